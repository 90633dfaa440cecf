"""Learned split network on the GPU: forward and backward kernels against the
FP64 oracle (itself pinned by finite differences in test_mlp_oracle.py),
training determinism and progress, and learned-split builds."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package, recall_at_k

pytestmark = pytest.mark.gpu


def _params(rng, n, scale):
    return (scale * rng.standard_normal(n)).astype(np.float32)


def _kink_free_case(acknn, oracle, rng, d, B, margin):
    """Parameters and rows whose triplet hinges are all well away from 0."""
    n = acknn.mlp_param_count(d)
    for _ in range(20):
        p = _params(rng, n, 1.0 / np.sqrt(max(d, 8)))
        rows = rng.standard_normal((3 * B, d)).astype(np.float32)
        # pull half of the positives towards their anchors so both hinge signs occur
        rows[B:B + B // 2] = rows[:B // 2] + np.float32(0.2) * rows[B:B + B // 2]
        loss, grad, hinge = oracle.mlp_loss_grad(p, rows, margin)
        if np.min(np.abs(hinge)) > 1e-2 and 0 < np.count_nonzero(hinge > 0) < B:
            return p, rows, loss, grad
    pytest.fail("no kink-free case found")


@pytest.mark.parametrize("d,B", [(5, 7), (37, 200), (128, 1024), (784, 96)])
def test_gradient_matches_oracle(acknn, oracle, d, B):
    """GPU FP32 forward + backward (tiled GEMMs, split-K weight gradients,
    GELU backward, triplet loss) against the FP64 oracle: loss within 1e-5
    relative, gradient within 1e-4 relative in L2 and 1e-3 of the largest
    component elementwise."""
    rng = np.random.Generator(np.random.PCG64(100 + d))
    margin = 4.0
    p, rows, loss_o, grad_o = _kink_free_case(acknn, oracle, rng, d, B, margin)
    loss_g, grad_g = acknn.mlp_loss_grad(p, rows, margin)
    assert loss_g == pytest.approx(loss_o, rel=1e-5)
    err = np.linalg.norm(grad_g - grad_o) / np.linalg.norm(grad_o)
    assert err < 1e-4, err
    assert np.max(np.abs(grad_g - grad_o)) <= 1e-3 * np.max(np.abs(grad_o))


@pytest.mark.parametrize("d,metric", [(16, 0), (96, 0), (130, 0), (96, 2)])
def test_embedding_matches_oracle(acknn, oracle, d, metric):
    rng = np.random.Generator(np.random.PCG64(200 + d + metric))
    n = 3000
    x = (3.0 * rng.standard_normal((n, d)) + 1.0).astype(np.float32)
    if metric == 2:
        x[7] = 0.0  # a zero row stays zero
    p = _params(rng, acknn.mlp_param_count(d), 1.0 / np.sqrt(d))
    mean = x.mean(0).astype(np.float32)
    inv_std = (1.0 / x.std(0)).astype(np.float32)
    z = acknn.mlp_embed(x, p, mean, inv_std, metric)
    u = x
    if metric == 2:
        nrm = np.sqrt((x.astype(np.float64) ** 2).sum(1)).astype(np.float32)
        sc = np.where(nrm > 0, np.float32(1.0) / np.where(nrm > 0, nrm, 1), np.float32(1.0))
        u = x * sc[:, None].astype(np.float32)
    s = (u - mean) * inv_std  # float32 roundings in the kernel's order
    zo = oracle.mlp_forward(p, s)
    np.testing.assert_allclose(z, zo, rtol=1e-4, atol=1e-4 * np.max(np.abs(zo)))


def test_training_is_deterministic_and_lowers_the_loss(acknn):
    x = acknn.workloads.gaussian_mixture(20000, 32, 16, 3)
    a = acknn.mlp_train(x, 10, seed=5, mlp_sample=8000, mlp_steps=200)
    b = acknn.mlp_train(x, 10, seed=5, mlp_sample=8000, mlp_steps=200)
    for u, v in zip(a, b):
        np.testing.assert_array_equal(u, v)
    curve = a[3]
    assert np.all(np.isfinite(curve))
    assert curve[-20:].mean() < 0.8 * curve[:20].mean(), (curve[:20].mean(), curve[-20:].mean())
    np.testing.assert_allclose(a[1], x[(np.arange(8000) * 20000) // 8000].mean(0), rtol=1e-4, atol=1e-4)


def test_learned_build_is_a_valid_graph(acknn, oracle):
    x = acknn.workloads.gaussian_mixture(20000, 24, 8, 11)
    k = 10
    idx, dist = acknn.knn_build(x, k, 4, 64, 2, 0, seed=1, learned=True, mlp_sample=10000,
                                mlp_steps=100)
    n = x.shape[0]
    assert idx.min() >= 0 and idx.max() < n
    assert not np.any(idx == np.arange(n)[:, None])
    assert all(len(set(r.tolist())) == k for r in idx[:2000])
    assert np.all(np.diff(dist, axis=1) >= 0)
    # distances are exact FP32 keys of the listed pairs
    q = np.arange(0, n, 97)
    d64 = oracle.pair_dist(x, np.repeat(q, k), idx[q].ravel()).reshape(-1, k)
    np.testing.assert_allclose(dist[q], d64, rtol=1e-5)
    ex, _ = oracle.exact(x, k, queries=q)
    plain, _ = acknn.knn_build(x, k, 4, 64, 2, 0, seed=1)
    # isotropic 24-dim clusters: the network matches random projections
    assert recall_at_k(idx[q], ex) > recall_at_k(plain[q], ex) - 0.05


@pytest.mark.parametrize("metric", [1, 2])
def test_learned_build_other_metrics(acknn, oracle, metric):
    x = acknn.workloads.gaussian_mixture(8000, 20, 6, 12 + metric) + np.float32(30.0)
    k = 8
    idx, dist = acknn.knn_build(x, k, 4, 64, 2, metric, seed=2, learned=True, mlp_sample=4000,
                                mlp_steps=60)
    q = np.arange(0, x.shape[0], 53)
    ex, _ = oracle.exact(x, k, queries=q, metric=metric)
    plain, _ = acknn.knn_build(x, k, 4, 64, 2, metric, seed=2)
    assert recall_at_k(idx[q], ex) > recall_at_k(plain[q], ex) - 0.05


def _recall_gpu(acknn, x, idx, k, metric, nq=2000):
    q = np.arange(0, x.shape[0], max(1, x.shape[0] // nq))
    ex, _ = acknn.exact_fp64(x, k, q, metric)
    return recall_at_k(idx[q], ex)


# (name, points, k, trees, leaf, props, metric, lower bound on learned - plain)
def _ab_cases(acknn):
    W = acknn.workloads
    return [
        ("scaled-norm directions d=64, COSINE", lambda: W.scaled_directions(0, 100_000, 64),
         10, 8, 64, 2, 2, 0.15),
        ("unit-norm 1000-cluster mixture d=96, COSINE (C4 shape)",
         lambda: W.normalized_mixture(0, 100_000, 96).astype(np.float32), 10, 12, 64, 4, 2, -0.03),
        ("integer 256-cluster mixture d=128, EUCLIDEAN (C2 shape)",
         lambda: W.integer_mixture(0, 100_000, 128), 16, 10, 1024, 1, 0, -0.01),
    ]


@pytest.mark.parametrize("case", range(3))
def test_learned_splits_ab(acknn, capsys, case):
    """A/B of the trained network against random-projection splits at equal
    trees, leaf size and propagations; recall against the FP64 exact k-NN.

    The network gains where raw coordinates misrepresent the metric (COSINE on
    rows whose norms spread over two decades: the unit-row input plus the
    network recover the angular neighbourhoods).  On isotropic Gaussian
    clusters random two-point directions are already as good as any direction
    (neighbour differences and node spread have the same covariance shape), so
    the network can only match them; the bound there is a small loss."""
    name, make, k, T, leaf, P, metric, bound = _ab_cases(acknn)[case]
    x = make()
    plain, _, sp = acknn.knn_build(x, k, T, leaf, P, metric, seed=3, stats=True)
    learned, _, sl = acknn.knn_build(x, k, T, leaf, P, metric, seed=3, stats=True, learned=True)
    rp = _recall_gpu(acknn, x, plain, k, metric)
    rl = _recall_gpu(acknn, x, learned, k, metric)
    with capsys.disabled():
        print(f"\n[learned A/B] {name}: n={x.shape[0]} k={k} T={T} leaf={leaf} P={P}: "
              f"recall plain {rp:.4f} ({sp['ms_total']:.1f} ms), learned {rl:.4f} "
              f"({sl['ms_total']:.1f} ms, of which training+embedding {sl['ms_learn']:.1f} ms), "
              f"gain {rl - rp:+.4f}")
    assert rl - rp >= bound, (rp, rl)

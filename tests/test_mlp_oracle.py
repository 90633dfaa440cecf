"""The learned split network's FP64 oracle (forward pass and triplet-loss
gradient) pinned by central finite differences on the CPU; it is then the reference
of the GPU forward and backward kernels (test_mlp_gpu.py)."""
from __future__ import annotations

import numpy as np
import pytest

H, E = 256, 64


def _param_count(d):
    return H * d + H + E * H + E


def _params(rng, d, scale=0.4):
    return (scale * rng.standard_normal(_param_count(d))).astype(np.float32)


def _numpy_forward(p, d, rows):
    p = p.astype(np.float64)
    W1 = p[: H * d].reshape(H, d)
    b1 = p[H * d: H * d + H]
    W2 = p[H * d + H: H * d + H + E * H].reshape(E, H)
    b2 = p[H * d + H + E * H:]
    a = rows.astype(np.float64) @ W1.T + b1
    g = 0.5 * a * (1 + np.tanh(np.sqrt(2 / np.pi) * (a + 0.044715 * a ** 3)))
    return g @ W2.T + b2


def test_forward_matches_numpy(oracle):
    rng = np.random.Generator(np.random.PCG64(1))
    d = 7
    p = _params(rng, d)
    rows = rng.standard_normal((9, d)).astype(np.float32)
    np.testing.assert_allclose(oracle.mlp_forward(p, rows), _numpy_forward(p, d, rows), rtol=1e-12,
                               atol=1e-12)


def _loss_numpy(p, d, rows, margin):
    z = _numpy_forward(p, d, rows)
    b = rows.shape[0] // 3
    za, zp, zn = z[:b], z[b:2 * b], z[2 * b:]
    l = margin + ((za - zp) ** 2).sum(1) - ((za - zn) ** 2).sum(1)
    return np.maximum(l, 0).mean(), l


def test_loss_matches_numpy(oracle):
    rng = np.random.Generator(np.random.PCG64(2))
    d = 6
    p = _params(rng, d)
    rows = rng.standard_normal((12, d)).astype(np.float32)
    loss, _, hinge = oracle.mlp_loss_grad(p, rows, margin=3.0)
    ref, l = _loss_numpy(p, d, rows, 3.0)
    assert loss == pytest.approx(ref, rel=1e-12)
    np.testing.assert_allclose(hinge, l, rtol=1e-12)


@pytest.mark.parametrize("d", [3, 8])
def test_gradient_matches_central_differences(oracle, d):
    """d loss / d theta_i against (L(theta + h e_i) - L(theta - h e_i)) / 2h for
    coordinates in every parameter block; h = 2^-12 is exact in float32 for
    these magnitudes, and every hinge is kept well away from its kink."""
    rng = np.random.Generator(np.random.PCG64(10 + d))
    margin = 2.0
    for _ in range(50):
        p = _params(rng, d)
        rows = rng.standard_normal((3 * 5, d)).astype(np.float32)
        _, grad, hinge = oracle.mlp_loss_grad(p, rows, margin)
        if np.min(np.abs(hinge)) > 0.5 and np.any(hinge > 0):
            break
    else:
        pytest.fail("no kink-free case found")
    npar = p.shape[0]
    blocks = [(0, H * d), (H * d, H * d + H), (H * d + H, H * d + H + E * H), (npar - E, npar)]
    coords = np.concatenate([rng.integers(lo, hi, size=12) for lo, hi in blocks])
    h = np.float32(2.0 ** -12)
    for i in coords:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        assert float(pp[i]) - float(p[i]) == float(h)  # exact perturbation
        lp, _, _ = oracle.mlp_loss_grad(pp, rows, margin)
        lm, _, _ = oracle.mlp_loss_grad(pm, rows, margin)
        fd = (lp - lm) / (2 * float(h))
        assert fd == pytest.approx(grad[i], rel=2e-4, abs=1e-6), (i, fd, grad[i])


def test_gradient_zero_when_all_hinges_inactive(oracle):
    rng = np.random.Generator(np.random.PCG64(5))
    d = 4
    p = _params(rng, d)
    rows = rng.standard_normal((6, d)).astype(np.float32)
    loss, grad, hinge = oracle.mlp_loss_grad(p, rows, margin=-1e6)
    assert loss == 0.0 and np.all(hinge < 0) and not np.any(grad)

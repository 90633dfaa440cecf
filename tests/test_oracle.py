"""The CPU oracle, pinned against the known-answer fixtures and checked for the
invariants every k-NN graph of this path must satisfy.  No GPU needed."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, load_package, recall_at_k

KATS = sorted(p.stem for p in GOLDEN.glob("kat_*.npz"))


def _kat(name):
    z = np.load(GOLDEN / f"{name}.npz")
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", KATS)
def test_oracle_exact_matches_kat(oracle, name):
    c = _kat(name)
    k, metric = int(c["k"]), int(c["metric"])
    idx, dist = oracle.exact(c["points"], k, metric=metric)
    np.testing.assert_array_equal(idx, c["idx"])
    np.testing.assert_allclose(dist, c["dist"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("name", KATS)
@pytest.mark.parametrize("props", [0, 2])
def test_oracle_build_one_leaf_is_exact(oracle, name, props):
    """n <= leaf: one leaf holds every point, so the graph is the exact one."""
    c = _kat(name)
    x = c["points"]
    k, metric = int(c["k"]), int(c["metric"])
    idx, dist = oracle.knn_build(x, k, trees=3, leaf=x.shape[0], props=props, metric=metric)
    np.testing.assert_array_equal(idx, c["idx"])
    np.testing.assert_allclose(dist, c["dist"], rtol=1e-6, atol=1e-6)


def _random(n, d, seed, kind="gauss"):
    rng = np.random.Generator(np.random.PCG64(seed))
    if kind == "int":
        return rng.integers(0, 8, size=(n, d)).astype(np.float32)
    return rng.standard_normal((n, d), dtype=np.float32)


def _check_graph(idx, dist, n, k):
    assert idx.shape == (n, k)
    assert np.all(idx >= 0) and np.all(idx < n)
    assert not np.any(idx == np.arange(n)[:, None]), "self in list"
    for row in idx:
        assert len(set(row.tolist())) == k, "duplicate neighbour"
    assert np.all(np.diff(dist, axis=1) >= 0), "rows not sorted"


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("kind", ["gauss", "int"])
def test_oracle_graph_invariants(oracle, metric, kind):
    n, d, k = 700, 9, 7
    x = _random(n, d, 11, kind)
    idx, dist = oracle.knn_build(x, k, trees=4, leaf=20, props=2, metric=metric)
    _check_graph(idx, dist, n, k)


def test_oracle_thread_count_does_not_change_result(oracle):
    x = _random(1500, 12, 2)
    a = oracle.knn_build(x, 8, trees=5, leaf=24, props=2, threads=1)
    b = oracle.knn_build(x, 8, trees=5, leaf=24, props=2, threads=8)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_oracle_trees_are_permutations_with_median_splits(oracle):
    n, d, leaf = 1000, 5, 16
    x = _random(n, d, 4)
    perm = oracle.build_trees(x, trees=3, leaf=leaf, seed=9)
    for t in range(3):
        assert np.array_equal(np.sort(perm[t]), np.arange(n))
    # leaf sizes are floor/ceil(n / 2^depth) and never exceed `leaf`
    depth = oracle.lib.oracle_tree_depth(n, leaf)
    bounds = [(j * n) >> depth for j in range((1 << depth) + 1)]
    sizes = np.diff(bounds)
    assert sizes.max() <= leaf and sizes.min() >= n // (1 << depth)


def test_oracle_seed_changes_trees(oracle):
    x = _random(800, 6, 5)
    a = oracle.build_trees(x, 2, 16, seed=1)
    b = oracle.build_trees(x, 2, 16, seed=2)
    assert not np.array_equal(a, b)


def test_oracle_rejects_n_le_k(oracle):
    x = _random(5, 3, 1)
    with pytest.raises(ValueError):
        oracle.knn_build(x, 5, trees=1, leaf=4, props=0)


def test_oracle_exact_vs_numpy(oracle):
    x = _random(300, 7, 8, "int")  # integer data: many exact distance ties
    for metric in (0, 1):
        idx, dist = oracle.exact(x, 6, metric=metric)
        x64 = x.astype(np.float64)
        for i in range(0, 300, 37):
            if metric == 0:
                dv = np.sqrt(((x64 - x64[i]) ** 2).sum(1))
            else:
                dv = np.abs(x64 - x64[i]).sum(1)
            order = sorted((dv[j], j) for j in range(300) if j != i)[:6]
            assert idx[i].tolist() == [j for _, j in order]


def test_oracle_recall_small_gaussians(oracle):
    """The plain path on the small 10-cluster case (k=10, 10 trees, leaf 32,
    3 propagations) against the FP64 exact graph."""
    acknn = load_package()
    x = acknn.workloads.small_gaussians(0)
    idx, _ = oracle.knn_build(x, 10, trees=10, leaf=32, props=3)
    ex, _ = oracle.exact(x, 10)
    assert recall_at_k(idx, ex) > 0.93


def _pairs_key(x, i, j, metric):
    # float32 key in the reference order for d <= 256 (one chunk)
    a, b = x[i], x[j]
    acc = np.float32(0)
    for e in range(x.shape[1]):
        if metric == 0:
            df = np.float32(a[e] - b[e])
            acc = np.float32(np.float64(df) * np.float64(df) + np.float64(acc))  # exact fma for small ints
        else:
            acc = np.float32(acc + np.float32(abs(np.float32(a[e] - b[e]))))
    return acc


def test_flag_skip_rule_equals_full_jacobi(oracle):
    """Propagation that skips pairs (a, j) with a and j both unchanged since the
    previous step gives exactly the full Jacobi result (the rule the GPU kernel
    relies on); checked over several steps on integer data with many ties."""
    n, d, k = 240, 3, 6
    x = _random(n, d, 21, "int")
    perm = oracle.build_trees(x, 2, 12, seed=3)
    idx, key = oracle.leaf_stage(x, k, perm, 12, metric=0)
    keymat = {}

    def kk(i, j):
        if (i, j) not in keymat:
            keymat[(i, j)] = float(_pairs_key(x, i, j, 0))
        return keymat[(i, j)]

    cur_idx, cur_key = idx.copy(), key.copy()
    flags = np.ones((n, k), dtype=bool)
    full_idx, full_key = idx.copy(), key.copy()
    for step in range(4):
        full_idx, full_key = oracle.propagate(x, full_idx, full_key, metric=0)
        new_idx = np.empty_like(cur_idx)
        new_key = np.empty_like(cur_key)
        new_flags = np.zeros_like(flags)
        for i in range(n):
            old = [(float(cur_key[i, s]), int(cur_idx[i, s])) for s in range(k)]
            seen = {i} | {j for _, j in old}
            cand = []
            for s in range(k):
                a = int(cur_idx[i, s])
                for r in range(k):
                    j = int(cur_idx[a, r])
                    if not (flags[i, s] or flags[a, r]) or j in seen:
                        continue
                    seen.add(j)
                    cand.append((kk(i, j), j))
            merged = sorted([(v, j, False) for v, j in old] + [(v, j, True) for v, j in cand])[:k]
            new_idx[i] = [j for _, j, _ in merged]
            new_key[i] = [v for v, _, _ in merged]
            new_flags[i] = [f for _, _, f in merged]
        cur_idx, cur_key, flags = new_idx, new_key, new_flags
        np.testing.assert_array_equal(cur_idx, full_idx, err_msg=f"step {step}")
        np.testing.assert_array_equal(cur_key, full_key, err_msg=f"step {step}")

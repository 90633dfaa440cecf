"""Mixed-precision leaf stage (BF16 tcgen05 tiles + FP32 re-rank of the best
min(2k, 32) candidates) against the plain FP32 path and the oracle.

* Integer coordinates in [0, 255] with d * 255^2 < 2^24: every BF16 product and
  FP32 sum of |x|^2 + |y|^2 - 2 x.y is exact, so the mixed path must return the
  plain path's graph bit for bit (which is the oracle's).
* Float data: every returned distance is the exact FP32 key of its pair (the
  re-rank), and recall against the FP64 exact graph stays within 0.02 of the
  plain path's."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package, recall_at_k

pytestmark = pytest.mark.gpu


def _ints(n, d, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.uniform(0, 255, size=(12, d))
    x = centres[rng.integers(0, 12, n)] + rng.normal(0, 20, size=(n, d))
    return np.clip(np.rint(x), 0, 255).astype(np.float32)


@pytest.fixture(scope="module")
def lib():
    acknn = load_package()
    acknn.load_library()
    return acknn


@pytest.mark.parametrize("n,d,k,trees,leaf,props", [
    (20000, 128, 16, 4, 64, 0),
    (20000, 128, 16, 4, 64, 2),
    (30000, 128, 16, 3, 512, 1),
    (9000, 200, 10, 2, 300, 1),     # Kp = 256, three 128-query tiles per leaf
    (5000, 64, 8, 3, 40, 1),        # Kp = 64, short blocks
    (4000, 96, 24, 2, 130, 1),      # kq = 32 for k > 16
    (20000, 128, 16, 3, 2048, 0),   # first tree with the bounding pass; later trees mask listed ids
    (24000, 64, 5, 2, 3000, 1),     # bounding pass over more than 64 column slices (groups wrap)
])
def test_mixed_equals_plain_on_exact_integer_data(lib, oracle, n, d, k, trees, leaf, props):
    x = _ints(n, d, n + d)
    mi, md = lib.knn_build(x, k, trees, leaf, props, 0, seed=4, precision=lib.PREC_BF16_RERANK)
    pi, pd = lib.knn_build(x, k, trees, leaf, props, 0, seed=4)
    np.testing.assert_array_equal(mi, pi)
    np.testing.assert_array_equal(md.view(np.uint32), pd.view(np.uint32))
    oi, od = oracle.knn_build(x, k, trees, leaf, props, 0, seed=4)
    np.testing.assert_array_equal(mi, oi)


@pytest.mark.parametrize("metric", [0, 2])
def test_mixed_float_data_exact_keys_and_recall(lib, oracle, metric):
    n, d, k = 12000, 48, 10
    x = lib.workloads.gaussian_mixture(n, d, 20, seed=7)
    mi, md = lib.knn_build(x, k, 6, 200, 2, metric, seed=1, precision=lib.PREC_BF16_RERANK)
    pi, pd = lib.knn_build(x, k, 6, 200, 2, metric, seed=1)
    # sorted rows, no self, unique neighbours
    assert np.all(np.diff(md, axis=1) >= 0)
    assert not np.any(mi == np.arange(n)[:, None])
    # returned distances are the exact FP32 keys of their pairs
    for i in range(0, n, 997):
        for s in range(k):
            key = oracle.pair_key(x[i], x[mi[i, s]], metric)
            want = np.sqrt(np.float32(key)) if metric == 0 else np.float32(key)
            assert md[i, s] == want
    q = np.arange(0, n, 5)
    ei, _ = oracle.exact(x, k, q, metric)
    rm = recall_at_k(mi[q], ei)
    rp = recall_at_k(pi[q], ei)
    assert rm >= rp - 0.02, (rm, rp)


def test_taxicab_request_falls_back_to_fp32(lib):
    x = _ints(3000, 32, 3)
    a = lib.knn_build(x, 6, 2, 40, 1, 1, precision=lib.PREC_BF16_RERANK)
    b = lib.knn_build(x, 6, 2, 40, 1, 1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("n,d,k,trees,leaf,props", [
    (20000, 128, 16, 4, 64, 0),
    (20000, 128, 16, 3, 2048, 0),
    (9000, 200, 10, 2, 300, 1),
])
def test_f16_tiles_equal_plain_on_exact_integer_data(lib, n, d, k, trees, leaf, props):
    """FP16 tiles (11 significant bits) hold integers up to 2048 exactly; the
    EUCLIDEAN rows are scaled by a power of two into [2^14, 2^15), which keeps
    them exact, so the graph equals the plain one bit for bit."""
    x = _ints(n, d, n + d + 1)
    mi, md = lib.knn_build(x, k, trees, leaf, props, 0, seed=4, precision=lib.PREC_F16_RERANK)
    pi, pd = lib.knn_build(x, k, trees, leaf, props, 0, seed=4)
    np.testing.assert_array_equal(mi, pi)
    np.testing.assert_array_equal(md.view(np.uint32), pd.view(np.uint32))


@pytest.mark.parametrize("scale", [1e-6, 1.0, 1e6])
def test_f16_tiles_any_euclidean_scale(lib, scale):
    """Rows far outside the FP16 range (or deep in its subnormals) still rank
    as the plain path does: on integer data times a power of two the graph is
    identical; on float data times any scale, recall stays within 0.02."""
    n, d, k = 12000, 64, 10
    x = _ints(n, d, 5) * np.float32(2.0 ** round(np.log2(scale)))
    mi, md = lib.knn_build(x, k, 4, 128, 1, 0, seed=2, precision=lib.PREC_F16_RERANK)
    pi, pd = lib.knn_build(x, k, 4, 128, 1, 0, seed=2)
    np.testing.assert_array_equal(mi, pi)
    np.testing.assert_array_equal(md.view(np.uint32), pd.view(np.uint32))
    y = lib.workloads.gaussian_mixture(n, d, 20, seed=9) * np.float32(scale)
    mi, _ = lib.knn_build(y, k, 4, 128, 1, 0, seed=2, precision=lib.PREC_F16_RERANK)
    pi, _ = lib.knn_build(y, k, 4, 128, 1, 0, seed=2)
    q = np.arange(0, n, 7)
    ei, _ = lib.exact_fp64(y, k, q, 0)
    assert recall_at_k(mi[q], ei) >= recall_at_k(pi[q], ei) - 0.02


def test_precision_stats_report_the_leaf_path(lib):
    x = lib.workloads.gaussian_mixture(3000, 32, 6, seed=1)
    for prec, metric, path, fallback in ((lib.PREC_FP32, 0, 0, 0), (lib.PREC_BF16_RERANK, 0, 1, 0),
                                         (lib.PREC_F16_RERANK, 2, 2, 0), (lib.PREC_BF16_RERANK, 1, 0, 1)):
        _, _, st = lib.knn_build(x, 6, 2, 64, 1, metric, precision=prec, stats=True)
        assert (st["leaf_path"], st["leaf_fallback"]) == (path, fallback)


@pytest.mark.parametrize("metric", [0, 2])
@pytest.mark.parametrize("n,d,k,leaf", [(20000, 64, 10, 48), (30000, 96, 10, 64), (9000, 32, 8, 30),
                                        (5000, 128, 15, 40)])
def test_grouped_sibling_leaves_equal_single_leaf_tiles(lib, metric, n, d, k, leaf):
    """Two or four sibling leaves in one 128-row tile (each row masked to its
    own leaf's columns) give the one-leaf-per-tile graph bit for bit."""
    x = lib.workloads.gaussian_mixture(n, d, 16, seed=n + leaf)
    want = None
    for g in (1, 2, 4):
        for prec in (lib.PREC_BF16_RERANK, lib.PREC_F16_RERANK):
            opts = dict(precision=prec, tc_group=g)
            gi, gd, st = lib.knn_build(x, k, 4, leaf, 1, metric, seed=3, stats=True, **opts)
            assert st["tc_group"] <= g
            key = prec
            if g == 1:
                want = want or {}
                want[key] = (gi, gd)
            else:
                np.testing.assert_array_equal(gi, want[key][0])
                np.testing.assert_array_equal(gd.view(np.uint32), want[key][1].view(np.uint32))


def test_grouped_tiles_in_batches_and_on_exact_data(lib):
    """Batches of sets with different depths: each set's graph is its single
    build's with any group; on exact-integer data every grouping equals the
    plain FP32 graph."""
    xs = [_ints(3000 + 1100 * i, 32, 40 + i) for i in range(5)]
    base = lib.knn_build_batch(xs, 12, 3, 48, 1, 0, seeds=list(range(5)), precision=lib.PREC_BF16_RERANK,
                               tc_group=1)
    for g in (2, 4):
        got = lib.knn_build_batch(xs, 12, 3, 48, 1, 0, seeds=list(range(5)), precision=lib.PREC_BF16_RERANK,
                                  tc_group=g)
        for (bi, bd), (gi, gd) in zip(base, got):
            np.testing.assert_array_equal(bi, gi)
            np.testing.assert_array_equal(bd.view(np.uint32), gd.view(np.uint32))
    for i, x in enumerate(xs):
        pi, pd = lib.knn_build(x, 12, 3, 48, 1, 0, seed=i)
        np.testing.assert_array_equal(base[i][0], pi)
        np.testing.assert_array_equal(base[i][1].view(np.uint32), pd.view(np.uint32))


def test_grouped_tiles_autotuned(lib):
    x = lib.workloads.gaussian_mixture(40000, 64, 16, seed=5)
    a = lib.knn_build(x, 10, 3, 40, 1, 0, precision=lib.PREC_BF16_RERANK, autotune=True)
    b = lib.knn_build(x, 10, 3, 40, 1, 0, precision=lib.PREC_BF16_RERANK, tc_group=1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))

"""Reference-rule trees (split_rule = KNN_SPLIT_REFERENCE): the sign split
through the origin with per-level shared pivots, pivots forced apart, nodes
split until they hold at most `leaf` points.  The GPU build equals the CPU
restatement bit for bit (plain FP32), including leaves smaller than k+1 whose
blocks are ancestors, and its recall is printed beside the reference's own
sm_100a build on the same (normalised) data."""
from __future__ import annotations

import zlib

import numpy as np
import pytest

from conftest import load_package, recall_at_k

pytestmark = pytest.mark.gpu

REF = 1  # KNN_SPLIT_REFERENCE

CASES = [
    # name, n, d, k, trees, leaf, props, normalise
    ("gauss16_norm", 4000, 16, 10, 4, 32, 2, True),
    ("gauss37_raw", 3000, 37, 8, 3, 40, 1, False),
    ("leaf_below_k", 2500, 12, 10, 3, 6, 1, True),   # leaves < k+1: blocks are ancestors
    ("d257_norm", 900, 257, 5, 2, 30, 1, True),
]


def _data(acknn, name, n, d, norm):
    x = acknn.workloads.gaussian_mixture(n, d, 8, zlib.crc32(name.encode()) & 0xFFFF)
    return acknn.normalize_reference(x) if norm else x


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_rule_bit_parity(acknn, oracle, case, metric):
    name, n, d, k, trees, leaf, props, norm = case
    x = _data(acknn, name, n, d, norm)
    gi, gd = acknn.knn_build(x, k, trees, leaf, props, metric, seed=3, split_rule=REF)
    oi, od = oracle.knn_build_faithful(x, k, trees, leaf, props, metric, seed=3)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))


def test_reference_rule_mixed_precision_on_exact_data(acknn):
    """BF16 tiles over the explicit leaf table: on integer data every product
    and sum is exact, so the mixed build equals the plain one."""
    rng = np.random.Generator(np.random.PCG64(8))
    x = (rng.integers(0, 40, size=(6000, 32)) - 20).astype(np.float32)
    a = acknn.knn_build(x, 12, 4, 48, 1, 0, seed=5, split_rule=REF)
    b = acknn.knn_build(x, 12, 4, 48, 1, 0, seed=5, split_rule=REF, precision=1)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_reference_rule_trees_are_unbalanced(acknn, oracle):
    """Splits through the origin on data far from the origin are lopsided; the
    build still ends (pivots on both sides) and every list is complete."""
    x = acknn.workloads.gaussian_mixture(5000, 8, 4, 2) + np.float32(50.0)
    idx, dist = acknn.knn_build(x, 6, 2, 16, 0, 0, seed=1, split_rule=REF)
    assert idx.min() >= 0 and idx.max() < x.shape[0]
    assert not np.any(idx == np.arange(x.shape[0])[:, None])
    oi, _ = oracle.knn_build_faithful(x, 6, 2, 16, 0, 0, seed=1)
    np.testing.assert_array_equal(idx, oi)

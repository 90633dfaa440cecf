"""Autotuned launch shapes change no result: every FP32 leaf tile and every
propagation block size gives the same graph, the tuner picks one of them, and
tuned single and batched builds equal the untuned ones bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_forced_shapes_give_identical_graphs(acknn, oracle, metric):
    x = acknn.workloads.gaussian_mixture(12000, 40, 16, 20 + metric)
    k, T, leaf, P = 12, 4, 48, 2
    ref = acknn.knn_build(x, k, T, leaf, P, metric, seed=4)
    oi, od = oracle.knn_build(x, k, T, leaf, P, metric, seed=4)
    np.testing.assert_array_equal(ref[0], oi)
    np.testing.assert_array_equal(ref[1], od)
    for tile in (32, 64):
        for warps in (1, 2, 4, 8):
            idx, dist = acknn.knn_build(x, k, T, leaf, P, metric, seed=4, leaf_tile=tile, prop_warps=warps)
            np.testing.assert_array_equal(idx, ref[0])
            np.testing.assert_array_equal(dist, ref[1])


def test_autotuned_build_equals_default(acknn):
    ctx = acknn.Context()
    x = acknn.workloads.gaussian_mixture(50000, 64, 16, 5)
    ref = acknn.knn_build(x, 15, 6, 48, 3, 0, seed=1)
    idx, dist, st = acknn.knn_build(x, 15, 6, 48, 3, 0, seed=1, autotune=True, stats=True, context=ctx.handle)
    np.testing.assert_array_equal(idx, ref[0])
    np.testing.assert_array_equal(dist, ref[1])
    assert st["leaf_tile"] in (32, 64) and st["prop_warps"] in (2, 4, 8)
    # the second call reuses the cached choice
    idx2, _, st2 = acknn.knn_build(x, 15, 6, 48, 3, 0, seed=1, autotune=True, stats=True, context=ctx.handle)
    np.testing.assert_array_equal(idx2, ref[0])
    assert (st2["leaf_tile"], st2["prop_warps"]) == (st["leaf_tile"], st["prop_warps"])
    ctx.close()


def test_autotuned_batch_equals_single_builds(acknn):
    ctx = acknn.Context()
    xs = [acknn.workloads.gaussian_mixture(n, d, 16, i) for i, (n, d) in
          enumerate([(3000, 32), (15000, 32), (800, 64), (7000, 64), (2500, 128)])]
    seeds = [3, 4, 5, 6, 7]
    for _ in range(3):  # eager + tuning, captured, replayed
        outs = acknn.knn_build_batch(xs, 15, 8, 48, 3, 0, seeds=seeds, autotune=True, context=ctx.handle)
        for x, (idx, dist), s in zip(xs, outs, seeds):
            ri, rd = acknn.knn_build(x, 15, 8, 48, 3, 0, seed=s)
            np.testing.assert_array_equal(idx, ri)
            np.testing.assert_array_equal(dist, rd)
    ctx.close()

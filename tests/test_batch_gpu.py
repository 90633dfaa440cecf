"""Batched builds (knn_build_batch): every set of a batch gets exactly the
graph that a build of that set alone produces with the same seed -- bit for bit
in plain FP32 and in the mixed BF16 + FP32 re-rank mode -- across uneven sizes,
several d, all metrics, repeated calls (eager, captured, replayed graph) and
FP16 input."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sets(acknn, spec, seed0=0):
    return [acknn.workloads.gaussian_mixture(n, d, 16, seed0 + i) for i, (n, d) in enumerate(spec)]


SPEC = [(16, 32), (1000, 32), (4321, 32), (20000, 32), (777, 64), (12345, 64), (3000, 7), (250, 7),
        (9000, 128), (1500, 256)]


def _check_equal(acknn, xs, outs, k, trees, leaf, props, metric, seeds, precision=0):
    for x, (idx, dist), s in zip(xs, outs, seeds):
        ri, rd = acknn.knn_build(x, k, trees, leaf, props, metric, seed=s, precision=precision)
        np.testing.assert_array_equal(idx, ri)
        np.testing.assert_array_equal(dist, rd)


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_batch_equals_individual_builds(acknn, metric):
    k, trees, leaf, props = 15, 4, 48, 2
    xs = _sets(acknn, SPEC)
    seeds = [11 * i + 1 for i in range(len(xs))]
    outs = acknn.knn_build_batch(xs, k, trees, leaf, props, metric, seeds=seeds)
    _check_equal(acknn, xs, outs, k, trees, leaf, props, metric, seeds)


@pytest.mark.parametrize("metric", [0, 2])
def test_batch_mixed_precision_equals_individual_builds(acknn, metric):
    k, trees, leaf, props = 15, 4, 48, 2
    xs = _sets(acknn, SPEC, seed0=50)
    seeds = list(range(len(xs)))
    outs = acknn.knn_build_batch(xs, k, trees, leaf, props, metric, seeds=seeds, precision=1)
    _check_equal(acknn, xs, outs, k, trees, leaf, props, metric, seeds, precision=1)


def test_batch_member_matches_oracle(acknn, oracle):
    xs = _sets(acknn, [(3000, 16), (5000, 16), (400, 16)], seed0=7)
    outs = acknn.knn_build_batch(xs, 10, 3, 32, 2, 0, seeds=[5, 6, 7])
    for x, (idx, dist), s in zip(xs, outs, [5, 6, 7]):
        oi, od = oracle.knn_build(x, 10, 3, 32, 2, 0, seed=s)
        np.testing.assert_array_equal(idx, oi)
        np.testing.assert_array_equal(dist, od)


def test_repeated_batches_replay_the_captured_graph(acknn):
    """First call launches directly, the second captures the group graphs, the
    third and later replay them; a new seed is a new shape signature."""
    ctx = acknn.Context()
    k, trees, leaf, props = 15, 4, 48, 3
    xs = _sets(acknn, SPEC, seed0=100)
    seeds = list(range(len(xs)))
    first = acknn.knn_build_batch(xs, k, trees, leaf, props, 0, seeds=seeds, context=ctx.handle)
    runs = [acknn.knn_build_batch(xs, k, trees, leaf, props, 0, seeds=seeds, context=ctx.handle)
            for _ in range(3)]
    for r in runs:
        for (a, b), (c, e) in zip(first, r):
            np.testing.assert_array_equal(a, c)
            np.testing.assert_array_equal(b, e)
    # fresh inputs of the same shapes through the replayed graphs
    ys = _sets(acknn, SPEC, seed0=300)
    outs = acknn.knn_build_batch(ys, k, trees, leaf, props, 0, seeds=seeds, context=ctx.handle)
    _check_equal(acknn, ys, outs, k, trees, leaf, props, 0, seeds)
    seeds2 = [s + 1 for s in seeds]
    outs = acknn.knn_build_batch(ys, k, trees, leaf, props, 0, seeds=seeds2, context=ctx.handle)
    _check_equal(acknn, ys, outs, k, trees, leaf, props, 0, seeds2)
    ctx.close()


def test_batch_fp16_input(acknn):
    xs = [x.astype(np.float16) for x in _sets(acknn, [(2000, 24), (6000, 24), (900, 40)], seed0=9)]
    outs = acknn.knn_build_batch(xs, 8, 3, 40, 2, 2, seeds=[1, 2, 3])
    _check_equal(acknn, xs, outs, 8, 3, 40, 2, 2, [1, 2, 3])


def test_batch_of_one_equals_single_build(acknn):
    x = acknn.workloads.gaussian_mixture(30000, 48, 16, 4)
    (idx, dist), = acknn.knn_build_batch([x], 12, 5, 64, 2, 0, seeds=[9])
    ri, rd = acknn.knn_build(x, 12, 5, 64, 2, 0, seed=9)
    np.testing.assert_array_equal(idx, ri)
    np.testing.assert_array_equal(dist, rd)

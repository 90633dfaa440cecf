"""Sparse-row FP32 leaf tiles (knn_options.sparse_dims) on the GPU.

Each leaf block reads only the dims that are non-zero in some of its rows.
The graph must be bit-identical to the all-dims tiles and to the CPU oracle:
rows with large zero supports (prototype supports, as in the sparse-prototype
workload), dims past 256 (two and four 256-dim groups), negative zeros, leaf
blocks made only of zero rows, dense rows where the list saves nothing,
climbed blocks of small leaves, and the automatic switch at 1024-point leaves."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _prototypes(n, d, protos, density, seed, zero_rows=0.0, negzero=False):
    rng = np.random.Generator(np.random.PCG64(seed))
    supports = rng.random((protos, d)) < density
    lab = rng.integers(0, protos, size=n)
    x = np.where(supports[lab], 1.0 - rng.random((n, d), dtype=np.float32), np.float32(0.0)).astype(np.float32)
    if zero_rows:
        x[rng.random(n) < zero_rows] = 0.0
    if negzero:
        x[(x == 0) & (rng.random((n, d)) < 0.5)] = np.float32(-0.0)
    return x


def _same(a, b, what):
    np.testing.assert_array_equal(a[0], b[0], err_msg=f"{what}: neighbour ids differ")
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32), err_msg=f"{what}: distances differ")


@pytest.fixture(scope="module")
def lib():
    acknn = load_package()
    acknn.load_library()
    return acknn


CASES = [
    # name, n, d, k, trees, leaf, props, x kwargs
    ("proto_d300", 5000, 300, 10, 2, 1200, 1, dict(protos=4, density=0.2)),
    ("proto_d784_k30", 4000, 784, 30, 2, 2048, 1, dict(protos=6, density=0.2)),
    ("proto_d1030", 2500, 1030, 8, 2, 1100, 0, dict(protos=3, density=0.1)),
    ("negzero_d200", 3000, 200, 6, 3, 300, 1, dict(protos=5, density=0.3, negzero=True)),
    ("zero_rows", 4000, 96, 5, 2, 500, 1, dict(protos=2, density=0.4, zero_rows=0.5)),
    ("dense", 3000, 64, 8, 2, 1500, 1, dict(protos=1, density=1.0)),
    ("climbed_blocks", 2000, 128, 12, 3, 6, 1, dict(protos=4, density=0.15)),
]


@pytest.mark.parametrize("pairs", [0, -1], ids=["tile_pairs", "one_sided"])
@pytest.mark.parametrize("metric", [0, 1])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_sparse_tiles_bit_identical(lib, oracle, case, metric, pairs):
    """With tile pairs each pair reads the union of its two tiles' dims (each
    leaf's positions ordered by row pattern first); one-sided tiles read the
    leaf block's dims."""
    name, n, d, k, trees, leaf, props, kw = case
    x = _prototypes(n, d, seed=len(name) * 31 + d, **kw)
    *on, st_on = lib.knn_build(x, k, trees, leaf, props, metric, seed=3, sparse_dims=1, tile_pairs=pairs,
                               stats=True)
    *off, st_off = lib.knn_build(x, k, trees, leaf, props, metric, seed=3, sparse_dims=-1, tile_pairs=pairs,
                                 stats=True)
    assert st_on["sparse_dims"] == 1 and st_off["sparse_dims"] == 0
    _same(on, off, f"{name}/metric{metric}: sparse vs all dims")
    _same(on, oracle.knn_build(x, k, trees, leaf, props, metric, seed=3), f"{name}/metric{metric}: vs oracle")


def test_automatic_switch(lib):
    x = _prototypes(4096, 160, protos=4, density=0.2, seed=9)
    big = lib.knn_build(x, 8, 2, 2048, 0, 1, seed=1, stats=True)[2]   # leaves of 2048 points
    small = lib.knn_build(x, 8, 2, 512, 0, 1, seed=1, stats=True)[2]  # leaves of 512 points
    cos = lib.knn_build(x, 8, 2, 2048, 0, 2, seed=1, stats=True)[2]   # COSINE reads all dims
    assert (big["sparse_dims"], small["sparse_dims"], cos["sparse_dims"]) == (1, 0, 0)


def test_batch_sparse_tile_pairs(lib, oracle):
    """Batched sets of sparse rows (segments of different sizes and depths):
    the per-leaf ordering, the tile masks and the pair lists work across
    segments, and every set gets the oracle's graph."""
    sets = [_prototypes(n, 200, protos=3, density=0.2, seed=40 + i) for i, n in enumerate((2600, 1500, 3900))]
    got = lib.knn_build_batch(sets, 9, 2, 700, 1, 1, seeds=[5, 6, 7], sparse_dims=1)
    off = lib.knn_build_batch(sets, 9, 2, 700, 1, 1, seeds=[5, 6, 7], sparse_dims=-1, tile_pairs=-1)
    for i, x in enumerate(sets):
        _same(got[i], off[i], f"set {i}: sparse tile pairs vs all dims one-sided")
        _same(got[i], oracle.knn_build(x, 9, 2, 700, 1, 1, seed=5 + i), f"set {i}: vs oracle")


def test_autotuned_sparse_tile_pairs(lib, oracle):
    """The leaf-tile tuner times both tiles on tree 0 with the same shortcuts;
    the graph does not depend on its choice."""
    x = _prototypes(3000, 300, protos=4, density=0.2, seed=77)
    tuned = lib.knn_build(x, 10, 3, 1500, 1, 0, seed=2, sparse_dims=1, autotune=True)
    _same(tuned, oracle.knn_build(x, 10, 3, 1500, 1, 0, seed=2), "autotuned sparse tile pairs vs oracle")

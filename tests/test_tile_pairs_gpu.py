"""Symmetric tile pairs of the FP32 leaf stage (knn_options.tile_pairs) on the GPU.

Where every leaf is its own block, each tile pair of a leaf is computed once
and merged into both tiles' rows.  The graph must be bit-identical to the
one-sided tiles and to the CPU oracle: all three metrics, list widths of one,
two and four warps' lanes (k 10, 40, 100), an odd and an even number of tiles
per leaf, 32- and 64-row tiles, sparse rows together with pairs, and batches."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _same(a, b, what):
    np.testing.assert_array_equal(a[0], b[0], err_msg=f"{what}: neighbour ids differ")
    np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32), err_msg=f"{what}: distances differ")


@pytest.fixture(scope="module")
def lib():
    acknn = load_package()
    acknn.load_library()
    return acknn


CASES = [
    # name, n, d, k, trees, leaf, props, leaf_tile
    ("two_tiles", 2000, 24, 10, 2, 128, 1, 64),        # leaves of 125: 2 tiles
    ("odd_tiles", 3000, 40, 10, 3, 200, 1, 64),        # leaves of 188: 3 tiles
    ("many_tiles_k40", 4096, 17, 40, 2, 1100, 0, 64),  # leaves of 1024: 16 tiles
    ("k100", 2600, 9, 100, 2, 700, 1, 64),             # leaves of 650: 11 tiles
    ("tile32", 3000, 33, 12, 2, 400, 1, 32),           # leaves of 375: 12 tiles of 32
]


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_pairs_bit_identical(lib, oracle, case, metric):
    name, n, d, k, trees, leaf, props, tile = case
    rng = np.random.Generator(np.random.PCG64(n + d + metric))
    x = rng.standard_normal((n, d), dtype=np.float32)
    *on, st_on = lib.knn_build(x, k, trees, leaf, props, metric, seed=4, leaf_tile=tile, stats=True)
    *off, st_off = lib.knn_build(x, k, trees, leaf, props, metric, seed=4, leaf_tile=tile, tile_pairs=-1,
                                 stats=True)
    assert st_on["tile_pairs"] == 1 and st_off["tile_pairs"] == 0
    assert st_on["leaf_pairs"] == st_off["leaf_pairs"]
    _same(on, off, f"{name}/metric{metric}: pairs vs one-sided tiles")
    _same(on, oracle.knn_build(x, k, trees, leaf, props, metric, seed=4), f"{name}/metric{metric}: vs oracle")


def test_pairs_with_sparse_rows(lib, oracle):
    rng = np.random.Generator(np.random.PCG64(5))
    sup = rng.random((3, 300)) < 0.2
    lab = rng.integers(0, 3, size=4000)
    x = np.where(sup[lab], rng.random((4000, 300), dtype=np.float32), np.float32(0)).astype(np.float32)
    for metric in (0, 1):
        *on, st = lib.knn_build(x, 16, 2, 1100, 1, metric, seed=2, sparse_dims=1, stats=True)
        assert st["tile_pairs"] == 1 and st["sparse_dims"] == 1
        off = lib.knn_build(x, 16, 2, 1100, 1, metric, seed=2, sparse_dims=-1, tile_pairs=-1)
        _same(on, off, f"metric{metric}: sparse pairs vs all dims one-sided")
        _same(on, oracle.knn_build(x, 16, 2, 1100, 1, metric, seed=2), f"metric{metric}: vs oracle")


def test_climbed_blocks_run_one_sided(lib):
    """Leaves below k+1 points climb to a larger block: no pairs there."""
    x = np.random.Generator(np.random.PCG64(8)).standard_normal((3000, 8), dtype=np.float32)
    st = lib.knn_build(x, 20, 2, 12, 0, 0, seed=1, stats=True)[2]
    assert st["tile_pairs"] == 0


def test_batch_with_pairs(lib, oracle):
    rng = np.random.Generator(np.random.PCG64(21))
    sets = [rng.standard_normal((n, d), dtype=np.float32) for n, d in ((1500, 16), (2300, 16), (900, 16))]
    got = lib.knn_build_batch(sets, 10, 2, 300, 1, 1, seeds=[3, 4, 5])
    off = lib.knn_build_batch(sets, 10, 2, 300, 1, 1, seeds=[3, 4, 5], tile_pairs=-1)
    for i, x in enumerate(sets):
        _same(got[i], off[i], f"set {i}: batch pairs vs one-sided")
        _same(got[i], oracle.knn_build(x, 10, 2, 300, 1, 1, seed=3 + i), f"set {i}: vs oracle")

"""GPU plain-FP32 path against the CPU oracle, through the C ABI.

Bar: bit-identical neighbour lists and bit-identical float32 distances (the
path's stated tolerance is 1e-5 relative; the kernels follow the oracle's
operation order exactly, so equality is required here)."""
from __future__ import annotations

import zlib

import numpy as np
import pytest

from conftest import GOLDEN, load_package

pytestmark = pytest.mark.gpu


def _rand(n, d, seed, kind="gauss"):
    rng = np.random.Generator(np.random.PCG64(seed))
    if kind == "int":
        return rng.integers(0, 6, size=(n, d)).astype(np.float32)
    if kind == "zeros":
        x = rng.standard_normal((n, d), dtype=np.float32)
        x[::7] = 0.0
        return x
    return rng.standard_normal((n, d), dtype=np.float32)


def _same(a, b, what):
    ai, ad = a
    bi, bd = b
    np.testing.assert_array_equal(ai, bi, err_msg=f"{what}: neighbour ids differ")
    np.testing.assert_array_equal(ad.view(np.uint32), bd.view(np.uint32),
                                  err_msg=f"{what}: distances differ")


@pytest.fixture(scope="module")
def lib():
    acknn = load_package()
    acknn.load_library()
    return acknn


def test_small_gaussians_bit_parity(lib, oracle):
    """N=10,000, d=16, 10 clusters; k=10, 10 trees, leaf 32, 3 propagations."""
    x = lib.workloads.small_gaussians(0)
    got = lib.knn_build(x, 10, 10, 32, 3, 0, seed=0)
    want = oracle.knn_build(x, 10, 10, 32, 3, 0, seed=0)
    _same(got, want, "small_gaussians")


CASES = [
    # name, n, d, k, trees, leaf, props, kind
    ("gauss_d37", 3000, 37, 12, 4, 40, 2, "gauss"),
    ("int_ties", 2000, 8, 8, 3, 24, 2, "int"),
    ("d257", 600, 257, 5, 2, 30, 1, "gauss"),
    ("line_d1", 500, 1, 4, 3, 16, 2, "gauss"),
    ("climb_leaf4_k10", 1000, 6, 10, 3, 4, 1, "gauss"),
    ("k40", 1500, 10, 40, 2, 90, 1, "gauss"),
    ("k100", 900, 7, 100, 2, 220, 1, "gauss"),
    ("n_k_plus_1", 9, 5, 8, 2, 4, 1, "gauss"),
    ("odd_n_deep", 4097, 3, 3, 2, 5, 2, "gauss"),
]


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_build_bit_parity(lib, oracle, case, metric):
    name, n, d, k, trees, leaf, props, kind = case
    x = _rand(n, d, zlib.crc32(name.encode()) & 0xFFFF, kind)
    got = lib.knn_build(x, k, trees, leaf, props, metric, seed=5)
    want = oracle.knn_build(x, k, trees, leaf, props, metric, seed=5)
    _same(got, want, f"{name}/metric{metric}")


def test_cosine_zero_rows(lib, oracle):
    x = _rand(800, 12, 3, "zeros")
    _same(lib.knn_build(x, 6, 3, 20, 2, 2), oracle.knn_build(x, 6, 3, 20, 2, 2), "cosine zeros")


@pytest.mark.parametrize("n,d,leaf", [(1000, 5, 16), (4097, 33, 7), (20000, 16, 64), (3, 2, 1)])
def test_trees_identical(lib, oracle, n, d, leaf):
    x = _rand(n, d, n + d)
    np.testing.assert_array_equal(lib.build_trees(x, 3, leaf, seed=11),
                                  oracle.build_trees(x, 3, leaf, seed=11))


def test_tree_large_node_path(lib, oracle):
    """Nodes above the shared-memory key limit (12288 points) take the
    streamed-select path."""
    x = _rand(60000, 8, 77)
    np.testing.assert_array_equal(lib.build_trees(x, 2, 50, seed=1),
                                  oracle.build_trees(x, 2, 50, seed=1))


def test_tree_multiblock_split_ties(lib, oracle):
    """Top levels with few, large nodes are split by several blocks per node
    (global digit histograms, then a stable scatter); integer data gives many
    tied projections, ordered by id."""
    x = _rand(150000, 4, 5, "int")
    np.testing.assert_array_equal(lib.build_trees(x, 3, 100, seed=3),
                                  oracle.build_trees(x, 3, 100, seed=3))


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_leaf_stage_identical(lib, oracle, metric):
    x = _rand(5000, 20, 9)
    perm = oracle.build_trees(x, 4, 40, seed=2)
    gi, gk = lib.leaf_stage(x, 9, perm, 40, metric)
    oi, ok = oracle.leaf_stage(x, 9, perm, 40, metric)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gk.view(np.uint32), ok.view(np.uint32))


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_propagate_step_identical(lib, oracle, metric):
    x = _rand(4000, 24, 10)
    perm = oracle.build_trees(x, 2, 30, seed=3)
    idx, key = oracle.leaf_stage(x, 8, perm, 30, metric)
    for _ in range(2):
        gi, gk = lib.propagate_step(x, idx, key, metric)
        oi, ok = oracle.propagate(x, idx, key, metric)
        np.testing.assert_array_equal(gi, oi)
        np.testing.assert_array_equal(gk.view(np.uint32), ok.view(np.uint32))
        idx, key = oi, ok


KATS = sorted(p.stem for p in GOLDEN.glob("kat_*.npz"))


@pytest.mark.parametrize("name", KATS)
def test_kat_on_gpu(lib, name):
    z = np.load(GOLDEN / f"{name}.npz")
    x, k, metric = z["points"], int(z["k"]), int(z["metric"])
    idx, dist = lib.knn_build(x, k, 2, x.shape[0], 1, metric)
    np.testing.assert_array_equal(idx, z["idx"])
    np.testing.assert_allclose(dist, z["dist"], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_exact_fp64_matches_cpu(lib, oracle, metric):
    x = _rand(3000, 19, 4, "int" if metric == 1 else "gauss")
    q = np.arange(0, 3000, 7)
    gi, gd = lib.exact_fp64(x, 11, q, metric)
    oi, od = oracle.exact(x, 11, q, metric)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)


@pytest.mark.parametrize("metric", [0, 1, 2])
@pytest.mark.parametrize("n,d,k", [(2000, 16, 7), (3000, 37, 12), (2500, 130, 33), (4000, 300, 5)])
def test_float16_input_matches_float32_of_same_values(lib, oracle, metric, n, d, k):
    """FP16 input: propagation gathers the FP16 rows themselves (row slices of
    128 dims, rows padded to 8); the FP16 -> FP32 conversion is exact, so the
    graph equals the oracle's on the same values as float32."""
    x16 = _rand(n, d, 12 + d).astype(np.float16)
    got = lib.knn_build(x16, k, 3, 32 + k, 2, metric)
    want = oracle.knn_build(x16.astype(np.float32), k, 3, 32 + k, 2, metric)
    _same(got, want, f"f16 d={d} metric={metric}")


def test_device_pointers_and_stats(lib, oracle):
    import ctypes

    import torch
    x = _rand(3000, 12, 13)
    xd = torch.from_numpy(x).cuda()
    k = 9
    idx = torch.empty((3000, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((3000, k), dtype=torch.float32, device="cuda")
    opt = lib.default_options(points_on_device=1, outputs_on_device=1)
    st = lib.KnnStats()
    st.struct_size = ctypes.sizeof(lib.KnnStats)
    rc = lib.load_library().knn_build_ex(None, xd.data_ptr(), 3000, 12, k, 3, 24, 2, 0, 0,
                                         idx.data_ptr(), dist.data_ptr(), ctypes.byref(opt),
                                         ctypes.byref(st))
    assert rc == 0
    want = oracle.knn_build(x, k, 3, 24, 2, 0)
    _same((idx.cpu().numpy(), dist.cpu().numpy()), want, "device pointers")
    assert st.depth == 7 and st.ms_total > 0 and st.leaf_pairs > 0
    assert st.prop_candidates[0] > st.prop_candidates[1] > 0  # flags skip settled pairs


def test_repeated_calls_same_context(lib):
    x = _rand(2500, 10, 14)
    ctx = lib.Context()
    a = lib.knn_build(x, 5, 2, 20, 1, 0, context=ctx.handle)
    b = lib.knn_build(x, 5, 2, 20, 1, 0, context=ctx.handle)
    _same(a, b, "repeat")
    assert ctx.scratch_bytes > 0
    ctx.close()


def test_normalize_reference_matches_numpy_order(lib):
    """Column mean by sequential float32 sums, then division of dims < 256 by
    the largest |x| over those dims (dims >= 256 centred only)."""
    x = _rand(300, 260, 15)
    got = lib.normalize_reference(x)
    want = x.copy()
    for dim in range(260):
        s = np.float32(0)
        for v in x[:, dim]:
            s = np.float32(s + v)
        want[:, dim] = x[:, dim] - np.float32(s / np.float32(300))
    m = np.float32(np.abs(want[:, :256]).max())
    want[:, :256] = want[:, :256] / m
    np.testing.assert_array_equal(got, want)


def test_errors_on_gpu(lib):
    x = _rand(10, 3, 1)
    with pytest.raises(lib.KnnError) as e:
        lib.knn_build(x, 10, 1, 4, 0, 0)
    assert e.value.status == -2

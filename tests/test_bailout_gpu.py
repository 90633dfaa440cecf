"""The tensor-core tile kernel's give-up path, made to run without a real
timeout: knn_test_fail_next_tile_wait sets the build's error words before its
launches, so every block of k_leaf_tc issues no MMA, frees its tensor memory
and returns.  The build must report KNN_ERR_TIMEOUT (at once when synchronous,
through knn_context_status when asynchronous), report it only once, and the
next build on the same context must give the normal graph bit for bit.  The
real wait limit is untouched; nothing here makes a device wait run out."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

TIMEOUT = -5


def _case():
    acknn = load_package()
    x = acknn.workloads.integer_mixture(seed=3, n=30_000, d=64)
    return acknn, x, dict(k=16, trees=4, leaf=256, props=1, metric=0)


def test_synchronous_build_reports_timeout_then_recovers():
    acknn, x, p = _case()
    lib = acknn.load_library()
    ctx = acknn.Context(0)
    try:
        good_i, good_d = acknn.knn_build(x, p["k"], p["trees"], p["leaf"], p["props"], p["metric"],
                                         precision=acknn.PREC_BF16_RERANK, context=ctx.handle)
        assert lib.knn_test_fail_next_tile_wait(ctx.handle) == 0
        with pytest.raises(acknn.KnnError) as e:
            acknn.knn_build(x, p["k"], p["trees"], p["leaf"], p["props"], p["metric"],
                            precision=acknn.PREC_BF16_RERANK, context=ctx.handle)
        assert e.value.status == TIMEOUT
        assert lib.knn_context_status(ctx.handle, None) == 0  # reported once
        idx, dist = acknn.knn_build(x, p["k"], p["trees"], p["leaf"], p["props"], p["metric"],
                                    precision=acknn.PREC_BF16_RERANK, context=ctx.handle)
        assert np.array_equal(idx, good_i)
        assert np.array_equal(dist.view(np.uint32), good_d.view(np.uint32))
    finally:
        ctx.close()


def test_asynchronous_build_reports_timeout_through_context_status():
    import torch

    acknn, x, p = _case()
    lib = acknn.load_library()
    torch.cuda.set_device(0)
    n, d = x.shape
    xd = torch.from_numpy(x).cuda()
    oi = torch.empty((n, p["k"]), dtype=torch.int32, device="cuda")
    od = torch.empty((n, p["k"]), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    ctx = acknn.Context(0)

    def build():
        opt = acknn.default_options(points_on_device=1, outputs_on_device=1, stream=stream.cuda_stream,
                                    precision=acknn.PREC_BF16_RERANK)
        return lib.knn_build_ex(ctx.handle, xd.data_ptr(), n, d, p["k"], p["trees"], p["leaf"], p["props"],
                                p["metric"], 0, oi.data_ptr(), od.data_ptr(), ctypes.byref(opt), None)

    try:
        assert build() == 0
        assert lib.knn_context_status(ctx.handle, ctypes.c_void_p(stream.cuda_stream)) == 0
        good_i, good_d = oi.cpu().clone(), od.cpu().clone()
        assert lib.knn_test_fail_next_tile_wait(ctx.handle) == 0
        assert build() == 0  # queued: the failure cannot be known yet
        assert lib.knn_context_status(ctx.handle, ctypes.c_void_p(stream.cuda_stream)) == TIMEOUT
        assert lib.knn_context_status(ctx.handle, ctypes.c_void_p(stream.cuda_stream)) == 0
        assert build() == 0
        assert lib.knn_context_status(ctx.handle, ctypes.c_void_p(stream.cuda_stream)) == 0
        assert torch.equal(oi.cpu(), good_i) and torch.equal(od.cpu(), good_d)
    finally:
        stream.synchronize()
        ctx.close()


def test_batch_build_reports_timeout_then_recovers():
    acknn, _, p = _case()
    lib = acknn.load_library()
    xs = [acknn.workloads.gaussian_mixture(3000 + 500 * i, 32, 8, seed=i) for i in range(3)]
    ctx = acknn.Context(0)
    try:
        good = acknn.knn_build_batch(xs, 8, 3, 64, 1, 0, seeds=[0, 1, 2], precision=acknn.PREC_BF16_RERANK,
                                     context=ctx.handle)
        assert lib.knn_test_fail_next_tile_wait(ctx.handle) == 0
        with pytest.raises(acknn.KnnError) as e:
            acknn.knn_build_batch(xs, 8, 3, 64, 1, 0, seeds=[0, 1, 2], precision=acknn.PREC_BF16_RERANK,
                                  context=ctx.handle)
        assert e.value.status == TIMEOUT
        again = acknn.knn_build_batch(xs, 8, 3, 64, 1, 0, seeds=[0, 1, 2], precision=acknn.PREC_BF16_RERANK,
                                      context=ctx.handle)
        for (gi, gd), (ai, ad) in zip(good, again):
            assert np.array_equal(gi, ai) and np.array_equal(gd.view(np.uint32), ad.view(np.uint32))
    finally:
        ctx.close()

"""knn_exact_fp64_noalloc: the FP64 exact k-NN for callers that cannot allocate
device memory while they run (for example a process that hands all device
memory to its own pool at start-up).  It works from caller-owned device buffers
and one fixed scratch array compiled into the library.

Checked through the C ABI against knn_exact_fp64 (the allocating entry point):
the two must agree exactly, on two calls in a row that reuse the shared
scratch.  This file is collected last so a stop-at-first-failure run has
already run every other test; it also passes alone in a fresh process."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _noalloc(lib, xd, n, d, k, metric, qd, nq, torch):
    idx = torch.full((nq, k), -7, dtype=torch.int32, device="cuda")
    dist = torch.full((nq, k), -7.0, dtype=torch.float64, device="cuda")
    rc = lib.knn_exact_fp64_noalloc(xd.data_ptr(), n, d, k, metric, qd.data_ptr(), nq,
                                    idx.data_ptr(), dist.data_ptr(), None)
    return rc, idx.cpu().numpy(), dist.cpu().numpy()


def test_noalloc_matches_allocating_entry_twice():
    torch = pytest.importorskip("torch")
    acknn = load_package()
    lib = acknn.load_library()
    rng = np.random.Generator(np.random.PCG64(42))
    cases = [  # (n, d, k, metric): calls in a row, different shapes and metrics
        (5000, 24, 10, 0),
        (3000, 7, 16, 2),
        (4000, 33, 12, 1),
    ]
    for n, d, k, metric in cases:
        x = rng.standard_normal((n, d), dtype=np.float32)
        q = np.sort(rng.choice(n, size=700, replace=False)).astype(np.int64)
        want_i, want_d = acknn.exact_fp64(x, k, q, metric)
        xd = torch.from_numpy(x).cuda()
        qd = torch.from_numpy(q).cuda()
        rc, got_i, got_d = _noalloc(lib, xd, n, d, k, metric, qd, len(q), torch)
        assert rc == 0, lib.knn_last_error()
        np.testing.assert_array_equal(got_i, want_i)
        np.testing.assert_array_equal(got_d, want_d)


def test_noalloc_rejects_oversize_and_bad_ids():
    torch = pytest.importorskip("torch")
    acknn = load_package()
    lib = acknn.load_library()
    n, d, k = 2000, 8, 8
    x = torch.randn((n, d), dtype=torch.float32, device="cuda")
    # 200,000 queries x 8 neighbours need ~25 MB of scratch: more than it holds
    big = torch.zeros(200_000, dtype=torch.int64, device="cuda")
    rc, _, _ = _noalloc(lib, x, n, d, k, 0, big, big.numel(), torch)
    assert rc == -1 and b"scratch" in lib.knn_last_error()
    bad = torch.tensor([0, 5, n + 3], dtype=torch.int64, device="cuda")
    rc, _, _ = _noalloc(lib, x, n, d, k, 0, bad, 3, torch)
    assert rc == -1 and b"out of range" in lib.knn_last_error()
    # the scratch is usable again after a rejected call
    good = torch.arange(0, n, 9, dtype=torch.int64, device="cuda")
    rc, gi, gd = _noalloc(lib, x, n, d, k, 0, good, good.numel(), torch)
    assert rc == 0
    wi, wd = acknn.exact_fp64(x.cpu().numpy(), k, good.cpu().numpy(), 0)
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gd, wd)


def test_noalloc_allocates_no_device_memory():
    """After a warm-up call, further calls (the same request and a larger one
    that still fits) leave the device's free memory unchanged: the outputs
    are the caller's and the scratch is the library's fixed array."""
    torch = pytest.importorskip("torch")
    acknn = load_package()
    lib = acknn.load_library()
    n, d, k = 20_000, 40, 16
    x = torch.randn((n, d), dtype=torch.float32, device="cuda")
    small = torch.arange(0, n, 40, dtype=torch.int64, device="cuda")
    large = torch.arange(0, n, 4, dtype=torch.int64, device="cuda")
    outs = {q.numel(): (torch.empty((q.numel(), k), dtype=torch.int32, device="cuda"),
                        torch.empty((q.numel(), k), dtype=torch.float64, device="cuda")) for q in (small, large)}

    def call(q, metric):
        oi, od = outs[q.numel()]
        return lib.knn_exact_fp64_noalloc(x.data_ptr(), n, d, k, metric, q.data_ptr(), q.numel(),
                                          oi.data_ptr(), od.data_ptr(), None)

    assert call(small, 0) == 0, lib.knn_last_error()  # warm-up: module and scratch set up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for q, metric in ((small, 0), (large, 1), (large, 2), (small, 0)):
        assert call(q, metric) == 0, lib.knn_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0

"""Sharded builds over torch.distributed (gloo, world size 2 and 3, CPU): the
exchange logic of approximate-cuda-knn_b200/sharded.py -- tree shares, the
all-gather and merge of every rank's lists, range-wise propagation -- gives
the single build's graph bit for bit.  Each rank's compute is the CPU
restatement (oracle) here; tests/test_sharded_gpu.py runs the library's
kernels through the same steps."""
from __future__ import annotations

import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ORACLE_DIR, Oracle, load_package


def merge_lists_host(idx_all, key_all, k):
    """The merge rule: per point, the k best distinct ids by (key, id)."""
    lists, n, _ = idx_all.shape
    out_i = np.full((n, k), -1, dtype=np.int32)
    out_k = np.full((n, k), np.inf, dtype=np.float32)
    for i in range(n):
        ids = idx_all[:, i, :].ravel()
        keys = key_all[:, i, :].ravel()
        ok = ids >= 0
        ids, keys = ids[ok], keys[ok]
        order = np.lexsort((ids.astype(np.uint32), keys))
        seen, m = set(), 0
        for j in order:
            if ids[j] in seen:
                continue
            seen.add(ids[j])
            out_i[i, m], out_k[i, m] = ids[j], keys[j]
            m += 1
            if m == k:
                break
    return out_i, out_k


class OracleBackend:
    """Per-rank compute by the CPU restatement, on torch CPU tensors."""

    def __init__(self, oracle, sharded):
        self.o = oracle
        self.Lists = sharded.Lists
        self.share = sharded.tree_share

    def local_trees(self, x, k, trees, leaf, metric, seed, rank, world):
        xn = x.numpy()
        n = xn.shape[0]
        count = self.share(trees, rank, world)
        if count == 0:
            return self.Lists(torch.full((n, k), -1, dtype=torch.int32), torch.full((n, k), float("inf")))
        perm = self.o.build_trees_ex(xn, count, leaf, seed, rank, world)
        idx, key = self.o.leaf_stage(xn, k, perm, leaf, metric)
        return self.Lists(torch.from_numpy(idx), torch.from_numpy(key))

    def merge(self, idx_all, key_all, k, metric, as_distance=False):
        i, kk = merge_lists_host(idx_all.numpy(), key_all.numpy(), k)
        if as_distance:
            kk = self.o.finalize(kk, metric)
        return self.Lists(torch.from_numpy(i), torch.from_numpy(kk))

    def propagate_range(self, x, lst, k, metric, r0, r1):
        oi, ok = self.o.propagate(x.numpy(), lst.idx.numpy(), lst.key.numpy(), metric)
        idx, key = lst.idx.clone(), lst.key.clone()
        idx[r0:r1] = torch.from_numpy(oi[r0:r1])
        key[r0:r1] = torch.from_numpy(ok[r0:r1])
        return self.Lists(idx, key, torch.zeros((x.shape[0], (k + 31) // 32), dtype=torch.int32))


def _worker(rank, world, port, case, out_path):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        acknn = load_package()
        sharded = acknn.sharded
        oracle = Oracle(ORACLE_DIR / "liboracle.so")
        n, d, k, trees, leaf, props, metric, seed = case
        x = torch.from_numpy(acknn.workloads.gaussian_mixture(n, d, 6, 31))
        idx, dist_ = sharded.build_sharded(OracleBackend(oracle, sharded), sharded.TorchComm(), x, k, trees, leaf,
                                           props, metric, seed)
        if rank == 0:
            np.savez(out_path, idx=idx.numpy(), dist=dist_.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world,case", [
    (2, (3000, 12, 8, 5, 40, 2, 0, 7)),
    (2, (2500, 9, 6, 4, 30, 2, 2, 3)),
    (3, (2000, 8, 5, 4, 25, 1, 1, 11)),   # uneven tree shares (2, 1, 1)
    (2, (1500, 6, 5, 1, 30, 1, 0, 2)),    # one tree: rank 1 contributes empty lists
])
def test_sharded_equals_single_build(oracle, world, case):
    n, d, k, trees, leaf, props, metric, seed = case
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "r0.npz")
        mp.start_processes(_worker, args=(world, _free_port(), case, out), nprocs=world, join=True,
                           start_method="spawn")
        got = np.load(out)
    acknn = load_package()
    x = acknn.workloads.gaussian_mixture(n, d, 6, 31)
    wi, wd = oracle.knn_build(x, k, trees, leaf, props, metric, seed=seed)
    np.testing.assert_array_equal(got["idx"], wi)
    np.testing.assert_array_equal(got["dist"].view(np.uint32), wd.view(np.uint32))


def test_tree_shares_and_ranges():
    sharded = load_package().sharded
    assert [sharded.tree_share(10, r, 4) for r in range(4)] == [3, 3, 2, 2]
    assert sum(sharded.tree_share(7, r, 3) for r in range(3)) == 7
    n, w = 1001, 4
    rs = [sharded.point_range(n, r, w) for r in range(w)]
    assert rs[0][0] == 0 and rs[-1][1] == n
    assert all(rs[i][1] == rs[i + 1][0] for i in range(w - 1))

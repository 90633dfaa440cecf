"""The sharded build's GPU primitives (global tree indices, the device list
merge, range-wise propagation) run as G virtual ranks on one GPU and give the
single build's graph bit for bit; one rank over NCCL runs build_sharded end
to end."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch

from conftest import load_package

pytestmark = pytest.mark.gpu


def _virtual_sharded(acknn, x, k, trees, leaf, props, metric, seed, world):
    sh = acknn.sharded
    be = sh.LibraryBackend(acknn, 0)
    xd = torch.from_numpy(x).cuda()
    n = x.shape[0]
    parts = [be.local_trees(xd, k, trees, leaf, metric, seed, r, world) for r in range(world)]
    # as build_sharded: each rank merges the G lists of its own point range
    idx_all, key_all = torch.stack([p.idx for p in parts]), torch.stack([p.key for p in parts])
    idx, key = torch.empty_like(parts[0].idx), torch.empty_like(parts[0].key)
    for r in range(world):
        a, b = sh.point_range(n, r, world)
        m = be.merge(idx_all[:, a:b].contiguous(), key_all[:, a:b].contiguous(), k, metric)
        idx[a:b], key[a:b] = m.idx, m.key
    lst = sh.Lists(idx, key)
    for _ in range(props):
        nxt = [be.propagate_range(xd, lst, k, metric, *sh.point_range(n, r, world)) for r in range(world)]
        idx, key, flags = lst.idx.clone(), lst.key.clone(), nxt[0].flags.clone()
        for r, p in enumerate(nxt):
            a, b = sh.point_range(n, r, world)
            idx[a:b], key[a:b], flags[a:b] = p.idx[a:b], p.key[a:b], p.flags[a:b]
        lst = sh.Lists(idx, key, flags)
    fin = be.merge(lst.idx.unsqueeze(0), lst.key.unsqueeze(0), k, metric, as_distance=True)
    return fin.idx.cpu().numpy(), fin.key.cpu().numpy()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("metric", [0, 1, 2])
def test_virtual_ranks_equal_single_build(acknn, world, metric):
    x = acknn.workloads.gaussian_mixture(20000, 24, 16, 40 + metric)
    k, trees, leaf, props, seed = 12, 5, 48, 2, 9
    gi, gd = _virtual_sharded(acknn, x, k, trees, leaf, props, metric, seed, world)
    wi, wd = acknn.knn_build(x, k, trees, leaf, props, metric, seed=seed)
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gd.view(np.uint32), wd.view(np.uint32))


def test_merge_of_tree_shares_is_the_initial_graph(acknn):
    """Lists of the trees {0, 2} and {1} merged = the lists of trees {0, 1, 2}."""
    x = acknn.workloads.gaussian_mixture(15000, 16, 8, 5)
    gi, gd = _virtual_sharded(acknn, x, 10, 3, 40, 0, 0, 1, 2)
    wi, wd = acknn.knn_build(x, 10, 3, 40, 0, 0, seed=1)
    np.testing.assert_array_equal(gi, wi)
    np.testing.assert_array_equal(gd, wd)


def test_merge_lists_host_and_device_agree(acknn):
    rng = np.random.Generator(np.random.PCG64(3))
    lists, n, k = 3, 500, 8
    idx = np.empty((lists, n, k), dtype=np.int32)
    key = np.empty((lists, n, k), dtype=np.float32)
    for l in range(lists):
        for i in range(n):
            ids = rng.choice(60, size=k, replace=False).astype(np.int32)
            keys = (ids % 17).astype(np.float32)  # equal keys across lists for equal ids, ties by id
            o = np.lexsort((ids, keys))
            idx[l, i], key[l, i] = ids[o], keys[o]
    idx[1, 7, 3:] = -1
    key[1, 7, 3:] = np.inf
    lib = acknn.load_library()
    oi = np.empty((n, k), dtype=np.int32)
    ok = np.empty((n, k), dtype=np.float32)
    opt = acknn.default_options()
    import ctypes
    assert lib.knn_merge_lists(None, idx.ctypes.data, key.ctypes.data, lists, n, k, 1, 0, oi.ctypes.data,
                               ok.ctypes.data, ctypes.byref(opt)) == 0
    for i in range(n):
        cand = {}
        for l in range(lists):
            for s in range(k):
                if idx[l, i, s] >= 0:
                    cand[int(idx[l, i, s])] = float(key[l, i, s])
        best = sorted(cand.items(), key=lambda t: (t[1], t[0]))[:k]
        assert [b[0] for b in best] == oi[i].tolist()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_build_sharded_one_rank_nccl(acknn):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        x = acknn.workloads.gaussian_mixture(30000, 32, 16, 8)
        sh = acknn.sharded
        gi, gd = sh.build_sharded(sh.LibraryBackend(acknn, 0), sh.TorchComm(), torch.from_numpy(x).cuda(), 15,
                                  6, 64, 2, 0, 4)
        wi, wd = acknn.knn_build(x, 15, 6, 64, 2, 0, seed=4)
        np.testing.assert_array_equal(gi.cpu().numpy(), wi)
        np.testing.assert_array_equal(gd.cpu().numpy(), wd)
    finally:
        dist.destroy_process_group()

"""Sharded k-NN graph builds: one process per GPU, torch.distributed for the
exchanges, the library's kernels for all compute.

Rank r of G builds the global trees r, r+G, r+2G, ... (the same trees a
single build would make: a tree's splits depend on its global index and the
seed only) and the initial lists over them.  The rows of every point range
then go to the range's owner (one all-to-all: each rank receives the G lists
of its n/G points), which merges them (the k best distinct ids of their union
-- the initial graph over all trees, since the k best of a union are the k
best of the union of each part's k best), and one all-gather of the merged
ranges gives every rank the whole initial graph: 2 n k 8 bytes received per
rank instead of the G n k 8 of gathering every rank's full lists, and each
point merged once instead of on every rank.  Each propagation step then runs
on a contiguous point range per rank and the ranges are all-gathered.  The
graph is therefore the single-GPU build's, bit for bit.

The per-rank compute goes through a backend object (`LibraryBackend`: the
C ABI on device tensors).  The exchange goes through torch.distributed
(NCCL between GPUs; any backend whose all_gather takes the tensors).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass


def tree_share(trees: int, rank: int, world: int) -> int:
    """Number of global trees rank builds: those t < trees with t % world == rank."""
    return len(range(rank, trees, world))


def point_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous point range of a rank for the propagation steps."""
    return n * rank // world, n * (rank + 1) // world


@dataclass
class Lists:
    """Per-point neighbour lists: idx int32 [n, k], key float32 [n, k] (keys:
    squared L2 / L1 / 1-cos), flags uint32 [n, ceil(k/32)] or None (all new)."""
    idx: object
    key: object
    flags: object = None


class LibraryBackend:
    """Per-rank compute on one GPU through the C ABI (device tensors)."""

    def __init__(self, acknn, device: int = 0, precision: int = 0):
        import torch

        self.torch = torch
        self.acknn = acknn
        self.precision = precision  # leaf stage of the local trees (knn_options.precision)
        self.lib = acknn.load_library()
        self.device = device
        self.ctx = acknn.Context(device)

    def _opt(self, x=None, **kw):
        # torch's current stream: the library's launches are ordered after the
        # torch ops that allocate and fill the tensors it reads and writes
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        if x is not None:
            kw["dtype"] = self.acknn.F16 if x.dtype == self.torch.float16 else self.acknn.F32
        return self.acknn.default_options(device=self.device, points_on_device=1, outputs_on_device=1,
                                          stream=stream, **kw)

    def empty_lists(self, n: int, k: int) -> Lists:
        t = self.torch
        return Lists(t.full((n, k), -1, dtype=t.int32, device=f"cuda:{self.device}"),
                     t.full((n, k), float("inf"), dtype=t.float32, device=f"cuda:{self.device}"))

    def local_trees(self, x, k, trees, leaf, metric, seed, rank, world) -> Lists:
        """Initial lists over the global trees rank, rank+world, ..."""
        n, d = x.shape
        count = tree_share(trees, rank, world)
        out = self.empty_lists(n, k)
        if count == 0:
            return out
        opt = self._opt(x, tree_offset=rank, tree_stride=world, raw_keys=1, precision=self.precision)
        rc = self.lib.knn_build_ex(self.ctx.handle, x.data_ptr(), n, d, k, count, leaf, 0, metric, seed,
                                   out.idx.data_ptr(), out.key.data_ptr(), ctypes.byref(opt), None)
        self._check(rc)
        return out

    def merge(self, idx_all, key_all, k, metric, as_distance=False) -> Lists:
        """k best distinct ids of the stacked lists [lists, n, k]."""
        lists, n = idx_all.shape[0], idx_all.shape[1]
        out = self.empty_lists(n, k)
        rc = self.lib.knn_merge_lists(self.ctx.handle, idx_all.data_ptr(), key_all.data_ptr(), lists, n, k, metric,
                                      int(as_distance), out.idx.data_ptr(), out.key.data_ptr(),
                                      ctypes.byref(self._opt()))
        self._check(rc)
        return out

    def propagate_range(self, x, lst: Lists, k, metric, r0, r1) -> Lists:
        t = self.torch
        n, d = x.shape
        kw = (k + 31) // 32
        out = Lists(lst.idx.clone(), lst.key.clone(),
                    t.zeros((n, kw), dtype=t.int32, device=f"cuda:{self.device}"))
        flags = lst.flags.data_ptr() if lst.flags is not None else None
        rc = self.lib.knn_propagate_range(self.ctx.handle, x.data_ptr(), n, d, k, metric, r0, r1,
                                          lst.idx.data_ptr(), lst.key.data_ptr(), flags, out.idx.data_ptr(),
                                          out.key.data_ptr(), out.flags.data_ptr(), ctypes.byref(self._opt(x)))
        self._check(rc)
        return out

    def _check(self, rc):
        if rc:
            raise self.acknn.KnnError(rc, self.lib.knn_last_error().decode())


class TorchComm:
    """All-gather over torch.distributed (the default process group)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    def all_gather_stack(self, t):
        """[world, *t.shape] of every rank's t (same shape on all ranks)."""
        import torch

        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(parts, t.contiguous(), group=self.group)
        return torch.stack(parts)

    def all_gather_rows(self, t, n):
        """Rows [n*r/world, n*(r+1)/world) of t from every rank r, assembled."""
        r0, r1 = point_range(n, self.rank, self.world)
        return self.all_gather_range(t[r0:r1], n)

    def all_gather_range(self, part, n):
        """[n, ...] assembled from every rank's rows of its own point range
        (`part`: this rank's rows, [r1 - r0, ...])."""
        import torch

        chunk = (n + self.world - 1) // self.world
        r0, r1 = point_range(n, self.rank, self.world)
        pad = torch.zeros((chunk,) + tuple(part.shape[1:]), dtype=part.dtype, device=part.device)
        pad[: r1 - r0] = part
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        self.dist.all_gather(parts, pad, group=self.group)
        out = torch.empty((n,) + tuple(part.shape[1:]), dtype=part.dtype, device=part.device)
        for r, p in enumerate(parts):
            a, b = point_range(n, r, self.world)
            out[a:b] = p[: b - a]
        return out

    def all_to_all_rows(self, t, n):
        """Rows of every rank's point range to that rank: returns [world,
        r1 - r0, ...], the rows of this rank's range [r0, r1) from every rank
        (t: [n, ...], this rank's rows of all points)."""
        import torch

        chunk = (n + self.world - 1) // self.world
        tail = tuple(t.shape[1:])
        send = torch.zeros((self.world * chunk,) + tail, dtype=t.dtype, device=t.device)
        for q in range(self.world):
            a, b = point_range(n, q, self.world)
            send[q * chunk: q * chunk + (b - a)] = t[a:b]
        recv = torch.empty_like(send)
        self.dist.all_to_all_single(recv, send, group=self.group)
        r0, r1 = point_range(n, self.rank, self.world)
        return recv.view((self.world, chunk) + tail)[:, : r1 - r0]


def build_sharded(backend, comm, x, k: int, trees: int, leaf: int, props: int, metric: int = 0,
                  seed: int = 0):
    """k-NN graph of x ([n, d] on this rank's device, the same on every rank)
    built by comm.world ranks.  Returns (idx [n, k], dist [n, k]) on every rank."""
    n = x.shape[0]
    world, rank = comm.world, comm.rank
    local = backend.local_trees(x, k, trees, leaf, metric, seed, rank, world)
    # this rank's point range: its G lists, merged here, then assembled everywhere
    idx_mine = comm.all_to_all_rows(local.idx, n).contiguous()
    key_mine = comm.all_to_all_rows(local.key, n).contiguous()
    merged = backend.merge(idx_mine, key_mine, k, metric)
    lst = Lists(comm.all_gather_range(merged.idx, n), comm.all_gather_range(merged.key, n))
    for _ in range(props):
        r0, r1 = point_range(n, rank, world)
        nxt = backend.propagate_range(x, lst, k, metric, r0, r1)
        lst = Lists(comm.all_gather_rows(nxt.idx, n), comm.all_gather_rows(nxt.key, n),
                    comm.all_gather_rows(nxt.flags, n))
    final = backend.merge(lst.idx.unsqueeze(0), lst.key.unsqueeze(0), k, metric, as_distance=True)
    return final.idx, final.key

"""List semantics of the tensor-core leaf stage's merge (k_leaf_tc), restated on the CPU.

A row's list is 32 (key, id) entries ascending by (key, id); the first kq are written back. Per
tree, candidates arrive in rounds of up to 64 columns. The merge admits them in one of these ways:
  * one by one: warp_insert1, which places a candidate before the first entry it precedes and
    drops the last entry, or drops the candidate when it precedes none;
  * a round's half of many survivors: sorted and merged, keeping the 32 smallest (first tree);
  * duplicates either dropped by an id check against the first kq entries, or removed before the
    filter when the row's listed ids are known up front (the exclusion).
The filter may let through extra candidates (it is widened to cover rounding). Whatever the path,
the first kq entries must equal the kq smallest distinct (key, id) of the initial list and every
candidate.
"""
from __future__ import annotations

import numpy as np

INF = np.float32(np.inf)
NOID = 0xFFFFFFFF


def less(a, b):
    return (a[0], a[1]) < (b[0], b[1])


def insert1(L, c):
    for p in range(32):
        if less(c, L[p]):
            L.insert(p, c)
            L.pop()
            return


def merge_batch(L, batch):
    return sorted(L + batch, key=lambda e: (e[0], e[1]))[:32]


def run_tree(L, cands, kq, first, exclude, widen, rng):
    """cands: (key, id) of one tree's block for this row, each id once, in column order."""
    listed = {e[1] for e in L[:kq] if e[1] != NOID}
    for r0 in range(0, len(cands), 64):
        tail = L[kq - 1][0]
        for h0 in (r0, r0 + 32):
            half = cands[h0:h0 + 32]
            surv = []
            for c in half:
                if exclude and c[1] in listed:
                    continue
                passes = c[0] <= tail or (widen and c[0] <= tail * 1.0001 + 1e-6)
                if passes:
                    surv.append(c)
            if first and len(surv) >= 12:
                L = merge_batch(L, surv)
                continue
            for c in surv:
                if not first and not exclude and any(e[1] == c[1] for e in L[:kq]):
                    continue
                insert1(L, c)
    return L


def run_tree_tile(L, cands, kq, first, exclude, widen, rng):
    """The per-tile schedule: the filter bound is the tail at the tile's start
    for all 128 columns; then the tile's 32-column slices are merged in column
    order, a slice with many survivors sorted and merged in one go (first tree
    only), the others one survivor at a time."""
    listed = {e[1] for e in L[:kq] if e[1] != NOID}
    for t0 in range(0, len(cands), 128):
        tail = L[kq - 1][0]
        slices = []
        for h0 in range(t0, min(t0 + 128, len(cands)), 32):
            surv = []
            for c in cands[h0:h0 + 32]:
                if exclude and c[1] in listed:
                    continue
                if c[0] <= tail or (widen and c[0] <= tail * 1.0001 + 1e-6):
                    surv.append(c)
            slices.append(surv)
        for surv in slices:
            if first and len(surv) >= 12:
                L = merge_batch(L, surv)
                continue
            for c in surv:
                if not first and not exclude and any(e[1] == c[1] for e in L[:kq]):
                    continue
                insert1(L, c)
    return L


def expected(initial, trees, kq):
    best = {}
    for e in initial:
        if e[1] != NOID:
            best[e[1]] = e[0]
    for cands in trees:
        for k, i in cands:
            best[i] = k
    return sorted(((k, i) for i, k in best.items()), key=lambda e: (e[0], e[1]))[:kq]


def test_every_merge_path_keeps_the_kq_best():
    rng = np.random.Generator(np.random.PCG64(4))
    for trial in range(300):
        kq = int(rng.choice([8, 16, 20, 32]))
        npts = 400
        key_of = np.round(rng.random(npts) * 50).astype(np.float32)  # ties on purpose
        T = 4
        trees = []
        for _ in range(T):
            nb = int(rng.integers(40, 300))
            ids = rng.choice(npts, size=nb, replace=False)
            trees.append([(float(key_of[i]), int(i)) for i in ids])
        want = expected([], trees, kq)
        for exclude in (False, True):
            for widen in (False, True):
                L = [(float(INF), NOID)] * 32
                for t, cands in enumerate(trees):
                    L = run_tree(L, cands, kq, t == 0, exclude and t > 0, widen, rng)
                    L = L[:kq] + [(float(INF), NOID)] * (32 - kq)  # only kq entries are kept
                got = [e for e in L[:kq] if e[1] != NOID]
                assert got == want[:len(got)] and len(got) == min(kq, len(want)), (trial, exclude, widen)


def test_tile_schedule_keeps_the_kq_best():
    """One filter bound per 128-column tile (looser than a bound refreshed
    after every 64 columns): the kq best are still kept, as the result of
    every path is the kq smallest of the union."""
    rng = np.random.Generator(np.random.PCG64(9))
    for trial in range(300):
        kq = int(rng.choice([8, 16, 20, 32]))
        npts = 600
        key_of = np.round(rng.random(npts) * 60).astype(np.float32)  # ties on purpose
        trees = []
        for _ in range(4):
            nb = int(rng.integers(40, 500))
            ids = rng.choice(npts, size=nb, replace=False)
            trees.append([(float(key_of[i]), int(i)) for i in ids])
        want = expected([], trees, kq)
        for exclude in (False, True):
            for widen in (False, True):
                L = [(float(INF), NOID)] * 32
                for t, cands in enumerate(trees):
                    L = run_tree_tile(L, cands, kq, t == 0, exclude and t > 0, widen, rng)
                    L = L[:kq] + [(float(INF), NOID)] * (32 - kq)
                got = [e for e in L[:kq] if e[1] != NOID]
                assert got == want[:len(got)] and len(got) == min(kq, len(want)), (trial, exclude, widen)

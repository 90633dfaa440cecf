"""Listed-id exclusion of the tensor-core leaf stage (k_leaf_tc, later trees), restated on the CPU.

At block start each row's listed ids that lie in the block are turned into sorted column
positions (kXEnd = 0xFFFF after them). Thread (row, half) then walks those positions with one
pointer over all of the block's steps: for tile c0 (128 columns) and round rb (64 columns) its
32 columns are [c0 + rb + 32 half, +32). Entries below that range belong to the other half, or
to ranges already passed, and are skipped; the ones inside set bits of its exclusion mask. Each
listed column must be excluded exactly once, by the thread that owns it, and no other column.
"""
from __future__ import annotations

import numpy as np

X_END = 0xFFFF
TILE, ROUND = 128, 64


def masks_by_walk(positions: np.ndarray, nb: int) -> dict:
    xp = list(np.sort(positions)) + [X_END] * (33 - len(positions))
    out = {}
    for half in (0, 1):
        ptr = 0
        for c0 in range(0, nb, TILE):
            mc = min(TILE, nb - c0)
            for rb in range(0, mc, ROUND):
                lo_c = c0 + rb + 32 * half
                ex = 0
                p = xp[ptr]
                while p < lo_c + 32:
                    if p >= lo_c:
                        ex |= 1 << (p - lo_c)
                    ptr += 1
                    p = xp[ptr]
                out[(c0, rb, half)] = ex
    return out


def test_walk_marks_exactly_the_listed_columns():
    rng = np.random.Generator(np.random.PCG64(2))
    for _ in range(2000):
        nb = int(rng.integers(1, 3000))
        kq = int(rng.integers(1, 33))
        cnt = int(rng.integers(0, min(kq, nb) + 1))
        pos = rng.choice(nb, size=cnt, replace=False)
        if cnt and rng.random() < 0.3:  # positions on range boundaries
            pos[0] = (pos[0] // 32) * 32
            pos = np.unique(pos)
        got = masks_by_walk(pos, nb)
        marked = set()
        for (c0, rb, half), ex in got.items():
            for b in range(32):
                if ex >> b & 1:
                    col = c0 + rb + 32 * half + b
                    assert col < nb
                    assert col not in marked
                    marked.add(col)
        assert marked == set(int(p) for p in pos)

"""CPU restatement of the FP32 leaf stage's tile-pair schedule (csrc/leaf_knn.cu,
k_leaf_pair) and of the key symmetry it rests on.

A leaf of T tiles is swept in T' rounds (T' = T rounded up to even): rounds
r < T'-1 pair tile r with tile T'-1 and (r + i) mod (T'-1) with
(r - i) mod (T'-1) for i = 1 .. T'/2 - 1 (the circle method); round T'-1 takes
the diagonal tiles.  Every unordered pair of tiles must come up exactly once,
and the pairs of a round must be disjoint, since each block merges into both
of its tiles' rows.  The keys must be symmetric bit for bit, because a pair's
key tile is read from both sides."""
from __future__ import annotations

import itertools

import numpy as np
import pytest


def schedule(tp: int):
    """Rounds of (a, b) pairs, as the kernel computes them from (round, blockIdx.y)."""
    rounds = []
    m = tp - 1
    for r in range(tp):
        if r == tp - 1:
            rounds.append([(y, y) for y in range(tp)])
            continue
        pairs = []
        for i in range(tp // 2):
            a = r if i == 0 else (r + i) % m
            b = m if i == 0 else (r - i + m) % m
            pairs.append((a, b))
        rounds.append(pairs)
    return rounds


def pair_tiles(maxleaf: int, tile: int) -> int:
    t = (maxleaf + tile - 1) // tile
    tp = (t + 1) // 2 * 2
    return tp if t >= 2 and tp <= 65535 else 0


@pytest.mark.parametrize("T", [2, 3, 4, 5, 8, 31, 32, 33, 100, 2048])
def test_every_pair_once_and_rounds_disjoint(T):
    tp = (T + 1) // 2 * 2
    seen = {}
    for r, pairs in enumerate(schedule(tp)):
        tiles = [t for ab in pairs for t in set(ab)]
        assert len(tiles) == len(set(tiles)), f"round {r}: a tile in two pairs"
        for a, b in pairs:
            if a >= T or b >= T:  # pairs with the padding tile are skipped
                continue
            key = (min(a, b), max(a, b))
            assert key not in seen, f"pair {key} in rounds {seen[key]} and {r}"
            seen[key] = r
    want = {(a, b) for a in range(T) for b in range(a, T)}
    assert set(seen) == want


@pytest.mark.parametrize("n_leaf,tile", [(64, 64), (65, 64), (128, 64), (1953, 64), (131072, 64), (1953, 32),
                                         (40, 32), (4_200_000, 64)])
def test_rounds_cover_each_leaf(n_leaf, tile):
    """Leaves of one tree differ by at most one point; the rounds follow the
    largest, and a smaller leaf skips the pairs past its own tiles."""
    tp = pair_tiles(n_leaf, tile)
    t = -(-n_leaf // tile)
    if t < 2 or t > 65534:
        assert tp == 0
        return
    assert tp >= t and tp % 2 == 0
    small = -(-(n_leaf - 1) // tile)
    covered = {(min(a, b), max(a, b)) for pairs in schedule(tp) for a, b in pairs if a < small and b < small}
    assert covered == {(a, b) for a in range(small) for b in range(a, small)}


def _key(q, c, metric):
    """The tile kernel's key: a sequential float32 partial per 256-dim group."""
    total = np.float32(0)
    part = np.float32(0)
    d = len(q)
    for dim in range(d):
        if metric == 2:
            part = np.float32(np.float64(q[dim]) * np.float64(c[dim]) + np.float64(part))  # fma, one rounding
        else:
            df = np.float32(q[dim] - c[dim])
            part = np.float32(np.float64(df) * np.float64(df) + np.float64(part)) if metric == 0 \
                else np.float32(part + abs(df))
        if (dim + 1) % 256 == 0 or dim == d - 1:
            total = np.float32(total + part)
            part = np.float32(0)
    return total


@pytest.mark.parametrize("metric", [0, 1, 2])
def test_keys_symmetric_bitwise(metric):
    rng = np.random.Generator(np.random.PCG64(11 + metric))
    for d in (3, 37, 300):
        x = rng.standard_normal((6, d)).astype(np.float32)
        x[0, ::3] = np.float32(-0.0)
        x[1] *= np.float32(1e-38)  # subnormal products and differences
        x[2, : d // 2] = x[3, : d // 2]  # exact cancellations
        for i, j in itertools.permutations(range(6), 2):
            a, b = _key(x[i], x[j], metric), _key(x[j], x[i], metric)
            assert a.view(np.uint32) == b.view(np.uint32), (d, i, j, a, b)

"""CPU restatement of the sparse-row leaf tiles' bookkeeping (csrc/leaf_knn.cu,
k_leaf_dim_mask / k_leaf_dim_list and the compact staging of k_leaf).

A leaf block's dim list keeps every dim that is non-zero in some row of the
block, in increasing order, with each 256-dim group padded by -1 to whole
32-dim chunks.  The tile kernel sums each group's terms sequentially into a
partial and adds the partial to the total at the group's end, so the keys
over the list must equal the keys over all dims bit for bit: the dims left
out add exact zeros to sums that are never negative."""
from __future__ import annotations

import numpy as np
import pytest


def mask_words(block: np.ndarray, dpad: int) -> np.ndarray:
    """k_leaf_dim_mask: bit (dim & 31) of word dim >> 5 set when a row is non-zero there."""
    W = dpad // 32 + 1
    nz = np.zeros(W * 32, dtype=bool)
    nz[:dpad] = (block != 0).any(axis=0)
    return np.packbits(nz.reshape(W, 32)[:, ::-1], axis=1, bitorder="big").view(">u4").ravel().astype(np.uint32)


def dim_list(mask: np.ndarray, d: int, dpad: int):
    """k_leaf_dim_list, lane by lane: lane l of group g holds dims 256 g + 8 l .. + 7."""
    W = len(mask)
    out = []
    for g in range((dpad + 255) // 256):
        counts, bits_of = [], []
        for lane in range(32):
            w = 8 * g + (lane >> 2)
            bits = (int(mask[w]) >> (8 * (lane & 3))) & 0xFF if w < W else 0
            bits_of.append(bits)
            counts.append(bin(bits).count("1"))
        excl = np.concatenate(([0], np.cumsum(counts)[:-1]))
        total = int(sum(counts))
        grp = [None] * total
        for lane in range(32):
            at = int(excl[lane])
            b = bits_of[lane]
            while b:
                low = (b & -b).bit_length() - 1
                grp[at] = 256 * g + 8 * lane + low
                at += 1
                b &= b - 1
        padded = (total + 31) & ~31
        out.extend(grp + [-1] * (padded - total))
    nch = len(out) // 32
    return np.array(out, dtype=np.int64), (nch if nch < (d + 31) // 32 else -1)


def key_dense(q, c, metric):
    """k_leaf over all dims: per 256-dim group a sequential float32 partial, added at the group end."""
    total = np.float32(0)
    part = np.float32(0)
    d = len(q)
    nch = (d + 31) // 32
    for ch in range(nch):
        for dim in range(32 * ch, 32 * ch + 32):
            qa = q[dim] if dim < d else np.float32(0)
            cb = c[dim] if dim < d else np.float32(0)
            df = np.float32(qa - cb)
            part = np.float32(part + (np.float32(df * df) if metric == 0 else abs(df)))
        if ((32 * ch + 32) & 255) == 0 or ch == nch - 1:
            total = np.float32(total + part)
            part = np.float32(0)
    return total


def key_listed(q, c, lst, nch, metric):
    """k_leaf over the listed dims: group ends where the next chunk's first dim lies in another group."""
    total = np.float32(0)
    part = np.float32(0)
    for ch in range(nch):
        for e in lst[32 * ch: 32 * ch + 32]:
            qa = q[e] if e >= 0 else np.float32(0)
            cb = c[e] if e >= 0 else np.float32(0)
            df = np.float32(qa - cb)
            part = np.float32(part + (np.float32(df * df) if metric == 0 else abs(df)))
        if ch == nch - 1 or (lst[32 * ch + 32] >> 8) != (lst[32 * ch] >> 8):
            total = np.float32(total + part)
            part = np.float32(0)
    return total


def _block(rng, rows, d, density, negzero=False):
    x = np.where(rng.random((rows, d)) < density, rng.standard_normal((rows, d)), 0.0).astype(np.float32)
    support = rng.random(d) < 0.5  # dims outside it are zero in every row
    x[:, ~support] = 0.0
    if negzero:
        x[:, ~support] = np.float32(-0.0)
    return x


@pytest.mark.parametrize("d", [5, 31, 64, 200, 256, 300, 784, 1030])
@pytest.mark.parametrize("density", [0.0, 0.05, 0.3, 1.0])
def test_list_holds_the_union_in_groups(d, density):
    rng = np.random.Generator(np.random.PCG64(d * 7 + int(density * 100)))
    dpad = (d + 3) // 4 * 4
    x = _block(rng, 40, d, density)
    xp = np.zeros((40, dpad), dtype=np.float32)
    xp[:, :d] = x
    lst, nch = dim_list(mask_words(xp, dpad), d, dpad)
    union = np.flatnonzero((x != 0).any(axis=0))
    np.testing.assert_array_equal(lst[lst >= 0], union)
    assert len(lst) % 32 == 0 and len(lst) <= 256 * ((dpad + 255) // 256)
    for ch in range(len(lst) // 32):
        chunk = lst[32 * ch: 32 * ch + 32]
        assert chunk[0] >= 0, "a chunk starts with a listed dim"
        valid = chunk[chunk >= 0]
        assert len(set(valid >> 8)) <= 1, "a chunk stays inside one 256-dim group"
        assert np.all(chunk[len(valid):] == -1), "padding only at a chunk's tail"
    if nch >= 0:
        assert nch < (d + 31) // 32


@pytest.mark.parametrize("metric", [0, 1])
@pytest.mark.parametrize("d,density,negzero", [(300, 0.2, False), (784, 0.2, False), (600, 0.6, True),
                                               (40, 0.3, False), (257, 0.02, True)])
def test_listed_keys_equal_dense_keys_bitwise(metric, d, density, negzero):
    rng = np.random.Generator(np.random.PCG64(d + metric))
    x = _block(rng, 12, d, density, negzero)
    dpad = (d + 3) // 4 * 4
    xp = np.zeros((12, dpad), dtype=np.float32)
    xp[:, :d] = x
    lst, nch = dim_list(mask_words(xp, dpad), d, dpad)
    if nch < 0:
        pytest.skip("the list saves no chunk: the kernel reads rows whole")
    for i in range(12):
        for j in range(12):
            a = key_dense(x[i], x[j], metric)
            b = key_listed(x[i], x[j], lst, nch, metric)
            assert a.view(np.uint32) == b.view(np.uint32), (i, j, a, b)


def test_planted_group_merge_is_caught():
    """With the groups' partials merged into one sequential sum (the group
    boundary ignored), the keys differ: the test sees the summation order."""
    rng = np.random.Generator(np.random.PCG64(3))
    d = 700
    x = _block(rng, 8, d, 0.4)
    dpad = 700
    lst, nch = dim_list(mask_words(x, dpad), d, dpad)

    def key_one_sum(q, c):
        s = np.float32(0)
        for e in lst[lst >= 0]:
            df = np.float32(q[e] - c[e])
            s = np.float32(s + abs(df))
        return s

    diff = sum(key_one_sum(x[i], x[j]).view(np.uint32) != key_dense(x[i], x[j], 1).view(np.uint32)
               for i in range(8) for j in range(8) if i != j)
    assert diff > 0

"""The first tree's bounding pass in the tensor-core leaf stage (k_leaf_tc,
approximate-cuda-knn_b200/csrc/leaf_umma.cu), restated on the CPU.

Pass 0 records, per query row, the smallest exact key of each 32-column slice of the block's
columns (slice s goes to group s mod 64; the row's own column is left out). The bound is the
kq-th smallest of the 64 group minima. Pass 1 filters against it, which is safe only if the bound
is never below the row's true kq-th smallest key. The kernel selects the kq-th smallest minimum
with a warp network: lanes' first halves sorted ascending, second halves descending, their
lane-wise minimum (the 32 smallest, a bitonic sequence), merged ascending.
"""
from __future__ import annotations

import numpy as np

GROUPS = 64


def group_minima(keys: np.ndarray, self_col: int) -> np.ndarray:
    """keys: one row's exact keys over the block's columns."""
    g = np.full(GROUPS, np.inf, dtype=np.float32)
    k = keys.copy()
    if 0 <= self_col < len(k):
        k[self_col] = np.inf
    for s0 in range(0, len(k), 32):
        grp = (s0 // 32) % GROUPS
        g[grp] = min(g[grp], k[s0:s0 + 32].min())
    return g


def bitonic_sort(v: np.ndarray, ascending: bool) -> np.ndarray:
    """The 32-lane bitonic network of the kernel (compare-exchange by lane xor m)."""
    v = v.copy()
    lanes = np.arange(32)
    size = 2
    while size <= 32:
        m = size // 2
        while m >= 1:
            o = v[lanes ^ m]
            keep_min = ((lanes & size) == 0) == ((lanes & m) == 0)
            if not ascending:
                keep_min = ~keep_min
            v = np.where(keep_min, np.minimum(v, o), np.maximum(v, o))
            m //= 2
        size *= 2
    return v


def network_kth(g: np.ndarray, kq: int) -> float:
    a = bitonic_sort(g[:32], True)
    b = bitonic_sort(g[32:], False)
    c = np.minimum(a, b)
    lanes = np.arange(32)
    m = 16
    while m >= 1:
        o = c[lanes ^ m]
        c = np.where((lanes & m) == 0, np.minimum(c, o), np.maximum(c, o))
        m //= 2
    return float(c[kq - 1])


def test_network_selects_the_kth_smallest_minimum():
    rng = np.random.Generator(np.random.PCG64(5))
    for _ in range(300):
        g = rng.standard_normal(GROUPS).astype(np.float32)
        g[rng.random(GROUPS) < 0.2] = np.inf  # empty groups
        g[rng.integers(0, GROUPS, 4)] = g[0]  # ties
        for kq in (1, 10, 20, 32):
            assert network_kth(g, kq) == float(np.sort(g)[kq - 1])


def test_bound_is_never_below_the_true_kth_key():
    rng = np.random.Generator(np.random.PCG64(9))
    for _ in range(200):
        nb = int(rng.integers(1024, 6000))      # blocks that get the bounding pass
        keys = rng.standard_normal(nb).astype(np.float32) ** 2
        if rng.random() < 0.3:
            keys = np.round(keys * 4).astype(np.float32)  # many ties
        self_col = int(rng.integers(0, nb))
        for kq in (10, 20, 32):
            bound = network_kth(group_minima(keys, self_col), kq)
            others = np.delete(keys, self_col)
            assert np.sort(others)[kq - 1] <= bound


def test_bound_is_useful():
    """On random keys the bound keeps a small fraction of a 2048-column block."""
    rng = np.random.Generator(np.random.PCG64(1))
    keys = rng.random(2048).astype(np.float32)
    bound = network_kth(group_minima(keys, 100), 32)
    assert (keys <= bound).sum() < 150

"""CPU restatement of k_leaf_bucket_sort (csrc/leaf_knn.cu): each leaf's
positions stably ordered by the rows' pattern bucket.

The kernel splits a leaf's n positions into 32 equal warp ranges, counts each
range per bucket, takes the exclusive prefix over (bucket, warp) and lets each
warp scatter its range in order, ranking equal buckets within 32 positions by
a match mask.  The result must be a permutation of the leaf's ids, sorted by
bucket and stable within a bucket."""
from __future__ import annotations

import numpy as np
import pytest

NB = 256


def bucket_sort(ids: np.ndarray, bucket: np.ndarray) -> np.ndarray:
    n = len(ids)
    per = (n + 31) // 32
    cnt = np.zeros((32, NB), dtype=np.int64)
    ranges = []
    for w in range(32):
        r0 = min(n, w * per)
        r1 = min(n, r0 + per)
        ranges.append((r0, r1))
        for r in range(r0, r1):
            cnt[w, bucket[ids[r]]] += 1
    tot = cnt.sum(axis=0)
    base = np.concatenate(([0], np.cumsum(tot)[:-1]))
    for b in range(NB):  # exclusive prefix over warps within each bucket
        run = base[b]
        for w in range(32):
            c = cnt[w, b]
            cnt[w, b] = run
            run += c
    out = np.full(n, -1, dtype=np.int64)
    for w, (r0, r1) in enumerate(ranges):
        for c0 in range(r0, r1, 32):
            lanes = [(lane, ids[c0 + lane]) for lane in range(32) if c0 + lane < r1]
            for lane, i in lanes:
                b = bucket[i]
                rank = sum(1 for l2, j in lanes if l2 < lane and bucket[j] == b)  # popc(peers & lt)
                out[cnt[w, b] + rank] = i
            for b in {bucket[i] for _, i in lanes}:
                cnt[w, b] += sum(1 for _, j in lanes if bucket[j] == b)
    return out


@pytest.mark.parametrize("n", [1, 31, 32, 33, 100, 1023, 1025, 4096, 5000])
@pytest.mark.parametrize("nbuckets", [1, 3, 10, 256])
def test_stable_sort_by_bucket(n, nbuckets):
    rng = np.random.Generator(np.random.PCG64(n * 7 + nbuckets))
    ids = rng.permutation(10 * n + 5)[:n]
    bucket = rng.integers(0, nbuckets, size=10 * n + 5)
    got = bucket_sort(ids, bucket)
    order = np.argsort(bucket[ids], kind="stable")
    np.testing.assert_array_equal(got, ids[order])


def test_planted_unstable_rank_is_caught():
    """Ranking by lane without the match mask (every lane's rank = its lane)
    overwrites entries: the restatement detects it."""
    rng = np.random.Generator(np.random.PCG64(1))
    n = 200
    ids = np.arange(n)
    bucket = rng.integers(0, 4, size=n)

    def broken(ids, bucket):
        out = np.full(n, -1)
        pos = {b: int(np.sum(bucket < b)) for b in range(4)}
        for r, i in enumerate(ids):
            out[min(n - 1, pos[bucket[i]] + (r % 32))] = i
        return out

    assert not np.array_equal(broken(ids, bucket), ids[np.argsort(bucket, kind="stable")])

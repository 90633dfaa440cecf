"""Generates the known-answer fixtures in this directory.

The reference ships no tests, golden vectors or fixtures (its only self-check
writes "Everything is OK." unconditionally, euclideandistancematrixgpu.cu:2967-2971),
so these cases are built from first principles.  Each case has n <= leaf, where
one leaf holds every point: the approximate graph must then equal the exact
k-NN graph, whose answer is written here analytically or by a float64 brute
force with ties broken by index.

    python tests/golden/make_golden.py      # rewrites kat_*.npz
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def exact_graph(x: np.ndarray, k: int, metric: int):
    """float64 brute force; ranks by (distance, index); self excluded."""
    x64 = x.astype(np.float64)
    n = x.shape[0]
    idx = np.empty((n, k), dtype=np.int32)
    dist = np.empty((n, k), dtype=np.float64)
    norms = np.sqrt((x64 * x64).sum(1))
    for i in range(n):
        if metric == 0:
            dv = np.sqrt(((x64 - x64[i]) ** 2).sum(1))
        elif metric == 1:
            dv = np.abs(x64 - x64[i]).sum(1)
        else:
            den = norms * norms[i]
            dot = x64 @ x64[i]
            dv = np.where(den == 0, 1.0, 1.0 - dot / np.where(den == 0, 1.0, den))
        order = sorted((dv[j], j) for j in range(n) if j != i)[:k]
        idx[i] = [j for _, j in order]
        dist[i] = [v for v, _ in order]
    return idx, dist


def case_line(n=64, k=4, shuffle=False, seed=3):
    """Points 0..n-1 on a line (d=1); integer distances are exact in float32."""
    x = np.arange(n, dtype=np.float32)[:, None]
    if shuffle:
        rng = np.random.Generator(np.random.PCG64(seed))
        x = x[rng.permutation(n)]
    idx, dist = exact_graph(x, k, 0)
    return dict(points=x, k=k, metric=0, idx=idx, dist=dist.astype(np.float32))


def case_duplicates(k=3, seed=5):
    """20 distinct points, each stored twice: each point's nearest is its twin."""
    rng = np.random.Generator(np.random.PCG64(seed))
    base = rng.integers(-8, 8, size=(20, 3)).astype(np.float32)
    x = np.concatenate([base, base])
    idx, dist = exact_graph(x, k, 0)
    return dict(points=x, k=k, metric=0, idx=idx, dist=dist.astype(np.float32))


def case_k_plus_one(k=4, seed=7):
    """n = k + 1: every point lists all the others."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.integers(-5, 6, size=(k + 1, 4)).astype(np.float32)
    idx, dist = exact_graph(x, k, 1)
    return dict(points=x, k=k, metric=1, idx=idx, dist=dist.astype(np.float32))


def case_taxicab_grid(k=6):
    """A 6x6 integer grid under L1 (many ties, broken by index)."""
    g = np.array([[i, j] for i in range(6) for j in range(6)], dtype=np.float32)
    idx, dist = exact_graph(g, k, 1)
    return dict(points=g, k=k, metric=1, idx=idx, dist=dist.astype(np.float32))


def case_cosine_axes(k=3):
    """Scaled unit axes and their negatives in 4-D, plus two zero rows
    (1 - cos of a zero row is 1 by definition)."""
    rows = []
    for a in range(4):
        for s in (1.0, 2.0, -1.0):
            v = np.zeros(4, dtype=np.float32)
            v[a] = s
            rows.append(v)
    rows.append(np.zeros(4, dtype=np.float32))
    rows.append(np.zeros(4, dtype=np.float32))
    x = np.stack(rows)
    idx, dist = exact_graph(x, k, 2)
    return dict(points=x, k=k, metric=2, idx=idx, dist=dist.astype(np.float32))


CASES = {
    "kat_line": lambda: case_line(),
    "kat_line_shuffled": lambda: case_line(shuffle=True),
    "kat_duplicates": case_duplicates,
    "kat_k_plus_one": case_k_plus_one,
    "kat_taxicab_grid": case_taxicab_grid,
    "kat_cosine_axes": case_cosine_axes,
}


def main() -> None:
    for name, fn in CASES.items():
        c = fn()
        np.savez(HERE / f"{name}.npz", **c)
        print(name, c["points"].shape, "k", c["k"], "metric", c["metric"])


if __name__ == "__main__":
    main()

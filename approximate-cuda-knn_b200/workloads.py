"""Seeded synthetic point sets with the shapes and value distributions of the
benchmark configurations (the reference names no public dataset; its input is
any CSV of N points in d dimensions, README.md:31-47).

All generators use numpy's PCG64 stream seeded by ``seed`` and return a
C-contiguous ``float32`` (or ``float16``) array of shape ``[n, d]``.
"""
from __future__ import annotations

import math

import numpy as np

_CHUNK = 1 << 18


def gaussian_mixture(n: int, d: int, clusters: int, seed: int, lo: float = -10.0,
                     hi: float = 10.0, sigma: float = 1.0) -> np.ndarray:
    """Equal-weight mixture of isotropic Gaussians, centres uniform in [lo, hi]^d."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.uniform(lo, hi, size=(clusters, d)).astype(np.float32)
    labels = rng.integers(0, clusters, size=n)
    out = np.empty((n, d), dtype=np.float32)
    for s in range(0, n, _CHUNK):
        e = min(n, s + _CHUNK)
        noise = rng.standard_normal((e - s, d), dtype=np.float32)
        out[s:e] = centres[labels[s:e]] + np.float32(sigma) * noise
    return out


def small_gaussians(seed: int = 0, n: int = 10_000, d: int = 16) -> np.ndarray:
    """10 isotropic Gaussians, centres U[-10,10]^16, sigma 1 (N=10,000, d=16)."""
    return gaussian_mixture(n, d, 10, seed)


def integer_mixture(seed: int = 0, n: int = 1_000_000, d: int = 128) -> np.ndarray:
    """256-cluster mixture, centres U[0,255]^d, per-dim sigma 20, rounded and
    clamped to the integers 0..255, stored as float32 (N=1,000,000, d=128)."""
    x = gaussian_mixture(n, d, 256, seed, lo=0.0, hi=255.0, sigma=20.0)
    np.rint(x, out=x)
    np.clip(x, 0.0, 255.0, out=x)
    return x


def sparse_prototypes(seed: int = 0, n: int = 1_000_000, d: int = 784,
                      prototypes: int = 10, density: float = 0.2) -> np.ndarray:
    """Rows in [0,1]: each row takes the support of one of 10 prototypes (a fixed
    random ~20% subset of the d dims) with values U(0,1] there and exact zeros
    elsewhere (N=1,000,000, d=784)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = int(round(density * d))
    supports = np.zeros((prototypes, d), dtype=bool)
    for p in range(prototypes):
        supports[p, rng.choice(d, size=m, replace=False)] = True
    labels = rng.integers(0, prototypes, size=n)
    out = np.zeros((n, d), dtype=np.float32)
    for s in range(0, n, _CHUNK):
        e = min(n, s + _CHUNK)
        u = 1.0 - rng.random((e - s, d), dtype=np.float32)  # (0, 1]
        out[s:e] = np.where(supports[labels[s:e]], u, np.float32(0.0))
    return out


def normalized_mixture(seed: int = 0, n: int = 10_000_000, d: int = 96,
                       clusters: int = 1000, sigma: float = 0.3,
                       dtype=np.float16) -> np.ndarray:
    """1000-cluster mixture, centres N(0, I_d), sigma 0.3, rows L2-normalised,
    stored as float16 (N=10,000,000, d=96)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.standard_normal((clusters, d), dtype=np.float32)
    labels = rng.integers(0, clusters, size=n)
    out = np.empty((n, d), dtype=dtype)
    for s in range(0, n, _CHUNK):
        e = min(n, s + _CHUNK)
        x = centres[labels[s:e]] + np.float32(sigma) * rng.standard_normal((e - s, d), dtype=np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        out[s:e] = x.astype(dtype)
    return out


def scaled_directions(seed: int = 0, n: int = 200_000, d: int = 64, clusters: int = 100,
                      sigma: float = 0.3, scale_lo: float = 0.1, scale_hi: float = 10.0) -> np.ndarray:
    """Rows of :func:`normalized_mixture` (float32) each multiplied by a
    log-uniform scale in [scale_lo, scale_hi].  COSINE neighbours are those of
    the unit rows, while raw-coordinate geometry is dominated by the scales."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.standard_normal((clusters, d), dtype=np.float32)
    labels = rng.integers(0, clusters, size=n)
    out = np.empty((n, d), dtype=np.float32)
    lo, hi = math.log(scale_lo), math.log(scale_hi)
    for s in range(0, n, _CHUNK):
        e = min(n, s + _CHUNK)
        x = centres[labels[s:e]] + np.float32(sigma) * rng.standard_normal((e - s, d), dtype=np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        x *= np.exp(rng.uniform(lo, hi, size=(e - s, 1))).astype(np.float32)
        out[s:e] = x
    return out


def batch_dataset(seed: int) -> np.ndarray:
    """One member of the 256-dataset batch: N log-uniform in [1e3, 2e5],
    d uniform over {32, 64, 128, 256}, 16-cluster mixture (centres U[-10,10]^d,
    sigma 1)."""
    rng = np.random.Generator(np.random.PCG64(10_000 + seed))
    n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5)))))
    d = int(rng.choice([32, 64, 128, 256]))
    return gaussian_mixture(n, d, 16, seed)


# name -> (generator, k, trees, leaf, propagations, metric)
CONFIGS = {
    "small_gaussians": dict(gen=small_gaussians, n=10_000, d=16, k=10, trees=10, leaf=32,
                            props=3, metric=0),
    "integer_mixture": dict(gen=integer_mixture, n=1_000_000, d=128, k=16, trees=16, leaf=64,
                            props=5, metric=0),
    "sparse_prototypes": dict(gen=sparse_prototypes, n=1_000_000, d=784, k=30, trees=8,
                              leaf=128, props=4, metric=1),
    "normalized_mixture": dict(gen=normalized_mixture, n=10_000_000, d=96, k=10, trees=12,
                               leaf=64, props=4, metric=2),
    "dataset_batch": dict(gen=batch_dataset, n=None, d=None, k=15, trees=8, leaf=48, props=3,
                          metric=0, count=256),
}

"""The tensor-core leaf stage's survivor filter admits every key the exact rule admits.

k_leaf_tc (approximate-cuda-knn_b200/csrc/leaf_umma.cu, the epilogue's row filter) checks each
(query, candidate) pair with three instructions:
    key' = fma(-2, dot, |y|^2)       (EUCLIDEAN)   or   0 - dot   (COSINE)
    pass = sign(thr - key') == 0
against a per-row threshold, widened by 2^-21 (|tk| + |x|^2 + max|y|^2) (EUCLIDEAN) or
2^-21 (|tk| + 2) (COSINE), where tk is the row's list tail. The merge then applies the exact
rule: key = fma(-2, dot, |x|^2 + |y|^2) (or 1 - dot), admitted when key <= tk. Parity holds only
if every pair the exact rule admits also passes the filter. This test restates both computations
in float32, with the kernel's operation order (the library is built without FMA contraction), and
checks that implication on random and adversarial inputs: tails equal to the key or one ulp away,
large norms and near-cancelling products.
"""
from __future__ import annotations

import numpy as np

F = np.float32
SLACK = F(2.0 ** -21)
MAXF = np.finfo(np.float32).max


def fma32(a, b, c):
    # a*b is exact in float64 for float32 inputs; one rounding to float64 and one to float32 can
    # differ from a single rounding only at float32 ties, which random inputs do not hit
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def euclid_exact(dot, xn, yn):
    return fma32(F(-2.0) * np.ones_like(dot), dot, (xn + yn).astype(np.float32))


def euclid_filter(dot, xn, yn, tk, cmax):
    kp = fma32(F(-2.0) * np.ones_like(dot), dot, yn)
    t1 = (tk - xn).astype(np.float32)
    t3 = ((np.abs(tk) + xn).astype(np.float32) + cmax).astype(np.float32)
    thr = np.minimum((t1 + (SLACK * t3).astype(np.float32)).astype(np.float32), F(MAXF))
    diff = (thr - kp).astype(np.float32)
    return ~np.signbit(diff)


def cosine_exact(dot):
    return (F(1.0) - dot).astype(np.float32)


def cosine_filter(dot, tk):
    kp = (F(0.0) - dot).astype(np.float32)
    t1 = (tk - F(1.0)).astype(np.float32)
    t3 = (np.abs(tk) + F(2.0)).astype(np.float32)
    thr = np.minimum((t1 + (SLACK * t3).astype(np.float32)).astype(np.float32), F(MAXF))
    diff = (thr - kp).astype(np.float32)
    return ~np.signbit(diff)


def _tails_around(key):
    """The key itself and its float32 neighbours: the boundary of the exact rule."""
    up = np.nextafter(key, np.float32(np.inf))
    dn = np.nextafter(key, np.float32(-np.inf))
    return [key, up, dn, np.nextafter(up, np.float32(np.inf))]


def _euclid_cases(rng, m, scale, cancel):
    d = 128
    x = (rng.standard_normal((m, d)) * scale).astype(np.float32)
    if cancel:  # candidates close to the query: tiny keys from large norms
        y = (x + rng.standard_normal((m, d)).astype(np.float32) * F(scale * 1e-3)).astype(np.float32)
    else:
        y = (rng.standard_normal((m, d)) * scale).astype(np.float32)
    xn = np.einsum("ij,ij->i", x, x, dtype=np.float32).astype(np.float32)
    yn = np.einsum("ij,ij->i", y, y, dtype=np.float32).astype(np.float32)
    dot = np.einsum("ij,ij->i", x, y, dtype=np.float32).astype(np.float32)
    return dot, xn, yn


def test_euclidean_filter_keeps_every_admitted_key():
    rng = np.random.Generator(np.random.PCG64(7))
    for scale in (1e-3, 1.0, 255.0, 1e4):
        for cancel in (False, True):
            dot, xn, yn = _euclid_cases(rng, 20000, scale, cancel)
            cmax = F(yn.max())
            key = euclid_exact(dot, xn, yn)
            for tk in _tails_around(key) + [key * F(1.5) + F(1.0), key * F(0.5)]:
                tk = tk.astype(np.float32)
                admitted = key <= tk
                passed = euclid_filter(dot, xn, yn, tk, cmax)
                bad = admitted & ~passed
                assert not bad.any(), (scale, cancel, int(bad.sum()))


def test_cosine_filter_keeps_every_admitted_key():
    rng = np.random.Generator(np.random.PCG64(11))
    d = 96
    for spread in (1.0, 1e-3):
        x = rng.standard_normal((20000, d)).astype(np.float32)
        y = (x + rng.standard_normal((20000, d)).astype(np.float32) * F(spread)).astype(np.float32)
        x /= np.linalg.norm(x, axis=1, keepdims=True).astype(np.float32)
        y /= np.linalg.norm(y, axis=1, keepdims=True).astype(np.float32)
        dot = np.einsum("ij,ij->i", x, y, dtype=np.float32).astype(np.float32)
        key = cosine_exact(dot)
        for tk in _tails_around(key) + [key + F(0.25), key * F(0.5)]:
            tk = tk.astype(np.float32)
            admitted = key <= tk
            passed = cosine_filter(dot, tk)
            bad = admitted & ~passed
            assert not bad.any(), (spread, int(bad.sum()))


def test_filter_is_tight():
    """The widening is small: keys well above the tail are rejected (the filter filters)."""
    rng = np.random.Generator(np.random.PCG64(3))
    dot, xn, yn = _euclid_cases(rng, 20000, 1.0, False)
    key = euclid_exact(dot, xn, yn)
    tk = (key * F(0.99)).astype(np.float32)
    passed = euclid_filter(dot, xn, yn, tk, F(yn.max()))
    assert passed.mean() < 0.01

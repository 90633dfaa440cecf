"""Shared fixtures: the package (loaded from its directory), the CPU oracle
(test infrastructure under oracle/), and the gpu marker."""
from __future__ import annotations

import ctypes
import importlib.util
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "approximate-cuda-knn_b200"
ORACLE_DIR = ROOT / "oracle"
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    """Import approximate-cuda-knn_b200/ (not a valid module name) as `acknn`."""
    if "acknn" in sys.modules:
        return sys.modules["acknn"]
    spec = importlib.util.spec_from_file_location(
        "acknn", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["acknn"] = mod
    spec.loader.exec_module(mod)
    return mod


class Oracle:
    """ctypes binding of oracle/liboracle.so (the CPU restatement)."""

    def __init__(self, path: Path):
        P, I32, I64, U64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64
        lib = ctypes.CDLL(str(path))
        sig = {
            "oracle_tree_depth": (ctypes.c_int, [I64, I32]),
            "oracle_project": (ctypes.c_float, [P, P, I32]),
            "oracle_pair_key": (ctypes.c_float, [P, P, I32, I32]),
            "oracle_build_trees": (ctypes.c_int, [P, I64, I32, I32, I32, U64, P, I32]),
            "oracle_build_trees_ex": (ctypes.c_int, [P, I64, I32, I32, I32, U64, I32, I32, P, I32]),
            "oracle_knn_build_faithful": (ctypes.c_int, [P, I64, I32, I32, I32, I32, I32, I32, U64, P, P, I32]),
            "oracle_leaf_stage": (ctypes.c_int, [P, I64, I32, I32, I32, I32, I32, P, P, P, I32]),
            "oracle_propagate": (ctypes.c_int, [P, I64, I32, I32, I32, P, P, P, P, I32]),
            "oracle_finalize": (None, [I64, I32, P, P]),
            "oracle_knn_build": (ctypes.c_int, [P, I64, I32, I32, I32, I32, I32, I32, U64, P, P, I32]),
            "oracle_exact_knn": (ctypes.c_int, [P, I64, I32, I32, I32, P, I64, P, P, I32]),
            "oracle_pair_dist_fp64": (ctypes.c_int, [P, I64, I32, I32, P, P, I64, P]),
            "oracle_mlp_forward": (ctypes.c_int, [P, I32, P, I64, P]),
            "oracle_mlp_loss_grad": (ctypes.c_int, [P, I32, P, I32, ctypes.c_double, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    @staticmethod
    def _x(points):
        return np.ascontiguousarray(points, dtype=np.float32)

    def build_trees(self, points, trees, leaf, seed=0, threads=0):
        x = self._x(points)
        n, d = x.shape
        perm = np.empty((trees, n), dtype=np.int32)
        assert self.lib.oracle_build_trees(x.ctypes.data, n, d, trees, leaf, seed,
                                           perm.ctypes.data, threads) == 0
        return perm

    def build_trees_ex(self, points, trees, leaf, seed, tree_offset, tree_stride, threads=0):
        x = self._x(points)
        n, d = x.shape
        perm = np.empty((trees, n), dtype=np.int32)
        assert self.lib.oracle_build_trees_ex(x.ctypes.data, n, d, trees, leaf, seed, tree_offset,
                                              tree_stride, perm.ctypes.data, threads) == 0
        return perm

    def leaf_stage(self, points, k, perm, leaf, metric=0, threads=0):
        x = self._x(points)
        n, d = x.shape
        perm = np.ascontiguousarray(perm, dtype=np.int32)
        idx = np.empty((n, k), dtype=np.int32)
        key = np.empty((n, k), dtype=np.float32)
        assert self.lib.oracle_leaf_stage(x.ctypes.data, n, d, k, perm.shape[0], leaf, metric,
                                          perm.ctypes.data, idx.ctypes.data, key.ctypes.data,
                                          threads) == 0
        return idx, key

    def propagate(self, points, idx, key, metric=0, threads=0):
        x = self._x(points)
        n, d = x.shape
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        key = np.ascontiguousarray(key, dtype=np.float32)
        oi, ok = np.empty_like(idx), np.empty_like(key)
        assert self.lib.oracle_propagate(x.ctypes.data, n, d, idx.shape[1], metric,
                                         idx.ctypes.data, key.ctypes.data, oi.ctypes.data,
                                         ok.ctypes.data, threads) == 0
        return oi, ok

    def knn_build(self, points, k, trees, leaf, props, metric=0, seed=0, threads=0):
        x = self._x(points)
        n, d = x.shape
        idx = np.empty((n, k), dtype=np.int32)
        dist = np.empty((n, k), dtype=np.float32)
        rc = self.lib.oracle_knn_build(x.ctypes.data, n, d, k, trees, leaf, props, metric, seed,
                                       idx.ctypes.data, dist.ctypes.data, threads)
        if rc:
            raise ValueError(f"oracle_knn_build rc={rc}")
        return idx, dist

    def knn_build_faithful(self, points, k, trees, leaf, props, metric=0, seed=0, threads=0):
        """The build with reference-rule trees (sign split through the origin)."""
        x = self._x(points)
        n, d = x.shape
        idx = np.empty((n, k), dtype=np.int32)
        dist = np.empty((n, k), dtype=np.float32)
        rc = self.lib.oracle_knn_build_faithful(x.ctypes.data, n, d, k, trees, leaf, props, metric, seed,
                                                idx.ctypes.data, dist.ctypes.data, threads)
        if rc:
            raise ValueError(f"oracle_knn_build_faithful rc={rc}")
        return idx, dist

    def exact(self, points, k, queries=None, metric=0, threads=0):
        x = self._x(points)
        n, d = x.shape
        q = np.arange(n, dtype=np.int64) if queries is None else np.ascontiguousarray(queries, dtype=np.int64)
        idx = np.empty((q.shape[0], k), dtype=np.int32)
        dist = np.empty((q.shape[0], k), dtype=np.float64)
        assert self.lib.oracle_exact_knn(x.ctypes.data, n, d, k, metric, q.ctypes.data,
                                         q.shape[0], idx.ctypes.data, dist.ctypes.data,
                                         threads) == 0
        return idx, dist

    def pair_dist(self, points, qi, cj, metric=0):
        x = self._x(points)
        n, d = x.shape
        qi = np.ascontiguousarray(qi, dtype=np.int64)
        cj = np.ascontiguousarray(cj, dtype=np.int32)
        out = np.empty(qi.shape[0], dtype=np.float64)
        assert self.lib.oracle_pair_dist_fp64(x.ctypes.data, n, d, metric, qi.ctypes.data,
                                              cj.ctypes.data, qi.shape[0], out.ctypes.data) == 0
        return out

    def pair_key(self, a, b, metric=0):
        a = self._x(a)
        b = self._x(b)
        return self.lib.oracle_pair_key(a.ctypes.data, b.ctypes.data, a.shape[0], metric)

    def project(self, x, v):
        x = self._x(x)
        v = self._x(v)
        return self.lib.oracle_project(x.ctypes.data, v.ctypes.data, x.shape[0])

    def finalize(self, key, metric=0):
        """Keys -> distances (sqrt for EUCLIDEAN), float32."""
        k = np.ascontiguousarray(key, dtype=np.float32)
        out = np.empty_like(k)
        self.lib.oracle_finalize(k.size, metric, k.ctypes.data, out.ctypes.data)
        return out

    def mlp_forward(self, params, rows):
        """FP64 f(rows) of the learned split network: [m, 64]."""
        p = self._x(params)
        r = self._x(rows)
        z = np.empty((r.shape[0], 64), dtype=np.float64)
        assert self.lib.oracle_mlp_forward(p.ctypes.data, r.shape[1], r.ctypes.data, r.shape[0],
                                           z.ctypes.data) == 0
        return z

    def mlp_loss_grad(self, params, rows, margin=1.0):
        """FP64 (loss, grad, per-triplet hinge argument) of the triplet loss."""
        p = self._x(params)
        r = self._x(rows)
        b = r.shape[0] // 3
        grad = np.empty(p.shape[0], dtype=np.float64)
        loss = np.zeros(1, dtype=np.float64)
        hinge = np.empty(b, dtype=np.float64)
        assert self.lib.oracle_mlp_loss_grad(p.ctypes.data, r.shape[1], r.ctypes.data, b, margin,
                                             grad.ctypes.data, loss.ctypes.data,
                                             hinge.ctypes.data) == 0
        return float(loss[0]), grad, hinge


@pytest.fixture(scope="session")
def oracle() -> Oracle:
    lib = ORACLE_DIR / "liboracle.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(ORACLE_DIR), "liboracle.so"], check=True,
                       capture_output=True)
    return Oracle(lib)


@pytest.fixture(scope="session")
def acknn():
    return load_package()


def recall_at_k(approx_idx: np.ndarray, exact_idx: np.ndarray) -> float:
    """Mean |approx_i n exact_i| / k."""
    k = exact_idx.shape[1]
    hits = 0
    for a, e in zip(approx_idx, exact_idx):
        hits += len(np.intersect1d(a, e, assume_unique=False))
    return hits / (k * exact_idx.shape[0])

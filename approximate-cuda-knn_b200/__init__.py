"""B200 approximate k-NN graph builder -- Python host side over libacknn.so.

The compute path is the C ABI in ``include/knn.h`` (CUDA kernels for sm_100a).
This module loads it with ctypes and offers

* functional calls: :func:`knn_build`, :func:`build_trees`, :func:`leaf_stage`,
  :func:`propagate_step`, :func:`exact_fp64`, :func:`normalize_reference`;
* :class:`EuclideanDistanceMatrixGPU`, a mirror of the reference's class of the
  same name (euclideandistancematrixgpu.h:50-63): setDataFile, setResultsFile,
  initialize, calculate, saveResultToResultFile, deinitialize, each returning
  ``True`` on error as the reference does.

There is no CPU fallback: if the shared library is missing, or no CUDA device
is usable, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from . import formats  # noqa: F401  (CSV / binary result formats)
from . import workloads  # noqa: F401  (seeded synthetic point sets)
from . import sharded  # noqa: F401  (multi-GPU builds over torch.distributed)

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libacknn.so"

METRIC_EUCLIDEAN = 0
METRIC_TAXICAB = 1
METRIC_COSINE = 2
METRICS = {"EUCLIDEAN": 0, "TAXICAB": 1, "COSINE": 2}

F32, F16, BF16 = 0, 1, 2
PREC_FP32, PREC_BF16_RERANK, PREC_F16_RERANK = 0, 1, 2
MAX_K = 128
MAX_PROPS = 64

STATUS = {
    0: "ok", -1: "invalid argument", -2: "n must exceed k", -3: "out of memory",
    -4: "CUDA error", -5: "device wait timed out", -6: "unsupported request",
    -7: "no CUDA device",
}


class KnnError(RuntimeError):
    """A negative status from the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, 'unknown status')} ({status}): {message}")
        self.status = status


class KnnOptions(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("points_on_device", ctypes.c_int32),
        ("outputs_on_device", ctypes.c_int32),
        ("dtype", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("learned_splits", ctypes.c_int32),
        ("timing", ctypes.c_int32),
        ("ld", ctypes.c_int64),
        ("stream", ctypes.c_void_p),
        ("mlp_sample", ctypes.c_int32),
        ("mlp_steps", ctypes.c_int32),
        ("autotune", ctypes.c_int32),
        ("leaf_tile", ctypes.c_int32),
        ("prop_warps", ctypes.c_int32),
        ("tree_offset", ctypes.c_int32),
        ("tree_stride", ctypes.c_int32),
        ("raw_keys", ctypes.c_int32),
        ("split_rule", ctypes.c_int32),
        ("tc_group", ctypes.c_int32),
        ("sparse_dims", ctypes.c_int32),
        ("tile_pairs", ctypes.c_int32),
    ]


class KnnStats(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("depth", ctypes.c_int32),
        ("ms_total", ctypes.c_float),
        ("ms_upload", ctypes.c_float),
        ("ms_trees", ctypes.c_float),
        ("ms_leaf", ctypes.c_float),
        ("ms_propagate", ctypes.c_float),
        ("ms_download", ctypes.c_float),
        ("launches", ctypes.c_int32),
        ("props_run", ctypes.c_int32),
        ("leaf_pairs", ctypes.c_int64),
        ("prop_candidates", ctypes.c_int64 * MAX_PROPS),
        ("ms_prop_iter", ctypes.c_float * MAX_PROPS),
        ("ms_learn", ctypes.c_float),
        ("leaf_tile", ctypes.c_int32),
        ("prop_warps", ctypes.c_int32),
        ("ms_leaf_tiles", ctypes.c_float),
        ("leaf_path", ctypes.c_int32),
        ("leaf_fallback", ctypes.c_int32),
        ("tc_group", ctypes.c_int32),
        ("sparse_dims", ctypes.c_int32),
        ("tile_pairs", ctypes.c_int32),
        ("reserved32", ctypes.c_int32),
        ("reserved", ctypes.c_int64 * 3),
    ]

    def as_dict(self) -> dict:
        n = self.props_run
        return {
            "depth": self.depth, "ms_total": self.ms_total, "ms_upload": self.ms_upload,
            "ms_learn": self.ms_learn, "ms_trees": self.ms_trees, "ms_leaf": self.ms_leaf,
            "ms_propagate": self.ms_propagate, "ms_download": self.ms_download,
            "ms_leaf_tiles": self.ms_leaf_tiles,
            "launches": self.launches, "leaf_pairs": self.leaf_pairs,
            "leaf_tile": self.leaf_tile, "prop_warps": self.prop_warps,
            "leaf_path": self.leaf_path, "leaf_fallback": self.leaf_fallback, "tc_group": self.tc_group,
            "sparse_dims": self.sparse_dims, "tile_pairs": self.tile_pairs,
            "prop_candidates": [self.prop_candidates[i] for i in range(n)],
        }


class KnnDataset(ctypes.Structure):
    _fields_ = [
        ("points", ctypes.c_void_p),
        ("n", ctypes.c_int64),
        ("d", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("out_idx", ctypes.c_void_p),
        ("out_dist", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_I32, _I64, _U64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64

# name -> (restype, argtypes); every symbol declared in include/knn.h
EXPORTS = {
    "knn_default_options": (None, [_P]),
    "knn_version": (ctypes.c_int, []),
    "knn_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "knn_last_error": (ctypes.c_char_p, []),
    "knn_device_capability": (ctypes.c_int, [_I32, _P, _P]),
    "knn_context_create": (_P, [_I32]),
    "knn_context_destroy": (None, [_P]),
    "knn_context_scratch_bytes": (_I64, [_P]),
    "knn_context_status": (ctypes.c_int, [_P, _P]),
    "knn_test_fail_next_tile_wait": (ctypes.c_int, [_P]),
    "knn_build": (ctypes.c_int, [_P, _I64, _I32, _I32, _I32, _I32, _I32, _I32, _U64, _P, _P]),
    "knn_build_ex": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _I32, _I32, _I32, _U64, _P,
                                    _P, _P, _P]),
    "knn_build_trees": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _U64, _P]),
    "knn_leaf_stage": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _I32, _I32, _P, _P, _P]),
    "knn_propagate_step": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _P, _P, _P, _P]),
    "knn_exact_fp64": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _P, _I64, _P, _P, _P]),
    "knn_normalize_reference": (ctypes.c_int, [_P, _I64, _I32]),
    "knn_exact_fp64_noalloc": (ctypes.c_int, [_P, _I64, _I32, _I32, _I32, _P, _I64, _P, _P, _P]),
    "knn_build_batch": (ctypes.c_int, [_P, _P, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "knn_merge_lists": (ctypes.c_int, [_P, _P, _P, _I32, _I64, _I32, _I32, _I32, _P, _P, _P]),
    "knn_propagate_range": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _I64, _I64, _P, _P, _P, _P, _P,
                                           _P, _P]),
    "knn_mlp_param_count": (_I64, [_I32]),
    "knn_mlp_loss_grad": (ctypes.c_int, [_P, _I32, _P, _I32, ctypes.c_float, _P, _P]),
    "knn_mlp_train": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _I32, _U64, _P, _P, _P, _P, _P]),
    "knn_mlp_embed": (ctypes.c_int, [_P, _P, _I64, _I32, _I32, _P, _P, _P, _P, _P]),
}

_lib_handle = None


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load libacknn.so (built by ``make -C approximate-cuda-knn_b200``)."""
    global _lib_handle
    if _lib_handle is not None and path is None:
        return _lib_handle
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `make -C {PKG_DIR}` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib_handle = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        msg = load_library().knn_last_error()
        raise KnnError(rc, msg.decode() if msg else "")


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _points(points) -> np.ndarray:
    x = np.ascontiguousarray(points)
    if x.ndim != 2:
        raise ValueError("points must be a 2-D array [n, d]")
    if x.dtype not in (np.float32, np.float16):
        x = x.astype(np.float32)
    return x


def default_options(**kw) -> KnnOptions:
    o = KnnOptions()
    load_library().knn_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def knn_build(points, k: int, trees: int, leaf: int, props: int, metric: int = 0,
              seed: int = 0, precision: int = PREC_FP32, learned: bool = False,
              stats: bool = False, context=None, mlp_sample: int = 0, mlp_steps: int = 0,
              autotune: bool = False, leaf_tile: int = 0, prop_warps: int = 0,
              split_rule: int = 0, tc_group: int = 0, sparse_dims: int = 0, tile_pairs: int = 0):
    """k-NN graph of ``points`` ([n, d] float32/float16, host memory).

    ``sparse_dims`` (FP32 leaf tiles, EUCLIDEAN/TAXICAB): 1 each leaf block
    reads only its rows' non-zero dims, -1 never, 0 when leaves hold >= 1024
    points; the graph is the same either way.  ``tile_pairs`` -1 computes
    every FP32 leaf key from both of its points instead of once (same graph).
    ``learned`` builds the trees on the learned split network's embedding
    (trained on a sample of ``mlp_sample`` points for ``mlp_steps`` steps; 0
    picks the library default).  Returns ``(idx int32 [n, k], dist float32
    [n, k])`` sorted by (distance, index), plus a stats dict when ``stats``."""
    x = _points(points)
    n, d = x.shape
    lib = load_library()
    idx = np.empty((n, k), dtype=np.int32)
    dist = np.empty((n, k), dtype=np.float32)
    opt = default_options(dtype=F16 if x.dtype == np.float16 else F32, precision=precision,
                          learned_splits=int(bool(learned)), mlp_sample=mlp_sample,
                          mlp_steps=mlp_steps, autotune=int(bool(autotune)), leaf_tile=leaf_tile,
                          prop_warps=prop_warps, split_rule=split_rule, tc_group=tc_group,
                          sparse_dims=sparse_dims, tile_pairs=tile_pairs)
    st = KnnStats()
    st.struct_size = ctypes.sizeof(KnnStats)
    rc = lib.knn_build_ex(context, _ptr(x), n, d, k, trees, leaf, props, metric, seed,
                          _ptr(idx), _ptr(dist), ctypes.byref(opt),
                          ctypes.byref(st) if stats else None)
    _check(rc)
    return (idx, dist, st.as_dict()) if stats else (idx, dist)


def knn_build_batch(datasets, k: int, trees: int, leaf: int, props: int, metric: int = 0,
                    seeds=None, precision: int = PREC_FP32, stats: bool = False, context=None,
                    autotune: bool = False, leaf_tile: int = 0, prop_warps: int = 0, tc_group: int = 0,
                    sparse_dims: int = 0, tile_pairs: int = 0):
    """k-NN graphs of many independent point sets in one call.

    ``datasets``: sequence of [n_i, d_i] arrays (all float32 or all float16);
    ``seeds``: one seed per set (default 0).  Returns a list of ``(idx, dist)``
    per set (ids local to the set), plus a stats dict when ``stats``."""
    xs = [_points(x) for x in datasets]
    if len({x.dtype for x in xs}) > 1:
        raise ValueError("all datasets must share one element type")
    seeds = [0] * len(xs) if seeds is None else list(seeds)
    outs = []
    arr = (KnnDataset * max(1, len(xs)))()
    for i, x in enumerate(xs):
        n, d = x.shape
        idx = np.empty((n, k), dtype=np.int32)
        dist = np.empty((n, k), dtype=np.float32)
        outs.append((idx, dist))
        arr[i].points = _ptr(x)
        arr[i].n = n
        arr[i].d = d
        arr[i].seed = int(seeds[i])
        arr[i].out_idx = _ptr(idx)
        arr[i].out_dist = _ptr(dist)
    f16 = bool(xs) and xs[0].dtype == np.float16
    opt = default_options(dtype=F16 if f16 else F32, precision=precision,
                          autotune=int(bool(autotune)), leaf_tile=leaf_tile, prop_warps=prop_warps,
                          tc_group=tc_group, sparse_dims=sparse_dims, tile_pairs=tile_pairs)
    st = KnnStats()
    st.struct_size = ctypes.sizeof(KnnStats)
    _check(load_library().knn_build_batch(context, arr, len(xs), k, trees, leaf, props, metric,
                                          ctypes.byref(opt), ctypes.byref(st) if stats else None))
    return (outs, st.as_dict()) if stats else outs


def build_trees(points, trees: int, leaf: int, seed: int = 0) -> np.ndarray:
    """Leaf order of every tree, int32 [trees, n]."""
    x = _points(points).astype(np.float32, copy=False)
    n, d = x.shape
    perm = np.empty((trees, n), dtype=np.int32)
    _check(load_library().knn_build_trees(None, _ptr(x), n, d, trees, leaf, seed, _ptr(perm)))
    return perm


def leaf_stage(points, k: int, perm: np.ndarray, leaf: int, metric: int = 0):
    """Initial k-NN from given leaf orders: (idx [n, k], key [n, k])."""
    x = _points(points).astype(np.float32, copy=False)
    n, d = x.shape
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    idx = np.empty((n, k), dtype=np.int32)
    key = np.empty((n, k), dtype=np.float32)
    _check(load_library().knn_leaf_stage(None, _ptr(x), n, d, k, perm.shape[0], leaf, metric,
                                         _ptr(perm), _ptr(idx), _ptr(key)))
    return idx, key


def propagate_step(points, idx: np.ndarray, key: np.ndarray, metric: int = 0):
    """One Jacobi propagation step on (idx, key) lists."""
    x = _points(points).astype(np.float32, copy=False)
    n, d = x.shape
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    key = np.ascontiguousarray(key, dtype=np.float32)
    k = idx.shape[1]
    oi = np.empty_like(idx)
    ok = np.empty_like(key)
    _check(load_library().knn_propagate_step(None, _ptr(x), n, d, k, metric, _ptr(idx), _ptr(key),
                                             _ptr(oi), _ptr(ok)))
    return oi, ok


def exact_fp64(points, k: int, queries, metric: int = 0):
    """Exact FP64 k-NN of the given query rows on the GPU: (idx [nq,k], dist float64)."""
    x = _points(points).astype(np.float32, copy=False)
    n, d = x.shape
    q = np.ascontiguousarray(queries, dtype=np.int64)
    idx = np.empty((q.shape[0], k), dtype=np.int32)
    dist = np.empty((q.shape[0], k), dtype=np.float64)
    _check(load_library().knn_exact_fp64(None, _ptr(x), n, d, k, metric, _ptr(q), q.shape[0],
                                         _ptr(idx), _ptr(dist), None))
    return idx, dist


MLP_HIDDEN, MLP_EMBED = 256, 64


def mlp_param_count(d: int) -> int:
    """Length of the learned split network's parameter vector (W1, b1, W2, b2)."""
    return int(load_library().knn_mlp_param_count(d))


def mlp_loss_grad(params: np.ndarray, rows: np.ndarray, margin: float = 1.0):
    """Mean triplet loss and gradient on the GPU for standardised rows
    [3B, d] (anchors, positives, negatives): (loss, grad float32)."""
    rows = np.ascontiguousarray(rows, dtype=np.float32)
    params = np.ascontiguousarray(params, dtype=np.float32)
    d = rows.shape[1]
    if rows.shape[0] % 3:
        raise ValueError("rows must hold 3*batch rows")
    grad = np.empty(mlp_param_count(d), dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    _check(load_library().knn_mlp_loss_grad(_ptr(params), d, _ptr(rows), rows.shape[0] // 3,
                                            ctypes.c_float(margin), _ptr(grad), _ptr(loss)))
    return float(loss[0]), grad


def mlp_train(points, k: int, metric: int = 0, seed: int = 0, mlp_sample: int = 0,
              mlp_steps: int = 0):
    """Train the split network as a learned build would:
    (params, mean, inv_std, loss_curve)."""
    x = _points(points)
    n, d = x.shape
    steps = mlp_steps if mlp_steps > 0 else 300
    params = np.empty(mlp_param_count(d), dtype=np.float32)
    mean = np.empty(d, dtype=np.float32)
    inv_std = np.empty(d, dtype=np.float32)
    curve = np.empty(steps, dtype=np.float32)
    opt = default_options(dtype=F16 if x.dtype == np.float16 else F32, mlp_sample=mlp_sample,
                          mlp_steps=mlp_steps)
    _check(load_library().knn_mlp_train(None, _ptr(x), n, d, k, metric, seed, ctypes.byref(opt),
                                        _ptr(params), _ptr(mean), _ptr(inv_std), _ptr(curve)))
    return params, mean, inv_std, curve


def mlp_embed(points, params, mean, inv_std, metric: int = 0) -> np.ndarray:
    """f(points) on the GPU, float32 [n, 64] (COSINE feeds the unit rows)."""
    x = _points(points)
    n, d = x.shape
    params = np.ascontiguousarray(params, dtype=np.float32)
    mean = np.ascontiguousarray(mean, dtype=np.float32)
    inv_std = np.ascontiguousarray(inv_std, dtype=np.float32)
    out = np.empty((n, MLP_EMBED), dtype=np.float32)
    opt = default_options(dtype=F16 if x.dtype == np.float16 else F32)
    _check(load_library().knn_mlp_embed(None, _ptr(x), n, d, metric, _ptr(params), _ptr(mean),
                                        _ptr(inv_std), ctypes.byref(opt), _ptr(out)))
    return out


def normalize_reference(points: np.ndarray) -> np.ndarray:
    """The reference's normalisation (normalizeDataStep1/2) on a copy."""
    x = np.ascontiguousarray(points, dtype=np.float32).copy()
    _check(load_library().knn_normalize_reference(_ptr(x), x.shape[0], x.shape[1]))
    return x


class Context:
    """Owns a knn_context (device scratch reused across calls)."""

    def __init__(self, device: int = -1):
        self._lib = load_library()
        self.handle = self._lib.knn_context_create(device)
        if not self.handle:
            raise KnnError(-4, self._lib.knn_last_error().decode())

    @property
    def scratch_bytes(self) -> int:
        return int(self._lib.knn_context_scratch_bytes(self.handle))

    def close(self) -> None:
        if self.handle:
            self._lib.knn_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EuclideanDistanceMatrixGPU:
    """Mirror of the reference's class (euclideandistancematrixgpu.h:50-63).

    Methods return ``True`` on error, like the reference; the reason is kept in
    ``last_error``.  Differences: no cudaDeviceReset, no stdout logging, and the
    points are normalised by :func:`normalize_reference` inside ``calculate``
    exactly where the reference runs normalizeDataStep1/2 (.cu:2869-2875)."""

    def __init__(self, debugMode: bool = False):
        self.debugMode = bool(debugMode)
        self.inputFile = ""
        self.outputFile = ""
        self.last_error = ""
        self.elapsed_ms = 0.0
        self._data = None
        self._idx = None
        self._dist = None

    def setDataFile(self, nameOfFile: str) -> None:
        self.inputFile = nameOfFile

    def setResultsFile(self, nameOfFile: str) -> None:
        self.outputFile = nameOfFile

    def initialize(self, numberOfEntities: int, dimensionOfEntity: int, numberOfNeighbors: int,
                   device: int, typeOfDistance: int, klaster: bool, numberOfTrees: int,
                   numberOfPropagations: int, minSize: int) -> bool:
        try:
            load_library()
            self.N, self.d, self.k = numberOfEntities, dimensionOfEntity, numberOfNeighbors
            self.device, self.metric, self.klaster = device, typeOfDistance, klaster
            self.trees, self.props, self.leaf = numberOfTrees, numberOfPropagations, minSize
            self._data, _ = formats.read_csv(self.inputFile, self.N, self.d, klaster)
            return False
        except Exception as e:  # noqa: BLE001 - mirror the bool error protocol
            self.last_error = str(e)
            return True

    def calculate(self) -> bool:
        try:
            import time
            t = time.perf_counter()
            x = normalize_reference(self._data)
            self._idx, self._dist = knn_build(x, self.k, self.trees, self.leaf, self.props,
                                              self.metric)
            self.elapsed_ms = (time.perf_counter() - t) * 1e3
            return False
        except Exception as e:  # noqa: BLE001
            self.last_error = str(e)
            return True

    def saveResultToResultFile(self) -> bool:
        try:
            formats.write_result(self.outputFile, self._idx, self._dist, self.metric,
                                 debug=self.debugMode)
            return False
        except Exception as e:  # noqa: BLE001
            self.last_error = str(e)
            return True

    def deinitialize(self) -> bool:
        self._data = self._idx = self._dist = None
        return False

#!/usr/bin/env python
"""k-NN graph build throughput on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full k-NN graph build (trees -> leaf blocks -> propagation ->
sorted lists) of the integer-mixture workload: N=1,000,000 points, d=128,
float32 integer values in [0,255] from a 256-cluster Gaussian mixture (seeded
synthetic data, no dataset needed); k=16, 16 trees, leaf 64, 5 propagations,
EUCLIDEAN.  `value` is points/s with the points already in HBM; `e2e` is the
same metric through the public C ABI with pinned host buffers (host->device
copy of the points and device->host copy of the graph inside the timed
region).  Recall@k and distance error are measured against the FP64 exact
graph on 10,000 seeded queries.

With --gpus N > 1 (launched by torchrun) every rank builds the graph of its own
dataset (seed = rank): independent replicas, weak scaling, no collective on
the data path.  `--impl reference` times the CPU rendition of the reference
algorithm (the reference itself has no CPU implementation) on a bounded
sample of the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "approximate-cuda-knn_b200"
METRIC_NAME = "k-NN graph points/s at recall@k≥0.95 vs FP64 exact, mixed/learned vs plain FP32"
METRIC_NAMES = {0: "EUCLIDEAN", 1: "TAXICAB", 2: "COSINE"}


def load_package():
    if "acknn" in sys.modules:
        return sys.modules["acknn"]
    spec = importlib.util.spec_from_file_location(
        "acknn", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["acknn"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- workloads --
WORKLOAD = dict(name="integer_mixture", n=1_000_000, d=128, k=16, trees=16, leaf=64, props=5,
                metric=0)


def workload_desc(w) -> str:
    return (f"integer_mixture N={w['n']:,} d={w['d']} float32 ints in [0,255] (256-cluster "
            f"mixture, sigma 20); k={w['k']}, {w['trees']} trees, leaf {w['leaf']}, "
            f"{w['props']} propagations, {METRIC_NAMES[w['metric']]}")


def make_points(acknn, n: int, seed: int) -> np.ndarray:
    return acknn.workloads.integer_mixture(seed=seed, n=n)


# ------------------------------------------------------------- accuracy --
def accuracy(acknn, x: np.ndarray, idx: np.ndarray, dist: np.ndarray, k: int, metric: int,
             nq: int = 10_000, seed: int = 12345) -> dict:
    n = x.shape[0]
    rng = np.random.Generator(np.random.PCG64(seed))
    q = np.sort(rng.choice(n, size=min(nq, n), replace=False)).astype(np.int64)
    ei, ed = acknn.exact_fp64(x, k, q, metric)
    ai, ad = idx[q], dist[q]
    # FP64 distance of the returned pairs
    a = x[q].astype(np.float64)
    pair = np.empty(ai.shape, dtype=np.float64)
    for s in range(k):
        b = x[ai[:, s]].astype(np.float64)
        if metric == 0:
            pair[:, s] = np.sqrt(((a - b) ** 2).sum(1))
        elif metric == 1:
            pair[:, s] = np.abs(a - b).sum(1)
        else:
            den = np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1)
            pair[:, s] = np.where(den == 0, 1.0, 1.0 - (a * b).sum(1) / np.where(den == 0, 1, den))
    kth = ed[:, -1:]
    tie_aware = float(np.mean(pair <= kth * (1 + 1e-12) + 1e-12))
    hits = sum(len(np.intersect1d(ai[i], ei[i])) for i in range(len(q)))
    rel = np.abs(ad.astype(np.float64) - pair) / np.maximum(np.abs(pair), 1e-30)
    return {"recall": tie_aware, "recall_id": hits / (k * len(q)),
            "dist_rel_err_max": float(rel.max()), "dist_rel_err_mean": float(rel.mean()),
            "queries": int(len(q))}


# ------------------------------------------------------------ CPU rendition --
def cpu_rendition(w, sample_n: int, repeats: int = 1) -> dict:
    """The oracle's OpenMP rendition of the algorithm on a bounded sample."""
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import Oracle  # noqa: E402  -- the CPU baseline leg only

    lib = ROOT / "oracle" / "liboracle.so"
    if not lib.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "liboracle.so"], check=True,
                       capture_output=True)
    orc = Oracle(lib)
    acknn = load_package()
    x = make_points(acknn, sample_n, seed=0)
    cores = os.cpu_count() or 1
    times = []
    for _ in range(repeats):
        t = time.perf_counter()
        orc.knn_build(x, w["k"], w["trees"], w["leaf"], w["props"], w["metric"], seed=0,
                      threads=cores)
        times.append(time.perf_counter() - t)
    sec = min(times)
    return {"value": sample_n / sec, "unit": "points/s", "cores": cores, "kind": "port",
            "sample": f"{sample_n:,} points of the same generator and parameters "
                      f"(full workload is {w['n']:,}); best of {repeats}; {sec:.2f} s",
            "seconds": sec}


# ------------------------------------------------------------------ main --
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, w):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    sample = args.cpu_sample
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_rendition(w, sample, repeats=1)
        if i >= args.warmup:
            vals.append(r)
    sec = sum(r["seconds"] for r in vals) / len(vals)
    value = sample / sec
    cores = vals[0]["cores"]
    line = {
        "impl": "reference", "metric": METRIC_NAME, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_desc(w), "sample_points": sample,
                   "implementation": "CPU rendition of the reference algorithm (OpenMP), the "
                                     "reference has no CPU path of its own"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port",
                         "sample": vals[0]["sample"]},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, w):
    import torch

    world, rank, local = dist_setup()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    acknn = load_package()
    lib = acknn.load_library()
    n, d, k = w["n"], w["d"], w["k"]
    x = make_points(acknn, n, seed=rank)
    xh = torch.from_numpy(x).pin_memory()
    xd = xh.to(f"cuda:{dev}")
    idx_d = torch.empty((n, k), dtype=torch.int32, device=f"cuda:{dev}")
    dist_d = torch.empty((n, k), dtype=torch.float32, device=f"cuda:{dev}")
    idx_h = torch.empty((n, k), dtype=torch.int32).pin_memory()
    dist_h = torch.empty((n, k), dtype=torch.float32).pin_memory()
    ctx = acknn.Context(dev)
    stream = torch.cuda.current_stream()
    prec = acknn.PREC_BF16_RERANK if args.precision == "bf16" else acknn.PREC_FP32

    opt_dev = acknn.default_options(device=dev, points_on_device=1, outputs_on_device=1,
                                    stream=stream.cuda_stream, precision=prec)
    opt_host = acknn.default_options(device=dev, points_on_device=0, outputs_on_device=0,
                                     stream=stream.cuda_stream, precision=prec)

    def step_device(stats=None):
        rc = lib.knn_build_ex(ctx.handle, xd.data_ptr(), n, d, k, w["trees"], w["leaf"],
                              w["props"], w["metric"], args.seed, idx_d.data_ptr(),
                              dist_d.data_ptr(), ctypes.byref(opt_dev),
                              ctypes.byref(stats) if stats is not None else None)
        if rc:
            raise acknn.KnnError(rc, lib.knn_last_error().decode())

    def step_host():
        rc = lib.knn_build_ex(ctx.handle, xh.data_ptr(), n, d, k, w["trees"], w["leaf"],
                              w["props"], w["metric"], args.seed, idx_h.data_ptr(),
                              dist_h.data_ptr(), ctypes.byref(opt_host), None)
        if rc:
            raise acknn.KnnError(rc, lib.knn_last_error().decode())

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up (allocates the context's scratch)
    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()

    # one instrumented call for stage times and counts
    st = acknn.KnnStats()
    st.struct_size = ctypes.sizeof(acknn.KnnStats)
    step_device(st)
    torch.cuda.synchronize()
    stages = st.as_dict()

    # timed: device-resident points and graph
    clocks = ClockSampler(dev)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_device()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    # timed: end to end through the public API with pinned host buffers
    barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        step_host()
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps)

    # the device and host results must agree (same build)
    same = bool(torch.equal(idx_d.cpu(), idx_h) and torch.equal(dist_d.cpu(), dist_h))

    acc = accuracy(acknn, x, idx_h.numpy(), dist_h.numpy(), k, w["metric"]) if rank == 0 else {}

    value = world * n / (ms / 1e3)
    value_e2e = world * n / (ms_e2e / 1e3)

    # roofline of the dominant stage (algorithmic bytes per launch / mean launch time)
    peak, peak_kind = measured_peaks()
    T, L, P = w["trees"], stages["depth"], w["props"]
    s = 4
    prop_bytes = sum(n * (k * k * 4 + 2 * k * 8) + c * d * s for c in stages["prop_candidates"])
    leaf_bytes = T * (n * d * s + n * k * 8)
    tree_bytes = T * L * (n * d * s + 16 * n)
    cand = {"propagate": (stages["ms_propagate"], prop_bytes, P),
            "leaf": (stages["ms_leaf"], leaf_bytes, T),
            "trees": (stages["ms_trees"], tree_bytes, 3 * L)}
    dom = max(cand, key=lambda kname: cand[kname][0])
    dms, dbytes, dlaunch = cand[dom]
    achieved = dbytes / (dms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": dbytes / max(1, dlaunch),
                "mean_launch_ms": dms / max(1, dlaunch)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_rendition(w, args.cpu_sample)
        cpu = {kk: r[kk] for kk in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": METRIC_NAME, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded integer Gaussian mixture; seed = rank)",
            "config": {"workload": workload_desc(w), "n": n, "d": d, "k": k,
                       "trees": w["trees"], "leaf": w["leaf"], "props": w["props"],
                       "metric": METRIC_NAMES[w["metric"]], "precision": args.precision,
                       "l2": "inputs larger than L2 (512 MB of points per step)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "accuracy": acc, "stages_ms": {kk: stages[kk] for kk in (
                "ms_upload", "ms_trees", "ms_leaf", "ms_propagate", "ms_download", "ms_total")},
            "prop_candidates": stages["prop_candidates"],
            "e2e": {"value": value_e2e, "unit": "points/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(n * d * 4),
                    "d2h_bytes_per_step": int(n * k * 8), "matches_device_run": same},
            "gpu_launches": int(stages["launches"]) * args.steps * 2,
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "bf16"], default="fp32")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n", type=int, default=None, help="override N (smaller runs)")
    ap.add_argument("--cpu-sample", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = dict(WORKLOAD)
    if args.n:
        w["n"] = args.n
    if args.impl == "reference":
        return run_reference(args, w)
    return run_ours(args, w)


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""k-NN graph build throughput on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (seeded synthetic data, no dataset needed): the integer mixture,
N=1,000,000 points, d=128, float32 integer values in [0,255] drawn from a
256-cluster Gaussian mixture (centres U[0,255], sigma 20); k=16, EUCLIDEAN.

Metric: k-NN graph points/s at recall@k >= 0.95 against the FP64 exact graph.
A step is one full graph build (trees -> leaf blocks -> propagation -> sorted
lists).  The headline path is the mixed-precision builder (BF16 tcgen05 leaf
tiles + exact FP32 re-rank) at its cheapest setting that reaches recall 0.95 on
this workload (8 trees, leaf 2048, no propagation); the plain FP32 builder is
timed at its own cheapest such setting (16 trees, leaf 512, 1 propagation),
which is the equal-recall comparison, and once at the mixed path's setting
(identical output on this data: every BF16 product and FP32 sum is exact).
Both also run at the configuration's literal parameters (16 trees, leaf 64,
5 propagations), which stay below 0.95.

`value` is points/s with the points already in HBM (512 MB, larger than L2);
`e2e` is the same build through the public C ABI with pinned host buffers
(host->device copy of the points and device->host copy of the graph inside the
timed region).  Recall@k and distance error are measured against the FP64
exact graph (knn_exact_fp64) on 10,000 seeded queries.

With --gpus N > 1 (launched by torchrun) every rank builds the graph of its own
dataset (seed = rank): independent replicas, weak scaling, no collective on
the data path.  `--impl reference` times the CPU rendition of the reference
algorithm (the reference itself has no CPU implementation) on a bounded sample
of the same workload with all host threads.
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

WORKLOAD = dict(name="integer_mixture", n=1_000_000, d=128, k=16, metric=0)
# the configuration's own parameters
CONFIG_PARAMS = dict(trees=16, leaf=64, props=5)
# cheapest settings found to reach recall@16 >= 0.95 on this workload in a sweep
# of trees {6..20} x leaf {64..2048} x propagations {0..5}, each path on its own:
# the mixed-precision builder ...
TARGET_PARAMS = dict(trees=8, leaf=2048, props=0)
# ... and the plain FP32 builder (equal-recall comparison)
PLAIN_TARGET_PARAMS = dict(trees=16, leaf=512, props=1)


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


def profiled_traffic(summary: str, config: dict, n: int):
    """DRAM bytes per launch from a committed ncu summary under profiles/: the
    line `traffic_bytes_per_launch: B n=N d=.. k=.. trees=.. leaf=..` gives the
    mean per launch on N points; it is scaled to n (a launch's traffic grows
    with the points it processes).  (None, reason) when the summary is absent
    or was taken on another configuration."""
    import re

    path = ROOT / "profiles" / summary
    if not path.exists():
        return None, f"profiles/{summary} absent"
    m = re.search(r"^traffic_bytes_per_launch: (\d+) n=(\d+) (.*)$", path.read_text(), flags=re.M)
    if not m:
        return None, f"no traffic line in profiles/{summary}"
    fields = dict(kv.split("=") for kv in m.group(3).split())
    if any(str(config[key]) != fields.get(key) for key in config):
        return None, f"profiles/{summary} was taken on another configuration ({m.group(3)})"
    b, pn = int(m.group(1)), int(m.group(2))
    return b * n / pn, (f"ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, mean over a build's "
                        f"launches at {pn:,} points (profiles/{summary}), scaled to {n:,} points")


def measured_tensor_peak() -> tuple[float, str]:
    """Dense bf16 TFLOP/s: the burst figure (the leaf kernel runs at full clock in the bench)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops"]), "measured (burst)"
    return 1590.0, "fallback (burst)"


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


def workload_desc(w, p) -> str:
    return (f"integer_mixture N={w['n']:,} d={w['d']} float32 ints in [0,255] (256-cluster "
            f"mixture, sigma 20); k={w['k']}, {p['trees']} trees, leaf {p['leaf']}, "
            f"{p['props']} propagation(s), {METRIC_NAMES[w['metric']]}")


def make_points(acknn, n: int, seed: int) -> np.ndarray:
    return acknn.workloads.integer_mixture(seed=seed, n=n)


# ------------------------------------------------------------- accuracy --
def accuracy(acknn, x, idx, dist, k, metric, exact, q, gathered: bool = False) -> dict:
    """Recall@k (tie-aware and by id) and distance error against the FP64 exact
    graph on the query rows q; ``gathered``: idx/dist hold only those rows."""
    ei, ed = exact
    ai, ad = (idx, dist) if gathered else (idx[q], dist[q])
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
def cpu_rendition(w, p, sample_n: int) -> dict:
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
    t = time.perf_counter()
    orc.knn_build(x, w["k"], p["trees"], p["leaf"], p["props"], w["metric"], seed=0,
                  threads=cores)
    sec = time.perf_counter() - t
    return {"value": sample_n / sec, "unit": "points/s", "cores": cores, "kind": "port",
            "sample": f"{sample_n:,} points of the same generator with {p['trees']} trees, leaf "
                      f"{p['leaf']}, {p['props']} propagation(s) (full workload {w['n']:,}); "
                      f"{sec:.2f} s",
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
    p = TARGET_PARAMS
    # every step is one bounded sample, so that --steps K --warmup W ends in minutes
    sample = min(args.cpu_sample, 10_000)
    secs, last = [], None
    for i in range(args.warmup + args.steps):
        r = cpu_rendition(w, p, sample)
        if i >= args.warmup:
            secs.append(r["seconds"])
            last = r
    sec = sum(secs) / len(secs)
    value = sample / sec
    line = {
        "impl": "reference", "metric": METRIC_NAME, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_desc(w, p), "sample_points": sample,
                   "implementation": "CPU rendition of the reference algorithm (OpenMP, keys of eight "
                                     "candidates interleaved); the reference has no CPU path of its own"},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": last["cores"],
                         "kind": "port", "sample": last["sample"]},
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
    n, d, k, metric = w["n"], w["d"], w["k"], w["metric"]
    x = make_points(acknn, n, seed=rank)
    xh = torch.from_numpy(x).pin_memory()
    xd = xh.to(f"cuda:{dev}")
    idx_d = torch.empty((n, k), dtype=torch.int32, device=f"cuda:{dev}")
    dist_d = torch.empty((n, k), dtype=torch.float32, device=f"cuda:{dev}")
    idx_h = torch.empty((n, k), dtype=torch.int32).pin_memory()
    dist_h = torch.empty((n, k), dtype=torch.float32).pin_memory()
    ctx = acknn.Context(dev)
    stream = torch.cuda.current_stream()
    MIXED, PLAIN = acknn.PREC_BF16_RERANK, acknn.PREC_FP32
    head = TARGET_PARAMS

    def build(p, prec, host=False, stats=None):
        opt = acknn.default_options(device=dev, points_on_device=0 if host else 1,
                                    outputs_on_device=0 if host else 1,
                                    stream=stream.cuda_stream, precision=prec)
        src = xh if host else xd
        oi, od = (idx_h, dist_h) if host else (idx_d, dist_d)
        rc = lib.knn_build_ex(ctx.handle, src.data_ptr(), n, d, k, p["trees"], p["leaf"],
                              p["props"], metric, args.seed, oi.data_ptr(), od.data_ptr(),
                              ctypes.byref(opt), ctypes.byref(stats) if stats is not None else None)
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

    def timed(fn, steps) -> float:
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # warm-up of the headline build (allocates the context's scratch)
    for _ in range(args.warmup):
        build(head, MIXED)
    torch.cuda.synchronize()
    st = acknn.KnnStats()
    st.struct_size = ctypes.sizeof(acknn.KnnStats)
    build(head, MIXED, stats=st)
    torch.cuda.synchronize()
    stages = st.as_dict()

    clocks = ClockSampler(dev)
    clocks.start()
    # the last timed step also records CUDA events around each leaf-tile kernel
    # launch (its statistics; the call then synchronises before returning)
    st_live = acknn.KnnStats()
    st_live.struct_size = ctypes.sizeof(acknn.KnnStats)
    step_no = [0]

    def headline_step():
        step_no[0] += 1
        build(head, MIXED, stats=st_live if step_no[0] == args.steps else None)

    ms = timed(headline_step, args.steps)
    leaf_kernel_ms = st_live.ms_leaf_tiles
    ms_e2e = timed(lambda: build(head, MIXED, host=True), args.steps)
    clk = clocks.stop()
    mixed_idx = idx_h.numpy().copy()
    mixed_dist = dist_h.numpy().copy()
    same_dev_host = bool(torch.equal(idx_d.cpu(), idx_h) and torch.equal(dist_d.cpu(), dist_h))

    # the plain FP32 builder at its own cheapest setting reaching recall 0.95
    build(PLAIN_TARGET_PARAMS, PLAIN)
    ms_plain = timed(lambda: build(PLAIN_TARGET_PARAMS, PLAIN), args.steps)
    plain_idx = idx_d.cpu().numpy()
    plain_dist = dist_d.cpu().numpy()
    # and at the mixed path's setting (one step): on this data every BF16 product
    # and FP32 sum is exact, so the two graphs must be identical
    build(head, PLAIN)
    ms_plain_same = timed(lambda: build(head, PLAIN), 1)
    plain_same = bool(np.array_equal(idx_d.cpu().numpy(), mixed_idx) and
                      np.array_equal(dist_d.cpu().numpy(), mixed_dist))
    # both at the configuration's literal parameters (one step each, after a warm-up)
    lit = {}
    for name, prec in (("plain_fp32", PLAIN), ("mixed", MIXED)):
        build(CONFIG_PARAMS, prec)
        lit[name] = {"ms": timed(lambda: build(CONFIG_PARAMS, prec), 1)}
    lit_idx = idx_d.cpu().numpy()
    lit_dist = dist_d.cpu().numpy()

    acc = lit_acc = plain_acc = {}
    if rank == 0:
        rng = np.random.Generator(np.random.PCG64(12345))
        q = np.sort(rng.choice(n, size=min(10_000, n), replace=False)).astype(np.int64)
        exact = acknn.exact_fp64(x, k, q, metric)
        acc = accuracy(acknn, x, mixed_idx, mixed_dist, k, metric, exact, q)
        lit_acc = accuracy(acknn, x, lit_idx, lit_dist, k, metric, exact, q)
        plain_acc = accuracy(acknn, x, plain_idx, plain_dist, k, metric, exact, q)
    for v in lit.values():
        v["points_per_s"] = world * n / (v["ms"] / 1e3)
        v["recall"] = lit_acc.get("recall")

    value = world * n / (ms / 1e3)
    value_e2e = world * n / (ms_e2e / 1e3)
    value_plain = world * n / (ms_plain / 1e3)

    # roofline of the dominant stage (algorithmic bytes per launch / mean launch time)
    peak, peak_kind = measured_peaks()
    T, L, P = head["trees"], stages["depth"], head["props"]
    s = 4
    kq = min(32, 2 * k)
    prop_bytes = sum(n * (k * k * 4 + 2 * k * 8) + c * d * s for c in stages["prop_candidates"])
    # tensor-core leaf stage: the BF16 rows (d*2 B) and each point's kq-entry list per tree
    leaf_bytes = T * (n * d * 2 + n * kq * 8 * 2)
    tree_bytes = T * L * (n * d * s + 16 * n)
    cand = {"propagate": (stages["ms_propagate"], prop_bytes, max(1, P)),
            "leaf_tc": (leaf_kernel_ms if leaf_kernel_ms > 0 else stages["ms_leaf"], leaf_bytes, T),
            "trees": (stages["ms_trees"], tree_bytes, 3 * L)}
    dom = max(cand, key=lambda kname: cand[kname][0])
    dms, dbytes, dlaunch = cand[dom]
    achieved = dbytes / (dms / 1e3) / 1e9
    # DRAM bytes (read + write) per k_leaf_tc launch from the committed ncu
    # summary of this kernel on a smaller case of the same configuration,
    # scaled by the points a launch processes
    traffic, traffic_src = None, None
    if dom == "leaf_tc":
        traffic, traffic_src = profiled_traffic("k_leaf_tc_integer_mixture_500k.md",
                                                dict(d=d, k=k, trees=T, leaf=head["leaf"]), n)
    hbm_view = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "traffic_source": traffic_src,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": dbytes / dlaunch,
                "mean_launch_ms": dms / dlaunch,
                "mean_launch_source": "CUDA events around each k_leaf_tc launch of the last timed step"
                if dom == "leaf_tc" and leaf_kernel_ms > 0 else "stage time / launches"}
    roofline = hbm_view
    if dom == "leaf_tc":
        # the tile products: 2 d flops per (query, candidate) pair of every leaf
        # block (median trees: leaf j holds points [j n / 2^D, (j + 1) n / 2^D))
        nl = 1 << L
        pairs = sum(((j + 1) * n // nl - j * n // nl) ** 2 for j in range(nl))
        flops = 2.0 * d * pairs
        tpeak, tkind = measured_tensor_peak()
        tach = flops / (dms / dlaunch / 1e3) / 1e12
        tensor_view = {"bound": "tensor", "kernel": dom, "achieved": tach, "peak": tpeak, "unit": "TFLOP/s",
                       "frac": tach / tpeak, "traffic": traffic, "peak_source": tkind,
                       "algorithmic_flops_per_launch": flops, "mean_launch_ms": dms / dlaunch,
                       "mean_launch_source": hbm_view["mean_launch_source"]}
        # the roofline that binds: the larger of the two times at peak
        if flops / (tpeak * 1e12) >= (dbytes / dlaunch) / (peak * 1e9):
            roofline, hbm_view = tensor_view, {**hbm_view, "binding": False}
            roofline["hbm_view"] = hbm_view

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_rendition(w, head, args.cpu_sample)
        cpu = {kk: r[kk] for kk in ("value", "unit", "cores", "kind", "sample")}

    # the reference's own CUDA build on the same points (its CLI, its own timer),
    # after every timed region of this process: at the headline setting (about
    # 1.5 min) and at the configuration's literal setting (about 1 min)
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        settings = {"headline": head}
        if not args.reference_gpu_headline_only:
            settings["literal"] = CONFIG_PARAMS
        ref_gpu = reference_gpu_runs(acknn, x, k, q, exact[0], settings, args.ref_limit)
        for name, rr in ref_gpu.items():
            if isinstance(rr, dict) and rr.get("ms_calculate"):
                ours = value if rr["params"] == head else lit.get("mixed", {}).get("points_per_s")
                rr["ours_points_per_s_same_setting"] = ours

    if rank == 0:
        line = {
            "metric": METRIC_NAME, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16+f32",
            "data": "synthetic (seeded integer Gaussian mixture; seed = rank)",
            "config": {"workload": workload_desc(w, head), "n": n, "d": d, "k": k,
                       **head, "metric": METRIC_NAMES[metric],
                       "path": "mixed: BF16 tcgen05 leaf tiles + FP32 re-rank",
                       "l2": "inputs larger than L2 (512 MB of points per step)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "accuracy": acc,
            "plain_fp32_equal_recall": {"params": PLAIN_TARGET_PARAMS, "value": value_plain,
                                        "ms_per_step": ms_plain, "recall": plain_acc.get("recall"),
                                        "mixed_speedup": value / value_plain},
            "plain_fp32_same_setting": {"ms_per_step": ms_plain_same,
                                        "value": world * n / (ms_plain_same / 1e3),
                                        "identical_graph": plain_same},
            "config_literal_params": {"params": CONFIG_PARAMS, **lit},
            "stages_ms": {kk: stages[kk] for kk in (
                "ms_upload", "ms_trees", "ms_leaf", "ms_propagate", "ms_download", "ms_total")},
            "prop_candidates": stages["prop_candidates"],
            "e2e": {"value": value_e2e, "unit": "points/s", "ms_per_step": ms_e2e,
                    "h2d_bytes_per_step": int(n * d * 4),
                    "d2h_bytes_per_step": int(n * k * 8), "matches_device_run": same_dev_host},
            "gpu_launches": int(stages["launches"]) * args.steps * 2,
            "gpu_launches_note": "kernels of the timed device-resident and end-to-end mixed builds",
            "roofline": roofline, "cpu_baseline": cpu, "reference_gpu": ref_gpu, "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------- single-build case --
def run_single(args, w):
    """One configuration, W warm-up builds then K timed builds on device-resident
    points; prints per-stage times.  The case the ncu summaries in profiles/
    are taken on (a fixed, committed command line)."""
    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    lib = acknn.load_library()
    if args.workload == "integer_mixture":
        n, k, metric = w["n"], w["k"], w["metric"]
        p = dict(TARGET_PARAMS)
        xh = make_points(acknn, n, seed=args.seed)
        desc = workload_desc
    else:
        cfg = acknn.workloads.CONFIGS[args.workload]
        n, k, metric = args.n or cfg["n"], cfg["k"], cfg["metric"]
        p = {kk: cfg[kk] for kk in ("trees", "leaf", "props")}
        xh = cfg["gen"](args.seed, n=n)

        def desc(_w, pp):
            return (f"{args.workload} N={n:,} d={xh.shape[1]} {xh.dtype}; k={k}, {pp['trees']} trees, leaf "
                    f"{pp['leaf']}, {pp['props']} propagation(s), {METRIC_NAMES[metric]}")
    d = xh.shape[1]
    dtype = acknn.F16 if xh.dtype == np.float16 else acknn.F32
    for key in ("trees", "leaf", "props"):
        if getattr(args, key) is not None:
            p[key] = getattr(args, key)
    prec = {"mixed": acknn.PREC_BF16_RERANK, "mixed_f16": acknn.PREC_F16_RERANK}.get(args.single, acknn.PREC_FP32)
    x = torch.from_numpy(xh).cuda()
    idx = torch.empty((n, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((n, k), dtype=torch.float32, device="cuda")
    ctx = acknn.Context(0)
    stream = torch.cuda.current_stream()

    def build(stats=None):
        opt = acknn.default_options(points_on_device=1, outputs_on_device=1, stream=stream.cuda_stream,
                                    precision=prec, dtype=dtype)
        rc = lib.knn_build_ex(ctx.handle, x.data_ptr(), n, d, k, p["trees"], p["leaf"], p["props"], metric,
                              args.seed, idx.data_ptr(), dist.data_ptr(), ctypes.byref(opt),
                              ctypes.byref(stats) if stats is not None else None)
        if rc:
            raise acknn.KnnError(rc, lib.knn_last_error().decode())

    for _ in range(args.warmup):
        build()
    st = acknn.KnnStats()
    st.struct_size = ctypes.sizeof(acknn.KnnStats)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        build()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    build(stats=st)
    torch.cuda.synchronize()
    sd = st.as_dict()
    print(json.dumps({"case": args.single, "workload": desc(w, p), "ms_per_build": ms,
                      "points_per_s": n / (ms / 1e3),
                      "stages_ms": {kk: sd[kk] for kk in ("ms_trees", "ms_leaf", "ms_propagate", "ms_total")},
                      "prop_candidates": sd["prop_candidates"], "ms_leaf_tiles": sd["ms_leaf_tiles"],
                      "launches": sd["launches"], "depth": sd["depth"]}), flush=True)
    ctx.close()
    return 0


# ---------------------------------------------------------- dataset batch --
# Cheapest settings reaching aggregate recall@15 >= 0.95 over the batch, per
# path, from `--workload dataset_batch --sweep`.
BATCH_TARGETS = {"plain_fp32": (8, 512, 3), "mixed": (3, 4096, 0)}


def run_batch(args):
    """The 256-dataset batch: N log-uniform in [1e3, 2e5], d uniform over
    {32, 64, 128, 256}, 16-cluster Gaussian mixtures, seeds 0..255; k=15,
    EUCLIDEAN.  Each path at its own cheapest setting reaching aggregate
    recall 0.95 (BATCH_TARGETS; recall over the seeded queries of all sets,
    up to 500 per set, against FP64 exact), device-resident sets, autotuned
    shapes, captured graphs replayed; the mixed path also end to end from
    pinned host buffers.  At the configuration's literal parameters (8 trees,
    leaf 48, 3 propagations): a loop of single plain builds against the
    batched plain and mixed builds."""
    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    lib = acknn.load_library()
    cfg = acknn.workloads.CONFIGS["dataset_batch"]
    count = args.count or cfg["count"]
    k, metric = cfg["k"], cfg["metric"]
    lit = (cfg["trees"], cfg["leaf"], cfg["props"])
    xs = [acknn.workloads.batch_dataset(s) for s in range(count)]
    ntot = sum(x.shape[0] for x in xs)
    xh = [torch.from_numpy(x).pin_memory() for x in xs]
    xd = [t.cuda() for t in xh]
    oi = [torch.empty((x.shape[0], k), dtype=torch.int32, device="cuda") for x in xs]
    od = [torch.empty((x.shape[0], k), dtype=torch.float32, device="cuda") for x in xs]
    hi = [torch.empty((x.shape[0], k), dtype=torch.int32).pin_memory() for x in xs]
    hd = [torch.empty((x.shape[0], k), dtype=torch.float32).pin_memory() for x in xs]
    ctx = acknn.Context(0)
    stream = torch.cuda.current_stream()

    def table(host):
        arr = (acknn.KnnDataset * count)()
        for i, x in enumerate(xs):
            arr[i].points = (xh if host else xd)[i].data_ptr()
            arr[i].n, arr[i].d, arr[i].seed = x.shape[0], x.shape[1], i
            arr[i].out_idx = (hi if host else oi)[i].data_ptr()
            arr[i].out_dist = (hd if host else od)[i].data_ptr()
        return arr

    dev_tab, host_tab = table(False), table(True)

    def batch(prec, p, host=False, stats=None):
        opt = acknn.default_options(points_on_device=0 if host else 1, outputs_on_device=0 if host else 1,
                                    stream=stream.cuda_stream, precision=prec, autotune=1)
        rc = lib.knn_build_batch(ctx.handle, host_tab if host else dev_tab, count, k, p[0], p[1], p[2], metric,
                                 ctypes.byref(opt), ctypes.byref(stats) if stats is not None else None)
        if rc:
            raise acknn.KnnError(rc, lib.knn_last_error().decode())

    def loop(prec, p):
        for i, x in enumerate(xs):
            opt = acknn.default_options(points_on_device=1, outputs_on_device=1, stream=stream.cuda_stream,
                                        precision=prec)
            rc = lib.knn_build_ex(ctx.handle, xd[i].data_ptr(), x.shape[0], x.shape[1], k, p[0], p[1], p[2],
                                  metric, i, oi[i].data_ptr(), od[i].data_ptr(), ctypes.byref(opt), None)
            if rc:
                raise acknn.KnnError(rc, lib.knn_last_error().decode())

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    rng = np.random.Generator(np.random.PCG64(7))
    qs, exact = [], []
    for x in xs:
        q = np.sort(rng.choice(x.shape[0], size=min(500, x.shape[0]), replace=False)).astype(np.int64)
        qs.append(q)
        exact.append(acknn.exact_fp64(x, k, q, metric)[0])

    def recall():
        per, hits, total = [], 0, 0
        for i in range(count):
            ai = oi[i].cpu().numpy()[qs[i]]
            h = sum(len(np.intersect1d(a, b)) for a, b in zip(ai, exact[i]))
            per.append(h / (k * len(ai)))
            hits += h
            total += k * len(ai)
        return {"recall": hits / total, "recall_mean_of_sets": sum(per) / len(per), "recall_min": min(per),
                "sets_below_0.95": int(sum(r < 0.95 for r in per))}

    precs = {"plain_fp32": acknn.PREC_FP32, "mixed": acknn.PREC_BF16_RERANK}
    res = {}
    clocks = ClockSampler(0)
    clocks.start()
    for name, p in BATCH_TARGETS.items():
        ms = timed(lambda: batch(precs[name], p), args.steps)
        st = acknn.KnnStats()
        st.struct_size = ctypes.sizeof(acknn.KnnStats)
        batch(precs[name], p, stats=st)
        torch.cuda.synchronize()
        res[name + "@target"] = {"params": dict(zip(("trees", "leaf", "props"), p)), "ms_per_step": ms,
                                 "points_per_s": ntot / (ms / 1e3), "accuracy": recall(),
                                 "stages_ms": {"trees": st.ms_trees, "leaf": st.ms_leaf, "propagate": st.ms_propagate}}
    mp = BATCH_TARGETS["mixed"]
    ms_e2e = timed(lambda: batch(precs["mixed"], mp, host=True), args.steps)
    same = all(torch.equal(oi[i].cpu(), hi[i]) for i in range(count))
    for name, fn in (("loop_plain_fp32@literal", lambda: loop(acknn.PREC_FP32, lit)),
                     ("batch_plain_fp32@literal", lambda: batch(acknn.PREC_FP32, lit)),
                     ("batch_mixed@literal", lambda: batch(acknn.PREC_BF16_RERANK, lit))):
        ms = timed(fn, args.steps)
        res[name] = {"ms_per_step": ms, "points_per_s": ntot / (ms / 1e3)}
    res["batch_mixed@literal"]["accuracy"] = recall()
    clk = clocks.stop()
    value = res["mixed@target"]["points_per_s"]
    line = {
        "metric": "k-NN graph points/s over a batch of independent datasets (aggregate) at recall@k >= 0.95",
        "value": value, "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["mixed@target"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16+f32", "data": "synthetic (seeded Gaussian mixtures)",
        "config": {"workload": f"{count} datasets, N log-uniform in [1e3, 2e5] (total {ntot:,}), d in "
                               f"{{32,64,128,256}}, 16 clusters each, seeds 0..{count - 1}; k={k}, EUCLIDEAN",
                   "path": "knn_build_batch, BF16 tcgen05 leaf tiles + FP32 re-rank, autotuned shapes, "
                           "captured graphs replayed", "targets": BATCH_TARGETS},
        "paths": res,
        "mixed_vs_plain_at_equal_recall": value / res["plain_fp32@target"]["points_per_s"],
        "batch_vs_loop_plain_literal": res["batch_plain_fp32@literal"]["points_per_s"]
        / res["loop_plain_fp32@literal"]["points_per_s"],
        "e2e": {"value": ntot / (ms_e2e / 1e3), "unit": "points/s", "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": int(sum(x.nbytes for x in xs)), "d2h_bytes_per_step": int(ntot * k * 8),
                "matches_device_run": same},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# ------------------------------------------------------- other configurations --
# Cheapest settings reaching recall@k >= 0.95 per path, from `--sweep` runs
# of each configuration (trees, leaf, propagations); None: the path did not
# reach the target within the swept grid (its best setting is given instead).
CONFIG_TARGETS = {
    "sparse_prototypes": {"plain_fp32": (4, 131072, 1)},
    "normalized_mixture": {"plain_fp32": (24, 2048, 0), "mixed_f16": (15, 4096, 0),
                           "mixed_f16_learned": (16, 4096, 1)},
}
PATH_OPTIONS = {
    "plain_fp32": dict(precision=0),
    "plain_fp32_all_dims": dict(precision=0, sparse_dims=-1),
    "mixed": dict(precision=1),
    "mixed_f16": dict(precision=2),
    "mixed_learned": dict(precision=1, learned_splits=1),
    "mixed_f16_learned": dict(precision=2, learned_splits=1),
}


def prop_roofline(n, d, k, s, cands, ms_prop, peak):
    """Propagation against HBM: algorithmic bytes P N (k^2 4 + 2k 8) + sum over
    iterations of c-bar N d s (c-bar N = the keys evaluated in that iteration,
    each reading one candidate row of d elements of s bytes), over the
    propagation time."""
    if not cands or ms_prop <= 0:
        return None
    by = sum(n * (k * k * 4 + 2 * k * 8) + c * d * s for c in cands)
    ach = by / (ms_prop / 1e3) / 1e9
    return {"bound": "hbm", "kernel": "k_propagate", "algorithmic_bytes": by, "ms": ms_prop,
            "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "c_bar": [c / n for c in cands]}


def run_config(args):
    """One named configuration (sparse prototypes, d=784, TAXICAB; normalised
    mixture, 10M x 96 FP16, COSINE): each path at its own cheapest setting that
    reaches recall@k >= 0.95 (CONFIG_TARGETS, from the sweep) and the plain
    FP32 path at the configuration's literal parameters; points resident in
    HBM, recall@k and distance error against the FP64 exact graph on 10,000
    seeded queries, per-stage device times, the propagation kernel's HBM
    roofline and the ratio to plain FP32 at equal recall."""
    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    lib = acknn.load_library()
    cfg = acknn.workloads.CONFIGS[args.workload]
    n = args.n or cfg["n"]
    k, metric = cfg["k"], cfg["metric"]
    x = cfg["gen"](0, n=n)
    d = x.shape[1]
    s_bytes = 2 if x.dtype == np.float16 else 4
    dtype = acknn.F16 if x.dtype == np.float16 else acknn.F32
    xd = torch.from_numpy(x).cuda()
    idx = torch.empty((n, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((n, k), dtype=torch.float32, device="cuda")
    ctx = acknn.Context(0)
    stream = torch.cuda.current_stream()
    rng = np.random.Generator(np.random.PCG64(12345))
    q = np.sort(rng.choice(n, size=min(10_000, n), replace=False)).astype(np.int64)
    qt = torch.from_numpy(q).cuda()
    exact = acknn.exact_fp64(x, k, q, metric)
    peak, peak_kind = measured_peaks()
    runs = {f"{p}@target": (p, tuple(v)) for p, v in CONFIG_TARGETS[args.workload].items() if v}
    runs["plain_fp32@literal"] = ("plain_fp32", (cfg["trees"], cfg["leaf"], cfg["props"]))
    if args.ab_sparse and CONFIG_TARGETS[args.workload].get("plain_fp32"):
        # the same graph with every leaf block reading all dims
        runs["plain_fp32_all_dims@target"] = ("plain_fp32_all_dims", tuple(CONFIG_TARGETS[args.workload]["plain_fp32"]))
    res = {}
    for name, (path, (T, L, P)) in runs.items():
        kw = dict(PATH_OPTIONS[path])
        if kw.get("learned_splits"):
            kw["mlp_sample"] = min(n, 1_000_000)

        def build(stats=None, kw=kw, T=T, L=L, P=P):
            opt = acknn.default_options(points_on_device=1, outputs_on_device=1, dtype=dtype,
                                        stream=stream.cuda_stream, **kw)
            rc = lib.knn_build_ex(ctx.handle, xd.data_ptr(), n, d, k, T, L, P, metric, 0, idx.data_ptr(),
                                  dist.data_ptr(), ctypes.byref(opt), ctypes.byref(stats) if stats else None)
            if rc:
                raise acknn.KnnError(rc, lib.knn_last_error().decode())
        for _ in range(args.warmup):
            build()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            build()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        st = acknn.KnnStats()
        st.struct_size = ctypes.sizeof(acknn.KnnStats)
        build(stats=st)
        torch.cuda.synchronize()
        acc = accuracy(acknn, x, idx[qt].cpu().numpy(), dist[qt].cpu().numpy(), k, metric, exact, q, gathered=True)
        sd = st.as_dict()
        res[name] = {"params": {"trees": T, "leaf": L, "props": P}, "ms_per_build": ms,
                     "points_per_s": n / (ms / 1e3), "accuracy": acc, "leaf_path": sd["leaf_path"],
                     "sparse_dims": sd["sparse_dims"],
                     "stages_ms": {kk: sd[kk] for kk in ("ms_learn", "ms_trees", "ms_leaf", "ms_propagate")},
                     "propagate_roofline": prop_roofline(n, d, k, s_bytes, sd["prop_candidates"],
                                                         sd["ms_propagate"], peak)}
    plain = res.get("plain_fp32@target")
    ratios = {}
    if plain:
        for name, r in res.items():
            if name.endswith("@target") and not name.startswith("plain_fp32"):
                ratios[name.split("@")[0] + "_vs_plain_at_equal_recall"] = plain["ms_per_build"] / r["ms_per_build"]
        dense = res.get("plain_fp32_all_dims@target")
        if dense:
            ratios["sparse_rows_speedup"] = dense["ms_per_build"] / plain["ms_per_build"]
            ratios["sparse_rows_identical_recall"] = dense["accuracy"] == plain["accuracy"]
    print(json.dumps({"workload": args.workload, "n": n, "d": d, "k": k, "metric": METRIC_NAMES[metric],
                      "dtype": str(x.dtype), "queries": int(len(q)), "steps": args.steps, "warmup": args.warmup,
                      "peak_source": peak_kind, "paths": res, **ratios}), flush=True)
    ctx.close()
    return 0


# ------------------------------------------------ the reference's own build --
REF_BIN = ROOT / "oracle" / "_ref" / "hello"


def reference_gpu_runs(acknn, x, k, q, exact_ids, settings, limit_s: float) -> dict:
    """The reference's own CUDA program, built unmodified from its sources for
    sm_100a (oracle/Makefile `ref`), run through its CLI on the same points as
    CSV: per setting its self-reported device time of calculate()
    (euclideandistancematrixgpu.cu:2867, :2889-2893), the wall time of the
    whole process (CSV parse and file write included), and recall@k by id on
    the query rows from its output file.  A run past ``limit_s`` seconds is
    killed and recorded as not run."""
    import re
    import shutil
    import tempfile

    if not REF_BIN.exists():
        return {"not_run": "reference build absent (oracle/_ref/hello)"}
    tmp = Path(tempfile.mkdtemp(prefix="acknn_ref_"))
    out = {}
    try:
        csv = tmp / "points.csv"
        t = time.perf_counter()
        acknn.formats.write_csv_integers(str(csv), x)
        out["csv_write_s"] = time.perf_counter() - t
        out["csv_bytes"] = csv.stat().st_size
        for name, p in settings.items():
            res = tmp / f"{name}.bin"
            cmd = [str(REF_BIN), str(csv), str(res), str(k), str(p["trees"]), str(p["leaf"]),
                   str(p["props"]), "EUCLIDEAN", "0", "F"]
            t = time.perf_counter()
            try:
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=limit_s)
            except subprocess.TimeoutExpired:
                out[name] = {"params": p, "not_run": f"exceeded {limit_s:.0f} s"}
                continue
            wall = time.perf_counter() - t
            m = re.search(r"has done task in: ([0-9.eE+-]+) ms", r.stdout)
            if r.returncode != 0 or not m:
                out[name] = {"params": p, "not_run": f"exit {r.returncode}: {r.stdout[-300:]}"}
                continue
            _, _, ids, _ = acknn.formats.read_result(str(res))
            ai = ids[q]
            rec = sum(len(np.intersect1d(a, b)) for a, b in zip(ai, exact_ids)) / (k * len(q))
            ms = float(m.group(1))
            out[name] = {"params": p, "ms_calculate": ms, "points_per_s": x.shape[0] / (ms / 1e3),
                         "process_wall_s": wall, "recall_id": rec}
            res.unlink(missing_ok=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def run_reference_gpu_batch(args):
    """The 256-dataset batch through the reference's own build: one process
    per set (the reference builds one set per process), at the batch's
    literal parameters; its self-reported device time summed over the sets,
    the wall time of all processes, and recall@k by id per set against the
    FP64 exact graph (up to 500 seeded queries per set).  Our batched build of
    the same sets at the same parameters (plain FP32 and BF16 tiles) is timed
    beside it.  Sets are stopped once `--ref-limit` seconds of wall time have
    gone by."""
    import re
    import shutil
    import tempfile

    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    lib = acknn.load_library()
    cfg = acknn.workloads.CONFIGS["dataset_batch"]
    count = args.count or cfg["count"]
    k, T, L, P = cfg["k"], cfg["trees"], cfg["leaf"], cfg["props"]
    xs = [acknn.workloads.batch_dataset(s) for s in range(count)]
    tmp = Path(tempfile.mkdtemp(prefix="acknn_refb_"))
    ref_ms, ref_wall, ref_rec, done = 0.0, 0.0, [], 0
    ours_rec = {"plain_fp32": [], "mixed": []}
    rng = np.random.Generator(np.random.PCG64(7))
    t_all = time.perf_counter()
    try:
        for i, x in enumerate(xs):
            if time.perf_counter() - t_all > args.ref_limit:
                break
            q = np.sort(rng.choice(x.shape[0], size=min(500, x.shape[0]), replace=False)).astype(np.int64)
            csv = tmp / "set.csv"
            parsed = acknn.formats.write_csv_fixed(str(csv), x)
            xn = acknn.normalize_reference(parsed)
            ei, _ = acknn.exact_fp64(xn, k, q, 0)
            out = tmp / "set.bin"
            t = time.perf_counter()
            r = subprocess.run([str(REF_BIN), str(csv), str(out), str(k), str(T), str(L), str(P), "EUCLIDEAN", "0", "F"],
                               capture_output=True, text=True, timeout=max(30.0, args.ref_limit))
            ref_wall += time.perf_counter() - t
            m = re.search(r"has done task in: ([0-9.eE+-]+) ms", r.stdout)
            if r.returncode != 0 or not m:
                break
            ref_ms += float(m.group(1))
            _, _, ids, _ = acknn.formats.read_result(str(out))
            ref_rec.append(sum(len(np.intersect1d(a, b)) for a, b in zip(ids[q], ei)) / (k * len(q)))
            for name, prec in (("plain_fp32", acknn.PREC_FP32), ("mixed", acknn.PREC_BF16_RERANK)):
                oi, _ = acknn.knn_build(xn, k, T, L, P, 0, seed=i, precision=prec)
                ours_rec[name].append(sum(len(np.intersect1d(a, b)) for a, b in zip(oi[q], ei)) / (k * len(q)))
            done += 1
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    pts = sum(x.shape[0] for x in xs[:done])
    # our batched build of the same sets (device-resident, captured graphs replayed)
    stream = torch.cuda.current_stream()
    ctx = acknn.Context(0)
    sub = xs[:done]
    xd = [torch.from_numpy(acknn.normalize_reference(x)).cuda() for x in sub]
    oi = [torch.empty((x.shape[0], k), dtype=torch.int32, device="cuda") for x in sub]
    od = [torch.empty((x.shape[0], k), dtype=torch.float32, device="cuda") for x in sub]
    arr = (acknn.KnnDataset * max(1, done))()
    for i, x in enumerate(sub):
        arr[i].points = xd[i].data_ptr()
        arr[i].n, arr[i].d, arr[i].seed = x.shape[0], x.shape[1], i
        arr[i].out_idx, arr[i].out_dist = oi[i].data_ptr(), od[i].data_ptr()
    ours = {}
    for name, prec in (("plain_fp32", acknn.PREC_FP32), ("mixed", acknn.PREC_BF16_RERANK)):
        def b(prec=prec):
            opt = acknn.default_options(points_on_device=1, outputs_on_device=1, stream=stream.cuda_stream,
                                        precision=prec, autotune=1)
            rc = lib.knn_build_batch(ctx.handle, arr, done, k, T, L, P, 0, ctypes.byref(opt), None)
            if rc:
                raise acknn.KnnError(rc, lib.knn_last_error().decode())
        for _ in range(3):
            b()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            b()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        ours[name] = {"ms": ms, "points_per_s": pts / (ms / 1e3),
                      "recall_mean_of_sets": float(np.mean(ours_rec[name])) if ours_rec[name] else None}
    ctx.close()
    print(json.dumps({"reference_gpu_batch": {
        "sets_run": done, "sets": count, "points": pts, "params": {"k": k, "trees": T, "leaf": L, "props": P},
        "ms_calculate_sum": ref_ms, "process_wall_s": ref_wall,
        "points_per_s_calculate": pts / (ref_ms / 1e3) if ref_ms else None,
        "recall_mean_of_sets": float(np.mean(ref_rec)) if ref_rec else None,
        "recall_min": float(np.min(ref_rec)) if ref_rec else None},
        "ours_batched_same_sets": ours,
        "note": "the sets as CSV in fixed point with 9 decimals, normalised by the reference's rule on both sides"}),
        flush=True)
    return 0


def run_reference_gpu(args, w):
    """The reference's own build on the integer mixture at the configuration's
    literal parameters and at the headline setting (one run each); with
    --workload dataset_batch, the 256-set batch (run_reference_gpu_batch)."""
    import torch

    if args.workload == "dataset_batch":
        return run_reference_gpu_batch(args)
    torch.cuda.set_device(0)
    acknn = load_package()
    acknn.load_library()
    n, k = w["n"], w["k"]
    x = make_points(acknn, n, seed=0)
    rng = np.random.Generator(np.random.PCG64(12345))
    q = np.sort(rng.choice(n, size=min(10_000, n), replace=False)).astype(np.int64)
    ei, _ = acknn.exact_fp64(x, k, q, w["metric"])
    settings = {"literal": CONFIG_PARAMS, "headline": TARGET_PARAMS}
    if args.trees or args.leaf or args.props is not None:
        settings = {"custom": dict(trees=args.trees or 8, leaf=args.leaf or 2048,
                                   props=args.props if args.props is not None else 0)}
    r = reference_gpu_runs(acknn, x, k, q, ei, settings, args.ref_limit)
    print(json.dumps({"reference_gpu": r, "workload": workload_desc(w, TARGET_PARAMS)}), flush=True)
    return 0


# ------------------------------------------------------ sharded single dataset --
def run_sharded(args):
    """One dataset's graph built by all ranks together (sharded.build_sharded:
    trees split by rank, one all-to-all + merge + all-gather of the initial
    lists, propagation by point range with an all-gather per step).  Every
    rank holds the same points; `value` = n / (max over ranks of the device
    time of one build): strong scaling, the total work is fixed."""
    import datetime

    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    acknn = load_package()
    acknn.load_library()
    name = args.workload if args.workload != "dataset_batch" else "normalized_mixture"
    cfg = acknn.workloads.CONFIGS[name]
    n = args.n or cfg["n"]
    k, metric = cfg["k"], cfg["metric"]
    T = args.trees or cfg["trees"]
    L = args.leaf or cfg["leaf"]
    P = args.props if args.props is not None else cfg["props"]
    x = cfg["gen"](0, n=n)
    xd = torch.from_numpy(x).cuda(local)
    prec = acknn.PREC_FP32 if metric == 1 else acknn.PREC_F16_RERANK
    sh = acknn.sharded
    be, comm = sh.LibraryBackend(acknn, local, precision=prec), sh.TorchComm()
    stream = torch.cuda.current_stream(local)

    def build():
        return sh.build_sharded(be, comm, xd, k, T, L, P, metric, 0)

    for _ in range(args.warmup):
        build()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        gi, gd = build()
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1) / args.steps], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    if rank == 0:
        rng = np.random.Generator(np.random.PCG64(12345))
        q = np.sort(rng.choice(n, size=min(10_000, n), replace=False)).astype(np.int64)
        ei, _ = acknn.exact_fp64(x, k, q, metric)
        ai = gi[torch.from_numpy(q).cuda(local)].cpu().numpy()
        rec = sum(len(np.intersect1d(a, b)) for a, b in zip(ai, ei)) / (k * len(q))
        print(json.dumps({
            "metric": "k-NN graph points/s of one dataset built by all ranks", "value": n / (ms / 1e3),
            "unit": "points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f16+f32",
            "data": "synthetic",
            "config": {"workload": f"{name} N={n:,} d={x.shape[1]} {x.dtype}; k={k}, {T} trees, leaf {L}, {P} "
                                   f"propagation(s), {METRIC_NAMES[metric]}", "parallelism": f"sharded x{world}",
                       "exchange_bytes_received_per_rank": int(2 * n * k * 8 + P * n * (k * 8 + 4 * ((k + 31) // 32)))},
            "recall_id": rec}), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


# ------------------------------------------------------- the hello CLI itself --
HELLO_BIN = PKG_DIR / "hello"


def run_cli(args):
    """The drop-in CLI end to end on one configuration written as CSV: wall
    time of the `hello` process and its own split (CSV ingest, normalisation +
    build, binary write; ACKNN_TIMING=1), and recall@k by id from its output
    file against the FP64 exact graph of the points it read, normalised as the
    reference normalises them (10,000 seeded queries)."""
    import re
    import shutil
    import tempfile

    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    acknn.load_library()
    cfg = acknn.workloads.CONFIGS[args.workload]
    n = args.n or cfg["n"]
    k, metric = cfg["k"], cfg["metric"]
    T = args.trees or cfg["trees"]
    L = args.leaf or cfg["leaf"]
    P = args.props if args.props is not None else cfg["props"]
    x = cfg["gen"](0, n=n)
    tmp = Path(tempfile.mkdtemp(prefix="acknn_cli_"))
    try:
        csv = tmp / "points.csv"
        t = time.perf_counter()
        if args.workload == "integer_mixture":
            acknn.formats.write_csv_integers(str(csv), x)
            parsed = x
        elif args.workload == "sparse_prototypes":
            parsed = acknn.formats.write_csv_fixed(str(csv), x)
        else:
            raise SystemExit(f"--cli supports integer_mixture and sparse_prototypes, not {args.workload}")
        write_s = time.perf_counter() - t
        out = tmp / "graph.bin"
        env = dict(os.environ, ACKNN_TIMING="1")
        cmd = [str(HELLO_BIN), str(csv), str(out), str(k), str(T), str(L), str(P), METRIC_NAMES[metric], "0", "F"]
        t = time.perf_counter()
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=1800)
        wall = time.perf_counter() - t
        if r.returncode != 0:
            raise SystemExit(f"hello exited {r.returncode}: {r.stdout[-500:]} {r.stderr[-500:]}")
        tm = dict(re.findall(r"(\w+_ms)=([0-9.]+)", r.stderr))
        thr = re.search(r"threads=(\d+)", r.stderr)
        _, _, ids, _ = acknn.formats.read_result(str(out))
        xn = acknn.normalize_reference(parsed)
        rng = np.random.Generator(np.random.PCG64(12345))
        q = np.sort(rng.choice(n, size=min(10_000, n), replace=False)).astype(np.int64)
        ei, _ = acknn.exact_fp64(xn, k, q, metric)
        rec = sum(len(np.intersect1d(a, b)) for a, b in zip(ids[q], ei)) / (k * len(q))
        line = {"cli": args.workload, "n": n, "d": x.shape[1], "k": k, "trees": T, "leaf": L, "props": P,
                "metric": METRIC_NAMES[metric], "csv_bytes": csv.stat().st_size, "csv_write_s": write_s,
                "hello_wall_s": wall, "load_ms": float(tm.get("load_ms", "nan")),
                "build_ms": float(tm.get("build_ms", "nan")), "write_ms": float(tm.get("write_ms", "nan")),
                "parse_threads": int(thr.group(1)) if thr else None,
                "ingest_gb_per_s": csv.stat().st_size / (float(tm.get("load_ms", "nan")) / 1e3) / 1e9,
                "recall_id": rec, "queries": int(len(q))}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


# ------------------------------------------------------------ setting sweep --
# Grids searched per workload: trees x leaf, and for each pair propagations
# 0..max_props until the recall target is met.
SWEEP_GRIDS = {
    "integer_mixture": dict(trees=[6, 8, 10, 12, 16], leaf=[256, 512, 1024, 2048], max_props=3),
    "sparse_prototypes": dict(trees=[1, 2, 4], leaf=[32768, 131072], max_props=2),
    "normalized_mixture": dict(trees=[8, 12, 16, 24], leaf=[512, 1024, 2048, 4096], max_props=4),
    "dataset_batch": dict(trees=[4, 8, 12], leaf=[48, 128, 256, 512, 1024, 2048], max_props=6),
}


class _SingleRunner:
    """One configuration's points resident in HBM, its FP64 exact graph on
    10,000 seeded queries, and builds of any (path, trees, leaf, props)."""

    def __init__(self, acknn, lib, torch, name: str, n: int | None):
        cfg = acknn.workloads.CONFIGS[name]
        self.acknn, self.lib, self.torch = acknn, lib, torch
        self.n = n or cfg["n"]
        self.k, self.metric = cfg["k"], cfg["metric"]
        self.x = cfg["gen"](0, n=self.n)
        self.d = self.x.shape[1]
        self.dtype = acknn.F16 if self.x.dtype == np.float16 else acknn.F32
        self.xd = torch.from_numpy(self.x).cuda()
        self.idx = torch.empty((self.n, self.k), dtype=torch.int32, device="cuda")
        self.dist = torch.empty((self.n, self.k), dtype=torch.float32, device="cuda")
        self.ctx = acknn.Context(0)
        self.stream = torch.cuda.current_stream()
        rng = np.random.Generator(np.random.PCG64(12345))
        self.q = np.sort(rng.choice(self.n, size=min(10_000, self.n), replace=False)).astype(np.int64)
        self.exact = acknn.exact_fp64(self.x, self.k, self.q, self.metric)
        self.qt = torch.from_numpy(self.q).cuda()
        self.points = self.n

    def build(self, kw: dict, T: int, L: int, P: int, stats=None):
        opt = self.acknn.default_options(points_on_device=1, outputs_on_device=1, dtype=self.dtype,
                                         stream=self.stream.cuda_stream, **kw)
        rc = self.lib.knn_build_ex(self.ctx.handle, self.xd.data_ptr(), self.n, self.d, self.k, T, L, P,
                                   self.metric, 0, self.idx.data_ptr(), self.dist.data_ptr(),
                                   ctypes.byref(opt), ctypes.byref(stats) if stats is not None else None)
        if rc:
            raise self.acknn.KnnError(rc, self.lib.knn_last_error().decode())

    def accuracy(self) -> dict:
        return accuracy(self.acknn, self.x, self.idx[self.qt].cpu().numpy(), self.dist[self.qt].cpu().numpy(),
                        self.k, self.metric, self.exact, self.q, gathered=True)

    def close(self):
        self.ctx.close()


class _BatchRunner:
    """The 256-dataset batch resident in HBM; per-set FP64 exact graphs on up to
    500 seeded queries per set; one knn_build_batch per build."""

    def __init__(self, acknn, lib, torch, count: int | None):
        cfg = acknn.workloads.CONFIGS["dataset_batch"]
        self.acknn, self.lib, self.torch = acknn, lib, torch
        self.count = count or cfg["count"]
        self.k, self.metric = cfg["k"], cfg["metric"]
        self.xs = [acknn.workloads.batch_dataset(s) for s in range(self.count)]
        self.points = sum(x.shape[0] for x in self.xs)
        self.xd = [torch.from_numpy(x).cuda() for x in self.xs]
        self.oi = [torch.empty((x.shape[0], self.k), dtype=torch.int32, device="cuda") for x in self.xs]
        self.od = [torch.empty((x.shape[0], self.k), dtype=torch.float32, device="cuda") for x in self.xs]
        self.ctx = acknn.Context(0)
        self.stream = torch.cuda.current_stream()
        arr = (acknn.KnnDataset * self.count)()
        for i, x in enumerate(self.xs):
            arr[i].points = self.xd[i].data_ptr()
            arr[i].n, arr[i].d, arr[i].seed = x.shape[0], x.shape[1], i
            arr[i].out_idx = self.oi[i].data_ptr()
            arr[i].out_dist = self.od[i].data_ptr()
        self.table = arr
        rng = np.random.Generator(np.random.PCG64(7))
        self.qs, self.exact = [], []
        for x in self.xs:
            q = np.sort(rng.choice(x.shape[0], size=min(500, x.shape[0]), replace=False)).astype(np.int64)
            self.qs.append(q)
            self.exact.append(acknn.exact_fp64(x, self.k, q, self.metric))

    def build(self, kw: dict, T: int, L: int, P: int, stats=None):
        opt = self.acknn.default_options(points_on_device=1, outputs_on_device=1,
                                         stream=self.stream.cuda_stream, autotune=1, **kw)
        rc = self.lib.knn_build_batch(self.ctx.handle, self.table, self.count, self.k, T, L, P, self.metric,
                                      ctypes.byref(opt), ctypes.byref(stats) if stats is not None else None)
        if rc:
            raise self.acknn.KnnError(rc, self.lib.knn_last_error().decode())

    def accuracy(self) -> dict:
        per, hits, total = [], 0, 0
        for i, x in enumerate(self.xs):
            ai = self.oi[i].cpu().numpy()[self.qs[i]]
            ei = self.exact[i][0]
            h = sum(len(np.intersect1d(a, b)) for a, b in zip(ai, ei))
            per.append(h / (self.k * len(ai)))
            hits += h
            total += self.k * len(ai)
        return {"recall": hits / total, "recall_id": hits / total, "recall_min": min(per),
                "recall_mean_of_sets": sum(per) / len(per),
                "sets_below_0.95": int(sum(r < 0.95 for r in per)), "queries": total // self.k}

    def close(self):
        self.ctx.close()


def _sweep_paths(acknn, workload: str, metric: int, n: int) -> dict:
    """Paths compared at equal recall: plain FP32 always; for EUCLIDEAN the
    BF16 and FP16 tensor-core leaf tiles; for COSINE (FP16 data) the FP16
    tiles with and without learned splits."""
    names = ["plain_fp32"]
    if metric == 0:
        names += ["mixed", "mixed_f16"]
    elif metric == 2:
        names += ["mixed_f16"] + (["mixed_f16_learned"] if workload != "dataset_batch" else [])
    paths = {}
    for nm in names:
        kw = dict(PATH_OPTIONS[nm])
        if kw.get("learned_splits"):
            kw["mlp_sample"] = min(n, 1_000_000)
        paths[nm] = kw
    return paths


def run_sweep(args):
    """Cheapest (trees, leaf, propagations) reaching recall@k >= --target per
    path.  For each (trees, leaf), in order of growing leaf work, propagations
    rise from 0 until the target is met; a setting is timed (warm-up build,
    then --steps builds under CUDA events, points resident in HBM) only once
    it meets the target, and a pair is abandoned once an untimed build already
    takes longer than the best timed setting.  One JSON line per tried setting,
    then a summary line per path and the equal-recall ratios."""
    import torch

    torch.cuda.set_device(0)
    acknn = load_package()
    lib = acknn.load_library()
    name = args.workload
    grid = dict(SWEEP_GRIDS[name])
    if args.grid_trees:
        grid["trees"] = [int(v) for v in args.grid_trees.split(",")]
    if args.grid_leaf:
        grid["leaf"] = [int(v) for v in args.grid_leaf.split(",")]
    if args.max_props is not None:
        grid["max_props"] = args.max_props
    if name == "dataset_batch":
        R = _BatchRunner(acknn, lib, torch, args.count)
    else:
        R = _SingleRunner(acknn, lib, torch, name, args.n)
    paths = _sweep_paths(acknn, name, R.metric, R.points)
    if args.paths:
        paths = {p: paths[p] for p in args.paths.split(",")}
    stream = R.stream

    def timed(fn, steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    pairs = sorted(((T, L) for T in grid["trees"] for L in grid["leaf"]), key=lambda tl: (tl[0] * tl[1], tl[0]))
    summary = {}
    for pname, kw in paths.items():
        best = None
        top = None  # highest recall seen, for a path that never meets the target
        for T, L in pairs:
            for P in range(grid["max_props"] + 1):
                t0 = time.perf_counter()
                try:
                    R.build(kw, T, L, P)
                    torch.cuda.synchronize()
                except acknn.KnnError as e:
                    print(json.dumps({"trial": pname, "trees": T, "leaf": L, "props": P, "error": str(e)}),
                          flush=True)
                    break
                wall_ms = (time.perf_counter() - t0) * 1e3
                acc = R.accuracy()
                rec = acc["recall"]
                row = {"trial": pname, "trees": T, "leaf": L, "props": P, "recall": rec, "wall_ms_untimed": wall_ms}
                if top is None or rec > top["recall"]:
                    top = dict(row)
                if rec >= args.target:
                    R.build(kw, T, L, P)
                    ms = timed(lambda: R.build(kw, T, L, P), args.steps)
                    st = acknn.KnnStats()
                    st.struct_size = ctypes.sizeof(acknn.KnnStats)
                    R.build(kw, T, L, P, stats=st)
                    torch.cuda.synchronize()
                    sd = st.as_dict()
                    row.update(ms=ms, points_per_s=R.points / (ms / 1e3), accuracy=acc,
                               stages_ms={kk: sd[kk] for kk in ("ms_learn", "ms_trees", "ms_leaf", "ms_propagate")},
                               prop_candidates=sd["prop_candidates"], leaf_path=sd["leaf_path"])
                    print(json.dumps(row), flush=True)
                    if best is None or ms < best["ms"]:
                        best = row
                    break
                print(json.dumps(row), flush=True)
                if best is not None and wall_ms > 1.5 * best["ms"]:
                    break
        summary[pname] = best if best is not None else {"target_not_met": True, "best_recall_seen": top}
    out = {"sweep": name, "target": args.target, "points": R.points, "k": R.k,
           "metric": METRIC_NAMES[R.metric], "grid": grid, "steps": args.steps, "cheapest": summary}
    if "plain_fp32" in summary and summary["plain_fp32"].get("ms"):
        for pname, row in summary.items():
            if pname != "plain_fp32" and row.get("ms"):
                out[f"{pname}_vs_plain_at_equal_recall"] = summary["plain_fp32"]["ms"] / row["ms"]
    print(json.dumps(out), flush=True)
    R.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n", type=int, default=None, help="override N (smaller runs)")
    ap.add_argument("--cpu-sample", type=int, default=20_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["integer_mixture", "dataset_batch", "sparse_prototypes",
                                           "normalized_mixture"], default="integer_mixture")
    ap.add_argument("--count", type=int, default=None, help="datasets in the batch workload")
    ap.add_argument("--single", choices=["mixed", "mixed_f16", "plain"], default=None,
                    help="time one configuration only (the profiling case)")
    ap.add_argument("--trees", type=int, default=None)
    ap.add_argument("--leaf", type=int, default=None)
    ap.add_argument("--props", type=int, default=None)
    ap.add_argument("--sweep", action="store_true",
                    help="search the cheapest setting reaching --target recall per path")
    ap.add_argument("--target", type=float, default=0.95)
    ap.add_argument("--grid-trees", default=None, help="comma-separated trees to sweep")
    ap.add_argument("--grid-leaf", default=None, help="comma-separated leaf sizes to sweep")
    ap.add_argument("--max-props", type=int, default=None)
    ap.add_argument("--paths", default=None, help="comma-separated paths to sweep")
    ap.add_argument("--ab-sparse", action="store_true",
                    help="configurations: also time the plain target with sparse-row leaf tiles off")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="time the reference's own sm_100a build (oracle/_ref/hello) on the workload")
    ap.add_argument("--ref-limit", type=float, default=300.0, help="seconds per reference run")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own build in the default run")
    ap.add_argument("--reference-gpu-headline-only", action="store_true",
                    help="run the reference's own build at the headline setting only (not also the literal one)")
    ap.add_argument("--sharded", action="store_true",
                    help="one dataset built by all ranks together (strong scaling; launch with torchrun for N > 1)")
    ap.add_argument("--cli", action="store_true",
                    help="time the hello CLI end to end (CSV ingest, build, binary write) on the workload")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    w = dict(WORKLOAD)
    if args.n:
        w["n"] = args.n
    if args.impl == "reference":
        return run_reference(args, w)
    if args.sweep:
        return run_sweep(args)
    if args.reference_gpu:
        return run_reference_gpu(args, w)
    if args.cli:
        return run_cli(args)
    if args.sharded:
        return run_sharded(args)
    if args.workload == "dataset_batch":
        return run_batch(args)
    if args.single:
        return run_single(args, w)
    if args.workload in ("sparse_prototypes", "normalized_mixture"):
        return run_config(args)
    return run_ours(args, w)


if __name__ == "__main__":
    sys.exit(main())

"""Benchmark: kriged cells/s on one B200 — FP32-refined (headline) vs FP64 plain.

Workload (default): ordinary kriging on the 256x256x128 grid (8.4M cells), 1%
seeded conditioning cells with lognormal(0, 0.5) values, exponential model
ranges (30,15,6) azimuth 30, nugget 0.05, radiuses (30,15,6), max_neighbours 32
(geo_bsd.workloads.sk_ok_large; synthetic, no dataset).

A step is one whole-grid kriging call through the engine's C ABI
(hpgl_b200_cont_kriging_ex): neighbour search + per-cell solves + estimate and
variance for every uninformed cell. `value` has the inputs resident in HBM
(device pointers, CUDA events on the launching stream); `e2e` repeats the call
with pinned HOST buffers, so each step includes the host->device copy of data
and mask and the device->host copy of estimate, mask and variance.

`--kind sk|lvm` runs simple kriging or kriging with a locally varying mean
(a smooth trend, geo_bsd.workloads.lvm_means) on the same grid instead;
`--kind cok` times simple collocated cokriging (Markov model I, k=32) of that
grid with a correlated secondary field informed on half of the cells, against
the reference's own single-threaded hpgl_simple_cokriging_mark1 on a smaller
grid of the same generator; `--kind sgs` times sequential Gaussian simulation (SK, k=32, seed 42) of every
uninformed cell of that grid, against the reference's own single-threaded
hpgl_sgs_simulation on a smaller grid of the same generator; `--kind sis` times
sequential indicator simulation (5 categories, k=24, seed 42) of the 200x200x100
indicator grid (geo_bsd.workloads.indicator) against the reference's own
single-threaded hpgl_sis_simulation on a smaller grid of that generator.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
For N > 1 the driver runs it under torchrun; every rank runs its own replica
(cells are independent given the conditioning data, so no collective is on the
data path) and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hpgl-reborn_b200"))

METRIC = "kriged cells/s, 1 B200: FP32-refined vs FP64 plain at <=1e-6 rel err"
UNIT = "cells/s"


def rank_max(dist, x, device):
    """Maximum of x over all ranks (x itself without a process group): a
    step's device time is the slowest rank's."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms):
    """Units per second of the whole job: every rank processes
    units_per_rank (independent replicas) and the job takes the slowest
    rank's ms."""
    return units_per_rank * world / (ms / 1e3)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="sk_ok_large")
    ap.add_argument("--kind", choices=["ok", "sk", "lvm", "sgs", "cok", "sis"], default="ok")
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--skip-configs", action="store_true",
                    help="leave out the other benchmark configurations (100x100x50, clustered 512x512x64, "
                         "indicator 200x200x100, leave-one-out 200x200x50)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--profile-case", type=float, default=0.0, metavar="SCALE",
                    help="run one device call on the workload shrunk by SCALE and exit "
                         "(the case profiled with ncu)")
    ap.add_argument("--profile-precision", choices=["fp32_refined", "fp64"], default="fp32_refined",
                    help="precision of the --profile-case call")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workloads_module():
    """geo_bsd/workloads.py loaded by file path: the seeded generators without
    importing the geo_bsd package (whose import loads the engine library), so
    the reference arm never maps the product library."""
    name = "hb_bench_workloads"
    if name in sys.modules:
        return sys.modules[name]
    import importlib.util
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "hpgl-reborn_b200", "geo_bsd",
                                                                     "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workload(name):
    return workloads_module().ALL[name](1.0)


def lvm_means(wl):
    return workloads_module().lvm_means(wl.dims)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


KIND_NAMES = {"ok": "ordinary kriging", "sk": "simple kriging", "lvm": "LVM kriging (smooth trend mean)"}


# ---------------------------------------------------------------- CPU baseline
def z_slab(wl, z0, nz):
    """Layers z0 .. z0+nz-1 of a workload as a grid of their own (the slab's
    own conditioning cells; x fastest, so a slab is a contiguous range)."""
    nx, ny, _ = wl.dims
    a, b = nx * ny * z0, nx * ny * (z0 + nz)
    return (nx, ny, nz), np.ascontiguousarray(wl.data[a:b]), np.ascontiguousarray(wl.mask[a:b])


def ref_api_slab(wl, kind, nz, threads):
    """One whole call of the reference library's own public entry point
    (hpgl_ordinary_kriging / hpgl_simple_kriging from oracle/_ref/libhpgl.so,
    built from the reference's sources: the call geo.ordinary_kriging /
    simple_kriging make), lookup construction included, on the middle nz
    layers of the workload at `threads` OpenMP threads. Returns (kriged
    cells/s, info)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    z0 = max(0, wl.dims[2] // 2 - nz // 2)
    dims, data, mask = z_slab(wl, z0, nz)
    t0 = time.perf_counter()
    _, om = O.ref_cont_api(0 if kind == "ok" else 1, dims, data, mask, wl.cov, wl.radiuses, wl.max_neighbours,
                           threads=threads)
    dt = time.perf_counter() - t0
    kriged = int(((om == 1) & (mask == 0)).sum())
    return kriged / dt, {"slab": f"layers {z0}..{z0 + nz - 1} of z as a {dims[0]}x{dims[1]}x{nz} grid",
                         "kriged_cells": kriged, "seconds": dt, "threads": threads}


def slab_layers(wl, kind, target_seconds, threads):
    """Layers of a slab that one reference call finishes in about
    `target_seconds` (from a 2-layer probe)."""
    rate, _ = ref_api_slab(wl, kind, 2, threads)
    per_layer = wl.dims[0] * wl.dims[1]
    return int(max(2, min(wl.dims[2], round(rate * target_seconds / per_layer))))


def cpu_baseline_api(wl, kind, target_seconds):
    """cpu_baseline of the reference library's own entry point: all host
    threads on a slab of about `target_seconds`, and one thread on 2 layers."""
    threads = os.cpu_count() or 1
    nz = slab_layers(wl, kind, target_seconds, threads)
    v, info = ref_api_slab(wl, kind, nz, threads)
    v1, info1 = ref_api_slab(wl, kind, 2, 1)
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"one whole hpgl_{'ordinary' if kind == 'ok' else 'simple'}_kriging call of the reference "
                      f"library ({info['slab']}, {info['kriged_cells']} kriged cells, {info['seconds']:.2f} s, "
                      f"lookup construction included)",
            "value_1_thread": v1, "sample_1_thread": f"{info1['slab']}, {info1['seconds']:.2f} s",
            "cpu_model": cpu_model()}


def cpu_reference(wl, kind, target_seconds, threads):
    """Reference CPU path (oracle/_ref, the reference's own code) on a sample of
    uninformed cells; falls back to the CPU restatement if the reference build
    is absent. Returns (cells/s, dict)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    which = "ref" if O.available("ref") else "port"
    unk = np.flatnonzero(wl.mask == 0)
    rng = np.random.default_rng(123)
    k = 0 if kind == "ok" else 1
    mean = float(wl.data[wl.mask == 1].astype(np.float64).mean()) if kind == "sk" else 0.0
    means = lvm_means(wl) if kind == "lvm" else None

    def timed(nodes):
        t0 = time.perf_counter()
        O.krige_nodes(which, k, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours, mean=mean,
                      nodes=nodes, threads=threads, want_idx=False, means=means)
        return time.perf_counter() - t0

    setup = timed(np.zeros(0, np.int32))  # template + clusterizer construction only
    probe = np.sort(rng.choice(unk, min(4000, len(unk)), replace=False)).astype(np.int32)
    t_probe = max(timed(probe) - setup, 1e-3)
    rate = len(probe) / t_probe
    n = int(min(len(unk), max(len(probe), rate * target_seconds)))
    sample = np.sort(rng.choice(unk, n, replace=False)).astype(np.int32)
    t = timed(sample) - setup
    return n / t, {"which": which, "sample_cells": n, "seconds": t, "setup_seconds": setup, "threads": threads}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------- engine runs
def peak_table():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = {}
    if os.path.exists(path):
        with open(path) as f:
            peaks = json.load(f)
    mhz = peaks.get("sm_max_mhz", 1965.0)
    src = "measured sm_max_mhz" if "sm_max_mhz" in peaks else "fallback 1965 MHz"
    # CUDA-core peaks: 148 SMs x (128 FP32 | 64 FP64) lanes x 2 flop/FMA x clock
    return {"fp32": 148 * 128 * 2 * mhz * 1e6 / 1e12, "fp64": 148 * 64 * 2 * mhz * 1e6 / 1e12,
            "hbm_gbs": peaks.get("hbm_gbs", 6650.0), "source": src}


def traffic_per_cell():
    """DRAM bytes per kriged cell of the dominant solve kernel from the committed
    ncu summary (profiles/solve_kernel_traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "solve_kernel_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_cell")


SGS_METRIC = "simulated cells/s, 1 B200: sequential Gaussian simulation (SK, k=32)"
SGS_SEED = 42


def sgs_workload(scale):
    WL = workloads_module()
    wl = WL.sk_ok_large(scale)
    cov = WL.CovSpec(wl.cov.cov_type, wl.cov.ranges, wl.cov.angles, 1.0, wl.cov.nugget / wl.cov.sill)
    return wl, cov


def sgs_reference(target_seconds):
    """The reference's own SGS (oracle/_ref/libhpgl.so, single-threaded as it is)
    on a grid of the same generator sized for about target_seconds; returns
    (cells/s, info)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    wl, cov = sgs_workload(0.25)
    t0 = time.perf_counter()
    O.ref_sgs(wl.dims, wl.data, wl.mask, cov, wl.radiuses, wl.max_neighbours, SGS_SEED)
    rate = int((wl.mask == 0).sum()) / max(time.perf_counter() - t0, 1e-3)
    scale = min(1.0, max(0.25, (rate * target_seconds / (256 * 256 * 128)) ** (1.0 / 3.0)))
    wl, cov = sgs_workload(scale)
    t0 = time.perf_counter()
    O.ref_sgs(wl.dims, wl.data, wl.mask, cov, wl.radiuses, wl.max_neighbours, SGS_SEED)
    dt = time.perf_counter() - t0
    cells = int((wl.mask == 0).sum())
    return cells / dt, {"dims": wl.dims, "cells": cells, "seconds": dt}


def bench_sgs(args, rank, world, local):
    import torch
    if args.impl == "reference":
        if rank == 0:
            vals, info = [], None
            for i in range(args.warmup + args.steps):
                v, info = sgs_reference(min(args.cpu_seconds, 2.0))
                if i >= args.warmup:
                    vals.append(v)
            value = float(np.median(vals))
            d = "x".join(str(x) for x in info["dims"])
            print(json.dumps({"impl": "reference", "metric": SGS_METRIC, "value": value, "unit": UNIT,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded, geo_bsd.workloads)",
                              "config": {"workload": f"SGS SK k=32 seed {SGS_SEED}, grid {d} of the 256x256x128 "
                                                     "generator (1% lognormal conditioning, exponential (30,15,6))"},
                              "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                                               "sample": f"whole simulation of a {d} grid ({info['cells']} cells) "
                                                         "per step; the reference's SGS is single-threaded"},
                              "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    from geo_bsd import hpgl_wrap as W
    wl, cov = sgs_workload(args.profile_case if args.profile_case > 0 else 1.0)
    n = wl.n_cells
    dev = torch.device("cuda", local)
    d_data0 = torch.from_numpy(np.ascontiguousarray(wl.data)).to(dev)
    d_mask0 = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
    d_data = d_data0.clone()
    d_mask = d_mask0.clone()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    dims = (C.c_int * 3)(*wl.dims)
    p = W._HPGL_SGS_PARAMS(covariance_type=cov.cov_type, ranges=cov.ranges, angles=cov.angles, sill=cov.sill,
                           nugget=cov.nugget, radiuses=wl.radiuses, max_neighbours=wl.max_neighbours, kriging_kind=1,
                           seed=SGS_SEED, min_neighbours=0)

    def dev_call():
        o = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=W.FLAG_DEVICE_POINTERS, stream=stream.cuda_stream,
                                 estimate64=None, variance=None, status=None, ik_probs=None)
        rc = W._hpgl_so.hpgl_b200_sgs_ex(dims, d_data.data_ptr(), d_mask.data_ptr(), None, None, None, C.byref(p),
                                         C.byref(o))
        W.check(rc, "sgs_ex")
        return W.last_stats()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(dist, x, dev)

    def restore():
        d_data.copy_(d_data0)
        d_mask.copy_(d_mask0)

    if args.profile_case > 0:
        st = dev_call()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": wl.dims, "stats": st}), flush=True)
        return
    for _ in range(args.warmup):
        restore()
        dev_call()
    times, stats = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            restore()
            flush.zero_()  # L2 flush between steps (outside the timed region)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = dev_call()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
    barrier()
    ms = max_over_ranks(float(np.mean(times)))
    last = stats[-1]
    cells = last["kriged_cells"]
    value = cells * world / (ms / 1e3)
    pk = peak_table()
    solve_ms = float(np.mean([s["stage_solve_ms"] for s in stats]))
    achieved = last["sgs_flops"] / (solve_ms / 1e3) / 1e12
    roofline = {"bound": "fp64", "kernel": "k_sgs_solve_fold<simple> (FP64, two nodes per warp, one launch per level)",
                "achieved": achieved, "peak": pk["fp64"], "unit": "TFLOP/s", "frac": achieved / pk["fp64"],
                "traffic": None, "peak_source": f"CUDA-core FP64 peak 148 SM x 64 lanes x 2 x {pk['source']}",
                "algorithmic_flops_per_call": last["sgs_flops"], "solve_stage_ms": solve_ms,
                "levels": last["sgs_levels"]}

    # end to end with pinned host buffers (data and mask in, simulated data and mask out)
    lib = W._hpgl_so
    h_data = lib.hpgl_b200_host_alloc(n * 4)
    h_mask = lib.hpgl_b200_host_alloc(n)
    src_d = np.ascontiguousarray(wl.data)
    src_m = np.ascontiguousarray(wl.mask)

    def host_call():
        C.memmove(h_data, src_d.ctypes.data, n * 4)
        C.memmove(h_mask, src_m.ctypes.data, n)
        o = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                                 status=None, ik_probs=None)
        t0 = time.perf_counter()
        rc = lib.hpgl_b200_sgs_ex(dims, h_data, h_mask, None, None, None, C.byref(p), C.byref(o))
        dt = time.perf_counter() - t0
        W.check(rc, "sgs_ex (host)")
        return dt, W.last_stats()

    for _ in range(args.warmup):
        host_call()
    e2e_t = []
    for _ in range(args.steps):
        barrier()
        dt, st = host_call()
        e2e_t.append(dt)
    barrier()
    e2e_s = max_over_ranks(float(np.mean(e2e_t)))
    e2e_value = st["kriged_cells"] * world / e2e_s
    lib.hpgl_b200_host_free(h_data)
    lib.hpgl_b200_host_free(h_mask)
    cpu = None
    if rank == 0 and not args.skip_cpu_baseline:
        v, info = sgs_reference(args.cpu_seconds)
        d = "x".join(str(x) for x in info["dims"])
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
               "sample": f"the reference's hpgl_sgs_simulation of a {d} grid of the same generator "
                         f"({info['cells']} cells, {info['seconds']:.1f} s); single-threaded as the reference is"}
    if rank == 0:
        print(json.dumps({
            "metric": SGS_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, geo_bsd.workloads)",
            "config": {"workload": f"SGS SK {wl.dims[0]}x{wl.dims[1]}x{wl.dims[2]}, 1% lognormal conditioning, "
                                   f"exponential (30,15,6) az 30 (sill-normalised), k={wl.max_neighbours}, "
                                   f"seed {SGS_SEED}", "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "stages_ms": {k[len("stage_"):-len("_ms")]: round(v, 3) for k, v in last.items() if k.startswith("stage_")},
            "host_draws_ms": last["sgs_draws_ms"],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(st["h2d_bytes"]),
                    "d2h_bytes_per_step": int(st["d2h_bytes"]), "timing": "wall clock per call"},
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "clocks": clk.summary(),
        }), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


SIS_METRIC = "simulated cells/s, 1 B200: sequential indicator simulation (5 categories, k=24)"
SIS_SEED = 42


def sis_workload(scale):
    WL = workloads_module()
    wl = WL.indicator(scale)
    data = np.where(wl.mask == 1, wl.data, 0).astype(np.uint8)
    return wl, data


def sis_reference(target_seconds):
    """The reference's own SIS (oracle/_ref/libhpgl.so, single-threaded as it is)
    on a grid of the same generator sized for about target_seconds; returns
    (cells/s, info)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    def run(scale):
        wl, data = sis_workload(scale)
        ks = [wl.max_neighbours] * wl.categories
        t0 = time.perf_counter()
        O.ref_sis(wl.dims, data, wl.mask, wl.cat_covs, wl.cat_radiuses, ks, wl.marginals, SIS_SEED)
        return wl, time.perf_counter() - t0

    wl, dt = run(0.2)
    rate = int((wl.mask == 0).sum()) / max(dt, 1e-3)
    scale = min(1.0, max(0.2, (rate * target_seconds / (200 * 200 * 100)) ** (1.0 / 3.0)))
    wl, dt = run(scale)
    cells = int((wl.mask == 0).sum())
    return cells / dt, {"dims": wl.dims, "cells": cells, "seconds": dt}


def bench_sis(args, rank, world, local):
    import torch
    if args.impl == "reference":
        if rank == 0:
            vals, info = [], None
            for i in range(args.warmup + args.steps):
                v, info = sis_reference(min(args.cpu_seconds, 2.0))
                if i >= args.warmup:
                    vals.append(v)
            value = float(np.median(vals))
            d = "x".join(str(x) for x in info["dims"])
            print(json.dumps({"impl": "reference", "metric": SIS_METRIC, "value": value, "unit": UNIT,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded, geo_bsd.workloads)",
                              "config": {"workload": f"SIS 5 categories k=24 seed {SIS_SEED}, grid {d} of the "
                                                     "200x200x100 indicator generator (1.5% conditioning)"},
                              "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                                               "sample": f"whole simulation of a {d} grid ({info['cells']} cells) "
                                                         "per step; the reference's SIS is single-threaded"},
                              "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    from geo_bsd import hpgl_wrap as W
    wl, data = sis_workload(args.profile_case if args.profile_case > 0 else 1.0)
    n = wl.n_cells
    m = wl.categories
    dev = torch.device("cuda", local)
    d_data0 = torch.from_numpy(np.ascontiguousarray(data)).to(dev)
    d_mask0 = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
    d_data = d_data0.clone()
    d_mask = d_mask0.clone()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    dims = (C.c_int * 3)(*wl.dims)
    params = (W._HPGL_IK_PARAMS * m)()
    for i, c in enumerate(wl.cat_covs):
        params[i] = W._HPGL_IK_PARAMS(covariance_type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill,
                                      nugget=c.nugget, radiuses=wl.cat_radiuses[i], max_neighbours=wl.max_neighbours,
                                      marginal_prob=wl.marginals[i])

    def dev_call():
        o = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=W.FLAG_DEVICE_POINTERS, stream=stream.cuda_stream,
                                 estimate64=None, variance=None, status=None, ik_probs=None)
        rc = W._hpgl_so.hpgl_b200_sis_ex(dims, d_data.data_ptr(), d_mask.data_ptr(), None, params, m, None, SIS_SEED,
                                         0, C.byref(o))
        W.check(rc, "sis_ex")
        return W.last_stats()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(dist, x, dev)

    def restore():
        d_data.copy_(d_data0)
        d_mask.copy_(d_mask0)

    if args.profile_case > 0:
        st = dev_call()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": wl.dims, "stats": st}), flush=True)
        return
    for _ in range(args.warmup):
        restore()
        dev_call()
    times, stats = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            restore()
            flush.zero_()  # L2 flush between steps (outside the timed region)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = dev_call()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
    barrier()
    ms = max_over_ranks(float(np.mean(times)))
    last = stats[-1]
    cells = last["kriged_cells"]
    value = cells * world / (ms / 1e3)
    pk = peak_table()
    solve_ms = float(np.mean([s["stage_solve_ms"] for s in stats]))
    achieved = last["sgs_flops"] / (solve_ms / 1e3) / 1e12
    roofline = {"bound": "fp64", "kernel": "k_sis_level (FP64, two systems per warp, every category of a level "
                                            "in one launch, the node's last system draws)",
                "achieved": achieved, "peak": pk["fp64"], "unit": "TFLOP/s", "frac": achieved / pk["fp64"],
                "traffic": None, "peak_source": f"CUDA-core FP64 peak 148 SM x 64 lanes x 2 x {pk['source']}",
                "algorithmic_flops_per_call": last["sgs_flops"], "solve_stage_ms": solve_ms,
                "levels": last["sgs_levels"]}

    # end to end with pinned host buffers (categories and mask in, simulated categories and mask out)
    lib = W._hpgl_so
    h_data = lib.hpgl_b200_host_alloc(n)
    h_mask = lib.hpgl_b200_host_alloc(n)
    src_d = np.ascontiguousarray(data)
    src_m = np.ascontiguousarray(wl.mask)

    def host_call():
        C.memmove(h_data, src_d.ctypes.data, n)
        C.memmove(h_mask, src_m.ctypes.data, n)
        o = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                                 status=None, ik_probs=None)
        t0 = time.perf_counter()
        rc = lib.hpgl_b200_sis_ex(dims, h_data, h_mask, None, params, m, None, SIS_SEED, 0, C.byref(o))
        dt = time.perf_counter() - t0
        W.check(rc, "sis_ex (host)")
        return dt, W.last_stats()

    for _ in range(args.warmup):
        host_call()
    e2e_t = []
    for _ in range(args.steps):
        barrier()
        dt, st = host_call()
        e2e_t.append(dt)
    barrier()
    e2e_s = max_over_ranks(float(np.mean(e2e_t)))
    e2e_value = st["kriged_cells"] * world / e2e_s
    lib.hpgl_b200_host_free(h_data)
    lib.hpgl_b200_host_free(h_mask)
    cpu = None
    if rank == 0 and not args.skip_cpu_baseline:
        v, info = sis_reference(args.cpu_seconds)
        d = "x".join(str(x) for x in info["dims"])
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
               "sample": f"the reference's hpgl_sis_simulation of a {d} grid of the same generator "
                         f"({info['cells']} cells, {info['seconds']:.1f} s); single-threaded as the reference is"}
    if rank == 0:
        print(json.dumps({
            "metric": SIS_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, geo_bsd.workloads)",
            "config": {"workload": f"SIS {wl.dims[0]}x{wl.dims[1]}x{wl.dims[2]}, 1.5% conditioning, 5 categories "
                                   f"(spherical, ranges 12-25), k={wl.max_neighbours} per category, seed {SIS_SEED}",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "stages_ms": {k[len("stage_"):-len("_ms")]: round(v, 3) for k, v in last.items() if k.startswith("stage_")},
            "host_draws_ms": last["sgs_draws_ms"],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(st["h2d_bytes"]),
                    "d2h_bytes_per_step": int(st["d2h_bytes"]), "timing": "wall clock per call"},
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "clocks": clk.summary(),
        }), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


COK_METRIC = "cokriged cells/s, 1 B200: simple collocated cokriging, Markov model I (k=32)"


def cok_workload(scale):
    """The kriging grid's generator with a secondary field: 0.6 x the primary
    values plus seeded N(0,1) noise, informed on half of the cells."""
    WL = workloads_module()
    wl = WL.sk_ok_large(scale)
    rng = np.random.default_rng(4)
    sdata = (0.6 * np.where(wl.mask == 1, wl.data, 0) + rng.normal(size=wl.n_cells)).astype(np.float32)
    smask = (rng.random(wl.n_cells) < 0.5).astype(np.uint8)
    pm = float(wl.data[wl.mask == 1].astype(np.float64).mean())
    sm = float(sdata[smask == 1].astype(np.float64).mean())
    return wl, sdata, smask, pm, sm


def cok_reference(target_seconds):
    """The reference's own cokriging (oracle/_ref/libhpgl.so, single-threaded as
    it is) on a grid of the same generator sized for about target_seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    def run(scale):
        wl, sd, smk, pm, sm = cok_workload(scale)
        t0 = time.perf_counter()
        O.ref_cokriging_mark1(wl.dims, wl.data, wl.mask, sd, smk, wl.cov, wl.radiuses, wl.max_neighbours, pm, sm,
                              0.9, 0.6)
        return wl, time.perf_counter() - t0

    wl, dt = run(0.12)
    rate = int((wl.mask == 0).sum()) / max(dt, 1e-3)
    scale = min(1.0, max(0.12, (rate * target_seconds / (256 * 256 * 128)) ** (1.0 / 3.0)))
    wl, dt = run(scale)
    cells = int((wl.mask == 0).sum())
    return cells / dt, {"dims": wl.dims, "cells": cells, "seconds": dt}


def bench_cok(args, rank, world, local):
    import torch
    if args.impl == "reference":
        if rank == 0:
            vals, info = [], None
            for i in range(args.warmup + args.steps):
                v, info = cok_reference(min(args.cpu_seconds, 2.0))
                if i >= args.warmup:
                    vals.append(v)
            value = float(np.median(vals))
            d = "x".join(str(x) for x in info["dims"])
            print(json.dumps({"impl": "reference", "metric": COK_METRIC, "value": value, "unit": UNIT,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded, geo_bsd.workloads)",
                              "config": {"workload": f"cokriging Markov I k=32 on a {d} grid of the 256x256x128 "
                                                     "generator"},
                              "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                                               "sample": f"whole {d} grid ({info['cells']} cells) per step; the "
                                                         "reference's cokriging is single-threaded"},
                              "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    from geo_bsd import hpgl_wrap as W
    wl, sdata, smask, pm, sm = cok_workload(args.profile_case if args.profile_case > 0 else 1.0)
    n = wl.n_cells
    dev = torch.device("cuda", local)
    arrays = [torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (wl.data, wl.mask, sdata, smask)]
    d_out = torch.empty(n, dtype=torch.float32, device=dev)
    d_om = torch.empty(n, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    dims = (C.c_int * 3)(*wl.dims)
    c = wl.cov
    p = W._HPGL_COK_M1_PARAMS(covariance_type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill,
                              nugget=c.nugget, radiuses=wl.radiuses, max_neighbours=wl.max_neighbours,
                              primary_mean=pm, secondary_mean=sm, secondary_variance=0.9, correlation_coef=0.6)

    def call(ptrs, out, om, flags, strm):
        o = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=flags, stream=strm, estimate64=None,
                                 variance=None, status=None, ik_probs=None)
        rc = W._hpgl_so.hpgl_b200_cokriging_ex(1, dims, *ptrs, C.byref(p), None, out, om, C.byref(o))
        W.check(rc, "cokriging_ex")
        return W.last_stats()

    def dev_call():
        return call([a.data_ptr() for a in arrays], d_out.data_ptr(), d_om.data_ptr(), W.FLAG_DEVICE_POINTERS,
                    stream.cuda_stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(dist, x, dev)

    if args.profile_case > 0:
        st = dev_call()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": wl.dims, "stats": st}), flush=True)
        return
    for _ in range(args.warmup):
        dev_call()
    times, stats = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = dev_call()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
    barrier()
    ms = max_over_ranks(float(np.mean(times)))
    last = stats[-1]
    value = last["kriged_cells"] * world / (ms / 1e3)
    # end to end with pinned host buffers
    lib = W._hpgl_so
    sizes = (n * 4, n, n * 4, n, n * 4, n)
    h = [lib.hpgl_b200_host_alloc(sz) for sz in sizes]
    for ptr, src, sz in zip(h[:4], (wl.data, wl.mask, sdata, smask), sizes[:4]):
        C.memmove(ptr, np.ascontiguousarray(src).ctypes.data, sz)
    for _ in range(args.warmup):
        call(h[:4], h[4], h[5], 0, None)
    e2e_t = []
    for _ in range(args.steps):
        barrier()
        t0 = time.perf_counter()
        st = call(h[:4], h[4], h[5], 0, None)
        e2e_t.append(time.perf_counter() - t0)
    barrier()
    e2e_value = st["kriged_cells"] * world / max_over_ranks(float(np.mean(e2e_t)))
    for ptr in h:
        lib.hpgl_b200_host_free(ptr)
    cpu = None
    if rank == 0 and not args.skip_cpu_baseline:
        v, info = cok_reference(args.cpu_seconds)
        d = "x".join(str(x) for x in info["dims"])
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
               "sample": f"the reference's hpgl_simple_cokriging_mark1 of a {d} grid of the same generator "
                         f"({info['cells']} cells, {info['seconds']:.1f} s); single-threaded as the reference is"}
    if rank == 0:
        print(json.dumps({
            "metric": COK_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, geo_bsd.workloads)",
            "config": {"workload": f"cokriging Markov I {wl.dims[0]}x{wl.dims[1]}x{wl.dims[2]}, 1% lognormal "
                                   f"conditioning, exponential (30,15,6) az 30, secondary 0.6 x primary + N(0,1) "
                                   f"on half the cells, rho 0.6, k={wl.max_neighbours}",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "stages_ms": {k[len("stage_"):-len("_ms")]: round(v, 3) for k, v in last.items() if k.startswith("stage_")},
            "search": {"prefilter": bool(last["prefilter_active"]), "exact_cells": int(last["prefilter_exact_cells"])},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(st["h2d_bytes"]),
                    "d2h_bytes_per_step": int(st["d2h_bytes"]), "timing": "wall clock per call"},
            "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
            "clocks": clk.summary(),
        }), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def bucket_kernel(W, b, cov_type, precision, ordinary):
    """Name of the solve kernel that ran bucket b (0..4) for this key."""
    if b == 4:
        return "k_solve_large (n > 64, one block per system, FP64)"
    np_ = [8, 16, 32, 64][b]
    v = W.solve_variant(np_, cov_type, precision) if hasattr(W, "solve_variant") else 1
    kind = "ordinary" if ordinary else "simple"
    if np_ == 64 and v in (getattr(W, "VARIANT_WIDE", -1), W.VARIANT_DEFAULT):
        th, pr = (256, "FP64 plain") if precision == 0 else (256, "FP32 refined")
        return f"k_solve_wide{64 if precision == 0 else 32}<{kind}, {th}> ({pr}, one warp per system, rolled phases)"
    if precision == 0:
        th = 384 if (np_ <= 32 and v == W.VARIANT_FOLD) else 256
        return f"k_solve_fold64<NP={np_}, {kind}, {th}> (FP64 plain, NP/2 lanes per system)"
    if np_ == 32 and v in (getattr(W, "VARIANT_TILE", -1), getattr(W, "VARIANT_TILE_NARROW", -1)):
        th = 384 if v == W.VARIANT_TILE else 192
        return f"k_solve_tile<NP=32, {kind}, {th}> (FP32 refined, union tiles of {th // 8} systems, NP/4 lanes per system)"
    if np_ <= 32 and v in (W.VARIANT_QUAD, W.VARIANT_QUAD_NARROW):
        th = 384 if v == W.VARIANT_QUAD else 256
        return f"k_solve_quad<NP={np_}, {kind}, {th}> (FP32 refined, NP/4 lanes per system)"
    th = 512 if (np_ <= 32 and v == W.VARIANT_FOLD) else 256
    return f"k_solve_fold<NP={np_}, {kind}, {th}> (FP32 refined, NP/2 lanes per system)"


def solve_roofline(W, stats_list, cov_type, precision, ordinary, pk):
    """Dominant solve kernel of a run (the bucket with the largest time) and its
    algorithmic rate against the derived CUDA-core peak of the precision."""
    last = stats_list[-1]
    b = int(np.argmax([last[f"bucket_ms_{i}"] for i in range(5)]))
    ms = float(np.mean([s[f"bucket_ms_{b}"] for s in stats_list]))
    flops = last[f"bucket_flops_{b}"]
    tf = flops / (ms / 1e3) / 1e12 if ms > 0 else 0.0
    peak = pk["fp32"] if precision else pk["fp64"]
    return {"kernel": bucket_kernel(W, b, cov_type, precision, ordinary), "kernel_ms": ms,
            "algorithmic_flops": flops, "achieved_tflops": tf, "peak_tflops": peak, "frac": tf / peak,
            "bound": "fp32" if precision else "fp64"}


def bench_other_configs(args, W, dev, stream, pk):
    """The benchmark's other configurations at one GPU (device pointers, CUDA
    events on the launching stream, inputs resident in HBM): FP64-plain and
    FP32-refined OK of the 100x100x50 grid (k = 12) and of the clustered
    512x512x64 grid (k = 64, nugget 1e-3, with the error of both against the
    FP64 oracle on sampled cells), full and median IK of the 200x200x100
    five-category grid (k = 24), and the leave-one-out forward and adjoint
    kernels on the 200x200x50 Gaussian-field grid (k = 24)."""
    import torch
    WL = workloads_module()
    steps = max(1, min(args.steps, 3))
    out = {}

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        times, stats = [], []
        for _ in range(n):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = fn()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
        return float(np.mean(times)), stats

    def cont_case(wl, n_steps, kind=0):
        d_data = torch.from_numpy(np.ascontiguousarray(wl.data)).to(dev)
        d_mask = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
        d_out, d_om = d_data.clone(), d_mask.clone()
        d_est = torch.empty(wl.n_cells, dtype=torch.float64, device=dev)
        dims = (C.c_int * 3)(*wl.dims)
        p = W._HPGL_SK_PARAMS(covariance_type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                              sill=wl.cov.sill, nugget=wl.cov.nugget, radiuses=wl.radiuses,
                              max_neighbours=wl.max_neighbours, automatic_mean=1, mean=0.0)
        res, ests = {}, {}
        for prec, name in ((0, "fp64_plain"), (1, "fp32_refined")):
            def call():
                o = W._HPGL_B200_OPTIONS(precision=prec, refine_steps=2,
                                         flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                                         stream=stream.cuda_stream, estimate64=d_est.data_ptr(), variance=None,
                                         status=None, ik_probs=None)
                rc = W._hpgl_so.hpgl_b200_cont_kriging_ex(kind, dims, d_data.data_ptr(), d_mask.data_ptr(),
                                                          C.byref(p), d_out.data_ptr(), d_om.data_ptr(), C.byref(o))
                W.check(rc, "cont_kriging_ex")
                return W.last_stats()
            ms, stats = timed(call, n_steps)
            cells = stats[-1]["kriged_cells"]
            res[name] = {"value": cells / (ms / 1e3), "unit": "kriged cells/s", "ms_per_call": ms,
                         "kriged_cells": cells, "escalated_cells": stats[-1]["escalated_cells"],
                         "roofline": solve_roofline(W, stats, wl.cov.cov_type, prec, kind == 0, pk)}
            ests[name] = d_est.cpu().numpy()
        res["fp32_refined_over_fp64_plain"] = res["fp32_refined"]["value"] / res["fp64_plain"]["value"]
        ok = np.isfinite(ests["fp64_plain"]) & (wl.mask == 0)
        res["rel_err_fp32_refined_vs_fp64_plain"] = float(
            np.abs(ests["fp32_refined"][ok] - ests["fp64_plain"][ok]).max() / np.abs(ests["fp64_plain"][ok]).max())
        return res, ests

    # 100x100x50, spherical, k = 12
    wl = WL.ok_small()
    out["ok_100x100x50_k12"], _ = cont_case(wl, max(steps, 3))

    # clustered 512x512x64, Gaussian nugget 1e-3, k = 64; error against the FP64 oracle on sampled cells
    wl = WL.clustered()
    res, ests = cont_case(wl, 2)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    which = "ref" if O.available("ref") else "port"
    rng = np.random.default_rng(55)
    cand = np.flatnonzero((wl.mask == 0) & np.isfinite(ests["fp64_plain"]))
    nodes = np.sort(rng.choice(cand, min(2000, len(cand)), replace=False)).astype(np.int32)
    r = O.krige_nodes(which, 0, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours, nodes=nodes,
                      want_idx=False)
    okn = r["status"] == 0
    ref = r["est"][okn]
    scale = np.abs(ref).max()
    for name in ("fp64_plain", "fp32_refined"):
        e = ests[name][nodes][okn]
        per = np.abs(e - ref) / np.maximum(np.abs(ref), 1e-300)
        res[name]["error_vs_fp64_oracle"] = {"normwise": float(np.abs(e - ref).max() / scale),
                                             "per_cell_p999": float(np.quantile(per, 0.999)),
                                             "sampled_cells": int(okn.sum()), "oracle": which}
    out["clustered_512x512x64_k64"] = res

    # 200x200x100, five categories, k = 24: full IK and median IK
    wl = WL.indicator()
    m = len(wl.cat_covs)
    d_data = torch.from_numpy(np.ascontiguousarray(wl.data)).to(dev)
    d_mask = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
    d_out, d_om = d_data.clone(), d_mask.clone()
    dims = (C.c_int * 3)(*wl.dims)
    arr = (W._HPGL_IK_PARAMS * m)()
    for i in range(m):
        c = wl.cat_covs[i]
        arr[i] = W._HPGL_IK_PARAMS(covariance_type=c.cov_type, ranges=tuple(c.ranges), angles=tuple(c.angles),
                                   sill=c.sill, nugget=c.nugget, radiuses=tuple(wl.cat_radiuses[i]),
                                   max_neighbours=wl.max_neighbours, marginal_prob=float(wl.marginals[i]))
    d_mik = (d_data >= 2).to(torch.uint8)
    c2 = wl.cat_covs[2]
    mp = (1.0 - float(sum(wl.marginals[2:])), float(sum(wl.marginals[2:])))
    pm = W._HPGL_MEDIAN_IK_PARAMS(covariance_type=c2.cov_type, ranges=tuple(c2.ranges), angles=tuple(c2.angles),
                                  sill=c2.sill, nugget=c2.nugget, radiuses=tuple(wl.cat_radiuses[2]),
                                  max_neighbours=wl.max_neighbours, marginal_probs=mp)
    ik = {}
    for prec, name in ((0, "fp64_plain"), (1, "fp32_refined")):
        def ik_call():
            o = W._HPGL_B200_OPTIONS(precision=prec, refine_steps=2, flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                                     stream=stream.cuda_stream, estimate64=None, variance=None, status=None,
                                     ik_probs=None)
            rc = W._hpgl_so.hpgl_b200_indicator_kriging_ex(dims, d_data.data_ptr(), d_mask.data_ptr(), arr, m,
                                                           d_out.data_ptr(), d_om.data_ptr(), C.byref(o))
            W.check(rc, "indicator_kriging_ex")
            return W.last_stats()

        def mik_call():
            o = W._HPGL_B200_OPTIONS(precision=prec, refine_steps=2, flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                                     stream=stream.cuda_stream, estimate64=None, variance=None, status=None,
                                     ik_probs=None)
            rc = W._hpgl_so.hpgl_b200_median_ik_ex(dims, d_mik.data_ptr(), d_mask.data_ptr(), C.byref(pm),
                                                   d_out.data_ptr(), d_om.data_ptr(), C.byref(o))
            W.check(rc, "median_ik_ex")
            return W.last_stats()
        ms, stats = timed(ik_call, steps)
        ik[f"ik_{name}"] = {"value": wl.n_cells * m / (ms / 1e3), "unit": "category-cells/s", "ms_per_call": ms,
                            "cells_per_s": wl.n_cells / (ms / 1e3),
                            "roofline": solve_roofline(W, stats, c2.cov_type, prec, False, pk)}
        ms, stats = timed(mik_call, steps)
        ik[f"median_ik_{name}"] = {"value": wl.n_cells / (ms / 1e3), "unit": "cells/s", "ms_per_call": ms,
                                   "roofline": solve_roofline(W, stats, c2.cov_type, prec, False, pk)}
    out["indicator_200x200x100_k24"] = ik

    # 200x200x50 Gaussian field, k = 24: leave-one-out forward and adjoint kernels
    wl = WL.gauss_cv()
    from geo_bsd import geo as GEO
    from geo_bsd import loo as LOO
    prop = GEO.ContProperty(wl.data.reshape(wl.dims, order="F"), wl.mask.reshape(wl.dims, order="F"))
    grid = GEO.SugarboxGrid(*wl.dims)
    cm = GEO.CovarianceModel(type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles, sill=wl.cov.sill,
                             nugget=wl.cov.nugget)
    geom = LOO.loo_geometry(prop, grid, wl.radiuses, wl.max_neighbours, cm)
    ranges = torch.tensor(wl.cov.ranges, dtype=torch.float64, requires_grad=True)
    sill = torch.tensor(wl.cov.sill, dtype=torch.float64, requires_grad=True)
    nug = torch.tensor(wl.cov.nugget, dtype=torch.float64, requires_grad=True)
    vals = geom.values.clone().requires_grad_(True)
    fwd_ms, _ = timed(lambda: LOO.loo_estimates(geom, ranges, wl.cov.angles, sill, nug, vals), steps)
    loss = None

    def both():
        nonlocal loss
        loss = LOO.loo_cv_mse(geom, ranges, wl.cov.angles, sill, nug, vals)
        loss.backward()
    both_ms, _ = timed(both, steps)
    t = int(geom.targets.numel())
    k = wl.max_neighbours
    f_sys = k ** 3 / 3 + k ** 2 / 2 + 2 * 2 * k ** 2 + 30 * (k * (k + 1) / 2 + k) + 2 * 2 * k  # F(k, 2)
    out["loo_200x200x50_k24"] = {"targets": t, "forward_ms": fwd_ms, "forward_and_adjoint_ms": both_ms,
                                 "adjoint_ms": both_ms - fwd_ms, "targets_per_s_forward": t / (fwd_ms / 1e3),
                                 "forward_roofline": {"kernel": "k_loo_forward (FP64, one warp per target)",
                                                      "algorithmic_flops": t * f_sys,
                                                      "achieved_tflops": t * f_sys / (fwd_ms / 1e3) / 1e12,
                                                      "peak_tflops": pk["fp64"],
                                                      "frac": t * f_sys / (fwd_ms / 1e3) / 1e12 / pk["fp64"],
                                                      "note": "forward call time includes the torch layer"}}
    return out


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.kind == "sgs":
        bench_sgs(args, rank, world, local)
        return
    if args.kind == "sis":
        return bench_sis(args, rank, world, local)
    if args.kind == "cok":
        bench_cok(args, rank, world, local)
        return
    import torch

    if args.impl == "reference":
        # The reference's own CPU implementation (no GPU, none of this
        # repository's engine: the package is not imported). ok / sk: each
        # step is one whole call of the reference library's public entry point
        # on a z-slab of the workload; lvm: its per-node code on sampled cells.
        if rank == 0:
            wl = load_workload(args.workload)
            threads = os.cpu_count() or 1
            vals, info = [], None
            if args.kind in ("ok", "sk"):
                nz = slab_layers(wl, args.kind, 3.0, threads)
                for i in range(args.warmup + args.steps):
                    v, info = ref_api_slab(wl, args.kind, nz, threads)
                    if i >= args.warmup:
                        vals.append(v)
                sample = (f"one whole hpgl_{'ordinary' if args.kind == 'ok' else 'simple'}_kriging call of the "
                          f"reference library per step ({info['slab']}, {info['kriged_cells']} kriged cells, lookup "
                          f"construction included)")
                v1, info1 = ref_api_slab(wl, args.kind, 2, 1)
                extra = {"value_1_thread": v1, "sample_1_thread": f"{info1['slab']}, {info1['seconds']:.2f} s"}
            else:
                for i in range(args.warmup + args.steps):
                    v, info = cpu_reference(wl, args.kind, min(args.cpu_seconds, 8.0), threads)
                    if i >= args.warmup:
                        vals.append(v)
                sample = f"{info['sample_cells']} random uninformed cells per step, lookup built once"
                extra = {}
            value = float(np.median(vals))
            d = wl.dims
            line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, geo_bsd.workloads)",
                    "config": {"workload": f"{KIND_NAMES[args.kind]} {d[0]}x{d[1]}x{d[2]}, k={wl.max_neighbours}",
                               "sample": sample},
                    "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                     "sample": sample, "cpu_model": cpu_model(), **extra},
                    "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    from geo_bsd import hpgl_wrap as W

    if args.profile_case > 0:
        WL = workloads_module()
        wl = WL.ALL[args.workload](args.profile_case)
    else:
        wl = load_workload(args.workload)
    kind = 0 if args.kind == "ok" else 1
    lvm = args.kind == "lvm"
    n = wl.n_cells
    dev = torch.device("cuda", local)
    d_data = torch.from_numpy(np.ascontiguousarray(wl.data)).to(dev)
    d_mask = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
    d_out = d_data.clone()
    d_omask = d_mask.clone()
    d_var = torch.empty(n, dtype=torch.float64, device=dev)
    d_est = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    dims = (C.c_int * 3)(*wl.dims)
    p = W._HPGL_SK_PARAMS(covariance_type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                          sill=wl.cov.sill, nugget=wl.cov.nugget, radiuses=wl.radiuses,
                          max_neighbours=wl.max_neighbours, automatic_mean=1, mean=0.0)
    p_ok = W._HPGL_OK_PARAMS(covariance_type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                             sill=wl.cov.sill, nugget=wl.cov.nugget, radiuses=wl.radiuses,
                             max_neighbours=wl.max_neighbours)
    h_means = lvm_means(wl) if lvm else None
    d_means = torch.from_numpy(h_means).to(dev) if lvm else None

    def krige(data, mask, means, out, omask, o):
        if lvm:
            return W._hpgl_so.hpgl_b200_lvm_kriging_ex(dims, data, mask, means, C.byref(p_ok), out, omask,
                                                       C.byref(o))
        return W._hpgl_so.hpgl_b200_cont_kriging_ex(kind, dims, data, mask, C.byref(p), out, omask, C.byref(o))

    def dev_call(precision, est=False):
        o = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=3,
                                 flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE, stream=stream.cuda_stream,
                                 estimate64=d_est.data_ptr() if est else None, variance=d_var.data_ptr(),
                                 status=None, ik_probs=None)
        rc = krige(d_data.data_ptr(), d_mask.data_ptr(), d_means.data_ptr() if lvm else None, d_out.data_ptr(),
                   d_omask.data_ptr(), o)
        W.check(rc, "kriging_ex")
        return W.last_stats()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(dist, x, dev)

    def timed_device(precision):
        for _ in range(args.warmup):
            dev_call(precision)
        times, stats = [], []
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between steps (outside the timed region)
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = dev_call(precision)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            stats.append(st)
        barrier()
        return times, stats

    if args.profile_case > 0:
        st = dev_call(1 if args.profile_precision == "fp32_refined" else 0)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": wl.dims, "stats": st}), flush=True)
        return

    # accuracy of the FP32-refined estimate against the FP64 plain one, same grid
    dev_call(0, est=True)
    est64 = d_est.clone()
    dev_call(1, est=True)
    kriged = torch.isfinite(est64) & (d_mask == 0)
    diff = (d_est - est64)[kriged].abs().max().item()
    scale = est64[kriged].abs().max().item()
    rel_err = diff / scale if scale > 0 else 0.0

    t64, s64 = timed_device(0)
    with ClockSampler(local) as clk:
        t32, s32 = timed_device(1)
    ms32 = max_over_ranks(float(np.mean(t32)))
    ms64 = max_over_ranks(float(np.mean(t64)))
    cells = s32[-1]["kriged_cells"]
    value = whole_job_rate(cells, world, ms32)
    value64 = whole_job_rate(s64[-1]["kriged_cells"], world, ms64)
    launches = int(sum(s["kernel_launches"] for s in s32))

    # roofline of the dominant kernel (the solve bucket with the largest time)
    last = s32[-1]
    b = int(np.argmax([last[f"bucket_ms_{i}"] for i in range(5)])) if "bucket_ms_0" in last else 2
    pk = peak_table()
    b_ms = float(np.mean([s[f"bucket_ms_{b}"] for s in s32]))
    b_flops = last[f"bucket_flops_{b}"]
    achieved = b_flops / (b_ms / 1e3) / 1e12
    tpc = traffic_per_cell()
    kname = bucket_kernel(W, b, wl.cov.cov_type, 1, kind == 0 and not lvm)
    roofline = {"bound": "fp32", "kernel": kname,
                "achieved": achieved, "peak": pk["fp32"], "unit": "TFLOP/s", "frac": achieved / pk["fp32"],
                "traffic": (tpc * last[f"bucket_items_{b}"]) if tpc else None,
                "peak_source": f"CUDA-core FP32 peak 148 SM x 128 lanes x 2 x {pk['source']}",
                "algorithmic_flops_per_launch": b_flops, "kernel_ms": b_ms}
    s64b = s64[-1]
    b64 = int(np.argmax([s64b[f"bucket_ms_{i}"] for i in range(5)]))
    fp64_kernel_tflops = s64b[f"bucket_flops_{b64}"] / (np.mean([s[f"bucket_ms_{b64}"] for s in s64]) / 1e3) / 1e12

    # end to end through the C ABI with pinned host buffers; the call reads back what the
    # reference's hpgl_ordinary_kriging / hpgl_simple_kriging return (the output values and
    # mask), not the kriging variance
    lib = W._hpgl_so
    nbytes = n * 4
    h_ptrs = [lib.hpgl_b200_host_alloc(sz) for sz in (nbytes, n, nbytes, n, nbytes)]
    h_data, h_mask, h_out, h_omask, h_mean = h_ptrs
    if lvm:
        C.memmove(h_mean, h_means.ctypes.data, nbytes)
    C.memmove(h_data, np.ascontiguousarray(wl.data).ctypes.data, nbytes)
    C.memmove(h_mask, np.ascontiguousarray(wl.mask).ctypes.data, n)
    C.memmove(h_out, h_data, nbytes)
    C.memmove(h_omask, h_mask, n)

    def host_call(precision):
        o = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=3, flags=W.FLAG_OUT_IS_CLONE, stream=None,
                                 estimate64=None, variance=None, status=None, ik_probs=None)
        rc = krige(h_data, h_mask, h_mean if lvm else None, h_out, h_omask, o)
        W.check(rc, "kriging_ex (host)")
        return W.last_stats()

    def timed_host(precision):
        for _ in range(args.warmup):
            host_call(precision)
        times = []
        stats = None
        for _ in range(args.steps):
            barrier()
            t0 = time.perf_counter()
            stats = host_call(precision)
            times.append(time.perf_counter() - t0)
        barrier()
        return stats, stats["kriged_cells"] * world / max_over_ranks(float(np.mean(times)))

    st, e2e_value = timed_host(1)
    _, e2e_value64 = timed_host(0)
    for ptr in h_ptrs:
        lib.hpgl_b200_host_free(ptr)

    # end to end through the public Python API (geo_bsd.ordinary_kriging / simple_kriging) with
    # pageable numpy arrays: validation, the output clone and the copies included
    e2e_api = None
    if not lvm:
        from geo_bsd import geo as GEO
        prop = GEO.ContProperty(wl.data.reshape(wl.dims, order="F"), wl.mask.reshape(wl.dims, order="F"))
        grid = GEO.SugarboxGrid(*wl.dims)
        cm = GEO.CovarianceModel(type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                                 sill=wl.cov.sill, nugget=wl.cov.nugget)
        api_fn = GEO.ordinary_kriging if kind == 0 else GEO.simple_kriging
        times = []
        for i in range(2 + min(args.steps, 3)):
            barrier()
            t0 = time.perf_counter()
            api_fn(prop, grid, wl.radiuses, wl.max_neighbours, cm, precision="fp32_refined")
            if i >= 2:
                times.append(time.perf_counter() - t0)
        barrier()
        api_cells = W.last_stats()["kriged_cells"]
        e2e_api = {"value": api_cells * world / max_over_ranks(float(np.mean(times))), "unit": UNIT,
                   "path": f"geo_bsd.{api_fn.__name__}(..., precision='fp32_refined'), pageable numpy inputs, "
                           "wall clock per call"}

    configs = None
    if world == 1 and args.kind == "ok" and not args.skip_configs:
        configs = bench_other_configs(args, W, dev, stream, peak_table())

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        if args.kind in ("ok", "sk"):
            cpu = cpu_baseline_api(wl, args.kind, args.cpu_seconds)
        else:
            threads = os.cpu_count() or 1
            v, info = cpu_reference(wl, args.kind, args.cpu_seconds, threads)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference" if info["which"] == "ref" else "port",
                   "sample": f"{info['sample_cells']} random uninformed cells of the same grid; the reference's own "
                             f"per-node code (kriging_interpolation) over OpenMP, lookup construction excluded "
                             f"({info['setup_seconds']:.2f}s)", "cpu_model": cpu_model()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64-refined residuals)", "data": "synthetic (seeded, geo_bsd.workloads)",
            "config": {"workload": f"{KIND_NAMES[args.kind]} {wl.dims[0]}x{wl.dims[1]}x"
                                   f"{wl.dims[2]}, 1% lognormal conditioning, exponential (30,15,6) az 30, "
                                   f"k={wl.max_neighbours}", "precision": "fp32_refined",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "fp64_plain": {"value": value64, "ms_per_step": ms64, "kernel_tflops": fp64_kernel_tflops,
                           "kernel_frac_of_fp64_peak": fp64_kernel_tflops / pk["fp64"], "e2e_value": e2e_value64},
            "fp32_refined_over_fp64_plain": value / value64,
            "rel_err_fp32_refined_vs_fp64": rel_err,
            "escalated_cells": last["escalated_cells"],
            "stages_ms": {k[len("stage_"):-len("_ms")]: round(v, 3) for k, v in last.items() if k.startswith("stage_")},
            "tie_resolved_cells": last["tie_cells"],
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(st["h2d_bytes"]),
                    "d2h_bytes_per_step": int(st["d2h_bytes"]),
                    "timing": "wall clock per call (host tables, copies and kernels); outputs read back: "
                              "values and mask, as the reference's call returns them"},
            "e2e_api": e2e_api,
            "configs": configs,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the coupled MPM-LBM FSI step on B200.

Default workload (one FSI step = one "step"): duct with a cantilevered elastic
plate on a 128 x 64 x 64 D3Q19 lattice (walls at j in {0,63}, k in {0,63}),
MRT tau = 0.55, velocity inlet u_x = 0.05 / pressure outlet rho = 1 with
the reference's default equilibrium-reset open boundaries, plate 2 x 32 x 48 cells at 8 particles per cell (24,576
particles, E = 0.02 and nu = 0.3 in lattice units, density 1.2, clamped base),
moving_boundary coupling subcycled with 120 LBM substeps per FSI step and
40 MPM substeps per FSI step (the explicit MPM limit for this plate).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                       [--storage fp32|fp16] [--workload NAME]
Prints one JSON line (rank 0).  Multi-GPU runs are independent replicas
(weak scaling): every rank advances its own case, no data-path collective.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Workloads: the duct with a cantilevered plate of the benchmark configurations
# (mpm_lbm_b200.cases.DuctPlateCase).
#   duct_plate_128x64x64: 128 x 64 x 64 lattice, tau 0.55, inlet u_x 0.05, plate
#     2 x 32 x 48 cells (24,576 particles); the metric's configuration (default).
#   duct_plate_256x128x128: 256 x 128 x 128 lattice, tau 0.52, inlet u_x 0.04,
#     plate 4 x 64 x 96 cells (196,608 particles); the precision form's
#     configuration, and a lattice larger than L2 for DRAM profiles.
# Both: E = 0.02 and nu = 0.3 in lattice units, density 1.2, moving_boundary
# coupling subcycled with S = 120 LBM substeps per FSI step and M = 40 MPM
# substeps per FSI step (the explicit MPM limit for E = 0.02: c dt / dx ~ 0.45
# at 3 lattice steps per MPM substep; M = 1 would give c dt / dx ~ 15).  The
# open boundaries are the reference's default (equilibrium reset): its
# regularized variants diverge after ~450 substeps in this duct with the
# reference's own operator (the CPU oracle and the CUDA path agree), so they
# are exercised by the parity tests, not by the benchmark run.
WORKLOADS = {
    "duct_plate_128x64x64": dict(lattice=(128, 64, 64), tau=0.55, u_in=0.05, plate=(2, 32, 48)),
    "duct_plate_256x128x128": dict(lattice=(256, 128, 128), tau=0.52, u_in=0.04, plate=(4, 64, 96)),
}
DEFAULT_WORKLOAD = "duct_plate_128x64x64"
FALLBACK_HBM_GBS = 6650.0


class Workload:
    def __init__(self, name):
        from mpm_lbm_b200.cases import DuctPlateCase

        if name not in WORKLOADS:
            raise SystemExit(f"unknown workload {name!r}; choose from {sorted(WORKLOADS)}")
        self.name = name
        self.case = DuctPlateCase(**WORKLOADS[name])
        self.nx, self.ny, self.nz = self.case.lattice
        self.cells = self.case.cells
        self.S, self.M = self.case.lbm_substeps, self.case.mpm_substeps

    def tag(self):
        return f"{self.name}_S{self.S}_M{self.M}"


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: read-only NVML queries every 5 ms from a thread (nvidia-smi's
    100 ms polling as the fallback).  The sampler is started and its first
    sample awaited before the timed region opens."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, gpu_index=0, interval_s=0.005):
        self.gpu = gpu_index
        self.interval = interval_s
        self.samples = []  # (time, sm_mhz, max_mhz, reason bits)
        self.marks = []
        self._stop = threading.Event()
        self.proc = None
        self.source = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def read():
                return (time.time(), float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)), float(mx),
                        int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))

            read()
            self.source = "nvml"
        except Exception:
            read = None
        if read is not None:
            def loop():
                while not self._stop.is_set():
                    try:
                        self.samples.append(read())
                    except Exception:
                        break
                    time.sleep(self.interval)

            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
        else:
            self._start_smi()
        t0 = time.time()
        while not self.samples and time.time() - t0 < 5.0:
            time.sleep(0.005)
        return self

    def _start_smi(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"

            def read():
                for line in self.proc.stdout:
                    p = [x.strip() for x in line.split(",")]
                    try:
                        self.samples.append((time.time(), float(p[1]), float(p[2]), int(p[4], 16)))
                    except (ValueError, IndexError):
                        continue

            self.t = threading.Thread(target=read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def open_region(self):
        self.marks = [time.time()]

    def close_region(self):
        self.marks.append(time.time())

    def __exit__(self, *a):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        lo, hi = (self.marks + [None, None])[:2] if self.marks else (None, None)
        sm, mx, reasons = [], None, set()
        for ts, mhz, mmax, bits in list(self.samples):
            if lo is not None and hi is not None and not (lo <= ts <= hi):
                continue
            sm.append(mhz)
            mx = mmax
            for name, bit in self.REASONS.items():
                if bits & bit:
                    reasons.add(name)
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
               "samples": len(sm), "source": self.source}
        if not sm and self.samples:  # region shorter than one sample: the nearest one
            ts, mhz, mmax, bits = min(self.samples, key=lambda r: abs(r[0] - (lo or r[0])))
            out.update(sm_mhz=mhz, sm_max_mhz=mmax, samples=0,
                       reasons=sorted(n for n, b in self.REASONS.items() if bits & b))
        return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def oracle_driver(wl, substeps, mpm_substeps, threads=None):
    """The CPU oracle (C++ restatement, OpenMP over cells; all host threads by
    default) on the same case: FSI steps of `substeps` LBM and `mpm_substeps`
    MPM substeps."""
    from oracle import oracle as orc

    threads = threads or os.cpu_count() or 1
    return orc.fsi_driver_for_case(wl.case, substeps=substeps, mpm_substeps=mpm_substeps, threads=threads), threads


def cpu_sample_text(wl, steps, substeps, mpm_substeps):
    return (f"{steps} FSI step(s) x ({substeps} LBM substeps + {mpm_substeps} MPM substeps) of the same "
            f"{wl.nx}x{wl.ny}x{wl.nz} case, CPU oracle (C++ restatement, OpenMP over cells)")


def cpu_baseline(wl, steps=1):
    """MLUPS of the CPU oracle on a bounded sample of the workload: one FSI
    step on all host threads, and a shorter FSI step (12 LBM + 4 MPM
    substeps, the same 3:1 ratio per LBM substep) on one thread."""
    substeps, mpm_substeps = wl.S, wl.M
    drv, threads = oracle_driver(wl, substeps, mpm_substeps)
    t0 = time.perf_counter()
    for _ in range(steps):
        drv.step_once()
    dt = time.perf_counter() - t0
    one_sub, one_msub = 12, 4
    drv1, _ = oracle_driver(wl, one_sub, one_msub, threads=1)
    t0 = time.perf_counter()
    drv1.step_once()
    dt1 = time.perf_counter() - t0
    return {"value": steps * substeps * wl.cells / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "cpu_model": cpu_model(), "nproc": os.cpu_count(),
            "sample": cpu_sample_text(wl, steps, substeps, mpm_substeps),
            "one_thread": {"value": one_sub * wl.cells / dt1 / 1e6, "unit": "MLUPS", "cores": 1,
                           "sample": cpu_sample_text(wl, 1, one_sub, one_msub)}}


def dist_setup():
    """One process per GPU under torchrun: NCCL over the node's GPUs, or gloo
    for a host-only run (the reference arm on a machine without a GPU)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            backend = "nccl"
        else:
            backend = "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(x, device=None):
    """x maximised over the ranks of the default process group (x itself when
    there is none): independent replicas are done when the slowest is."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, wl, ws, rank):
    """The reference arm: the reference's algorithm on the host CPU cores.  The
    reference itself (Taichi) is not installed on this image, so its CPU
    restatement (the oracle) runs; each step is a bounded sample of the
    workload: one FSI step of --ref-substeps LBM substeps."""
    if rank != 0:
        return
    sub = args.ref_substeps
    msub = max(1, sub // 3)
    drv, threads = oracle_driver(wl, sub, msub)
    for _ in range(args.warmup):
        drv.step_once()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        drv.step_once()
    secs = time.perf_counter() - t0
    value = args.steps * sub * wl.cells / secs / 1e6
    cb = {"value": value, "unit": "MLUPS", "cores": threads, "kind": "port", "cpu_model": cpu_model(),
          "sample": cpu_sample_text(wl, args.steps, sub, msub)}
    print(json.dumps({"impl": "reference", "metric": "coupled-FSI MLUPS", "value": value, "unit": "MLUPS",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": {"workload": wl.tag(), "reference_step": f"{sub} LBM + {msub} MPM substeps",
                                 "reference_runtime": "CPU restatement of the reference (taichi is not installed "
                                                      "on this image)"},
                      "cpu_baseline": cb,
                      "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_batched(args):
    """Batching form: 64 cases of the batching configuration (per-axis edges in
    {32, 48, 64, 96}, tau ~ U[0.52, 0.8], block or plate of 4^3-16^3 cells,
    E ~ U[0.01, 0.1], penalty or moving_boundary), one batched launch per
    phase replayed as one CUDA graph per FSI step, against the same cases
    advanced one at a time (each with its own CUDA-graph step) on the same GPU.
    A step is one FSI step (one LBM step + 10 MPM substeps) of every case."""
    import torch

    from mpm_lbm_b200.batch import FSIBatch, sample_box_cases

    from mpm_lbm_b200.autotune import tune_batch

    cases = sample_box_cases(args.cases, seed=0)
    cells = sum(c.cells for c in cases)
    if args.no_autotune:
        tuning = {"lbm_tune": 0 if args.lbm_tune is None else args.lbm_tune, "mpm_ctas": 0, "ms_per_step": None}
    else:
        tuning = tune_batch(lambda: [c.make_driver(storage=args.storage) for c in cases], storage=args.storage,
                            mpm_substeps=10)
        torch.cuda.empty_cache()
    batch = FSIBatch(capacity=len(cases), storage=args.storage, mpm_substeps=10, lbm_tune=tuning["lbm_tune"],
                     mpm_ctas=tuning["mpm_ctas"])
    for c in cases:
        batch.add(c.make_driver(storage=args.storage))
    for _ in range(max(args.warmup, 3)):
        batch.step(use_graph=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        batch.step(use_graph=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    out = {"metric": "batched coupled-FSI MLUPS", "value": cells / (ms * 1e-3) / 1e6, "unit": "MLUPS",
           "form": "batched", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "dtype": "f32" if args.storage == "fp32" else "f16-storage/f32-compute",
           "data": "synthetic", "config": {"workload": f"batch_{len(cases)}_box_cases", "cases": len(cases),
                                           "cells": cells, "kernels_per_step": batch.graph_kernels,
                                           "lbm_tune": batch.dims.lbm_tune, "mpm_ctas": batch.dims.mpm_ctas,
                                           "tuning_ms_per_step": tuning["ms_per_step"]}}
    del batch
    if not args.no_one_by_one:
        tot = 0.0
        for c in cases:
            drv = c.make_driver(storage=args.storage)
            drv.use_cuda_graph = True
            for _ in range(3):
                drv.step_once()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(args.steps):
                drv.step_once()
            e1.record()
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1) / args.steps
            del drv
        out["one_by_one"] = {"ms_per_step": tot, "value": cells / (tot * 1e-3) / 1e6, "unit": "MLUPS"}
    print(json.dumps(out), flush=True)


def run_served(args):
    """Serving form: a Poisson stream (20 requests/s) of FSI solves, cubic
    grids from {32, 48, 64, 96, 128} with weights {.3, .3, .2, .15, .05}, 100-2000
    LBM steps each, solid / tau / mode as in the batching form, admitted into a
    continuous batch under a 150 GB HBM budget."""
    from mpm_lbm_b200.serve import FSIServer, poisson_requests

    reqs = poisson_requests(args.requests, rate_per_s=20.0, seed=1, steps=(100, 2000))
    srv = FSIServer(slots=64, hbm_budget_bytes=150e9, storage=args.storage)
    srv.run(reqs, time_limit_s=1800)
    rep = srv.report()
    out = {"metric": "served coupled-FSI MLUPS", "value": rep["aggregate_mlups"], "unit": "MLUPS", "form": "served",
           "n_gpus": 1, "higher_is_better": True,
           "dtype": "f32" if args.storage == "fp32" else "f16-storage/f32-compute", "data": "synthetic",
           "p50_latency_s": rep["p50_latency_s"], "p99_latency_s": rep["p99_latency_s"],
           "config": {"workload": f"poisson_20ps_{args.requests}_requests", **rep}}
    print(json.dumps(out), flush=True)


def time_lbm_kernel(drv, storage, n_k1=40, reps=5):
    """Average duration of the fused LBM step kernel: a CUDA graph of n_k1
    back-to-back moving-boundary substeps, replayed reps times between events on
    the stream the kernels run on."""
    import torch

    lbm = drv.lbm
    stream = torch.cuda.current_stream()
    graph = torch.cuda.CUDAGraph()
    lbm.dirstats_enabled = False
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        for _ in range(n_k1):
            lbm.step_moving_bounceback()
    torch.cuda.synchronize()
    graph.replay()  # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    k1_ms = e0.elapsed_time(e1) / (reps * n_k1)
    del graph
    return k1_ms


def time_mpm_phase(drv, reps=5):
    """Average duration of one binned MPM substep with its reaction transfer:
    a CUDA graph of the FSI step's MPM phase (re-binning, then the M substeps
    of fsi_mpm_substeps_binned), replayed reps times between events."""
    import torch

    solid, lbm = drv.solid, drv.lbm
    coupler = drv.mb_coupler if drv.mb_coupler is not None else drv.link_area_coupler
    M = drv.config.mpm_substeps_per_lbm_step
    stream = torch.cuda.current_stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        solid.rebin()
        solid.substeps_binned(M, coupler, lbm)
    graph.replay()  # warm
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        graph.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    del graph
    return e0.elapsed_time(e1) / (reps * M)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one k_lbm_step
# launch, from an ncu capture of the same workload's kernel
# (profiles/k_lbm_step_<workload>.md).  The 128x64x64 lattice fits in L2: the
# capture (caches flushed before the launch) reads the populations from DRAM
# and its writes stay in L2.
NCU_LBM_TRAFFIC = {
    ("duct_plate_128x64x64", "fp32"): 42.6e6,
    ("duct_plate_256x128x128", "fp32"): 590.5e6,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="default launch variants")
    ap.add_argument("--lbm-tune", type=int, default=None, help="fixed FsiLbmParams.tune (no autotuning)")
    ap.add_argument("--ref-substeps", type=int, default=30,
                    help="LBM substeps per timed step of the reference arm (bounded CPU sample)")
    ap.add_argument("--form", default="single", choices=["single", "batched", "served"],
                    help="single: the metric's case; batched / served: the batching and serving forms")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--requests", type=int, default=100)
    ap.add_argument("--no-one-by-one", action="store_true")
    args = ap.parse_args()
    if args.form == "batched":
        run_batched(args)
        return
    if args.form == "served":
        run_served(args)
        return
    wl = Workload(args.workload)
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, wl, ws, rank)
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    import torch

    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    drv = wl.case.make_driver(storage=args.storage, graph=True, device=device)
    lbm = drv.lbm
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # > L2 (126 MB)
    stream = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 3)):
        drv.step_once()
    torch.cuda.synchronize()
    tuning = None
    if args.lbm_tune is not None:
        # a fixed launch variant (profiling a given variant); the step graph is recaptured
        drv._graph = None
        drv.lbm.tune = args.lbm_tune
        tuning = {"lbm": {"choice": drv.lbm.tune, "ms_per_substep": None}}
        for _ in range(2):
            drv.step_once()
        torch.cuda.synchronize()
    elif not args.no_autotune:
        tuning = drv.autotune()  # launch variants timed on this state; the step graph is recaptured
        for _ in range(2):
            drv.step_once()
        torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    # ---- timed region: K FSI steps, each bracketed by events; L2 flushed in between
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        clk.open_region()
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            drv.step_once()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        clk.close_region()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms, device)
    fluid_cells = int(lbm.fluid_mask().sum().item())
    value = ws * args.steps * wl.S * wl.cells / (total_ms * 1e-3) / 1e6
    ms_step = total_ms / args.steps
    rows_ok = bool(np.isfinite(drv.lbm.get_stats()["rho_max"]))
    kernels_per_step = drv.graph_kernels_per_step

    # ---- dominant kernel: the fused LBM step (the chosen variant; every valid variant listed)
    from mpm_lbm_b200.autotune import lbm_candidates

    chosen = drv.lbm.tune
    variant_ms = {}
    for t in lbm_candidates(drv.lbm):
        drv.lbm.tune = t
        variant_ms[int(t)] = time_lbm_kernel(drv, args.storage)
    drv.lbm.tune = chosen
    k1_ms = variant_ms[int(chosen)]
    pop_bytes = 2 if args.storage == "fp16" else 4
    alg_bytes = fluid_cells * 19 * 2 * pop_bytes + wl.cells * 1
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (k1_ms * 1e-3) / 1e9
    traffic = NCU_LBM_TRAFFIC.get((wl.name, args.storage))
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": f"{peak_kind} (hbm_gbs)", "kernel": "k_lbm_step",
                "kernel_ms": k1_ms, "kernel_variant": int(chosen),
                "kernel_ms_by_variant": variant_ms, "alg_bytes_per_launch": alg_bytes,
                "alg_bytes_per_cell": f"2*19*{pop_bytes} per fluid cell + 1 (flags) per cell"}

    # ---- the MPM phase (second in the step after the LBM substeps)
    mpm_ms = time_mpm_phase(drv)
    mpm = {"kernel": "k_mpm_seq", "ms_per_substep": mpm_ms, "launches_per_substep": (wl.M + 2) / wl.M,
           "share_of_step": wl.M * mpm_ms / ms_step}

    # ---- the whole coupled FSI step against the same roofline: per step
    # S LBM substeps (alg_bytes each), M MPM substeps of 204 B per particle and
    # 48 B per active grid node, and 25 B per cell for projection and mask
    n_p = drv.solid.n_particles
    active_nodes = int((drv.solid._last_grid()[1] > 0).sum().item())
    step_bytes = wl.S * alg_bytes + wl.M * (n_p * 204 + active_nodes * 48) + wl.cells * 25
    coupled = step_bytes / (ms_step * 1e-3) / 1e9
    roofline["coupled_frac"] = coupled / peak
    roofline["coupled"] = {"achieved": coupled, "bytes_per_step": step_bytes, "active_grid_nodes": active_nodes,
                           "bytes": "S*(2*19*s*fluid_cells + cells) + M*(204*particles + 48*active_nodes) + 25*cells"}

    # ---- end to end through the public API with host buffers
    pinned_in = torch.tensor([wl.case.u_in, 0.0, 0.0], dtype=torch.float32).pin_memory()
    n = drv.solid.n_particles
    pinned_out = torch.empty(3, n, dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    e_steps = max(3, args.steps // 2)
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for k in range(e_steps):
        pinned_in[0] = wl.case.u_in
        drv.lbm.set_inlet_velocity_async(pinned_in)
        drv.step_once()
        pinned_out.copy_(drv.solid.t_x, non_blocking=True)
        torch.cuda.current_stream().synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, device)
    e2e_value = ws * e_steps * wl.S * wl.cells / e2e_s / 1e6

    result = {
        "metric": "coupled-FSI MLUPS", "value": value, "unit": "MLUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.storage == "fp32" else "f16-storage/f32-compute",
        "data": "synthetic",
        "config": {"workload": wl.tag(), "lattice": [wl.nx, wl.ny, wl.nz],
                   "lbm_substeps_per_fsi_step": wl.S, "mpm_substeps_per_fsi_step": wl.M,
                   "particles": int(n), "fluid_cells": fluid_cells, "collision": "mrt", "tau": wl.case.tau,
                   "coupling": "moving_boundary/engineering/subcycled",
                   "open_boundary": wl.case.open_boundary, "reaction_cap": wl.case.reaction_cap,
                   "population_storage": args.storage,
                   "l2": "flushed (256 MB write) between timed FSI steps", "cuda_graph": True,
                   "launch_variants": None if tuning is None else
                   {"lbm_tune": tuning["lbm"]["choice"], "lbm_ms_per_substep": tuning["lbm"]["ms_per_substep"]},
                   "parallelism": f"replicas x{ws}"},
        "particle_updates_per_s": ws * args.steps * wl.M * n / (total_ms * 1e-3),
        "roofline": roofline,
        "mpm": mpm,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": 12, "d2h_bytes_per_step": 12 * n,
                "api": "FSIDriver3D.step_once + inlet velocity H2D from pinned host + particle positions D2H"},
        "gpu_launches": None if kernels_per_step is None else int(round(args.steps * kernels_per_step)),
        "gpu_launches_per_step": kernels_per_step,
        "finite": rows_ok,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            result["cpu_baseline"] = cpu_baseline(wl)
        except Exception as exc:  # reported, not fatal
            result["cpu_baseline"] = {"error": str(exc)}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if ws > 1:
        drv._graph = None
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

"""Serving loop: FSI solve requests admitted into a running batch.

Requests arrive over time (a Poisson stream in the benchmark).  The server
keeps every admitted request's state resident on the device in a slot of an
FSIBatch and advances all occupied slots together, one FSI step per batched
launch sequence.  Between steps it
  * retires requests that have run their LBM steps (their summary is read
    back, their slot and memory are freed), and
  * admits waiting requests in arrival order while a slot is free and the
    estimated device memory of the admitted requests stays within the HBM
    budget,
so requests that arrive while others are on the GPU join the batch as soon
as room frees up, and their work overlaps with the others' on the device
(continuous batching).  Each request's result is the same as when it runs
alone (the batched kernels perform each case's own arithmetic).

Latency of a request = completion time - arrival time (wall clock, queueing
included); throughput = cell updates of the completed requests / makespan.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from .batch import BoxCase

GRID_SIZES = (32, 48, 64, 96, 128)
GRID_WEIGHTS = (0.3, 0.3, 0.2, 0.15, 0.05)


@dataclass
class Request:
    rid: int
    case: BoxCase
    arrival_s: float
    admit_s: Optional[float] = None
    finish_s: Optional[float] = None
    result: Optional[dict] = None
    error: Optional[str] = None

    @property
    def lbm_steps(self):
        return self.case.lbm_steps

    @property
    def latency_s(self):
        return None if self.finish_s is None else self.finish_s - self.arrival_s


def poisson_requests(n, rate_per_s=20.0, seed=0, sizes=GRID_SIZES, weights=GRID_WEIGHTS, steps=(100, 2000),
                     mpm_substeps=10):
    """n requests with exponential inter-arrival times (mean 1 / rate): a cubic
    grid drawn from `sizes` with `weights`, an LBM step count uniform in
    `steps`, and the solid, tau, material and mode of the batching
    configuration."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        g = int(rng.choice(sizes, p=np.asarray(weights) / np.sum(weights)))
        solid = "block" if rng.random() < 0.5 else "plate"
        L = int(rng.integers(4, 17))
        L = min(L, g - 4) if solid == "block" else min(L, g - 4)
        case = BoxCase(lattice=(g, g, g), tau=float(rng.uniform(0.52, 0.8)),
                       mode="penalty" if rng.random() < 0.5 else "moving_boundary", solid=solid,
                       solid_cells=max(L, 2), e_lu=float(rng.uniform(0.01, 0.1)),
                       lbm_steps=int(rng.integers(steps[0], steps[1] + 1)), mpm_substeps=mpm_substeps,
                       seed=int(seed * 100000 + i))
        out.append(Request(rid=i, case=case, arrival_s=t))
    return out


def estimate_bytes(case: BoxCase, storage="fp32"):
    """Device memory a resident case holds (lattice fields, MPM grid buffers,
    particles and bins), from the allocation sizes of LBMFluid3D and
    MPMSolid3D."""
    cells = case.cells
    pitch = (cells + 127) // 128 * 128
    pop = 19 * pitch * (2 if storage == "fp16" else 4)
    # flags, nbr, rho, vel, static, old, reinit, phi, smass, svel, cf, hydro, accum, hpp(2x3), change list,
    # readout buffers (pop 19 + rho + vel, float) made on first readout
    lattice = pitch * (1 + 4 + 4 + 12 + 1 + 1 + 1 + 4 + 4 + 12 + 12 + 12 + 12 + 24 + 4) + pitch * 4 * 23
    n = case.n_grid ** 3
    grid = 2 * n * 7 * 4
    parts = case.n_particles * (4 * (3 + 3 + 9 + 9 + 1 + 1 + 1 + 3) + 1 + 4 * (32 + 2)) + 64 * 1024
    return int(pop + lattice + grid + parts)


def request_summary(drv):
    """Small result of a finished request, read back from the device."""
    st = drv.lbm.get_stats()
    ms = drv.solid.get_stats()
    tip = drv.flap_tip_displacement()
    return {"rho_min": st["rho_min"], "rho_max": st["rho_max"], "max_v": st["max_v"], "mass_total": st["mass_total"],
            "min_J": ms["min_J"], "max_speed": ms["max_speed"],
            "tip_displacement": None if tip is None else [float(v) for v in tip.cpu().tolist()]}


class AdmissionQueue:
    """FIFO admission under a slot limit and a device-memory budget (host
    logic only; the engine that holds the slots is separate)."""

    def __init__(self, slots, budget_bytes, estimate: Callable[[Request], int]):
        self.slots = int(slots)
        self.budget = int(budget_bytes)
        self.estimate = estimate
        self.waiting: List[Request] = []
        self.resident = {}  # rid -> bytes

    @property
    def used_bytes(self):
        return sum(self.resident.values())

    def arrive(self, req: Request):
        need = self.estimate(req)
        if need > self.budget:
            req.error = f"request needs {need} bytes, above the {self.budget}-byte budget"
            return False
        self.waiting.append(req)
        return True

    def admissible(self):
        """Requests to admit now, in arrival order; stops at the first that does
        not fit (no overtaking, so a large request is not starved)."""
        out = []
        while self.waiting and len(self.resident) < self.slots:
            req = self.waiting[0]
            need = self.estimate(req)
            if self.used_bytes + need > self.budget:
                break
            self.waiting.pop(0)
            self.resident[req.rid] = need
            out.append(req)
        return out

    def release(self, req: Request):
        self.resident.pop(req.rid, None)


class FSIServer:
    """Continuous-batching FSI server on one GPU."""

    def __init__(self, slots=64, hbm_budget_bytes=150e9, storage="fp32", mpm_substeps=10, device="cuda",
                 clock=time.perf_counter, engine=None, make_driver=None, summarize=request_summary):
        """engine: an FSIBatch-like object (add / remove / step / steps_done);
        make_driver(case) builds an initialised case; summarize(driver) reads
        a finished case's result.  Defaults: FSIBatch and BoxCase.make_driver."""
        self.storage = storage
        if engine is None:
            from .batch import FSIBatch

            engine = FSIBatch(capacity=slots, storage=storage, mpm_substeps=mpm_substeps, device=device)
        self.batch = engine
        self.make_driver = make_driver or (lambda case: case.make_driver(storage=storage, device=device))
        self.summarize = summarize
        self.queue = AdmissionQueue(slots, hbm_budget_bytes, lambda r: estimate_bytes(r.case, storage))
        self.device = device
        self.clock = clock
        self.slot_of = {}
        self.running = {}
        self.done: List[Request] = []
        self.batch_steps = 0
        self.keep_drivers = False

    def _admit(self, now):
        for req in self.queue.admissible():
            try:
                drv = self.make_driver(req.case)
                slot = self.batch.add(drv)
            except Exception as exc:  # a failed set-up fails this request only
                req.error = f"admission failed: {exc}"
                req.finish_s = self.clock() - self.t0
                self.queue.release(req)
                self.done.append(req)
                continue
            req.admit_s = now
            self.slot_of[req.rid] = slot
            self.running[req.rid] = req

    def _retire(self):
        for rid in list(self.running):
            req = self.running[rid]
            slot = self.slot_of[rid]
            if self.batch.steps_done[slot] < req.lbm_steps:
                continue
            drv = self.batch.remove(slot)
            try:
                req.result = self.summarize(drv)
                if not all(math.isfinite(v) for v in (req.result["rho_min"], req.result["rho_max"])):
                    req.error = "non-finite density"
            except Exception as exc:
                req.error = f"readout failed: {exc}"
            if self.keep_drivers:
                req.driver = drv
            req.finish_s = self.clock() - self.t0
            del self.running[rid]
            del self.slot_of[rid]
            self.queue.release(req)
            self.done.append(req)

    def run(self, requests: List[Request], time_limit_s=600.0):
        """Serve `requests` (arrival_s relative to the start) in real time."""
        pending = sorted(requests, key=lambda r: r.arrival_s)
        self.t0 = self.clock()
        i = 0
        while i < len(pending) or self.running or self.queue.waiting:
            now = self.clock() - self.t0
            if now > time_limit_s:
                raise TimeoutError(f"serving did not finish within {time_limit_s} s")
            while i < len(pending) and pending[i].arrival_s <= now:
                if not self.queue.arrive(pending[i]):
                    pending[i].finish_s = now
                    self.done.append(pending[i])
                i += 1
            self._admit(now)
            if self.running:
                self.batch.step(use_graph=False)
                self.batch_steps += 1
                self._retire()
            elif i < len(pending):
                time.sleep(max(0.0, min(0.01, pending[i].arrival_s - now)))
        self.makespan_s = self.clock() - self.t0
        return self.done

    def report(self):
        ok = [r for r in self.done if r.error is None and r.finish_s is not None]
        lat = np.array([r.latency_s for r in ok]) if ok else np.zeros(1)
        cell_updates = sum(r.case.cells * r.lbm_steps for r in ok)
        return {"requests": len(self.done), "completed": len(ok), "failed": len(self.done) - len(ok),
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_latency_s": float(lat.mean()), "makespan_s": self.makespan_s,
                "aggregate_mlups": cell_updates / self.makespan_s / 1e6, "batch_steps": self.batch_steps,
                "storage": self.storage}

"""Batched FSI: many independent cases advanced with one launch per phase.

Each case is a full FSIDriver3D (its own lattice of any shape, particles,
MPM grid, relaxation time, material and coupling mode), built and
initialised as usual.  FSIBatch then advances all active cases together:
per FSI step, every phase of FSIDriver3D.step_once (one LBM step per FSI
step, src/mpm_lbm/sim/drivers/fsi_driver.py:484-531) runs as one batched
launch for all cases (fsi_batch_* in include/fsi_b200.h):

  penalty cases:          project -> LBM step with the penalty force
  moving-boundary cases:  project -> mask rebuild -> LBM step (moving walls)
  all:                    rebin -> M x binned MPM substep with the case's
                          reaction transfer

The per-case step state (AA parity, ping-pong slot, MPM grid buffer) lives in
a device array of FsiBatchCase records and advances on the device, so the
whole batched FSI step can be captured in one CUDA graph and replayed.
Slots can be filled and emptied between steps (the serving loop does); a
case's driver object reads its fields as usual after `sync_case(slot)`.

Restrictions: every case in a batch shares the population storage and the
number M of MPM substeps per FSI step, and has no open boundaries.
"""

from __future__ import annotations

import ctypes
import math
import tempfile
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np
import torch

from ._lib import (FSI_BATCH_MOVING, FSI_BATCH_PENALTY, FSI_MODE_DIRSTATS, FSI_MODE_MOVING_BB, FSI_MODE_PENALTY,
                   FSI_TUNE_LBM_OCC3, FSI_TUNE_LBM_PAIR, FsiBatchCase, FsiBatchDims, call, launch_count,
                   stream_handle)
from .config import FSIDriverConfig
from .geometry import jittered_block, walled_channel


@dataclass(frozen=True)
class BoxCase:
    """A walled box (periodic in x, solid planes at j in {0, ny-1} and k in
    {0, nz-1}) driven by a body force along x, holding an elastic block
    (free, centred) or a plate cantilevered from the y-min wall at x = nx/4
    (thickness max(2, L/4) along x, height and span L, clamped base), with 8
    particles per cell.  tau and E are lattice-unit values; the MPM grid and
    the normalised units span the longest lattice edge (dx = 1 / max edge)."""

    lattice: Tuple[int, int, int] = (32, 32, 32)
    tau: float = 0.6
    mode: str = "moving_boundary"        # or "penalty"
    solid: str = "block"                 # or "plate"
    solid_cells: int = 8                 # L
    e_lu: float = 0.05
    nu_poisson: float = 0.3
    rho_s: float = 1.2
    body_force: Tuple[float, float, float] = (1.0e-5, 0.0, 0.0)
    mpm_substeps: int = 10               # M per FSI step (= per LBM step)
    dt_lbm: float = 1.0e-3
    lbm_steps: int = 200                 # FSI steps a request runs (serving)
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def n_grid(self):
        return max(self.lattice)

    @property
    def cells(self):
        return self.lattice[0] * self.lattice[1] * self.lattice[2]

    def _box(self):
        nx, ny, nz = self.lattice
        L = int(self.solid_cells)
        if self.solid == "block":
            if L > min(ny, nz) - 4 or L > nx - 2:
                raise ValueError(f"block of {L} cells does not fit the {self.lattice} box")
            lo = (nx // 2 - L // 2, ny // 2 - L // 2, nz // 2 - L // 2)
            return lo, (lo[0] + L, lo[1] + L, lo[2] + L)
        if self.solid == "plate":
            t = max(2, L // 4)
            if L > ny - 3 or L > nz - 4:
                raise ValueError(f"plate of {L} cells does not fit the {self.lattice} box")
            x0, z0 = nx // 4, (nz - L) // 2
            return (x0, 1, z0), (x0 + t, 1 + L, z0 + L)
        raise ValueError("solid must be 'block' or 'plate'")

    @property
    def n_particles(self):
        lo, hi = self._box()
        return 8 * (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2])

    def config(self) -> FSIDriverConfig:
        n = self.n_grid
        nu_phys = (self.tau - 0.5) / 3.0 * (1.0 / n) ** 2 / self.dt_lbm
        kw = dict(coupling_mode=self.mode, n_grid=n, n_particles=self.n_particles, n_lbm_steps=self.lbm_steps,
                  mpm_substeps_per_lbm_step=self.mpm_substeps, mpm_dt=self.dt_lbm / self.mpm_substeps,
                  lbm_viscosity_semantics="physical_nu_mapping", physical_duct_length_m=1.0,
                  fluid_kinematic_viscosity_m2_s=nu_phys, mb_force_cap_norm=1.0e-8 * (128.0 / n) ** 3,
                  output_interval=max(1, self.lbm_steps))
        kw.update(self.extra)
        return FSIDriverConfig(**kw)

    def geometry(self):
        nx, ny, nz = self.lattice
        solid = walled_channel(nx, ny, nz)
        lo, hi = self._box()
        dx = 1.0 / self.n_grid
        x = jittered_block(lo, hi, dx, 2, self.seed)
        vol0 = np.full(len(x), dx ** 3 / 8.0, np.float32)
        mass = (vol0 * np.float32(self.rho_s)).astype(np.float32)
        if self.solid == "plate":
            ycell = x[:, 1] / dx
            base_h = max(hi[0] - lo[0], 0.2 * (hi[1] - lo[1]))
            fixed = (ycell < 1 + base_h).astype(np.int8)
            tip = (ycell >= hi[1] - base_h).astype(np.int8)
        else:
            fixed = np.zeros(len(x), np.int8)
            tip = np.ones(len(x), np.int8)
        return solid, {"x": x, "vol0": vol0, "mass": mass, "fixed": fixed, "free_tip": tip}

    def material(self):
        e_norm = self.e_lu * ((1.0 / self.n_grid) / self.dt_lbm) ** 2
        return {"young_modulus": e_norm, "poisson_ratio": self.nu_poisson, "p_rho": self.rho_s}

    def make_driver(self, storage="fp32", device="cuda", out_dir=None):
        from .driver import FSIDriver3D

        solid, parts = self.geometry()
        drv = FSIDriver3D(self.config(), out_dir or tempfile.mkdtemp(prefix="fsi_box_"), population_storage=storage,
                          lattice_shape=tuple(self.lattice), material=self.material(), static_solid=solid,
                          initial_particles=parts, device=device)
        drv.initialize()
        drv.lbm.set_force(self.body_force)
        return drv


def sample_box_cases(n, seed=0, edges=(32, 48, 64, 96), lbm_steps=200, mpm_substeps=10):
    """n cases drawn as the batching configuration: per-axis edges uniform in
    `edges`, tau ~ U[0.52, 0.8], a block or plate of 4^3..16^3 cells
    (clipped to fit), E ~ U[0.01, 0.1], mode penalty or moving_boundary."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        lat = tuple(int(rng.choice(edges)) for _ in range(3))
        solid = "block" if rng.random() < 0.5 else "plate"
        L = int(rng.integers(4, 17))
        nx, ny, nz = lat
        L = min(L, min(ny, nz) - 4, nx - 2) if solid == "block" else min(L, ny - 3, nz - 4)
        out.append(BoxCase(lattice=lat, tau=float(rng.uniform(0.52, 0.8)),
                           mode="penalty" if rng.random() < 0.5 else "moving_boundary", solid=solid,
                           solid_cells=max(L, 2), e_lu=float(rng.uniform(0.01, 0.1)), lbm_steps=lbm_steps,
                           mpm_substeps=mpm_substeps, seed=int(seed * 1000 + i)))
    return out


class FSIBatch:
    """Up to `capacity` independent FSI cases, advanced together."""

    def __init__(self, capacity, storage="fp32", mpm_substeps=10, device="cuda", lbm_tune=None, mpm_ctas=0):
        """lbm_tune: FSI_TUNE_LBM_OCC3 (0, default) or FSI_TUNE_LBM_PAIR (2, every
        case's nx even); mpm_ctas: CTAs per case of the batched MPM substeps (0:
        about one per chunk of the largest case).  autotune.tune_batch picks
        both by timing."""
        self.capacity = int(capacity)
        self.storage = storage
        self.M = int(mpm_substeps)
        self.device = torch.device(device)
        self.lbm_tune = lbm_tune
        self.mpm_ctas = int(mpm_ctas)
        self.slots = [None] * self.capacity          # FSIDriver3D per slot
        self.records = (FsiBatchCase * self.capacity)()
        self.t_cases = torch.zeros(ctypes.sizeof(self.records), dtype=torch.uint8, device=self.device)
        self.dims = FsiBatchDims(n_cases=self.capacity, store_fp16=int(storage == "fp16"))
        self.steps_done = [0] * self.capacity
        self.graph = None
        self.graph_kernels = None

    # ---------------------------------------------------------- slots
    def free_slots(self):
        return [i for i, d in enumerate(self.slots) if d is None]

    def add(self, drv, slot=None):
        """Put an initialised FSIDriver3D into a free slot (between steps)."""
        if drv.config.coupling_mode not in ("penalty", "moving_boundary"):
            raise ValueError("batched cases must use penalty or moving_boundary coupling")
        if drv.config.fsi_exchange_mode != "one_lbm_step_per_fsi_step":
            raise ValueError("batched cases run one LBM step per FSI step")
        if drv.config.mpm_substeps_per_lbm_step != self.M:
            raise ValueError(f"batched cases share M = {self.M} MPM substeps per FSI step")
        if drv.population_storage != self.storage:
            raise ValueError(f"batched cases share the population storage ({self.storage})")
        if drv.mpm_path != "binned":
            raise ValueError("batched cases use the binned MPM substep")
        lbm = drv.lbm
        if lbm.bc_x_left or lbm.bc_x_right:
            raise ValueError("batched cases have no open boundaries")
        if lbm.params.ob_semantics >= 8:
            raise ValueError("batched cases run no outlet flux controller (open-boundary semantics 8 and 9)")
        if slot is None:
            free = self.free_slots()
            if not free:
                raise RuntimeError("no free batch slot")
            slot = free[0]
        if self.slots[slot] is not None:
            raise RuntimeError(f"slot {slot} is busy")
        self.slots[slot] = drv
        self.steps_done[slot] = 0
        self._write_record(slot)
        return slot

    def remove(self, slot):
        """Take the case out of its slot (between steps); returns its driver,
        synchronised for readout."""
        drv = self.slots[slot]
        if drv is None:
            return None
        self.sync_case(slot)
        self.slots[slot] = None
        self.records[slot] = FsiBatchCase()
        self._upload(slot)
        self._update_dims()
        return drv

    def _write_record(self, slot):
        drv = self.slots[slot]
        lbm, solid = drv.lbm, drv.solid
        moving = drv.config.coupling_mode == "moving_boundary"
        # the phases of FSIDriver3D.step_once outside the step: flush a pending
        # open boundary (none here), make the readout state current
        lbm.flush_open_boundary()
        solid._ensure_binned()
        if not solid._binned_clean or solid._binned_mode != "seq":
            for b in range(3):
                for t in solid._buffers(b):
                    t.zero_()
            solid._bins["t"]["meta"][1:].zero_()
            solid._binned_last, solid._binned_clean, solid._binned_mode = None, True, "seq"
        if moving:
            coupler = drv.mb_coupler if drv.mb_coupler is not None else drv.link_area_coupler
            mode = FSI_MODE_MOVING_BB | FSI_MODE_DIRSTATS
        else:
            coupler = drv.penalty_coupler
            pc = drv.penalty_coupler
            lbm._penalty = (pc.beta_lbm, pc.phi_min, pc.force_cap_lbm)
            mode = FSI_MODE_PENALTY
        lbm._sync_params()
        coupler.binned_stats.t.zero_()
        rec = FsiBatchCase()
        rec.lbm = lbm.state
        rec.lp = lbm.params
        rec.ctl.parity, rec.ctl.bc_pending, rec.ctl.pp, rec.ctl.mode = lbm.parity, 0, lbm.pp, mode
        rec.pt = solid.particles
        for b in range(3):
            rec.grid[b] = solid._bins["grids"][b]
        rec.bins = solid._bins["struct"]
        rec.mp = solid.params
        rec.cp = coupler.params
        rec.proj_stats = drv.projector.stats.t.data_ptr()
        rec.react_stats = coupler.binned_stats.t.data_ptr()
        rec.mask_threshold = float(drv.config.dynamic_solid_threshold)
        rec.mode = FSI_BATCH_MOVING if moving else FSI_BATCH_PENALTY
        rec.active = 1
        self.records[slot] = rec
        self._coupler = getattr(self, "_coupler", {})
        self._coupler[slot] = coupler
        self._upload(slot)
        self._update_dims()

    def _upload(self, slot):
        size = ctypes.sizeof(FsiBatchCase)
        raw = ctypes.string_at(ctypes.addressof(self.records[slot]), size)
        host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
        self.t_cases[slot * size:(slot + 1) * size].copy_(host)

    def _update_dims(self):
        d = self.dims
        act = [drv for drv in self.slots if drv is not None]
        d.n_cases = self.capacity
        d.store_fp16 = int(self.storage == "fp16")
        d.mpm_ctas = int(self.mpm_ctas)
        all_even = all(x.lbm.nx % 2 == 0 for x in act)
        if self.lbm_tune is None:
            d.lbm_tune = FSI_TUNE_LBM_OCC3  # the faster of the two on B200 (see profiles/)
        else:
            if self.lbm_tune == FSI_TUNE_LBM_PAIR and not all_even:
                raise ValueError("the paired LBM kernel needs an even nx in every case")
            d.lbm_tune = int(self.lbm_tune)
        if not act:
            d.max_lbm_tiles = d.max_particles = d.max_chunks = d.max_bins = 1
            d.max_cells = 1
            return
        d.max_lbm_tiles = max(((l.nx + 31) // 32) * ((l.ny + 7) // 8) * l.nz for l in (x.lbm for x in act))
        d.max_cells = max(x.lbm.ncell for x in act)
        d.max_particles = max(x.solid.n_particles for x in act)
        d.max_chunks = max(x.solid._bins["struct"].max_chunks for x in act)
        d.max_bins = max(x.solid._bins["struct"].n_bins for x in act)

    # ---------------------------------------------------------- stepping
    def _ptr(self):
        return ctypes.c_void_p(self.t_cases.data_ptr())

    def step_eager(self):
        """One FSI step of every active case (six batched calls + M substeps)."""
        st = stream_handle()
        d = ctypes.byref(self.dims)
        call("fsi_batch_project", self._ptr(), d, st)
        call("fsi_batch_mask_rebuild", self._ptr(), d, st)
        call("fsi_batch_lbm_substep", self._ptr(), d, st)
        call("fsi_batch_mpm_bin", self._ptr(), d, st)
        call("fsi_batch_mpm_substeps", self._ptr(), d, self.M, st)

    def capture(self):
        """Capture one batched FSI step in a CUDA graph (for the current slots)."""
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        n0 = launch_count()
        with torch.cuda.graph(g):
            self.step_eager()
        self.graph_kernels = launch_count() - n0
        self.graph = g
        return g

    def step(self, use_graph=True):
        if use_graph:
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self.step_eager()
        for i, drv in enumerate(self.slots):
            if drv is not None:
                self.steps_done[i] += 1

    def invalidate_graph(self):
        """Slot changes alter the launch geometry: recapture on the next step."""
        self.graph = None

    # ---------------------------------------------------------- readout
    def sync_case(self, slot):
        """Bring the Python-side mirrors of the case's driver up to date with the
        device records (call after steps, before reading its fields)."""
        drv = self.slots[slot]
        if drv is None:
            return None
        size = ctypes.sizeof(FsiBatchCase)
        raw = self.t_cases[slot * size:(slot + 1) * size].cpu().numpy().tobytes()
        rec = FsiBatchCase.from_buffer_copy(raw)
        lbm, solid = drv.lbm, drv.solid
        k = self.steps_done[slot]
        lbm.parity, lbm.pp = int(rec.ctl.parity), int(rec.ctl.pp)
        lbm.last_pp = lbm.pp ^ 1
        lbm.bc_pending = False
        lbm._penalty = None
        lbm._hydro_src = lbm.last_pp if rec.mode == FSI_BATCH_MOVING else "hydro"
        lbm._old_equals_solid = False
        lbm.steps += k - getattr(lbm, "_batch_steps_seen", 0)
        lbm._batch_steps_seen = k
        lbm._version += 1
        if k > 0 and self.M > 0:
            solid._binned_last = (self.M - 1) % 3
        solid._since_bin = 0
        coupler = self._coupler[slot]
        if k > 0 and self.M > 0:
            coupler._binned_slot = (self.M - 1) % 3
        drv.current_lbm_step = k
        drv.total_lbm_substeps = k
        drv.total_mpm_substeps = k * self.M
        return drv

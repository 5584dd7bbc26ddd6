"""MPMSolid3D: the reference's MLS-MPM solid on B200 kernels.

Same constructor (MPMConfig, n_particles), fields and methods as
src/mpm_lbm/sim/mpm/solid.py:11-419.  Particle state lives in planar device
tensors ([comp][n]); the MPM grid is n_grid^3, x fastest.
"""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from ._lib import (FsiCouplingStats, FsiGrid, FsiMpmBins, FsiMpmParams, FsiParticles, call,
                   ptr, stream_handle)
from .config import MPMConfig
from .fields import ParticleField


class _GridField:
    """grid_v / grid_m / grid_f_ext in the reference shape (n, n, n[, 3]).

    get() returns the tensor holding the reference's values; for_write()
    returns the tensor a write must go to (the one-phase grid)."""

    def __init__(self, get, n, comps, for_write=None):
        self._get, self.ng, self.comps = get, n, comps
        self._for_write = for_write if for_write is not None else get

    @property
    def shape(self):
        return (self.ng,) * 3

    def to_numpy(self):
        t = self._get()
        g = self.ng
        if self.comps:
            return t.reshape(self.comps, g, g, g).permute(3, 2, 1, 0).contiguous().cpu().numpy()
        return t.reshape(g, g, g).permute(2, 1, 0).contiguous().cpu().numpy()

    def from_numpy(self, arr):
        t = self._for_write()
        a = torch.as_tensor(np.ascontiguousarray(arr), device=t.device)
        if self.comps:
            t.copy_(a.permute(3, 2, 1, 0).reshape(t.shape).to(t.dtype))
        else:
            t.copy_(a.permute(2, 1, 0).reshape(t.shape).to(t.dtype))


class MPMSolid3D:
    def __init__(self, config: MPMConfig, n_particles: int, device=None):
        if n_particles <= 0:
            raise ValueError("n_particles must be positive")
        if config.mpm_planar_constraint_mode not in ("disabled", "lock_z"):
            raise ValueError("mpm_planar_constraint_mode must be one of ('disabled', 'lock_z')")
        if config.mpm_planar_constraint_axis != "z":
            raise ValueError("mpm_planar_constraint_axis currently supports only z")
        if config.mpm_velocity_damping < 0.0:
            raise ValueError("mpm_velocity_damping must be non-negative")
        if config.mpm_damping_application not in ("disabled", "particle_velocity_post_g2p"):
            raise ValueError("mpm_damping_application must be one of ('disabled', 'particle_velocity_post_g2p')")
        if config.mpm_damping_application == "disabled" and config.mpm_velocity_damping != 0.0:
            raise ValueError("mpm_velocity_damping must be 0 when damping is disabled")
        self.config = config
        self.dim = 3
        self.n_grid = int(config.n_grid)
        self.dx = float(config.dx)
        self.inv_dx = 1.0 / self.dx
        self.dt = float(config.dt)
        self.n_particles = int(n_particles)
        self.bound = int(config.bound)
        self.use_apic = config.use_apic
        self.gravity_x, self.gravity_y, self.gravity_z = (float(g) for g in config.gravity)
        self.box_min_x, self.box_min_y, self.box_min_z = config.box_min
        self.box_max_x, self.box_max_y, self.box_max_z = config.box_max
        self.young_modulus, self.poisson_ratio = config.young_modulus, config.poisson_ratio
        self.mu = config.young_modulus / (2.0 * (1.0 + config.poisson_ratio))
        self.la = config.young_modulus * config.poisson_ratio / ((1.0 + config.poisson_ratio) *
                                                                 (1.0 - 2.0 * config.poisson_ratio))
        box_volume = np.prod([b - a for a, b in zip(config.box_min, config.box_max)])
        self.p_vol0 = float(box_volume) / float(n_particles)
        self.p_mass0 = self.p_vol0 * config.p_rho
        self.particles_per_axis = max(1, math.ceil(n_particles ** (1.0 / 3.0)))
        self.mpm_planar_lock_z_enabled = 1 if config.mpm_planar_constraint_mode == "lock_z" else 0
        self.mpm_damping_enabled = 1 if config.mpm_damping_application == "particle_velocity_post_g2p" else 0
        self.mpm_velocity_damping = float(config.mpm_velocity_damping)
        self.device = torch.device(device if device is not None else "cuda")
        n, dev = self.n_particles, self.device
        f32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)  # noqa: E731
        self.t_x, self.t_v = f32(3, n), f32(3, n)
        self.t_C, self.t_F = f32(9, n), f32(9, n)
        self.t_F[0].fill_(1.0)
        self.t_F[4].fill_(1.0)
        self.t_F[8].fill_(1.0)
        self.t_Jp, self.t_mass, self.t_vol0 = torch.ones(n, device=dev), f32(n), f32(n)
        self.t_fixed = torch.zeros(n, dtype=torch.uint8, device=dev)
        self.t_fixed_x = f32(3, n)
        G = self.n_grid ** 3
        self.t_gv, self.t_gm, self.t_gf = f32(3, G), f32(G), f32(3, G)
        self.particles = FsiParticles(n=n, x=ptr(self.t_x), v=ptr(self.t_v), C=ptr(self.t_C), F=ptr(self.t_F),
                                      Jp=ptr(self.t_Jp), mass=ptr(self.t_mass), vol0=ptr(self.t_vol0),
                                      fixed=ptr(self.t_fixed), fixed_x=ptr(self.t_fixed_x))
        self.grid = FsiGrid(n=self.n_grid, v=ptr(self.t_gv), m=ptr(self.t_gm), f_ext=ptr(self.t_gf))
        self.params = FsiMpmParams(dx=self.dx, inv_dx=self.inv_dx, dt=self.dt, mu=self.mu, la=self.la,
                                   damping=self.mpm_velocity_damping if self.mpm_damping_enabled else 0.0,
                                   bound=self.bound, lock_z=self.mpm_planar_lock_z_enabled)
        self.params.gravity[:] = [self.gravity_x, self.gravity_y, self.gravity_z]
        self.x = ParticleField(lambda: self.t_x, (3,), np.float32, name="x")
        self.v = ParticleField(lambda: self.t_v, (3,), np.float32, name="v")
        self.C = ParticleField(lambda: self.t_C, (3, 3), np.float32, name="C")
        self.F = ParticleField(lambda: self.t_F, (3, 3), np.float32, name="F")
        self.Jp = ParticleField(lambda: self.t_Jp, (), np.float32, name="Jp")
        self.mass = ParticleField(lambda: self.t_mass, (), np.float32, name="mass")
        self.vol0 = ParticleField(lambda: self.t_vol0, (), np.float32, name="vol0")
        self.fixed_mask = ParticleField(lambda: self.t_fixed, (), np.int8, name="fixed_mask")
        self.fixed_x = ParticleField(lambda: self.t_fixed_x, (3,), np.float32, name="fixed_x")
        self.grid_v = _GridField(self._grid_velocity, self.n_grid, 3, lambda: self._one_phase_grid()[0])
        self.grid_m = _GridField(lambda: self._last_grid()[1], self.n_grid, 0, lambda: self._one_phase_grid()[1])
        self.grid_f_ext = _GridField(lambda: self._last_grid()[2], self.n_grid, 3, lambda: self._one_phase_grid()[2])
        # binned substeps (fsi_mpm_substeps_binned): three grid buffers and bins, made on first use
        self._bins = None
        self._binned_last = None  # buffer of the last binned substep while the grid holds its result
        self._binned_clean = True  # the buffers are zero outside the recorded boxes
        self._binned_mode = "seq"
        self._since_bin = 0
        self.rebin_interval = 64  # binned substeps between automatic re-binnings

    def _stream(self):
        return stream_handle()

    # solid.py:126-159 (deterministic lattice of particles in the box)
    def init_box(self):
        ppa = self.particles_per_axis
        p = np.arange(self.n_particles)
        idx = np.stack([p % ppa, (p // ppa) % ppa, (p // (ppa * ppa)) % ppa], axis=1).astype(np.float32)
        denom = np.float32(max(1, ppa - 1) + 1)
        local = (idx + np.float32(0.5)) / denom
        bmin = np.array([self.box_min_x, self.box_min_y, self.box_min_z], dtype=np.float32)
        span = np.array([self.box_max_x - self.box_min_x, self.box_max_y - self.box_min_y,
                         self.box_max_z - self.box_min_z], dtype=np.float32)
        x = bmin + span * local
        self.x.from_numpy(x)
        self.fixed_x.from_numpy(x)
        self.t_v.zero_()
        self.reset_deformation_state()
        self.t_mass.fill_(self.p_mass0)
        self.t_vol0.fill_(self.p_vol0)
        self.t_fixed.zero_()

    def reset_deformation_state(self):
        self.t_C.zero_()
        self.t_F.zero_()
        self.t_F[0].fill_(1.0)
        self.t_F[4].fill_(1.0)
        self.t_F[8].fill_(1.0)
        self.t_Jp.fill_(1.0)

    # solid.py:168-210
    def init_from_numpy(self, x_np, vol0_np, mass_np, v_np=None, fixed_mask_np=None):
        n = self.n_particles
        x = np.asarray(x_np, dtype=np.float32)
        vol = np.asarray(vol0_np, dtype=np.float32)
        mass = np.asarray(mass_np, dtype=np.float32)
        if x.shape != (n, 3):
            raise ValueError(f"x_np must have shape ({n}, 3)")
        if vol.shape != (n,):
            raise ValueError(f"vol0_np must have shape ({n},)")
        if mass.shape != (n,):
            raise ValueError(f"mass_np must have shape ({n},)")
        v = np.zeros_like(x) if v_np is None else np.asarray(v_np, dtype=np.float32)
        if v.shape != (n, 3):
            raise ValueError(f"v_np must have shape ({n}, 3)")
        fixed = np.zeros(n, np.int8) if fixed_mask_np is None else np.asarray(fixed_mask_np, dtype=np.int8)
        if fixed.shape != (n,):
            raise ValueError(f"fixed_mask_np must have shape ({n},)")
        if not np.all(np.isfinite(x)):
            raise ValueError("x_np must be finite")
        if not np.all(np.isfinite(v)):
            raise ValueError("v_np must be finite")
        if not np.all((fixed == 0) | (fixed == 1)):
            raise ValueError("fixed_mask_np must contain only 0/1 values")
        if not np.all(np.isfinite(vol)) or np.any(vol <= 0.0):
            raise ValueError("vol0_np must be finite and positive")
        if not np.all(np.isfinite(mass)) or np.any(mass <= 0.0):
            raise ValueError("mass_np must be finite and positive")
        self.x.from_numpy(x)
        self.v.from_numpy(v)
        self.vol0.from_numpy(vol)
        self.mass.from_numpy(mass)
        self.fixed_x.from_numpy(x)
        self.fixed_mask.from_numpy(fixed)
        self.reset_deformation_state()
        self.apply_fixed_particle_constraints()

    def apply_fixed_particle_constraints(self):  # solid.py:331-339
        m = self.t_fixed != 0
        self.t_x[:, m] = self.t_fixed_x[:, m]
        self.t_v[:, m] = 0.0
        self.t_C[:, m] = 0.0
        eye = torch.eye(3, device=self.device).reshape(9, 1)
        self.t_F[:, m] = eye.expand(9, int(m.sum().item())) if bool(m.any()) else self.t_F[:, m]
        self.t_Jp[m] = 1.0

    def set_uniform_velocity(self, vx, vy, vz):  # solid.py:323-329
        self.t_v[0].fill_(float(vx))
        self.t_v[1].fill_(float(vy))
        self.t_v[2].fill_(float(vz))
        self.t_v[:, self.t_fixed != 0] = 0.0

    def clear_grid(self):
        self._one_phase_grid()
        self.t_gv.zero_()
        self.t_gm.zero_()
        self.t_gf.zero_()

    def p2g(self):
        self._one_phase_grid()
        call("fsi_mpm_p2g", ctypes.byref(self.particles), ctypes.byref(self.grid), ctypes.byref(self.params),
             self._stream())

    def grid_update(self):
        self._one_phase_grid()
        call("fsi_mpm_grid_update", ctypes.byref(self.grid), ctypes.byref(self.params), self._stream())

    def g2p(self):
        self._one_phase_grid()
        call("fsi_mpm_g2p", ctypes.byref(self.particles), ctypes.byref(self.grid), ctypes.byref(self.params),
             self._stream())

    def substep(self):
        self.clear_grid()
        self.p2g()
        self.grid_update()
        self.g2p()

    # ---- binned substep -------------------------------------------------
    def _ensure_binned(self):
        if self._bins is not None:
            return
        nb, mc = ctypes.c_int32(), ctypes.c_int32()
        call("fsi_mpm_bins_layout", self.n_particles, self.n_grid, ctypes.byref(nb), ctypes.byref(mc))
        dev, n, G = self.device, self.n_particles, self.n_grid ** 3
        i32 = lambda *s: torch.zeros(*s, dtype=torch.int32, device=dev)  # noqa: E731
        f32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)  # noqa: E731
        t = {"key": i32(n), "count": i32(nb.value), "start": i32(nb.value), "perm": i32(n),
             "chunk": i32(mc.value, 2), "box": i32(3, mc.value, 6), "meta": i32(8)}
        self.t_gv1, self.t_gm1, self.t_gf1 = f32(3, G), f32(G), f32(3, G)
        self.t_gv2, self.t_gm2, self.t_gf2 = f32(3, G), f32(G), f32(3, G)
        grids = (FsiGrid * 3)()
        grids[0] = self.grid
        grids[1] = FsiGrid(n=self.n_grid, v=ptr(self.t_gv1), m=ptr(self.t_gm1), f_ext=ptr(self.t_gf1))
        grids[2] = FsiGrid(n=self.n_grid, v=ptr(self.t_gv2), m=ptr(self.t_gm2), f_ext=ptr(self.t_gf2))
        bins = FsiMpmBins(n_bins=nb.value, max_chunks=mc.value, **{k: ptr(v) for k, v in t.items()})
        self._bins = {"t": t, "grids": grids, "struct": bins}
        self._binned_clean = True
        self._since_bin = None

    def _buffers(self, b):
        return ((self.t_gv, self.t_gm, self.t_gf), (self.t_gv1, self.t_gm1, self.t_gf1),
                (self.t_gv2, self.t_gm2, self.t_gf2))[b]

    def _last_grid(self):
        """(momentum or velocity, mass, f_ext) tensors of the last grid state."""
        return self._buffers(self._binned_last) if self._binned_last is not None else (self.t_gv, self.t_gm, self.t_gf)

    def _grid_velocity(self):
        if self._binned_last is None:
            return self.t_gv
        b = self._binned_last
        out = torch.empty_like(self.t_gv)
        call("fsi_mpm_grid_velocity", ctypes.byref(self._bins["grids"][b]), ctypes.byref(self.params), ptr(out),
             self._stream())
        return out

    def _one_phase_grid(self):
        """Switch the grid to the one-phase layout (buffer 0 holds grid_v as
        velocity), materialising the last binned substep's grid first."""
        if self._binned_last is not None:
            v = self._grid_velocity()
            m, f = self._last_grid()[1:]
            self.t_gv.copy_(v)
            if self._binned_last != 0:
                self.t_gm.copy_(m)
                self.t_gf.copy_(f)
            self._binned_last = None
        self._binned_clean = False
        return self.t_gv, self.t_gm, self.t_gf

    # ---- state snapshots (trial substeps, e.g. autotuning) ----------------
    _SNAPSHOT = ("t_x", "t_v", "t_C", "t_F", "t_Jp", "t_gv", "t_gm", "t_gf")
    _SNAPSHOT_ATTRS = ("_binned_last", "_binned_clean", "_binned_mode", "_since_bin")

    def snapshot(self, extra=()):
        """Device copies of the mutable particle, grid and bin state (plus the
        given extra tensors)."""
        names = list(self._SNAPSHOT)
        if self._bins is not None:
            names += ["t_gv1", "t_gm1", "t_gf1", "t_gv2", "t_gm2", "t_gf2"]
        tensors = {k: getattr(self, k).clone() for k in names}
        bins = {} if self._bins is None else {k: v.clone() for k, v in self._bins["t"].items()}
        return (tensors, bins, [(t, t.clone()) for t in extra], {k: getattr(self, k) for k in self._SNAPSHOT_ATTRS})

    def restore(self, snap):
        tensors, bins, extra, attrs = snap
        for k, t in tensors.items():
            getattr(self, k).copy_(t)
        for k, t in bins.items():
            self._bins["t"][k].copy_(t)
        for t, c in extra:
            t.copy_(c)
        for k, v in attrs.items():
            setattr(self, k, v)

    def rebin(self):
        """Sort particle ids by 8x8x8 block of base cells, and by base cell
        within a block (fsi_mpm_bin)."""
        self._ensure_binned()
        call("fsi_mpm_bin", ctypes.byref(self.particles), ctypes.byref(self.grid), ctypes.byref(self.params),
             ctypes.byref(self._bins["struct"]), self._stream())
        self._since_bin = 0

    def substep_binned(self, coupler=None, lbm=None):
        """One substep through the binned path: the same update as substep()
        (plus the coupler's reaction transfer when given, as the driver's MPM
        loops call it), with binned, shared-memory-staged P2G."""
        self.substeps_binned(1, coupler, lbm)

    def substeps_binned(self, count, coupler=None, lbm=None):
        """`count` substeps through fsi_mpm_substeps_binned (one launch per
        substep: the gather of one substep, the stress, reaction and scatter
        of the next), re-binning first when the bins are due."""
        if count <= 0:
            return
        self._ensure_binned()
        if self._binned_mode != "seq" or not self._binned_clean:
            for b in range(3):
                for t in self._buffers(b):
                    t.zero_()
            self._bins["t"]["meta"][1:].zero_()  # no recorded boxes; the chunk table stays valid
            self._binned_last, self._binned_clean, self._binned_mode = None, True, "seq"
        if self._since_bin is None or self._since_bin >= self.rebin_interval:
            self.rebin()
        if coupler is not None:
            state, hydro, cp, stats = coupler._binned_args(lbm)
            args = (ctypes.byref(state), ptr(hydro), ctypes.byref(cp), stats)
        else:
            args = (None, None, None, None)
        call("fsi_mpm_substeps_binned", ctypes.byref(self.particles), self._bins["grids"],
             ctypes.byref(self._bins["struct"]), ctypes.byref(self.params), int(count), *args, self._stream())
        last = (count - 1) % 3
        if coupler is not None:
            coupler._binned_slot = last
        self._binned_last = last
        self._since_bin += count

    def inside_grid(self, I):
        return all(0 <= int(i) < self.n_grid for i in I)

    # solid.py:341-375 (reductions on the device)
    def get_stats(self):
        x, v, J, m = self.t_x, self.t_v, self.t_Jp, self.t_mass
        sp = torch.linalg.vector_norm(v.double(), dim=0)
        vals = torch.cat([x.min(dim=1).values.double(), x.max(dim=1).values.double(),
                          torch.stack([sp.max(), J.min().double(), J.max().double(), m.double().sum()])]).cpu().tolist()
        return {"min_x": tuple(vals[0:3]), "max_x": tuple(vals[3:6]), "min_y": vals[1], "max_y": vals[4],
                "max_speed": vals[6], "min_J": vals[7], "max_J": vals[8], "total_mass": vals[9]}

    def get_fixed_particle_stats(self):
        mask = self.fixed_mask.to_numpy().astype(bool)
        count = int(np.count_nonzero(mask))
        if count == 0:
            return {"fixed_base_constraint_applied": False, "fixed_base_particle_count": 0,
                    "fixed_base_max_displacement_norm": 0.0, "fixed_base_max_velocity_norm": 0.0}
        x, fx, v = self.x.to_numpy(), self.fixed_x.to_numpy(), self.v.to_numpy()
        return {"fixed_base_constraint_applied": True, "fixed_base_particle_count": count,
                "fixed_base_max_displacement_norm": float(np.max(np.linalg.norm(x[mask] - fx[mask], axis=1))),
                "fixed_base_max_velocity_norm": float(np.max(np.linalg.norm(v[mask], axis=1)))}

    def export_particles(self, out_dir: str, prefix: str = "particles"):
        os.makedirs(out_dir, exist_ok=True)
        np.save(os.path.join(out_dir, f"{prefix}_x.npy"), self.x.to_numpy())
        np.save(os.path.join(out_dir, f"{prefix}_v.npy"), self.v.to_numpy())
        np.save(os.path.join(out_dir, f"{prefix}_F.npy"), self.F.to_numpy())
        np.save(os.path.join(out_dir, f"{prefix}_J.npy"), self.Jp.to_numpy())

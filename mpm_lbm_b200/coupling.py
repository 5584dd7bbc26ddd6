"""MPM <-> LBM couplers on B200 kernels, with the reference's class names and
methods (src/mpm_lbm/sim/coupling/{projection,penalty,moving_boundary,
link_area,link_area_accounting}.py)."""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import FsiCouplingParams, FsiCouplingStats, FsiProjectScratch, call, ptr, stream_handle

AREA_POLICIES = ("uniform", "inverse_length", "length")


class _StatsBuffer:
    """count consecutive FsiCouplingStats records on the device."""

    def __init__(self, device, count=1):
        size = ctypes.sizeof(FsiCouplingStats)
        self.t = torch.zeros((size * count + 255) // 256 * 256, dtype=torch.uint8, device=device)

    def read(self, i=0) -> FsiCouplingStats:
        size = ctypes.sizeof(FsiCouplingStats)
        return FsiCouplingStats.from_buffer_copy(self.t[i * size: (i + 1) * size].cpu().numpy().tobytes())

    def ptr(self):
        return ptr(self.t)


class _BinnedReaction:
    """Reaction transfer fused into MPMSolid3D.substeps_binned: the kernel
    writes the reductions of a substep with grid buffer b to record b."""

    def _init_binned(self, device):
        self.binned_stats = _StatsBuffer(device, count=3)
        self._binned_slot = None

    def _binned_args(self, lbm):
        self._lbm = lbm
        return lbm.state, lbm._hydro_tensor(), self.params, self.binned_stats.ptr()

    def _reaction_stats(self) -> FsiCouplingStats:
        if self._binned_slot is not None:
            return self.binned_stats.read(self._binned_slot)
        return self.stats.read()


def _base_params(sim_config):
    cp = FsiCouplingParams()
    dx = float(sim_config.dx_norm)
    dt = float(sim_config.lbm_dt_phys)
    cp.inv_dx_norm = 1.0 / dx
    cp.cell_volume_norm = dx ** 3
    cp.vel_scale = dt / dx
    cp.eps_mass = 1.0e-12
    cp.force_density_scale = dx / (dt ** 2)
    return cp


class MPMToLBMProjector3D:
    """projection.py:5-111."""

    def __init__(self, sim_config, device=None):
        self.n_grid = sim_config.n_grid
        self.dx_norm = sim_config.dx_norm
        self.inv_dx_norm = 1.0 / sim_config.dx_norm
        self.cell_volume_norm = sim_config.dx_norm ** 3
        self.vel_scale_norm_to_lbm = sim_config.lbm_dt_phys / sim_config.dx_norm
        self.eps_mass = 1.0e-12
        self.params = _base_params(sim_config)
        self.stats = _StatsBuffer(device if device is not None else "cuda")
        self._scratch = None
        self._scratch_t = None

    def _ordered_scratch(self, lbm, solid):
        """Device scratch of fsi_project_ordered, allocated on first use (the
        driver's first FSI step runs eagerly, before any graph capture)."""
        keys = (lbm.nx + 2) * (lbm.ny + 2) * (lbm.nz + 2)
        n = int(solid.n_particles)
        sc = self._scratch
        if sc is None or sc.key_capacity < keys or sc.particle_capacity < n:
            dev = lbm.device
            t = {"count": torch.zeros(keys + 1, dtype=torch.int32, device=dev),
                 "start": torch.empty(keys + 1, dtype=torch.int32, device=dev),
                 "list": torch.empty(max(n, 1), dtype=torch.int32, device=dev),
                 "key": torch.empty(max(n, 1), dtype=torch.int32, device=dev),
                 "box": torch.empty(8, dtype=torch.int32, device=dev)}
            sc = FsiProjectScratch()
            sc.key_capacity, sc.particle_capacity = keys, n
            for k, v in t.items():
                setattr(sc, k, v.data_ptr())
            self._scratch, self._scratch_t = sc, t
        return sc

    def project(self, solid, lbm, clear=True):
        """projection.py:21-97 with every cell's sums in particle order
        (fsi_project_ordered): the same bits as a serial run of the
        reference's loop, on every run."""
        if not clear:
            raise NotImplementedError("projection without clearing is not supported")
        sc = self._ordered_scratch(lbm, solid)
        call("fsi_project_ordered", ctypes.byref(lbm.state), ctypes.byref(solid.particles),
             ctypes.byref(self.params), ctypes.byref(sc), self.stats.ptr(), stream_handle())
        lbm._version += 1

    def project_unordered(self, solid, lbm):
        """The same projection with float atomics (fsi_project): the sums'
        order, and so their last bits, vary from run to run."""
        call("fsi_project", ctypes.byref(lbm.state), ctypes.byref(solid.particles), ctypes.byref(self.params),
             self.stats.ptr(), stream_handle())
        lbm._version += 1

    def get_stats(self):
        s = self.stats.read()
        return {"projected_mass": float(s.projected_mass), "projected_volume_raw": float(s.projected_volume_raw),
                "projected_volume_clamped": float(s.projected_volume_clamped), "max_phi_raw": float(s.max_phi_raw),
                "active_cell_count": int(s.active_cell_count),
                "vel_scale_norm_to_lbm": float(self.vel_scale_norm_to_lbm),
                "cell_volume_norm": float(self.cell_volume_norm)}


class PenaltyFSICoupler3D(_BinnedReaction):
    """penalty.py:5-152.  The penalty force is built inside the next LBM step
    from the same macroscopic state the reference uses (the step's fused
    prologue), so build_penalty_force() only arms it."""

    def __init__(self, sim_config, beta_lbm=1.0e-3, phi_min=1.0e-6, force_cap_lbm=1.0e-4, reaction_scale=1.0,
                 device=None):
        if beta_lbm <= 0.0:
            raise ValueError("beta_lbm must be positive")
        if phi_min < 0.0:
            raise ValueError("phi_min must be non-negative")
        if force_cap_lbm <= 0.0:
            raise ValueError("force_cap_lbm must be positive")
        if reaction_scale <= 0.0:
            raise ValueError("reaction_scale must be positive")
        self.n_grid = sim_config.n_grid
        self.dx_norm = sim_config.dx_norm
        self.inv_dx_norm = 1.0 / sim_config.dx_norm
        self.lbm_dt_phys = sim_config.lbm_dt_phys
        self.beta_lbm, self.phi_min = float(beta_lbm), float(phi_min)
        self.force_cap_lbm, self.reaction_scale = float(force_cap_lbm), float(reaction_scale)
        self.force_density_scale_lbm_to_norm = self.dx_norm / (self.lbm_dt_phys ** 2)
        self.params = _base_params(sim_config)
        self.params.kind = 0
        self.params.reaction_scale = self.reaction_scale
        self.stats = _StatsBuffer(device if device is not None else "cuda")
        self._init_binned(device if device is not None else "cuda")
        self._lbm = None

    def clear_force_fields(self, lbm):
        """Cells whose force vanishes are cleared by the step that builds the new force."""
        self._lbm = lbm

    def build_penalty_force(self, lbm):
        lbm._penalty = (self.beta_lbm, self.phi_min, self.force_cap_lbm)
        self._lbm = lbm

    def add_lbm_reaction_to_mpm_grid(self, solid, lbm):
        self._binned_slot = None
        call("fsi_reaction_to_grid", ctypes.byref(lbm.state), ptr(lbm._hydro_tensor()), ctypes.byref(solid.particles),
             ctypes.byref(solid.grid), ctypes.byref(self.params), self.stats.ptr(), stream_handle())

    def get_stats(self):
        s = self._reaction_stats()
        out = {"n_grid": self.n_grid, "dx_norm": self.dx_norm, "inv_dx_norm": self.inv_dx_norm,
               "lbm_dt_phys": self.lbm_dt_phys, "beta_lbm": self.beta_lbm, "phi_min": self.phi_min,
               "force_cap_lbm": self.force_cap_lbm, "reaction_scale": self.reaction_scale,
               "force_density_scale_lbm_to_norm": self.force_density_scale_lbm_to_norm,
               "max_reaction_grid_force_norm": float(s.max_grid_reaction_norm),
               "net_reaction_grid_force": tuple(float(v) for v in s.net_grid_reaction)}
        if self._lbm is not None:
            d = self._lbm._diag()
            net = tuple(float(v) for v in d.penalty_net)
            out.update({"active_force_cell_count": int(d.penalty_active),
                        "max_cell_force_norm": float(d.penalty_max_norm),
                        "max_hydro_force_norm": float(d.penalty_max_norm), "net_cell_force": net,
                        "net_hydro_force": tuple(-v for v in net)})
        return out


class MovingBoundaryFSICoupler3D(_BinnedReaction):
    """moving_boundary.py:5-130 (engineering reaction transfer)."""

    kind = 1

    def __init__(self, sim_config, reaction_scale=1.0, force_cap_norm=1.0e-2, phi_min=1.0e-6, device=None):
        if reaction_scale <= 0.0:
            raise ValueError("reaction_scale must be positive")
        if force_cap_norm <= 0.0:
            raise ValueError("force_cap_norm must be positive")
        if phi_min < 0.0:
            raise ValueError("phi_min must be non-negative")
        self.n_grid = sim_config.n_grid
        self.dx_norm = sim_config.dx_norm
        self.inv_dx_norm = 1.0 / sim_config.dx_norm
        self.lbm_dt_phys = sim_config.lbm_dt_phys
        self.reaction_scale, self.force_cap_norm, self.phi_min = float(reaction_scale), float(force_cap_norm), float(phi_min)
        self.force_density_scale_lbm_to_norm = self.dx_norm / (self.lbm_dt_phys ** 2)
        self.params = _base_params(sim_config)
        self.params.kind = self.kind
        self.params.reaction_scale = self.reaction_scale
        self.params.force_cap = self.force_cap_norm
        self.params.phi_min = self.phi_min
        self.stats = _StatsBuffer(device if device is not None else "cuda")
        self._init_binned(device if device is not None else "cuda")

    def clear_reaction_diagnostics(self):
        """The reaction entry point clears its reductions itself."""
        return None

    def _react(self, solid, lbm):
        self._binned_slot = None
        call("fsi_reaction_to_grid", ctypes.byref(lbm.state), ptr(lbm._hydro_tensor()), ctypes.byref(solid.particles),
             ctypes.byref(solid.grid), ctypes.byref(self.params), self.stats.ptr(), stream_handle())

    def add_moving_boundary_reaction_to_mpm_grid(self, solid, lbm):
        self._react(solid, lbm)

    def _common_stats(self):
        s = self._reaction_stats()
        return s, {"n_grid": self.n_grid, "dx_norm": self.dx_norm, "inv_dx_norm": self.inv_dx_norm,
                   "lbm_dt_phys": self.lbm_dt_phys, "reaction_scale": self.reaction_scale,
                   "force_cap_norm": self.force_cap_norm, "phi_min": self.phi_min,
                   "force_density_scale_lbm_to_norm": self.force_density_scale_lbm_to_norm,
                   "active_reaction_particle_count": int(s.active_reaction_particle_count),
                   "max_particle_reaction_norm": float(s.max_particle_reaction_norm),
                   "max_grid_reaction_norm": float(s.max_grid_reaction_norm),
                   "net_particle_reaction_force": tuple(float(v) for v in s.net_particle_reaction),
                   "net_grid_reaction_force": tuple(float(v) for v in s.net_grid_reaction)}

    def get_stats(self):
        return self._common_stats()[1]


class LinkAreaMovingBoundaryCoupler3D(MovingBoundaryFSICoupler3D):
    """link_area.py:10-221.  The global area scale is recomputed on the device
    from the last step's per-direction bounce-back reductions by the reaction
    kernel itself; update_area_scale_from_lbm() returns the host summary."""

    kind = 2

    def __init__(self, sim_config, area_policy="inverse_length", reaction_scale=1.0, force_cap_norm=1.0e-5,
                 phi_min=1.0e-6, area_scale_min=0.25, area_scale_max=2.0, device=None):
        if area_policy not in AREA_POLICIES:
            raise ValueError(f"area_policy must be one of {AREA_POLICIES}")
        if area_scale_min <= 0.0:
            raise ValueError("area_scale_min must be positive")
        if area_scale_max <= 0.0:
            raise ValueError("area_scale_max must be positive")
        if area_scale_min > area_scale_max:
            raise ValueError("area_scale_min must be <= area_scale_max")
        super().__init__(sim_config, reaction_scale=reaction_scale, force_cap_norm=force_cap_norm, phi_min=phi_min,
                         device=device)
        self.area_policy = area_policy
        self.area_scale_min, self.area_scale_max = float(area_scale_min), float(area_scale_max)
        self.params.area_policy = AREA_POLICIES.index(area_policy)
        self.params.area_scale_min = self.area_scale_min
        self.params.area_scale_max = self.area_scale_max

    def update_area_scale_from_lbm(self, lbm):
        d = lbm.get_moving_boundary_directional_stats()
        e = lbm.e.to_numpy().astype(np.float64)
        lengths = np.linalg.norm(e, axis=1)
        w = np.zeros(19)
        act = lengths > 0
        w[act] = {"uniform": 1.0, "inverse_length": 1.0 / lengths[act], "length": lengths[act]}[self.area_policy]
        solid_by_dir = np.asarray(d["solid_force_by_dir"], dtype=np.float64)
        weighted = np.sum(solid_by_dir * w[:, None], axis=0)
        scalar = np.asarray(lbm.get_moving_boundary_stats()["bb_net_solid_force"], dtype=np.float64)
        raw = abs(float(weighted[0])) / (abs(float(scalar[0])) + 1.0e-12)
        scale = float(np.clip(raw, self.area_scale_min, self.area_scale_max))
        if not np.isfinite(scale):
            scale = self.area_scale_min
        counts = np.asarray(d["link_count_by_dir"], dtype=np.int64)
        return {"policy": self.area_policy, "area_policy": self.area_policy, "raw_area_scale": raw,
                "area_scale": scale, "area_proxy_total": float(np.sum(counts * w)),
                "area_weighted_solid_force_x": float(weighted[0]), "area_weighted_solid_force_y": float(weighted[1]),
                "area_weighted_solid_force_z": float(weighted[2]), "bb_net_solid_force_x": float(scalar[0]),
                "total_link_count": int(counts.sum())}

    def add_link_area_reaction_to_mpm_grid(self, solid, lbm):
        self._react(solid, lbm)

    def get_stats(self):
        s, out = self._common_stats()
        out.update({"area_policy": self.area_policy, "area_scale_min": self.area_scale_min,
                    "area_scale_max": self.area_scale_max, "area_scale": float(s.area_scale),
                    "raw_area_scale": float(s.raw_area_scale)})
        return out

"""FSIDriver3D on B200 kernels: the reference's driver API
(src/mpm_lbm/sim/drivers/fsi_driver.py:61-858) over the CUDA objects of this
package.  Phase order per FSI step is the reference's
(fsi_driver.py:425-575); diagnostics rows carry the same keys
(DIAGNOSTIC_FIELDS, fsi_driver.py:27-53) and are reduced on the device.

Constructor extensions (keyword-only, outside FSIDriverConfig):
  population_storage  "fp32" (default) or "fp16" (deviation storage)
  collision           "mrt" (default, the reference's operator) or "bgk"
  lattice_shape       (nx, ny, nz) for a non-cubic lattice with dx = 1/nx
  material            {"young_modulus", "poisson_ratio", "p_rho"} MPM overrides
  device              torch device (default "cuda")
"""

from __future__ import annotations

import csv
import json
import os
import time

import numpy as np
import torch

from ._lib import launch_count
from .config import FSIDriverConfig, GridUnitMapper
from .coupling import (LinkAreaMovingBoundaryCoupler3D, MovingBoundaryFSICoupler3D, MPMToLBMProjector3D,
                       PenaltyFSICoupler3D)
from .geometry import GeometryConfig, duct_static_geometry, sample_particles
from .lbm import LBMFluid3D
from .mpm import MPMSolid3D

DIAGNOSTIC_FIELDS = [
    "step", "total_mpm_substeps", "coupling_mode", "rho_min", "rho_max", "lbm_max_v", "fluid_mean_ux",
    "projection_zone_fluid_mean_ux", "far_field_fluid_mean_ux", "solid_mean_vx_norm", "mpm_min_J", "mpm_max_speed",
    "projected_mass", "active_cell_count", "cell_force_max_norm", "hydro_force_max_norm", "bb_link_count",
    "bb_max_correction", "mb_subcycle_force_accumulation_mode", "mb_subcycle_force_sample_count",
    "mb_subcycle_force_accum_norm_max", "mb_subcycle_force_mean_norm_max", "active_reaction_particle_count",
    "max_grid_reaction_norm", "elapsed_seconds",
]
DIAGNOSTIC_TEXT_FIELDS = {"coupling_mode", "mb_subcycle_force_accumulation_mode"}


class FSIDriver3D:
    def __init__(self, config: FSIDriverConfig, out_dir: str, *, population_storage="fp32", collision="mrt",
                 lattice_shape=None, material=None, static_solid=None, initial_particles=None, use_cuda_graph=False,
                 mpm_path="binned", device=None):
        if mpm_path not in ("binned", "one_phase"):
            raise ValueError("mpm_path must be 'binned' (fsi_mpm_substeps_binned) or 'one_phase' (one kernel per phase)")
        self.mpm_path = mpm_path
        self.config = config
        self.out_dir = out_dir
        self.sim = config.make_unified_sim_config()
        self.mapper = GridUnitMapper.from_sim_config(self.sim)
        self.current_lbm_step = 0
        self.total_lbm_substeps = 0
        self.total_mpm_substeps = 0
        self.diagnostics_rows = []
        self.timing = {k: 0.0 for k in ("init_time", "projection_time", "coupling_time", "lbm_step_time",
                                         "mpm_substep_time", "diagnostics_time", "export_time",
                                         "wall_velocity_application_time", "geometry_motion_interface_time",
                                         "total_time")}
        self.population_storage = population_storage
        self.collision = collision
        self.lattice_shape = tuple(lattice_shape) if lattice_shape is not None else (config.n_grid,) * 3
        self.material = dict(material or {})
        self.device = torch.device(device if device is not None else "cuda")
        self.initialized = False
        self.start_time = None
        self.lbm = self.solid = self.projector = None
        self.penalty_coupler = self.mb_coupler = self.link_area_coupler = None
        self.initial_particle_positions = None
        self.free_tip_proxy_mask = None
        self.flap_tip_monitor_rows = []
        self.fluent_like_monitor_rows = []
        self.duct_static_geometry_report = None
        self.sampling_stats = None
        self.timed_sync = False  # synchronise around phases so the timing dict holds device time
        self.static_solid = None if static_solid is None else np.asarray(static_solid, np.int8)
        self.initial_particles = initial_particles
        self.use_cuda_graph = bool(use_cuda_graph)
        self._graph = None
        self._graph_steps = 0
        self._graph_warm = False
        self.graph_kernels_per_step = None
        self.tuning = None
        # wall velocity application (fsi_driver.py:458-482): the host builds the
        # phase grid (callables taking (application config, n_grid, phase) and
        # (application config, lbm_step), e.g. the reference's
        # build_wall_velocity_grid and phase_for_lbm_step); the device applies it
        self.wall_velocity_grid_builder = None
        self.wall_velocity_phase_for_step = None
        self.wall_velocity_application_report = None
        self.wall_velocity_application_reports = []

    # ------------------------------------------------------------ init
    def _geometry_config(self):
        if self.config.geometry_config_path is None:
            return None
        g = GeometryConfig.from_json(self.config.geometry_config_path)
        if g.geometry_type != self.config.geometry_type:
            raise ValueError("geometry_config_path geometry_type does not match FSIDriverConfig.geometry_type: "
                             f"{g.geometry_type} != {self.config.geometry_type}")
        if g.n_particles != self.config.n_particles:
            raise ValueError("geometry_config_path n_particles does not match FSIDriverConfig.n_particles: "
                             f"{g.n_particles} != {self.config.n_particles}")
        return g

    def _make_lbm_config(self):
        nx, ny, nz = self.lattice_shape
        over = dict(nx=nx, ny=ny, nz=nz, collision=self.collision, population_storage=self.population_storage)
        if self.config.lbm_boundary_condition_mode == "duct_velocity_inlet_pressure_outlet":
            t = tuple(float(v) for v in self.config.target_u_lbm)
            if self.config.velocity_inlet_side == "min":
                over.update(bc_x_left=2, bc_x_right=1, vel_bc_x_left=t, rho_bc_x_right=1.0)
            else:
                over.update(bc_x_left=1, bc_x_right=2, rho_bc_x_left=1.0, vel_bc_x_right=t)
        return self.sim.make_lbm_config(**over)

    def initialize(self):
        t0 = time.perf_counter()
        os.makedirs(self.out_dir, exist_ok=True)
        with open(os.path.join(self.out_dir, "driver_config.json"), "w", encoding="utf-8") as f:
            json.dump(self.config.to_dict(), f, indent=2)
        gcfg = self._geometry_config()
        nx, ny, nz = self.lattice_shape
        if self.static_solid is not None:
            if self.static_solid.shape != (nx, ny, nz):
                raise ValueError(f"static_solid shape {self.static_solid.shape} != lattice {(nx, ny, nz)}")
            solid = self.static_solid
        elif self.config.lbm_boundary_condition_mode == "duct_velocity_inlet_pressure_outlet":
            if gcfg is None or gcfg.geometry_type != "duct_flap_proxy":
                raise ValueError("duct_velocity_inlet_pressure_outlet requires duct_flap_proxy geometry_config")
            if self.lattice_shape != (self.config.n_grid,) * 3:
                raise ValueError("the duct geometry file path builds a cubic lattice")
            solid, self.duct_static_geometry_report = duct_static_geometry(self.config.n_grid, gcfg)
        else:
            solid = np.zeros((nx, ny, nz), np.int8)
        self.lbm = LBMFluid3D(self._make_lbm_config(), device=self.device)
        self.lbm.init_geo_array(solid)
        self.lbm.init_simulation()
        mpm_over = {"gravity": self.config.gravity, "box_min": self.config.box_min, "box_max": self.config.box_max}
        mpm_over.update(self.config.make_mpm_control_overrides())
        if gcfg is not None and gcfg.geometry_type == "duct_flap_proxy":
            mat = gcfg.material_reference or {}
            if bool(mat.get("used_for_mpm_config", False)):
                mpm_over.update(p_rho=float(mat["density"]), young_modulus=float(mat["youngs_modulus"]),
                                poisson_ratio=float(mat["poisson_ratio"]))
        mpm_over.update(self.material)
        self.solid = MPMSolid3D(self.sim.make_mpm_config(**mpm_over), n_particles=self.config.n_particles,
                                device=self.device)
        if self.initial_particles is not None:
            ip = self.initial_particles
            self.solid.init_from_numpy(ip["x"], ip["vol0"], ip["mass"], fixed_mask_np=ip.get("fixed"))
            self.initial_particle_positions = np.asarray(ip["x"], np.float32).copy()
            tip = ip.get("free_tip")
            self.free_tip_proxy_mask = None if tip is None else np.asarray(tip, bool)
        elif self.config.geometry_type == "box" and self.config.geometry_config_path is None:
            self.solid.init_box()
        else:
            cloud = sample_particles(gcfg)
            self.sampling_stats = dict(cloud["sampling_stats"])
            self.initial_particle_positions = np.asarray(cloud["x"], np.float32).copy()
            self.free_tip_proxy_mask = np.asarray(cloud.get("free_tip_proxy_mask",
                                                            np.zeros(self.config.n_particles, np.int8)), bool)
            self.solid.init_from_numpy(cloud["x"], cloud["vol0"], cloud["mass"],
                                       fixed_mask_np=cloud.get("fixed_base_mask"))
        v0 = self.config.initial_solid_velocity_norm
        self.solid.set_uniform_velocity(float(v0[0]), float(v0[1]), float(v0[2]))
        self._make_couplers()
        self.initialized = True
        self.start_time = time.perf_counter()
        self.timing["init_time"] += self.start_time - t0

    def _make_couplers(self):
        cfg, dev = self.config, self.device
        self.projector = MPMToLBMProjector3D(self.sim, device=dev)
        if cfg.coupling_mode == "penalty":
            self.penalty_coupler = PenaltyFSICoupler3D(self.sim, beta_lbm=cfg.beta_lbm,
                                                       force_cap_lbm=cfg.penalty_force_cap_lbm, device=dev)
        if cfg.coupling_mode == "moving_boundary" and cfg.reaction_transfer_mode == "engineering":
            self.mb_coupler = MovingBoundaryFSICoupler3D(self.sim, reaction_scale=cfg.mb_reaction_scale,
                                                         force_cap_norm=cfg.mb_force_cap_norm, phi_min=1.0e-6,
                                                         device=dev)
        if cfg.coupling_mode == "moving_boundary" and cfg.reaction_transfer_mode == "link_area_experimental":
            self.link_area_coupler = LinkAreaMovingBoundaryCoupler3D(
                self.sim, area_policy=cfg.link_area_policy, reaction_scale=cfg.mb_reaction_scale,
                force_cap_norm=cfg.mb_force_cap_norm, phi_min=1.0e-6, area_scale_min=cfg.link_area_scale_min,
                area_scale_max=cfg.link_area_scale_max, device=dev)

    def set_initial_state(self, solid=None, x=None, vol0=None, mass=None, fixed_mask=None, free_tip_mask=None,
                          velocity=None):
        """Replace the initial geometry / particle cloud after initialize() (the
        reference's callers do this with lbm.init_geo and solid.init_from_numpy)."""
        if solid is not None:
            self.lbm.init_geo_array(solid)
            self.lbm.init_simulation()
        if x is not None:
            self.solid.init_from_numpy(x, vol0, mass, v_np=velocity, fixed_mask_np=fixed_mask)
            self.initial_particle_positions = np.asarray(x, np.float32).copy()
            if free_tip_mask is not None:
                self.free_tip_proxy_mask = np.asarray(free_tip_mask, bool)

    # ------------------------------------------------------------ tuning
    def autotune(self):
        """Time the launch variants of the step kernels on this case's state and
        keep the fastest (results are identical across variants).  Drops a
        captured step graph so that the next step recaptures with the choice."""
        from .autotune import tune_lbm

        if not self.initialized:
            self.initialize()
        self._graph = None
        self._graph_steps = 0
        step = self.lbm.step_moving_bounceback if self.config.coupling_mode == "moving_boundary" else self.lbm.step
        # time the substep the FSI step runs most: subcycled steps produce the
        # per-direction reductions only on their last substep
        subcycled = self.config.fsi_exchange_mode == "lbm_subcycled_per_fsi_step"
        saved = self.lbm.dirstats_enabled
        self.lbm.dirstats_enabled = not subcycled
        try:
            self.tuning = {"lbm": tune_lbm(self.lbm, step)}
        finally:
            self.lbm.dirstats_enabled = saved
        return self.tuning

    # ------------------------------------------------------------ steps
    def _t(self, key, t0):
        if self.timed_sync:
            torch.cuda.synchronize()
        self.timing[key] += time.perf_counter() - t0

    def _graph_period(self):
        # the captured sequence must return the AA layout parity and the ping-pong slot to their
        # start values (the binned MPM substeps of every FSI step start from the same buffers)
        S = self.config.lbm_substeps_per_fsi_step if self.config.fsi_exchange_mode == "lbm_subcycled_per_fsi_step" else 1
        return 2 if S % 2 else 1

    def step_once(self):
        if not self.initialized:
            self.initialize()
        if self.use_cuda_graph and self.config.wall_velocity_application_mode == "disabled":
            self._step_graph()
            return
        self._step_eager()

    def _step_graph(self):
        """Replay a CUDA graph of whole FSI steps (captured after one eager step)."""
        if self._graph is None and not self._graph_warm:
            # warm-up: allocates lazily created buffers (bins, grid buffers, readout
            # arrays) outside any capture, and leaves bc_pending set; also the first
            # step of a driver restored from a restart file
            self._step_eager()
            self._graph_warm = True
            return
        period = self._graph_period()
        if self._graph is None:
            if self.current_lbm_step % period:
                self._step_eager()
                return
            torch.cuda.synchronize()
            snap = self._counters()
            g = torch.cuda.CUDAGraph()
            n0 = launch_count()
            with torch.cuda.graph(g):
                for _ in range(period):
                    self._step_eager()
            # this library's kernels per replayed FSI step (torch's own fills/copies not included)
            self.graph_kernels_per_step = (launch_count() - n0) / period
            self._graph_delta = tuple(b - a for a, b in zip(snap, self._counters()))
            self._restore_counters(snap)
            self._graph = g
            self._graph_steps = 0
        if self._graph_steps == 0:
            self._graph.replay()
            self.lbm._version += 1  # device state advanced outside Python: invalidate readout caches
            self._graph_steps = period
        self._graph_steps -= 1
        d = self._graph_delta
        self.current_lbm_step += 1
        self.total_lbm_substeps += d[1] // period
        self.total_mpm_substeps += d[2] // period

    def _counters(self):
        return (self.current_lbm_step, self.total_lbm_substeps, self.total_mpm_substeps)

    def _restore_counters(self, snap):
        self.current_lbm_step, self.total_lbm_substeps, self.total_mpm_substeps = snap

    def _step_eager(self):
        if self.config.fsi_exchange_mode == "lbm_subcycled_per_fsi_step":
            if self.config.coupling_mode != "moving_boundary":
                raise ValueError("subcycled FSI exchange currently supports only moving_boundary coupling")
            self._step_moving_boundary_subcycled()
            self.current_lbm_step += 1
            return
        mode = self.config.coupling_mode
        if mode == "none":
            self._step_none()
        elif mode == "penalty":
            self._step_penalty()
        elif mode == "moving_boundary":
            self._step_moving_boundary()
        else:
            raise ValueError(f"unsupported coupling_mode: {mode}")
        self.current_lbm_step += 1
        self.total_lbm_substeps += 1

    def _project(self):
        t0 = time.perf_counter()
        self.projector.project(self.solid, self.lbm)
        self._t("projection_time", t0)
        self._apply_wall_velocity_application_if_enabled()

    def _apply_wall_velocity_application_if_enabled(self):
        """fsi_driver.py:458-482: the opt-in solid_vel overwrite after each
        projection (one device kernel; the phase grid is uploaded once)."""
        mode = self.config.wall_velocity_application_mode
        if mode == "disabled":
            return None
        if mode != "solid_vel_experimental":
            raise ValueError(f"unsupported wall_velocity_application_mode: {mode}")
        if self.config.boundary_motion_mode != "prescribed_kinematic":
            raise ValueError("solid_vel_experimental wall velocity application requires prescribed_kinematic "
                             "boundary motion")
        from .wall_velocity import apply_wall_velocity_application_to_lbm

        t0 = time.perf_counter()
        report_path = None
        if self.config.wall_velocity_application_report_enabled:
            report_path = os.path.join(self.out_dir, "wall_velocity_application_report.json")
        report = apply_wall_velocity_application_to_lbm(
            self.lbm, self.config.wall_velocity_application_config_path, self.config.n_grid, self.current_lbm_step,
            report_path=report_path, grid_builder=self.wall_velocity_grid_builder,
            phase_for_step=self.wall_velocity_phase_for_step)
        self.wall_velocity_application_report = report
        self.wall_velocity_application_reports.append(report)
        self._t("wall_velocity_application_time", t0)
        return report

    def _mpm_loop(self, coupler=None, one_phase_reaction=None):
        """The FSI step's MPM substeps, each with the coupler's reaction
        transfer when given (fsi_driver.py's MPM loops)."""
        t0 = time.perf_counter()
        M = self.config.mpm_substeps_per_lbm_step
        if self.mpm_path == "binned":
            self.solid.rebin()
            self.solid.substeps_binned(M, coupler, self.lbm if coupler is not None else None)
            self.total_mpm_substeps += M
        else:
            for _ in range(M):
                self.solid.clear_grid()
                self.solid.p2g()
                if one_phase_reaction is not None:
                    one_phase_reaction()
                self.solid.grid_update()
                self.solid.g2p()
                self.total_mpm_substeps += 1
        self._t("mpm_substep_time", t0)

    def _step_none(self):
        self._project()
        t0 = time.perf_counter()
        self.lbm.step()
        self._t("lbm_step_time", t0)
        self._mpm_loop()

    def _step_penalty(self):
        self._project()
        t0 = time.perf_counter()
        self.penalty_coupler.clear_force_fields(self.lbm)
        self.penalty_coupler.build_penalty_force(self.lbm)
        self._t("coupling_time", t0)
        t0 = time.perf_counter()
        self.lbm.step()
        self._t("lbm_step_time", t0)
        pc = self.penalty_coupler
        self._mpm_loop(pc, lambda: pc.add_lbm_reaction_to_mpm_grid(self.solid, self.lbm))

    def _step_moving_boundary(self):
        self._project()
        t0 = time.perf_counter()
        self.lbm.update_dynamic_solid(self.config.dynamic_solid_threshold)
        self.lbm.reinitialize_new_fluid_cells()
        self._t("coupling_time", t0)
        t0 = time.perf_counter()
        self.lbm.dirstats_enabled = True
        self.lbm.step_moving_bounceback()
        self._t("lbm_step_time", t0)
        self._advance_mpm_with_moving_boundary_reaction()

    def _step_moving_boundary_subcycled(self):
        self._project()
        self.lbm.clear_moving_boundary_force_accumulator()
        S = self.config.lbm_substeps_per_fsi_step
        for s in range(S):
            t0 = time.perf_counter()
            if s == 0:
                self.lbm.update_dynamic_solid(self.config.dynamic_solid_threshold)
            else:
                # phi is unchanged within the FSI step: the reference's repeat call only copies solid -> old_solid
                self.lbm.mark_repeat_mask_update()
            self.lbm.reinitialize_new_fluid_cells()
            self._t("coupling_time", t0)
            t0 = time.perf_counter()
            # the per-direction reductions are read only after the last substep
            self.lbm.dirstats_enabled = s == S - 1
            self.lbm.step_moving_bounceback()
            self._t("lbm_step_time", t0)
            self.lbm.accumulate_moving_boundary_force_sample()
            self.total_lbm_substeps += 1
        self.lbm.finalize_moving_boundary_force_accumulator()
        self._advance_mpm_with_moving_boundary_reaction()

    def _advance_mpm_with_moving_boundary_reaction(self):
        coupler = self.mb_coupler if self.config.reaction_transfer_mode == "engineering" else self.link_area_coupler
        if coupler is None:
            raise ValueError(f"unsupported reaction_transfer_mode: {self.config.reaction_transfer_mode}")

        def react():
            coupler.clear_reaction_diagnostics()
            coupler._react(self.solid, self.lbm)

        self._mpm_loop(coupler, react)

    def run(self):
        total = time.perf_counter()
        if not self.initialized:
            self.initialize()
        self.collect_diagnostics(0)
        for _ in range(self.config.n_lbm_steps):
            self.step_once()
            if self.current_lbm_step % self.config.output_interval == 0 or \
                    self.current_lbm_step == self.config.n_lbm_steps:
                self.collect_diagnostics(self.current_lbm_step)
        self.export_outputs(self.current_lbm_step)
        self.save_timeseries()
        self.timing["total_time"] = time.perf_counter() - total
        return self.diagnostics_rows

    # ------------------------------------------------------- diagnostics
    def _device_row_values(self):
        lbm, solid = self.lbm, self.solid
        n = lbm.ncell
        _, rho, vel = lbm._readout()
        fluid = lbm.fluid_mask()
        v = vel[:, :n].double()
        phi = lbm.t_phi[:n].double()
        zero = torch.zeros((), dtype=torch.float64, device=lbm.device)
        r = rho[:n][fluid].double()
        vf = v[:, fluid]
        fluid_mean = vf.mean(dim=1) if vf.shape[1] else torch.zeros(3, dtype=torch.float64, device=lbm.device)
        act = phi > 1.0e-6
        wsum = phi[act].sum()
        pz = (v[:, act] * phi[act]).sum(dim=1) / wsum if bool(act.any()) else torch.zeros(3, dtype=torch.float64,
                                                                                          device=lbm.device)
        ff = fluid & (phi <= 1.0e-6)
        far = v[:, ff].mean(dim=1) if bool(ff.any()) else torch.zeros(3, dtype=torch.float64, device=lbm.device)
        m = solid.t_mass.double()
        smean = (solid.t_v.double() * m).sum(dim=1) / m.sum()
        cfn = torch.linalg.vector_norm(lbm.t_cf[:, :n].double(), dim=0).max()
        hfn = torch.linalg.vector_norm(lbm._hydro_tensor()[:, :n].double(), dim=0).max()
        vn = torch.linalg.vector_norm(vf, dim=0).max() if vf.shape[1] else zero
        vals = torch.stack([r.min() if r.numel() else zero, r.max() if r.numel() else zero, vn, fluid_mean[0], pz[0],
                            far[0], smean[0], cfn, hfn]).cpu().tolist()
        return vals

    def collect_diagnostics(self, step: int):
        t0 = time.perf_counter()
        cfg = self.config
        vals = self._device_row_values()
        mpm = self.solid.get_stats()
        proj = self.projector.get_stats()
        bb_link, bb_max = 0, 0.0
        if cfg.coupling_mode == "moving_boundary":
            mb = self.lbm.get_moving_boundary_stats()
            bb_link, bb_max = mb["bb_link_count"], mb["bb_max_correction"]
        acc = self.lbm.get_moving_boundary_accumulation_stats()
        mode = "mean_force_accumulator" if (cfg.fsi_exchange_mode == "lbm_subcycled_per_fsi_step" and
                                            acc["mb_subcycle_force_sample_count"] > 0) else "not_active"
        arp, mgr = 0, 0.0
        if cfg.coupling_mode == "moving_boundary":
            c = self.mb_coupler if self.mb_coupler is not None else self.link_area_coupler
            st = c.get_stats()
            arp, mgr = st["active_reaction_particle_count"], st["max_grid_reaction_norm"]
        elif cfg.coupling_mode == "penalty":
            mgr = self.penalty_coupler.get_stats()["max_reaction_grid_force_norm"]
        row = {"step": int(step), "total_mpm_substeps": int(self.total_mpm_substeps), "coupling_mode": cfg.coupling_mode,
               "rho_min": vals[0], "rho_max": vals[1], "lbm_max_v": vals[2], "fluid_mean_ux": vals[3],
               "projection_zone_fluid_mean_ux": vals[4], "far_field_fluid_mean_ux": vals[5],
               "solid_mean_vx_norm": vals[6], "mpm_min_J": mpm["min_J"], "mpm_max_speed": mpm["max_speed"],
               "projected_mass": proj["projected_mass"], "active_cell_count": proj["active_cell_count"],
               "cell_force_max_norm": vals[7], "hydro_force_max_norm": vals[8], "bb_link_count": int(bb_link),
               "bb_max_correction": float(bb_max), "mb_subcycle_force_accumulation_mode": mode,
               "mb_subcycle_force_sample_count": int(acc["mb_subcycle_force_sample_count"]),
               "mb_subcycle_force_accum_norm_max": float(acc["mb_subcycle_force_accum_norm_max"]),
               "mb_subcycle_force_mean_norm_max": float(acc["mb_subcycle_force_mean_norm_max"]),
               "active_reaction_particle_count": int(arp), "max_grid_reaction_norm": float(mgr),
               "elapsed_seconds": 0.0 if self.start_time is None else time.perf_counter() - self.start_time}
        numeric = [v for v in row.values() if isinstance(v, (int, float))]
        if not np.all(np.isfinite(numeric)):
            raise RuntimeError("driver diagnostics contains NaN or Inf")
        self.diagnostics_rows.append(row)
        self.collect_flap_tip_monitor(step)
        self.timing["diagnostics_time"] += time.perf_counter() - t0
        return row

    def flap_tip_displacement(self):
        """Mean displacement of the free-tip particles (normalised units), on the device."""
        if self.initial_particle_positions is None or self.free_tip_proxy_mask is None or \
                not np.any(self.free_tip_proxy_mask):
            return None
        m = torch.as_tensor(self.free_tip_proxy_mask, device=self.device)
        x0 = torch.as_tensor(self.initial_particle_positions, device=self.device).t()
        return (self.solid.t_x[:, m] - x0[:, m]).double().mean(dim=1)

    def collect_flap_tip_monitor(self, step: int):
        d = self.flap_tip_displacement()
        if d is None:
            return None
        d = d.cpu().numpy()
        row = {"step": int(step), "time_s": float(step) * float(self.sim.lbm_dt_phys),
               "flap_tip_total_displacement_m": float(np.linalg.norm(d)), "flap_tip_x_displacement_m": float(d[0]),
               "flap_tip_y_displacement_m": float(d[1])}
        self.flap_tip_monitor_rows.append(row)
        return row

    def export_outputs(self, step: int):
        t0 = time.perf_counter()
        if self.config.write_particles:
            self.solid.export_particles(self.out_dir)
        if self.config.write_vtk:
            self.lbm.export_VTK(step, out_prefix=os.path.join(self.out_dir, "LBMFluid"))
        self.timing["export_time"] += time.perf_counter() - t0

    def save_timeseries(self):
        os.makedirs(self.out_dir, exist_ok=True)
        with open(os.path.join(self.out_dir, "diagnostics_timeseries.csv"), "w", newline="", encoding="utf-8") as f:
            w = csv.DictWriter(f, fieldnames=DIAGNOSTIC_FIELDS)
            w.writeheader()
            for r in self.diagnostics_rows:
                w.writerow({k: r.get(k, "") for k in DIAGNOSTIC_FIELDS})
        payload = {"columns": np.asarray(DIAGNOSTIC_FIELDS),
                   "modes": np.asarray([r["coupling_mode"] for r in self.diagnostics_rows])}
        for k in DIAGNOSTIC_FIELDS:
            if k in DIAGNOSTIC_TEXT_FIELDS:
                payload[k] = np.asarray([r[k] for r in self.diagnostics_rows])
            else:
                payload[k] = np.asarray([r[k] for r in self.diagnostics_rows], dtype=np.float64)
        np.savez(os.path.join(self.out_dir, "diagnostics_timeseries.npz"), **payload)

    def final_diagnostics(self):
        return self.diagnostics_rows[-1] if self.diagnostics_rows else None

    def performance_row(self):
        row = {"mode": self.config.coupling_mode}
        row.update(self.timing)
        return row

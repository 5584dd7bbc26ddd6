"""Generate golden fixtures by running the reference's own kernels.

TEST INFRASTRUCTURE.  Run in a container that holds the reference checkout
(read-only) at REF_ROOT; taichi need not be installed: ``taichi_shim`` stands
in for it (sequential, f32 storage).  Outputs ``tests/golden/*.npz``, which
the CPU tests use to pin the oracle and the GPU tests use to pin the CUDA
path.  Usage::

    python tests/golden/make_fixtures.py --ref PATH [--only NAME]

Each fixture stores its inputs and the reference's outputs in the reference's
own layouts (cell fields (nx, ny, nz[, c]), particle fields (n[, c])).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def install_shim(ref_root):
    sys.path.insert(0, HERE)
    import taichi_shim  # noqa: E402

    sys.modules["taichi"] = taichi_shim
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    return taichi_shim


def rand_state(rng, nx, ny, nz, solid_frac=0.15):
    from src.mpm_lbm.sim.lbm.fluid import LBMFluid3D  # noqa: F401

    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    F = (w[None, None, None, :] * (1.0 + 0.05 * rng.standard_normal((nx, ny, nz, 19)))).astype(np.float32)
    rho = (1.0 + 0.01 * rng.standard_normal((nx, ny, nz))).astype(np.float32)
    v = (0.02 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
    cf = (1e-4 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
    solid = (rng.random((nx, ny, nz)) < solid_frac).astype(np.int8)
    svel = (0.01 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
    return F, rho, v, cf, solid, svel


def make_lbm(cfg_kwargs):
    from src.mpm_lbm.sim.lbm.config import LBMConfig
    from src.mpm_lbm.sim.lbm.fluid import LBMFluid3D

    lbm = LBMFluid3D(LBMConfig(**cfg_kwargs))
    lbm.init_simulation()
    return lbm


def fixture_lbm_kernels(out):
    """collision / streaming / moving bounce-back / macros / mask update / reinit."""
    rng = np.random.default_rng(0)
    nx, ny, nz = 6, 5, 4
    F, rho, v, cf, solid, svel = rand_state(rng, nx, ny, nz)
    force = (1.0e-5, -2.0e-6, 3.0e-6)
    cfg = dict(nx=nx, ny=ny, nz=nz, niu=1.0 / 30.0, relaxation_semantics="standard_lattice_kinematic_viscosity",
               force=force)
    data = dict(F=F, rho=rho, v=v, cell_force=cf, solid=solid, solid_vel=svel, force=np.array(force),
                niu=np.float64(1.0 / 30.0))
    lbm = make_lbm(cfg)
    for name in ("F", "rho", "v", "cell_force", "solid", "solid_vel"):
        getattr(lbm, name).from_numpy(data[name])
    lbm.f.from_numpy(np.zeros_like(F))
    lbm.colission()
    data["collide_f"] = lbm.f.to_numpy()
    # streaming1 from the collided state
    f_post = lbm.f.to_numpy()
    lbm.F.from_numpy(F)
    lbm.streaming1()
    data["stream_static_F"] = lbm.F.to_numpy()
    # moving bounce-back from the same collided state
    lbm.F.from_numpy(F)
    lbm.f.from_numpy(f_post)
    lbm.clear_moving_boundary_diagnostics()
    lbm.streaming_moving_bounceback()
    lbm.finalize_moving_boundary_diagnostics()
    data["stream_moving_F"] = lbm.F.to_numpy()
    data["stream_moving_hydro"] = lbm.hydro_force.to_numpy()
    st = lbm.get_moving_boundary_stats()
    dst = lbm.get_moving_boundary_directional_stats()
    data["bb_link_count"] = np.int64(st["bb_link_count"])
    data["bb_max_correction"] = np.float64(st["bb_max_correction"])
    data["bb_net_solid_force"] = np.array(st["bb_net_solid_force"])
    for k, val in dst.items():
        data["dir_" + k] = np.asarray(val)
    # streaming3 on the moving-bounce-back result
    lbm.streaming3()
    data["macros_f"] = lbm.f.to_numpy()
    data["macros_rho"] = lbm.rho.to_numpy()
    data["macros_v"] = lbm.v.to_numpy()
    # dynamic mask + reinit
    phi = rng.random((nx, ny, nz)).astype(np.float32)
    static = (rng.random((nx, ny, nz)) < 0.1).astype(np.int8)
    lbm.solid.from_numpy(solid)
    lbm.static_solid.from_numpy(static)
    lbm.solid_phi.from_numpy(phi)
    lbm.update_dynamic_solid(0.5)
    data.update(mask_phi=phi, mask_static=static, mask_solid=lbm.solid.to_numpy(), mask_old=lbm.old_solid.to_numpy(),
                mask_reinit=lbm.reinit_flag.to_numpy())
    lbm.reinitialize_new_fluid_cells()
    data.update(reinit_F=lbm.F.to_numpy(), reinit_f=lbm.f.to_numpy(), reinit_rho=lbm.rho.to_numpy(),
                reinit_v=lbm.v.to_numpy())
    np.savez_compressed(out, **data)


BC_CASES = [
    # name, semantics, bc_x_left, bc_x_right, limiter
    ("legacy_vin_pout", "equilibrium_all_population_reset", 2, 1, False),
    ("legacy_pin_vout", "equilibrium_all_population_reset", 1, 2, False),
    ("reg_vin_pout", "regularized_velocity_pressure", 2, 1, False),
    ("reg_pin_vout", "regularized_velocity_pressure", 1, 2, False),
    ("lim_vin_pout", "regularized_velocity_pressure_limited", 2, 1, True),
    ("conv_vin_pout", "convective_pressure_outlet_experimental", 2, 1, False),
]


def fixture_boundaries(out):
    rng = np.random.default_rng(1)
    nx, ny, nz = 7, 5, 4
    F, rho, v, cf, solid, svel = rand_state(rng, nx, ny, nz, solid_frac=0.2)
    rho[3, 2, 1] = 0.0  # exercises the rho <= 1e-6 fallback of the velocity inlet
    rho[nx - 2, 2, 2] = 0.0
    data = dict(F=F, rho=rho, v=v, solid=solid)
    for name, sem, bl, br, lim in BC_CASES:
        cfg = dict(nx=nx, ny=ny, nz=nz, open_boundary_semantics=sem, bc_x_left=bl, bc_x_right=br,
                   vel_bc_x_left=(0.04, 0.003, -0.002), vel_bc_x_right=(0.03, 0.0, 0.001),
                   rho_bc_x_left=1.01, rho_bc_x_right=0.99, open_boundary_limiter_enabled=lim,
                   open_boundary_u_max=0.035, open_boundary_noneq_cap=0.004, open_boundary_rho_min=0.995,
                   open_boundary_rho_max=1.005, open_boundary_population_floor=0.0 if lim else None)
        lbm = make_lbm(cfg)
        for nm in ("F", "rho", "v", "solid"):
            getattr(lbm, nm).from_numpy(data[nm])
        lbm.Boundary_condition()
        data[name + "_F"] = lbm.F.to_numpy()
        if lim:
            s = lbm.get_open_boundary_limiter_stats()
            data[name + "_counts"] = np.array([s["rho_clip_count_step"], s["velocity_clip_count_step"],
                                               s["noneq_clip_count_step"], s["population_floor_count_step"],
                                               s["reconstructed_population_count_step"]], dtype=np.int64)
    data["cases"] = np.array(json.dumps(BC_CASES))
    np.savez_compressed(out, **data)


# outlet repairs and the plane-flux controller (fluid.py:1105-1346, 1495-1792):
# name, semantics, LBMConfig overrides
REPAIR_CASES = [
    ("rmb", "regularized_mass_balanced_pressure_outlet", {}),
    ("cmb_floor", "convective_mass_balanced_pressure_outlet",
     {"open_boundary_limiter_enabled": True, "open_boundary_population_floor": 0.0}),
    ("rfm", "regularized_flux_matched_pressure_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.5, "open_boundary_flux_feedback_gain_rho": 0.3,
      "open_boundary_flux_filter_alpha": 0.2}),
    ("cfm", "convective_flux_matched_damped_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.5, "open_boundary_convective_blend_weight": 0.3}),
    ("rpf_mn", "regularized_plane_flux_controlled_pressure_outlet",
     {"open_boundary_flux_feedback_gain_u": 1.0, "open_boundary_flux_feedback_gain_rho": 0.1,
      "open_boundary_flux_filter_alpha": 0.5, "open_boundary_flux_correction_cap_u": 0.004,
      "open_boundary_flux_feedback_delta_cap_u": 0.001, "open_boundary_flux_feedback_slew_alpha": 0.5,
      "open_boundary_flux_control_measure_plane_offset": 1, "open_boundary_outlet_flux_drop_guard_enabled": True,
      "open_boundary_outlet_flux_drop_guard_min_ratio": 0.9,
      "open_boundary_mass_neutral_flux_control_enabled": True,
      "open_boundary_mass_neutral_flux_control_mode": "global_mass_error_density_offset",
      "open_boundary_mass_neutral_mass_error_gain": 2.0, "open_boundary_mass_neutral_mass_error_cap": 0.001,
      "open_boundary_mass_neutral_correction_blend": 0.5}),
    ("cpf", "convective_plane_flux_controlled_damped_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.05, "open_boundary_flux_control_measure_plane_offset": 2,
      "open_boundary_flux_control_target_scale": 1.1, "open_boundary_convective_blend_weight": 0.25,
      "open_boundary_mass_neutral_flux_control_enabled": True,
      "open_boundary_mass_neutral_flux_control_mode": "global_mass_error_density_offset",
      "open_boundary_mass_neutral_mass_error_gain": 0.5, "open_boundary_mass_neutral_mass_error_cap": 0.01,
      "open_boundary_mass_neutral_correction_blend": 1.0}),
]
# the numeric entries of get_open_boundary_limiter_stats the fixture keeps
REPAIR_STAT_KEYS = [
    "mass_balance_correction_count_step", "mass_balance_correction_count_run",
    "mass_balance_correction_abs_sum_step", "mass_balance_correction_abs_sum_run",
    "unknown_population_delta_abs_sum_step", "unknown_population_delta_abs_sum_run",
    "flow_correction_delta_abs_sum_step", "flow_correction_delta_abs_sum_run",
    "flow_outlet_flux_error_filtered_run", "flow_correction_gain_effective_step",
    "population_floor_count_step", "mass_neutral_mass_current", "mass_neutral_mass_initial_reference",
    "mass_neutral_mass_error", "mass_neutral_rho_feedback", "mass_neutral_feedback_saturation_count_run",
    "mass_neutral_feedback_update_count_run", "near_outlet_flux_xminus1", "near_outlet_flux_xminus2",
    "near_outlet_flux_xminus3", "controller_true_outlet_flux_for_guard", "controller_target_outlet_flux",
    "controller_measured_outlet_flux", "controller_filtered_flux_error", "controller_outlet_fluid_area",
    "controller_u_feedback", "controller_density_feedback", "controller_saturation_count_run",
    "controller_update_count_run", "controller_drop_guard_active_step", "controller_drop_guard_activation_count_run",
    "controller_drop_guard_reference_flux",
]


def fixture_outlet_repair(out):
    """Boundary_condition, streaming3, Boundary_condition for each repair case
    (the second call sees the first's controller and filter state)."""
    rng = np.random.default_rng(2)
    nx, ny, nz = 7, 5, 4
    F, rho, v, cf, solid, svel = rand_state(rng, nx, ny, nz, solid_frac=0.2)
    rho[nx - 2, 2, 2] = 0.0
    data = dict(F=F, rho=rho, v=v, solid=solid)
    for name, sem, over in REPAIR_CASES:
        cfg = dict(nx=nx, ny=ny, nz=nz, open_boundary_semantics=sem, bc_x_left=2, bc_x_right=1,
                   vel_bc_x_left=(0.04, 0.003, -0.002), vel_bc_x_right=(0.03, 0.0, 0.001),
                   rho_bc_x_left=1.01, rho_bc_x_right=0.99)
        cfg.update(over)
        lbm = make_lbm(cfg)
        for nm in ("F", "rho", "v", "solid"):
            getattr(lbm, nm).from_numpy(data[nm])
        for call in (1, 2):
            lbm.Boundary_condition()
            data[f"{name}_F{call}"] = lbm.F.to_numpy()
            st = lbm.get_open_boundary_limiter_stats()
            data[f"{name}_stats{call}"] = np.array([float(st[k]) for k in REPAIR_STAT_KEYS])
            if call == 1:
                lbm.streaming3()
                data[f"{name}_rho1"] = lbm.rho.to_numpy()
                data[f"{name}_v1"] = lbm.v.to_numpy()
    data["cases"] = np.array(json.dumps(REPAIR_CASES))
    data["stat_keys"] = np.array(json.dumps(REPAIR_STAT_KEYS))
    np.savez_compressed(out, **data)


def fixture_mpm(out):
    from src.mpm_lbm.sim.mpm.config import MPMConfig
    from src.mpm_lbm.sim.mpm.solid import MPMSolid3D

    rng = np.random.default_rng(2)
    n = 40
    ng = 8
    cfg = MPMConfig(n_grid=ng, dx=1.0 / ng, dt=4.0e-4, gravity=(0.0, -9.8, 0.5), young_modulus=400.0,
                    poisson_ratio=0.2, p_rho=1.2, box_min=(0.3, 0.3, 0.3), box_max=(0.7, 0.7, 0.7))
    s = MPMSolid3D(cfg, n_particles=n)
    x = rng.uniform(0.2, 0.8, (n, 3)).astype(np.float32)
    x[0] = (0.02, 0.5, 0.99)  # clamp + boundary nodes
    vol0 = np.full(n, (1.0 / ng) ** 3 / 8.0, np.float32)
    mass = (vol0 * 1.2).astype(np.float32)
    fixed = (rng.random(n) < 0.2).astype(np.int8)
    s.init_from_numpy(x, vol0, mass, v_np=rng.normal(0, 0.3, (n, 3)).astype(np.float32), fixed_mask_np=fixed)
    Fdef = (np.eye(3)[None] + 0.05 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    Fdef[1] = np.diag([1.1, -0.9, 1.0]).astype(np.float32)  # inverted element: det < 0
    C = (0.5 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    s.F.from_numpy(Fdef)
    s.C.from_numpy(C)
    data = dict(x=s.x.to_numpy(), v=s.v.to_numpy(), F=Fdef, C=C, vol0=vol0, mass=mass, fixed=fixed,
                fixed_x=s.fixed_x.to_numpy(), n_grid=np.int64(ng), dt=np.float64(4e-4),
                gravity=np.array([0.0, -9.8, 0.5]), E=np.float64(400.0), nu=np.float64(0.2))
    s.clear_grid()
    s.p2g()
    data.update(p2g_grid_v=s.grid_v.to_numpy(), p2g_grid_m=s.grid_m.to_numpy(), p2g_Jp=s.Jp.to_numpy())
    fext = (1e-3 * rng.standard_normal((ng, ng, ng, 3))).astype(np.float32)
    s.grid_f_ext.from_numpy(fext)
    s.grid_update()
    data.update(grid_f_ext=fext, update_grid_v=s.grid_v.to_numpy())
    s.g2p()
    data.update(g2p_x=s.x.to_numpy(), g2p_v=s.v.to_numpy(), g2p_C=s.C.to_numpy(), g2p_F=s.F.to_numpy(),
                g2p_Jp=s.Jp.to_numpy())
    np.savez_compressed(out, **data)


def fixture_coupling(out):
    from src.mpm_lbm.sim.coupling.moving_boundary import MovingBoundaryFSICoupler3D
    from src.mpm_lbm.sim.coupling.penalty import PenaltyFSICoupler3D
    from src.mpm_lbm.sim.coupling.projection import MPMToLBMProjector3D
    from src.mpm_lbm.sim.drivers.sim_config import UnifiedSimConfig
    from src.mpm_lbm.sim.mpm.solid import MPMSolid3D

    rng = np.random.default_rng(3)
    ng = 8
    sim = UnifiedSimConfig(n_grid=ng, mpm_dt=4e-4, mpm_substeps_per_lbm_step=10)
    lbm = make_lbm(dict(nx=ng, ny=ng, nz=ng))
    n = 50
    s = MPMSolid3D(sim.make_mpm_config(), n_particles=n)
    x = rng.uniform(0.15, 0.85, (n, 3)).astype(np.float32)
    vol0 = np.full(n, (1.0 / ng) ** 3 / 8.0, np.float32)
    mass = vol0 * np.float32(1.1)
    s.init_from_numpy(x, vol0, mass, v_np=rng.normal(0, 0.2, (n, 3)).astype(np.float32))
    Jp = rng.uniform(0.9, 1.1, n).astype(np.float32)
    s.Jp.from_numpy(Jp)
    proj = MPMToLBMProjector3D(sim)
    proj.project(s, lbm)
    pst = proj.get_stats()
    data = dict(x=x, v=s.v.to_numpy(), Jp=Jp, vol0=vol0, mass=mass, n_grid=np.int64(ng),
                lbm_dt_phys=np.float64(sim.lbm_dt_phys), dx_norm=np.float64(sim.dx_norm),
                proj_phi=lbm.solid_phi.to_numpy(), proj_mass=lbm.solid_mass.to_numpy(),
                proj_vel=lbm.solid_vel.to_numpy(),
                proj_stats=np.array([pst["projected_mass"], pst["projected_volume_raw"],
                                     pst["projected_volume_clamped"], pst["max_phi_raw"], pst["active_cell_count"]]))
    # penalty force on a random fluid state
    rho = (1.0 + 0.01 * rng.standard_normal((ng, ng, ng))).astype(np.float32)
    vel = (0.01 * rng.standard_normal((ng, ng, ng, 3))).astype(np.float32)
    solid = (rng.random((ng, ng, ng)) < 0.1).astype(np.int8)
    lbm.rho.from_numpy(rho)
    lbm.v.from_numpy(vel)
    lbm.solid.from_numpy(solid)
    pen = PenaltyFSICoupler3D(sim, beta_lbm=0.05, force_cap_lbm=2.0e-4)
    pen.clear_force_fields(lbm)
    pen.build_penalty_force(lbm)
    ps = pen.get_stats()
    data.update(pen_rho=rho, pen_v=vel, pen_solid=solid, pen_cell_force=lbm.cell_force.to_numpy(),
                pen_hydro=lbm.hydro_force.to_numpy(),
                pen_stats=np.array([ps["active_force_cell_count"], ps["max_cell_force_norm"],
                                    *ps["net_cell_force"]]))
    # reaction transfers with a random hydro force field
    hydro = (1e-3 * rng.standard_normal((ng, ng, ng, 3))).astype(np.float32)
    lbm.hydro_force.from_numpy(hydro)
    s.clear_grid()
    pen.add_lbm_reaction_to_mpm_grid(s, lbm)
    data.update(react_hydro=hydro, react_pen_gfe=s.grid_f_ext.to_numpy())
    mb = MovingBoundaryFSICoupler3D(sim, force_cap_norm=2.0e-5)
    s.clear_grid()
    mb.clear_reaction_diagnostics()
    mb.add_moving_boundary_reaction_to_mpm_grid(s, lbm)
    st = mb.get_stats()
    data.update(react_mb_gfe=s.grid_f_ext.to_numpy(),
                react_mb_stats=np.array([st["active_reaction_particle_count"], st["max_particle_reaction_norm"],
                                         st["max_grid_reaction_norm"], *st["net_grid_reaction_force"]]))
    np.savez_compressed(out, **data)


DRIVER_CASES = {
    "drv_mb_eng": dict(coupling_mode="moving_boundary", n_grid=8, n_particles=64, n_lbm_steps=3,
                       mpm_substeps_per_lbm_step=2, box_min=(0.3, 0.3, 0.3), box_max=(0.7, 0.7, 0.7),
                       initial_solid_velocity_norm=(0.5, 0.0, 0.0), gravity=(0.0, -1.0, 0.0), output_interval=1),
    "drv_penalty": dict(coupling_mode="penalty", n_grid=8, n_particles=64, n_lbm_steps=3,
                        mpm_substeps_per_lbm_step=2, box_min=(0.3, 0.3, 0.3), box_max=(0.7, 0.7, 0.7),
                        initial_solid_velocity_norm=(0.5, 0.0, 0.0), beta_lbm=0.05, output_interval=1),
    "drv_none": dict(coupling_mode="none", n_grid=8, n_particles=27, n_lbm_steps=2, mpm_substeps_per_lbm_step=2,
                     box_min=(0.3, 0.3, 0.3), box_max=(0.6, 0.6, 0.6), gravity=(0.0, -9.8, 0.0), output_interval=1),
    "drv_mb_link": dict(coupling_mode="moving_boundary", reaction_transfer_mode="link_area_experimental", n_grid=8,
                        n_particles=64, n_lbm_steps=3, mpm_substeps_per_lbm_step=2, box_min=(0.3, 0.3, 0.3),
                        box_max=(0.7, 0.7, 0.7), initial_solid_velocity_norm=(0.5, 0.0, 0.0),
                        mb_force_cap_norm=1.0e-3, output_interval=1),
    "drv_mb_sub": dict(coupling_mode="moving_boundary", n_grid=8, n_particles=64, n_lbm_steps=2,
                       mpm_substeps_per_lbm_step=1, box_min=(0.3, 0.3, 0.3), box_max=(0.7, 0.7, 0.7),
                       initial_solid_velocity_norm=(0.5, 0.0, 0.0), fsi_exchange_mode="lbm_subcycled_per_fsi_step",
                       lbm_substeps_per_fsi_step=3, lbm_dt_phys_override_s=1.0e-3, official_fsi_dt_s=3.0e-3,
                       target_u_lbm=(0.02, 0.0, 0.0), target_u_lbm_for_dimensional_mapping=0.02,
                       physical_duct_length_m=1.0, target_inlet_velocity_mps=0.02 * (1.0 / 8) / 1.0e-3,
                       output_interval=1),
}


def _duct_geometry_json(path, n_particles):
    geo = {
        "geometry_type": "duct_flap_proxy",
        "n_particles": n_particles,
        "duct": {"x": [0.0, 1.0], "y": [0.2, 0.8], "z": [0.2, 0.8]},
        "flap": {"anchor_x": 0.5, "anchor_y": 0.2, "height_over_duct_height": 0.5, "thickness_over_duct_height": 0.2,
                 "normalized_height": 0.3, "normalized_thickness": 0.12, "z": [0.3, 0.7], "fixed_base": True,
                 "mirrored_pair": False},
        "material_reference": {"density": 1.5, "youngs_modulus": 40.0, "poisson_ratio": 0.3,
                               "used_for_exact_structural_model": False, "used_for_mpm_config": True},
    }
    with open(path, "w", encoding="utf-8") as f:
        json.dump(geo, f)


def fixture_driver(name, out, tmpdir):
    from src.mpm_lbm.sim.drivers.fsi_config import FSIDriverConfig
    from src.mpm_lbm.sim.drivers.fsi_driver import FSIDriver3D

    if name == "drv_duct_lim":
        gpath = os.path.join(tmpdir, "duct_geo.json")
        _duct_geometry_json(gpath, 96)
        kwargs = dict(coupling_mode="moving_boundary", geometry_type="duct_flap_proxy", geometry_config_path=gpath,
                      n_grid=10, n_particles=96, n_lbm_steps=2, mpm_substeps_per_lbm_step=1,
                      lbm_boundary_condition_mode="duct_velocity_inlet_pressure_outlet",
                      lbm_open_boundary_semantics="regularized_velocity_pressure_limited",
                      open_boundary_limiter_enabled=True, target_u_lbm=(0.03, 0.0, 0.0),
                      fsi_exchange_mode="lbm_subcycled_per_fsi_step", lbm_substeps_per_fsi_step=3,
                      lbm_dt_phys_override_s=1.0e-3, official_fsi_dt_s=3.0e-3,
                      target_u_lbm_for_dimensional_mapping=0.03, physical_duct_length_m=1.0,
                      target_inlet_velocity_mps=0.03 * 0.1 / 1.0e-3, output_interval=1)
    else:
        kwargs = dict(DRIVER_CASES[name])
    cfg = FSIDriverConfig(**kwargs)
    drv = FSIDriver3D(cfg, os.path.join(tmpdir, name))
    drv.initialize()
    init = dict(init_x=drv.solid.x.to_numpy(), init_v=drv.solid.v.to_numpy(), init_vol0=drv.solid.vol0.to_numpy(),
                init_mass=drv.solid.mass.to_numpy(), init_fixed=drv.solid.fixed_mask.to_numpy(),
                init_solid=drv.lbm.solid.to_numpy(), mpm_mu=np.float64(drv.solid.mu), mpm_la=np.float64(drv.solid.la))
    rows = drv.run()
    data = dict(init)
    data["config"] = np.array(json.dumps(cfg.to_dict()))
    data["rows"] = np.array(json.dumps(rows))
    lbm, solid = drv.lbm, drv.solid
    for nm in ("F", "rho", "v", "solid", "solid_phi", "solid_vel", "hydro_force", "cell_force"):
        data["lbm_" + nm] = getattr(lbm, nm).to_numpy()
    for nm in ("x", "v", "C", "F", "Jp"):
        data["mpm_" + nm] = getattr(solid, nm).to_numpy()
    if drv.link_area_coupler is not None:
        data["area_scale"] = np.float64(drv.link_area_coupler.area_scale[None])
    if drv.free_tip_proxy_mask is not None:
        data["free_tip_mask"] = drv.free_tip_proxy_mask.astype(np.int8)
    np.savez_compressed(out, **data)


UNIT = {
    "lbm_kernels": fixture_lbm_kernels,
    "lbm_boundaries": fixture_boundaries,
    "lbm_outlet_repair": fixture_outlet_repair,
    "mpm_kernels": fixture_mpm,
    "coupling_kernels": fixture_coupling,
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF_ROOT"), help="reference checkout (or set REF_ROOT)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or REF_ROOT")
    install_shim(args.ref)
    names = list(UNIT) + list(DRIVER_CASES) + ["drv_duct_lim"]
    if args.only:
        names = [n for n in names if n == args.only]
    with tempfile.TemporaryDirectory() as tmp:
        for name in names:
            t0 = time.time()
            out = os.path.join(HERE, name + ".npz")
            if name in UNIT:
                UNIT[name](out)
            else:
                fixture_driver(name, out, tmp)
            print(f"{name}: {time.time() - t0:.1f}s -> {os.path.getsize(out)} bytes", flush=True)


if __name__ == "__main__":
    main()

"""GPU parity of the outlet repairs and the plane-flux controller
(open-boundary semantics 4-9, fluid.py:1105-1346, 1495-1792) against the CPU
oracle, which tests/test_oracle_golden.py pins to the reference's kernels.

Tolerances (FP32): populations as the other LBM parity tests (rtol 2e-5 /
atol 1e-7); plane and repair sums rtol 1e-4 / atol 1e-6 (device atomics sum
in another order than the reference's sequential loop); counters exact.  The
flow filter of semantics 6 and 7 (one record per repaired population) is
folded in the reference's sequential order from per-row composites, so it
agrees with the oracle to the same tolerance and lies in the hull of the
recorded errors."""

import numpy as np
import pytest

from oracle import oracle as orc

from tests.test_gpu_lbm import POP_TOL, VEL_TOL, channel_with_obstacle, use_tune

pytestmark = pytest.mark.gpu

VEL = ((0.04, 0.002, 0.0), (0.03, 0.0, 0.001), (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0))
MASS_NEUTRAL = {"open_boundary_mass_neutral_flux_control_enabled": True,
                "open_boundary_mass_neutral_flux_control_mode": "global_mass_error_density_offset",
                "open_boundary_mass_neutral_mass_error_gain": 2.0, "open_boundary_mass_neutral_mass_error_cap": 0.001,
                "open_boundary_mass_neutral_correction_blend": 0.5}
CASES = [
    ("regularized_mass_balanced_pressure_outlet", {}),
    ("convective_mass_balanced_pressure_outlet", {}),
    ("regularized_flux_matched_pressure_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.5, "open_boundary_flux_feedback_gain_rho": 0.3,
      "open_boundary_flux_filter_alpha": 0.2}),
    ("convective_flux_matched_damped_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.5, "open_boundary_convective_blend_weight": 0.3}),
    ("regularized_plane_flux_controlled_pressure_outlet",
     {"open_boundary_flux_feedback_gain_u": 1.0, "open_boundary_flux_feedback_gain_rho": 0.1,
      "open_boundary_flux_filter_alpha": 0.5, "open_boundary_flux_correction_cap_u": 0.004,
      "open_boundary_flux_feedback_delta_cap_u": 0.001, "open_boundary_flux_feedback_slew_alpha": 0.5,
      "open_boundary_flux_control_measure_plane_offset": 1, "open_boundary_outlet_flux_drop_guard_enabled": True,
      "open_boundary_outlet_flux_drop_guard_min_ratio": 0.9, **MASS_NEUTRAL}),
    ("convective_plane_flux_controlled_damped_outlet",
     {"open_boundary_flux_feedback_gain_u": 0.05, "open_boundary_flux_control_measure_plane_offset": 2,
      "open_boundary_flux_control_target_scale": 1.1, "open_boundary_convective_blend_weight": 0.25,
      **MASS_NEUTRAL}),
]
COUNT_KEYS = ["mass_balance_correction_count_step", "mass_balance_correction_count_run",
              "controller_update_count_step", "controller_update_count_run", "controller_saturation_count_run",
              "controller_drop_guard_activation_count_run", "controller_drop_guard_active_step",
              "mass_neutral_feedback_update_count_run", "mass_neutral_feedback_saturation_count_run"]
SUM_KEYS = ["mass_balance_correction_abs_sum_step", "mass_balance_correction_abs_sum_run",
            "unknown_population_delta_abs_sum_step", "unknown_population_delta_abs_sum_run",
            "flow_correction_delta_abs_sum_step", "flow_correction_delta_abs_sum_run",
            "flow_correction_gain_effective_step", "near_outlet_flux_xminus1", "near_outlet_flux_xminus2",
            "near_outlet_flux_xminus3", "controller_true_outlet_flux_for_guard", "controller_target_outlet_flux",
            "controller_measured_outlet_flux", "controller_filtered_flux_error", "controller_outlet_fluid_area",
            "controller_u_feedback", "controller_density_feedback", "controller_drop_guard_reference_flux",
            "mass_neutral_mass_current", "mass_neutral_mass_initial_reference", "mass_neutral_mass_error",
            "mass_neutral_rho_feedback"]


def make_repair_pair(nx, ny, nz, solid, sem, over, seed=3):
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    gpu = LBMFluid3D(LBMConfig(nx=nx, ny=ny, nz=nz, open_boundary_semantics=sem, bc_x_left=2, bc_x_right=1,
                               rho_bc_x_left=1.01, rho_bc_x_right=0.99, vel_bc_x_left=VEL[0],
                               vel_bc_x_right=VEL[1], **over))
    ora = orc.OracleLBM(nx, ny, nz, open_boundary_semantics=sem, bc=(2, 1, 0, 0, 0, 0),
                        rho_bc=(1.01, 0.99, 1, 1, 1, 1), vel_bc=VEL, flux_control=over)
    ora.init_geo_array(solid)
    gpu.init_geo_array(solid)
    ora.init_simulation()
    gpu.init_simulation()
    rng = np.random.default_rng(seed)
    F = ora.F * (1.0 + 0.02 * rng.standard_normal(ora.F.shape)).astype(np.float32)
    rho = F.sum(axis=-1).astype(np.float32)
    v = ((F @ orc.E.astype(np.float32)) / rho[..., None]).astype(np.float32)
    v[..., 0] += np.float32(0.02)  # a mean flow toward the outlet
    ora.F[...] = F
    ora.f[...] = F
    ora.rho[...] = rho
    ora.v[...] = v
    gpu.F.from_numpy(F)
    gpu.rho.from_numpy(rho)
    gpu.v.from_numpy(v)
    return ora, gpu


def outlet_errors(ora, vx_in):
    """vx_bcxl - v[ni, j, k][0] over the fluid outlet cells, from the state the
    next Boundary_condition reads."""
    nx = ora.nx
    face = ora.solid[nx - 1] == 0
    ni_solid = ora.solid[nx - 2] > 0
    u = np.where(ni_solid, ora.v[nx - 1, :, :, 0], ora.v[nx - 2, :, :, 0])
    return (np.float32(vx_in) - u)[face]


@pytest.mark.parametrize("tune", [0, 2, 4])
@pytest.mark.parametrize("nx", [20, 64])
@pytest.mark.parametrize("sem,over", CASES, ids=[c[0] for c in CASES])
def test_outlet_repair_matches_oracle(sem, over, nx, tune):
    ny, nz = 9, 8
    solid = channel_with_obstacle(nx, ny, nz)
    solid[nx - 2, 4, 4] = 1  # an outlet cell whose neighbour is solid -> ni = face
    ora, gpu = make_repair_pair(nx, ny, nz, solid, sem, over)
    use_tune(gpu, tune)
    lo, hi = 0.0, 0.0
    for _ in range(6):
        e = outlet_errors(ora, VEL[0][0])
        lo, hi = min(lo, float(e.min())), max(hi, float(e.max()))
        ora.step_moving_bounceback()
        gpu.step_moving_bounceback()
        np.testing.assert_allclose(gpu.F.to_numpy(), ora.F, **POP_TOL)
        np.testing.assert_allclose(gpu.rho.to_numpy(), ora.rho, **POP_TOL)
        np.testing.assert_allclose(gpu.v.to_numpy(), ora.v, **VEL_TOL)
    go, oo = gpu.get_open_boundary_limiter_stats(), ora.get_open_boundary_limiter_stats()
    for k in COUNT_KEYS:
        assert go[k] == oo[k], (k, go[k], oo[k])
    for k in SUM_KEYS:
        assert abs(go[k] - oo[k]) <= 1e-6 + 1e-4 * abs(oo[k]), (k, go[k], oo[k])
    filt = go["flow_outlet_flux_error_filtered_run"]
    if "flux_matched" in sem:
        assert lo - 1e-6 <= filt <= hi + 1e-6, (filt, lo, hi)
        assert filt != 0.0
    assert abs(filt - oo["flow_outlet_flux_error_filtered_run"]) <= 1e-6 + 1e-4 * abs(filt)


def test_plane_flux_controller_contract_gpu():
    """tests/test_step131_plane_flux_controller_contract.py:205-235 on the
    product: a cleared run starts from zero, and with the inlet plane's flux
    above the outlet's the feedback saturates at +cap (-cap the other way)."""
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    cfg = LBMConfig(nx=8, ny=6, nz=6, open_boundary_semantics="regularized_plane_flux_controlled_pressure_outlet",
                    bc_x_left=2, bc_x_right=1, open_boundary_flux_feedback_gain_u=1.0,
                    open_boundary_flux_feedback_gain_rho=0.0, open_boundary_flux_filter_alpha=1.0,
                    open_boundary_flux_correction_cap_u=0.002, open_boundary_convective_blend_weight=0.02)
    lbm = LBMFluid3D(cfg)
    lbm.init_simulation()
    lbm.clear_open_boundary_limiter_run_counters()
    st = lbm.get_open_boundary_limiter_stats()
    assert st["controller_target_outlet_flux"] == 0.0
    assert st["controller_measured_outlet_flux"] == 0.0
    assert st["controller_u_feedback"] == 0.0
    assert st["controller_saturation_count_run"] == 0
    for inlet, outlet, sign in ((1.0, 0.0, 1.0), (0.0, 1.0, -1.0)):
        lbm.clear_open_boundary_limiter_run_counters()
        rho = np.ones((8, 6, 6), np.float32)
        vel = np.zeros((8, 6, 6, 3), np.float32)
        vel[0, :, :, 0] = inlet
        vel[-1, :, :, 0] = outlet
        lbm.solid.from_numpy(np.zeros((8, 6, 6), np.int8))
        lbm.rho.from_numpy(rho)
        lbm.v.from_numpy(vel)
        lbm.update_open_boundary_plane_flux_controller()
        st = lbm.get_open_boundary_limiter_stats()
        assert sign * (st["controller_target_outlet_flux"] - st["controller_measured_outlet_flux"]) > 0.0
        assert sign * st["controller_raw_flux_error"] > 0.0
        assert st["controller_u_feedback"] == pytest.approx(sign * 0.002)
        assert st["controller_saturation_count_run"] == 1
        assert st["controller_outlet_fluid_area"] == 36.0


def test_periodic_plane_flux_controller_runs_without_open_faces():
    """Semantics 8 with periodic x faces: the reference still runs the
    controller each step (fluid.py:561-564) and applies no outlet."""
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    over = {"open_boundary_flux_feedback_gain_u": 1.0, "open_boundary_flux_filter_alpha": 0.5}
    nx, ny, nz = 20, 9, 8
    solid = channel_with_obstacle(nx, ny, nz)
    sem = "regularized_plane_flux_controlled_pressure_outlet"
    gpu = LBMFluid3D(LBMConfig(nx=nx, ny=ny, nz=nz, open_boundary_semantics=sem, **over))
    ora = orc.OracleLBM(nx, ny, nz, open_boundary_semantics=sem, flux_control=over)
    for m in (ora, gpu):
        m.init_geo_array(solid)
        m.init_simulation()
    F = ora.F * (1.0 + 0.02 * np.random.default_rng(5).standard_normal(ora.F.shape)).astype(np.float32)
    ora.F[...] = F
    gpu.F.from_numpy(F)
    rho = F.sum(axis=-1).astype(np.float32)
    v = ((F @ orc.E.astype(np.float32)) / rho[..., None]).astype(np.float32)
    ora.rho[...] = rho
    ora.v[...] = v
    gpu.rho.from_numpy(rho)
    gpu.v.from_numpy(v)
    for _ in range(3):
        ora.step()
        gpu.step()
    np.testing.assert_allclose(gpu.F.to_numpy(), ora.F, **POP_TOL)
    go, oo = gpu.get_open_boundary_limiter_stats(), ora.get_open_boundary_limiter_stats()
    assert go["controller_update_count_run"] == oo["controller_update_count_run"] == 3
    for k in ("controller_target_outlet_flux", "controller_measured_outlet_flux", "controller_u_feedback"):
        assert abs(go[k] - oo[k]) <= 1e-6 + 1e-4 * abs(oo[k]), (k, go[k], oo[k])

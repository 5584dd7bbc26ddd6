"""GPU parity of the LBM step (CUDA path through the C ABI) against the CPU
oracle on seeded inputs.  Tolerances (FP32): populations rtol 2e-5 /
atol 1e-7 after N steps; link forces rtol 1e-4 / atol 1e-7 (a solid cell sums
up to 18 partly cancelling link terms whose order differs between the
oracle's sequential loop and device atomics); masks and link counts
bit-exact."""

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

POP_TOL = dict(rtol=2e-5, atol=1e-7)
VEL_TOL = dict(rtol=1e-4, atol=2e-7)


def make_pair(nx, ny, nz, solid, seed=0, perturb=True, **kw):
    import torch  # noqa: F401

    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    okw = dict(kw)
    gcfg = dict(nx=nx, ny=ny, nz=nz)
    mapping = dict(niu="niu", relaxation_semantics="relaxation_semantics",
                   open_boundary_semantics="open_boundary_semantics")
    for k in mapping:
        if k in okw:
            gcfg[k] = okw[k]
    bc = okw.get("bc", (0, 0, 0, 0, 0, 0))
    rho_bc = okw.get("rho_bc", (1.0,) * 6)
    vel_bc = okw.get("vel_bc", ((0.0, 0.0, 0.0),) * 6)
    gcfg.update(bc_x_left=bc[0], bc_x_right=bc[1], rho_bc_x_left=rho_bc[0], rho_bc_x_right=rho_bc[1],
                vel_bc_x_left=tuple(vel_bc[0]), vel_bc_x_right=tuple(vel_bc[1]),
                force=tuple(okw.get("force", (0.0, 0.0, 0.0))),
                open_boundary_limiter_enabled=okw.get("limiter_enabled", False),
                open_boundary_u_max=okw.get("ob_u_max", 0.1), open_boundary_noneq_cap=okw.get("ob_noneq_cap", 0.05),
                open_boundary_rho_min=okw.get("ob_rho_min", 0.8), open_boundary_rho_max=okw.get("ob_rho_max", 1.2),
                open_boundary_population_floor=okw.get("ob_floor", None))
    if "collision" in okw:
        gcfg["collision"] = okw["collision"]
    gpu = LBMFluid3D(LBMConfig(**gcfg))
    ora = orc.OracleLBM(nx, ny, nz, **kw)
    ora.init_geo_array(solid)
    gpu.init_geo_array(solid)
    ora.init_simulation()
    gpu.init_simulation()
    if perturb:
        rng = np.random.default_rng(seed)
        F = ora.F * (1.0 + 0.02 * rng.standard_normal(ora.F.shape)).astype(np.float32)
        rho = F.sum(axis=-1).astype(np.float32)
        e = orc.E.astype(np.float32)
        v = (F @ e) / rho[..., None]
        ora.F[...] = F
        ora.f[...] = F
        ora.rho[...] = rho
        ora.v[...] = v.astype(np.float32)
        gpu.F.from_numpy(F)
        gpu.rho.from_numpy(rho)
        gpu.v.from_numpy(ora.v)
    return ora, gpu


def compare(ora, gpu, what=("F", "rho", "v")):
    if "F" in what:
        np.testing.assert_allclose(gpu.F.to_numpy(), ora.F, **POP_TOL)
    if "rho" in what:
        np.testing.assert_allclose(gpu.rho.to_numpy(), ora.rho, **POP_TOL)
    if "v" in what:
        np.testing.assert_allclose(gpu.v.to_numpy(), ora.v, **VEL_TOL)


# FsiLbmParams.tune: 0 one cell per thread (3 CTAs/SM), 2 two x-adjacent cells
# per thread on the paired FP32 pipe (nx even)
TUNES = [0, 2]


def use_tune(gpu, tune):
    gpu.tune = tune
    gpu._sync_params()


def channel_with_obstacle(nx, ny, nz):
    s = np.zeros((nx, ny, nz), np.int8)
    s[:, 0, :] = s[:, -1, :] = 1
    s[:, :, 0] = s[:, :, -1] = 1
    s[nx // 2 - 1: nx // 2 + 1, ny // 2 - 1: ny // 2 + 2, nz // 2 - 1: nz // 2 + 1] = 1
    return s


@pytest.mark.parametrize("tune", TUNES)
@pytest.mark.parametrize("collision", ["mrt", "bgk"])
def test_static_bounceback_steps_match_oracle(collision, tune):
    nx, ny, nz = 70, 10, 9  # nx > 64: two warps per row in both layouts
    solid = channel_with_obstacle(nx, ny, nz)
    ora, gpu = make_pair(nx, ny, nz, solid, niu=1.0 / 30.0, relaxation_semantics="standard_lattice_kinematic_viscosity",
                         force=(1e-5, 2e-6, -1e-6), collision=collision)
    use_tune(gpu, tune)
    for step in range(7):  # odd count: ends on the swapped AA layout
        ora.step()
        gpu.step()
        if step in (0, 1, 6):
            compare(ora, gpu)


@pytest.mark.parametrize("nx,tune", [(33, 0), (34, 2), (66, 2)])
def test_moving_bounceback_matches_oracle(nx, tune):
    ny, nz = 8, 7  # nx % 32 == 1 without open boundaries is allowed
    solid = channel_with_obstacle(nx, ny, nz)
    ora, gpu = make_pair(nx, ny, nz, solid, force=(2e-5, 0.0, 0.0))
    use_tune(gpu, tune)
    rng = np.random.default_rng(5)
    sv = (0.01 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32) * solid[..., None]
    ora.solid_vel[...] = sv
    gpu.solid_vel.from_numpy(sv)
    for step in range(5):
        ora.step_moving_bounceback()
        gpu.step_moving_bounceback()
        compare(ora, gpu)
        np.testing.assert_allclose(gpu.hydro_force.to_numpy(), ora.hydro_force, rtol=1e-4, atol=1e-7)
        go, oo = gpu.get_moving_boundary_directional_stats(), ora.get_moving_boundary_directional_stats()
        np.testing.assert_array_equal(go["link_count_by_dir"], oo["link_count_by_dir"])
        np.testing.assert_allclose(go["solid_force_by_dir"], oo["solid_force_by_dir"], rtol=1e-4, atol=1e-7)
        np.testing.assert_allclose(go["correction_abs_max_by_dir"], oo["correction_abs_max_by_dir"], rtol=1e-5,
                                   atol=1e-10)
        assert gpu.get_moving_boundary_stats()["bb_link_count"] == ora.get_moving_boundary_stats()["bb_link_count"]


BC_CASES = [
    ("equilibrium_all_population_reset", 2, 1, False),
    ("equilibrium_all_population_reset", 1, 2, False),
    ("regularized_velocity_pressure", 2, 1, False),
    ("regularized_velocity_pressure", 1, 2, False),
    ("regularized_velocity_pressure_limited", 2, 1, True),
    ("convective_pressure_outlet_experimental", 2, 1, False),
]


@pytest.mark.parametrize("tune", TUNES)
@pytest.mark.parametrize("sem,bl,br,lim", BC_CASES)
@pytest.mark.parametrize("nx", [20, 48, 64])
def test_open_boundaries_match_oracle(sem, bl, br, lim, nx, tune):
    ny, nz = 9, 8
    solid = channel_with_obstacle(nx, ny, nz)
    solid[1, 3, 3] = 1  # neighbour of the inlet face is solid -> ni = face
    solid[nx - 2, 4, 4] = 1
    vel = ((0.04, 0.002, 0.0), (0.03, 0.0, 0.001), (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0))
    ora, gpu = make_pair(nx, ny, nz, solid, open_boundary_semantics=sem, bc=(bl, br, 0, 0, 0, 0),
                         rho_bc=(1.01, 0.99, 1, 1, 1, 1), vel_bc=vel, limiter_enabled=lim, ob_u_max=0.035,
                         ob_noneq_cap=0.004, ob_rho_min=0.995, ob_rho_max=1.005, ob_floor=0.0 if lim else None)
    use_tune(gpu, tune)
    for step in range(6):
        ora.step_moving_bounceback()
        gpu.step_moving_bounceback()
        compare(ora, gpu)
    if lim:
        go, oo = gpu.get_open_boundary_limiter_stats(), ora.get_open_boundary_limiter_stats()
        for k in ("rho_clip_count_run", "velocity_clip_count_run", "noneq_clip_count_run",
                  "population_floor_count_run", "reconstructed_population_count_run",
                  "reconstructed_population_count_step"):
            assert go[k] == oo[k], k


@pytest.mark.parametrize("tune", TUNES)
@pytest.mark.parametrize("steps_before", [1, 2])
def test_dynamic_mask_reinit_matches_oracle(steps_before, tune):
    nx, ny, nz = 24, 10, 10
    solid = channel_with_obstacle(nx, ny, nz)
    solid[nx // 2 - 1: nx // 2 + 1, ny // 2 - 1: ny // 2 + 2, nz // 2 - 1: nz // 2 + 1] = 0
    ora, gpu = make_pair(nx, ny, nz, solid, force=(1e-5, 0, 0))
    use_tune(gpu, tune)
    rng = np.random.default_rng(11)
    sv = (0.01 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
    for phase in range(4):
        phi = np.zeros((nx, ny, nz), np.float32)
        c = 6 + 3 * phase
        phi[c: c + 4, 3:7, 3:7] = 0.9
        phi[c, 3, 3] = 0.49
        for o in (ora, gpu):
            if o is ora:
                o.solid_phi[...] = phi
                o.solid_vel[...] = sv
            else:
                o.solid_phi.from_numpy(phi)
                o.solid_vel.from_numpy(sv)
        ora.update_dynamic_solid(0.5)
        ora.reinitialize_new_fluid_cells()
        gpu.update_dynamic_solid(0.5)
        np.testing.assert_array_equal(gpu.solid.to_numpy(), ora.solid)
        for _ in range(steps_before):
            ora.step_moving_bounceback()
            gpu.step_moving_bounceback()
        compare(ora, gpu)
        np.testing.assert_allclose(gpu.hydro_force.to_numpy(), ora.hydro_force, rtol=1e-4, atol=1e-7)


@pytest.mark.parametrize("tune", TUNES)
def test_subcycled_accumulator_matches_oracle(tune):
    nx, ny, nz = 16, 8, 8
    solid = channel_with_obstacle(nx, ny, nz)
    ora, gpu = make_pair(nx, ny, nz, solid, force=(3e-5, 0, 0))
    use_tune(gpu, tune)
    for o in (ora, gpu):
        o.clear_moving_boundary_force_accumulator()
    for _ in range(3):
        for o in (ora, gpu):
            o.step_moving_bounceback()
            o.accumulate_moving_boundary_force_sample()
    for o in (ora, gpu):
        o.finalize_moving_boundary_force_accumulator()
    np.testing.assert_allclose(gpu.hydro_force.to_numpy(), ora.hydro_force, rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(gpu.hydro_force_accum.to_numpy(), ora.hydro_force_accum, rtol=1e-4, atol=1e-7)
    a, b = gpu.get_moving_boundary_accumulation_stats(), ora.get_moving_boundary_accumulation_stats()
    assert a["mb_subcycle_force_sample_count"] == b["mb_subcycle_force_sample_count"] == 3
    np.testing.assert_allclose(a["mb_subcycle_force_accum_norm_max"], b["mb_subcycle_force_accum_norm_max"], rtol=1e-4)
    np.testing.assert_allclose(a["mb_subcycle_force_mean_norm_max"], b["mb_subcycle_force_mean_norm_max"], rtol=1e-4)


def test_step115_accumulator_known_answer_gpu():
    # tests/test_step115_lbm_open_boundary_and_force_accumulation_contract.py:25-45 of the reference
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    lbm = LBMFluid3D(LBMConfig(nx=4, ny=4, nz=4))
    lbm.clear_moving_boundary_force_accumulator()
    lbm.hydro_force[1, 1, 1] = (1.0, 0.0, 0.0)
    lbm.accumulate_moving_boundary_force_sample()
    lbm.hydro_force[1, 1, 1] = (3.0, 0.0, 0.0)
    lbm.accumulate_moving_boundary_force_sample()
    lbm.finalize_moving_boundary_force_accumulator()
    st = lbm.get_moving_boundary_accumulation_stats()
    np.testing.assert_allclose(lbm.hydro_force.to_numpy()[1, 1, 1], [2.0, 0.0, 0.0], rtol=0, atol=1e-6)
    assert st["mb_subcycle_force_sample_count"] == 2
    assert abs(st["mb_subcycle_force_accum_norm_max"] - 4.0) <= 1e-6
    assert abs(st["mb_subcycle_force_mean_norm_max"] - 2.0) <= 1e-6


@pytest.mark.parametrize("tune", TUNES)
def test_penalty_step_matches_oracle(tune):
    nx, ny, nz = 16, 10, 9
    solid = channel_with_obstacle(nx, ny, nz)
    ora, gpu = make_pair(nx, ny, nz, solid, force=(1e-5, 0, 0))
    use_tune(gpu, tune)
    rng = np.random.default_rng(3)
    cpl = orc.OracleCoupling(nx, 1.0 / nx, 4e-3, beta_lbm=0.05, penalty_force_cap=2e-4)
    for step in range(4):
        phi = np.clip(rng.random((nx, ny, nz)) * 1.4 - 0.6, 0, 1).astype(np.float32)
        sv = (0.02 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
        ora.solid_phi[...] = phi
        ora.solid_vel[...] = sv
        gpu.solid_phi.from_numpy(phi)
        gpu.solid_vel.from_numpy(sv)
        cpl.build_penalty_force(ora)
        gpu._penalty = (0.05, 1e-6, 2e-4)
        ora.step()
        gpu.step()
        compare(ora, gpu)
        np.testing.assert_allclose(gpu.cell_force.to_numpy(), ora.cell_force, rtol=1e-4, atol=2e-9)
        np.testing.assert_allclose(gpu.hydro_force.to_numpy(), ora.hydro_force, rtol=1e-4, atol=2e-9)


@pytest.mark.parametrize("moving", [False, True])
def test_launch_variants_are_bit_identical(moving):
    """FsiLbmParams.tune 0, 1, 3, 4 only change the register budget of the step
    kernel and whether it prefetches the next wave's tiles into L2: populations
    and macroscopic fields agree bit for bit; the link forces are float atomic
    sums whose order (and last-bit rounding) varies between any two launches."""
    nx, ny, nz = 40, 12, 10
    solid = channel_with_obstacle(nx, ny, nz)
    outs = []
    for tune in (0, 1, 3, 4):
        _, gpu = make_pair(nx, ny, nz, solid, force=(2e-5, 0.0, 0.0), seed=7)
        gpu.tune = tune
        rng = np.random.default_rng(9)
        sv = (0.01 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32) * solid[..., None]
        gpu.solid_vel.from_numpy(sv)
        for _ in range(5):
            gpu.step_moving_bounceback() if moving else gpu.step()
        outs.append((gpu.F.to_numpy(), gpu.rho.to_numpy(), gpu.v.to_numpy(), gpu.hydro_force.to_numpy()))
    for other in outs[1:]:
        for a, b in zip(outs[0][:3], other[:3]):
            np.testing.assert_array_equal(a, b)
        # link forces: float atomic sums of terms up to ~0.3 that cancel to ~1e-4;
        # their order varies, so compare within one ulp of the largest term
        np.testing.assert_allclose(outs[0][3], other[3], rtol=1e-5, atol=2e-8)

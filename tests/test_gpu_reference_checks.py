"""The reference's own regression checks on this path, run on the drop-in.

- Zero-velocity moving bounce-back equals static bounce-back
  (baseline_tests/run_step8_static_bounceback_regression.py:90-118): a 32^3
  lattice with solid walls at y = 0 and y = 31, 100 steps with `step()` and
  100 with `step_moving_bounceback()` at zero wall velocity; the moving run
  finds solid links, its largest correction is at most 1e-12, velocity and
  density agree within 1e-6, the static run leaves cell_force at zero, and
  both stay in the accepted density and speed ranges.
- Projection of a static and of a moving block
  (baseline_tests/run_step5_projection_static_block.py:48-105,
  run_step5_projection_moving_block.py:42-108): 4,096 particles of the
  default box on an all-fluid 32^3 lattice; the projected mass within 1e-5
  of the particle mass, solid_phi in [0, 1], the mass-weighted mean solid
  velocity equal to the block's (x within 1e-6, y and z within 1e-8; zero for
  the static block within 1e-8), and cell_force / hydro_force untouched.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lbm(sim, solid):
    from mpm_lbm_b200.lbm import LBMFluid3D

    lbm = LBMFluid3D(sim.make_lbm_config())
    lbm.init_geo_array(solid)
    lbm.init_simulation()
    return lbm


def _stats_ok(stats):
    vals = [stats["max_v"], stats["rho_min"], stats["rho_max"], stats["mass_total"]]
    assert np.all(np.isfinite(vals))
    assert 0.95 < stats["rho_min"] and stats["rho_max"] < 1.05, stats
    assert stats["max_v"] < 0.1, stats


def test_zero_velocity_moving_bounceback_equals_static():
    import torch

    from mpm_lbm_b200.config import UnifiedSimConfig

    sim = UnifiedSimConfig(n_grid=32, mpm_dt=4.0e-4, mpm_substeps_per_lbm_step=10)
    n = sim.n_grid
    geo = np.zeros((n, n, n), np.int8)
    geo[:, 0, :] = 1
    geo[:, n - 1, :] = 1
    static, moving = _lbm(sim, geo), _lbm(sim, geo)
    for step in range(1, 101):
        static.step()
        moving.step_moving_bounceback()
        if step % 25 == 0:
            _stats_ok(static.get_stats())
            _stats_ok(moving.get_stats())
    torch.cuda.synchronize()
    bb = moving.get_moving_boundary_stats()
    assert bb["bb_link_count"] > 0
    assert abs(bb["bb_max_correction"]) <= 1.0e-12
    dv = np.abs(moving.v.to_numpy() - static.v.to_numpy()).max()
    drho = np.abs(moving.rho.to_numpy() - static.rho.to_numpy()).max()
    assert np.isfinite(dv) and np.isfinite(drho)
    assert dv < 1.0e-6 and drho < 1.0e-6
    assert float(np.max(np.linalg.norm(static.cell_force.to_numpy(), axis=3))) == 0.0


@pytest.mark.parametrize("moving", [False, True])
def test_block_projection_mass_and_velocity(moving):
    import torch

    from mpm_lbm_b200.config import GridUnitMapper, UnifiedSimConfig
    from mpm_lbm_b200.coupling import MPMToLBMProjector3D
    from mpm_lbm_b200.mpm import MPMSolid3D

    sim = UnifiedSimConfig(n_grid=32)
    n = sim.n_grid
    lbm = _lbm(sim, np.zeros((n, n, n), np.int8))
    solid = MPMSolid3D(sim.make_mpm_config(gravity=(0.0, 0.0, 0.0)), n_particles=4096)
    solid.init_box()
    target = (0.03, 0.0, 0.0) if moving else (0.0, 0.0, 0.0)
    if moving:
        u = GridUnitMapper.from_sim_config(sim).velocity_lbm_to_norm(target)
        solid.set_uniform_velocity(float(u[0]), float(u[1]), float(u[2]))
    proj = MPMToLBMProjector3D(sim)
    proj.project(solid, lbm)
    torch.cuda.synchronize()
    st = proj.get_stats()
    phi, mass, vel = lbm.solid_phi.to_numpy(), lbm.solid_mass.to_numpy(), lbm.solid_vel.to_numpy()
    assert np.all(np.isfinite(phi)) and np.all(np.isfinite(mass)) and np.all(np.isfinite(vel))
    total = float(np.sum(solid.mass.to_numpy().astype(np.float64)))
    assert abs(st["projected_mass"] - total) / max(total, 1.0e-12) < 1.0e-5
    assert st["active_cell_count"] > 0
    assert float(phi.min()) >= 0.0 and float(phi.max()) <= 1.0
    active = mass > 1.0e-12
    assert np.any(active)
    mean = np.average(vel[active].astype(np.float64), axis=0, weights=mass[active].astype(np.float64))
    if moving:
        assert abs(mean[0] - target[0]) < 1.0e-6
        assert abs(mean[1]) < 1.0e-8 and abs(mean[2]) < 1.0e-8
    else:
        assert float(np.max(np.linalg.norm(vel[active], axis=1))) < 1.0e-8
    assert float(np.max(np.linalg.norm(lbm.cell_force.to_numpy(), axis=3))) == 0.0
    assert float(np.max(np.linalg.norm(lbm.hydro_force.to_numpy(), axis=3))) == 0.0

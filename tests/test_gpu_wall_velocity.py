"""The wall velocity application to solid_vel on the device against the
reference's apply_wall_velocity_to_lbm_solid_vel on the same seeded inputs
(tests/golden/wall_velocity_ref.npz / .json).  The FP64 arithmetic follows
numpy's rounding step by step, so the written solid_vel is bit-identical;
the statistics agree to rtol 1e-12 (sums in another order)."""

import json
import os

import numpy as np
import pytest

from tests.diag_compare import assert_same
from tests.golden.make_wall_velocity_fixture import N, inputs, make_root
from tests.test_wall_velocity import base_config

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("policy", ["additive_capped", "replace_capped"])
def test_wall_velocity_matches_reference(policy, tmp_path):
    from mpm_lbm_b200 import wall_velocity as wv
    from mpm_lbm_b200._lib import launch_count
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    with open(os.path.join(GOLD, "wall_velocity_ref.json")) as fh:
        ref = json.load(fh)["apply"][policy]
    want_after = np.load(os.path.join(GOLD, "wall_velocity_ref.npz"))[policy + "_after"]
    make_root(str(tmp_path))
    before, grid = inputs()
    lbm = LBMFluid3D(LBMConfig(nx=N, ny=N, nz=N))
    lbm.init_simulation()
    lbm.solid_vel.from_numpy(before)
    n0 = launch_count()
    got = wv.apply_wall_velocity_to_lbm_solid_vel(lbm, grid, base_config(application_policy=policy),
                                                  root=str(tmp_path))
    assert launch_count() > n0
    np.testing.assert_array_equal(lbm.solid_vel.to_numpy(), want_after)
    assert_same(got, ref, rtol=1e-12)


def test_wall_velocity_grid_shape_is_checked(tmp_path):
    from mpm_lbm_b200 import wall_velocity as wv
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    make_root(str(tmp_path))
    lbm = LBMFluid3D(LBMConfig(nx=N, ny=N, nz=N - 1))
    lbm.init_simulation()
    _, grid = inputs()
    with pytest.raises(ValueError, match="does not match"):
        wv.apply_wall_velocity_to_lbm_solid_vel(lbm, grid, base_config(), root=str(tmp_path))


def test_driver_applies_wall_velocity_after_projection(tmp_path):
    """fsi_driver.py:452-482: after each projection the driver writes the
    capped phase grid into solid_vel (replace policy: the capped grid)."""
    from mpm_lbm_b200.config import FSIDriverConfig
    from mpm_lbm_b200.driver import FSIDriver3D
    from tests.test_wall_velocity import _driver_cfg

    make_root(str(tmp_path))
    cfg_app = base_config(application_policy="replace_capped").to_dict()
    for k in ("wall_velocity_config_path", "boundary_motion_config_path", "geometry_config_path",
              "region_config_path"):
        cfg_app[k] = str(tmp_path / cfg_app[k])
    app_path = tmp_path / "app.json"
    app_path.write_text(json.dumps(cfg_app))
    cfg = _driver_cfg(tmp_path, boundary_motion_mode="prescribed_kinematic",
                      boundary_motion_config_path=cfg_app["boundary_motion_config_path"],
                      wall_velocity_application_mode="solid_vel_experimental",
                      wall_velocity_application_config_path=str(app_path),
                      wall_velocity_application_report_enabled=True)
    drv = FSIDriver3D(FSIDriverConfig(**cfg), str(tmp_path / "out"))
    n = cfg["n_grid"]
    box = (slice(1, 3), slice(2, 5), slice(0, n))

    def builder(config, n_grid, phase):
        g = np.zeros((n_grid, n_grid, n_grid, 3))
        g[box] = (0.02 * (1.0 + phase), -0.005, 0.0)
        return g, {"selected_phase": phase, "finite_pass": True}

    drv.wall_velocity_grid_builder = builder
    drv.wall_velocity_phase_for_step = lambda config, step: (step % 4) / 4.0
    drv.initialize()
    for step in range(2):
        drv.step_once()
        sv = drv.lbm.solid_vel.to_numpy()
        g = np.array([0.02 * (1.0 + step / 4.0), -0.005, 0.0])
        want = (g * (0.01 / np.linalg.norm(g))).astype(np.float32)
        assert np.all(sv[box] == want)
        rep = drv.wall_velocity_application_report["summary"]
        assert rep["applied_cell_count"] == 2 * 3 * n
        assert rep["driver_lbm_step"] == step and rep["report_pass"] and rep["cap_pass"]
    assert len(drv.wall_velocity_application_reports) == 2
    assert os.path.isfile(tmp_path / "out" / "wall_velocity_application_report.json")

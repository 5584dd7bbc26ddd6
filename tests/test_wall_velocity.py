"""Wall velocity application config rules against the reference's own
validation of the same configs (tests/golden/wall_velocity_ref.json, made by
tests/golden/make_wall_velocity_fixture.py).  The device application is
tested in tests/test_gpu_wall_velocity.py."""

import json
import os

import pytest

from mpm_lbm_b200 import wall_velocity as wv
from tests.golden.make_wall_velocity_fixture import CONFIG_FILES, config_variants, make_root

REF = os.path.join(os.path.dirname(__file__), "golden", "wall_velocity_ref.json")


def base_config(**over):
    fields = dict(application_id="fixture_application", **CONFIG_FILES,
                  scope_note="Step 36 opt-in experimental solid_vel application smoke only")
    fields.update(over)
    return wv.WallVelocityApplicationConfig(**fields)


def test_validation_matches_reference(tmp_path):
    with open(REF) as fh:
        ref = json.load(fh)["validation"]
    make_root(str(tmp_path))
    for name, over in config_variants().items():
        rows = wv.validate_wall_velocity_application_config(base_config(**over), root=str(tmp_path))
        assert [[r["check"], r["pass"]] for r in rows] == ref[name], name


def test_invalid_config_raises(tmp_path):
    make_root(str(tmp_path))
    wv.assert_valid_wall_velocity_application_config(base_config(), root=str(tmp_path))
    with pytest.raises(ValueError, match="validation failed"):
        wv.assert_valid_wall_velocity_application_config(base_config(wall_velocity_cap_lbm=0.2), root=str(tmp_path))


def test_config_json_round_trip(tmp_path):
    make_root(str(tmp_path))
    cfg = base_config(application_policy="replace_capped")
    path = tmp_path / "app.json"
    path.write_text(json.dumps(cfg.to_dict()))
    loaded = wv.load_wall_velocity_application_config(str(path), root=str(tmp_path))
    assert loaded == cfg


def test_application_without_grid_builder_fails_loudly(tmp_path):
    with pytest.raises(NotImplementedError, match="grid_builder"):
        wv.apply_wall_velocity_application_to_lbm(None, "x.json", 12, 0)


def _driver_cfg(tmp_path, **over):
    import numpy as np

    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "drv_mb_eng.npz"), allow_pickle=False)
    cfg = json.loads(str(d["config"]))
    cfg.update(over)
    return cfg


def test_driver_config_rules_match_reference(tmp_path):
    """fsi_config.py:184-200."""
    from mpm_lbm_b200.config import FSIDriverConfig

    app = tmp_path / "app.json"
    app.write_text("{}")
    with pytest.raises(ValueError, match="requires boundary_motion_mode='prescribed_kinematic'"):
        FSIDriverConfig(**_driver_cfg(tmp_path, wall_velocity_application_mode="solid_vel_experimental",
                                      wall_velocity_application_config_path=str(app)))
    with pytest.raises(ValueError, match="boundary_motion_config_path is required"):
        FSIDriverConfig(**_driver_cfg(tmp_path, boundary_motion_mode="prescribed_kinematic"))
    with pytest.raises(ValueError, match="must be None when wall_velocity_application_mode='disabled'"):
        FSIDriverConfig(**_driver_cfg(tmp_path, wall_velocity_application_config_path=str(app)))
    with pytest.raises(ValueError, match="must exist"):
        FSIDriverConfig(**_driver_cfg(tmp_path, boundary_motion_mode="prescribed_kinematic",
                                      boundary_motion_config_path="motion.json",
                                      wall_velocity_application_mode="solid_vel_experimental",
                                      wall_velocity_application_config_path=str(tmp_path / "absent.json")))
    FSIDriverConfig(**_driver_cfg(tmp_path, boundary_motion_mode="prescribed_kinematic",
                                  boundary_motion_config_path="motion.json",
                                  wall_velocity_application_mode="solid_vel_experimental",
                                  wall_velocity_application_config_path=str(app)))

"""LBM restart npz format (src/mpm_lbm/sim/lbm/restart.py:10-147) against a
file written by the reference's own writer (tests/golden/lbm_restart_ref.npz,
made by tests/golden/make_restart_fixture.py): reading it, writing the same
arrays, the statistics dictionary, the metadata guard and the errors.  Array
contents and dtypes are compared exactly."""

import json
import os

import numpy as np
import pytest

from mpm_lbm_b200 import restart as rs
from tests.golden.make_restart_fixture import fixture_arrays, fixture_metadata

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REF_NPZ = os.path.join(GOLDEN, "lbm_restart_ref.npz")


def test_reads_the_reference_file():
    arrays, metadata = rs.read_lbm_restart_npz(REF_NPZ)
    want = fixture_arrays()
    assert metadata == fixture_metadata()
    for key in rs.RESTART_ARRAY_KEYS:
        assert arrays[key].dtype == want[key].dtype and arrays[key].shape == want[key].shape
        np.testing.assert_array_equal(arrays[key], want[key])


def test_writes_what_the_reference_writes(tmp_path):
    out = tmp_path / "sub" / "restart.npz"
    stats = rs.write_lbm_restart_npz(out, fixture_arrays(), fixture_metadata())
    with np.load(REF_NPZ) as ref, np.load(out) as got:
        assert sorted(ref.files) == sorted(got.files)
        for key in ref.files:
            assert ref[key].dtype == got[key].dtype and ref[key].shape == got[key].shape, key
            np.testing.assert_array_equal(ref[key], got[key])
    with open(os.path.join(GOLDEN, "lbm_restart_ref_stats.json")) as fh:
        assert json.loads(json.dumps(stats)) == json.load(fh)


def test_extra_keys_are_invisible_to_the_reference_reader(tmp_path):
    out = tmp_path / "restart.npz"
    rs.write_lbm_restart_npz(out, fixture_arrays(), fixture_metadata(), extra={"ext_note": np.arange(3)})
    arrays, metadata = rs.read_lbm_restart_npz(out)
    assert sorted(arrays) == sorted(rs.RESTART_ARRAY_KEYS) and metadata == fixture_metadata()
    with pytest.raises(ValueError, match="collides"):
        rs.write_lbm_restart_npz(out, fixture_arrays(), fixture_metadata(), extra={"rho": np.zeros(1)})


def test_errors_and_guard(tmp_path):
    arrays = fixture_arrays()
    del arrays["static_solid"]
    with pytest.raises(ValueError, match="missing LBM restart arrays: static_solid"):
        rs.write_lbm_restart_npz(tmp_path / "x.npz", arrays, {})
    with pytest.raises(FileNotFoundError):
        rs.read_lbm_restart_npz(tmp_path / "absent.npz")
    assert rs.load_lbm_restart_to_lbm(None, tmp_path / "absent.npz", fixture_metadata()) == {
        "restart_loaded": False, "restart_missing": True}
    with pytest.raises(FileNotFoundError):
        rs.load_lbm_restart_to_lbm(None, tmp_path / "absent.npz", fixture_metadata(), required=True)
    meta = fixture_metadata()
    guard = rs.validate_lbm_restart_metadata(meta, dict(meta, n_grid=8))
    assert guard == {"restart_lbm_boundary_condition_mode_matches": True, "restart_n_grid_matches": False,
                     "restart_target_u_lbm_matches": True}
    with pytest.raises(ValueError, match="metadata mismatch"):
        rs.load_lbm_restart_to_lbm(None, REF_NPZ, dict(meta, target_u_lbm=[0.04, 0.0, 0.0]))
    with pytest.raises(ValueError, match="shape mismatch"):
        rs._validate_restart_shapes(fixture_arrays(), 8)


def test_expected_metadata_from_config():
    from mpm_lbm_b200.config import FSIDriverConfig

    cfg = FSIDriverConfig(n_grid=32)
    meta = rs.expected_restart_metadata_from_config(cfg)
    assert meta == {"lbm_boundary_condition_mode": cfg.lbm_boundary_condition_mode,
                    "lbm_restart_scope": "rho_velocity_populations", "n_grid": 32,
                    "target_u_lbm": [float(u) for u in cfg.target_u_lbm]}

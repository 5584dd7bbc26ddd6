"""End-to-end parity of the CUDA FSIDriver3D against the reference itself.

The fixtures tests/golden/drv_*.npz hold FSIDriver3D.run() of the reference
(its own Taichi kernel code executed by tests/golden/taichi_shim.py) for the
modes none / penalty / moving_boundary (engineering and link-area) /
subcycled / duct with the limited regularized open boundary.  The CUDA driver
runs the same config; tolerances (FP32 after a few coupled steps): fields
rtol 1e-3 on rho/v-scale quantities, particle positions atol 1e-6 (normalised
units), diagnostics rows rtol 2e-3 / atol 2e-7 (the reference's f32 rest state
carries ~4e-9 round-off velocities); masks and link counts exact.
"""

import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["drv_mb_eng", "drv_penalty", "drv_none", "drv_mb_link", "drv_mb_sub", "drv_duct_lim"]


def _load(name):
    p = os.path.join(GOLD, name + ".npz")
    if not os.path.exists(p):
        pytest.skip(f"missing fixture {name}")
    return np.load(p, allow_pickle=False)


@pytest.mark.parametrize("mpm_path", ["binned", "one_phase"])
@pytest.mark.parametrize("name", CASES)
def test_driver_matches_reference(name, mpm_path, tmp_path):
    from mpm_lbm_b200.config import FSIDriverConfig
    from mpm_lbm_b200.driver import FSIDriver3D

    d = _load(name)
    cfg = json.loads(str(d["config"]))
    if cfg.get("geometry_config_path"):
        from tests.golden.make_fixtures import _duct_geometry_json

        gp = str(tmp_path / "duct_geo.json")
        _duct_geometry_json(gp, cfg["n_particles"])
        cfg["geometry_config_path"] = gp
    drv = FSIDriver3D(FSIDriverConfig(**cfg), str(tmp_path / "out"), mpm_path=mpm_path)
    drv.initialize()
    np.testing.assert_array_equal(drv.lbm.solid.to_numpy(), d["init_solid"])
    np.testing.assert_allclose(drv.solid.x.to_numpy(), d["init_x"], rtol=0, atol=1e-7)
    np.testing.assert_array_equal(drv.solid.fixed_mask.to_numpy(), d["init_fixed"])
    np.testing.assert_allclose(drv.solid.mass.to_numpy(), d["init_mass"], rtol=1e-6)
    rows = drv.run()
    ref_rows = json.loads(str(d["rows"]))
    assert len(rows) == len(ref_rows)
    # the measured differences, relative to each field's largest magnitude
    got_f = {"rho": drv.lbm.rho.to_numpy(), "v": drv.lbm.v.to_numpy(), "F": drv.lbm.F.to_numpy(),
             "phi": drv.lbm.solid_phi.to_numpy(), "hydro": drv.lbm.hydro_force.to_numpy(),
             "x": drv.solid.x.to_numpy(), "mpm_v": drv.solid.v.to_numpy(), "mpm_F": drv.solid.F.to_numpy()}
    ref_f = {"rho": d["lbm_rho"], "v": d["lbm_v"], "F": d["lbm_F"], "phi": d["lbm_solid_phi"],
             "hydro": d["lbm_hydro_force"], "x": d["mpm_x"], "mpm_v": d["mpm_v"], "mpm_F": d["mpm_F"]}
    errs = {k: float(np.abs(got_f[k].astype(np.float64) - ref_f[k]).max() / max(np.abs(ref_f[k]).max(), 1e-30))
            for k in got_f}
    row_err = 0.0
    for got, ref in zip(rows, ref_rows):
        for k, v in ref.items():
            if isinstance(v, (int, float)) and not isinstance(v, bool) and k != "elapsed_seconds":
                row_err = max(row_err, abs(got[k] - v) / max(abs(v), 1e-6))
    print(name, mpm_path, {k: f"{e:.1e}" for k, e in errs.items()}, f"rows {row_err:.1e}")
    np.testing.assert_array_equal(drv.lbm.solid.to_numpy(), d["lbm_solid"])
    np.testing.assert_allclose(drv.lbm.rho.to_numpy(), d["lbm_rho"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(drv.lbm.v.to_numpy(), d["lbm_v"], rtol=1e-3, atol=2e-7)
    np.testing.assert_allclose(drv.lbm.F.to_numpy(), d["lbm_F"], rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(drv.lbm.solid_phi.to_numpy(), d["lbm_solid_phi"], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(drv.lbm.hydro_force.to_numpy(), d["lbm_hydro_force"], rtol=2e-3, atol=1e-7)
    np.testing.assert_allclose(drv.solid.x.to_numpy(), d["mpm_x"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(drv.solid.v.to_numpy(), d["mpm_v"], rtol=2e-3, atol=1e-5)
    np.testing.assert_allclose(drv.solid.F.to_numpy(), d["mpm_F"], rtol=0, atol=1e-5)
    for got, ref in zip(rows, ref_rows):
        for k, v in ref.items():
            if k in ("elapsed_seconds",):
                continue
            if isinstance(v, str):
                assert got[k] == v, (k, got[k], v)
            elif k in ("bb_link_count", "active_cell_count", "mb_subcycle_force_sample_count", "step",
                       "total_mpm_substeps"):
                assert int(got[k]) == int(v), (k, got[k], v)
            else:
                assert np.isclose(got[k], v, rtol=2e-3, atol=2e-7), (k, got[k], v)

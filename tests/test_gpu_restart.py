"""LBM restarts and FSI resume on the device.

1. A restart file written by the reference's own writer
   (tests/golden/lbm_restart_ref.npz) loads into LBMFluid3D through
   load_lbm_restart_to_lbm (restart.py:50-78): every restart field reads back
   exactly, and save_lbm_restart_from_lbm writes the same arrays again.
2. save_fsi_restart / load_fsi_restart: a fresh driver of the same
   configuration, loaded from a file saved after K = 2 FSI steps and advanced
   2 steps, matches the saved driver advanced the same 2 steps -- populations,
   density and velocity rtol 1e-5 / atol 1e-7, particle positions atol 1e-6,
   deformation gradients atol 1e-5 (float atomic sums differ in order between
   runs); solid masks and step counters exactly.
"""

import os

import numpy as np
import pytest

from tests.golden.make_restart_fixture import N, fixture_arrays, fixture_metadata

pytestmark = pytest.mark.gpu

REF_NPZ = os.path.join(os.path.dirname(__file__), "golden", "lbm_restart_ref.npz")
K = 2


def test_reference_restart_loads_and_saves_back(tmp_path):
    from mpm_lbm_b200 import restart as rs
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    lbm = LBMFluid3D(LBMConfig(nx=N, ny=N, nz=N))
    lbm.init_geo_array(np.zeros((N, N, N), np.int8))
    lbm.init_simulation()
    report = rs.load_lbm_restart_to_lbm(lbm, REF_NPZ, fixture_metadata(), required=True)
    assert report["restart_loaded"] and report["restart_n_grid_matches"]
    want = fixture_arrays()
    got = {"rho": lbm.rho.to_numpy(), "v": lbm.v.to_numpy(), "F": lbm.F.to_numpy(), "f": lbm.f.to_numpy(),
           "solid": lbm.solid.to_numpy(), "static_solid": lbm.static_solid.to_numpy()}
    for key, value in got.items():
        np.testing.assert_array_equal(value, want[key], err_msg=key)
    out = tmp_path / "again.npz"
    rs.save_lbm_restart_from_lbm(lbm, out, fixture_metadata())
    arrays, metadata = rs.read_lbm_restart_npz(out)
    assert metadata == fixture_metadata()
    for key in rs.RESTART_ARRAY_KEYS:
        assert arrays[key].dtype == want[key].dtype, key
        np.testing.assert_array_equal(arrays[key], want[key], err_msg=key)


def _box_case():
    from mpm_lbm_b200.batch import BoxCase

    return BoxCase(lattice=(32, 32, 48), tau=0.6, mode="moving_boundary", solid="block", solid_cells=6, e_lu=0.05,
                   mpm_substeps=4, seed=1)


def _duct_case():
    from mpm_lbm_b200.cases import DuctPlateCase

    return DuctPlateCase(lattice=(64, 32, 32), plate=(2, 16, 24), lbm_substeps=12, mpm_substeps=4)


def _state(drv):
    return {"F": drv.lbm.F.to_numpy(), "rho": drv.lbm.rho.to_numpy(), "v": drv.lbm.v.to_numpy(),
            "solid": drv.lbm.solid.to_numpy(), "x": drv.solid.x.to_numpy(), "Fp": drv.solid.F.to_numpy(),
            "counters": (drv.current_lbm_step, drv.total_lbm_substeps, drv.total_mpm_substeps)}


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("which", ["box_moving_boundary", "duct_subcycled"])
def test_fsi_resume_continues_the_saved_run(tmp_path, which, graph):
    import torch

    from mpm_lbm_b200 import restart as rs

    case = _box_case() if which == "box_moving_boundary" else _duct_case()
    a = case.make_driver()
    a.use_cuda_graph = graph
    for _ in range(K):  # K steps end on a graph-replay boundary in both cases
        a.step_once()
    path = tmp_path / "fsi.npz"
    rs.save_fsi_restart(a, path)
    for _ in range(2):
        a.step_once()
    torch.cuda.synchronize()
    want = _state(a)

    b = case.make_driver()
    b.use_cuda_graph = graph
    report = rs.load_fsi_restart(b, path)
    assert report["counters"]["current_lbm_step"] == K
    for _ in range(2):
        b.step_once()
    torch.cuda.synchronize()
    got = _state(b)
    assert got["counters"] == want["counters"]
    np.testing.assert_array_equal(got["solid"], want["solid"])
    np.testing.assert_allclose(got["F"], want["F"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(got["rho"], want["rho"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(got["v"], want["v"], rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(got["x"], want["x"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(got["Fp"], want["Fp"], rtol=0, atol=1e-5)
    # the LBM part of the file is a reference-format restart
    arrays, metadata = rs.read_lbm_restart_npz(path)
    assert arrays["F"].shape == tuple(a.lbm.dims) + (19,)


def test_fsi_resume_rejects_another_configuration(tmp_path):
    from mpm_lbm_b200 import restart as rs

    a = _box_case().make_driver()
    a.step_once()
    path = tmp_path / "fsi.npz"
    rs.save_fsi_restart(a, path)
    other = _duct_case().make_driver()
    with pytest.raises(ValueError, match="does not match"):
        rs.load_fsi_restart(other, path)
    plain = tmp_path / "plain.npz"
    rs.save_lbm_restart_from_lbm(a.lbm, plain, {"n_grid": 48})
    with pytest.raises(ValueError, match="no FSI resume state"):
        rs.load_fsi_restart(a, plain)

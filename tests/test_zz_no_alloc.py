"""fsi_mask_rebuild_static_scratch (the mask rebuild whose changed-cell list
lives in the library's own device array) against fsi_mask_rebuild with a
caller-provided change_list: two twin lattices, two consecutive rebuilds with
a moving solid-fraction blob, both called through the C ABI.  The twin that
uses the built-in list is handed a state whose change_list is NULL, so the
caller's buffer cannot be what makes it work, and the device's free memory is
the same before and after its second call."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ = 40, 24, 20
CAP = 1 << 20  # cells the built-in change list holds


def _lattice(seed=0):
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    solid = np.zeros((NX, NY, NZ), np.int8)
    solid[:, 0, :] = solid[:, -1, :] = 1
    solid[:, :, 0] = solid[:, :, -1] = 1
    lbm = LBMFluid3D(LBMConfig(nx=NX, ny=NY, nz=NZ, force=(1e-5, 0.0, 0.0)))
    lbm.init_geo_array(solid)
    lbm.init_simulation()
    rng = np.random.default_rng(seed)
    F = lbm.F.to_numpy()
    F = (F * (1.0 + 0.02 * rng.standard_normal(F.shape))).astype(np.float32)
    lbm.F.from_numpy(F)
    rho = F.sum(axis=-1).astype(np.float32)
    lbm.rho.from_numpy(rho)
    for _ in range(2):
        lbm.step_moving_bounceback()
    return lbm


def _blob(center, radius):
    i, j, k = np.meshgrid(np.arange(NX), np.arange(NY), np.arange(NZ), indexing="ij")
    d = np.sqrt((i - center[0]) ** 2 + (j - center[1]) ** 2 + (k - center[2]) ** 2)
    return np.clip(radius + 0.5 - d, 0.0, 1.0).astype(np.float32)


def _rebuild(lbm, name, threshold=0.5, no_scratch=False):
    from mpm_lbm_b200._lib import FsiLbmState, call

    lbm.flush_open_boundary()
    state = lbm.state
    if no_scratch:
        state = FsiLbmState.from_buffer_copy(lbm.state)
        state.change_list = None
    call(name, ctypes.byref(state), ctypes.byref(lbm.params), ctypes.byref(lbm._ctl()), ctypes.c_float(threshold),
         lbm._stream())
    lbm._old_equals_solid = False
    lbm._version += 1


def _compare(a, b):
    np.testing.assert_array_equal(b.solid.to_numpy(), a.solid.to_numpy())
    np.testing.assert_array_equal(b.t_flags.cpu().numpy(), a.t_flags.cpu().numpy())
    assert b._diag().change_count == a._diag().change_count
    np.testing.assert_allclose(b.F.to_numpy(), a.F.to_numpy(), rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(b.rho.to_numpy(), a.rho.to_numpy(), rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(b.v.to_numpy(), a.v.to_numpy(), rtol=1e-5, atol=1e-7)


def test_static_scratch_rebuild_matches_caller_scratch():
    import torch

    a, b = _lattice(), _lattice()
    _compare(a, b)
    changes = []
    for call_no, (center, radius) in enumerate((((14, 12, 10), 5.0), ((17, 12, 10), 6.0))):
        phi = _blob(center, radius)
        for lbm in (a, b):
            lbm.solid_phi.from_numpy(phi)
        _rebuild(a, "fsi_mask_rebuild")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _rebuild(b, "fsi_mask_rebuild_static_scratch", no_scratch=True)
        torch.cuda.synchronize()
        if call_no == 1:  # the first call looked the array up; the second must not allocate at all
            assert torch.cuda.mem_get_info()[0] == free_before
        _compare(a, b)
        changes.append(a._diag().change_count)
        for lbm in (a, b):
            lbm.step_moving_bounceback()
        _compare(a, b)
    assert all(c > 0 for c in changes)  # both rebuilds flipped cells


def test_static_scratch_rejects_lattices_beyond_capacity():
    from mpm_lbm_b200._lib import FsiError, FsiLbmState, call

    lbm = _lattice()
    big = FsiLbmState.from_buffer_copy(lbm.state)
    big.nx, big.ny, big.nz = 128, 128, 65  # 1064960 cells > CAP; rejected before any launch
    assert big.nx * big.ny * big.nz > CAP
    with pytest.raises(FsiError, match="exceeds the built-in change list"):
        call("fsi_mask_rebuild_static_scratch", ctypes.byref(big), ctypes.byref(lbm.params),
             ctypes.byref(lbm._ctl()), ctypes.c_float(0.5), lbm._stream())

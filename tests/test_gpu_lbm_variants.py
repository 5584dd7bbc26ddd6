"""Launch variants of the LBM step agree bit for bit.

FsiLbmParams.tune picks how the step maps onto the SMs, not what it
computes: one cell per thread with 3 or 4 CTAs per SM, with or without an L2
prefetch.  Two lattices with the same seeded state advance the same steps,
one per variant; populations, density, velocity and the per-direction link
counts must be identical (link forces and directional sums, float atomics,
to 1e-5).  Cases: a channel with an obstacle and moving solid walls (moving
bounce-back), open x faces with the regularized-limited outlet, the penalty
force, FP32 and FP16 storage.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(nx, ny, nz, storage, sem="equilibrium_all_population_reset", bc=(0, 0), seed=0):
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    rng = np.random.default_rng(seed)
    solid = np.zeros((nx, ny, nz), np.int8)
    solid[:, 0, :] = solid[:, -1, :] = 1
    solid[:, :, 0] = solid[:, :, -1] = 1
    solid[nx // 3: nx // 3 + 3, 2: ny // 2, 2: nz - 2] = 1
    out = []
    for _ in range(2):
        cfg = LBMConfig(nx=nx, ny=ny, nz=nz, bc_x_left=bc[0], bc_x_right=bc[1], vel_bc_x_left=(0.04, 0.0, 0.0),
                        open_boundary_semantics=sem, force=(2e-6, 0.0, 0.0), population_storage=storage,
                        open_boundary_limiter_enabled=sem.endswith("limited"))
        lbm = LBMFluid3D(cfg)
        lbm.init_geo_array(solid)
        lbm.init_simulation()
        out.append(lbm)
    F = out[0].F.to_numpy()
    F = (F * (1.0 + 0.02 * rng.standard_normal(F.shape))).astype(np.float32)
    sv = (0.01 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32) * solid[..., None]
    for lbm in out:
        lbm.F.from_numpy(F)
        lbm.rho.from_numpy(F.sum(axis=-1).astype(np.float32))
        lbm.solid_vel.from_numpy(sv)
    return out, solid


def _set_tune(lbm, tune):
    lbm.tune = tune
    lbm._sync_params()


def _same(a, b):
    for name in ("F", "rho", "v"):
        x, y = getattr(a, name).to_numpy(), getattr(b, name).to_numpy()
        assert np.array_equal(x, y), f"{name}: {int((x != y).sum())} values differ"
    # link forces and the directional sums are float atomics (their order
    # differs from launch to launch, in any variant); link counts are exact.
    # A solid cell's force is a sum of link terms of up to |0.4| that may
    # cancel, so its rounding is bounded by a few ulps of the largest term,
    # not by the (possibly tiny) result: 4 * 2^-23 * 0.4 = 2e-7.
    ha, hb = a.hydro_force.to_numpy(), b.hydro_force.to_numpy()
    np.testing.assert_allclose(ha, hb, rtol=1e-5, atol=4 * 2.0**-23 * max(float(np.abs(ha).max()), 0.4))
    da, db = a.get_moving_boundary_directional_stats(), b.get_moving_boundary_directional_stats()
    np.testing.assert_array_equal(da["link_count_by_dir"], db["link_count_by_dir"])
    np.testing.assert_allclose(da["solid_force_by_dir"], db["solid_force_by_dir"], rtol=1e-5, atol=1e-9)


CASES = [
    dict(nx=64, ny=12, nz=10, storage="fp32"),
    dict(nx=96, ny=20, nz=9, storage="fp16"),
    dict(nx=64, ny=12, nz=10, storage="fp32", sem="regularized_velocity_pressure_limited", bc=(2, 1)),
    dict(nx=128, ny=16, nz=8, storage="fp16", sem="regularized_velocity_pressure_limited", bc=(2, 1)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("tune", [1, 3, 4])
def test_variants_are_bit_identical_in_moving_bounceback(case, tune):
    import torch

    (ref, var), _ = _pair(**CASES[case])
    _set_tune(var, tune)
    for _ in range(5):  # odd count: ends on the swapped AA layout
        ref.step_moving_bounceback()
        var.step_moving_bounceback()
    torch.cuda.synchronize()
    _same(ref, var)


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
@pytest.mark.parametrize("tune", [1, 4])
def test_variants_with_the_penalty_force(storage, tune):
    import torch

    (ref, var), solid = _pair(64, 12, 10, storage)
    _set_tune(var, tune)
    phi = np.where(solid > 0, 0.9, 0.0).astype(np.float32)
    phi[20:24, 3:6, 3:6] = 0.4  # fluid cells inside the penalty zone
    for lbm in (ref, var):
        lbm.solid_phi.from_numpy(phi)
    for _ in range(4):
        for lbm in (ref, var):
            lbm._penalty = (1.0e-3, 1.0e-6, 1.0e-4)  # armed for the next step, as build_penalty_force does
            lbm.step()
    torch.cuda.synchronize()
    for name in ("F", "rho", "v"):
        assert np.array_equal(getattr(ref, name).to_numpy(), getattr(var, name).to_numpy()), name


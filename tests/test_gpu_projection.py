"""MPM -> LBM projection (coupling/projection.py:21-97) on the GPU against the
CPU oracle, bit for bit.

fsi_project_ordered sums every cell's terms in particle order with IEEE FP32
adds, the order of a serial run of the reference's particle loop, which is
the order the oracle sums in.  So for the same particle state solid_phi,
solid_mass and solid_vel are identical to the oracle's bits, and identical
from run to run; the solid mask built from solid_phi >= threshold
(fluid.py:1847-1861) then cannot flip on a cell whose phi sits a few ulps
from the threshold.  The atomic projection (fsi_project) agrees to FP32
rounding only.

Cases: a jittered plate with random velocities and J (the benchmark's
particle layout); particles packed so densely that a cell has more
contributors than the shared-memory ranking holds (the merge fallback);
particles on the lattice edges and outside it (base cells -2, -1 and beyond).
"""

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N = 40
DT_LBM = 1.0e-3


def _particles(kind, seed=0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / N
    if kind == "plate":
        from mpm_lbm_b200.geometry import jittered_block

        x = jittered_block((10, 3, 8), (12, 30, 32), dx, ppc_axis=2, seed=seed)
    elif kind == "packed":
        # 3 x 3 x 3 cells holding 60 particles each: ~1600 contributors per cell
        c = rng.integers(18, 21, size=(1620, 3)).astype(np.float64)
        x = ((c + rng.uniform(0.0, 1.0, size=c.shape)) * dx).astype(np.float32)
        x = np.concatenate([x, jittered_block_small(rng, dx)])
    else:  # edges
        k = rng.integers(-3, N + 3, size=(3000, 3)).astype(np.float64)
        frac = rng.choice([0.0, 0.25, 0.5, 0.75, 0.999], size=k.shape)
        x = ((k + frac) * dx).astype(np.float32)
    n = len(x)
    v = (0.05 * rng.standard_normal((n, 3))).astype(np.float32)
    jp = rng.uniform(0.6, 1.4, size=n).astype(np.float32)
    jp[:5] = -0.1  # max(J, 0) clamps these to zero volume
    vol0 = np.full(n, dx ** 3 / 8.0, np.float32)
    mass = (vol0 * np.float32(1.2)).astype(np.float32)
    return x, v, jp, vol0, mass


def jittered_block_small(rng, dx):
    c = rng.integers(5, 9, size=(400, 3)).astype(np.float64)
    return ((c + rng.uniform(0.0, 1.0, size=c.shape)) * dx).astype(np.float32)


def _setup(kind):
    from mpm_lbm_b200.config import LBMConfig, MPMConfig, UnifiedSimConfig
    from mpm_lbm_b200.coupling import MPMToLBMProjector3D
    from mpm_lbm_b200.lbm import LBMFluid3D
    from mpm_lbm_b200.mpm import MPMSolid3D

    x, v, jp, vol0, mass = _particles(kind)
    n = len(x)
    sim = UnifiedSimConfig(n_grid=N, mpm_dt=4e-4, lbm_dt_phys_override_s=DT_LBM)
    lbm = LBMFluid3D(LBMConfig(nx=N, ny=N, nz=N))
    lbm.init_geo_array(np.zeros((N, N, N), np.int8))
    lbm.init_simulation()
    solid = MPMSolid3D(MPMConfig(n_grid=N, dx=1.0 / N, dt=4e-4), n)
    solid.init_from_numpy(x, vol0, mass, v_np=v)
    solid.Jp.from_numpy(jp)
    proj = MPMToLBMProjector3D(sim)
    ol = orc.OracleLBM(N, N, N)
    om = orc.OracleMPM(N, 1.0 / N, 4e-4, n)
    om.x[...] = x
    om.v[...] = v
    om.Jp[...] = jp
    om.vol0[...] = vol0
    om.mass[...] = mass
    oc = orc.OracleCoupling(N, sim.dx_norm, sim.lbm_dt_phys)
    oc.project(om, ol)
    return lbm, solid, proj, ol, oc


@pytest.mark.parametrize("kind", ["plate", "packed", "edges"])
def test_ordered_projection_is_bit_identical_to_oracle(kind):
    import torch

    lbm, solid, proj, ol, oc = _setup(kind)
    for rep in range(2):  # the same bits on a second call (scratch reused)
        proj.project(solid, lbm)
        torch.cuda.synchronize()
        phi, m, sv = lbm.solid_phi.to_numpy(), lbm.solid_mass.to_numpy(), lbm.solid_vel.to_numpy()
        assert np.array_equal(phi, ol.solid_phi), f"phi differs in {int((phi != ol.solid_phi).sum())} cells"
        assert np.array_equal(m, ol.solid_mass)
        assert np.array_equal(sv, ol.solid_vel)
        st = proj.get_stats()
        assert st["active_cell_count"] == oc.stats.active_cell_count
        assert st["max_phi_raw"] == pytest.approx(oc.stats.max_phi_raw, rel=0, abs=0)
        # the statistic is an FP64 sum on the device (the oracle accumulates it in FP32)
        assert st["projected_mass"] == pytest.approx(float(np.sum(ol.solid_mass.astype(np.float64))), rel=1e-12)
    if kind == "packed":
        assert float(ol.solid_phi.max()) == 1.0  # clamped: the dense cells do exceed the ranking capacity
    # the atomic projection agrees to FP32 rounding
    proj.project_unordered(solid, lbm)
    torch.cuda.synchronize()
    np.testing.assert_allclose(lbm.solid_phi.to_numpy(), ol.solid_phi, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(lbm.solid_mass.to_numpy(), ol.solid_mass, rtol=1e-5, atol=1e-12)

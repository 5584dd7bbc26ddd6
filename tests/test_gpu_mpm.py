"""MPM substep and reaction transfer on the GPU against the CPU oracle.

Covers the one-phase kernels (fsi_mpm_p2g / grid_update / g2p and
fsi_reaction_to_grid, mpm/solid.py:212-315, coupling/*.py reaction
transfers), the binned substeps (fsi_mpm_bin + fsi_mpm_substeps_binned) and the
particle binning itself, which is integer work and must be bit-exact.

Tolerances: grid sums are FP32 atomics whose order differs between the GPU and
the sequential oracle, so particle state agrees to a few FP32 ulps of the
largest value of each field after several substeps."""

import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N_GRID = 32
DX = 1.0 / N_GRID
DT = 2.0e-4
YOUNG, NU, RHO = 400.0, 0.2, 1.0
GRAVITY = (0.0, -9.8, 0.0)


def _particles(seed=0):
    from mpm_lbm_b200.geometry import jittered_block

    rng = np.random.default_rng(seed)
    x = jittered_block((10, 9, 11), (18, 15, 17), DX, ppc_axis=2, seed=seed)
    n = len(x)
    vol0 = np.full(n, DX ** 3 / 8.0, np.float32)
    mass = (vol0 * np.float32(RHO)).astype(np.float32)
    v = (0.3 * rng.standard_normal((n, 3))).astype(np.float32)
    fixed = (x[:, 1] < 9.6 * DX).astype(np.int8)
    F = (np.eye(3) + 0.05 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    C = (2.0 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    return x, vol0, mass, v, fixed, F, C


def make_solids(seed=0, lock_z=False, damping=0.0):
    from mpm_lbm_b200.config import MPMConfig
    from mpm_lbm_b200.mpm import MPMSolid3D

    x, vol0, mass, v, fixed, F, C = _particles(seed)
    n = len(x)
    cfg = MPMConfig(n_grid=N_GRID, dx=DX, dt=DT, gravity=GRAVITY, young_modulus=YOUNG, poisson_ratio=NU, p_rho=RHO,
                    mpm_planar_constraint_mode="lock_z" if lock_z else "disabled",
                    mpm_velocity_damping=damping,
                    mpm_damping_application="particle_velocity_post_g2p" if damping > 0 else "disabled")
    gpu = MPMSolid3D(cfg, n)
    gpu.init_from_numpy(x, vol0, mass, v_np=v, fixed_mask_np=fixed)
    ora = orc.OracleMPM(N_GRID, DX, DT, n, gravity=GRAVITY, p_rho=RHO, young_modulus=YOUNG, poisson_ratio=NU,
                        lock_z=lock_z, damping=damping)
    ora.init_from_numpy(x, vol0, mass, v_np=v, fixed_mask_np=fixed)
    free = fixed == 0
    Fg, Cg = np.tile(np.eye(3, dtype=np.float32), (n, 1, 1)), np.zeros_like(C)
    Fg[free], Cg[free] = F[free], C[free]
    ora.F[...] = Fg
    ora.C[...] = Cg
    gpu.F.from_numpy(Fg)
    gpu.C.from_numpy(Cg)
    return gpu, ora


def _close(a, b, rel, name):
    scale = max(float(np.max(np.abs(b))), 1e-30)
    err = float(np.max(np.abs(a - b)))
    assert err <= rel * scale, f"{name}: max |diff| {err:.3e} > {rel:.1e} x {scale:.3e}"


def compare_particles(gpu, ora, rel=2e-5):
    _close(gpu.x.to_numpy(), ora.x, 1e-6, "x")
    _close(gpu.v.to_numpy(), ora.v, rel, "v")
    _close(gpu.C.to_numpy(), ora.C, rel, "C")
    _close(gpu.F.to_numpy(), ora.F, rel, "F")
    _close(gpu.Jp.to_numpy(), ora.Jp, rel, "Jp")


def compare_grid(gpu, ora, rel=2e-5):
    _close(gpu.grid_m.to_numpy(), ora.grid_m, rel, "grid_m")
    _close(gpu.grid_v.to_numpy(), ora.grid_v, rel, "grid_v")
    _close(gpu.grid_f_ext.to_numpy(), ora.grid_f_ext, rel, "grid_f_ext")


def expected_chunks(counts, start):
    """Chunk table of fsi_mpm_bin: each bin of c particles cut into
    ceil(c / FSI_BIN_CHUNK) chunks of equal size (the first c % n one
    larger)."""
    from mpm_lbm_b200._lib import FSI_BIN_CHUNK

    cap = FSI_BIN_CHUNK
    chunks = []
    for s, k in zip(start, counts):
        k = int(k)
        if k == 0:
            continue
        n = (k + cap - 1) // cap
        sz, rem = divmod(k, n)
        off = int(s)
        for i in range(n):
            m = sz + (1 if i < rem else 0)
            chunks.append((off, m))
            off += m
    return np.array(chunks, np.int32).reshape(-1, 2)


def expected_bins(x, n_grid, edge=8):
    """Bin keys, counts and chunk table restated on the CPU in FP32."""
    inv_dx = np.float32(n_grid)
    xp = (x.astype(np.float32) * inv_dx).astype(np.float32)
    base = (xp - np.float32(0.5)).astype(np.int32)  # truncation toward zero
    c = np.clip(base, 0, n_grid - 1) // edge
    nb = (n_grid + edge - 1) // edge
    key = (c[:, 2] * nb + c[:, 1]) * nb + c[:, 0]
    counts = np.bincount(key, minlength=nb ** 3)
    start = np.concatenate([[0], np.cumsum(counts)[:-1]])
    return key.astype(np.int32), counts, start, expected_chunks(counts, start)


@pytest.mark.parametrize("case", ["block", "edges"])
def test_binning_is_bit_exact(case):
    gpu, _ = make_solids()
    x = gpu.x.to_numpy()
    if case == "edges":
        # positions on cell faces, on the 0.5-offset the base cell truncates at,
        # and outside [dx, 1 - dx] (clamped into the first/last bin)
        rng = np.random.default_rng(5)
        k = rng.integers(0, N_GRID, size=x.shape).astype(np.float32)
        pick = rng.integers(0, 4, size=x.shape)
        x = np.where(pick == 0, k * np.float32(DX), x)
        x = np.where(pick == 1, (k + np.float32(0.5)) * np.float32(DX), x)
        x = np.where(pick == 2, rng.uniform(-0.02, 1.02, size=x.shape), x).astype(np.float32)
        gpu.x.from_numpy(x)
    gpu.rebin()
    t = gpu._bins["t"]
    key, counts, start, chunks = expected_bins(x, N_GRID)
    # after the scatter, start holds each bin's end offset
    np.testing.assert_array_equal(t["start"].cpu().numpy(), start + counts)
    assert int(t["meta"][0]) == len(chunks)
    np.testing.assert_array_equal(t["chunk"][: len(chunks)].cpu().numpy(), chunks)
    assert int(t["count"].abs().sum()) == 0  # reset for the next binning
    perm = t["perm"].cpu().numpy()
    assert sorted(perm.tolist()) == list(range(len(x)))
    for b in np.nonzero(counts)[0]:
        got = np.sort(perm[start[b]: start[b] + counts[b]])
        np.testing.assert_array_equal(got, np.nonzero(key == b)[0])
    # within each bin the particles are ordered by base cell (z, y, x within the 8^3 block)
    xp = (x.astype(np.float32) * np.float32(N_GRID)).astype(np.float32)
    local = np.clip((xp - np.float32(0.5)).astype(np.int32), 0, N_GRID - 1) % 8
    cell = (local[:, 2] * 8 + local[:, 1]) * 8 + local[:, 0]
    for b in np.nonzero(counts)[0]:
        assert np.all(np.diff(cell[perm[start[b]: start[b] + counts[b]]]) >= 0)


def test_one_phase_substeps_match_oracle():
    gpu, ora = make_solids()
    for _ in range(4):
        gpu.substep()
        ora.substep()
    compare_particles(gpu, ora)
    compare_grid(gpu, ora)


META_OVERFLOW = 4  # bins->meta[4]: chunks scattered without the shared-memory tile


@pytest.mark.parametrize("calls", [[1] * 5, [5], [2, 4, 1], [7]])
@pytest.mark.parametrize("lock_z,damping", [(False, 0.0), (True, 0.0), (False, 5.0)])
def test_binned_substeps_match_oracle(lock_z, damping, calls):
    """fsi_mpm_substeps_binned called with the given substep counts in turn:
    every buffer of the rotation, the zeroing of recorded boxes within a call
    and by the next call's prologue are exercised."""
    gpu, ora = make_solids(lock_z=lock_z, damping=damping)
    for count in calls:
        gpu.substeps_binned(count)
        for _ in range(count):
            ora.substep()
        compare_grid(gpu, ora)
    compare_particles(gpu, ora)
    compare_grid(gpu, ora)
    assert int(gpu._bins["t"]["meta"][META_OVERFLOW]) == 0  # every chunk was staged in shared memory


def test_binned_then_one_phase_switches_grid_layout():
    gpu, ora = make_solids()
    gpu.substep_binned()
    ora.substep()
    gpu.substep()
    ora.substep()
    gpu.substep_binned()
    ora.substep()
    compare_particles(gpu, ora)
    compare_grid(gpu, ora)


def test_binned_with_stale_bins_takes_the_unstaged_path():
    """Bins left stale after the particles are scattered across the domain:
    chunk boxes overflow the shared-memory tile and the global-atomic path
    runs; results still match the oracle."""
    gpu, ora = make_solids(seed=3)
    gpu.rebin()
    gpu.rebin_interval = 10 ** 9
    rng = np.random.default_rng(9)
    x = ora.x + rng.uniform(-6 * DX, 6 * DX, ora.x.shape).astype(np.float32)
    x = np.clip(x, 4 * DX, 1 - 4 * DX).astype(np.float32)
    ora.x[...] = x
    gpu.x.from_numpy(x)
    gpu.substeps_binned(3)
    for _ in range(3):
        ora.substep()
    assert int(gpu._bins["t"]["meta"][META_OVERFLOW]) > 0
    compare_particles(gpu, ora)
    compare_grid(gpu, ora)


def _lbm_and_coupling(kind, seed=1):
    import torch  # noqa: F401

    from mpm_lbm_b200.config import LBMConfig, UnifiedSimConfig
    from mpm_lbm_b200.coupling import (LinkAreaMovingBoundaryCoupler3D, MovingBoundaryFSICoupler3D,
                                       PenaltyFSICoupler3D)
    from mpm_lbm_b200.lbm import LBMFluid3D

    sim = UnifiedSimConfig(n_grid=N_GRID, mpm_dt=DT, lbm_dt_phys_override_s=1.0e-3)
    rng = np.random.default_rng(seed)
    hydro = (1e-6 * rng.standard_normal((N_GRID,) * 3 + (3,))).astype(np.float32)
    phi = rng.uniform(0.0, 1.0, (N_GRID,) * 3).astype(np.float32)
    phi[phi < 0.3] = 0.0  # some particles fall below phi_min and are gated off
    lbm = LBMFluid3D(LBMConfig(nx=N_GRID, ny=N_GRID, nz=N_GRID))
    lbm.init_geo_array(np.zeros((N_GRID,) * 3, np.int8))
    lbm.init_simulation()
    lbm.hydro_force.from_numpy(hydro)
    lbm.solid_phi.from_numpy(phi)
    cap = 2e-9
    if kind == 0:
        cpl = PenaltyFSICoupler3D(sim)
    elif kind == 1:
        cpl = MovingBoundaryFSICoupler3D(sim, force_cap_norm=cap)
    else:
        cpl = LinkAreaMovingBoundaryCoupler3D(sim, force_cap_norm=cap)
    olbm = orc.OracleLBM(N_GRID, N_GRID, N_GRID)
    olbm.hydro_force[...] = hydro
    olbm.solid_phi[...] = phi
    oc = orc.OracleCoupling(N_GRID, sim.dx_norm, sim.lbm_dt_phys, mb_force_cap_norm=cap)
    if kind == 2:
        oc.update_area_scale(olbm)
    return lbm, cpl, olbm, oc


def _react_stats(st):
    return (int(st.active_reaction_particle_count), float(st.max_particle_reaction_norm),
            float(st.max_grid_reaction_norm), np.array(st.net_particle_reaction), np.array(st.net_grid_reaction))


def _oracle_react_stats(st, kind):
    if kind == 0:
        return (0, 0.0, float(st.max_reaction_grid_force_norm), np.zeros(3), np.array(st.net_reaction_grid_force))
    return (int(st.active_reaction_particle_count), float(st.max_particle_reaction_norm),
            float(st.max_grid_reaction_norm), np.array(st.net_particle_reaction_force),
            np.array(st.net_grid_reaction_force))


@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("path", ["binned", "binned_sequence", "one_phase"])
def test_reaction_substeps_match_oracle(kind, path):
    gpu, ora = make_solids(seed=2)
    lbm, cpl, olbm, oc = _lbm_and_coupling(kind)
    if path == "binned_sequence":
        gpu.substeps_binned(3, cpl, lbm)
    for _ in range(3):
        if path == "binned":
            gpu.substep_binned(cpl, lbm)
        elif path == "binned_sequence":
            pass
        else:
            gpu.clear_grid()
            gpu.p2g()
            if kind == 0:
                cpl.add_lbm_reaction_to_mpm_grid(gpu, lbm)
            else:
                cpl._react(gpu, lbm)
            gpu.grid_update()
            gpu.g2p()
        ora.clear_grid()
        ora.p2g()
        oc.stats = orc.CouplingStats()
        oc.reaction(kind, ora, olbm)
        ora.grid_update()
        ora.g2p()
    compare_particles(gpu, ora)
    compare_grid(gpu, ora)
    got, exp = _react_stats(cpl._reaction_stats()), _oracle_react_stats(oc.stats, kind)
    if kind != 0:
        assert got[0] == exp[0]
        np.testing.assert_allclose(got[1], exp[1], rtol=1e-5)
        np.testing.assert_allclose(got[3], exp[3], rtol=1e-4, atol=1e-6 * np.abs(exp[3]).max())
    np.testing.assert_allclose(got[2], exp[2], rtol=1e-5)
    np.testing.assert_allclose(got[4], exp[4], rtol=1e-4, atol=1e-6 * np.abs(exp[4]).max())
    if kind == 2:
        st = cpl._reaction_stats()
        np.testing.assert_allclose(st.area_scale, oc.cp.area_scale, rtol=1e-6)


def test_binned_layout_and_argument_checks():
    from mpm_lbm_b200._lib import FsiError, FsiMpmBins, call

    nb, mc = ctypes.c_int32(), ctypes.c_int32()
    call("fsi_mpm_bins_layout", 1000, 50, ctypes.byref(nb), ctypes.byref(mc))
    # ceil(50 / 8)^3 bins; ceil(1000 / FSI_BIN_CHUNK) + min(1000, bins) chunks
    assert nb.value == 7 ** 3 and mc.value == 8 + 7 ** 3
    with pytest.raises(FsiError):
        call("fsi_mpm_bins_layout", 0, 50, ctypes.byref(nb), ctypes.byref(mc))
    gpu, _ = make_solids()
    gpu.rebin()
    bad = FsiMpmBins.from_buffer_copy(gpu._bins["struct"])
    bad.max_chunks = 1
    with pytest.raises(FsiError, match="max_chunks"):
        call("fsi_mpm_bin", ctypes.byref(gpu.particles), ctypes.byref(gpu.grid), ctypes.byref(gpu.params),
             ctypes.byref(bad), None)
    with pytest.raises(FsiError, match="n_substeps"):
        call("fsi_mpm_substeps_binned", ctypes.byref(gpu.particles), gpu._bins["grids"],
             ctypes.byref(gpu._bins["struct"]), ctypes.byref(gpu.params), -1, None, None, None, None, None)
    bad_grids = (type(gpu._bins["grids"][0]) * 3)(*gpu._bins["grids"])
    bad_grids[2].n = gpu.n_grid + 1
    with pytest.raises(FsiError, match="differ in size"):
        call("fsi_mpm_substeps_binned", ctypes.byref(gpu.particles), bad_grids,
             ctypes.byref(gpu._bins["struct"]), ctypes.byref(gpu.params), 1, None, None, None, None, None)

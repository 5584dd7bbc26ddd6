"""Seeded draws of the batching configuration, each run alone through the
CUDA FSIDriver3D and through the CPU oracle.

The cases come from `sample_box_cases` (per-axis edges in {32, 48} here so
that the oracle finishes in seconds, tau ~ U[0.52, 0.8], a block or a
cantilevered plate of 4..16 cells, E ~ U[0.01, 0.1] in lattice units,
penalty or moving_boundary), 20 FSI steps of one LBM step and 10 MPM
substeps each.  This covers the corners the fixed fixtures do not: tau near
0.52, anisotropic boxes (nx != ny != nz), plates clamped to the wall, and
particle counts that leave partial chunks.

Tolerances (FP32), as in the box-case test: solid masks exact; populations
and density rtol 2e-5 / atol 1e-7; velocity relative L2 within 1e-2 and every
cell within 1e-2 of the largest speed; particle positions atol 1e-6 and
deformation gradients atol 2e-5 (normalised units; the MPM grid sums are
float atomics).
"""

import os

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

STEPS = 20
N_CASES = 6
SEED = 11


def _cases():
    from mpm_lbm_b200.batch import sample_box_cases

    return sample_box_cases(N_CASES, seed=SEED, edges=(32, 48), lbm_steps=STEPS)


_ORACLE = {}


def _oracle(i):
    """The oracle's state after STEPS FSI steps of case i (shared by the
    single-case and the batched test)."""
    if i not in _ORACLE:
        ora = orc.fsi_driver_for_box_case(_cases()[i], threads=min(8, os.cpu_count() or 1))
        for _ in range(STEPS):
            ora.step_once()
        _ORACLE[i] = ora
    return _ORACLE[i]


def _compare(drv, ora, case):
    tag = f"{case.lattice} tau {case.tau:.3f} {case.mode} {case.solid} L={case.solid_cells} E={case.e_lu:.3f}"
    np.testing.assert_array_equal(drv.lbm.solid.to_numpy(), ora.lbm.solid, err_msg=tag)
    np.testing.assert_allclose(drv.lbm.F.to_numpy(), ora.lbm.F, rtol=2e-5, atol=1e-7, err_msg=tag)
    np.testing.assert_allclose(drv.lbm.rho.to_numpy(), ora.lbm.rho, rtol=2e-5, atol=1e-7, err_msg=tag)
    v, vo = drv.lbm.v.to_numpy().astype(np.float64), ora.lbm.v.astype(np.float64)
    umax = float(np.abs(vo).max())
    assert umax > 0.0, tag
    rel_l2 = float(np.linalg.norm(v - vo) / np.linalg.norm(vo))
    dmax = float(np.abs(v - vo).max())
    print(f"{tag}: velocity rel L2 {rel_l2:.2e}, max |dv| {dmax:.2e} of max |v| {umax:.2e}")
    assert rel_l2 <= 1e-2, tag
    assert dmax <= 1e-2 * umax, tag
    np.testing.assert_allclose(drv.solid.x.to_numpy(), ora.solid.x, rtol=0, atol=1e-6, err_msg=tag)
    np.testing.assert_allclose(drv.solid.F.to_numpy(), ora.solid.F, rtol=0, atol=2e-5, err_msg=tag)


@pytest.mark.parametrize("i", range(N_CASES))
def test_sampled_case_matches_oracle(i):
    import torch

    case = _cases()[i]
    drv = case.make_driver()
    for _ in range(STEPS):
        drv.step_once()
    torch.cuda.synchronize()
    _compare(drv, _oracle(i), case)


def test_sampled_cases_batched_match_oracle():
    """The same six cases in one FSIBatch (one launch per phase for all of
    them, replayed from a CUDA graph), each against the oracle."""
    from mpm_lbm_b200.batch import FSIBatch

    cases = _cases()
    batch = FSIBatch(capacity=8, mpm_substeps=cases[0].mpm_substeps)
    slots = [batch.add(c.make_driver()) for c in cases]
    for _ in range(STEPS):
        batch.step(use_graph=True)
    for i, (slot, case) in enumerate(zip(slots, cases)):
        _compare(batch.sync_case(slot), _oracle(i), case)

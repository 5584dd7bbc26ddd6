"""Batched FSI (FSIBatch, fsi_batch_* entry points) against the same cases
advanced one at a time by FSIDriver3D.

Three cases of different lattice shapes, relaxation times, materials and
coupling modes share one batch.  After N batched FSI steps -- eager and
replayed from a CUDA graph -- every case matches its own FSIDriver3D run:
populations, density and velocity rtol 1e-5 / atol 1e-7, particle positions
atol 1e-6 (normalised units), deformation gradients atol 1e-5 (the MPM grid
sums are float atomics whose order differs between runs); solid masks
bit-exact.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 6


def _cases():
    from mpm_lbm_b200.batch import BoxCase

    return [
        BoxCase(lattice=(32, 32, 48), tau=0.6, mode="moving_boundary", solid="block", solid_cells=6, e_lu=0.05,
                mpm_substeps=4, seed=1),
        BoxCase(lattice=(48, 32, 32), tau=0.7, mode="penalty", solid="plate", solid_cells=8, e_lu=0.02,
                mpm_substeps=4, seed=2),
        BoxCase(lattice=(32, 48, 32), tau=0.55, mode="moving_boundary", solid="plate", solid_cells=6, e_lu=0.08,
                mpm_substeps=4, seed=3),
    ]


def _fields(drv):
    return {"F": drv.lbm.F.to_numpy(), "rho": drv.lbm.rho.to_numpy(), "v": drv.lbm.v.to_numpy(),
            "solid": drv.lbm.solid.to_numpy(), "x": drv.solid.x.to_numpy(), "Fp": drv.solid.F.to_numpy()}


def _compare(got, ref):
    np.testing.assert_array_equal(got["solid"], ref["solid"])
    np.testing.assert_allclose(got["F"], ref["F"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(got["rho"], ref["rho"], rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(got["v"], ref["v"], rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(got["x"], ref["x"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(got["Fp"], ref["Fp"], rtol=0, atol=1e-5)


@pytest.fixture(scope="module")
def alone():
    import torch

    out = []
    for case in _cases():
        drv = case.make_driver()
        for _ in range(STEPS):
            drv.step_once()
        torch.cuda.synchronize()
        out.append(_fields(drv))
    return out


@pytest.mark.parametrize("lbm_tune", [0, 2])
@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_cases_match_single_case_runs(alone, use_graph, lbm_tune):
    """lbm_tune 0: one cell per thread (the single runs' kernel); 2: two cells
    per thread on the paired FP32 pipe (agrees to FP32 rounding)."""
    from mpm_lbm_b200.batch import FSIBatch

    cases = _cases()
    batch = FSIBatch(capacity=4, mpm_substeps=4, lbm_tune=lbm_tune)
    slots = [batch.add(c.make_driver()) for c in cases]
    for _ in range(STEPS):
        batch.step(use_graph=use_graph)
    for slot, ref in zip(slots, alone):
        _compare(_fields(batch.sync_case(slot)), ref)
    if use_graph:
        # one launch per phase: project 3, mask 4, LBM 3, bin 4, MPM prologue + M + 1
        assert batch.graph_kernels == 3 + 4 + 3 + 4 + 4 + 2


def test_slot_reuse_and_empty_slots(alone):
    """A case added to a slot emptied by another case, next to an empty slot,
    evolves exactly as when alone."""
    from mpm_lbm_b200.batch import FSIBatch

    cases = _cases()
    batch = FSIBatch(capacity=3, mpm_substeps=4)
    s0 = batch.add(cases[1].make_driver())
    batch.step(use_graph=False)
    batch.remove(s0)
    s1 = batch.add(cases[0].make_driver(), slot=s0)
    for _ in range(STEPS):
        batch.step(use_graph=False)
    _compare(_fields(batch.sync_case(s1)), alone[0])

"""Continuous batching on the GPU: the real FSIServer over FSIBatch.

Seven FSI solve requests of mixed lattice sizes, coupling modes, solids and
step counts arrive over time into a server with three slots, so that
requests arrive while others are running, wait for a slot, are admitted into
a batch that is already stepping, and reuse the slots of retired requests.
Time is a deterministic counter (one tick per clock read), so the
interleaving is the same on every run.  Each finished request's final state
-- solid mask, populations, density, velocity, particle positions and
deformation gradients -- equals the same case run alone through FSIDriver3D,
within the tolerances of the batched-form test (tests/test_gpu_batch.py:
populations and density rtol 1e-5 / atol 1e-7, velocity rtol 1e-4 / atol
1e-7, positions atol 1e-6, deformation gradients atol 1e-5; masks
bit-exact).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MPM_SUBSTEPS = 4


def _requests():
    from mpm_lbm_b200.batch import BoxCase
    from mpm_lbm_b200.serve import Request

    spec = [  # (lattice, tau, mode, solid, cells, E, LBM steps, arrival tick)
        ((32, 32, 32), 0.6, "moving_boundary", "block", 6, 0.05, 9, 0),
        ((48, 32, 32), 0.7, "penalty", "plate", 8, 0.02, 5, 0),
        ((32, 48, 32), 0.55, "moving_boundary", "plate", 6, 0.08, 12, 3),
        ((32, 32, 32), 0.65, "penalty", "block", 4, 0.03, 4, 5),
        ((48, 48, 48), 0.58, "moving_boundary", "block", 8, 0.04, 6, 8),
        ((32, 32, 48), 0.75, "penalty", "plate", 6, 0.06, 7, 9),
        ((32, 32, 32), 0.52, "moving_boundary", "block", 5, 0.1, 5, 20),
    ]
    out = []
    for rid, (lat, tau, mode, solid, cells, e, steps, tick) in enumerate(spec):
        case = BoxCase(lattice=lat, tau=tau, mode=mode, solid=solid, solid_cells=cells, e_lu=e, lbm_steps=steps,
                       mpm_substeps=MPM_SUBSTEPS, seed=10 + rid)
        out.append(Request(rid=rid, case=case, arrival_s=float(tick)))
    return out


def _fields(drv):
    return {"F": drv.lbm.F.to_numpy(), "rho": drv.lbm.rho.to_numpy(), "v": drv.lbm.v.to_numpy(),
            "solid": drv.lbm.solid.to_numpy(), "x": drv.solid.x.to_numpy(), "Fp": drv.solid.F.to_numpy()}


class _Ticks:
    """A clock that advances one unit per read."""

    def __init__(self):
        self.t = -1.0

    def __call__(self):
        self.t += 1.0
        return self.t


@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_served_requests_equal_their_runs_alone(storage):
    import torch

    from mpm_lbm_b200.serve import FSIServer

    reqs = _requests()
    srv = FSIServer(slots=3, hbm_budget_bytes=4e9, storage=storage, mpm_substeps=MPM_SUBSTEPS, clock=_Ticks())
    srv.keep_drivers = True
    done = srv.run(reqs, time_limit_s=1e9)
    assert len(done) == len(reqs) and all(r.error is None for r in done), [r.error for r in done]
    # requests waited for a slot, and later requests took the slots of retired ones
    assert any(r.admit_s > r.arrival_s for r in done)
    assert max(r.admit_s for r in done) > min(r.finish_s for r in done)
    assert srv.report()["completed"] == len(reqs)
    for r in sorted(done, key=lambda q: q.rid):
        got = _fields(r.driver)  # FSIBatch.remove synchronised it at retirement
        alone = r.case.make_driver(storage=storage)
        for _ in range(r.lbm_steps):
            alone.step_once()
        torch.cuda.synchronize()
        ref = _fields(alone)
        np.testing.assert_array_equal(got["solid"], ref["solid"])
        np.testing.assert_allclose(got["F"], ref["F"], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(got["rho"], ref["rho"], rtol=1e-5, atol=1e-7)
        np.testing.assert_allclose(got["v"], ref["v"], rtol=1e-4, atol=1e-7)
        np.testing.assert_allclose(got["x"], ref["x"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(got["Fp"], ref["Fp"], rtol=0, atol=1e-5)
        assert r.result["tip_displacement"] is None or np.all(np.isfinite(r.result["tip_displacement"]))

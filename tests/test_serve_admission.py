"""Host logic of the serving loop (no GPU): request generation, admission
under a slot limit and a memory budget, and continuous batching with a
stand-in engine whose steps take no device time."""

import numpy as np

from mpm_lbm_b200.batch import BoxCase
from mpm_lbm_b200.serve import (GRID_SIZES, AdmissionQueue, FSIServer, Request, estimate_bytes,
                                poisson_requests)


def _req(rid, g=32, steps=10, t=0.0):
    return Request(rid=rid, case=BoxCase(lattice=(g, g, g), solid_cells=4, lbm_steps=steps), arrival_s=t)


def test_poisson_requests_follow_the_configuration():
    reqs = poisson_requests(2000, rate_per_s=20.0, seed=3)
    t = np.array([r.arrival_s for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 0.05) < 0.005
    g = np.array([r.case.lattice[0] for r in reqs])
    freq = np.array([np.mean(g == s) for s in GRID_SIZES])
    np.testing.assert_allclose(freq, [0.3, 0.3, 0.2, 0.15, 0.05], atol=0.03)
    steps = np.array([r.lbm_steps for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 2000
    assert all(r.case.lattice[0] == r.case.lattice[1] == r.case.lattice[2] for r in reqs)
    assert {r.case.mode for r in reqs} == {"penalty", "moving_boundary"}
    taus = np.array([r.case.tau for r in reqs])
    assert taus.min() >= 0.52 and taus.max() <= 0.8
    # same seed, same stream
    again = poisson_requests(2000, rate_per_s=20.0, seed=3)
    assert [r.case for r in again] == [r.case for r in reqs]


def test_memory_estimate_grows_with_the_case_and_storage():
    small, big = BoxCase(lattice=(32,) * 3), BoxCase(lattice=(128,) * 3)
    assert estimate_bytes(big) > 50 * estimate_bytes(small)
    assert estimate_bytes(big, "fp16") < estimate_bytes(big, "fp32")
    # a 128^3 case holds at least its populations and two MPM grid buffers
    assert estimate_bytes(big) > 19 * 4 * 128 ** 3 + 2 * 7 * 4 * 128 ** 3


def test_admission_respects_slots_budget_and_order():
    size = {0: 40, 1: 40, 2: 30, 3: 10}
    q = AdmissionQueue(slots=3, budget_bytes=100, estimate=lambda r: size[r.rid])
    for rid in range(4):
        assert q.arrive(_req(rid))
    got = [r.rid for r in q.admissible()]
    assert got == [0, 1]  # request 2 would exceed the budget; 3 may not overtake it
    q.release(_req(0))
    assert [r.rid for r in q.admissible()] == [2, 3]
    assert q.used_bytes == 80 and len(q.resident) == 3


def test_request_above_the_budget_is_rejected():
    q = AdmissionQueue(slots=4, budget_bytes=100, estimate=lambda r: 500)
    r = _req(0)
    assert not q.arrive(r)
    assert "budget" in r.error
    assert q.admissible() == []


class _FakeEngine:
    """Stands in for FSIBatch: slots, per-slot step counts, instant steps."""

    def __init__(self, capacity):
        self.slots = [None] * capacity
        self.steps_done = [0] * capacity
        self.max_occupancy = 0

    def add(self, drv):
        i = self.slots.index(None)
        self.slots[i] = drv
        self.steps_done[i] = 0
        self.max_occupancy = max(self.max_occupancy, sum(s is not None for s in self.slots))
        return i

    def remove(self, slot):
        drv, self.slots[slot] = self.slots[slot], None
        return drv

    def step(self, use_graph=False):
        for i, s in enumerate(self.slots):
            if s is not None:
                self.steps_done[i] += 1
                s["steps"] += 1


def test_continuous_batching_admits_as_slots_free_up():
    clock = {"t": 0.0}

    def tick():
        clock["t"] += 0.001  # every clock read advances 1 ms
        return clock["t"]

    eng = _FakeEngine(2)
    srv = FSIServer(slots=2, hbm_budget_bytes=1e12, engine=eng, clock=tick,
                    make_driver=lambda case: {"case": case, "steps": 0},
                    summarize=lambda d: {"steps": d["steps"], "rho_min": 1.0, "rho_max": 1.0})
    reqs = [_req(i, steps=5 + 3 * i, t=0.0) for i in range(5)]
    done = srv.run(reqs, time_limit_s=60)
    assert len(done) == 5 and all(r.error is None for r in done)
    assert eng.max_occupancy == 2
    for r in done:
        assert r.result["steps"] == r.lbm_steps
        assert r.admit_s is not None and r.finish_s >= r.admit_s
    # requests 2.. waited for a slot: admitted only after an earlier one finished
    first_finish = min(r.finish_s for r in done[:2])
    assert all(r.admit_s >= first_finish for r in reqs[2:])
    rep = srv.report()
    assert rep["completed"] == 5 and rep["p99_latency_s"] >= rep["p50_latency_s"] > 0

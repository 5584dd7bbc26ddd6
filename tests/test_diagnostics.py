"""The host part of the LBM diagnostics (record statistics, x sampling)
against the reference's own functions' results
(tests/golden/lbm_diagnostics_ref.json, made by
tests/golden/make_diagnostics_fixture.py).  The device reductions are tested
in tests/test_gpu_diagnostics.py."""

import json
import os

import pytest

from mpm_lbm_b200 import lbm_boundary_diagnostics as bd
from mpm_lbm_b200 import lbm_stability_diagnostics as sd
from tests.diag_compare import assert_same
from tests.golden.make_diagnostics_fixture import records

REF = os.path.join(os.path.dirname(__file__), "golden", "lbm_diagnostics_ref.json")


@pytest.fixture(scope="module")
def ref():
    with open(REF) as fh:
        return json.load(fh)["records"]


def test_record_statistics_match_reference(ref):
    rows = records()
    assert_same(bd.summarize_timeseries_trends(rows), ref["summarize_timeseries_trends"])
    assert_same(bd.summarize_timeseries_trends(rows, tail_fraction=0.5), ref["summarize_timeseries_trends_half"])
    assert_same(sd.mass_source_sink_by_step(rows), ref["mass_source_sink_by_step"])
    assert_same(sd.mass_source_sink_by_step([]), ref["mass_source_sink_by_step_empty"])
    assert_same(sd.first_gate_failure_detector(rows), ref["first_gate_failure_detector"])
    assert_same(sd.first_gate_failure_detector(rows, rho_high=1.1, max_v=0.1),
                ref["first_gate_failure_detector_tight"])


def test_sampled_indices_match_reference(ref):
    for n, want in ref["sampled_x_profile_indices"].items():
        assert bd.sampled_x_profile_indices(int(n)) == want


def test_record_errors_match_reference():
    with pytest.raises(ValueError, match="records must not be empty"):
        bd.summarize_timeseries_trends([])
    with pytest.raises(ValueError, match="tail_fraction"):
        bd.summarize_timeseries_trends(records(), tail_fraction=0.0)
    with pytest.raises(ValueError, match="side must be"):
        sd.boundary_population_stats({}, "y_min")

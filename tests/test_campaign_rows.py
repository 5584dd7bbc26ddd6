"""The campaign rows of mpm_lbm_b200.campaign against the reference's own
_stability_row and _mass_flux_row (solvers/official_subcycled_flow_solver.py:
443-515), whose outputs on seeded host snapshots are committed
(tests/golden/make_campaign_fixture.py).  Here the sums the rows are built
from are taken on the host with the reference's numpy expressions, so the
rows must be identical, gates and all; tests/test_gpu_campaign.py takes the
same sums on the device."""

import json
import os

import numpy as np

from mpm_lbm_b200 import campaign

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture():
    d = np.load(os.path.join(GOLDEN, "campaign_fields.npz"))
    snaps = [{k: d[f"s{i}_{k}"] for k in ("rho", "velocity", "population", "solid")} for i in range(3)]
    masks = {"boundary": {"velocity_inlet_mask": d["inlet"], "pressure_outlet_mask": d["outlet"]},
             "geometry": {"fluid_mask": d["fluid_mask"]}}
    with open(os.path.join(GOLDEN, "campaign_rows_ref.json")) as fh:
        ref = json.load(fh)
    return snaps, masks, ref


def host_sums(snap, regions):
    fluid = snap["solid"] == 0
    rho = snap["rho"].astype(np.float64)
    ux = snap["velocity"][..., 0].astype(np.float64)
    return {"fluid_mass": float(np.sum(rho[fluid])),
            "flux": {k: float(np.sum(rho[m] * ux[m])) for k, m in regions.items()},
            "fluid_cells": int(fluid.sum()),
            "rho_finite": bool(np.all(np.isfinite(snap["rho"][fluid]))),
            "velocity_finite": bool(np.all(np.isfinite(snap["velocity"][fluid]))),
            "population_finite": bool(np.all(np.isfinite(snap["population"][fluid])))}


def compare_rows(got, want, rtol, atol=0.0):
    assert set(got) == set(want)
    for k, w in want.items():
        g = got[k]
        if isinstance(w, (bool, str, int)):
            assert g == w, k
        else:
            np.testing.assert_allclose(g, w, rtol=rtol, atol=atol, err_msg=k)


def test_rows_equal_the_reference_rows():
    snaps, masks, ref = load_fixture()
    regions = campaign.campaign_regions(masks)
    initial = None
    for k, snap in enumerate(snaps):
        sums = host_sums(snap, regions)
        compare_rows(campaign.stability_row(ref["base"][k], ref["diagnostics"][k], sums), ref["rows"]["stability"][k],
                     rtol=0)
        if k < len(ref["rows"]["mass_flux"]):
            row, initial = campaign.mass_flux_row(ref["base"][k], sums, initial)
            compare_rows(row, ref["rows"]["mass_flux"][k], rtol=0)
    # the gates the fixture exercises: all pass at first, all fail at the end
    st = ref["rows"]["stability"]
    assert st[0]["finite_gate_pass_step"] and st[0]["density_gate_pass_step"] and st[0]["mpm_j_gate_pass_step"]
    assert not (st[2]["finite_gate_pass_step"] or st[2]["density_gate_pass_step"] or st[2]["mpm_j_gate_pass_step"])

"""Device reductions of the subcycled-flow campaign (fsi_campaign_sums,
fsi_campaign_sums_arrays, mpm_lbm_b200.campaign).

1. Against the reference's own rows: the reference's _stability_row and
   _mass_flux_row (solvers/official_subcycled_flow_solver.py:443-515) ran on
   seeded host snapshots (tests/golden/make_campaign_fixture.py); the same
   snapshots go to the device, fsi_campaign_sums_arrays sums them and
   campaign builds the rows.  FP64 sums of FP32 fields in another order: rtol
   1e-12 (mass_delta_rel, a difference of two near-equal sums: atol 1e-12);
   gates, flags and counts exact.
2. On the drop-in's own state: fsi_campaign_sums over the lattice state of a
   duct/plate case with open x faces after FSI steps (the open boundary of
   the last substep pending, so the readout applies it) against the same
   sums of the host copies _copy_lbm_fields makes (352-365).  A non-finite
   population written into one fluid cell clears population_finite and the
   finite gate.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_rows(fields, masks, diagnostics):
    """solver.py:465-540 on host arrays (the expected values)."""
    rho = fields["rho"].astype(np.float64)
    ux = fields["velocity"][..., 0].astype(np.float64)
    fluid = fields["solid"] == 0
    boundary, geometry = masks["boundary"], masks["geometry"]
    inlet = boundary["velocity_inlet_mask"].astype(bool)
    outlet = boundary["pressure_outlet_mask"].astype(bool)
    static_fluid = geometry["fluid_mask"].astype(bool)
    mid = np.zeros_like(static_fluid)
    mid[static_fluid.shape[0] // 2] = static_fluid[static_fluid.shape[0] // 2]
    finite = {"rho": bool(np.all(np.isfinite(fields["rho"][fluid]))),
              "velocity": bool(np.all(np.isfinite(fields["velocity"][fluid]))),
              "population": bool(np.all(np.isfinite(fields["population"][fluid])))}
    return {"mass": float(np.sum(rho[fluid])), "inlet": float(np.sum(rho[inlet] * ux[inlet])),
            "outlet": float(np.sum(rho[outlet] * ux[outlet])), "midplane": float(np.sum(rho[mid] * ux[mid])),
            "cells": int(fluid.sum()), **finite}


def test_device_rows_equal_the_reference_rows():
    from mpm_lbm_b200 import campaign
    from tests.test_campaign_rows import compare_rows, load_fixture

    snaps, masks, ref = load_fixture()
    regions = campaign.campaign_regions(masks)
    initial = None
    for k, snap in enumerate(snaps):
        sums = campaign.campaign_sums_from_fields(snap, regions)
        assert sums["fluid_cells"] == int((snap["solid"] == 0).sum())
        compare_rows(campaign.stability_row(ref["base"][k], ref["diagnostics"][k], sums), ref["rows"]["stability"][k],
                     rtol=1e-12)
        if k < len(ref["rows"]["mass_flux"]):
            row, initial = campaign.mass_flux_row(ref["base"][k], sums, initial)
            compare_rows(row, ref["rows"]["mass_flux"][k], rtol=1e-12, atol=1e-12)


def _masks(drv):
    nx, ny, nz = drv.lbm.dims
    static = drv.lbm.static_solid.to_numpy() == 0
    inlet = np.zeros((nx, ny, nz), bool)
    outlet = np.zeros((nx, ny, nz), bool)
    inlet[0] = static[0]
    outlet[-1] = static[-1]
    return {"boundary": {"velocity_inlet_mask": inlet, "pressure_outlet_mask": outlet},
            "geometry": {"fluid_mask": static}}


def test_campaign_sums_match_host_rows():
    import torch

    from mpm_lbm_b200 import campaign
    from mpm_lbm_b200.cases import DuctPlateCase

    drv = DuctPlateCase(lattice=(64, 32, 32), plate=(2, 16, 24), lbm_substeps=12, mpm_substeps=4).make_driver()
    masks = _masks(drv)
    red = campaign.CampaignReductions(drv.lbm, campaign.campaign_regions(masks))
    initial = None
    for step in range(3):
        if step:
            drv.step_once()
        torch.cuda.synchronize()
        assert drv.lbm.bc_pending == (step > 0)
        diag = drv.collect_diagnostics(step)
        sums = red()
        fields = campaign.copy_lbm_fields(drv)
        want = _host_rows(fields, masks, diag)
        assert sums["fluid_cells"] == want["cells"]
        for key in ("rho", "velocity", "population"):
            assert sums[f"{key}_finite"] == want[key]
        np.testing.assert_allclose(sums["fluid_mass"], want["mass"], rtol=1e-12)
        for name in ("inlet", "outlet", "midplane"):
            np.testing.assert_allclose(sums["flux"][name], want[name], rtol=1e-12, atol=1e-12)
        base = {"official_step": step, "time_s": 0.1 * step, "lbm_substeps_per_fsi_step": 12,
                "total_lbm_substeps": drv.total_lbm_substeps, "fsi_exchange_mode": drv.config.fsi_exchange_mode}
        row, initial = campaign.mass_flux_row(base, sums, initial)
        assert row["total_fluid_mass"] == sums["fluid_mass"]
        assert row["flux_imbalance_rel"] == (sums["flux"]["outlet"] - sums["flux"]["inlet"]) / max(
            abs(sums["flux"]["inlet"]), 1e-30)
        srow = campaign.stability_row(base, diag, sums)
        assert srow["finite_gate_pass_step"] and srow["density_gate_pass_step"] and srow["mpm_j_gate_pass_step"]
    assert sums["flux"]["inlet"] > 0.0  # the inlet drives the flow


def test_nonfinite_population_clears_the_finite_gate():
    import torch

    from mpm_lbm_b200 import campaign
    from mpm_lbm_b200.cases import DuctPlateCase

    drv = DuctPlateCase(lattice=(64, 32, 32), plate=(2, 16, 24), lbm_substeps=12, mpm_substeps=4).make_driver()
    drv.step_once()
    F = drv.lbm.F.to_numpy()
    fluid = np.argwhere(drv.lbm.solid.to_numpy() == 0)[100]
    F[tuple(fluid)][5] = np.inf
    drv.lbm.F.from_numpy(F)
    torch.cuda.synchronize()
    sums = campaign.CampaignReductions(drv.lbm, campaign.campaign_regions(_masks(drv)))()
    assert not sums["population_finite"] and sums["rho_finite"]
    row = campaign.stability_row({"official_step": 1}, {"rho_min": 0.9, "rho_max": 1.1, "lbm_max_v": 0.05,
                                                        "mpm_min_J": 1.0, "mpm_max_speed": 0.0}, sums)
    assert not row["finite_gate_pass_step"]

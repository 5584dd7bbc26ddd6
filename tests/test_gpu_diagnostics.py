"""The LBM boundary and stability diagnostics reduced on the device against
the reference's own numpy implementation run on the same snapshots
(tests/golden/lbm_diagnostics_ref.json, made by
tests/golden/make_diagnostics_fixture.py), both from a snapshot dict and
from an LBMFluid3D holding the snapshot.  Tolerances: counts, locations,
flags and FP32 extrema exact; FP64 sums and derived means / deviations
rtol 1e-9 (summation order, one-pass deviations)."""

import json
import os

import pytest

from tests.diag_compare import assert_same
from tests.golden.make_diagnostics_fixture import snapshots

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(__file__), "golden", "lbm_diagnostics_ref.json")


def results(obj, nx):
    from mpm_lbm_b200 import lbm_boundary_diagnostics as bd
    from mpm_lbm_b200 import lbm_stability_diagnostics as sd

    return {
        "summary_boundary": bd.summarize_lbm_boundary_diagnostics(obj, step=7),
        "summary_boundary_mass": bd.summarize_lbm_boundary_diagnostics(obj, step=8, mass_initial=1234.5),
        "plane_flux_x": {str(x): bd.plane_flux_x(obj, x) for x in (-1, 0, 1, nx // 2, nx - 1, nx + 3)},
        "plane_mean_velocity_x": {str(x): bd.plane_mean_velocity_x(obj, x) for x in (0, 4, nx - 2)},
        "plane_mean_density_x": {str(x): bd.plane_mean_density_x(obj, x) for x in (0, 4, nx - 2)},
        "centerline_profile_x": bd.centerline_profile_x(obj, y_index=1, z_index=3),
        "plane_velocity_x_stats": bd.plane_velocity_x_stats(obj, 2),
        "plane_density_stats": bd.plane_density_stats(obj, nx - 1),
        "outlet_reflection_proxy": bd.outlet_reflection_proxy(obj),
        "density_stats": bd.density_stats(obj),
        "mass_total": bd.mass_total(obj),
        "summary_stability": sd.summarize_lbm_stability_diagnostics(obj, step=7),
        "density_outlier_stats": sd.density_outlier_stats(obj, low=0.99, high=1.01),
        "velocity_outlier_stats": sd.velocity_outlier_stats(obj, max_v_threshold=0.07),
        "boundary_population_stats_x_min": sd.boundary_population_stats(obj, "x_min"),
        "boundary_population_stats_x_max": sd.boundary_population_stats(obj, "x_max"),
        "population_stats": sd.population_stats(obj),
        "negative_population_stats": sd.negative_population_stats(obj),
        "classify_first_failure_location": sd.classify_first_failure_location(obj),
    }


@pytest.fixture(scope="module")
def ref():
    with open(REF) as fh:
        return json.load(fh)["snapshots"]


@pytest.mark.parametrize("name", ["ducta", "smallb"])
def test_diagnostics_from_snapshot(ref, name):
    snap = snapshots()[name]
    assert_same(results(snap, snap["rho"].shape[0]), ref[name])


@pytest.mark.parametrize("name", ["ducta", "smallb"])
def test_diagnostics_from_lattice(ref, name):
    from mpm_lbm_b200._lib import launch_count
    from mpm_lbm_b200.config import LBMConfig
    from mpm_lbm_b200.lbm import LBMFluid3D

    snap = snapshots()[name]
    nx, ny, nz = snap["rho"].shape
    lbm = LBMFluid3D(LBMConfig(nx=nx, ny=ny, nz=nz))
    lbm.init_geo_array(snap["solid"])
    lbm.init_simulation()
    lbm.F.from_numpy(snap["F"])
    lbm.rho.from_numpy(snap["rho"])
    lbm.v.from_numpy(snap["v"])
    before = launch_count()
    got = results(lbm, nx)
    assert launch_count() > before
    assert_same(got, ref[name])

"""Generate the LBM diagnostics fixture with the reference's own diagnostics.

TEST INFRASTRUCTURE.  Run in a container that holds the reference checkout
(read-only) at REF_ROOT.  The reference's diagnostics modules
(src/mpm_lbm/sim/diagnostics/lbm_boundary_diagnostics.py and
lbm_stability_diagnostics.py) need only numpy, so they are loaded from their
files directly.  They run on seeded snapshots that ``snapshots()`` rebuilds
(the tests call it too) and on seeded diagnostic records; their results go to
tests/golden/lbm_diagnostics_ref.json, which pins
mpm_lbm_b200.lbm_boundary_diagnostics and mpm_lbm_b200.lbm_stability_diagnostics
(tests/test_diagnostics.py on the CPU, tests/test_gpu_diagnostics.py on the
device).  Usage::

    python tests/golden/make_diagnostics_fixture.py --ref PATH
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "lbm_diagnostics_ref.json")


def _snapshot(rng, nx, ny, nz):
    solid = np.zeros((nx, ny, nz), np.int8)
    solid[:, 0, :] = 1
    solid[:, :, 0] = 1
    solid[nx // 3: nx // 3 + 2, ny // 2 - 1: ny // 2 + 1, nz // 2 - 1: nz // 2 + 1] = 1
    rho = (1.0 + 0.01 * rng.standard_normal((nx, ny, nz))).astype(np.float32)
    v = (0.02 * rng.standard_normal((nx, ny, nz, 3))).astype(np.float32)
    v[..., 0] += np.float32(0.05)
    F = rng.uniform(-0.01, 0.2, (nx, ny, nz, 19)).astype(np.float32)
    # the device state keeps rho0 and zero velocity in solid cells
    rho[solid > 0] = 1.0
    v[solid > 0] = 0.0
    return {"rho": rho, "v": v, "solid": solid, "f": F.copy(), "F": F}


def snapshots():
    """name -> snapshot dict (rho, v, solid, f, F) in the reference's layouts."""
    rng = np.random.default_rng(11)
    a = _snapshot(rng, 50, 6, 5)
    a["rho"][7, 2, 3] = -0.1   # negative density
    a["rho"][30, 4, 1] = 1.5   # high density
    a["rho"][12, 2, 2] = 1.3
    a["v"][20, 3, 3] = (0.3, 0.1, 0.0)   # velocity outliers
    a["v"][9, 1, 4] = (-0.2, 0.0, 0.05)
    b = _snapshot(rng, 9, 5, 4)
    b["solid"][4] = 1          # a plane without fluid
    b["rho"][4] = 1.0
    b["v"][4] = 0.0
    b["rho"][2, 3, 2] = np.nan
    b["v"][6, 2, 1, 1] = np.inf
    b["F"][1, 1, 1, 5] = np.nan
    b["f"][1, 1, 1, 5] = np.nan
    b["rho"][8, 3, 3] = 2.0
    return {"ducta": a, "smallb": b}


def records(seed=5, n=12):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        rows.append({
            "step": 10 * i, "rho_min": float(0.95 - 0.02 * i + 0.01 * rng.standard_normal()),
            "rho_max": float(1.05 + 0.02 * i), "mass_total_delta_rel": float(0.01 * i * rng.standard_normal()),
            "max_v": float(0.05 + 0.02 * i), "mach_proxy_observed": float(0.1 + 0.03 * i),
            "inlet_flux": float(1.0 + 0.1 * rng.standard_normal()), "outlet_flux": float(0.9 + 0.1 * rng.standard_normal()),
            "flux_imbalance_rel": float(0.1 * rng.standard_normal()), "inlet_mean_ux": float(0.05 + 0.001 * i),
            "midplane_mean_ux": float(0.048 + 0.001 * i),
            "outlet_reflection_proxy": {"negative_ux_fraction": float(0.01 * i), "rho_std": float(0.001 * i),
                                        "ux_std": float(0.002 * i)},
        })
    rows[3]["rho_min"] = float("nan")
    return rows


def _load(ref, name):
    path = os.path.join(ref, "src", "mpm_lbm", "sim", "diagnostics", name + ".py")
    spec = importlib.util.spec_from_file_location("reference_" + name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _jsonable(value):
    if isinstance(value, dict):
        return {str(k): _jsonable(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_jsonable(v) for v in value]
    if isinstance(value, (np.integer,)):
        return int(value)
    if isinstance(value, (np.floating,)):
        return float(value)
    if isinstance(value, np.bool_):
        return bool(value)
    return value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF_ROOT"), help="reference checkout (or set REF_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or REF_ROOT")
    bd = _load(args.ref, "lbm_boundary_diagnostics")
    sd = _load(args.ref, "lbm_stability_diagnostics")
    out = {"snapshots": {}, "records": {}}
    for name, snap in snapshots().items():
        nx = snap["rho"].shape[0]
        res = {
            "summary_boundary": bd.summarize_lbm_boundary_diagnostics(snap, step=7),
            "summary_boundary_mass": bd.summarize_lbm_boundary_diagnostics(snap, step=8, mass_initial=1234.5),
            "plane_flux_x": {str(x): bd.plane_flux_x(snap, x) for x in (-1, 0, 1, nx // 2, nx - 1, nx + 3)},
            "plane_mean_velocity_x": {str(x): bd.plane_mean_velocity_x(snap, x) for x in (0, 4, nx - 2)},
            "plane_mean_density_x": {str(x): bd.plane_mean_density_x(snap, x) for x in (0, 4, nx - 2)},
            "centerline_profile_x": bd.centerline_profile_x(snap, y_index=1, z_index=3),
            "plane_velocity_x_stats": bd.plane_velocity_x_stats(snap, 2),
            "plane_density_stats": bd.plane_density_stats(snap, nx - 1),
            "outlet_reflection_proxy": bd.outlet_reflection_proxy(snap),
            "density_stats": bd.density_stats(snap),
            "mass_total": bd.mass_total(snap),
            "summary_stability": sd.summarize_lbm_stability_diagnostics(snap, step=7),
            "density_outlier_stats": sd.density_outlier_stats(snap, low=0.99, high=1.01),
            "velocity_outlier_stats": sd.velocity_outlier_stats(snap, max_v_threshold=0.07),
            "boundary_population_stats_x_min": sd.boundary_population_stats(snap, "x_min"),
            "boundary_population_stats_x_max": sd.boundary_population_stats(snap, "x_max"),
            "population_stats": sd.population_stats(snap),
            "negative_population_stats": sd.negative_population_stats(snap),
            "classify_first_failure_location": sd.classify_first_failure_location(snap),
        }
        out["snapshots"][name] = _jsonable(res)
    rows = records()
    out["records"] = _jsonable({
        "summarize_timeseries_trends": bd.summarize_timeseries_trends(rows),
        "summarize_timeseries_trends_half": bd.summarize_timeseries_trends(rows, tail_fraction=0.5),
        "mass_source_sink_by_step": sd.mass_source_sink_by_step(rows),
        "mass_source_sink_by_step_empty": sd.mass_source_sink_by_step([]),
        "first_gate_failure_detector": sd.first_gate_failure_detector(rows),
        "first_gate_failure_detector_tight": sd.first_gate_failure_detector(rows, rho_high=1.1, max_v=0.1),
        "sampled_x_profile_indices": {str(n): bd.sampled_x_profile_indices(n) for n in (1, 2, 5, 9, 47, 48, 50, 128)},
    })
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()

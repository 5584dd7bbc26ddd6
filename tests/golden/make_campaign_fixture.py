"""Generate the campaign-row fixture with the reference's own row functions.

TEST INFRASTRUCTURE.  Run in a container that holds the reference checkout
(read-only); its path comes from --ref or the REF_ROOT environment variable.
taichi need not be installed (``taichi_shim`` stands in for it) and the
plotting package the solver file imports is stubbed (the row functions do
not plot).  The reference's _stability_row and _mass_flux_row
(src/mpm_lbm/solvers/official_subcycled_flow_solver.py:443-515) run on
seeded host snapshots in the layouts of _copy_lbm_fields (352-365) -- rho,
velocity, population and solid of a walled duct with a plate -- and on
seeded diagnostics; the snapshots go to campaign_fields.npz and the rows to
campaign_rows_ref.json.  tests/test_campaign_rows.py (CPU) and
tests/test_gpu_campaign.py (device sums) compare mpm_lbm_b200.campaign with
them.  Usage::

    python tests/golden/make_campaign_fixture.py --ref PATH
"""

from __future__ import annotations

import argparse
import importlib.abc
import importlib.machinery
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = os.path.join(HERE, "campaign_fields.npz")
ROWS = os.path.join(HERE, "campaign_rows_ref.json")
NX, NY, NZ = 16, 10, 8
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)


def _snapshot(rng):
    solid = np.zeros((NX, NY, NZ), np.int8)
    solid[:, 0, :] = solid[:, -1, :] = 1
    solid[:, :, 0] = solid[:, :, -1] = 1
    solid[NX // 3: NX // 3 + 2, 1:6, 2:6] = 1  # the plate
    rho = (1.0 + 0.01 * rng.standard_normal((NX, NY, NZ))).astype(np.float32)
    v = (0.01 * rng.standard_normal((NX, NY, NZ, 3))).astype(np.float32)
    v[..., 0] += np.float32(0.04)
    pop = (W * (1.0 + 0.05 * rng.standard_normal((NX, NY, NZ, 19)))).astype(np.float32)
    rho[solid > 0] = 1.0
    v[solid > 0] = 0.0
    return {"rho": rho, "velocity": v, "population": pop, "solid": solid}


def snapshots():
    """Three host snapshots of successive official steps; the last holds a
    non-finite population and a non-finite velocity in fluid cells."""
    rng = np.random.default_rng(157)
    out = [_snapshot(rng) for _ in range(3)]
    fluid = np.argwhere(out[2]["solid"] == 0)
    i, j, k = fluid[40]
    out[2]["population"][i, j, k, 7] = np.nan
    i, j, k = fluid[90]
    out[2]["velocity"][i, j, k, 1] = np.inf
    return out


def masks(solid_static):
    static_fluid = solid_static == 0
    inlet = np.zeros_like(static_fluid)
    outlet = np.zeros_like(static_fluid)
    inlet[0] = static_fluid[0]
    outlet[-1] = static_fluid[-1]
    return {"boundary": {"velocity_inlet_mask": inlet, "pressure_outlet_mask": outlet},
            "geometry": {"fluid_mask": static_fluid}}


def diagnostics(k):
    return [{"rho_min": 0.97, "rho_max": 1.04, "lbm_max_v": 0.081, "mpm_min_J": 0.995, "mpm_max_speed": 0.012},
            {"rho_min": 0.96, "rho_max": 1.05, "lbm_max_v": 0.083, "mpm_min_J": 0.99, "mpm_max_speed": 0.015},
            {"rho_min": 0.95, "rho_max": 5.2, "lbm_max_v": 0.09, "mpm_min_J": -0.1, "mpm_max_speed": 0.02}][k]


def base(k):
    return {"official_step": k + 1, "time_s": 0.125 * (k + 1), "lbm_substeps_per_fsi_step": 120,
            "total_lbm_substeps": 120 * (k + 1), "fsi_exchange_mode": "lbm_subcycled_per_fsi_step"}


class _Stub(types.ModuleType):
    """Stands in for the plotting package the solver file imports."""

    __path__: list = []

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return type(name, (), {"__init__": lambda self, *a, **k: None, "__call__": lambda self, *a, **k: None})


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name == "matplotlib" or name.startswith("matplotlib."):
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        return _Stub(spec.name)

    def exec_module(self, module):
        pass


def _jsonable(v):
    if isinstance(v, dict):
        return {k: _jsonable(x) for k, x in v.items()}
    if isinstance(v, (np.bool_, bool)):
        return bool(v)
    if isinstance(v, (np.integer,)):
        return int(v)
    if isinstance(v, (np.floating, float)):
        return float(v)
    return v


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("REF_ROOT"), help="reference checkout (or set REF_ROOT)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or REF_ROOT")
    sys.path.insert(0, HERE)
    import taichi_shim  # noqa: E402

    sys.modules["taichi"] = taichi_shim
    sys.meta_path.insert(0, _StubFinder())
    sys.path.insert(0, args.ref)
    from src.mpm_lbm.solvers import official_subcycled_flow_solver as solver

    snaps = snapshots()
    m = masks(snaps[0]["solid"])
    rows = {"stability": [], "mass_flux": []}
    initial = None
    for k, snap in enumerate(snaps):
        rows["stability"].append(solver._stability_row(base(k), diagnostics(k), snap))
        if k < 2:  # _mass_flux_row raises on the last snapshot's non-finite velocity
            row, initial = solver._mass_flux_row(base(k), snap, m, initial)
            rows["mass_flux"].append(row)
    payload = {}
    for k, snap in enumerate(snaps):
        for name, arr in snap.items():
            payload[f"s{k}_{name}"] = arr
    payload["inlet"] = m["boundary"]["velocity_inlet_mask"]
    payload["outlet"] = m["boundary"]["pressure_outlet_mask"]
    payload["fluid_mask"] = m["geometry"]["fluid_mask"]
    np.savez_compressed(FIELDS, **payload)
    out = {"rows": _jsonable(rows), "diagnostics": [diagnostics(k) for k in range(3)],
           "base": [base(k) for k in range(3)]}
    with open(ROWS, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", FIELDS, os.path.getsize(FIELDS), "bytes and", ROWS)


if __name__ == "__main__":
    main()

"""The reference's LBM stability diagnostics
(src/mpm_lbm/sim/diagnostics/lbm_stability_diagnostics.py), same names,
arguments and result keys, reduced on the device.

Each function takes an LBMFluid3D or a snapshot dict (rho, v, solid and
optionally f, F in the reference's layouts).  On an LBMFluid3D the
populations f and F are the readout populations (one array: the reference's
``f`` equals ``F`` on fluid cells after each macroscopic update).  Minima
and maxima are exact (FP32 values); first-outlier locations follow numpy's
argwhere order (x, then y, then z); counts are exact.
"""

from __future__ import annotations

import math
from typing import Any, Dict, Iterable, List, Optional

import numpy as np

from ._field_stats import KEY_NONE_MIN, PlaneTable, decode_keys, field_stats


def snapshot_from_lbm(lbm: Any) -> Dict[str, np.ndarray]:
    """lbm_stability_diagnostics.py:9-16: a host copy (the caller asks for one)."""
    return {
        "rho": np.asarray(lbm.rho.to_numpy(), dtype=float),
        "v": np.asarray(lbm.v.to_numpy(), dtype=float),
        "solid": np.asarray(lbm.solid.to_numpy(), dtype=np.int8),
        "f": np.asarray(lbm.f.to_numpy(), dtype=float),
        "F": np.asarray(lbm.F.to_numpy(), dtype=float),
    }


def _table(data: Any, **kw) -> PlaneTable:
    if isinstance(data, PlaneTable):
        return data
    return field_stats(data, **kw)


def _key_col(t: PlaneTable, name: str, w: int, sel, smallest: bool) -> float:
    k = np.asarray(t[name][sel, w]).reshape(-1)
    k = k[k != (np.uint32(KEY_NONE_MIN) if smallest else 0)]
    if not k.size:
        return float("nan")
    return float(decode_keys(k.min() if smallest else k.max()))


def _pop_stats(t: PlaneTable, w: int, sel=slice(None)):
    """nanmin, nanmax, negative and non-finite counts of population array w
    (0: f, 1: F) over the selected planes."""
    return (_key_col(t, "pop_min", w, sel, True), _key_col(t, "pop_max", w, sel, False),
            int(np.sum(t["pop_negative"][sel, w], dtype=np.int64)),
            int(np.sum(t["pop_nonfinite"][sel, w], dtype=np.int64)))


def population_stats(lbm_or_snapshot: Any) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:19-31 (nanmin / nanmax over all cells)."""
    t = _table(lbm_or_snapshot)
    f_min, f_max, _, f_bad = _pop_stats(t, 0)
    F_min, F_max, _, F_bad = _pop_stats(t, 1)
    return {
        "f_min": _finite_float(f_min),
        "f_max": _finite_float(f_max),
        "F_min": _finite_float(F_min),
        "F_max": _finite_float(F_max),
        "f_all_finite": f_bad == 0,
        "F_all_finite": F_bad == 0,
        "all_finite": f_bad == 0 and F_bad == 0,
    }


def negative_population_stats(lbm_or_snapshot: Any) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:34-48."""
    t = _table(lbm_or_snapshot)
    f_neg = int(np.sum(t["pop_negative"][:, 0], dtype=np.int64))
    F_neg = int(np.sum(t["pop_negative"][:, 1], dtype=np.int64))
    nx, ny, nz = t.shape
    total = 2 * nx * ny * nz * 19
    count = f_neg + F_neg
    return {
        "negative_population_count": count,
        "negative_population_fraction": _finite_float(count / total if total else 0.0),
        "f_negative_population_count": f_neg,
        "F_negative_population_count": F_neg,
        "population_entry_count": total,
    }


def boundary_population_stats(lbm_or_snapshot: Any, side: str) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:51-72."""
    if side not in ("x_min", "x_max"):
        raise ValueError("side must be 'x_min' or 'x_max'")
    t = _table(lbm_or_snapshot)
    nx, ny, nz = t.shape
    x = 0 if side == "x_min" else nx - 1
    sel = slice(x, x + 1)
    f_min, f_max, f_neg, f_bad = _pop_stats(t, 0, sel)
    F_min, F_max, F_neg, F_bad = _pop_stats(t, 1, sel)
    total = 2 * ny * nz * 19
    neg = f_neg + F_neg
    return {
        "side": side,
        "x_index": int(x),
        "f_min": _finite_float(f_min),
        "f_max": _finite_float(f_max),
        "F_min": _finite_float(F_min),
        "F_max": _finite_float(F_max),
        "negative_population_count": neg,
        "negative_population_fraction": _finite_float(neg / total if total else 0.0),
        "all_finite": f_bad == 0 and F_bad == 0,
    }


def _first(t: PlaneTable, count_key: str, first_key: str) -> Optional[List[int]]:
    nz = t.shape[2]
    hits = np.nonzero(t[count_key] > 0)[0]
    if hits.size == 0:
        return None
    x = int(hits[0])
    jk = int(t[first_key][x])
    return [x, jk // nz, jk % nz]


def _fluid(t: PlaneTable) -> int:
    return int(np.sum(t["fluid_cells"], dtype=np.int64))


def density_outlier_stats(lbm_or_snapshot: Any, low: float = 0.0, high: float = 1.2) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:75-92."""
    t = _table(lbm_or_snapshot, rho_low=low, rho_high=high)
    return _density(t, low, high)


def _density(t: PlaneTable, low: float, high: float) -> Dict[str, Any]:
    n = _fluid(t)
    return {
        "rho_min": _finite_float(t.key_min("rho_min")) if n else 0.0,
        "rho_max": _finite_float(t.key_max("rho_max")) if n else 0.0,
        "rho_low_threshold": float(low),
        "rho_high_threshold": float(high),
        "rho_below_low_count": int(np.sum(t["rho_low"], dtype=np.int64)),
        "rho_above_high_count": int(np.sum(t["rho_high"], dtype=np.int64)),
        "first_negative_density_location": _first(t, "rho_low", "rho_low_first"),
        "first_high_density_location": _first(t, "rho_high", "rho_high_first"),
        "all_finite": (int(np.sum(t["rho_nonfinite"])) == 0) if n else True,
    }


def velocity_outlier_stats(lbm_or_snapshot: Any, max_v_threshold: float = 0.2) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:95-118."""
    t = _table(lbm_or_snapshot, vel_high=max_v_threshold)
    return _velocity(t, max_v_threshold)


def _velocity(t: PlaneTable, max_v_threshold: float) -> Dict[str, Any]:
    n = _fluid(t)
    if n == 0:
        return {"max_v": 0.0, "max_v_threshold": float(max_v_threshold), "velocity_outlier_count": 0,
                "velocity_outlier_fraction": 0.0, "first_velocity_outlier_location": None, "all_finite": True}
    count = int(np.sum(t["vel_high"], dtype=np.int64))
    all_nan = int(np.sum(t["vel_nan"], dtype=np.int64)) == n
    return {
        "max_v": _finite_float(float("nan") if all_nan else t.speed_max()),
        "max_v_threshold": float(max_v_threshold),
        "velocity_outlier_count": count,
        "velocity_outlier_fraction": _finite_float(count / n),
        "first_velocity_outlier_location": _first(t, "vel_high", "vel_high_first"),
        "all_finite": int(np.sum(t["vel_nonfinite"])) == 0,
    }


def mass_source_sink_by_step(records: Iterable[Dict[str, Any]]) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:121-138 (host arithmetic on the records)."""
    rows = list(records)
    if not rows:
        return {"record_count": 0, "mass_drift_initial": None, "mass_drift_final": None,
                "mass_drift_delta_final": None, "mass_drift_abs_max": None}
    values = [_record_float(row, "mass_total_delta_rel") for row in rows]
    return {
        "record_count": int(len(rows)),
        "mass_drift_initial": values[0],
        "mass_drift_final": values[-1],
        "mass_drift_delta_final": _finite_float(values[-1] - values[0]),
        "mass_drift_abs_max": _finite_float(max(abs(value) for value in values)),
    }


def first_gate_failure_detector(records: Iterable[Dict[str, Any]], rho_low: float = 0.0, rho_high: float = 1.2,
                                mass_drift_abs: float = 0.05, max_v: float = 0.2) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:141-190 (host arithmetic on the records)."""
    rows = list(records)
    result = {"record_count": int(len(rows)), "all_records_finite": True, "first_nonfinite_step": None,
              "first_negative_density_step": None, "first_high_density_step": None, "first_mass_drift_step": None,
              "first_max_v_step": None, "first_failure_step": None, "first_failure_reason": None}
    failures = []
    for row in rows:
        step = int(_record_float(row, "step"))
        rmin, rmax = _record_float(row, "rho_min"), _record_float(row, "rho_max")
        drift, vmax = _record_float(row, "mass_total_delta_rel"), _record_float(row, "max_v")
        if not all(math.isfinite(value) for value in (rmin, rmax, drift, vmax)):
            result["all_records_finite"] = False
            _set_first(result, "first_nonfinite_step", step)
            failures.append((step, "nonfinite"))
        checks = ((rmin < float(rho_low), "first_negative_density_step", "negative_density"),
                  (rmax > float(rho_high), "first_high_density_step", "high_density"),
                  (abs(drift) > float(mass_drift_abs), "first_mass_drift_step", "mass_drift"),
                  (vmax > float(max_v), "first_max_v_step", "max_v"))
        for failed, key, reason in checks:
            if failed:
                _set_first(result, key, step)
                failures.append((step, reason))
    if failures:
        failures.sort(key=lambda item: item[0])
        result["first_failure_step"] = int(failures[0][0])
        result["first_failure_reason"] = failures[0][1]
    return result


def classify_first_failure_location(lbm_or_snapshot: Any) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:193-206 (default thresholds)."""
    t = _table(lbm_or_snapshot)
    return _classify(t)


def _classify(t: PlaneTable) -> Dict[str, Any]:
    density, velocity = _density(t, 0.0, 1.2), _velocity(t, 0.2)
    candidates = [density["first_negative_density_location"], density["first_high_density_location"],
                  velocity["first_velocity_outlier_location"]]
    location = next((candidate for candidate in candidates if candidate is not None), None)
    return {"first_failure_location": _location_label(location, t.shape) if location is not None else None,
            "first_failure_cell": location}


def summarize_lbm_stability_diagnostics(lbm_or_snapshot: Any, step: int) -> Dict[str, Any]:
    """lbm_stability_diagnostics.py:209-237 from one device pass."""
    t = _table(lbm_or_snapshot)
    density, velocity = _density(t, 0.0, 1.2), _velocity(t, 0.2)
    inlet, outlet = boundary_population_stats(t, "x_min"), boundary_population_stats(t, "x_max")
    location = _classify(t)
    return {
        "step": int(step),
        **population_stats(t),
        **negative_population_stats(t),
        "rho_min": density["rho_min"],
        "rho_max": density["rho_max"],
        "max_v": velocity["max_v"],
        "rho_below_low_count": density["rho_below_low_count"],
        "rho_above_high_count": density["rho_above_high_count"],
        "first_negative_density_location": density["first_negative_density_location"],
        "first_high_density_location": density["first_high_density_location"],
        "velocity_outlier_count": velocity["velocity_outlier_count"],
        "first_velocity_outlier_location": velocity["first_velocity_outlier_location"],
        "boundary_x_min_negative_population_count": inlet["negative_population_count"],
        "boundary_x_max_negative_population_count": outlet["negative_population_count"],
        "first_failure_location": location["first_failure_location"],
        "first_failure_cell": location["first_failure_cell"],
        "stability_all_finite": bool(density["all_finite"] and velocity["all_finite"] and inlet["all_finite"]
                                     and outlet["all_finite"]),
    }


def _location_label(location: Optional[List[int]], shape: Any) -> Optional[str]:
    if location is None:
        return None
    x, y, z = location
    nx, ny, nz = shape
    if x == 0:
        return "inlet"
    if x == nx - 1:
        return "outlet"
    if y in (0, ny - 1) or z in (0, nz - 1):
        return "wall_or_open_boundary_corner"
    return "interior"


def _set_first(result: Dict[str, Any], key: str, step: int) -> None:
    if result[key] is None:
        result[key] = int(step)


def _record_float(record: Dict[str, Any], key: str) -> float:
    value = record.get(key, 0.0)
    if value is None:
        return float("nan")
    return float(value)


def _finite_float(value: Any) -> float:
    # the reference's stability module returns non-finite values unchanged
    return float(value)

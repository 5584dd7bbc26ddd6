"""The reference's LBM boundary diagnostics
(src/mpm_lbm/sim/diagnostics/lbm_boundary_diagnostics.py), same names,
arguments and result keys, reduced on the device.

Each function takes an LBMFluid3D (its readout state, with a pending open
boundary applied) or a snapshot dict with rho, v and solid in the reference's
layouts.  The reductions run in one device pass (``_field_stats``), so a
summary costs one kernel and ~160 bytes per x plane of device-to-host copy
instead of the full rho and v fields.  Sums are FP64 like the reference's
numpy reductions of the float64 copies; they agree to FP64 rounding (the
summation order differs).  Standard deviations come from FP64 sums of x and
of squares (densities shifted by 1), not from numpy's two-pass form.
"""

from __future__ import annotations

import math
from typing import Any, Dict, List, Optional

import numpy as np

from ._field_stats import PlaneTable, field_stats


def snapshot_from_lbm(lbm: Any) -> Dict[str, np.ndarray]:
    """lbm_boundary_diagnostics.py:9-14: a host copy (the caller asks for one)."""
    return {
        "rho": np.asarray(lbm.rho.to_numpy(), dtype=float),
        "v": np.asarray(lbm.v.to_numpy(), dtype=float),
        "solid": np.asarray(lbm.solid.to_numpy(), dtype=np.int8),
    }


def _table(data: Any, **kw) -> PlaneTable:
    if isinstance(data, PlaneTable):
        return data
    return field_stats(data, **kw)


def fluid_mask(lbm_or_snapshot: Any) -> np.ndarray:
    if isinstance(lbm_or_snapshot, dict):
        return np.asarray(np.asarray(lbm_or_snapshot["solid"]) == 0, dtype=bool)
    return np.asarray(lbm_or_snapshot.solid.to_numpy() == 0, dtype=bool)


def _plane(t: PlaneTable, x_index: int) -> int:
    return _clamp_index(int(x_index), t.nx)


def plane_flux_x(lbm_or_snapshot: Any, x_index: int) -> float:
    """lbm_boundary_diagnostics.py:32-39."""
    t = _table(lbm_or_snapshot)
    x = _plane(t, x_index)
    if t["fluid_cells"][x] == 0:
        return 0.0
    return _finite_float(t["flux"][x])


def plane_mean_velocity_x(lbm_or_snapshot: Any, x_index: int) -> float:
    t = _table(lbm_or_snapshot)
    x = _plane(t, x_index)
    n = int(t["fluid_cells"][x])
    return _finite_float(t["ux_sum"][x] / n) if n else 0.0


def plane_mean_density_x(lbm_or_snapshot: Any, x_index: int) -> float:
    t = _table(lbm_or_snapshot)
    x = _plane(t, x_index)
    n = int(t["fluid_cells"][x])
    return _finite_float(t["rho_sum"][x] / n) if n else 0.0


def _rho_std(rho_sum: float, rho_sq_shifted: float, n: int) -> float:
    dm = rho_sum / n - 1.0
    return math.sqrt(max(rho_sq_shifted / n - dm * dm, 0.0)) if math.isfinite(dm) else float("nan")


def _std(total: float, sq: float, n: int) -> float:
    m = total / n
    var = sq / n - m * m
    return math.sqrt(max(var, 0.0)) if math.isfinite(var) else float("nan")


def _min_nan(t: PlaneTable, key: str, nan_key: str, sel=slice(None)) -> float:
    """np.min over the selected fluid cells (a NaN anywhere gives NaN)."""
    if int(np.sum(t[nan_key][sel])):
        return float("nan")
    return t.key_min(key, sel)


def _max_nan(t: PlaneTable, key: str, nan_key: str, sel=slice(None)) -> float:
    if int(np.sum(t[nan_key][sel])):
        return float("nan")
    return t.key_max(key, sel)


def density_stats(lbm_or_snapshot: Any) -> Dict[str, float]:
    """lbm_boundary_diagnostics.py:62-80."""
    t = _table(lbm_or_snapshot)
    n = int(np.sum(t["fluid_cells"], dtype=np.int64))
    if n == 0:
        return {"fluid_cell_count": 0, "rho_min": 0.0, "rho_max": 0.0, "rho_mean": 0.0, "rho_std": 0.0}
    total, sq = float(np.sum(t["rho_sum"])), float(np.sum(t["rho_sq"]))
    return {
        "fluid_cell_count": n,
        "rho_min": _finite_float(_min_nan(t, "rho_min", "rho_nan")),
        "rho_max": _finite_float(_max_nan(t, "rho_max", "rho_nan")),
        "rho_mean": _finite_float(total / n),
        "rho_std": _finite_float(_rho_std(total, sq, n)),
    }


def mass_total(lbm_or_snapshot: Any) -> float:
    t = _table(lbm_or_snapshot)
    if int(np.sum(t["fluid_cells"])) == 0:
        return 0.0
    return _finite_float(np.sum(t["rho_sum"]))


def centerline_profile_x(lbm_or_snapshot: Any, y_index: Optional[int] = None,
                         z_index: Optional[int] = None) -> Dict[str, Any]:
    """lbm_boundary_diagnostics.py:91-114."""
    if isinstance(lbm_or_snapshot, PlaneTable):
        raise TypeError("centerline_profile_x needs the lattice (its centerline cell is chosen here)")
    if isinstance(lbm_or_snapshot, dict):
        _, ny, nz = np.asarray(lbm_or_snapshot["rho"]).shape
    else:
        _, ny, nz = lbm_or_snapshot.dims
    y = _clamp_index(ny // 2 if y_index is None else int(y_index), ny)
    z = _clamp_index(nz // 2 if z_index is None else int(z_index), nz)
    t = field_stats(lbm_or_snapshot, cy=y, cz=z)
    return _centerline(t, y, z)


def _centerline(t: PlaneTable, y: int, z: int) -> Dict[str, Any]:
    values, source = [], []
    for x in range(t.nx):
        if t["center_fluid"][x]:
            values.append(_finite_float(t["center_ux"][x]))
            source.append("centerline")
        else:
            n = int(t["fluid_cells"][x])
            values.append(_finite_float(t["ux_sum"][x] / n) if n else 0.0)
            source.append("plane_mean_fallback")
    return {"axis": "x", "y_index": int(y), "z_index": int(z), "ux": values, "source": source}


def outlet_reflection_proxy(lbm_or_snapshot: Any) -> Dict[str, float]:
    """lbm_boundary_diagnostics.py:117-143."""
    t = _table(lbm_or_snapshot)
    nx = t.nx
    x = _clamp_index(nx - 2 if nx > 2 else nx - 1, nx)
    n = int(t["fluid_cells"][x])
    if n == 0:
        return {"proxy_name": "outlet_near_plane_ux_density_variation", "x_index": int(x), "fluid_cell_count": 0,
                "ux_std": 0.0, "negative_ux_fraction": 0.0, "rho_std": 0.0, "rho_peak_to_peak": 0.0}
    sel = slice(x, x + 1)
    return {
        "proxy_name": "outlet_near_plane_ux_density_variation",
        "x_index": int(x),
        "fluid_cell_count": n,
        "ux_std": _finite_float(_std(float(t["ux_sum"][x]), float(t["ux_sq"][x]), n)),
        "negative_ux_fraction": _finite_float(int(t["ux_negative"][x]) / n),
        "rho_std": _finite_float(_rho_std(float(t["rho_sum"][x]), float(t["rho_sq"][x]), n)),
        "rho_peak_to_peak": _finite_float(_max_nan(t, "rho_max", "rho_nan", sel)
                                          - _min_nan(t, "rho_min", "rho_nan", sel)),
    }


def plane_velocity_x_stats(lbm_or_snapshot: Any, x_index: int) -> Dict[str, float]:
    """lbm_boundary_diagnostics.py:146-168."""
    t = _table(lbm_or_snapshot)
    x = _plane(t, x_index)
    n = int(t["fluid_cells"][x])
    if n == 0:
        return {"x_index": int(x), "fluid_cell_count": 0, "ux_min": 0.0, "ux_max": 0.0, "ux_mean": 0.0,
                "negative_ux_fraction": 0.0}
    sel = slice(x, x + 1)
    return {
        "x_index": int(x),
        "fluid_cell_count": n,
        "ux_min": _finite_float(_min_nan(t, "ux_min", "ux_nan", sel)),
        "ux_max": _finite_float(_max_nan(t, "ux_max", "ux_nan", sel)),
        "ux_mean": _finite_float(t["ux_sum"][x] / n),
        "negative_ux_fraction": _finite_float(int(t["ux_negative"][x]) / n),
    }


def plane_density_stats(lbm_or_snapshot: Any, x_index: int) -> Dict[str, float]:
    """lbm_boundary_diagnostics.py:171-189."""
    t = _table(lbm_or_snapshot)
    x = _plane(t, x_index)
    n = int(t["fluid_cells"][x])
    if n == 0:
        return {"x_index": int(x), "fluid_cell_count": 0, "rho_mean": 0.0, "rho_std": 0.0}
    return {
        "x_index": int(x),
        "fluid_cell_count": n,
        "rho_mean": _finite_float(t["rho_sum"][x] / n),
        "rho_std": _finite_float(_rho_std(float(t["rho_sum"][x]), float(t["rho_sq"][x]), n)),
    }


def sampled_x_profile_indices(nx: int) -> List[int]:
    """lbm_boundary_diagnostics.py:192-198."""
    count = max(1, int(nx))
    if count >= 48:
        requested = [0, 6, 12, 18, 24, 30, 36, 42, 45, 46, 47]
    else:
        requested = [0, count // 4, count // 2, (3 * count) // 4, count - 3, count - 2, count - 1]
    return sorted({_clamp_index(index, count) for index in requested})


def sampled_x_profile_flux_map(lbm_or_snapshot: Any) -> Dict[str, float]:
    t = _table(lbm_or_snapshot)
    return {str(x): plane_flux_x(t, x) for x in sampled_x_profile_indices(t.nx)}


def sampled_x_profile_ux_mean_map(lbm_or_snapshot: Any) -> Dict[str, float]:
    t = _table(lbm_or_snapshot)
    return {str(x): plane_mean_velocity_x(t, x) for x in sampled_x_profile_indices(t.nx)}


def sampled_x_profile_rho_mean_map(lbm_or_snapshot: Any) -> Dict[str, float]:
    t = _table(lbm_or_snapshot)
    return {str(x): plane_mean_density_x(t, x) for x in sampled_x_profile_indices(t.nx)}


def sampled_x_profile_flux(lbm_or_snapshot: Any) -> str:
    flux = sampled_x_profile_flux_map(lbm_or_snapshot)
    return ";".join(f"{x}:{value:.12g}" for x, value in flux.items())


def _max_velocity(t: PlaneTable) -> float:
    if int(np.sum(t["fluid_cells"])) == 0:
        return 0.0
    if int(np.sum(t["vel_nan"])):
        return 0.0  # np.max over a NaN norm is NaN, which the reference reports as 0.0
    return _finite_float(t.speed_max())


def summarize_lbm_boundary_diagnostics(lbm_or_snapshot: Any, step: int,
                                       mass_initial: Optional[float] = None) -> Dict[str, Any]:
    """lbm_boundary_diagnostics.py:224-286 from one device pass."""
    t = _table(lbm_or_snapshot)
    density = density_stats(t)
    mass = mass_total(t)
    if mass_initial is None:
        mass_initial = mass
    mass_delta = mass - float(mass_initial)
    mass_delta_rel = 0.0 if float(mass_initial) == 0.0 else mass_delta / float(mass_initial)
    nx, ny, nz = t.shape
    mid_x = nx // 2
    inlet_flux = plane_flux_x(t, 0)
    outlet_flux = plane_flux_x(t, nx - 1)
    midplane_flux = plane_flux_x(t, mid_x)
    near1 = plane_flux_x(t, nx - 2)
    outlet_plane = plane_velocity_x_stats(t, nx - 1)
    outlet_plane_density = plane_density_stats(t, nx - 1)
    scale = max(abs(inlet_flux), abs(outlet_flux), 1.0e-12)
    flux_imbalance_abs = abs(inlet_flux - outlet_flux)
    max_v = _max_velocity(t)
    return {
        "step": int(step),
        **density,
        "mass_total": mass,
        "mass_total_delta_from_initial": _finite_float(mass_delta),
        "mass_total_delta_rel": _finite_float(mass_delta_rel),
        "inlet_mean_ux": plane_mean_velocity_x(t, 0),
        "outlet_mean_ux": plane_mean_velocity_x(t, nx - 1),
        "midplane_mean_ux": plane_mean_velocity_x(t, mid_x),
        "inlet_flux": inlet_flux,
        "outlet_flux": outlet_flux,
        "midplane_flux": midplane_flux,
        "near_outlet_flux_xminus1": near1,
        "near_outlet_flux_xminus2": plane_flux_x(t, nx - 3),
        "near_outlet_flux_xminus3": plane_flux_x(t, nx - 4),
        "near_outlet_to_outlet_flux_ratio": _safe_ratio(near1, outlet_flux),
        "flux_imbalance_abs": _finite_float(flux_imbalance_abs),
        "flux_imbalance_rel": _finite_float(flux_imbalance_abs / scale),
        "flux_balance_reported": True,
        "max_v": max_v,
        "mach_proxy_observed": _finite_float(max_v / math.sqrt(1.0 / 3.0)),
        "centerline_ux_profile": _centerline(t, ny // 2, nz // 2),
        "x_profile_flux_samples": sampled_x_profile_flux_map(t),
        "x_profile_ux_mean_samples": sampled_x_profile_ux_mean_map(t),
        "x_profile_rho_mean_samples": sampled_x_profile_rho_mean_map(t),
        "sampled_x_profile_flux": sampled_x_profile_flux(t),
        "outlet_reflection_proxy": outlet_reflection_proxy(t),
        "outlet_plane_ux_min": outlet_plane["ux_min"],
        "outlet_plane_ux_max": outlet_plane["ux_max"],
        "outlet_plane_ux_mean": outlet_plane["ux_mean"],
        "outlet_plane_negative_ux_fraction": outlet_plane["negative_ux_fraction"],
        "outlet_plane_rho_mean": outlet_plane_density["rho_mean"],
        "outlet_plane_rho_std": outlet_plane_density["rho_std"],
        "all_finite": int(np.sum(t["cell_nonfinite"])) == 0,
    }


def summarize_timeseries_trends(records: Any, tail_fraction: float = 0.2) -> Dict[str, Any]:
    """lbm_boundary_diagnostics.py:289-338 (host arithmetic on the records)."""
    rows = list(records)
    if not rows:
        raise ValueError("records must not be empty")
    if tail_fraction <= 0.0 or tail_fraction > 1.0:
        raise ValueError("tail_fraction must be in (0, 1]")
    tail_count = max(1, int(math.ceil(len(rows) * float(tail_fraction))))
    tail = rows[-tail_count:]
    final = rows[-1]

    def col(rows_, key):
        return [_record_float(row, key) for row in rows_]

    inlet_tail, outlet_tail = col(tail, "inlet_flux"), col(tail, "outlet_flux")
    imbalance_tail = col(tail, "flux_imbalance_rel")
    inlet_mean, outlet_mean = _finite_float(np.mean(inlet_tail)), _finite_float(np.mean(outlet_tail))
    inlet_ux_mean = _finite_float(np.mean(col(tail, "inlet_mean_ux")))
    mid_ux_mean = _finite_float(np.mean(col(tail, "midplane_mean_ux")))
    drift = col(rows, "mass_total_delta_rel")
    return {
        "record_count": int(len(rows)),
        "tail_fraction": float(tail_fraction),
        "tail_record_count": int(tail_count),
        "step_initial": int(_record_float(rows[0], "step")),
        "step_final": int(_record_float(final, "step")),
        "rho_min_global": _finite_float(min(col(rows, "rho_min"))),
        "rho_max_global": _finite_float(max(col(rows, "rho_max"))),
        "mass_drift_final": _record_float(final, "mass_total_delta_rel"),
        "mass_drift_abs_max": _finite_float(max(abs(v) for v in drift)),
        "mass_drift_tail_mean": _finite_float(np.mean(col(tail, "mass_total_delta_rel"))),
        "flux_imbalance_rel_final": _record_float(final, "flux_imbalance_rel"),
        "flux_imbalance_rel_min": _finite_float(min(col(rows, "flux_imbalance_rel"))),
        "flux_imbalance_rel_max": _finite_float(max(col(rows, "flux_imbalance_rel"))),
        "flux_imbalance_rel_tail_mean": _finite_float(np.mean(imbalance_tail)),
        "flux_imbalance_rel_tail_max": _finite_float(max(imbalance_tail)),
        "outlet_flux_final": _record_float(final, "outlet_flux"),
        "inlet_flux_tail_mean": inlet_mean,
        "outlet_flux_tail_mean": outlet_mean,
        "outlet_flux_tail_cv": _safe_cv(outlet_tail),
        "outlet_to_inlet_flux_ratio_tail_mean": _safe_ratio(outlet_mean, inlet_mean),
        "inlet_mean_ux_tail_mean": inlet_ux_mean,
        "midplane_mean_ux_tail_mean": mid_ux_mean,
        "midplane_to_inlet_flux_ratio_tail_mean": _safe_ratio(mid_ux_mean, inlet_ux_mean),
        "max_v_global": _finite_float(max(col(rows, "max_v"))),
        "mach_proxy_observed_max": _finite_float(max(col(rows, "mach_proxy_observed"))),
        "negative_ux_fraction_tail_mean": _finite_float(
            np.mean([_outlet_proxy_float(row, "negative_ux_fraction") for row in tail])),
        "rho_std_outlet_tail_mean": _finite_float(np.mean([_outlet_proxy_float(row, "rho_std") for row in tail])),
        "ux_std_outlet_tail_mean": _finite_float(np.mean([_outlet_proxy_float(row, "ux_std") for row in tail])),
    }


def _record_float(record: Dict[str, Any], key: str) -> float:
    return _finite_float(record.get(key, 0.0))


def _outlet_proxy_float(record: Dict[str, Any], key: str) -> float:
    proxy = record.get("outlet_reflection_proxy", {})
    if not isinstance(proxy, dict):
        return 0.0
    return _finite_float(proxy.get(key, 0.0))


def _safe_ratio(numerator: float, denominator: float) -> float:
    if abs(float(denominator)) < 1.0e-12:
        return 0.0
    return _finite_float(float(numerator) / float(denominator))


def _safe_cv(values: Any) -> float:
    array = np.asarray(list(values), dtype=float)
    if array.size == 0:
        return 0.0
    mean = _finite_float(np.mean(array))
    if abs(mean) < 1.0e-12:
        return 0.0
    return _finite_float(np.std(array) / abs(mean))


def _clamp_index(index: int, size: int) -> int:
    if size <= 0:
        raise ValueError("axis size must be positive")
    return max(0, min(index, size - 1))


def _finite_float(value: Any) -> float:
    result = float(value)
    if not math.isfinite(result):
        return 0.0
    return result

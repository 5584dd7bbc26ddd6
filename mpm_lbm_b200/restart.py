"""LBM restart files in the reference's npz format, plus an FSI resume
extension.

The reference format (src/mpm_lbm/sim/lbm/restart.py:10-147) is one
compressed npz with six arrays in the reference's field shapes and one JSON
string:
  rho (nx, ny, nz) f32, v (nx, ny, nz, 3) f32, f / F (nx, ny, nz, 19) f32,
  solid / static_solid (nx, ny, nz) i8, metadata_json (0-d unicode, sorted
  keys).
The functions below keep the reference's names, arguments, dictionaries and
errors, so a campaign script that saves or loads LBM restarts runs unchanged
on LBMFluid3D, and files move between the two implementations in both
directions.

Extension (not in the reference): save_fsi_restart / load_fsi_restart write
the same six arrays and metadata, and add the complete device state of an
FSIDriver3D under keys prefixed "ext_": the lattice in its device layout
(populations in the current AA parity, flags, link-force ping-pong,
subcycle accumulator, projected solid fields), the particles, and the step
counters.  A driver of the same configuration resumes from it exactly where
the saved one stood; readers of the reference format ignore the extra keys.
"""

from __future__ import annotations

import json
from pathlib import Path
from typing import Any

import numpy as np
import torch

RESTART_ARRAY_KEYS = ("rho", "v", "f", "F", "solid", "static_solid")
RESTART_METADATA_KEY = "metadata_json"

EXT_PREFIX = "ext_"
EXT_STATE_KEY = "ext_state_json"
EXT_VERSION = 3
# device tensors of LBMFluid3D / MPMSolid3D that a resume restores
_LBM_TENSORS = ("t_pop", "t_flags", "t_nbr", "t_rho", "t_vel", "t_static", "t_old", "t_reinit", "t_phi", "t_smass",
                "t_svel", "t_cf", "t_hydro", "t_accum", "t_hpp", "t_plane", "t_vin", "t_diag")
_LBM_ATTRS = ("parity", "bc_pending", "pp", "last_pp", "steps", "_accumulating", "_fused_accumulation",
              "_sample_count", "_hydro_src", "_old_equals_solid", "_penalty")
_MPM_TENSORS = ("t_x", "t_v", "t_C", "t_F", "t_Jp", "t_mass", "t_vol0", "t_fixed", "t_fixed_x")
_DRIVER_COUNTERS = ("current_lbm_step", "total_lbm_substeps", "total_mpm_substeps")


# ---------------------------------------------------------------- reference format
def write_lbm_restart_npz(path: str | Path, arrays: dict[str, np.ndarray], metadata: dict[str, Any],
                          extra: dict[str, np.ndarray] | None = None) -> dict:
    """restart.py:14-24.  `extra` (keys outside the reference's six) is
    written alongside; the reference's reader ignores it."""
    path = Path(path)
    missing = [key for key in RESTART_ARRAY_KEYS if key not in arrays]
    if missing:
        raise ValueError("missing LBM restart arrays: " + ", ".join(missing))
    path.parent.mkdir(parents=True, exist_ok=True)
    payload = {key: np.asarray(arrays[key]) for key in RESTART_ARRAY_KEYS}
    payload[RESTART_METADATA_KEY] = np.asarray(json.dumps(metadata, sort_keys=True))
    for key, value in (extra or {}).items():
        if key in payload:
            raise ValueError(f"extra restart key {key!r} collides with the LBM restart arrays")
        payload[key] = np.asarray(value)
    np.savez_compressed(path, **payload)
    return restart_payload_stats(payload, metadata)


def read_lbm_restart_npz(path: str | Path) -> tuple[dict[str, np.ndarray], dict[str, Any]]:
    """restart.py:27-34."""
    path = Path(path)
    if not path.is_file():
        raise FileNotFoundError(f"LBM restart not found: {path}")
    with np.load(path, allow_pickle=False) as data:
        arrays = {key: np.asarray(data[key]) for key in RESTART_ARRAY_KEYS}
        metadata_raw = str(np.asarray(data[RESTART_METADATA_KEY]).item())
    return arrays, json.loads(metadata_raw)


def validate_lbm_restart_metadata(metadata: dict[str, Any], expected: dict[str, Any]) -> dict:
    """restart.py:37-47: n_grid, boundary mode and target velocity must agree."""
    return {
        "restart_lbm_boundary_condition_mode_matches": bool(
            str(metadata.get("lbm_boundary_condition_mode", "")) == str(expected.get("lbm_boundary_condition_mode", ""))),
        "restart_n_grid_matches": bool(int(metadata.get("n_grid", -1)) == int(expected.get("n_grid", -2))),
        "restart_target_u_lbm_matches": bool(
            _float_list(metadata.get("target_u_lbm", [])) == _float_list(expected.get("target_u_lbm", []))),
    }


def load_lbm_restart_to_lbm(lbm, path: str | Path, expected_metadata: dict[str, Any], required: bool = False) -> dict:
    """restart.py:50-78: validate the metadata and shapes, then set rho, v, f,
    F, solid and static_solid in that order (f and F are one population field
    here, so F's values stand, as after the reference's streaming3 f = F)."""
    try:
        arrays, metadata = read_lbm_restart_npz(path)
    except FileNotFoundError:
        if required:
            raise
        return {"restart_loaded": False, "restart_missing": True}
    guard = validate_lbm_restart_metadata(metadata, expected_metadata)
    if not all(guard.values()):
        raise ValueError(f"LBM restart metadata mismatch: {guard}")
    _validate_restart_shapes(arrays, int(expected_metadata["n_grid"]), getattr(lbm, "dims", None))
    lbm.rho.from_numpy(arrays["rho"].astype(np.float32, copy=False))
    lbm.v.from_numpy(arrays["v"].astype(np.float32, copy=False))
    lbm.f.from_numpy(arrays["f"].astype(np.float32, copy=False))
    lbm.F.from_numpy(arrays["F"].astype(np.float32, copy=False))
    lbm.solid.from_numpy(arrays["solid"].astype(np.int8, copy=False))
    lbm.static_solid.from_numpy(arrays["static_solid"].astype(np.int8, copy=False))
    report = restart_payload_stats(arrays, metadata)
    report.update(guard)
    report.update({"restart_loaded": True, "restart_missing": False, "restart_path": str(path)})
    return report


def save_lbm_restart_from_lbm(lbm, path: str | Path, metadata: dict[str, Any]) -> dict:
    """restart.py:81-90."""
    return write_lbm_restart_npz(path, _lbm_arrays(lbm), metadata)


def expected_restart_metadata_from_config(config) -> dict:
    """restart.py:93-99."""
    return {
        "lbm_boundary_condition_mode": config.lbm_boundary_condition_mode,
        "lbm_restart_scope": config.lbm_restart_scope,
        "n_grid": int(config.n_grid),
        "target_u_lbm": [float(value) for value in config.target_u_lbm],
    }


def restart_payload_stats(arrays: dict[str, np.ndarray], metadata: dict[str, Any]) -> dict:
    """restart.py:102-129: density range and largest speed over fluid cells,
    NaN / Inf flags over the six arrays."""
    rho = np.asarray(arrays["rho"], dtype=np.float64)
    v = np.asarray(arrays["v"], dtype=np.float64)
    fluid = np.asarray(arrays["solid"]) == 0
    if np.any(fluid):
        rho_min, rho_max = float(np.min(rho[fluid])), float(np.max(rho[fluid]))
        max_v = float(np.max(np.linalg.norm(v[fluid], axis=1)))
    else:
        rho_min = rho_max = max_v = 0.0
    numeric = [np.asarray(arrays[key]) for key in RESTART_ARRAY_KEYS]
    floating = [a for a in numeric if np.issubdtype(a.dtype, np.floating)]
    return {
        "array_keys": list(RESTART_ARRAY_KEYS),
        "has_inf": bool(any(np.isinf(a).any() for a in floating)),
        "has_nan": bool(any(np.isnan(a).any() for a in floating)),
        "metadata": dict(metadata),
        "rho_max": rho_max,
        "rho_min": rho_min,
        "velocity_max_norm": max_v,
    }


def _validate_restart_shapes(arrays: dict[str, np.ndarray], n_grid: int, dims=None) -> None:
    """restart.py:132-143.  The reference's lattices are n_grid^3; a lattice
    of another shape (lattice_shape) is checked against its own dims."""
    dims = tuple(int(d) for d in dims) if dims is not None else (n_grid, n_grid, n_grid)
    expected = {"F": dims + (19,), "f": dims + (19,), "rho": dims, "solid": dims, "static_solid": dims,
                "v": dims + (3,)}
    bad = {key: arrays[key].shape for key, shape in expected.items() if arrays[key].shape != shape}
    if bad:
        raise ValueError(f"LBM restart array shape mismatch: {bad}")


def _float_list(values) -> list[float]:
    return [float(value) for value in values]


def _lbm_arrays(lbm) -> dict[str, np.ndarray]:
    F = lbm.F.to_numpy()
    return {"rho": lbm.rho.to_numpy(), "v": lbm.v.to_numpy(), "f": F.copy(), "F": F,
            "solid": lbm.solid.to_numpy(), "static_solid": lbm.static_solid.to_numpy()}


# ---------------------------------------------------------------- FSI resume extension
def _jsonable(value):
    if isinstance(value, tuple):
        return {"tuple": [_jsonable(v) for v in value]}
    return value


def _from_jsonable(value):
    if isinstance(value, dict) and "tuple" in value:
        return tuple(_from_jsonable(v) for v in value["tuple"])
    return value


def _device_counters(driver) -> dict:
    """Step counters of the state on the device.  A driver replaying a CUDA
    graph of `period` FSI steps runs the whole period at the first step_once
    of it, so between its steps the device is _graph_steps steps ahead of the
    counters; the file records the counters of the state it holds."""
    counters = {k: int(getattr(driver, k)) for k in _DRIVER_COUNTERS}
    ahead = int(getattr(driver, "_graph_steps", 0) or 0)
    if ahead and getattr(driver, "_graph", None) is not None:
        delta = driver._graph_delta
        period = max(1, delta[0])
        counters["current_lbm_step"] += ahead
        counters["total_lbm_substeps"] += ahead * (delta[1] // period)
        counters["total_mpm_substeps"] += ahead * (delta[2] // period)
    return counters


def save_fsi_restart(driver, path: str | Path, metadata: dict[str, Any] | None = None) -> dict:
    """Write the reference's LBM restart arrays of `driver.lbm` and, under
    "ext_" keys, the driver's complete device state (lattice in its device
    layout, particles, step counters).  Returns the payload statistics of
    the LBM arrays (as save_lbm_restart_from_lbm).  Between the steps of a
    replayed multi-step CUDA graph the device state is the one after the
    replay; the counters saved are that state's."""
    lbm, solid = driver.lbm, driver.solid
    if metadata is None:
        metadata = expected_restart_metadata_from_config(driver.config) if hasattr(driver.config, "lbm_restart_scope") \
            else {"n_grid": int(max(lbm.dims))}
    torch.cuda.synchronize(lbm.device)
    extra = {EXT_PREFIX + "lbm_" + k: getattr(lbm, k).cpu().numpy() for k in _LBM_TENSORS}
    extra.update({EXT_PREFIX + "mpm_" + k: getattr(solid, k).cpu().numpy() for k in _MPM_TENSORS})
    state = {
        "version": EXT_VERSION,
        "lattice": [int(d) for d in lbm.dims],
        "pitch": int(lbm.pitch),
        "population_storage": "fp16" if lbm.fp16 else "fp32",
        "n_particles": int(solid.n_particles),
        "n_grid": int(solid.n_grid),
        "lbm_attrs": {k: _jsonable(getattr(lbm, k)) for k in _LBM_ATTRS},
        "counters": _device_counters(driver),
    }
    extra[EXT_STATE_KEY] = np.asarray(json.dumps(state, sort_keys=True))
    return write_lbm_restart_npz(path, _lbm_arrays(lbm), metadata, extra=extra)


def load_fsi_restart(driver, path: str | Path) -> dict:
    """Restore a driver of the same configuration (lattice shape, population
    storage, particle count, MPM grid) from save_fsi_restart's file, so that
    its next steps continue the saved run.  Raises ValueError if the file has
    no extension or the configurations differ."""
    path = Path(path)
    if not path.is_file():
        raise FileNotFoundError(f"FSI restart not found: {path}")
    if not driver.initialized:
        driver.initialize()
    lbm, solid = driver.lbm, driver.solid
    with np.load(path, allow_pickle=False) as data:
        if EXT_STATE_KEY not in data.files:
            raise ValueError("restart file has no FSI resume state (written by save_lbm_restart_from_lbm?)")
        state = json.loads(str(np.asarray(data[EXT_STATE_KEY]).item()))
        want = {"lattice": [int(d) for d in lbm.dims], "pitch": int(lbm.pitch),
                "population_storage": "fp16" if lbm.fp16 else "fp32", "n_particles": int(solid.n_particles),
                "n_grid": int(solid.n_grid)}
        got = {k: state.get(k) for k in want}
        if state.get("version") != EXT_VERSION or got != want:
            raise ValueError(f"FSI restart does not match this driver: file {got}, driver {want}")
        tensors = {k: data[EXT_PREFIX + "lbm_" + k] for k in _LBM_TENSORS}
        tensors.update({("mpm", k): data[EXT_PREFIX + "mpm_" + k] for k in _MPM_TENSORS})
    for k in _LBM_TENSORS:
        dst = getattr(lbm, k)
        dst.copy_(torch.from_numpy(np.ascontiguousarray(tensors[k])).to(dst.device, dst.dtype))
    for k in _MPM_TENSORS:
        dst = getattr(solid, k)
        dst.copy_(torch.from_numpy(np.ascontiguousarray(tensors[("mpm", k)])).to(dst.device, dst.dtype))
    for k, v in state["lbm_attrs"].items():
        setattr(lbm, k, _from_jsonable(v))
    lbm._sync_params()
    lbm._version += 1
    # the MPM grid buffers are cleared, and the bins rebuilt, by the next FSI
    # step; they are allocated here, outside any CUDA-graph capture
    solid._ensure_binned()
    solid._binned_clean = False
    solid._since_bin = None
    for k, v in state["counters"].items():
        setattr(driver, k, int(v))
    driver._graph = None
    driver._graph_steps = 0
    driver._graph_warm = False
    return {"restart_loaded": True, "restart_path": str(path), "counters": dict(state["counters"])}

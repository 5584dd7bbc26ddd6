"""Opt-in wall velocity application to the lattice's solid_vel
(src/mpm_lbm/sim/wall_velocity/application.py, application_config.py).

The reference builds a capped velocity grid per motion phase on the host
(geometry sampling of its squid proxy, build_wall_velocity_grid,
application.py:46-115) and, after every projection of an FSI step, writes
it into ``lbm.solid_vel`` (apply_wall_velocity_to_lbm_solid_vel, 118-158):
host copies of solid_vel before and after and the arithmetic in numpy.
Here the grid goes to the device once per phase (cached) and one kernel
(fsi_apply_wall_velocity) applies it in FP64 and returns the statistics of
the reference's result dict; solid_vel never leaves the device.

The phase grid itself is host geometry work done once per phase; it comes
from a builder the caller provides (``grid_builder(config, n_grid, phase)
-> (grid (n, n, n, 3), summary)``, for instance the reference's
build_wall_velocity_grid).
"""

from __future__ import annotations

import ctypes
import json
import math
import os
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import Callable, Optional

import numpy as np
import torch

from ._lib import FSI_WALL_ADDITIVE, FSI_WALL_REPLACE, FsiWallVelocityStats, call, ptr, stream_handle

VALID_WALL_VELOCITY_APPLICATION_MODES = ("solid_vel_experimental",)
VALID_WALL_VELOCITY_APPLICATION_POLICIES = ("additive_capped", "replace_capped")
APPLICATION_FLAG_FIELDS = ("apply_to_lbm_solid_vel", "apply_to_lbm_populations", "apply_to_mpm", "apply_to_projector",
                           "modify_bounceback_formula", "jet_model_enabled", "actuation_claim_enabled",
                           "diagnostic_report_enabled")
APPLICATION_SCOPE_NOTE = "Step 36 opt-in experimental solid_vel application only; no bounce-back formula change"


@dataclass(frozen=True)
class WallVelocityApplicationConfig:
    """application_config.py:23-56, same fields and defaults."""

    application_id: str
    wall_velocity_config_path: str
    boundary_motion_config_path: str
    geometry_config_path: str
    region_config_path: str
    application_mode: str = "solid_vel_experimental"
    target_lbm_field: str = "solid_vel"
    application_policy: str = "additive_capped"
    wall_velocity_scale: float = 0.05
    wall_velocity_cap_lbm: float = 0.01
    apply_to_lbm_solid_vel: bool = True
    apply_to_lbm_populations: bool = False
    apply_to_mpm: bool = False
    apply_to_projector: bool = False
    modify_bounceback_formula: bool = False
    jet_model_enabled: bool = False
    actuation_claim_enabled: bool = False
    diagnostic_report_enabled: bool = True
    scope_note: str = "Step 36 opt-in experimental solid_vel application smoke only"

    def __post_init__(self):
        object.__setattr__(self, "wall_velocity_scale", float(self.wall_velocity_scale))
        object.__setattr__(self, "wall_velocity_cap_lbm", float(self.wall_velocity_cap_lbm))
        for name in APPLICATION_FLAG_FIELDS:
            object.__setattr__(self, name, bool(getattr(self, name)))

    @classmethod
    def from_json(cls, path, root=None):
        with _resolve(path, root).open("r", encoding="utf-8") as fh:
            return cls(**json.load(fh))

    def to_dict(self):
        return asdict(self)


def _resolve(path, root=None) -> Path:
    p = Path(os.fspath(path))
    if p.is_absolute():
        return p
    return Path(os.getcwd() if root is None else root) / p


def _check(name, passed, value, notes):
    return {"check": name, "pass": bool(passed), "value": value, "notes": notes}


def validate_wall_velocity_application_config(config: WallVelocityApplicationConfig, root=None) -> list:
    """application_config.py:59-89, the same checks in the same order.
    Relative paths resolve against ``root`` (default: the working
    directory; the reference resolves them against its package directory)."""
    def exists(path):
        return _resolve(path, root).is_file()

    c = config
    return [
        _check("application_id_present", bool(c.application_id), c.application_id, "application_id must be nonempty"),
        _check("wall_velocity_config_path_exists", exists(c.wall_velocity_config_path), c.wall_velocity_config_path,
               "Step 35 wall velocity config must exist"),
        _check("boundary_motion_config_path_exists", exists(c.boundary_motion_config_path),
               c.boundary_motion_config_path, "Step 34 boundary-motion config must exist"),
        _check("geometry_config_path_exists", exists(c.geometry_config_path), c.geometry_config_path,
               "Step 30 geometry config must exist"),
        _check("region_config_path_exists", exists(c.region_config_path), c.region_config_path,
               "Step 30 region config must exist"),
        _check("application_mode_valid", c.application_mode == "solid_vel_experimental", c.application_mode,
               "application_mode must be solid_vel_experimental"),
        _check("target_lbm_field_valid", c.target_lbm_field == "solid_vel", c.target_lbm_field,
               "target_lbm_field must be solid_vel"),
        _check("application_policy_valid", c.application_policy in VALID_WALL_VELOCITY_APPLICATION_POLICIES,
               c.application_policy, "application_policy must be supported"),
        _check("wall_velocity_scale_valid", math.isfinite(c.wall_velocity_scale) and 0.0 < c.wall_velocity_scale <= 1.0,
               c.wall_velocity_scale, "wall_velocity_scale must be in (0, 1]"),
        _check("wall_velocity_cap_lbm_valid",
               math.isfinite(c.wall_velocity_cap_lbm) and 0.0 < c.wall_velocity_cap_lbm <= 0.05,
               c.wall_velocity_cap_lbm, "wall_velocity_cap_lbm must be in (0, 0.05]"),
        _check("apply_to_lbm_solid_vel_true", c.apply_to_lbm_solid_vel is True, c.apply_to_lbm_solid_vel,
               "Step 36 applies only to lbm.solid_vel"),
        _check("apply_to_lbm_populations_false", c.apply_to_lbm_populations is False, c.apply_to_lbm_populations,
               "Step 36 must not write LBM populations"),
        _check("apply_to_mpm_false", c.apply_to_mpm is False, c.apply_to_mpm, "Step 36 must not write MPM state"),
        _check("apply_to_projector_false", c.apply_to_projector is False, c.apply_to_projector,
               "Step 36 must not write projector state"),
        _check("modify_bounceback_formula_false", c.modify_bounceback_formula is False, c.modify_bounceback_formula,
               "Step 36 must not modify bounce-back formulas"),
        _check("jet_model_enabled_false", c.jet_model_enabled is False, c.jet_model_enabled,
               "Step 36 must not enable a jet model"),
        _check("actuation_claim_enabled_false", c.actuation_claim_enabled is False, c.actuation_claim_enabled,
               "Step 36 must not enable actuation claims"),
        _check("diagnostic_report_enabled_true", c.diagnostic_report_enabled is True, c.diagnostic_report_enabled,
               "Step 36 must write diagnostic reports"),
        _check("scope_note_valid", "opt-in experimental" in c.scope_note and "solid_vel" in c.scope_note,
               c.scope_note, "scope_note must state opt-in experimental solid_vel application"),
    ]


def assert_valid_wall_velocity_application_config(config: WallVelocityApplicationConfig, root=None) -> None:
    rows = validate_wall_velocity_application_config(config, root=root)
    failed = [row for row in rows if not row["pass"]]
    if failed:
        raise ValueError(f"Step 36 wall velocity application config validation failed: {failed}")


def load_wall_velocity_application_config(path, root=None) -> WallVelocityApplicationConfig:
    config = WallVelocityApplicationConfig.from_json(path, root=root)
    assert_valid_wall_velocity_application_config(config, root=root)
    return config


class _DeviceGrid:
    """Velocity grids uploaded in lattice order (FP64), by caller key."""

    def __init__(self):
        self.cache = {}

    def get(self, lbm, grid, key=None):
        if isinstance(grid, torch.Tensor) and grid.is_cuda and grid.dtype == torch.float64 and grid.dim() == 2:
            return grid  # already [3][pitch] on the device
        if key is not None and key in self.cache:
            return self.cache[key]
        arr = np.asarray(grid, dtype=np.float64)
        t = torch.zeros(3, lbm.pitch, dtype=torch.float64, device=lbm.device)
        src = torch.from_numpy(np.ascontiguousarray(arr)).to(lbm.device)
        n = lbm.ncell
        t[:, :n] = src.permute(3, 2, 1, 0).reshape(3, n)
        if key is not None:
            self.cache[key] = t
        return t


_GRIDS = _DeviceGrid()


def apply_wall_velocity_to_lbm_solid_vel(lbm, velocity_grid, application_config, root=None, grid_key=None) -> dict:
    """application.py:118-158 on the device.  velocity_grid: (nx, ny, nz, 3)
    host array (or a [3][pitch] FP64 device tensor); grid_key caches the
    upload (e.g. the phase)."""
    if not isinstance(application_config, WallVelocityApplicationConfig):
        application_config = load_wall_velocity_application_config(application_config, root=root)
    assert_valid_wall_velocity_application_config(application_config, root=root)
    shape = tuple(lbm.dims) + (3,)
    if not isinstance(velocity_grid, torch.Tensor) and np.shape(velocity_grid) != shape:
        raise ValueError(f"velocity grid shape {np.shape(velocity_grid)} does not match lbm.solid_vel shape {shape}")
    policy = application_config.application_policy
    if policy == "replace_capped":
        code = FSI_WALL_REPLACE
    elif policy == "additive_capped":
        code = FSI_WALL_ADDITIVE
    else:
        raise ValueError(f"unsupported application_policy: {policy}")
    grid = _GRIDS.get(lbm, velocity_grid, grid_key)
    out = torch.zeros(ctypes.sizeof(FsiWallVelocityStats), dtype=torch.uint8, device=lbm.device)
    cap = float(application_config.wall_velocity_cap_lbm)
    call("fsi_apply_wall_velocity", ctypes.byref(lbm.state), ptr(grid), code, cap, ptr(out), stream_handle())
    lbm._version += 1
    st = FsiWallVelocityStats.from_buffer_copy(out.cpu().numpy().tobytes())
    n = int(st.applied_cells)
    return {
        "applied_cell_count": n,
        "max_applied_velocity_norm": float(st.delta_norm_max) if n else 0.0,
        "mean_applied_velocity_norm": float(st.delta_norm_sum) / n if n else 0.0,
        "before_solid_vel_norm_max": float(st.before_norm_max),
        "after_solid_vel_norm_max": float(st.after_norm_max),
        "after_solid_vel_norm_mean_active": float(st.after_norm_sum_active) / n if n else 0.0,
        "cap_pass": float(st.after_norm_max_active) <= cap + 1.0e-12 if n else True,
        "lbm_population_update_count": 0,
        "apply_to_lbm_solid_vel": bool(application_config.apply_to_lbm_solid_vel),
        "apply_to_lbm_populations": bool(application_config.apply_to_lbm_populations),
        "modify_bounceback_formula": bool(application_config.modify_bounceback_formula),
    }


def apply_wall_velocity_application_to_lbm(lbm, application_config_path, n_grid: int, lbm_step: int,
                                           report_path=None, grid_builder: Optional[Callable] = None,
                                           phase_for_step: Optional[Callable] = None, root=None) -> dict:
    """application.py:196-231.  grid_builder(config, n_grid, phase) ->
    (grid, grid_summary) builds the phase grid on the host (the reference's
    build_wall_velocity_grid fits); phase_for_step(config, lbm_step) gives
    the phase (the reference's phase_for_lbm_step)."""
    if grid_builder is None or phase_for_step is None:
        raise NotImplementedError("the wall velocity grid is built on the host from the reference's squid-proxy "
                                  "geometry: pass grid_builder and phase_for_step")
    config = load_wall_velocity_application_config(application_config_path, root=root)
    requested_phase = phase_for_step(config, lbm_step)
    velocity_grid, grid_summary = grid_builder(config, n_grid=n_grid, phase=requested_phase)
    key = (config.application_id, int(n_grid), float(grid_summary.get("selected_phase", requested_phase)))
    result = apply_wall_velocity_to_lbm_solid_vel(lbm, velocity_grid, config, root=root, grid_key=key)
    summary = dict(grid_summary)
    summary.update({
        "application_mode": config.application_mode,
        "target_lbm_field": config.target_lbm_field,
        "application_policy": config.application_policy,
        "apply_to_lbm_solid_vel": bool(config.apply_to_lbm_solid_vel),
        "apply_to_lbm_populations": bool(config.apply_to_lbm_populations),
        "apply_to_mpm": bool(config.apply_to_mpm),
        "apply_to_projector": bool(config.apply_to_projector),
        "driver_lbm_step": int(lbm_step),
    })
    summary.update(result)
    summary["report_pass"] = bool(
        summary.get("finite_pass", True) and summary["cap_pass"] and int(summary["applied_cell_count"]) > 0
        and float(summary["max_applied_velocity_norm"]) <= float(config.wall_velocity_cap_lbm) + 1.0e-12
        and int(summary["lbm_population_update_count"]) == 0 and not bool(summary["modify_bounceback_formula"]))
    report = {"summary": summary, "config": config.to_dict()}
    if report_path:
        path = Path(report_path)
        path.parent.mkdir(parents=True, exist_ok=True)
        with path.open("w", encoding="utf-8") as fh:
            json.dump(report, fh, indent=2, sort_keys=True)
            fh.write("\n")
    return report

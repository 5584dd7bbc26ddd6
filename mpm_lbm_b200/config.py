"""Configuration types of the FSI step, with the reference's field names,
defaults and validation rules, so a reference config (JSON or keyword form)
drives this package unchanged.

Reference anchors (lizhuoh9/MPM-LBM):
  FSIDriverConfig   src/mpm_lbm/sim/drivers/fsi_config.py:67-537
  UnifiedSimConfig  src/mpm_lbm/sim/drivers/sim_config.py:9-99
  LBMConfig         src/mpm_lbm/sim/lbm/config.py:37-165
  MPMConfig         src/mpm_lbm/sim/mpm/config.py:5-30
  tau conventions   src/mpm_lbm/sim/lbm/relaxation_semantics.py:14-19
  GridUnitMapper    src/mpm_lbm/sim/units/mapper.py:6-57
"""

from __future__ import annotations

import json
import math
from dataclasses import asdict, dataclass, field, fields
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER = "legacy_external_solver_relaxation_parameter"
STANDARD_LATTICE_KINEMATIC_VISCOSITY = "standard_lattice_kinematic_viscosity"


def tau_from_legacy_external_solver_parameter(niu: float) -> float:
    return float(niu) / 3.0 + 0.5


def tau_from_lattice_kinematic_viscosity(nu_lbm: float) -> float:
    return 3.0 * float(nu_lbm) + 0.5


OPEN_BOUNDARY_SEMANTICS = (
    "equilibrium_all_population_reset",
    "regularized_velocity_pressure",
    "regularized_velocity_pressure_limited",
    "convective_pressure_outlet_experimental",
    "regularized_mass_balanced_pressure_outlet",
    "convective_mass_balanced_pressure_outlet",
    "regularized_flux_matched_pressure_outlet",
    "convective_flux_matched_damped_outlet",
    "regularized_plane_flux_controlled_pressure_outlet",
    "convective_plane_flux_controlled_damped_outlet",
)
# FsiLbmParams.ob_semantics code of each (FSI_OB_* in the C header); the FSI
# driver config exposes the first four (fsi_config.py:32-37), LBMConfig all ten
KERNEL_OPEN_BOUNDARY_CODES = {name: code for code, name in enumerate(OPEN_BOUNDARY_SEMANTICS)}
OPEN_BOUNDARY_MASS_NEUTRAL_FLUX_CONTROL_MODES = (
    "disabled",
    "global_mass_error_density_offset",
    "outlet_population_projection_report_only",
)
OPEN_BOUNDARY_MASS_NEUTRAL_REFERENCE_MASS_MODES = ("initial",)


@dataclass
class LBMConfig:
    nx: int
    ny: int
    nz: int
    niu: float = 0.1
    rho0: float = 1.0
    relaxation_semantics: str = LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER
    open_boundary_semantics: str = "equilibrium_all_population_reset"
    open_boundary_limiter_enabled: bool = False
    open_boundary_rho_min: float = 0.8
    open_boundary_rho_max: float = 1.2
    open_boundary_u_max: float = 0.1
    open_boundary_noneq_cap: float = 0.05
    open_boundary_population_floor: Optional[float] = None
    open_boundary_flux_feedback_gain_u: float = 0.01
    open_boundary_flux_feedback_gain_rho: float = 0.005
    open_boundary_flux_filter_alpha: float = 0.05
    open_boundary_flux_correction_cap_u: float = 0.005
    open_boundary_flux_feedback_delta_cap_u: float = 0.0
    open_boundary_flux_feedback_slew_alpha: float = 1.0
    open_boundary_convective_blend_weight: float = 0.05
    open_boundary_flux_control_measure_plane_offset: int = 0
    open_boundary_flux_control_target_scale: float = 1.0
    open_boundary_outlet_flux_drop_guard_enabled: bool = False
    open_boundary_outlet_flux_drop_guard_min_ratio: float = 0.60
    open_boundary_mass_neutral_flux_control_enabled: bool = False
    open_boundary_mass_neutral_flux_control_mode: str = "disabled"
    open_boundary_mass_neutral_mass_error_gain: float = 0.0
    open_boundary_mass_neutral_mass_error_cap: float = 0.0
    open_boundary_mass_neutral_correction_blend: float = 0.0
    open_boundary_mass_neutral_reference_mass_mode: str = "initial"
    sparse_storage: bool = False
    force: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bc_x_left: int = 0
    bc_x_right: int = 0
    bc_y_left: int = 0
    bc_y_right: int = 0
    bc_z_left: int = 0
    bc_z_right: int = 0
    rho_bc_x_left: float = 1.0
    rho_bc_x_right: float = 1.0
    rho_bc_y_left: float = 1.0
    rho_bc_y_right: float = 1.0
    rho_bc_z_left: float = 1.0
    rho_bc_z_right: float = 1.0
    vel_bc_x_left: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    vel_bc_x_right: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    vel_bc_y_left: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    vel_bc_y_right: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    vel_bc_z_left: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    vel_bc_z_right: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    # B200 extensions (not in the reference): collision operator and population storage
    collision: str = "mrt"
    population_storage: str = "fp32"

    def __post_init__(self):
        if self.relaxation_semantics not in (LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER,
                                             STANDARD_LATTICE_KINEMATIC_VISCOSITY):
            raise ValueError("relaxation_semantics must be one of "
                             f"{(LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER, STANDARD_LATTICE_KINEMATIC_VISCOSITY)}")
        if self.open_boundary_semantics not in OPEN_BOUNDARY_SEMANTICS:
            raise ValueError(f"open_boundary_semantics must be one of {OPEN_BOUNDARY_SEMANTICS}")
        if self.open_boundary_rho_min <= 0.0:
            raise ValueError("open_boundary_rho_min must be positive")
        if self.open_boundary_rho_max <= self.open_boundary_rho_min:
            raise ValueError("open_boundary_rho_min must be less than open_boundary_rho_max")
        if self.open_boundary_u_max <= 0.0:
            raise ValueError("open_boundary_u_max must be positive")
        if self.open_boundary_noneq_cap <= 0.0:
            raise ValueError("open_boundary_noneq_cap must be positive")
        self._check_flux_control()
        if self.collision not in ("mrt", "bgk"):
            raise ValueError("collision must be 'mrt' or 'bgk'")
        if self.population_storage not in ("fp32", "fp16"):
            raise ValueError("population_storage must be 'fp32' or 'fp16'")

    def _check_flux_control(self):
        """The outlet repair and flux-controller rules of lbm/config.py:109-165,
        in the reference's order."""
        def nonneg(name):
            if getattr(self, name) < 0.0:
                raise ValueError(f"{name} must be non-negative")

        nonneg("open_boundary_flux_feedback_gain_u")
        nonneg("open_boundary_flux_feedback_gain_rho")
        if not (0.0 < self.open_boundary_flux_filter_alpha <= 1.0):
            raise ValueError("open_boundary_flux_filter_alpha must be in (0, 1]")
        if self.open_boundary_flux_correction_cap_u <= 0.0:
            raise ValueError("open_boundary_flux_correction_cap_u must be positive")
        nonneg("open_boundary_flux_feedback_delta_cap_u")
        if not (0.0 < self.open_boundary_flux_feedback_slew_alpha <= 1.0):
            raise ValueError("open_boundary_flux_feedback_slew_alpha must be in (0, 1]")
        if not (0.0 <= self.open_boundary_convective_blend_weight <= 1.0):
            raise ValueError("open_boundary_convective_blend_weight must be in [0, 1]")
        offset = self.open_boundary_flux_control_measure_plane_offset
        if int(offset) != offset:
            raise ValueError("open_boundary_flux_control_measure_plane_offset must be an integer")
        if not (0 <= int(offset) <= 2):
            raise ValueError("open_boundary_flux_control_measure_plane_offset must be 0, 1, or 2")
        self.open_boundary_flux_control_measure_plane_offset = int(offset)
        if self.open_boundary_flux_control_target_scale <= 0.0:
            raise ValueError("open_boundary_flux_control_target_scale must be positive")
        self.open_boundary_flux_control_target_scale = float(self.open_boundary_flux_control_target_scale)
        if not (0.0 < self.open_boundary_outlet_flux_drop_guard_min_ratio <= 1.0):
            raise ValueError("open_boundary_outlet_flux_drop_guard_min_ratio must be in (0, 1]")
        self.open_boundary_mass_neutral_flux_control_enabled = bool(self.open_boundary_mass_neutral_flux_control_enabled)
        if self.open_boundary_mass_neutral_flux_control_mode not in OPEN_BOUNDARY_MASS_NEUTRAL_FLUX_CONTROL_MODES:
            raise ValueError("open_boundary_mass_neutral_flux_control_mode must be one of "
                             f"{OPEN_BOUNDARY_MASS_NEUTRAL_FLUX_CONTROL_MODES}")
        if self.open_boundary_mass_neutral_reference_mass_mode not in OPEN_BOUNDARY_MASS_NEUTRAL_REFERENCE_MASS_MODES:
            raise ValueError("open_boundary_mass_neutral_reference_mass_mode must be one of "
                             f"{OPEN_BOUNDARY_MASS_NEUTRAL_REFERENCE_MASS_MODES}")
        if self.open_boundary_mass_neutral_flux_control_enabled and \
                self.open_boundary_mass_neutral_flux_control_mode == "disabled":
            raise ValueError("open_boundary_mass_neutral_flux_control_enabled cannot be true when mode is disabled")
        nonneg("open_boundary_mass_neutral_mass_error_gain")
        nonneg("open_boundary_mass_neutral_mass_error_cap")
        if not (0.0 <= self.open_boundary_mass_neutral_correction_blend <= 1.0):
            raise ValueError("open_boundary_mass_neutral_correction_blend must be in [0, 1]")
        for name in ("open_boundary_mass_neutral_mass_error_gain", "open_boundary_mass_neutral_mass_error_cap",
                     "open_boundary_mass_neutral_correction_blend"):
            setattr(self, name, float(getattr(self, name)))


@dataclass
class MPMConfig:
    n_grid: int = 32
    dx: float = 1.0 / 32.0
    dt: float = 4.0e-4
    gravity: Tuple[float, float, float] = (0.0, -9.8, 0.0)
    p_rho: float = 1.0
    particles_per_cell: int = 2
    young_modulus: float = 400.0
    poisson_ratio: float = 0.2
    bound: int = 3
    use_apic: bool = True
    box_min: Tuple[float, float, float] = (0.25, 0.35, 0.25)
    box_max: Tuple[float, float, float] = (0.55, 0.65, 0.55)
    mpm_planar_constraint_mode: str = "disabled"
    mpm_planar_constraint_axis: str = "z"
    mpm_velocity_damping: float = 0.0
    mpm_damping_application: str = "disabled"
    output_interval: int = 10


@dataclass(frozen=True)
class UnifiedSimConfig:
    n_grid: int = 32
    domain_length: float = 1.0
    mpm_dt: float = 4.0e-4
    mpm_substeps_per_lbm_step: int = 10
    lbm_niu: float = 0.1
    lbm_rho0: float = 1.0
    lbm_relaxation_semantics: str = LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER
    lbm_open_boundary_semantics: str = "equilibrium_all_population_reset"
    open_boundary_limiter_enabled: bool = False
    open_boundary_rho_min: float = 0.8
    open_boundary_rho_max: float = 1.2
    open_boundary_u_max: float = 0.1
    open_boundary_noneq_cap: float = 0.05
    open_boundary_population_floor: Optional[float] = None
    lbm_dt_phys_override_s: Optional[float] = None

    def __post_init__(self):
        checks = [
            (self.n_grid <= 0, "n_grid must be positive"),
            (self.domain_length <= 0.0, "domain_length must be positive"),
            (self.mpm_dt <= 0.0, "mpm_dt must be positive"),
            (self.mpm_substeps_per_lbm_step <= 0, "mpm_substeps_per_lbm_step must be positive"),
            (self.lbm_niu <= 0.0, "lbm_niu must be positive"),
            (self.lbm_rho0 <= 0.0, "lbm_rho0 must be positive"),
            (self.open_boundary_rho_min <= 0.0, "open_boundary_rho_min must be positive"),
            (self.open_boundary_rho_max <= self.open_boundary_rho_min,
             "open_boundary_rho_min must be less than open_boundary_rho_max"),
            (self.open_boundary_u_max <= 0.0, "open_boundary_u_max must be positive"),
            (self.open_boundary_noneq_cap <= 0.0, "open_boundary_noneq_cap must be positive"),
            (self.lbm_dt_phys_override_s is not None and self.lbm_dt_phys_override_s <= 0.0,
             "lbm_dt_phys_override_s must be positive when provided"),
        ]
        for bad, msg in checks:
            if bad:
                raise ValueError(msg)

    nx = property(lambda self: self.n_grid)
    ny = property(lambda self: self.n_grid)
    nz = property(lambda self: self.n_grid)

    @property
    def dx_norm(self) -> float:
        return self.domain_length / float(self.n_grid)

    @property
    def lbm_dt_phys(self) -> float:
        if self.lbm_dt_phys_override_s is not None:
            return float(self.lbm_dt_phys_override_s)
        return self.mpm_substeps_per_lbm_step * self.mpm_dt

    def make_lbm_config(self, **overrides) -> LBMConfig:
        values = dict(nx=self.nx, ny=self.ny, nz=self.nz, niu=self.lbm_niu, rho0=self.lbm_rho0,
                      relaxation_semantics=self.lbm_relaxation_semantics,
                      open_boundary_semantics=self.lbm_open_boundary_semantics,
                      open_boundary_limiter_enabled=self.open_boundary_limiter_enabled,
                      open_boundary_rho_min=self.open_boundary_rho_min,
                      open_boundary_rho_max=self.open_boundary_rho_max,
                      open_boundary_u_max=self.open_boundary_u_max,
                      open_boundary_noneq_cap=self.open_boundary_noneq_cap,
                      open_boundary_population_floor=self.open_boundary_population_floor)
        values.update(overrides)
        return LBMConfig(**values)

    def make_mpm_config(self, **overrides) -> MPMConfig:
        values = dict(n_grid=self.n_grid, dx=self.dx_norm, dt=self.mpm_dt)
        values.update(overrides)
        return MPMConfig(**values)


@dataclass(frozen=True)
class GridUnitMapper:
    n_grid: int
    dx_norm: float
    lbm_dt_phys: float

    @classmethod
    def from_sim_config(cls, sim):
        return cls(n_grid=sim.n_grid, dx_norm=sim.dx_norm, lbm_dt_phys=sim.lbm_dt_phys)

    def velocity_norm_to_lbm(self, v):
        return np.asarray(v, dtype=np.float64) * self.lbm_dt_phys / self.dx_norm

    def velocity_lbm_to_norm(self, v):
        return np.asarray(v, dtype=np.float64) * self.dx_norm / self.lbm_dt_phys

    def acceleration_norm_to_lbm(self, a):
        return np.asarray(a, dtype=np.float64) * self.lbm_dt_phys ** 2 / self.dx_norm

    def acceleration_lbm_to_norm(self, a):
        return np.asarray(a, dtype=np.float64) * self.dx_norm / self.lbm_dt_phys ** 2

    def viscosity_norm_to_lbm(self, nu):
        return float(nu) * self.lbm_dt_phys / (self.dx_norm ** 2)

    def viscosity_lbm_to_norm(self, nu):
        return float(nu) * (self.dx_norm ** 2) / self.lbm_dt_phys


_CHOICES = {
    "coupling_mode": ("none", "penalty", "moving_boundary"),
    "reaction_transfer_mode": ("engineering", "link_area_experimental", "interface_traction_conservative"),
    "link_area_policy": ("uniform", "inverse_length", "length"),
    "boundary_motion_mode": ("static", "prescribed_kinematic"),
    "wall_velocity_application_mode": ("disabled", "solid_vel_experimental"),
    "geometry_motion_mode": ("static", "prescribed_kinematic"),
    "geometry_motion_application_mode": ("disabled", "diagnostic_only"),
    "lbm_boundary_condition_mode": ("default_periodic", "duct_velocity_inlet_pressure_outlet"),
    "lbm_open_boundary_semantics": ("equilibrium_all_population_reset", "zou_he_reconstruct_unknowns",
                                    "regularized_velocity_pressure", "regularized_velocity_pressure_limited",
                                    "convective_pressure_outlet_experimental"),
    "lbm_viscosity_semantics": ("legacy_external", "physical_nu_mapping"),
    "lbm_tau_stability_policy": ("report_only", "strict"),
    "fsi_exchange_mode": ("one_lbm_step_per_fsi_step", "lbm_subcycled_per_fsi_step"),
    "lbm_restart_scope": ("rho_velocity_populations",),
    "mpm_planar_constraint_mode": ("disabled", "lock_z"),
    "mpm_planar_constraint_axis": ("z",),
    "mpm_damping_application": ("disabled", "particle_velocity_post_g2p"),
    "solid_model": ("finite_deformation_mpm", "small_strain_linear_elastic"),
    "solid_dimensionality": ("three_dimensional", "plane_strain_2d", "plane_stress_2d"),
    "flow_dimensionality_mode": ("three_dimensional", "thin_3d_no_slip_z_walls", "d2q9_planar",
                                 "d3q19_quasi_2d_periodic_z"),
    "velocity_inlet_axis": ("x",),
    "velocity_inlet_side": ("min", "max"),
    "pressure_outlet_side": ("min", "max"),
    "geometry_type": ("box", "ellipsoid", "squid_proxy", "duct_flap_proxy", "voxel", "mesh"),
}
_NOT_IMPLEMENTED = {
    "lbm_open_boundary_semantics": ("zou_he_reconstruct_unknowns",),
    "solid_model": ("small_strain_linear_elastic",),
    "solid_dimensionality": ("plane_strain_2d", "plane_stress_2d"),
    "flow_dimensionality_mode": ("d2q9_planar", "d3q19_quasi_2d_periodic_z"),
}


def _tuple3(v, name):
    if len(v) != 3:
        raise ValueError(f"{name} must contain exactly three values")
    return tuple(float(a) for a in v)


@dataclass(frozen=True)
class FSIDriverConfig:
    coupling_mode: str = "penalty"
    geometry_type: str = "box"
    geometry_config_path: Optional[str] = None
    n_grid: int = 32
    n_particles: int = 4096
    n_lbm_steps: int = 20
    mpm_substeps_per_lbm_step: int = 10
    mpm_dt: float = 4.0e-4
    target_u_lbm: Tuple[float, float, float] = (0.02, 0.0, 0.0)
    initial_solid_velocity_norm: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    gravity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    lbm_boundary_condition_mode: str = "default_periodic"
    lbm_open_boundary_semantics: str = "equilibrium_all_population_reset"
    open_boundary_limiter_enabled: bool = False
    open_boundary_rho_min: float = 0.8
    open_boundary_rho_max: float = 1.2
    open_boundary_u_max: float = 0.1
    open_boundary_noneq_cap: float = 0.05
    open_boundary_population_floor: Optional[float] = None
    velocity_inlet_axis: str = "x"
    velocity_inlet_side: str = "min"
    pressure_outlet_side: str = "max"
    physical_duct_length_m: float = 1.0
    target_inlet_velocity_mps: Optional[float] = None
    official_fsi_dt_s: Optional[float] = None
    target_u_lbm_for_dimensional_mapping: Optional[float] = None
    lbm_substeps_per_fsi_step: int = 1
    lbm_dt_phys_override_s: Optional[float] = None
    fluid_density_kg_m3: float = 1.225
    fluid_kinematic_viscosity_m2_s: float = 1.5e-5
    target_reynolds_number: Optional[float] = None
    lbm_viscosity_semantics: str = "legacy_external"
    lbm_min_tau_margin: float = 1.0e-4
    lbm_tau_stability_policy: str = "report_only"
    fsi_exchange_mode: str = "one_lbm_step_per_fsi_step"
    lbm_restart_path: Optional[str] = None
    lbm_restart_required: bool = False
    lbm_restart_scope: str = "rho_velocity_populations"
    box_min: Tuple[float, float, float] = (0.25, 0.35, 0.25)
    box_max: Tuple[float, float, float] = (0.55, 0.65, 0.55)
    dynamic_solid_threshold: float = 0.5
    beta_lbm: float = 1.0e-3
    penalty_force_cap_lbm: float = 1.0e-4
    mb_reaction_scale: float = 1.0
    mb_force_cap_norm: float = 1.0e-4
    reaction_transfer_mode: str = "engineering"
    solid_model: str = "finite_deformation_mpm"
    solid_dimensionality: str = "three_dimensional"
    flow_dimensionality_mode: str = "three_dimensional"
    link_area_policy: str = "inverse_length"
    link_area_scale_min: float = 0.25
    link_area_scale_max: float = 2.0
    boundary_motion_mode: str = "static"
    boundary_motion_config_path: Optional[str] = None
    boundary_motion_report_enabled: bool = False
    wall_velocity_application_mode: str = "disabled"
    wall_velocity_application_config_path: Optional[str] = None
    wall_velocity_application_report_enabled: bool = False
    geometry_motion_mode: str = "static"
    geometry_motion_config_path: Optional[str] = None
    geometry_motion_report_enabled: bool = False
    geometry_motion_application_mode: str = "disabled"
    geometry_motion_application_config_path: Optional[str] = None
    geometry_motion_application_report_enabled: bool = False
    mpm_planar_constraint_mode: str = "disabled"
    mpm_planar_constraint_axis: str = "z"
    mpm_velocity_damping: float = 0.0
    mpm_damping_application: str = "disabled"
    fluent_like_monitor_enabled: bool = False
    fluent_like_monitor_physical_point_m: Tuple[float, float] = (0.0505, 0.0095)
    fluent_like_monitor_nearest_count: int = 8
    fluent_like_monitor_radius_m: Optional[float] = None
    output_interval: int = 10
    write_vtk: bool = False
    write_particles: bool = False
    quality_check_enabled: bool = False
    quality_check_strict: bool = False
    quality_report_path: Optional[str] = None

    def __post_init__(self):
        for name in ("target_u_lbm", "initial_solid_velocity_norm", "gravity", "box_min", "box_max"):
            object.__setattr__(self, name, _tuple3(getattr(self, name), name))
        pt = self.fluent_like_monitor_physical_point_m
        if len(pt) != 2:
            raise ValueError("fluent_like_monitor_physical_point_m must contain exactly two values")
        object.__setattr__(self, "fluent_like_monitor_physical_point_m", tuple(float(v) for v in pt))
        for name, choices in _CHOICES.items():
            if getattr(self, name) not in choices:
                raise ValueError(f"{name} must be one of {choices}")
        for name, bad in _NOT_IMPLEMENTED.items():
            if getattr(self, name) in bad:
                raise ValueError(f"{name}={getattr(self, name)!r} is not implemented")
        if self.reaction_transfer_mode == "interface_traction_conservative":
            raise ValueError("reaction_transfer_mode='interface_traction_conservative' is planned but not implemented")
        if self.reaction_transfer_mode == "link_area_experimental" and self.coupling_mode != "moving_boundary":
            raise ValueError("reaction_transfer_mode='link_area_experimental' requires coupling_mode='moving_boundary'")
        if self.mpm_damping_application == "disabled" and float(self.mpm_velocity_damping) != 0.0:
            raise ValueError("mpm_velocity_damping must be 0 when mpm_damping_application is disabled")
        if self.mpm_damping_application == "particle_velocity_post_g2p" and float(self.mpm_velocity_damping) <= 0.0:
            raise ValueError("mpm_velocity_damping must be positive when damping is enabled")
        if self.lbm_restart_required and not self.lbm_restart_path:
            raise ValueError("lbm_restart_path is required when lbm_restart_required is true")
        if self.lbm_boundary_condition_mode == "duct_velocity_inlet_pressure_outlet":
            if self.velocity_inlet_side == self.pressure_outlet_side:
                raise ValueError("velocity_inlet_side and pressure_outlet_side must differ")
        positives = [("n_grid", self.n_grid), ("n_particles", self.n_particles), ("n_lbm_steps", self.n_lbm_steps),
                     ("mpm_substeps_per_lbm_step", self.mpm_substeps_per_lbm_step), ("mpm_dt", self.mpm_dt),
                     ("physical_duct_length_m", self.physical_duct_length_m),
                     ("lbm_substeps_per_fsi_step", self.lbm_substeps_per_fsi_step),
                     ("fluid_density_kg_m3", self.fluid_density_kg_m3),
                     ("fluid_kinematic_viscosity_m2_s", self.fluid_kinematic_viscosity_m2_s),
                     ("fluent_like_monitor_nearest_count", self.fluent_like_monitor_nearest_count),
                     ("beta_lbm", self.beta_lbm), ("penalty_force_cap_lbm", self.penalty_force_cap_lbm),
                     ("mb_reaction_scale", self.mb_reaction_scale), ("mb_force_cap_norm", self.mb_force_cap_norm),
                     ("link_area_scale_min", self.link_area_scale_min),
                     ("link_area_scale_max", self.link_area_scale_max), ("output_interval", self.output_interval),
                     ("lbm_min_tau_margin", self.lbm_min_tau_margin)]
        for name, value in positives:
            if value <= 0:
                raise ValueError(f"{name} must be positive")
        for name in ("target_inlet_velocity_mps", "official_fsi_dt_s", "target_u_lbm_for_dimensional_mapping",
                     "lbm_dt_phys_override_s", "target_reynolds_number", "fluent_like_monitor_radius_m"):
            v = getattr(self, name)
            if v is not None and float(v) <= 0.0:
                raise ValueError(f"{name} must be positive when provided")
        if self.link_area_scale_min > self.link_area_scale_max:
            raise ValueError("link_area_scale_min must be <= link_area_scale_max")
        if self.dynamic_solid_threshold < 0.0:
            raise ValueError("dynamic_solid_threshold must be non-negative")
        # fsi_config.py:184-200: prescribed boundary motion and the wall velocity application
        if self.boundary_motion_mode == "static" and self.boundary_motion_config_path is not None:
            raise ValueError("boundary_motion_config_path must be None when boundary_motion_mode='static'")
        if self.boundary_motion_mode == "prescribed_kinematic" and not self.boundary_motion_config_path:
            raise ValueError("boundary_motion_config_path is required when boundary_motion_mode='prescribed_kinematic'")
        if self.wall_velocity_application_mode == "disabled" and self.wall_velocity_application_config_path is not None:
            raise ValueError("wall_velocity_application_config_path must be None when "
                             "wall_velocity_application_mode='disabled'")
        if self.wall_velocity_application_mode == "solid_vel_experimental":
            if self.boundary_motion_mode != "prescribed_kinematic":
                raise ValueError("wall_velocity_application_mode='solid_vel_experimental' requires "
                                 "boundary_motion_mode='prescribed_kinematic'")
            if not self.wall_velocity_application_config_path:
                raise ValueError("wall_velocity_application_config_path is required when "
                                 "wall_velocity_application_mode='solid_vel_experimental'")
            if not Path(self.wall_velocity_application_config_path).is_file():
                raise ValueError("wall_velocity_application_config_path must exist when "
                                 "wall_velocity_application_mode='solid_vel_experimental'")
        # the geometry-motion application (a host-side mask schedule) is out of this package's scope
        if self.geometry_motion_application_mode != "disabled":
            raise ValueError("geometry-motion application is not supported by this backend")
        self._validate_fsi_exchange_mapping()
        mapping = self.lbm_viscosity_mapping_report()
        if not math.isfinite(float(mapping["tau"])) or float(mapping["tau"]) <= 0.5:
            raise ValueError("LBM viscosity mapping must produce finite tau > 0.5")
        if self.lbm_tau_stability_policy == "strict" and not bool(mapping["tau_margin_pass"]):
            raise ValueError("LBM tau stability margin failed strict policy")

    # fsi_config.py:334-374
    def _validate_fsi_exchange_mapping(self):
        if self.fsi_exchange_mode == "one_lbm_step_per_fsi_step":
            if self.lbm_substeps_per_fsi_step != 1:
                raise ValueError("lbm_substeps_per_fsi_step must be 1 when fsi_exchange_mode='one_lbm_step_per_fsi_step'")
            if self.lbm_dt_phys_override_s is not None:
                raise ValueError("lbm_dt_phys_override_s requires fsi_exchange_mode='lbm_subcycled_per_fsi_step'")
            return
        if self.coupling_mode != "moving_boundary":
            raise ValueError("lbm_subcycled_per_fsi_step currently requires coupling_mode='moving_boundary'")
        missing = [n for n in ("target_inlet_velocity_mps", "official_fsi_dt_s", "target_u_lbm_for_dimensional_mapping",
                               "lbm_dt_phys_override_s") if getattr(self, n) is None]
        if missing:
            raise ValueError("subcycled FSI exchange requires: " + ", ".join(missing))
        expected = float(self.lbm_substeps_per_fsi_step) * float(self.lbm_dt_phys_override_s)
        if not math.isclose(float(self.official_fsi_dt_s), expected, rel_tol=1.0e-12, abs_tol=1.0e-15):
            raise ValueError("official_fsi_dt_s must equal lbm_substeps_per_fsi_step * lbm_dt_phys_override_s")
        if not math.isclose(float(self.target_u_lbm[0]), float(self.target_u_lbm_for_dimensional_mapping),
                            rel_tol=1.0e-12, abs_tol=1.0e-15):
            raise ValueError("target_u_lbm[0] must equal target_u_lbm_for_dimensional_mapping")
        dx_phys = float(self.physical_duct_length_m) / float(self.n_grid)
        mapped = float(self.target_u_lbm_for_dimensional_mapping) * dx_phys / float(self.lbm_dt_phys_override_s)
        if not math.isclose(mapped, float(self.target_inlet_velocity_mps), rel_tol=1.0e-12, abs_tol=1.0e-9):
            raise ValueError("dimensional mapping does not recover target_inlet_velocity_mps")

    # fsi_config.py:376-445
    def lbm_viscosity_mapping_report(self) -> dict:
        if self.lbm_viscosity_semantics == "legacy_external":
            niu = 0.1
            tau = tau_from_legacy_external_solver_parameter(niu)
            return {"lbm_viscosity_semantics": self.lbm_viscosity_semantics, "physical_mapping_used": False,
                    "lbm_niu": niu, "nu_lbm": None, "tau": tau, "tau_minus_half": tau - 0.5,
                    "tau_margin_pass": (tau - 0.5) >= float(self.lbm_min_tau_margin),
                    "lbm_relaxation_semantics": LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER}
        dx = float(self.physical_duct_length_m) / float(self.n_grid)
        dt = float(self.lbm_dt_phys_override_s if self.lbm_dt_phys_override_s is not None
                   else self.mpm_substeps_per_lbm_step * self.mpm_dt)
        nu = float(self.fluid_kinematic_viscosity_m2_s) * dt / (dx * dx)
        tau = tau_from_lattice_kinematic_viscosity(nu)
        return {"lbm_viscosity_semantics": self.lbm_viscosity_semantics, "physical_mapping_used": True,
                "dx_phys_m": dx, "dt_phys_s": dt, "nu_lbm": nu, "lbm_niu": nu, "tau": tau,
                "tau_minus_half": tau - 0.5, "tau_margin_pass": (tau - 0.5) >= float(self.lbm_min_tau_margin),
                "lbm_relaxation_semantics": STANDARD_LATTICE_KINEMATIC_VISCOSITY}

    @classmethod
    def from_json(cls, path):
        with open(path, "r", encoding="utf-8") as f:
            return cls(**json.load(f))

    def to_dict(self):
        d = asdict(self)
        for k in ("target_u_lbm", "initial_solid_velocity_norm", "gravity", "box_min", "box_max",
                  "fluent_like_monitor_physical_point_m"):
            d[k] = list(d[k])
        return d

    def make_unified_sim_config(self):
        m = self.lbm_viscosity_mapping_report()
        return UnifiedSimConfig(n_grid=self.n_grid, mpm_dt=self.mpm_dt,
                                mpm_substeps_per_lbm_step=self.mpm_substeps_per_lbm_step,
                                lbm_dt_phys_override_s=self.lbm_dt_phys_override_s, lbm_niu=float(m["lbm_niu"]),
                                lbm_rho0=1.0, lbm_relaxation_semantics=str(m["lbm_relaxation_semantics"]),
                                lbm_open_boundary_semantics=self.lbm_open_boundary_semantics,
                                open_boundary_limiter_enabled=bool(self.open_boundary_limiter_enabled),
                                open_boundary_rho_min=float(self.open_boundary_rho_min),
                                open_boundary_rho_max=float(self.open_boundary_rho_max),
                                open_boundary_u_max=float(self.open_boundary_u_max),
                                open_boundary_noneq_cap=float(self.open_boundary_noneq_cap),
                                open_boundary_population_floor=self.open_boundary_population_floor)

    def make_mpm_control_overrides(self):
        return {"mpm_damping_application": self.mpm_damping_application,
                "mpm_planar_constraint_axis": self.mpm_planar_constraint_axis,
                "mpm_planar_constraint_mode": self.mpm_planar_constraint_mode,
                "mpm_velocity_damping": float(self.mpm_velocity_damping)}

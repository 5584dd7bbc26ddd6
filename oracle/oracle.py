"""Python front of the CPU oracle (``fsi_oracle.cpp``).

TEST INFRASTRUCTURE ONLY.  These classes drive the C++ restatement of the
reference kernels in the reference's call order and keep state in the
reference's AoS numpy layouts, so that parity tests can compare them field by
field with the CUDA product.  Only ``tests/``, ``__graft_entry__.smoke`` and
the CPU-baseline leg of ``bench.py`` import this module.

Reference anchors (lizhuoh9/MPM-LBM):
  LBMFluid3D              src/mpm_lbm/sim/lbm/fluid.py:32-2112
  MPMSolid3D              src/mpm_lbm/sim/mpm/solid.py:11-375
  MPMToLBMProjector3D     src/mpm_lbm/sim/coupling/projection.py:5-111
  PenaltyFSICoupler3D     src/mpm_lbm/sim/coupling/penalty.py:5-152
  MovingBoundaryFSICoupler3D  src/mpm_lbm/sim/coupling/moving_boundary.py:5-130
  LinkAreaMovingBoundaryCoupler3D src/mpm_lbm/sim/coupling/link_area.py:10-221
  FSIDriver3D.step_once   src/mpm_lbm/sim/drivers/fsi_driver.py:425-575
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libfsi_oracle.so")
SRC_PATH = os.path.join(HERE, "fsi_oracle.cpp")

_lock = threading.Lock()
_lib = None

OB_CODES = {
    "equilibrium_all_population_reset": 0,
    "regularized_velocity_pressure": 1,
    "regularized_velocity_pressure_limited": 2,
    "convective_pressure_outlet_experimental": 3,
    "regularized_mass_balanced_pressure_outlet": 4,
    "convective_mass_balanced_pressure_outlet": 5,
    "regularized_flux_matched_pressure_outlet": 6,
    "convective_flux_matched_damped_outlet": 7,
    "regularized_plane_flux_controlled_pressure_outlet": 8,
    "convective_plane_flux_controlled_damped_outlet": 9,
}
# LBMConfig defaults of the outlet repair and flux controller (lbm/config.py:53-69)
FLUX_CONTROL_DEFAULTS = {
    "open_boundary_flux_feedback_gain_u": 0.01,
    "open_boundary_flux_feedback_gain_rho": 0.005,
    "open_boundary_flux_filter_alpha": 0.05,
    "open_boundary_flux_correction_cap_u": 0.005,
    "open_boundary_flux_feedback_delta_cap_u": 0.0,
    "open_boundary_flux_feedback_slew_alpha": 1.0,
    "open_boundary_convective_blend_weight": 0.05,
    "open_boundary_flux_control_measure_plane_offset": 0,
    "open_boundary_flux_control_target_scale": 1.0,
    "open_boundary_outlet_flux_drop_guard_enabled": False,
    "open_boundary_outlet_flux_drop_guard_min_ratio": 0.60,
    "open_boundary_mass_neutral_flux_control_enabled": False,
    "open_boundary_mass_neutral_flux_control_mode": "disabled",
    "open_boundary_mass_neutral_mass_error_gain": 0.0,
    "open_boundary_mass_neutral_mass_error_cap": 0.0,
    "open_boundary_mass_neutral_correction_blend": 0.0,
}

# moment matrix of the reference (src/mpm_lbm/sim/lbm/fluid.py:231-249)
M_MATRIX = np.array(
    [
        [1] * 19,
        [-1, 0, 0, 0, 0, 0, 0] + [1] * 12,
        [1, -2, -2, -2, -2, -2, -2] + [1] * 12,
        [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
        [0, -2, 2, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
        [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1],
        [0, 0, 0, -2, 2, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1],
        [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1],
        [0, 0, 0, 0, 0, -2, 2, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1],
        [0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
        [0, -2, -2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
        [0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
        [0, 0, 0, -1, -1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
        [0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0],
        [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1],
        [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0],
        [0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0],
        [0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
        [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1],
    ],
    dtype=np.float64,
)
E = np.array(
    [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [-1, -1, 0],
     [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1],
     [0, -1, 1]],
    dtype=np.int32,
)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float64)


class LbmParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("ob_semantics", ctypes.c_int32),
        ("rho0", ctypes.c_double), ("force", ctypes.c_double * 3), ("S", ctypes.c_double * 19),
        ("inv_M", ctypes.c_double * 361), ("bc", ctypes.c_int32 * 6), ("rho_bc", ctypes.c_double * 6),
        ("vel_bc", (ctypes.c_double * 3) * 6), ("limiter_enabled", ctypes.c_int32), ("floor_enabled", ctypes.c_int32),
        ("ob_rho_min", ctypes.c_double), ("ob_rho_max", ctypes.c_double), ("ob_u_max", ctypes.c_double),
        ("ob_noneq_cap", ctypes.c_double), ("ob_floor", ctypes.c_double),
        ("flux_gain_u", ctypes.c_double), ("flux_gain_rho", ctypes.c_double), ("flux_filter_alpha", ctypes.c_double),
        ("flux_cap_u", ctypes.c_double), ("flux_delta_cap_u", ctypes.c_double), ("flux_slew_alpha", ctypes.c_double),
        ("convective_blend", ctypes.c_double), ("flux_target_scale", ctypes.c_double),
        ("drop_guard_min_ratio", ctypes.c_double), ("mn_gain", ctypes.c_double), ("mn_cap", ctypes.c_double),
        ("mn_blend", ctypes.c_double), ("measure_plane_offset", ctypes.c_int32),
        ("drop_guard_enabled", ctypes.c_int32), ("mass_neutral", ctypes.c_int32), ("pad_ob", ctypes.c_int32),
    ]


class LbmDiag(ctypes.Structure):
    _fields_ = [
        ("bb_link_count", ctypes.c_int32), ("pad0", ctypes.c_int32), ("bb_max_correction", ctypes.c_double),
        ("bb_net_fluid_impulse", ctypes.c_double * 3), ("bb_net_solid_force", ctypes.c_double * 3),
        ("bb_link_count_by_dir", ctypes.c_int32 * 19), ("pad1", ctypes.c_int32),
        ("bb_fluid_impulse_by_dir", (ctypes.c_double * 3) * 19), ("bb_solid_force_by_dir", (ctypes.c_double * 3) * 19),
        ("bb_correction_abs_sum_by_dir", ctypes.c_double * 19), ("bb_correction_abs_max_by_dir", ctypes.c_double * 19),
        ("mb_sample_count", ctypes.c_int32), ("pad2", ctypes.c_int32), ("mb_accum_norm_max", ctypes.c_double),
        ("mb_mean_norm_max", ctypes.c_double), ("ob_rho_clip", ctypes.c_int32 * 2),
        ("ob_velocity_clip", ctypes.c_int32 * 2), ("ob_noneq_clip", ctypes.c_int32 * 2),
        ("ob_floor_count", ctypes.c_int32 * 2), ("ob_reconstructed", ctypes.c_int32 * 2),
        ("mb_corr_count", ctypes.c_int32 * 2), ("mb_corr_abs_sum", ctypes.c_double * 2),
        ("pop_delta_abs_sum", ctypes.c_double * 2), ("flow_delta_abs_sum", ctypes.c_double * 2),
        ("flow_err_filtered_run", ctypes.c_double), ("flow_gain_effective_step", ctypes.c_double),
        ("target_flux", ctypes.c_double), ("measured_flux", ctypes.c_double), ("fluid_area", ctypes.c_double),
        ("true_outlet_flux", ctypes.c_double), ("near_flux", ctypes.c_double * 3),
        ("flux_err_filtered", ctypes.c_double), ("u_feedback", ctypes.c_double), ("rho_feedback", ctypes.c_double),
        ("guard_reference", ctypes.c_double), ("guard_active_step", ctypes.c_int32),
        ("guard_count_run", ctypes.c_int32), ("ctl_update", ctypes.c_int32 * 2),
        ("ctl_saturation", ctypes.c_int32 * 2), ("mn_mass_current", ctypes.c_double),
        ("mn_reference", ctypes.c_double), ("mn_error", ctypes.c_double), ("mn_rho_feedback", ctypes.c_double),
        ("mn_initialized", ctypes.c_int32), ("mn_update", ctypes.c_int32 * 2),
        ("mn_saturation", ctypes.c_int32 * 2), ("pad_mn", ctypes.c_int32),
    ]


class MpmParams(ctypes.Structure):
    _fields_ = [
        ("n_grid", ctypes.c_int32), ("n_particles", ctypes.c_int32), ("bound", ctypes.c_int32),
        ("damping_enabled", ctypes.c_int32), ("lock_z", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("dx", ctypes.c_double), ("inv_dx", ctypes.c_double), ("dt", ctypes.c_double), ("mu", ctypes.c_double),
        ("la", ctypes.c_double), ("gravity", ctypes.c_double * 3), ("damping", ctypes.c_double),
    ]


class MpmStats(ctypes.Structure):
    _fields_ = [
        ("min_x", ctypes.c_double * 3), ("max_x", ctypes.c_double * 3), ("max_speed", ctypes.c_double),
        ("min_J", ctypes.c_double), ("max_J", ctypes.c_double), ("total_mass", ctypes.c_double),
    ]


class CouplingParams(ctypes.Structure):
    _fields_ = [
        ("n_grid", ctypes.c_int32), ("pad", ctypes.c_int32), ("inv_dx_norm", ctypes.c_double),
        ("cell_volume_norm", ctypes.c_double), ("vel_scale", ctypes.c_double), ("eps_mass", ctypes.c_double),
        ("phi_min", ctypes.c_double), ("beta_lbm", ctypes.c_double), ("force_cap", ctypes.c_double),
        ("reaction_scale", ctypes.c_double), ("force_density_scale", ctypes.c_double), ("area_scale", ctypes.c_double),
    ]


class CouplingStats(ctypes.Structure):
    _fields_ = [
        ("projected_mass", ctypes.c_double), ("projected_volume_raw", ctypes.c_double),
        ("projected_volume_clamped", ctypes.c_double), ("max_phi_raw", ctypes.c_double),
        ("active_cell_count", ctypes.c_int32), ("active_force_cell_count", ctypes.c_int32),
        ("max_cell_force_norm", ctypes.c_double), ("max_hydro_force_norm", ctypes.c_double),
        ("net_cell_force", ctypes.c_double * 3), ("net_hydro_force", ctypes.c_double * 3),
        ("max_reaction_grid_force_norm", ctypes.c_double), ("net_reaction_grid_force", ctypes.c_double * 3),
        ("active_reaction_particle_count", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("max_particle_reaction_norm", ctypes.c_double), ("max_grid_reaction_norm", ctypes.c_double),
        ("net_particle_reaction_force", ctypes.c_double * 3), ("net_grid_reaction_force", ctypes.c_double * 3),
    ]


def build(force: bool = False) -> str:
    """Compile the oracle shared library (g++ -O2 -fopenmp)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(SRC_PATH):
        return LIB_PATH
    tmp = LIB_PATH + f".tmp{os.getpid()}"
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", "-o", tmp, SRC_PATH]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            _lib = ctypes.CDLL(build())
        return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _fn(prefix, name):
    return getattr(lib(), f"orc{prefix}_{name}")


def tau_from_config(niu: float, relaxation_semantics: str) -> float:
    """fluid.py:295-300 with relaxation_semantics.py:14-19."""
    if relaxation_semantics == "standard_lattice_kinematic_viscosity":
        return 3.0 * float(niu) + 0.5
    if relaxation_semantics == "legacy_external_solver_relaxation_parameter":
        return float(niu) / 3.0 + 0.5
    raise ValueError(f"unsupported LBM relaxation semantics: {relaxation_semantics}")


def relaxation_rates(tau: float, collision: str = "mrt") -> np.ndarray:
    """S_dig of fluid.py:301-304; 'bgk' relaxes every non-conserved moment at 1/tau."""
    s_v = 1.0 / tau
    s_o = 8.0 * (2.0 - s_v) / (8.0 - s_v)
    if collision == "bgk":
        s_o = s_v
    return np.array([0, s_v, s_v, 0, s_o, 0, s_o, 0, s_o, s_v, s_v, s_v, s_v, s_v, s_v, s_v, s_o, s_o, s_o],
                    dtype=np.float64)


class OracleLBM:
    """Numpy-state mirror of LBMFluid3D driven by the C++ restatement."""

    def __init__(self, nx, ny, nz, niu=0.1, rho0=1.0,
                 relaxation_semantics="legacy_external_solver_relaxation_parameter",
                 open_boundary_semantics="equilibrium_all_population_reset", bc=(0, 0, 0, 0, 0, 0),
                 rho_bc=(1.0,) * 6, vel_bc=((0.0, 0.0, 0.0),) * 6, force=(0.0, 0.0, 0.0),
                 limiter_enabled=False, ob_rho_min=0.8, ob_rho_max=1.2, ob_u_max=0.1, ob_noneq_cap=0.05,
                 ob_floor=None, collision="mrt", dtype=np.float32, flux_control=None):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dtype = np.dtype(dtype)
        self.pfx = "32" if self.dtype == np.float32 else "64"
        self.rho0 = float(rho0)
        self.niu = niu
        self.relaxation_semantics = relaxation_semantics
        self.collision = collision
        p = LbmParams()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.ob_semantics = OB_CODES[open_boundary_semantics]
        p.rho0 = self.rho0
        p.force[:] = [float(v) for v in force]
        inv_m = np.linalg.inv(M_MATRIX)
        p.inv_M[:] = [float(v) for v in inv_m.reshape(-1)]
        p.bc[:] = [int(v) for v in bc]
        p.rho_bc[:] = [float(v) for v in rho_bc]
        for i in range(6):
            p.vel_bc[i][:] = [float(v) for v in vel_bc[i]]
        p.limiter_enabled = int(bool(limiter_enabled))
        p.floor_enabled = int(ob_floor is not None)
        p.ob_rho_min, p.ob_rho_max, p.ob_u_max, p.ob_noneq_cap = ob_rho_min, ob_rho_max, ob_u_max, ob_noneq_cap
        p.ob_floor = float(ob_floor) if ob_floor is not None else -1.0e30
        fc = dict(FLUX_CONTROL_DEFAULTS)
        fc.update(flux_control or {})
        self.flux_control = fc
        p.flux_gain_u = fc["open_boundary_flux_feedback_gain_u"]
        p.flux_gain_rho = fc["open_boundary_flux_feedback_gain_rho"]
        p.flux_filter_alpha = fc["open_boundary_flux_filter_alpha"]
        p.flux_cap_u = fc["open_boundary_flux_correction_cap_u"]
        p.flux_delta_cap_u = fc["open_boundary_flux_feedback_delta_cap_u"]
        p.flux_slew_alpha = fc["open_boundary_flux_feedback_slew_alpha"]
        p.convective_blend = fc["open_boundary_convective_blend_weight"]
        p.flux_target_scale = fc["open_boundary_flux_control_target_scale"]
        p.drop_guard_min_ratio = fc["open_boundary_outlet_flux_drop_guard_min_ratio"]
        p.mn_gain = fc["open_boundary_mass_neutral_mass_error_gain"]
        p.mn_cap = fc["open_boundary_mass_neutral_mass_error_cap"]
        p.mn_blend = fc["open_boundary_mass_neutral_correction_blend"]
        p.measure_plane_offset = int(fc["open_boundary_flux_control_measure_plane_offset"])
        p.drop_guard_enabled = int(bool(fc["open_boundary_outlet_flux_drop_guard_enabled"]))
        p.mass_neutral = int(bool(fc["open_boundary_mass_neutral_flux_control_enabled"])
                             and fc["open_boundary_mass_neutral_flux_control_mode"]
                             == "global_mass_error_density_offset")
        self.p = p
        self.diag = LbmDiag()
        shp = (self.nx, self.ny, self.nz)
        z = lambda *extra: np.zeros(shp + extra, dtype=self.dtype)  # noqa: E731
        self.f, self.F = z(19), z(19)
        self.rho, self.v = z(), z(3)
        self.solid = np.zeros(shp, np.int8)
        self.static_solid = np.zeros(shp, np.int8)
        self.old_solid = np.zeros(shp, np.int8)
        self.reinit_flag = np.zeros(shp, np.int8)
        self.solid_phi, self.solid_mass = z(), z()
        self.solid_vel, self.cell_force = z(3), z(3)
        self.hydro_force, self.hydro_force_accum = z(3), z(3)
        self.threads = 1

    # fluid.py:347-353 (array form of init_geo)
    def init_geo_array(self, solid):
        s = (np.asarray(solid) > 0).astype(np.int8)
        self.solid[...] = s
        self.static_solid[...] = s
        self.old_solid[...] = s

    def init_simulation(self):
        tau = tau_from_config(self.niu, self.relaxation_semantics)
        self.tau = tau
        self.p.S[:] = [float(v) for v in relaxation_rates(tau, self.collision)]
        _fn(self.pfx, "lbm_init")(ctypes.byref(self.p), _ptr(self.f), _ptr(self.F), _ptr(self.rho), _ptr(self.v))

    def set_force(self, force):
        self.p.force[:] = [float(v) for v in force]

    def set_bc_vel_x0(self, vel):
        self.p.bc[0] = 2
        self.p.vel_bc[0][:] = [float(v) for v in vel]

    def colission(self):
        _fn(self.pfx, "lbm_collide")(ctypes.byref(self.p), _ptr(self.F), _ptr(self.rho), _ptr(self.v),
                                     _ptr(self.cell_force), _ptr(self.solid), _ptr(self.f), self.threads)

    def streaming1(self):
        _fn(self.pfx, "lbm_stream")(ctypes.byref(self.p), 0, _ptr(self.f), _ptr(self.F), _ptr(self.solid),
                                    _ptr(self.rho), _ptr(self.solid_vel), _ptr(self.hydro_force),
                                    ctypes.byref(self.diag), self.threads)

    def streaming_moving_bounceback(self):
        _fn(self.pfx, "lbm_stream")(ctypes.byref(self.p), 1, _ptr(self.f), _ptr(self.F), _ptr(self.solid),
                                    _ptr(self.rho), _ptr(self.solid_vel), _ptr(self.hydro_force),
                                    ctypes.byref(self.diag), self.threads)

    def Boundary_condition(self):
        _fn(self.pfx, "lbm_boundary")(ctypes.byref(self.p), _ptr(self.F), _ptr(self.rho), _ptr(self.v),
                                      _ptr(self.solid), ctypes.byref(self.diag))

    def update_open_boundary_plane_flux_controller(self):
        _fn(self.pfx, "lbm_plane_flux_controller")(ctypes.byref(self.p), _ptr(self.rho), _ptr(self.v),
                                                   _ptr(self.solid), ctypes.byref(self.diag))

    def streaming3(self):
        _fn(self.pfx, "lbm_macros")(ctypes.byref(self.p), _ptr(self.f), _ptr(self.F), _ptr(self.rho),
                                    _ptr(self.v), _ptr(self.solid), _ptr(self.cell_force), self.threads)

    def step(self):  # fluid.py:2099-2103
        self.colission()
        self.streaming1()
        self.Boundary_condition()
        self.streaming3()

    def step_moving_bounceback(self):  # fluid.py:2105-2111
        self.colission()
        self.streaming_moving_bounceback()
        self.Boundary_condition()
        self.streaming3()

    def update_dynamic_solid(self, threshold):
        _fn(self.pfx, "lbm_update_dynamic_solid")(ctypes.byref(self.p), ctypes.c_double(threshold),
                                                  _ptr(self.solid), _ptr(self.static_solid), _ptr(self.old_solid),
                                                  _ptr(self.solid_phi), _ptr(self.reinit_flag))

    def reinitialize_new_fluid_cells(self):
        _fn(self.pfx, "lbm_reinit")(ctypes.byref(self.p), _ptr(self.reinit_flag), _ptr(self.solid_vel),
                                    _ptr(self.rho), _ptr(self.v), _ptr(self.f), _ptr(self.F))

    def _accum(self, op):
        _fn(self.pfx, "lbm_force_accumulator")(ctypes.byref(self.p), op, _ptr(self.hydro_force),
                                               _ptr(self.hydro_force_accum), ctypes.byref(self.diag))

    def clear_moving_boundary_force_accumulator(self):
        self._accum(0)

    def accumulate_moving_boundary_force_sample(self):
        self._accum(1)

    def finalize_moving_boundary_force_accumulator(self):
        self._accum(2)

    # fluid.py:1931-1968
    def get_stats(self):
        fluid = self.solid == 0
        if not np.any(fluid):
            return {"max_v": 0.0, "rho_min": float("nan"), "rho_max": float("nan"), "mass_total": 0.0,
                    "force_norm_max": 0.0}
        vel_norm = np.linalg.norm(self.v[fluid], axis=1)
        force_norm = np.linalg.norm(self.cell_force[fluid], axis=1)
        rho_fluid = self.rho[fluid]
        return {"max_v": float(np.max(vel_norm)), "rho_min": float(np.min(rho_fluid)),
                "rho_max": float(np.max(rho_fluid)), "mass_total": float(np.sum(rho_fluid)),
                "force_norm_max": float(np.max(force_norm))}

    def get_moving_boundary_stats(self):
        d = self.diag
        return {"bb_link_count": int(d.bb_link_count), "bb_max_correction": float(d.bb_max_correction),
                "bb_net_fluid_impulse": tuple(d.bb_net_fluid_impulse), "bb_net_solid_force": tuple(d.bb_net_solid_force)}

    def get_moving_boundary_directional_stats(self):
        d = self.diag
        return {
            "link_count_by_dir": np.array(d.bb_link_count_by_dir[:], dtype=np.int32),
            "fluid_impulse_by_dir": np.array([list(r) for r in d.bb_fluid_impulse_by_dir], dtype=np.float64),
            "solid_force_by_dir": np.array([list(r) for r in d.bb_solid_force_by_dir], dtype=np.float64),
            "correction_abs_sum_by_dir": np.array(d.bb_correction_abs_sum_by_dir[:], dtype=np.float64),
            "correction_abs_max_by_dir": np.array(d.bb_correction_abs_max_by_dir[:], dtype=np.float64),
        }

    def get_moving_boundary_accumulation_stats(self):
        d = self.diag
        return {"mb_subcycle_force_sample_count": int(d.mb_sample_count),
                "mb_subcycle_force_accum_norm_max": float(d.mb_accum_norm_max),
                "mb_subcycle_force_mean_norm_max": float(d.mb_mean_norm_max)}

    def get_open_boundary_limiter_stats(self):
        d = self.diag
        return {"rho_clip_count_step": d.ob_rho_clip[0], "rho_clip_count_run": d.ob_rho_clip[1],
                "velocity_clip_count_step": d.ob_velocity_clip[0], "velocity_clip_count_run": d.ob_velocity_clip[1],
                "noneq_clip_count_step": d.ob_noneq_clip[0], "noneq_clip_count_run": d.ob_noneq_clip[1],
                "population_floor_count_step": d.ob_floor_count[0], "population_floor_count_run": d.ob_floor_count[1],
                "reconstructed_population_count_step": d.ob_reconstructed[0],
                "reconstructed_population_count_run": d.ob_reconstructed[1],
                "mass_balance_correction_count_step": d.mb_corr_count[0],
                "mass_balance_correction_count_run": d.mb_corr_count[1],
                "mass_balance_correction_abs_sum_step": d.mb_corr_abs_sum[0],
                "mass_balance_correction_abs_sum_run": d.mb_corr_abs_sum[1],
                "unknown_population_delta_abs_sum_step": d.pop_delta_abs_sum[0],
                "unknown_population_delta_abs_sum_run": d.pop_delta_abs_sum[1],
                "flow_correction_delta_abs_sum_step": d.flow_delta_abs_sum[0],
                "flow_correction_delta_abs_sum_run": d.flow_delta_abs_sum[1],
                "flow_outlet_flux_error_filtered_run": d.flow_err_filtered_run,
                "flow_correction_gain_effective_step": d.flow_gain_effective_step,
                "mass_neutral_mass_current": d.mn_mass_current,
                "mass_neutral_mass_initial_reference": d.mn_reference,
                "mass_neutral_mass_error": d.mn_error,
                "mass_neutral_rho_feedback": d.mn_rho_feedback,
                "mass_neutral_feedback_saturation_count_step": d.mn_saturation[0],
                "mass_neutral_feedback_saturation_count_run": d.mn_saturation[1],
                "mass_neutral_feedback_update_count_step": d.mn_update[0],
                "mass_neutral_feedback_update_count_run": d.mn_update[1],
                "near_outlet_flux_xminus1": d.near_flux[0],
                "near_outlet_flux_xminus2": d.near_flux[1],
                "near_outlet_flux_xminus3": d.near_flux[2],
                "controller_true_outlet_flux_for_guard": d.true_outlet_flux,
                "controller_target_outlet_flux": d.target_flux,
                "controller_measured_outlet_flux": d.measured_flux,
                "controller_raw_flux_error": d.target_flux - d.measured_flux,
                "controller_filtered_flux_error": d.flux_err_filtered,
                "controller_outlet_fluid_area": d.fluid_area,
                "controller_u_feedback": d.u_feedback,
                "controller_density_feedback": d.rho_feedback,
                "controller_saturation_count_step": d.ctl_saturation[0],
                "controller_saturation_count_run": d.ctl_saturation[1],
                "controller_update_count_step": d.ctl_update[0],
                "controller_update_count_run": d.ctl_update[1],
                "controller_drop_guard_active_step": d.guard_active_step,
                "controller_drop_guard_activation_count_run": d.guard_count_run,
                "controller_drop_guard_reference_flux": d.guard_reference}


class OracleMPM:
    """Numpy-state mirror of MPMSolid3D (mpm/solid.py:11-375)."""

    def __init__(self, n_grid, dx, dt, n_particles, gravity=(0.0, -9.8, 0.0), p_rho=1.0, young_modulus=400.0,
                 poisson_ratio=0.2, bound=3, box_min=(0.25, 0.35, 0.25), box_max=(0.55, 0.65, 0.55),
                 lock_z=False, damping=0.0, dtype=np.float32):
        if n_particles <= 0:
            raise ValueError("n_particles must be positive")
        self.dtype = np.dtype(dtype)
        self.pfx = "32" if self.dtype == np.float32 else "64"
        self.n_grid, self.n_particles = int(n_grid), int(n_particles)
        self.dx, self.inv_dx, self.dt = float(dx), 1.0 / float(dx), float(dt)
        self.box_min, self.box_max = tuple(box_min), tuple(box_max)
        self.mu = young_modulus / (2.0 * (1.0 + poisson_ratio))
        self.la = young_modulus * poisson_ratio / ((1.0 + poisson_ratio) * (1.0 - 2.0 * poisson_ratio))
        box_volume = np.prod([b - a for a, b in zip(box_min, box_max)])
        self.p_vol0 = float(box_volume) / float(n_particles)
        self.p_mass0 = self.p_vol0 * p_rho
        self.particles_per_axis = max(1, math.ceil(n_particles ** (1.0 / 3.0)))
        p = MpmParams()
        p.n_grid, p.n_particles, p.bound = self.n_grid, self.n_particles, int(bound)
        p.damping_enabled = int(damping > 0.0)
        p.lock_z = int(bool(lock_z))
        p.dx, p.inv_dx, p.dt, p.mu, p.la = self.dx, self.inv_dx, self.dt, self.mu, self.la
        p.gravity[:] = [float(g) for g in gravity]
        p.damping = float(damping)
        self.p = p
        n, g = self.n_particles, self.n_grid
        dt_ = self.dtype
        self.x, self.v = np.zeros((n, 3), dt_), np.zeros((n, 3), dt_)
        self.C, self.F = np.zeros((n, 3, 3), dt_), np.zeros((n, 3, 3), dt_)
        self.Jp, self.mass, self.vol0 = np.zeros(n, dt_), np.zeros(n, dt_), np.zeros(n, dt_)
        self.fixed_mask = np.zeros(n, np.int8)
        self.fixed_x = np.zeros((n, 3), dt_)
        self.grid_v, self.grid_m = np.zeros((g, g, g, 3), dt_), np.zeros((g, g, g), dt_)
        self.grid_f_ext = np.zeros((g, g, g, 3), dt_)

    # solid.py:126-159
    def init_box(self):
        ppa = self.particles_per_axis
        f = self.dtype.type
        p = np.arange(self.n_particles)
        idx = np.stack([p % ppa, (p // ppa) % ppa, (p // (ppa * ppa)) % ppa], axis=1)
        denom = max(1, ppa - 1)
        local = (idx.astype(self.dtype) + f(0.5)) / f(denom + 1)
        bmin = np.array(self.box_min, dtype=self.dtype)
        span = np.array([b - a for a, b in zip(self.box_min, self.box_max)], dtype=self.dtype)
        self.x[...] = bmin + span * local
        self.v[...] = 0
        self.C[...] = 0
        self.F[...] = np.eye(3, dtype=self.dtype)
        self.Jp[...] = 1
        self.mass[...] = self.p_mass0
        self.vol0[...] = self.p_vol0
        self.fixed_mask[...] = 0
        self.fixed_x[...] = self.x

    # solid.py:168-210 (validation restated in the product; the oracle trusts its inputs)
    def init_from_numpy(self, x_np, vol0_np, mass_np, v_np=None, fixed_mask_np=None):
        self.x[...] = np.asarray(x_np, dtype=self.dtype)
        self.v[...] = 0 if v_np is None else np.asarray(v_np, dtype=self.dtype)
        self.vol0[...] = np.asarray(vol0_np, dtype=self.dtype)
        self.mass[...] = np.asarray(mass_np, dtype=self.dtype)
        self.fixed_x[...] = self.x
        self.fixed_mask[...] = 0 if fixed_mask_np is None else np.asarray(fixed_mask_np, dtype=np.int8)
        self.C[...] = 0
        self.F[...] = np.eye(3, dtype=self.dtype)
        self.Jp[...] = 1
        self._apply_fixed()

    def _apply_fixed(self):  # solid.py:331-339
        m = self.fixed_mask != 0
        self.x[m] = self.fixed_x[m]
        self.v[m] = 0
        self.C[m] = 0
        self.F[m] = np.eye(3, dtype=self.dtype)
        self.Jp[m] = 1

    def set_uniform_velocity(self, vx, vy, vz):  # solid.py:323-329
        self.v[...] = np.array([vx, vy, vz], dtype=self.dtype)
        self.v[self.fixed_mask != 0] = 0

    def clear_grid(self):
        self.grid_v[...] = 0
        self.grid_m[...] = 0
        self.grid_f_ext[...] = 0

    def p2g(self):
        _fn(self.pfx, "mpm_p2g")(ctypes.byref(self.p), _ptr(self.x), _ptr(self.v), _ptr(self.C), _ptr(self.F),
                                 _ptr(self.Jp), _ptr(self.mass), _ptr(self.vol0), _ptr(self.grid_v),
                                 _ptr(self.grid_m))

    def grid_update(self):
        _fn(self.pfx, "mpm_grid_update")(ctypes.byref(self.p), _ptr(self.grid_v), _ptr(self.grid_m),
                                         _ptr(self.grid_f_ext))

    def g2p(self):
        _fn(self.pfx, "mpm_g2p")(ctypes.byref(self.p), _ptr(self.x), _ptr(self.v), _ptr(self.C), _ptr(self.F),
                                 _ptr(self.Jp), _ptr(self.fixed_mask), _ptr(self.fixed_x), _ptr(self.grid_v))

    def substep(self):
        self.clear_grid()
        self.p2g()
        self.grid_update()
        self.g2p()

    def get_stats(self):
        st = MpmStats()
        _fn(self.pfx, "mpm_stats")(ctypes.byref(self.p), _ptr(self.x), _ptr(self.v), _ptr(self.Jp),
                                   _ptr(self.mass), ctypes.byref(st))
        return {"min_x": tuple(st.min_x), "max_x": tuple(st.max_x), "min_y": st.min_x[1], "max_y": st.max_x[1],
                "max_speed": st.max_speed, "min_J": st.min_J, "max_J": st.max_J, "total_mass": st.total_mass}


class OracleCoupling:
    """Projection + penalty + moving-boundary + link-area couplers (coupling/*.py)."""

    def __init__(self, n_grid, dx_norm, lbm_dt_phys, beta_lbm=1.0e-3, penalty_force_cap=1.0e-4, phi_min=1.0e-6,
                 reaction_scale=1.0, mb_force_cap_norm=1.0e-2, link_area_policy="inverse_length",
                 area_scale_min=0.25, area_scale_max=2.0):
        cp = CouplingParams()
        cp.n_grid = int(n_grid)
        cp.inv_dx_norm = 1.0 / dx_norm
        cp.cell_volume_norm = dx_norm ** 3
        cp.vel_scale = lbm_dt_phys / dx_norm
        cp.eps_mass = 1.0e-12
        cp.phi_min = phi_min
        cp.beta_lbm = beta_lbm
        cp.reaction_scale = reaction_scale
        cp.force_density_scale = dx_norm / (lbm_dt_phys ** 2)
        cp.area_scale = 1.0
        self.cp = cp
        self.penalty_force_cap = penalty_force_cap
        self.mb_force_cap_norm = mb_force_cap_norm
        self.link_area_policy = link_area_policy
        self.area_scale_min, self.area_scale_max = area_scale_min, area_scale_max
        self.stats = CouplingStats()

    def project(self, solid: OracleMPM, lbm: OracleLBM):
        _fn(lbm.pfx, "couple_project")(ctypes.byref(self.cp), ctypes.byref(lbm.p), solid.n_particles,
                                       _ptr(solid.x), _ptr(solid.v), _ptr(solid.Jp), _ptr(solid.vol0),
                                       _ptr(solid.mass), _ptr(lbm.solid_phi), _ptr(lbm.solid_mass),
                                       _ptr(lbm.solid_vel), ctypes.byref(self.stats))

    def build_penalty_force(self, lbm: OracleLBM):
        self.cp.force_cap = self.penalty_force_cap
        _fn(lbm.pfx, "couple_penalty_force")(ctypes.byref(self.cp), ctypes.byref(lbm.p), _ptr(lbm.solid),
                                             _ptr(lbm.solid_phi), _ptr(lbm.rho), _ptr(lbm.v), _ptr(lbm.solid_vel),
                                             _ptr(lbm.cell_force), _ptr(lbm.hydro_force), ctypes.byref(self.stats))

    def reaction(self, kind, solid: OracleMPM, lbm: OracleLBM):
        self.cp.force_cap = self.mb_force_cap_norm
        _fn(lbm.pfx, "couple_reaction")(kind, ctypes.byref(self.cp), ctypes.byref(lbm.p), solid.n_particles,
                                        _ptr(solid.x), _ptr(solid.Jp), _ptr(solid.vol0), _ptr(lbm.hydro_force),
                                        _ptr(lbm.solid_phi), _ptr(solid.grid_f_ext), ctypes.byref(self.stats))

    # coupling/link_area.py:84-108 with link_area_accounting.py:42-148
    def update_area_scale(self, lbm: OracleLBM):
        d = lbm.get_moving_boundary_directional_stats()
        lengths = np.linalg.norm(E.astype(np.float64), axis=1)
        weights = np.zeros(19)
        active = lengths > 0
        if self.link_area_policy == "uniform":
            weights[active] = 1.0
        elif self.link_area_policy == "inverse_length":
            weights[active] = 1.0 / lengths[active]
        else:
            weights[active] = lengths[active]
        weighted_solid = np.sum(d["solid_force_by_dir"] * weights[:, None], axis=0, dtype=np.float64)
        scalar_solid = np.asarray(lbm.get_moving_boundary_stats()["bb_net_solid_force"], dtype=np.float64)
        raw = abs(float(weighted_solid[0])) / (abs(float(scalar_solid[0])) + 1.0e-12)
        scale = float(np.clip(raw, self.area_scale_min, self.area_scale_max))
        if not np.isfinite(scale):
            scale = self.area_scale_min
        self.cp.area_scale = np.float32(scale) if lbm.dtype == np.float32 else scale
        self.raw_area_scale = raw
        return scale


class OracleFSIDriver:
    """FSIDriver3D.step_once phase order (fsi_driver.py:425-575) over the oracle objects."""

    def __init__(self, lbm: OracleLBM, solid: OracleMPM, coupling: OracleCoupling, coupling_mode="moving_boundary",
                 reaction_transfer_mode="engineering", fsi_exchange_mode="one_lbm_step_per_fsi_step",
                 lbm_substeps_per_fsi_step=1, mpm_substeps_per_lbm_step=10, dynamic_solid_threshold=0.5):
        self.lbm, self.solid, self.coupling = lbm, solid, coupling
        self.coupling_mode = coupling_mode
        self.reaction_transfer_mode = reaction_transfer_mode
        self.fsi_exchange_mode = fsi_exchange_mode
        self.S = int(lbm_substeps_per_fsi_step)
        self.M = int(mpm_substeps_per_lbm_step)
        self.thr = float(dynamic_solid_threshold)
        self.current_lbm_step = 0
        self.total_lbm_substeps = 0
        self.total_mpm_substeps = 0

    def step_once(self):
        lbm, solid, cpl = self.lbm, self.solid, self.coupling
        if self.fsi_exchange_mode == "lbm_subcycled_per_fsi_step":
            cpl.project(solid, lbm)
            lbm.clear_moving_boundary_force_accumulator()
            for _ in range(self.S):
                lbm.update_dynamic_solid(self.thr)
                lbm.reinitialize_new_fluid_cells()
                lbm.step_moving_bounceback()
                lbm.accumulate_moving_boundary_force_sample()
                self.total_lbm_substeps += 1
            lbm.finalize_moving_boundary_force_accumulator()
            self._advance_mpm_mb()
            self.current_lbm_step += 1
            return
        cpl.project(solid, lbm)
        if self.coupling_mode == "none":
            lbm.step()
            for _ in range(self.M):
                solid.substep()
                self.total_mpm_substeps += 1
        elif self.coupling_mode == "penalty":
            cpl.build_penalty_force(lbm)
            lbm.step()
            for _ in range(self.M):
                solid.clear_grid()
                solid.p2g()
                cpl.reaction(0, solid, lbm)
                solid.grid_update()
                solid.g2p()
                self.total_mpm_substeps += 1
        elif self.coupling_mode == "moving_boundary":
            lbm.update_dynamic_solid(self.thr)
            lbm.reinitialize_new_fluid_cells()
            lbm.step_moving_bounceback()
            self._advance_mpm_mb()
        else:
            raise ValueError(f"unsupported coupling_mode: {self.coupling_mode}")
        self.current_lbm_step += 1
        self.total_lbm_substeps += 1

    def _advance_mpm_mb(self):
        lbm, solid, cpl = self.lbm, self.solid, self.coupling
        kind = 1
        if self.reaction_transfer_mode == "link_area_experimental":
            cpl.update_area_scale(lbm)
            kind = 2
        for _ in range(self.M):
            solid.clear_grid()
            solid.p2g()
            cpl.reaction(kind, solid, lbm)
            solid.grid_update()
            solid.g2p()
            self.total_mpm_substeps += 1


def fsi_driver_for_case(case, dtype=np.float32, substeps=None, mpm_substeps=None, threads=1):
    """The oracle set up on a duct/plate case of ``mpm_lbm_b200.cases``: the
    same geometry, particles, material, unit mapping and open boundaries as
    ``case.make_driver()``, moving_boundary subcycled, engineering transfer.
    substeps / mpm_substeps override the case's S and M per FSI step."""
    cfg = case.config()
    solid, parts = case.geometry()
    sim = cfg.make_unified_sim_config()
    nx, ny, nz = case.lattice
    vel = ((case.u_in, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0), (0, 0, 0))
    lbm = OracleLBM(nx, ny, nz, niu=sim.lbm_niu, relaxation_semantics=sim.lbm_relaxation_semantics,
                    open_boundary_semantics=cfg.lbm_open_boundary_semantics, bc=(2, 1, 0, 0, 0, 0),
                    rho_bc=(1.0,) * 6, vel_bc=vel, limiter_enabled=cfg.open_boundary_limiter_enabled, dtype=dtype)
    lbm.threads = int(threads)
    lbm.init_geo_array(solid)
    lbm.init_simulation()
    mc = sim.make_mpm_config(gravity=cfg.gravity, **case.material())
    mpm = OracleMPM(nx, mc.dx, mc.dt, len(parts["x"]), gravity=mc.gravity, young_modulus=mc.young_modulus,
                    poisson_ratio=mc.poisson_ratio, p_rho=mc.p_rho, dtype=dtype)
    mpm.init_from_numpy(parts["x"], parts["vol0"], parts["mass"], fixed_mask_np=parts["fixed"])
    cpl = OracleCoupling(nx, sim.dx_norm, sim.lbm_dt_phys, mb_force_cap_norm=cfg.mb_force_cap_norm)
    S = case.lbm_substeps if substeps is None else int(substeps)
    M = case.mpm_substeps if mpm_substeps is None else int(mpm_substeps)
    return OracleFSIDriver(lbm, mpm, cpl, fsi_exchange_mode="lbm_subcycled_per_fsi_step",
                           lbm_substeps_per_fsi_step=S, mpm_substeps_per_lbm_step=M)


def fsi_driver_for_box_case(case, dtype=np.float32, threads=1):
    """The oracle set up on a box case of ``mpm_lbm_b200.batch.BoxCase``: the
    same walls, particles, material, unit mapping, body force and coupling
    mode as ``case.make_driver()``, one LBM step per FSI step."""
    cfg = case.config()
    solid, parts = case.geometry()
    sim = cfg.make_unified_sim_config()
    nx, ny, nz = case.lattice
    lbm = OracleLBM(nx, ny, nz, niu=sim.lbm_niu, relaxation_semantics=sim.lbm_relaxation_semantics, dtype=dtype)
    lbm.threads = int(threads)
    lbm.init_geo_array(solid)
    lbm.init_simulation()
    lbm.set_force(case.body_force)
    mc = sim.make_mpm_config(gravity=cfg.gravity, **case.material())
    mpm = OracleMPM(case.n_grid, mc.dx, mc.dt, len(parts["x"]), gravity=mc.gravity, young_modulus=mc.young_modulus,
                    poisson_ratio=mc.poisson_ratio, p_rho=mc.p_rho, dtype=dtype)
    mpm.init_from_numpy(parts["x"], parts["vol0"], parts["mass"], fixed_mask_np=parts["fixed"])
    cpl = OracleCoupling(case.n_grid, sim.dx_norm, sim.lbm_dt_phys, beta_lbm=cfg.beta_lbm,
                         penalty_force_cap=cfg.penalty_force_cap_lbm, mb_force_cap_norm=cfg.mb_force_cap_norm)
    return OracleFSIDriver(lbm, mpm, cpl, coupling_mode=case.mode,
                           mpm_substeps_per_lbm_step=case.mpm_substeps,
                           dynamic_solid_threshold=cfg.dynamic_solid_threshold)

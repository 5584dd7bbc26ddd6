"""LBMFluid3D: the reference's D3Q19 fluid object on B200 kernels.

Same constructor (LBMConfig), fields and methods as
src/mpm_lbm/sim/lbm/fluid.py:32-2112; state lives in device tensors and every
step runs through libfsi_b200.so.  Differences a caller can observe:
  * update_dynamic_solid() also performs reinitialize_new_fluid_cells() (the
    reference's driver always calls the two back to back, fsi_driver.py:
    523-524, 540-541); reinitialize_new_fluid_cells() is then a no-op.
  * set_force() takes effect for every later step (the reference's Taichi
    kernels capture the force at their first compilation, fluid.py:393-396).
  * only the x faces may carry open boundaries (the driver uses only those,
    fsi_driver.py:238-257); the population storage can be FP16 (extension).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import (FSI_CELL_OVERRIDE, FSI_CELL_SOLID, FSI_MODE_DIRSTATS, FSI_MODE_MOVING_BB, FSI_MODE_PENALTY,
                   FSI_MODE_SUBCYCLED, FsiLbmDiag, FsiLbmParams, FsiLbmState, FsiStepCtl, call, ptr, stream_handle)
from .config import (KERNEL_OPEN_BOUNDARY_CODES, LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER,
                     STANDARD_LATTICE_KINEMATIC_VISCOSITY, LBMConfig, tau_from_lattice_kinematic_viscosity,
                     tau_from_legacy_external_solver_parameter)
from .fields import CellField, ConstField, ScalarField, lattice_to_ref, ref_to_lattice

E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [-1, -1, 0],
              [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1],
              [0, 1, -1], [0, -1, 1]], dtype=np.int32)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32)
LR = [0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17]


def pop_blocks(t: torch.Tensor) -> torch.Tensor:
    """[19][pitch] populations in the device storage order (blocks of 32
    cells, each holding 19 runs of 32 values; FsiLbmState.pop)."""
    n = t.shape[1]
    return t.reshape(19, n // 32, 32).permute(1, 0, 2).reshape(19, n)


def relaxation_rates(tau: float, collision: str = "mrt"):
    """S_dig of fluid.py:301-304 as (s_v, s_o); BGK relaxes all non-conserved moments at 1/tau."""
    s_v = 1.0 / tau
    s_o = s_v if collision == "bgk" else 8.0 * (2.0 - s_v) / (8.0 - s_v)
    return s_v, s_o


class LBMFluid3D:
    def __init__(self, config: LBMConfig, device=None):
        if config.sparse_storage:
            raise NotImplementedError("Step 2 only supports dense storage. Enable sparse storage after FSI coupling "
                                      "is validated.")
        if any((config.bc_y_left, config.bc_y_right, config.bc_z_left, config.bc_z_right)):
            raise NotImplementedError("the B200 kernels implement open boundaries on the x faces only")
        if config.open_boundary_semantics not in KERNEL_OPEN_BOUNDARY_CODES:
            raise NotImplementedError(f"open_boundary_semantics={config.open_boundary_semantics!r} is not "
                                      "implemented by the B200 kernels")
        self.config = config
        self.enable_projection = True
        self.sparse_storage = False
        self.nx, self.ny, self.nz = int(config.nx), int(config.ny), int(config.nz)
        self.dims = (self.nx, self.ny, self.nz)
        self.fx, self.fy, self.fz = (float(v) for v in config.force)
        self.niu = config.niu
        self.rho0 = float(config.rho0)
        self.relaxation_semantics = config.relaxation_semantics
        self.open_boundary_semantics = config.open_boundary_semantics
        self.collision = config.collision
        self.bc_x_left, self.rho_bcxl = int(config.bc_x_left), float(config.rho_bc_x_left)
        self.vx_bcxl, self.vy_bcxl, self.vz_bcxl = (float(v) for v in config.vel_bc_x_left)
        self.bc_x_right, self.rho_bcxr = int(config.bc_x_right), float(config.rho_bc_x_right)
        self.vx_bcxr, self.vy_bcxr, self.vz_bcxr = (float(v) for v in config.vel_bc_x_right)
        self.fp16 = config.population_storage == "fp16"
        self.device = torch.device(device if device is not None else "cuda")
        n = self.nx * self.ny * self.nz
        self.ncell = n
        self.pitch = ((n + 127) // 128) * 128
        P, dev = self.pitch, self.device
        z32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)  # noqa: E731
        z8 = lambda *s: torch.zeros(*s, dtype=torch.uint8, device=dev)  # noqa: E731
        self.t_pop = torch.zeros(19, P, dtype=torch.float16 if self.fp16 else torch.float32, device=dev)
        self.t_flags = z8(P)
        self.t_nbr = torch.zeros(P, dtype=torch.int32, device=dev)
        self.t_rho = torch.full((P,), self.rho0, dtype=torch.float32, device=dev)
        self.t_vel = z32(3, P)
        self.t_static, self.t_old, self.t_reinit = z8(P), z8(P), z8(P)
        self.t_phi, self.t_smass, self.t_svel = z32(P), z32(P), z32(3, P)
        self.t_cf, self.t_hydro, self.t_accum = z32(3, P), z32(3, P), z32(3, P)
        self.t_hpp = z32(2, 3, P)
        self.t_plane = z32(5, 4, self.ny * self.nz)
        self.t_change = torch.zeros(P, dtype=torch.int32, device=dev)
        self.t_diag = torch.zeros((ctypes.sizeof(FsiLbmDiag) + 255) // 256 * 256, dtype=torch.uint8, device=dev)
        self.t_out_pop = None
        # inlet velocity read on the device every step (bc_vel_x_left_dynamic, fluid.py:287-288)
        self.t_vin = torch.tensor([self.vx_bcxl, self.vy_bcxl, self.vz_bcxl], dtype=torch.float32, device=dev)
        self.state = FsiLbmState(
            nx=self.nx, ny=self.ny, nz=self.nz, store_fp16=int(self.fp16), pitch=P, pop=ptr(self.t_pop),
            flags=ptr(self.t_flags), nbr=ptr(self.t_nbr), rho=ptr(self.t_rho), vel=ptr(self.t_vel),
            static_solid=ptr(self.t_static), old_solid=ptr(self.t_old), reinit_flag=ptr(self.t_reinit),
            phi=ptr(self.t_phi), smass=ptr(self.t_smass), svel=ptr(self.t_svel), cell_force=ptr(self.t_cf),
            hydro=ptr(self.t_hydro), hpp=ptr(self.t_hpp), accum=ptr(self.t_accum), plane=ptr(self.t_plane),
            change_list=ptr(self.t_change), diag=ptr(self.t_diag), vel_left_dyn=ptr(self.t_vin))
        self.params = FsiLbmParams()
        self._penalty = None
        self.parity = 0
        self.bc_pending = False
        self.pp = 0
        self.last_pp = 0
        self.steps = 0
        self._accumulating = False
        self._fused_accumulation = False
        self._sample_count = 0
        self._hydro_src = "hydro"
        self._version = 0
        self._readout_version = -1
        self._old_equals_solid = False
        self.dirstats_enabled = True
        self.tune = 0  # FSI_TUNE_LBM_* launch variant (mpm_lbm_b200.autotune picks it)
        self.tau_f = None
        self._sync_params()
        self._make_fields()

    # ------------------------------------------------------------ params
    def _sync_params(self):
        p = self.params
        p.rho0 = self.rho0
        p.force[:] = [self.fx, self.fy, self.fz]
        if self.tau_f is not None:
            p.s_v, p.s_o = relaxation_rates(self.tau_f, self.collision)
        else:
            p.s_v = p.s_o = 1.0
        p.bc_left, p.bc_right = self.bc_x_left, self.bc_x_right
        p.ob_semantics = KERNEL_OPEN_BOUNDARY_CODES[self.open_boundary_semantics]
        cfg = self.config
        p.limiter = int(bool(cfg.open_boundary_limiter_enabled))
        p.floor_enabled = int(cfg.open_boundary_population_floor is not None)
        p.rho_bc_left, p.rho_bc_right = self.rho_bcxl, self.rho_bcxr
        p.vel_bc_left[:] = [self.vx_bcxl, self.vy_bcxl, self.vz_bcxl]
        p.vel_bc_right[:] = [self.vx_bcxr, self.vy_bcxr, self.vz_bcxr]
        p.ob_rho_min, p.ob_rho_max = cfg.open_boundary_rho_min, cfg.open_boundary_rho_max
        p.ob_u_max, p.ob_noneq_cap = cfg.open_boundary_u_max, cfg.open_boundary_noneq_cap
        p.ob_floor = float(cfg.open_boundary_population_floor) if cfg.open_boundary_population_floor is not None else -1e30
        p.ob_gain_u, p.ob_gain_rho = cfg.open_boundary_flux_feedback_gain_u, cfg.open_boundary_flux_feedback_gain_rho
        p.ob_filter_alpha, p.ob_cap_u = cfg.open_boundary_flux_filter_alpha, cfg.open_boundary_flux_correction_cap_u
        p.ob_delta_cap_u = cfg.open_boundary_flux_feedback_delta_cap_u
        p.ob_slew_alpha = cfg.open_boundary_flux_feedback_slew_alpha
        p.ob_blend = cfg.open_boundary_convective_blend_weight
        p.ob_target_scale = cfg.open_boundary_flux_control_target_scale
        p.ob_guard_min_ratio = cfg.open_boundary_outlet_flux_drop_guard_min_ratio
        p.ob_mn_gain = cfg.open_boundary_mass_neutral_mass_error_gain
        p.ob_mn_cap = cfg.open_boundary_mass_neutral_mass_error_cap
        p.ob_mn_blend = cfg.open_boundary_mass_neutral_correction_blend
        p.ob_measure_offset = int(cfg.open_boundary_flux_control_measure_plane_offset)
        p.ob_guard = int(bool(cfg.open_boundary_outlet_flux_drop_guard_enabled))
        p.ob_mass_neutral = int(self._mass_neutral_active())
        if self._penalty is not None:
            p.penalty_beta, p.penalty_phi_min, p.penalty_cap = self._penalty
        p.tune = int(self.tune)

    def _ctl(self, mode=0, pp=None):
        return FsiStepCtl(parity=self.parity, bc_pending=int(self.bc_pending), pp=self.pp if pp is None else pp,
                          mode=mode)

    def _stream(self):
        return stream_handle()

    # ------------------------------------------------- state snapshots
    _SNAPSHOT = ("t_pop", "t_flags", "t_nbr", "t_rho", "t_vel", "t_old", "t_reinit", "t_cf", "t_hydro", "t_accum",
                 "t_hpp", "t_plane", "t_diag")
    _SNAPSHOT_ATTRS = ("parity", "bc_pending", "pp", "last_pp", "steps", "_accumulating", "_fused_accumulation",
                       "_sample_count", "_hydro_src", "_old_equals_solid", "_penalty", "dirstats_enabled")

    def snapshot(self):
        """Device copies of the mutable state (for trial steps, e.g. autotuning)."""
        return ({k: getattr(self, k).clone() for k in self._SNAPSHOT},
                {k: getattr(self, k) for k in self._SNAPSHOT_ATTRS})

    def restore(self, snap):
        tensors, attrs = snap
        for k, t in tensors.items():
            getattr(self, k).copy_(t)
        for k, v in attrs.items():
            setattr(self, k, v)
        self._sync_params()
        self._version += 1

    # ------------------------------------------------------------ fields
    def _make_fields(self):
        d = self.dims
        self.f = self.F = CellField(d, 19, np.float32, lambda: self._readout()[0], self._put_pop, "F")
        self.rho = CellField(d, 0, np.float32, lambda: self._readout()[1], self._put_rho, "rho")
        self.v = CellField(d, 3, np.float32, lambda: self._readout()[2], self._put_vel, "v")
        self.solid = CellField(d, 0, np.int8, lambda: (self.t_flags & FSI_CELL_SOLID), self._put_solid, "solid")
        self.static_solid = CellField(d, 0, np.int8, lambda: self.t_static, self._put_static, "static_solid")
        self.old_solid = CellField(d, 0, np.int8,
                                   lambda: (self.t_flags & FSI_CELL_SOLID) if self._old_equals_solid else self.t_old,
                                   None, "old_solid")
        self.reinit_flag = CellField(d, 0, np.int8, lambda: self.t_reinit, None, "reinit_flag")
        self.solid_phi = CellField(d, 0, np.float32, lambda: self.t_phi, self._putter(self.t_phi), "solid_phi")
        self.solid_mass = CellField(d, 0, np.float32, lambda: self.t_smass, self._putter(self.t_smass), "solid_mass")
        self.solid_vel = CellField(d, 3, np.float32, lambda: self.t_svel, self._putter(self.t_svel, 3), "solid_vel")
        self.cell_force = CellField(d, 3, np.float32, lambda: self.t_cf, None, "cell_force")
        self.hydro_force = CellField(d, 3, np.float32, self._hydro_tensor, self._put_hydro, "hydro_force")
        self.hydro_force_accum = CellField(d, 3, np.float32, self._accum_tensor, None, "hydro_force_accum")
        self.e = ConstField(E)
        self.e_f = ConstField(E.astype(np.float32))
        self.w = ConstField(W)
        self.LR = list(LR)
        self.S_dig = ScalarField(self._s_dig)
        dg = self._diag
        self.bb_link_count = ScalarField(lambda: int(sum(dg().link_count)))
        self.bb_max_correction = ScalarField(lambda: float(max(dg().corr_abs_max)))
        self.bb_net_fluid_impulse = ScalarField(lambda: self._dir_impulse().sum(axis=0).astype(np.float32))
        self.bb_net_solid_force = ScalarField(lambda: -self._dir_impulse().sum(axis=0).astype(np.float32))
        self.bb_link_count_by_dir = ScalarField(lambda: np.array(dg().link_count[:], np.int32), shape=(19,))
        self.mb_subcycle_force_sample_count = ScalarField(lambda: self._sample_count)

    def _putter(self, t, comps=0):
        def put(a):
            ref_to_lattice(a, self.dims, comps, t)
            self._version += 1
        return put

    def _s_dig(self):
        s_v, s_o = self.params.s_v, self.params.s_o
        return np.array([0, s_v, s_v, 0, s_o, 0, s_o, 0, s_o] + [s_v] * 7 + [s_o] * 3, dtype=np.float32)

    def _diag(self) -> FsiLbmDiag:
        raw = self.t_diag[: ctypes.sizeof(FsiLbmDiag)].cpu().numpy().tobytes()
        return FsiLbmDiag.from_buffer_copy(raw)

    def _dir_impulse(self):
        return np.array([list(r) for r in self._diag().fluid_impulse], dtype=np.float64)

    def _hydro_tensor(self):
        if self._hydro_src == "hydro":
            return self.t_hydro
        return self.t_hpp[self._hydro_src]

    def _accum_tensor(self):
        if self._fused_accumulation:
            return self.t_accum + self.t_hpp[self.last_pp]
        return self.t_accum

    def _readout(self):
        if self.t_out_pop is None:
            P = self.pitch
            self.t_out_pop = torch.empty(19, P, dtype=torch.float32, device=self.device)
            self.t_out_rho = torch.empty(P, dtype=torch.float32, device=self.device)
            self.t_out_vel = torch.empty(3, P, dtype=torch.float32, device=self.device)
        if self._readout_version != self._version:
            call("fsi_lbm_readout", ctypes.byref(self.state), ctypes.byref(self.params), ctypes.byref(self._ctl()),
                 ptr(self.t_out_pop), ptr(self.t_out_rho), ptr(self.t_out_vel), self._stream())
            self._readout_version = self._version
        return self.t_out_pop, self.t_out_rho, self.t_out_vel

    def _materialize_macros(self):
        """Store the current rho/v and mark every cell to collide with them."""
        pop, rho, vel = self._readout()
        self.t_rho.copy_(rho)
        self.t_vel.copy_(vel)
        self.t_flags.bitwise_or_(FSI_CELL_OVERRIDE)
        return pop

    def _to_natural(self):
        self.flush_open_boundary()
        if self.parity == 1:
            call("fsi_lbm_to_natural", ctypes.byref(self.state), self._stream())
            self.parity = 0
            self._version += 1

    def _put_pop(self, arr):
        self._materialize_macros()
        self._to_natural()
        t = torch.empty(19, self.pitch, dtype=torch.float32, device=self.device)
        ref_to_lattice(arr, self.dims, 19, t)
        if self.fp16:
            w = torch.as_tensor(W, device=self.device)[:, None]
            t = t / w - self.rho0
        self.t_pop.copy_(pop_blocks(t).to(self.t_pop.dtype))
        self._version += 1

    def _put_rho(self, arr):
        self._materialize_macros()
        ref_to_lattice(arr, self.dims, 0, self.t_rho)
        self._version += 1

    def _put_vel(self, arr):
        self._materialize_macros()
        ref_to_lattice(arr, self.dims, 3, self.t_vel)
        self._version += 1

    def _put_solid(self, arr):
        s = (np.asarray(arr) > 0).astype(np.uint8)
        self._set_solid(s, keep_static=True)

    def _put_static(self, arr):
        """static_solid.from_numpy (a restart load, restart.py:76): the mask the
        dynamic solid update starts from; the current solid mask is unchanged."""
        ref_to_lattice((np.asarray(arr) > 0).astype(np.uint8), self.dims, 0, self.t_static)
        self._version += 1

    def _put_hydro(self, arr):
        ref_to_lattice(arr, self.dims, 3, self._hydro_tensor())
        self._version += 1

    # ------------------------------------------------------- geometry/init
    def _set_solid(self, solid_ref: np.ndarray, keep_static=False):
        self._to_natural()
        t = torch.zeros(self.pitch, dtype=torch.uint8, device=self.device)
        ref_to_lattice(solid_ref.astype(np.uint8), self.dims, 0, t)
        static_before = self.t_static.clone() if keep_static else None
        call("fsi_lbm_set_solid", ctypes.byref(self.state), ptr(t), self._stream())
        if keep_static:
            self.t_static.copy_(static_before)
        self._version += 1

    def init_geo(self, filename):
        """fluid.py:347-353: Fortran-ordered 0/1 .dat file -> solid, static_solid, old_solid."""
        in_dat = np.loadtxt(filename)
        in_dat[in_dat > 0] = 1
        self.init_geo_array(np.reshape(in_dat, self.dims, order="F"))

    def init_geo_array(self, solid):
        self._set_solid((np.asarray(solid) > 0).astype(np.uint8))

    def init_simulation(self):
        """fluid.py:285-317: relaxation rates + equilibrium at rest."""
        if self.relaxation_semantics == STANDARD_LATTICE_KINEMATIC_VISCOSITY:
            self.tau_f = tau_from_lattice_kinematic_viscosity(self.niu)
        elif self.relaxation_semantics == LEGACY_EXTERNAL_SOLVER_RELAXATION_PARAMETER:
            self.tau_f = tau_from_legacy_external_solver_parameter(self.niu)
        else:
            raise ValueError(f"unsupported LBM relaxation semantics: {self.relaxation_semantics}")
        self.s_v, self.s_other = relaxation_rates(self.tau_f, self.collision)
        self._sync_params()
        call("fsi_lbm_init_equilibrium", ctypes.byref(self.state), ctypes.byref(self.params), self._stream())
        self.parity = 0
        self.bc_pending = False
        self._version += 1

    def set_force(self, force):
        self.fx, self.fy, self.fz = (float(v) for v in force)
        self._sync_params()
        self._version += 1

    def set_viscosity(self, niu):
        self.niu = niu

    def set_bc_vel_x0(self, vel):
        self.bc_x_left = 2
        self.vx_bcxl, self.vy_bcxl, self.vz_bcxl = (float(v) for v in vel)
        self.t_vin.copy_(torch.tensor([self.vx_bcxl, self.vy_bcxl, self.vz_bcxl], dtype=torch.float32))
        self._sync_params()

    def set_inlet_velocity_async(self, vel_host):
        """Stream-ordered update of the x-min inlet velocity from a (pinned) host
        tensor of 3 floats; steps captured in a CUDA graph read the new value."""
        self.t_vin.copy_(vel_host, non_blocking=True)

    def set_bc_vel_x1(self, vel):
        self.bc_x_right = 2
        self.vx_bcxr, self.vy_bcxr, self.vz_bcxr = (float(v) for v in vel)
        self._sync_params()

    def set_bc_rho_x0(self, rho):
        self.bc_x_left = 1
        self.rho_bcxl = float(rho)
        self._sync_params()

    def set_bc_rho_x1(self, rho):
        self.bc_x_right = 1
        self.rho_bcxr = float(rho)
        self._sync_params()

    # --------------------------------------------------------------- steps
    def _substep(self, mode):
        if self.tau_f is None:
            raise RuntimeError("init_simulation() must run before stepping")
        if self._penalty is not None:
            mode |= FSI_MODE_PENALTY
        self._sync_params()
        ctl = self._ctl(mode)
        call("fsi_lbm_substep", ctypes.byref(self.state), ctypes.byref(self.params), ctypes.byref(ctl),
             self._stream())
        self.last_pp = self.pp
        self.pp ^= 1
        self.parity ^= 1
        self.bc_pending = bool(self.bc_x_left or self.bc_x_right)
        self.steps += 1
        self._version += 1
        self._penalty = None
        if mode & FSI_MODE_MOVING_BB:
            self._hydro_src = self.last_pp
        elif mode & FSI_MODE_PENALTY:
            self._hydro_src = "hydro"
        return mode

    def step(self):
        """colission -> streaming1 -> Boundary_condition -> streaming3 (fluid.py:2099-2103)."""
        self._substep(0)

    def step_moving_bounceback(self):
        """fluid.py:2105-2111, with the moving-wall link forces."""
        mode = FSI_MODE_MOVING_BB
        if self.dirstats_enabled:
            mode |= FSI_MODE_DIRSTATS
        if self._accumulating:
            mode |= FSI_MODE_SUBCYCLED
        self._fused_accumulation = bool(mode & FSI_MODE_SUBCYCLED)
        self._substep(mode)

    def flush_open_boundary(self):
        if self.bc_pending:
            call("fsi_lbm_flush_bc", ctypes.byref(self.state), ctypes.byref(self.params),
                 ctypes.byref(self._ctl()), self._stream())
            self.bc_pending = False
            self._version += 1

    def update_dynamic_solid(self, threshold):
        """fluid.py:1847-1861 followed by reinitialize_new_fluid_cells (1863-1877)."""
        self.flush_open_boundary()
        call("fsi_mask_rebuild", ctypes.byref(self.state), ctypes.byref(self.params), ctypes.byref(self._ctl()),
             ctypes.c_float(threshold), self._stream())
        self._old_equals_solid = False
        self._version += 1

    def reinitialize_new_fluid_cells(self):
        """Performed inside update_dynamic_solid (see module docstring)."""
        return None

    def mark_repeat_mask_update(self):
        """A second update_dynamic_solid with unchanged solid_phi is a no-op except
        that old_solid becomes equal to solid (fluid.py:1851)."""
        self._old_equals_solid = True

    # -------------------------------------------------- force accumulator
    def clear_moving_boundary_force_accumulator(self):
        self.t_accum.zero_()
        off = FsiLbmDiag.accum_norm_max.offset
        self.t_diag[off: off + 8].zero_()  # accum_norm_max, mean_norm_max
        self._sample_count = 0
        self._accumulating = True
        self._fused_accumulation = False
        self._version += 1

    def accumulate_moving_boundary_force_sample(self):
        """fluid.py:468-473.  After a fused subcycled step the sample is already
        folded on the device; otherwise the current hydro_force is added here."""
        self._sample_count += 1
        if not self._fused_accumulation:
            self.t_accum.add_(self._hydro_tensor())
            nrm = torch.linalg.vector_norm(self.t_accum[:, : self.ncell], dim=0).max()
            off = FsiLbmDiag.accum_norm_max.offset
            cur = torch.frombuffer(bytearray(self._diag_bytes(off, 4)), dtype=torch.float32)[0]
            val = torch.maximum(nrm.cpu(), cur)
            self.t_diag[off: off + 4].copy_(torch.tensor([float(val)], dtype=torch.float32).view(torch.uint8))
        self._version += 1

    def _diag_bytes(self, off, n):
        return self.t_diag[off: off + n].cpu().numpy().tobytes()

    def finalize_moving_boundary_force_accumulator(self):
        # after fused subcycled steps the last substep's link forces still sit in
        # the ping-pong slot of the last step and are folded here
        ctl = self._ctl(mode=FSI_MODE_SUBCYCLED if self._fused_accumulation else 0, pp=self.last_pp)
        call("fsi_force_accum_finalize", ctypes.byref(self.state), ctypes.byref(ctl),
             ctypes.c_int32(self._sample_count), self._stream())
        self._accumulating = False
        self._fused_accumulation = False
        self._hydro_src = "hydro"
        self._version += 1

    # -------------------------------------------------------- diagnostics
    def fluid_mask(self):
        return (self.t_flags[: self.ncell] & FSI_CELL_SOLID) == 0

    def get_stats(self):
        """fluid.py:1931-1968 (reductions on the device, FP64)."""
        _, rho, vel = self._readout()
        fluid = self.fluid_mask()
        if not bool(fluid.any()):
            return {"max_v": 0.0, "rho_min": float("nan"), "rho_max": float("nan"), "mass_total": 0.0,
                    "force_norm_max": 0.0}
        r = rho[: self.ncell][fluid].double()
        vn = torch.linalg.vector_norm(vel[:, : self.ncell][:, fluid].double(), dim=0)
        fn = torch.linalg.vector_norm(self.t_cf[:, : self.ncell][:, fluid].double(), dim=0)
        vals = torch.stack([vn.max(), r.min(), r.max(), r.sum(), fn.max()]).cpu().tolist()
        return {"max_v": vals[0], "rho_min": vals[1], "rho_max": vals[2], "mass_total": vals[3],
                "force_norm_max": vals[4]}

    def get_max_v(self):
        return self.get_stats()["max_v"]

    def get_moving_boundary_stats(self):
        d = self._diag()
        imp = np.array([list(r) for r in d.fluid_impulse], dtype=np.float32).sum(axis=0)
        return {"bb_link_count": int(sum(d.link_count)), "bb_max_correction": float(max(d.corr_abs_max)),
                "bb_net_fluid_impulse": tuple(float(v) for v in imp),
                "bb_net_solid_force": tuple(float(-v) for v in imp)}

    def get_moving_boundary_directional_stats(self):
        d = self._diag()
        imp = np.array([list(r) for r in d.fluid_impulse], dtype=np.float32)
        return {"link_count_by_dir": np.array(d.link_count[:], dtype=np.int32), "fluid_impulse_by_dir": imp,
                "solid_force_by_dir": -imp, "correction_abs_sum_by_dir": np.array(d.corr_abs_sum[:], np.float32),
                "correction_abs_max_by_dir": np.array(d.corr_abs_max[:], np.float32)}

    def get_moving_boundary_accumulation_stats(self):
        d = self._diag()
        return {"mb_subcycle_force_sample_count": int(self._sample_count),
                "mb_subcycle_force_accum_norm_max": float(d.accum_norm_max),
                "mb_subcycle_force_mean_norm_max": float(d.mean_norm_max)}

    def _mass_neutral_active(self) -> bool:
        cfg = self.config
        return bool(cfg.open_boundary_mass_neutral_flux_control_enabled
                    and cfg.open_boundary_mass_neutral_flux_control_mode == "global_mass_error_density_offset")

    def get_open_boundary_limiter_stats(self):
        """fluid.py:804-924 with the same keys.  Applies a pending open-boundary step first."""
        self.flush_open_boundary()
        d = self._diag()
        cfg = self.config
        st, run = list(d.ob_step), list(d.ob_run)
        names = ["rho_clip_count", "velocity_clip_count", "noneq_clip_count", "population_floor_count",
                 "reconstructed_population_count"]
        out = {}
        for i, nm in enumerate(names):
            out[nm + "_step"] = int(st[i])
            out[nm + "_run"] = int(run[i])
        out["limiter_activation_count_step"] = sum(st[:4])
        out["limiter_activation_count"] = sum(run[:4])
        out["limiter_activation_denominator"] = int(run[4])
        out["limiter_activation_fraction"] = float(sum(run[:4]) / run[4]) if run[4] else 0.0
        updates, saturations = int(d.pc_update_run), int(d.pc_sat_run)
        mn_updates, mn_saturations = int(d.mn_update_run), int(d.mn_sat_run)
        u_fb, rho_fb, mn_fb = float(d.pc_u_fb), float(d.pc_rho_fb), float(d.mn_rho_fb)
        cap = abs(float(cfg.open_boundary_flux_correction_cap_u))
        out.update({
            "mass_balance_correction_count_step": int(d.obr_count_step),
            "mass_balance_correction_count_run": int(d.obr_count_run),
            "mass_balance_correction_abs_sum_step": float(d.obr_corr_step),
            "mass_balance_correction_abs_sum_run": float(d.obr_corr_run),
            "unknown_population_delta_abs_sum_step": float(d.obr_delta_step),
            "unknown_population_delta_abs_sum_run": float(d.obr_delta_run),
            "flow_correction_delta_abs_sum_step": float(d.obf_delta_step),
            "flow_correction_delta_abs_sum_run": float(d.obf_delta_run),
            "flow_outlet_flux_error_filtered_run": float(d.obf_err_filtered_run),
            "flow_correction_gain_effective_step": float(d.obf_gain_step),
            "flow_feedback_gain_u": float(cfg.open_boundary_flux_feedback_gain_u),
            "flow_feedback_gain_rho": float(cfg.open_boundary_flux_feedback_gain_rho),
            "flow_filter_alpha": float(cfg.open_boundary_flux_filter_alpha),
            "flow_correction_cap_u": float(cfg.open_boundary_flux_correction_cap_u),
            "flow_feedback_delta_cap_u": float(cfg.open_boundary_flux_feedback_delta_cap_u),
            "flow_feedback_slew_alpha": float(cfg.open_boundary_flux_feedback_slew_alpha),
            "flow_convective_blend_weight": float(cfg.open_boundary_convective_blend_weight),
            "flow_control_measure_plane_offset": int(cfg.open_boundary_flux_control_measure_plane_offset),
            "flow_control_target_scale": float(cfg.open_boundary_flux_control_target_scale),
            "flow_outlet_flux_drop_guard_enabled": bool(cfg.open_boundary_outlet_flux_drop_guard_enabled),
            "flow_outlet_flux_drop_guard_min_ratio": float(cfg.open_boundary_outlet_flux_drop_guard_min_ratio),
            "mass_neutral_flux_control_enabled": bool(cfg.open_boundary_mass_neutral_flux_control_enabled),
            "mass_neutral_flux_control_mode": cfg.open_boundary_mass_neutral_flux_control_mode,
            "mass_neutral_mass_error_gain": float(cfg.open_boundary_mass_neutral_mass_error_gain),
            "mass_neutral_mass_error_cap": float(cfg.open_boundary_mass_neutral_mass_error_cap),
            "mass_neutral_correction_blend": float(cfg.open_boundary_mass_neutral_correction_blend),
            "mass_neutral_reference_mass_mode": cfg.open_boundary_mass_neutral_reference_mass_mode,
            "mass_neutral_projection_report_only": bool(
                cfg.open_boundary_mass_neutral_flux_control_mode == "outlet_population_projection_report_only"),
            "mass_neutral_runtime_behavior_active": self._mass_neutral_active(),
            "mass_neutral_mass_current": float(d.mn_mass),
            "mass_neutral_mass_initial_reference": float(d.mn_reference),
            "mass_neutral_mass_error": float(d.mn_error),
            "mass_neutral_rho_feedback": mn_fb,
            "mass_neutral_rho_feedback_abs": abs(mn_fb),
            "mass_neutral_feedback_saturation_count_step": int(d.mn_sat_step),
            "mass_neutral_feedback_saturation_count_run": mn_saturations,
            "mass_neutral_feedback_update_count_step": int(d.mn_update_step),
            "mass_neutral_feedback_update_count_run": mn_updates,
            "mass_neutral_feedback_saturation_fraction_run": float(mn_saturations / mn_updates if mn_updates else 0.0),
            "near_outlet_flux_xminus1": float(d.pc_near[0]),
            "near_outlet_flux_xminus2": float(d.pc_near[1]),
            "near_outlet_flux_xminus3": float(d.pc_near[2]),
            "controller_true_outlet_flux_for_guard": float(d.pc_true_outlet),
            "controller_target_outlet_flux": float(d.pc_target),
            "controller_measured_outlet_flux": float(d.pc_measured),
            "controller_raw_flux_error": float(d.pc_target) - float(d.pc_measured),
            "controller_filtered_flux_error": float(d.pc_err_filtered),
            "controller_outlet_fluid_area": float(d.pc_area),
            "controller_u_feedback": u_fb,
            "controller_u_feedback_abs": abs(u_fb),
            "controller_density_feedback": rho_fb,
            "controller_density_feedback_abs": abs(rho_fb),
            "controller_delta_cap_u": float(cfg.open_boundary_flux_feedback_delta_cap_u),
            "controller_slew_alpha": float(cfg.open_boundary_flux_feedback_slew_alpha),
            "controller_authority_ratio": float(abs(u_fb) / cap if cap else 0.0),
            "controller_saturation_count_step": int(d.pc_sat_step),
            "controller_saturation_count_run": saturations,
            "controller_update_count_step": int(d.pc_update_step),
            "controller_update_count_run": updates,
            "controller_saturation_fraction_run": float(saturations / updates if updates else 0.0),
            "controller_measure_plane_offset": int(cfg.open_boundary_flux_control_measure_plane_offset),
            "controller_target_scale": float(cfg.open_boundary_flux_control_target_scale),
            "controller_drop_guard_active_step": int(d.pc_guard_step),
            "controller_drop_guard_activation_count_run": int(d.pc_guard_run),
            "controller_drop_guard_reference_flux": float(d.pc_guard_ref),
            "controller_drop_guard_min_ratio": float(cfg.open_boundary_outlet_flux_drop_guard_min_ratio),
            "controller_drop_guard_activation_fraction_run": float(int(d.pc_guard_run) / updates if updates else 0.0),
        })
        return out

    # open-boundary counter and controller state of FsiLbmDiag (fluid.py:571-736)
    _OB_REPAIR_FIELDS = ("obr_count_step", "obr_corr_step", "obr_delta_step", "obf_delta_step", "obf_gain_step",
                         "obr_count_run", "obr_corr_run", "obr_delta_run", "obf_delta_run", "obf_err_filtered_run")
    _OB_CONTROLLER_FIELDS = ("pc_acc", "pc_target", "pc_measured", "pc_area", "pc_true_outlet", "pc_near",
                             "pc_err_filtered", "pc_u_fb", "pc_rho_fb", "pc_guard_ref", "pc_guard_step",
                             "pc_guard_run", "pc_update_step", "pc_update_run", "pc_sat_step", "pc_sat_run",
                             "mn_mass", "mn_reference", "mn_error", "mn_rho_fb", "mn_initialized", "mn_update_step",
                             "mn_update_run", "mn_sat_step", "mn_sat_run")

    def _diag_set(self, values: dict):
        """Write FsiLbmDiag fields (stream-ordered with the kernels)."""
        d = FsiLbmDiag()
        for name, value in values.items():
            setattr(d, name, value)
        raw = bytes(d)
        for name in values:
            f = getattr(FsiLbmDiag, name)
            src = torch.frombuffer(bytearray(raw[f.offset: f.offset + f.size]), dtype=torch.uint8)
            self.t_diag[f.offset: f.offset + f.size].copy_(src)

    def _diag_zero(self, names):
        for name in names:
            f = getattr(FsiLbmDiag, name)
            self.t_diag[f.offset: f.offset + f.size].zero_()

    def clear_open_boundary_limiter_run_counters(self):
        """fluid.py:589-636: every limiter, repair and controller counter and state to zero."""
        self.flush_open_boundary()
        self._diag_zero(("ob_step", "ob_run") + self._OB_REPAIR_FIELDS + self._OB_CONTROLLER_FIELDS)

    def set_open_boundary_limiter_run_counters(self, rho_clip_count, velocity_clip_count, noneq_clip_count,
                                               population_floor_count, reconstructed_population_count):
        """fluid.py:638-691 (restart of the limiter counters)."""
        self.flush_open_boundary()
        self._diag_zero(self._OB_REPAIR_FIELDS + self._OB_CONTROLLER_FIELDS)
        counts = [int(rho_clip_count), int(velocity_clip_count), int(noneq_clip_count), int(population_floor_count),
                  int(reconstructed_population_count)]
        self._diag_set({"ob_step": (ctypes.c_int32 * 5)(), "ob_run": (ctypes.c_int32 * 5)(*counts)})

    def set_open_boundary_repair_run_counters(self, mass_balance_correction_count, mass_balance_correction_abs_sum,
                                              unknown_population_delta_abs_sum):
        """fluid.py:693-736 (restart of the repair counters)."""
        self.flush_open_boundary()
        self._diag_zero(self._OB_REPAIR_FIELDS + self._OB_CONTROLLER_FIELDS)
        self._diag_set({"obr_count_run": int(mass_balance_correction_count),
                        "obr_corr_run": float(mass_balance_correction_abs_sum),
                        "obr_delta_run": float(unknown_population_delta_abs_sum)})

    def update_open_boundary_plane_flux_controller(self):
        """fluid.py:1141-1263 called on its own, from the current rho, v and
        solid fields (the step runs it by itself under semantics 8 and 9)."""
        self.flush_open_boundary()
        _, rho, vel = self._readout()
        call("fsi_ob_controller_update", ctypes.byref(self.state), ctypes.byref(self.params), ptr(rho), ptr(vel),
             self._stream())

    def get_lightweight_stability_stats(self):
        """fluid.py:738-802 on the device."""
        pop, rho, vel = self._readout()
        fluid = self.fluid_mask()
        n = self.ncell
        f = pop[:, :n][:, fluid]
        r = rho[:n][fluid].double()
        vn = torch.linalg.vector_norm(vel[:, :n][:, fluid].double(), dim=0)
        neg = int((f < 0).sum().item()) * 2
        entries = int(fluid.sum().item()) * 19 * 2
        x = torch.arange(n, device=self.device) % self.nx
        xm = x[fluid]
        negmask = (f < 0).any(dim=0)
        return {"rho_min": float(r.min()), "rho_max": float(r.max()), "max_v": float(vn.max()),
                "mass_total": float(r.sum()), "fluid_cell_count": int(fluid.sum()), "f_min": float(f.min()),
                "f_max": float(f.max()), "F_min": float(f.min()), "F_max": float(f.max()),
                "negative_population_count": neg,
                "negative_population_fraction": float(neg / entries) if entries else 0.0,
                "population_entry_count": entries,
                "boundary_x_min_negative_population_count": int(((f < 0) & (xm == 0)[None]).sum()) * 2,
                "boundary_x_max_negative_population_count": int(((f < 0) & (xm == self.nx - 1)[None]).sum()) * 2,
                "stability_all_finite": bool(torch.isfinite(f).all()) and bool(negmask is not None)}

    def export_VTK(self, n, out_prefix="./LBMFluid"):
        """Headless export: one .npz per call instead of VTK (no pyevtk dependency)."""
        np.savez_compressed(f"{out_prefix}_{n}.npz", rho=self.rho.to_numpy(), velocity=self.v.to_numpy(),
                            solid=self.solid.to_numpy(), solid_phi=self.solid_phi.to_numpy(),
                            hydro_force=self.hydro_force.to_numpy(), cell_force=self.cell_force.to_numpy())

"""ctypes binding of libfsi_b200.so (include/fsi_b200.h).

The library must have been built in-tree (``python -m mpm_lbm_b200.build``);
loading fails loudly otherwise -- there is no fallback implementation.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfsi_b200.so")
# FSI_ABI_VERSION of include/fsi_b200.h.  2: populations stored in blocks of 32
# cells, FsiLbmDiag with the FP64 mass-neutral sum, fsi_project_ordered.
ABI_VERSION = 2

c_i32, c_i64, c_f32, c_f64, c_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p

FSI_CELL_SOLID, FSI_CELL_NEAR, FSI_CELL_LINK, FSI_CELL_OVERRIDE, FSI_CELL_CF = 1, 2, 4, 8, 16
FSI_MODE_MOVING_BB, FSI_MODE_SUBCYCLED, FSI_MODE_DIRSTATS, FSI_MODE_PENALTY = 1, 2, 4, 8
FSI_TUNE_LBM_OCC3, FSI_TUNE_LBM_OCC4, FSI_TUNE_LBM_PAIR, FSI_TUNE_LBM_OCC3_PF, FSI_TUNE_LBM_OCC4_PF = 0, 1, 2, 3, 4


FSI_CAMPAIGN_REGIONS = 8
FSI_BIN_CHUNK, FSI_BIN_EDGE = 128, 8  # particles per chunk of a bin, bin edge in cells


class FsiCampaignSums(ctypes.Structure):
    _fields_ = [("fluid_mass", ctypes.c_double), ("region_flux", ctypes.c_double * FSI_CAMPAIGN_REGIONS),
                ("fluid_cells", c_i32), ("nonfinite_rho", c_i32), ("nonfinite_vel", c_i32), ("nonfinite_pop", c_i32)]


class FsiLbmDiag(ctypes.Structure):
    _fields_ = [
        ("link_count", c_i32 * 19), ("corr_abs_sum", c_f32 * 19), ("corr_abs_max", c_f32 * 19),
        ("fluid_impulse", (c_f32 * 3) * 19), ("accum_norm_max", c_f32), ("mean_norm_max", c_f32),
        ("ob_step", c_i32 * 5), ("ob_run", c_i32 * 5), ("penalty_active", c_i32), ("penalty_max_norm", c_f32),
        ("penalty_net", c_f32 * 3), ("change_count", c_i32), ("status", c_i32), ("pad", c_i32 * 2),
        ("obr_count_step", c_i32), ("obr_corr_step", c_f32), ("obr_delta_step", c_f32), ("obf_delta_step", c_f32),
        ("obf_gain_step", c_f32), ("obr_count_run", c_i32), ("obr_corr_run", c_f32), ("obr_delta_run", c_f32),
        ("obf_delta_run", c_f32), ("obf_err_filtered_run", c_f32), ("pc_acc", c_f32 * 8),
        ("pc_target", c_f32), ("pc_measured", c_f32), ("pc_area", c_f32), ("pc_true_outlet", c_f32),
        ("pc_near", c_f32 * 3), ("pc_err_filtered", c_f32), ("pc_u_fb", c_f32), ("pc_rho_fb", c_f32),
        ("pc_guard_ref", c_f32), ("pc_guard_step", c_i32), ("pc_guard_run", c_i32), ("pc_update_step", c_i32),
        ("pc_update_run", c_i32), ("pc_sat_step", c_i32), ("pc_sat_run", c_i32), ("mn_mass", c_f32),
        ("mn_reference", c_f32), ("mn_error", c_f32), ("mn_rho_fb", c_f32), ("mn_initialized", c_i32),
        ("mn_update_step", c_i32), ("mn_update_run", c_i32), ("mn_sat_step", c_i32), ("mn_sat_run", c_i32),
        ("pad2", c_i32), ("mn_mass_acc", c_f64),
    ]


class FsiLbmState(ctypes.Structure):
    _fields_ = [
        ("nx", c_i32), ("ny", c_i32), ("nz", c_i32), ("store_fp16", c_i32), ("pitch", c_i64),
        ("pop", c_p), ("flags", c_p), ("nbr", c_p), ("rho", c_p), ("vel", c_p), ("static_solid", c_p),
        ("old_solid", c_p), ("reinit_flag", c_p), ("phi", c_p), ("smass", c_p), ("svel", c_p),
        ("cell_force", c_p), ("hydro", c_p), ("hpp", c_p), ("accum", c_p), ("plane", c_p),
        ("change_list", c_p), ("diag", c_p), ("vel_left_dyn", c_p),
    ]


class FsiLbmParams(ctypes.Structure):
    _fields_ = [
        ("rho0", c_f32), ("force", c_f32 * 3), ("s_v", c_f32), ("s_o", c_f32), ("bc_left", c_i32),
        ("bc_right", c_i32), ("ob_semantics", c_i32), ("limiter", c_i32), ("floor_enabled", c_i32),
        ("rho_bc_left", c_f32), ("rho_bc_right", c_f32), ("vel_bc_left", c_f32 * 3), ("vel_bc_right", c_f32 * 3),
        ("ob_rho_min", c_f32), ("ob_rho_max", c_f32), ("ob_u_max", c_f32), ("ob_noneq_cap", c_f32),
        ("ob_floor", c_f32), ("penalty_beta", c_f32), ("penalty_phi_min", c_f32), ("penalty_cap", c_f32),
        ("tune", c_i32),
        ("ob_gain_u", c_f32), ("ob_gain_rho", c_f32), ("ob_filter_alpha", c_f32), ("ob_cap_u", c_f32),
        ("ob_delta_cap_u", c_f32), ("ob_slew_alpha", c_f32), ("ob_blend", c_f32), ("ob_target_scale", c_f32),
        ("ob_guard_min_ratio", c_f32), ("ob_mn_gain", c_f32), ("ob_mn_cap", c_f32), ("ob_mn_blend", c_f32),
        ("ob_measure_offset", c_i32), ("ob_guard", c_i32), ("ob_mass_neutral", c_i32), ("ob_pad", c_i32),
    ]


class FsiStepCtl(ctypes.Structure):
    _fields_ = [("parity", c_i32), ("bc_pending", c_i32), ("pp", c_i32), ("mode", c_i32)]


class FsiParticles(ctypes.Structure):
    _fields_ = [("n", c_i32), ("pad", c_i32), ("x", c_p), ("v", c_p), ("C", c_p), ("F", c_p), ("Jp", c_p),
                ("mass", c_p), ("vol0", c_p), ("fixed", c_p), ("fixed_x", c_p)]


class FsiGrid(ctypes.Structure):
    _fields_ = [("n", c_i32), ("pad", c_i32), ("v", c_p), ("m", c_p), ("f_ext", c_p)]


class FsiMpmBins(ctypes.Structure):
    _fields_ = [("n_bins", c_i32), ("max_chunks", c_i32), ("key", c_p), ("count", c_p), ("start", c_p),
                ("perm", c_p), ("chunk", c_p), ("box", c_p), ("meta", c_p)]


class FsiProjectScratch(ctypes.Structure):
    _fields_ = [("key_capacity", c_i32), ("particle_capacity", c_i32), ("count", c_p), ("start", c_p),
                ("list", c_p), ("key", c_p), ("box", c_p)]


class FsiMpmParams(ctypes.Structure):
    _fields_ = [("dx", c_f32), ("inv_dx", c_f32), ("dt", c_f32), ("mu", c_f32), ("la", c_f32),
                ("gravity", c_f32 * 3), ("damping", c_f32), ("bound", c_i32), ("lock_z", c_i32), ("pad", c_i32)]


class FsiCouplingParams(ctypes.Structure):
    _fields_ = [("inv_dx_norm", c_f32), ("cell_volume_norm", c_f32), ("vel_scale", c_f32), ("eps_mass", c_f32),
                ("phi_min", c_f32), ("force_cap", c_f32), ("reaction_scale", c_f32),
                ("force_density_scale", c_f32), ("kind", c_i32), ("area_policy", c_i32),
                ("area_scale_min", c_f32), ("area_scale_max", c_f32)]


class FsiCouplingStats(ctypes.Structure):
    _fields_ = [("projected_mass", c_f64), ("projected_volume_raw", c_f64), ("projected_volume_clamped", c_f64),
                ("max_phi_raw", c_f32), ("active_cell_count", c_i32), ("active_reaction_particle_count", c_i32),
                ("max_particle_reaction_norm", c_f32), ("max_grid_reaction_norm", c_f32), ("area_scale", c_f32),
                ("raw_area_scale", c_f32), ("pad", c_i32), ("net_particle_reaction", c_f64 * 3),
                ("net_grid_reaction", c_f64 * 3)]


class FsiBatchCase(ctypes.Structure):
    _fields_ = [("lbm", FsiLbmState), ("lp", FsiLbmParams), ("ctl", FsiStepCtl), ("pt", FsiParticles),
                ("grid", FsiGrid * 3), ("bins", FsiMpmBins), ("mp", FsiMpmParams), ("cp", FsiCouplingParams),
                ("proj_stats", c_p), ("react_stats", c_p), ("mask_threshold", c_f32), ("mode", c_i32),
                ("active", c_i32)]


class FsiBatchDims(ctypes.Structure):
    _fields_ = [("n_cases", c_i32), ("store_fp16", c_i32), ("max_lbm_tiles", c_i32), ("max_particles", c_i32),
                ("max_cells", c_i64), ("max_chunks", c_i32), ("max_bins", c_i32),
                ("lbm_tune", c_i32), ("mpm_ctas", c_i32)]


FSI_BATCH_PENALTY, FSI_BATCH_MOVING = 0, 1


class FsiPlaneStats(ctypes.Structure):
    _fields_ = [("flux", c_f64), ("ux_sum", c_f64), ("ux_sq", c_f64), ("rho_sum", c_f64), ("rho_sq", c_f64),
                ("speed_max", ctypes.c_uint64), ("fluid_cells", c_i32), ("ux_negative", c_i32),
                ("ux_min", ctypes.c_uint32), ("ux_max", ctypes.c_uint32), ("rho_min", ctypes.c_uint32),
                ("rho_max", ctypes.c_uint32), ("rho_nan", c_i32), ("rho_nonfinite", c_i32), ("vel_nan", c_i32),
                ("vel_nonfinite", c_i32), ("cell_nonfinite", c_i32), ("rho_low", c_i32), ("rho_high", c_i32),
                ("vel_high", c_i32), ("rho_low_first", c_i32), ("rho_high_first", c_i32),
                ("vel_high_first", c_i32), ("pop_min", ctypes.c_uint32 * 2), ("pop_max", ctypes.c_uint32 * 2),
                ("pop_negative", c_i32 * 2), ("pop_nonfinite", c_i32 * 2), ("center_ux", c_f32),
                ("center_fluid", c_i32), ("ux_nan", c_i32)]


class FsiWallVelocityStats(ctypes.Structure):
    _fields_ = [("delta_norm_max", c_f64), ("delta_norm_sum", c_f64), ("before_norm_max", c_f64),
                ("after_norm_max", c_f64), ("after_norm_max_active", c_f64), ("after_norm_sum_active", c_f64),
                ("applied_cells", c_i32), ("pad", c_i32)]


FSI_WALL_REPLACE, FSI_WALL_ADDITIVE = 0, 1


class FsiFieldStatsArgs(ctypes.Structure):
    _fields_ = [("rho_low", c_f32), ("rho_high", c_f32), ("vel_high", c_f32), ("cy", c_i32), ("cz", c_i32),
                ("pad", c_i32), ("rho", c_p), ("vel", c_p), ("solid", c_p), ("pop_f", c_p), ("pop_F", c_p)]

STRUCTS = {
    "FsiLbmDiag": FsiLbmDiag, "FsiLbmState": FsiLbmState, "FsiLbmParams": FsiLbmParams, "FsiStepCtl": FsiStepCtl,
    "FsiParticles": FsiParticles, "FsiGrid": FsiGrid, "FsiMpmParams": FsiMpmParams,
    "FsiCouplingParams": FsiCouplingParams, "FsiCouplingStats": FsiCouplingStats, "FsiMpmBins": FsiMpmBins,
    "FsiBatchCase": FsiBatchCase, "FsiBatchDims": FsiBatchDims, "FsiCampaignSums": FsiCampaignSums,
    "FsiPlaneStats": FsiPlaneStats, "FsiFieldStatsArgs": FsiFieldStatsArgs,
    "FsiWallVelocityStats": FsiWallVelocityStats,
    "FsiProjectScratch": FsiProjectScratch,
}

# entry point -> argtypes (all return int)
_P = ctypes.POINTER
SIGNATURES = {
    "fsi_lbm_init_equilibrium": [_P(FsiLbmState), _P(FsiLbmParams), c_p],
    "fsi_lbm_set_solid": [_P(FsiLbmState), c_p, c_p],
    "fsi_lbm_to_natural": [_P(FsiLbmState), c_p],
    "fsi_lbm_substep": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_p],
    "fsi_ob_controller_update": [_P(FsiLbmState), _P(FsiLbmParams), c_p, c_p, c_p],
    "fsi_lbm_flush_bc": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_p],
    "fsi_mask_rebuild": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_f32, c_p],
    "fsi_mask_rebuild_static_scratch": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_f32, c_p],
    "fsi_force_accum_finalize": [_P(FsiLbmState), _P(FsiStepCtl), c_i32, c_p],
    "fsi_lbm_readout": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_p, c_p, c_p, c_p],
    "fsi_campaign_sums": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), c_p, c_p, c_p],
    "fsi_campaign_sums_arrays": [c_i32, c_i32, c_i32, c_p, c_p, c_p, c_p, c_p, c_p, c_p],
    "fsi_lbm_field_stats": [_P(FsiLbmState), _P(FsiLbmParams), _P(FsiStepCtl), _P(FsiFieldStatsArgs), c_p, c_p],
    "fsi_field_stats_arrays": [c_i32, c_i32, c_i32, _P(FsiFieldStatsArgs), c_p, c_p],
    "fsi_apply_wall_velocity": [_P(FsiLbmState), c_p, c_i32, c_f64, c_p, c_p],
    "fsi_project": [_P(FsiLbmState), _P(FsiParticles), _P(FsiCouplingParams), c_p, c_p],
    "fsi_project_ordered": [_P(FsiLbmState), _P(FsiParticles), _P(FsiCouplingParams), _P(FsiProjectScratch), c_p,
                            c_p],
    "fsi_reaction_to_grid": [_P(FsiLbmState), c_p, _P(FsiParticles), _P(FsiGrid), _P(FsiCouplingParams), c_p, c_p],
    "fsi_mpm_p2g": [_P(FsiParticles), _P(FsiGrid), _P(FsiMpmParams), c_p],
    "fsi_mpm_grid_update": [_P(FsiGrid), _P(FsiMpmParams), c_p],
    "fsi_mpm_g2p": [_P(FsiParticles), _P(FsiGrid), _P(FsiMpmParams), c_p],
    "fsi_mpm_bins_layout": [c_i32, c_i32, _P(c_i32), _P(c_i32)],
    "fsi_mpm_bin": [_P(FsiParticles), _P(FsiGrid), _P(FsiMpmParams), _P(FsiMpmBins), c_p],
    "fsi_mpm_substeps_binned": [_P(FsiParticles), _P(FsiGrid), _P(FsiMpmBins), _P(FsiMpmParams), c_i32,
                                _P(FsiLbmState), c_p, _P(FsiCouplingParams), c_p, c_p],
    "fsi_mpm_grid_velocity": [_P(FsiGrid), _P(FsiMpmParams), c_p, c_p],
    "fsi_batch_project": [c_p, _P(FsiBatchDims), c_p],
    "fsi_batch_mask_rebuild": [c_p, _P(FsiBatchDims), c_p],
    "fsi_batch_lbm_substep": [c_p, _P(FsiBatchDims), c_p],
    "fsi_batch_mpm_bin": [c_p, _P(FsiBatchDims), c_p],
    "fsi_batch_mpm_substeps": [c_p, _P(FsiBatchDims), c_i32, c_p],
    "fsi_abi_version": [],
    "fsi_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "fsi_launch_count": [],
}
# entry points that do not return int
RESTYPES = {"fsi_launch_count": ctypes.c_uint64}

_lock = threading.Lock()
_lib = None


class FsiError(RuntimeError):
    pass


def load():
    """Load the in-tree library; raise if it is missing (no fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise FsiError(f"{LIB_PATH} is not built; run `python -m mpm_lbm_b200.build` (nvcc, sm_100a)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = RESTYPES.get(name, ctypes.c_int)
        if lib.fsi_abi_version() != ABI_VERSION:
            raise FsiError("libfsi_b200.so ABI version mismatch")
        _lib = lib
        return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    load().fsi_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def call(name, *args):
    rc = getattr(load(), name)(*args)
    if rc != 0:
        raise FsiError(f"{name} failed ({rc}): {last_error()}")
    return rc


def launch_count() -> int:
    """Kernel launches issued by libfsi_b200.so so far (graph nodes while capturing)."""
    return int(load().fsi_launch_count())


def ptr(t):
    """Device address of a torch tensor (or None)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_handle(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)

/*
 * fsi_b200.h -- C ABI of the B200 coupled MPM-LBM FSI step.
 *
 * The reference (lizhuoh9/MPM-LBM) has no native boundary: its hot path is a
 * set of Taichi kernels called from Python (src/mpm_lbm/sim/drivers/
 * fsi_driver.py:425-575).  Each entry point below replaces one or more of those
 * kernel calls; the Python package mpm_lbm_b200 binds them with ctypes behind
 * the reference's FSIDriver3D / LBMFluid3D / MPMSolid3D / coupler API.
 *
 * Conventions
 *  - Every pointer inside the structs is a DEVICE pointer owned by the caller
 *    (torch tensors); no entry point allocates or frees memory.
 *  - Calls are asynchronous and ordered on the given cudaStream_t (passed as
 *    void*, NULL = legacy default stream).  Return 0 on success or a negative
 *    FSI_E_* code; fsi_last_error() returns the message of the last failure
 *    on the calling thread.
 *  - Cell fields use the lattice layout: cell = (k * ny + j) * nx + i (x
 *    fastest); vector fields are planar: comp c of cell at [c * pitch + cell].
 *  - Populations use the in-place AA pattern: the layout of `pop` alternates
 *    with FsiStepCtl.parity (0: every cell holds its own populations; 1: each
 *    fluid-fluid link's pair of slots is swapped).  fsi_lbm_readout decodes it.
 */
#ifndef FSI_B200_H
#define FSI_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: populations in blocks of 32 cells (FsiLbmState.pop), FsiLbmDiag.mn_mass_acc,
 *    fsi_project_ordered.  1: populations in [19][pitch] planes. */
#define FSI_ABI_VERSION 2

enum {
  FSI_OK = 0,
  FSI_E_INVALID = -1,   /* bad argument or unsupported configuration */
  FSI_E_CUDA = -2,      /* a CUDA launch or runtime call failed */
  FSI_E_DEVICE = -3,    /* the device reported an error status */
};

/* cell flag bits */
enum {
  FSI_CELL_SOLID = 1,     /* solid (static or dynamic) */
  FSI_CELL_NEAR = 2,      /* fluid cell with a solid neighbour; FsiLbmState.nbr valid */
  FSI_CELL_LINK = 4,      /* solid cell with a fluid neighbour (receives link forces) */
  FSI_CELL_OVERRIDE = 8,  /* collide with the stored rho/vel instead of recomputing them */
  FSI_CELL_CF = 16,       /* cell_force / hydro hold a non-zero penalty force */
};

/* open-boundary semantics (src/mpm_lbm/sim/lbm/fluid.py:16-25, Boundary_condition 538-569).
 * 4-9 differ from 1 only at a right-face pressure outlet (bc_right == 1): a
 * repaired regularized population (4, 6, 8) or its blend with the convective
 * one (5, 7, 9), fed back from the neighbour's density and velocity (4-7) or
 * from the plane-flux controller (8, 9: update_open_boundary_plane_flux_controller,
 * fluid.py:1141-1263, run once per step after the step kernel). */
enum {
  FSI_OB_EQUILIBRIUM_RESET = 0,
  FSI_OB_REGULARIZED = 1,
  FSI_OB_REGULARIZED_LIMITED = 2,
  FSI_OB_CONVECTIVE = 3,
  FSI_OB_REG_MASS_BALANCED = 4,     /* regularized_mass_balanced_pressure_outlet */
  FSI_OB_CONV_MASS_BALANCED = 5,    /* convective_mass_balanced_pressure_outlet */
  FSI_OB_REG_FLUX_MATCHED = 6,      /* regularized_flux_matched_pressure_outlet */
  FSI_OB_CONV_FLUX_MATCHED = 7,     /* convective_flux_matched_damped_outlet */
  FSI_OB_REG_PLANE_FLUX = 8,        /* regularized_plane_flux_controlled_pressure_outlet */
  FSI_OB_CONV_PLANE_FLUX = 9,       /* convective_plane_flux_controlled_damped_outlet */
};

/* step mode bits */
enum {
  FSI_MODE_MOVING_BB = 1,  /* streaming_moving_bounceback (fluid.py:488) instead of streaming1 (431) */
  FSI_MODE_SUBCYCLED = 2,  /* link forces feed the subcycle accumulator (fluid.py:460-486) */
  FSI_MODE_DIRSTATS = 4,   /* produce the per-direction bounce-back reductions this step */
  FSI_MODE_PENALTY = 8,    /* build the penalty force in the step (coupling/penalty.py:59-88) */
};

/* device-resident reductions; zeroed by the caller where noted */
typedef struct FsiLbmDiag {
  int32_t link_count[19];            /* bb_link_count_by_dir */
  float corr_abs_sum[19];            /* bb_correction_abs_sum_by_dir */
  float corr_abs_max[19];            /* bb_correction_abs_max_by_dir (non-negative, max via int bits) */
  float fluid_impulse[19][3];        /* bb_fluid_impulse_by_dir (solid force = -this) */
  float accum_norm_max;              /* mb_subcycle_force_accum_norm_max */
  float mean_norm_max;               /* mb_subcycle_force_mean_norm_max */
  int32_t ob_step[5];                /* rho, velocity, noneq, floor, reconstructed counts of the last BC */
  int32_t ob_run[5];                 /* cumulative */
  int32_t penalty_active;            /* active_force_cell_count */
  float penalty_max_norm;            /* max_cell_force_norm == max_hydro_force_norm */
  float penalty_net[3];              /* net_cell_force (net hydro = -this) */
  int32_t change_count;              /* cells whose solid bit flipped in the last mask rebuild */
  int32_t status;                    /* non-zero: device-side error code */
  int32_t pad[2];
  /* open-boundary repair of semantics 4-9 (fluid.py:1115-1140): the last BC
   * (cleared before each) and cumulative: mass_balance_correction_count /
   * _abs_sum, unknown_population_delta_abs_sum, flow_correction_delta_abs_sum,
   * flow_correction_gain_effective_step, flow_outlet_flux_error_filtered_run */
  int32_t obr_count_step;
  float obr_corr_step, obr_delta_step, obf_delta_step, obf_gain_step;
  int32_t obr_count_run;
  float obr_corr_run, obr_delta_run, obf_delta_run, obf_err_filtered_run;
  /* plane-flux controller (fluid.py:1141-1263): sums the step kernel accumulates
   * from its macroscopic state (rho * u_x of the fluid cells of x = 0, the
   * measure plane, x = nx-1, nx-2, nx-3, nx-4; fluid cells of the measure plane;
   * [7] unused: the fluid mass goes to mn_mass_acc), consumed and cleared by the
   * controller update */
  float pc_acc[8];
  float pc_target, pc_measured, pc_area, pc_true_outlet;
  float pc_near[3];
  float pc_err_filtered, pc_u_fb, pc_rho_fb, pc_guard_ref;
  int32_t pc_guard_step, pc_guard_run;
  int32_t pc_update_step, pc_update_run, pc_sat_step, pc_sat_run;
  float mn_mass, mn_reference, mn_error, mn_rho_fb;
  int32_t mn_initialized;
  int32_t mn_update_step, mn_update_run, mn_sat_step, mn_sat_run;
  int32_t pad2;
  double mn_mass_acc;  /* the fluid mass for the mass-neutral feedback, summed in FP64 (pc_acc[7] unused) */
} FsiLbmDiag;

typedef struct FsiLbmState {
  int32_t nx, ny, nz;
  int32_t store_fp16;       /* 0: float populations; 1: half (f/w - rho0) */
  int64_t pitch;            /* >= nx*ny*nz, multiple of 32 */
  void* pop;                /* 19 * pitch float or __half, in blocks of 32 cells: population s of cell i
                               at (i / 32) * 608 + s * 32 + i % 32 */
  uint8_t* flags;           /* [pitch] FSI_CELL_* */
  uint32_t* nbr;            /* [pitch] bit s: cell + e_s is solid (valid with FSI_CELL_NEAR) */
  float* rho;               /* [pitch] stored density (override cells, readout) */
  float* vel;               /* [3][pitch] stored velocity */
  uint8_t* static_solid;    /* [pitch] */
  uint8_t* old_solid;       /* [pitch] */
  uint8_t* reinit_flag;     /* [pitch] */
  float* phi;               /* [pitch] solid_phi */
  float* smass;             /* [pitch] solid_mass */
  float* svel;              /* [3][pitch] solid_vel (lattice units) */
  float* cell_force;        /* [3][pitch] */
  float* hydro;             /* [3][pitch] hydro_force (penalty / subcycled mean) */
  float* hpp;               /* [2][3][pitch] per-step link forces, ping-pong */
  float* accum;             /* [3][pitch] hydro_force_accum */
  float* plane;             /* [5][4][ny*nz]: planes 0-3 rho,ux,uy,uz of x = 0, 1, nx-2, nx-1 of the last
                               step; plane 4 scratch of the outlet flow filter (semantics 6, 7), zeroed */
  int32_t* change_list;     /* [pitch] scratch for the mask rebuild */
  FsiLbmDiag* diag;         /* device */
  const float* vel_left_dyn;  /* optional [3]: x-min inlet velocity read on the device each step
                                 (bc_vel_x_left_dynamic, fluid.py:287-288, 1979); NULL = vel_bc_left */
} FsiLbmState;

typedef struct FsiLbmParams {
  float rho0;
  float force[3];           /* set_force (fluid.py:2025) */
  float s_v, s_o;           /* MRT rates (fluid.py:301-302); s_o == s_v gives the BGK form */
  int32_t bc_left, bc_right;   /* 0 periodic, 1 pressure, 2 velocity (x faces) */
  int32_t ob_semantics;     /* FSI_OB_* */
  int32_t limiter, floor_enabled;
  float rho_bc_left, rho_bc_right;
  float vel_bc_left[3], vel_bc_right[3];
  float ob_rho_min, ob_rho_max, ob_u_max, ob_noneq_cap, ob_floor;
  float penalty_beta, penalty_phi_min, penalty_cap;
  int32_t tune;             /* FSI_TUNE_LBM_*: launch variant of the step kernel (results are identical) */
  /* open-boundary semantics 4-9 (LBMConfig.open_boundary_*, lbm/config.py:53-69) */
  float ob_gain_u, ob_gain_rho, ob_filter_alpha, ob_cap_u, ob_delta_cap_u, ob_slew_alpha, ob_blend;
  float ob_target_scale, ob_guard_min_ratio, ob_mn_gain, ob_mn_cap, ob_mn_blend;
  int32_t ob_measure_offset;  /* 0..2: the controller measures x = nx - 1 - offset */
  int32_t ob_guard;           /* outlet flux drop guard */
  int32_t ob_mass_neutral;    /* mass-neutral density offset (mode global_mass_error_density_offset) */
  int32_t ob_pad;
} FsiLbmParams;

/* launch variants of fsi_lbm_substep (FsiLbmParams.tune) */
enum {
  FSI_TUNE_LBM_OCC3 = 0,  /* registers for 3 CTAs of 256 threads per SM (default) */
  FSI_TUNE_LBM_OCC4 = 1,  /* registers for 4 CTAs per SM (64 per thread) */
  FSI_TUNE_LBM_PAIR = 2,  /* two x-adjacent cells per thread on the paired FP32 pipe; nx even, and
                             nx % 64 != 2 with open boundaries (results agree to FP32 rounding) */
  FSI_TUNE_LBM_OCC3_PF = 3, /* OCC3, each CTA prefetching into L2 the tile one resident wave later */
  FSI_TUNE_LBM_OCC4_PF = 4, /* OCC4 with the same L2 prefetch */
};

typedef struct FsiStepCtl {
  int32_t parity;       /* AA layout parity of the input state */
  int32_t bc_pending;   /* 1: the open-boundary step of the previous step is still to be applied */
  int32_t pp;           /* ping-pong slot of hpp written by this step */
  int32_t mode;         /* FSI_MODE_* */
} FsiStepCtl;

/* ---- LBM (replaces LBMFluid3D kernels) ---------------------------------- */

/* init (fluid.py:328-344): populations feq(rho0, 0), rho = rho0, vel = 0,
 * flags = solid bits of static_solid | OVERRIDE, old_solid = static_solid,
 * neighbour masks rebuilt.  Layout parity 0. */
int fsi_lbm_init_equilibrium(const FsiLbmState* s, const FsiLbmParams* p, void* stream);

/* Rebuild neighbour masks and NEAR/LINK flags from the solid bits (init_geo,
 * fluid.py:347-353 + copy_solid_to_static 1841). Requires parity 0. */
int fsi_lbm_set_solid(const FsiLbmState* s, const uint8_t* solid, void* stream);

/* Convert a parity-1 state to parity 0 (pure data movement). */
int fsi_lbm_to_natural(const FsiLbmState* s, void* stream);

/* One fused LBM step: pending open boundary of the previous step
 * (Boundary_condition, fluid.py:538-569) -> macroscopic update (streaming3,
 * 1794-1814) -> optional penalty force (coupling/penalty.py:59-88) -> MRT
 * collision (398-413) -> AA streaming with static or moving half-way
 * bounce-back and momentum-exchange link forces (431-440 / 488-536). */
int fsi_lbm_substep(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, void* stream);
/* Under semantics 4-9 fsi_lbm_substep launches one more small kernel after the
 * step: the clear of the repair step counters and, under 8 and 9, the outlet
 * flux controller (update_open_boundary_plane_flux_controller, fluid.py:1141-1263)
 * from plane sums the step accumulated, ahead of the step's pending open boundary. */

/* update_open_boundary_plane_flux_controller (fluid.py:1141-1263) called on its
 * own, from given macroscopic fields rho [pitch] and vel [3][pitch] (the
 * readout of the state, or fields the caller set) and the solid bits of the
 * state.  Replaces LBMFluid3D.update_open_boundary_plane_flux_controller. */
int fsi_ob_controller_update(const FsiLbmState* s, const FsiLbmParams* p, const float* rho, const float* vel,
                             void* stream);

/* Apply a pending open-boundary step into the state (so that a mask rebuild
 * sees the same populations as the reference). */
int fsi_lbm_flush_bc(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, void* stream);

/* update_dynamic_solid + reinitialize_new_fluid_cells (fluid.py:1847-1877),
 * including the AA re-pairing of links whose fluid/solid status changed. */
int fsi_mask_rebuild(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, float threshold,
                     void* stream);

/* fsi_mask_rebuild without the change_list scratch: the list of flipped
 * cells lives in a file-scope device array of the library, so the caller
 * passes no scratch (s->change_list is ignored) and nothing is allocated.
 * No counterpart in the reference.  For callers that own the lattice state
 * but cannot provide one more device buffer (e.g. a host binding without a
 * device allocator).  Limits: nx*ny*nz <= 1048576 cells, else FSI_E_INVALID;
 * all calls on one device share the array, so calls must not overlap in
 * time (order them on one stream); the first call on each device looks the
 * array up (cudaGetSymbolAddress) and should be made outside stream capture.
 * The address is kept for the life of the process: do not call this entry
 * point after a cudaDeviceReset of that device. */
int fsi_mask_rebuild_static_scratch(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl,
                                    float threshold, void* stream);

/* finalize_moving_boundary_force_accumulator (fluid.py:475-486): folds the
 * last substep, hydro = accum / sample_count. */
int fsi_force_accum_finalize(const FsiLbmState* s, const FsiStepCtl* ctl, int32_t sample_count, void* stream);

/* Decode the public fields: F (== f) [19][pitch], rho [pitch], vel [3][pitch]
 * with any pending open boundary applied (read-only on the state). */
int fsi_lbm_readout(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, float* out_pop,
                    float* out_rho, float* out_vel, void* stream);

/* Per-FSI-step reductions of the subcycled flow campaign
 * (solvers/official_subcycled_flow_solver.py:352-365 copies rho, v, f and
 * solid to the host every step; 443-515 then sums them in FP64).  One pass
 * over the readout state of every cell (as fsi_lbm_readout returns it),
 * FP64 sums, ~100 bytes of output instead of the four fields:
 *   - over fluid cells: sum of rho, the cell count, and the number of cells
 *     with a non-finite rho, v or population;
 *   - over the cells whose regions[i] has bit r set (any solid state; NULL:
 *     none): sum of rho * v_x.
 * regions: [nx * ny * nz] in lattice order (x fastest).  out: device. */
#define FSI_CAMPAIGN_REGIONS 8
typedef struct FsiCampaignSums {
  double fluid_mass;
  double region_flux[FSI_CAMPAIGN_REGIONS];
  int32_t fluid_cells;
  int32_t nonfinite_rho, nonfinite_vel, nonfinite_pop;
} FsiCampaignSums;
int fsi_campaign_sums(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, const uint8_t* regions,
                      FsiCampaignSums* out, void* stream);
/* The same sums from plain device fields in lattice order (x fastest,
 * n = nx * ny * nz): rho [n], vel [3][n], pop [19][n] (NULL: no population
 * check), solid [n] (non-zero: solid) -- the host copies _copy_lbm_fields
 * makes (official_subcycled_flow_solver.py:352-365), held on the device. */
int fsi_campaign_sums_arrays(int32_t nx, int32_t ny, int32_t nz, const float* rho, const float* vel, const float* pop,
                             const uint8_t* solid, const uint8_t* regions, FsiCampaignSums* out, void* stream);

/* Per-x-plane statistics of the lattice fields, one device pass.  The
 * reference's diagnostics (sim/diagnostics/lbm_boundary_diagnostics.py,
 * lbm_stability_diagnostics.py) copy rho, v, solid, f and F to the host and
 * reduce them with numpy in FP64; every quantity they report is a function
 * of these per-plane records (host sums over planes give the totals).
 * Keys: order-preserving uint32 codes of FP32 values (a min key of
 * FSI_KEY_NONE_MIN or a max key of 0: no value); NaN is skipped by the
 * min / max keys and counted separately. */
#define FSI_KEY_NONE_MIN 0xffffffffu
typedef struct FsiPlaneStats {
  double flux;              /* fluid cells: sum of rho * v_x (FP64) */
  double ux_sum, ux_sq;     /* fluid: sum of v_x, of v_x^2 */
  double rho_sum, rho_sq;   /* fluid: sum of rho, of (rho - 1)^2 */
  uint64_t speed_max;       /* fluid: max |v| (bits of the FP64 norm, NaN skipped; 0: none) */
  int32_t fluid_cells;
  int32_t ux_negative;      /* fluid cells with v_x < 0 */
  uint32_t ux_min, ux_max, rho_min, rho_max;   /* fluid cells: keys */
  int32_t rho_nan, rho_nonfinite, vel_nan, vel_nonfinite;  /* fluid cells (vel: any component) */
  int32_t cell_nonfinite;   /* cells of any kind with a non-finite rho or v */
  int32_t rho_low, rho_high, vel_high;                     /* fluid: rho < low, rho > high, |v| > vel_high */
  int32_t rho_low_first, rho_high_first, vel_high_first;   /* smallest j * nz + k of those (INT32_MAX: none) */
  uint32_t pop_min[2], pop_max[2];      /* populations f, F of all cells: keys */
  int32_t pop_negative[2], pop_nonfinite[2];
  float center_ux;          /* v_x at (x, cy, cz) */
  int32_t center_fluid;     /* solid[x, cy, cz] == 0 */
  int32_t ux_nan;           /* fluid cells with a NaN v_x */
} FsiPlaneStats;

typedef struct FsiFieldStatsArgs {
  float rho_low, rho_high, vel_high;  /* density_outlier_stats low / high, velocity_outlier_stats threshold */
  int32_t cy, cz;                     /* centerline cell of centerline_profile_x */
  int32_t pad;
  /* fsi_field_stats_arrays only: fields in lattice order (x fastest), n = nx*ny*nz */
  const float* rho;       /* [n] */
  const float* vel;       /* [3][n] */
  const uint8_t* solid;   /* [n] non-zero: solid */
  const float* pop_f;     /* [19][n] or NULL (zeros, as the reference's snapshot without f) */
  const float* pop_F;     /* [19][n] or NULL */
} FsiFieldStatsArgs;

/* planes: [nx] device records, overwritten.  From the state's readout (as
 * fsi_lbm_readout returns it; f and F are the same array there, so index 0
 * and 1 of the population fields agree). */
int fsi_lbm_field_stats(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl,
                        const FsiFieldStatsArgs* a, FsiPlaneStats* planes, void* stream);
/* The same from plain device fields (a snapshot the caller holds). */
int fsi_field_stats_arrays(int32_t nx, int32_t ny, int32_t nz, const FsiFieldStatsArgs* a, FsiPlaneStats* planes,
                           void* stream);

/* apply_wall_velocity_to_lbm_solid_vel (wall_velocity/application.py:118-158):
 * cells whose grid velocity g has |g| > 0 get solid_vel = g (replace) or
 * solid_vel + g (additive), capped to |.| <= cap, all in FP64 from the FP32
 * solid_vel, written back as FP32.  grid: [3][pitch] FP64 in lattice order.
 * out (device) receives the statistics of the reference's result dict. */
#define FSI_WALL_REPLACE 0
#define FSI_WALL_ADDITIVE 1
typedef struct FsiWallVelocityStats {
  double delta_norm_max, delta_norm_sum;   /* |after - before| over applied cells */
  double before_norm_max, after_norm_max;  /* over all cells */
  double after_norm_max_active, after_norm_sum_active;
  int32_t applied_cells;
  int32_t pad;
} FsiWallVelocityStats;
int fsi_apply_wall_velocity(const FsiLbmState* s, const double* grid, int32_t policy, double cap,
                            FsiWallVelocityStats* out, void* stream);

/* ---- particles, projection, reaction transfer, MPM ---------------------- */

typedef struct FsiParticles {
  int32_t n;
  int32_t pad;
  float* x;          /* [3][n] */
  float* v;          /* [3][n] */
  float* C;          /* [9][n] row-major components */
  float* F;          /* [9][n] */
  float* Jp;         /* [n] */
  float* mass;       /* [n] */
  float* vol0;       /* [n] */
  uint8_t* fixed;    /* [n] */
  float* fixed_x;    /* [3][n] */
} FsiParticles;

typedef struct FsiGrid {
  int32_t n;         /* MPM grid edge (n^3 nodes, node = (k * n + j) * n + i) */
  int32_t pad;
  float* v;          /* [3][n^3] grid_v (momentum during P2G) */
  float* m;          /* [n^3] */
  float* f_ext;      /* [3][n^3] */
} FsiGrid;

typedef struct FsiMpmParams {
  float dx, inv_dx, dt, mu, la;
  float gravity[3];
  float damping;     /* >0 enables particle_velocity_post_g2p damping */
  int32_t bound;
  int32_t lock_z;
  int32_t pad;
} FsiMpmParams;


typedef struct FsiCouplingParams {
  float inv_dx_norm, cell_volume_norm, vel_scale, eps_mass;
  float phi_min, force_cap, reaction_scale, force_density_scale;
  int32_t kind;           /* 0 penalty, 1 engineering, 2 link-area */
  int32_t area_policy;    /* link-area: 0 uniform, 1 inverse_length, 2 length */
  float area_scale_min, area_scale_max;
} FsiCouplingParams;

/* f64 reductions of the coupling step */
typedef struct FsiCouplingStats {
  double projected_mass, projected_volume_raw, projected_volume_clamped;
  float max_phi_raw;
  int32_t active_cell_count;
  int32_t active_reaction_particle_count;
  float max_particle_reaction_norm;
  float max_grid_reaction_norm;
  float area_scale, raw_area_scale;
  int32_t pad;
  double net_particle_reaction[3];
  double net_grid_reaction[3];
} FsiCouplingStats;

/* MPMToLBMProjector3D.project (coupling/projection.py:21-97): clear, P2G of
 * phi/mass/momentum onto the lattice, normalise + clamp.  stats: device. */
int fsi_project(const FsiLbmState* s, const FsiParticles* pt, const FsiCouplingParams* cp, FsiCouplingStats* stats,
                void* stream);

/* The same projection with every cell's sums taken in the reference's order:
 * particle index ascending, each term added in FP32 with IEEE rounding and no
 * fused multiply-add (projection.py:39-65 run by one thread, the order a
 * serial ti.cpu run sums its atomic adds in).  solid_phi, solid_mass and
 * solid_vel are then bit-identical to that serial sum for the same particle
 * state and the same on every run, so the solid mask it feeds
 * (update_dynamic_solid, fluid.py:1847-1861) does not depend on the order of
 * float atomics even for cells whose phi sits within a few ulps of the
 * threshold.  fsi_project's float atomics sum in an unspecified order.
 * Particles are sorted by B-spline base cell over the bounding box of the
 * base cells; each cell then gathers its contributors (at most 27 base-cell
 * lists), ranks them by particle index and sums them in rank order. */
typedef struct FsiProjectScratch {
  int32_t key_capacity;       /* >= (nx + 2) * (ny + 2) * (nz + 2) */
  int32_t particle_capacity;  /* >= the particle count */
  int32_t* count;             /* [key_capacity + 1], zero before the first call; kept zero after each call */
  int32_t* start;             /* [key_capacity + 1] */
  int32_t* list;              /* [particle_capacity] particle ids by base cell, ascending within a cell */
  int32_t* key;               /* [particle_capacity] */
  int32_t* box;               /* [8] base-cell bounding box of the last call */
} FsiProjectScratch;
int fsi_project_ordered(const FsiLbmState* s, const FsiParticles* pt, const FsiCouplingParams* cp,
                        const FsiProjectScratch* scratch, FsiCouplingStats* stats, void* stream);

/* Reaction transfer LBM -> MPM grid: penalty (coupling/penalty.py:90-129),
 * engineering (moving_boundary.py:58-110) or link-area (link_area.py:84-193,
 * area scale computed on the device from the last directional reductions).
 * hydro: the hydro-force field to sample ([3][pitch]). */
int fsi_reaction_to_grid(const FsiLbmState* s, const float* hydro, const FsiParticles* pt, const FsiGrid* g,
                         const FsiCouplingParams* cp, FsiCouplingStats* stats, void* stream);

/* MPMSolid3D.p2g (mpm/solid.py:219-249): fixed-corotated stress with the
 * polar rotation computed in FP64; grid must be cleared by the caller. */
int fsi_mpm_p2g(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, void* stream);

/* MPMSolid3D.grid_update (mpm/solid.py:251-259, boundary 97-111). */
int fsi_mpm_grid_update(const FsiGrid* g, const FsiMpmParams* mp, void* stream);

/* MPMSolid3D.g2p (mpm/solid.py:261-315): APIC gather, advection, clamp,
 * F update, damping / z-lock controls, fixed-base reset. */
int fsi_mpm_g2p(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, void* stream);

/* ---- binned MPM substeps ------------------------------------------------
 * The same substep as clear -> p2g -> reaction -> grid_update -> g2p above
 * (one call of MPMSolid3D.substep plus the coupler's reaction transfer, as
 * driven by fsi_driver.py's MPM loops), organised around particle bins:
 *   - fsi_mpm_bin sorts particle ids by FSI_BIN_EDGE^3-cell block of their
 *     B-spline base cell, and within a block by base cell, and cuts every bin
 *     into ceil(count / FSI_BIN_CHUNK) chunks of equal size (sizes differ by
 *     at most one; bins may go stale between calls: that costs speed only);
 *   - fsi_mpm_substeps_binned runs substeps chunk by chunk: each chunk is
 *     scattered into a shared-memory tile covering its stencil box and the
 *     tile is flushed with one atomic per touched node value; the gather
 *     evaluates the grid update per node while staging the chunk's box.  A
 *     substep leaves momentum (not velocity), mass and f_ext in its grid
 *     buffer; three buffers rotate, and only the boxes recorded for a buffer
 *     are zeroed before it is reused, so no dense pass over the grid is made. */
#define FSI_BIN_CHUNK 128
#define FSI_BIN_EDGE 8

/* count, start and chunk must be 16-byte aligned */
typedef struct FsiMpmBins {
  int32_t n_bins;       /* ceil(n_grid / FSI_BIN_EDGE)^3 */
  int32_t max_chunks;   /* capacity of chunk[] and of each third of box[] */
  int32_t* key;         /* [n_particles] scratch (bin keys, then the in-bin sort) */
  int32_t* count;       /* [n_bins] zero before the first fsi_mpm_bin; kept zero after each call */
  int32_t* start;       /* [n_bins] end offset of each bin in perm after fsi_mpm_bin */
  int32_t* perm;        /* [n_particles] particle ids ordered by bin */
  int32_t* chunk;       /* [max_chunks][2] (first slot in perm, particle count) */
  int32_t* box;         /* [3][max_chunks][6] node box (lo xyz, hi xyz) touched per chunk and buffer */
  int32_t* meta;        /* [8] chunk count, records in box[0..2], chunks scattered without the tile,
                           buffer 0..2 holds unzeroed boxes; zero before the first call */
} FsiMpmBins;

/* n_bins and max_chunks for a particle count and grid edge */
int fsi_mpm_bins_layout(int32_t n_particles, int32_t n_grid, int32_t* n_bins, int32_t* max_chunks);

/* (re)bin the particles at their current positions */
int fsi_mpm_bin(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, const FsiMpmBins* bins,
                void* stream);

/* n_substeps binned MPM substeps (each one call of MPMSolid3D.substep plus,
 * with cp != NULL, the reaction transfer of kind cp->kind from s and hydro as
 * for fsi_reaction_to_grid, whose reductions go to stats[substep % 3]) as
 * n_substeps + 2 launches: launch s gathers substep s - 1 and, for the same
 * chunk of particles, builds and scatters substep s, rotating over three grid
 * buffers (substep s scatters into grid[s % 3]).
 *   - On entry every buffer must be zero apart from the boxes recorded in the
 *     bins (any earlier call of this function leaves it so).
 *   - On return grid[(n_substeps - 1) % 3] holds the last substep's momentum,
 *     mass and f_ext, and stats[(n_substeps - 1) % 3] its reaction reductions.
 *   - Zero the three buffers and bins->meta[1..7] after using grid[0] with
 *     the one-phase entry points (fsi_mpm_p2g etc.). */
int fsi_mpm_substeps_binned(const FsiParticles* pt, const FsiGrid grid[3], const FsiMpmBins* bins,
                            const FsiMpmParams* mp, int32_t n_substeps, const FsiLbmState* s, const float* hydro,
                            const FsiCouplingParams* cp, FsiCouplingStats stats[3], void* stream);

/* grid velocity after a binned substep (the grid_v of the reference after
 * grid_update) from grid's momentum, mass and f_ext, into out [3][n^3] */
int fsi_mpm_grid_velocity(const FsiGrid* g, const FsiMpmParams* mp, float* out, void* stream);

/* ---- batched cases -------------------------------------------------------
 * Many independent FSI cases (each its own lattice, particles, MPM grid,
 * parameters and coupling mode) advanced together: each fsi_batch_* call
 * runs one phase of the FSI step for every active case in one launch per
 * kernel (grid.y = case slot, grid.x strides over the case's work).  The
 * reference advances one FSIDriver3D per process (fsi_driver.py:425-531);
 * a batch of N cases performs, per case, exactly the phases of
 * FSIDriver3D.step_once with one LBM step per FSI step:
 *   penalty:          fsi_batch_project, fsi_batch_lbm_substep (penalty force
 *                     built in the step), then fsi_batch_mpm_substeps (M)
 *   moving_boundary:  fsi_batch_project, fsi_batch_mask_rebuild,
 *                     fsi_batch_lbm_substep, then fsi_batch_mpm_substeps (M)
 * with fsi_batch_mpm_bin before the MPM substeps.  Cases must have no open
 * boundaries (bc_left = bc_right = 0) and equal population storage.
 *
 * `cases` is a DEVICE array of FsiBatchCase; the calls read the descriptors
 * there and advance the per-case step state (ctl, buf) on the device, so a
 * sequence of calls can be captured in a CUDA graph and replayed.  The host
 * keeps `dims` current (maxima over the active cases). */
enum {
  FSI_BATCH_PENALTY = 0,
  FSI_BATCH_MOVING = 1,
};

typedef struct FsiBatchCase {
  FsiLbmState lbm;
  FsiLbmParams lp;
  FsiStepCtl ctl;                 /* parity, pp advanced by fsi_batch_lbm_substep */
  FsiParticles pt;
  FsiGrid grid[3];                /* MPM grid buffers of the binned substeps */
  FsiMpmBins bins;
  FsiMpmParams mp;
  FsiCouplingParams cp;           /* reaction kind 0 penalty, 1 engineering, 2 link-area */
  FsiCouplingStats* proj_stats;   /* device [1] */
  FsiCouplingStats* react_stats;  /* device [3] (as stats of fsi_mpm_substeps_binned) */
  float mask_threshold;           /* dynamic_solid_threshold */
  int32_t mode;                   /* FSI_BATCH_* */
  int32_t active;                 /* 0: empty slot, skipped */
} FsiBatchCase;

typedef struct FsiBatchDims {
  int32_t n_cases;                /* slots in `cases` (active or not) */
  int32_t store_fp16;             /* population storage of every case */
  int32_t max_lbm_tiles;          /* max over cases of ceil(nx / 32) * ceil(ny / 8) * nz */
  int32_t max_particles;
  int64_t max_cells;              /* max nx * ny * nz */
  int32_t max_chunks;             /* max FsiMpmBins.max_chunks */
  int32_t max_bins;               /* max FsiMpmBins.n_bins */
  int32_t lbm_tune;               /* FSI_TUNE_LBM_OCC3, or FSI_TUNE_LBM_PAIR when every case has an even nx */
  int32_t mpm_ctas;               /* CTAs per case of the batched MPM substeps (0: about one per chunk of the
                                     largest case); a launch variant picked by the batch autotuner */
} FsiBatchDims;

/* MPMToLBMProjector3D.project per case (coupling/projection.py:21-97). */
int fsi_batch_project(FsiBatchCase* cases, const FsiBatchDims* dims, void* stream);
/* update_dynamic_solid + reinitialize_new_fluid_cells per moving-boundary case
 * (fluid.py:1847-1877); penalty cases are skipped. */
int fsi_batch_mask_rebuild(FsiBatchCase* cases, const FsiBatchDims* dims, void* stream);
/* One LBM step per case: step_moving_bounceback (fluid.py:2105) for moving
 * cases, step (2099) with the penalty force (penalty.py:59-88) for penalty
 * cases; then the case's parity and ping-pong slot advance. */
int fsi_batch_lbm_substep(FsiBatchCase* cases, const FsiBatchDims* dims, void* stream);
/* fsi_mpm_bin per case. */
int fsi_batch_mpm_bin(FsiBatchCase* cases, const FsiBatchDims* dims, void* stream);
/* n_substeps binned MPM substeps per case with its reaction transfer
 * (penalty.py:90-129 / moving_boundary.py:58-110 / link_area.py:139-193) from
 * the last LBM step's force field, as fsi_mpm_substeps_binned does for one
 * case: n_substeps + 2 launches for the whole batch. */
int fsi_batch_mpm_substeps(FsiBatchCase* cases, const FsiBatchDims* dims, int32_t n_substeps, void* stream);

/* ---- misc --------------------------------------------------------------- */
int fsi_abi_version(void);
/* Kernel launches issued by this library since it was loaded (all threads).
 * During stream capture a launch becomes a graph node, so the difference
 * across a capture is the number of this library's kernels in the graph.
 * Instrumentation only: the reference has no counterpart. */
uint64_t fsi_launch_count(void);
int fsi_last_error(char* buf, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* FSI_B200_H */

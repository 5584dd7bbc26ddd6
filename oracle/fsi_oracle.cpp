// CPU restatement of the reference's coupled MPM-LBM FSI step.
//
// TEST INFRASTRUCTURE ONLY: this file is the parity oracle and the timed CPU
// baseline.  Nothing in the product links or calls it; only tests/, the
// smoke check of __graft_entry__ and bench.py's CPU-baseline leg do.
//
// Every function restates one reference Taichi kernel, in the reference's
// loop order (single-thread order, as the reference's own tests pin it with
// ti.init(arch=ti.cpu, cpu_max_num_threads=1)), on the reference's AoS
// field layout: cell fields are C-order (nx, ny, nz[, comp]), particle
// fields are (n[, comp]).  The arithmetic type R is float (the reference's
// ti.f32 fields) or double (the FP64 oracle).  Citations are
// path:line into lizhuoh9/MPM-LBM.
//
// When compiled with -fopenmp and the `threads` argument of the *_mt entry
// points is > 1, the cell-parallel kernels run with OpenMP (timed CPU
// baseline); the scatter kernels then use atomics, so sums lose the
// single-thread order.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// D3Q19 velocity set, weights and opposite map: src/mpm_lbm/sim/lbm/fluid.py:252, 359-373
const int E[19][3] = {{0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                      {0, 0, 1},  {0, 0, -1},  {1, 1, 0},  {-1, -1, 0}, {1, -1, 0},
                      {-1, 1, 0}, {1, 0, 1},   {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1},
                      {0, 1, 1},  {0, -1, -1}, {0, 1, -1}, {0, -1, 1}};
const int LR[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
const double W[19] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                      1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
// Moment matrix M: src/mpm_lbm/sim/lbm/fluid.py:257-275
const int MM[19][19] = {
    {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {-1, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {1, -2, -2, -2, -2, -2, -2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1},
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, -2, 2, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0},
    {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, -2, 2, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
    {0, 0, 0, 0, 0, -2, 2, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1},
    {0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, -2, -2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2},
    {0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    {0, 0, 0, -1, -1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0},
    {0, 0, 0, 0, 0, 0, 0, -1, 1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1},
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1}};
const int UNKNOWN_XMIN[5] = {1, 7, 9, 11, 13};   // fluid.py:26
const int UNKNOWN_XMAX[5] = {2, 8, 10, 12, 14};  // fluid.py:27

}  // namespace

extern "C" {

// Open-boundary semantics codes (src/mpm_lbm/sim/lbm/fluid.py:16-25)
enum {
  ORC_OB_EQUILIBRIUM_RESET = 0,
  ORC_OB_REGULARIZED = 1,
  ORC_OB_REGULARIZED_LIMITED = 2,
  ORC_OB_CONVECTIVE = 3,
  ORC_OB_REG_MASS_BALANCED = 4,
  ORC_OB_CONV_MASS_BALANCED = 5,
  ORC_OB_REG_FLUX_MATCHED = 6,
  ORC_OB_CONV_FLUX_MATCHED = 7,
  ORC_OB_REG_PLANE_FLUX = 8,
  ORC_OB_CONV_PLANE_FLUX = 9,
};

// LBM parameters.  Mirrors LBMFluid3D.__init__/init_simulation
// (src/mpm_lbm/sim/lbm/fluid.py:33-317).
struct OrcLbmParams {
  int32_t nx, ny, nz;
  int32_t ob_semantics;
  double rho0;
  double force[3];         // fx, fy, fz (set_force, fluid.py:2025)
  double S[19];            // S_dig (fluid.py:304)
  double inv_M[361];       // np.linalg.inv(M) (fluid.py:250, 277)
  int32_t bc[6];           // bc_x_left, bc_x_right, bc_y_left, bc_y_right, bc_z_left, bc_z_right
  double rho_bc[6];        // rho_bcxl, rho_bcxr, ...
  double vel_bc[6][3];     // bc velocities; vel_bc[0] is bc_vel_x_left_dynamic
  int32_t limiter_enabled;
  int32_t floor_enabled;
  double ob_rho_min, ob_rho_max, ob_u_max, ob_noneq_cap, ob_floor;
  // outlet repair and flux controller (LBMConfig.open_boundary_*, lbm/config.py:53-69)
  double flux_gain_u, flux_gain_rho, flux_filter_alpha, flux_cap_u, flux_delta_cap_u, flux_slew_alpha;
  double convective_blend, flux_target_scale, drop_guard_min_ratio;
  double mn_gain, mn_cap, mn_blend;
  int32_t measure_plane_offset;
  int32_t drop_guard_enabled;
  int32_t mass_neutral;  // enabled with mode global_mass_error_density_offset
  int32_t pad_ob;
};

// Scalar LBM diagnostics (fluid.py:98-146, 212-223).
struct OrcLbmDiag {
  int32_t bb_link_count;
  int32_t pad0;
  double bb_max_correction;
  double bb_net_fluid_impulse[3];
  double bb_net_solid_force[3];
  int32_t bb_link_count_by_dir[19];
  int32_t pad1;
  double bb_fluid_impulse_by_dir[19][3];
  double bb_solid_force_by_dir[19][3];
  double bb_correction_abs_sum_by_dir[19];
  double bb_correction_abs_max_by_dir[19];
  int32_t mb_sample_count;
  int32_t pad2;
  double mb_accum_norm_max;
  double mb_mean_norm_max;
  // open-boundary limiter counters: [0]=step, [1]=run
  int32_t ob_rho_clip[2], ob_velocity_clip[2], ob_noneq_clip[2], ob_floor_count[2], ob_reconstructed[2];
  // outlet repair (fluid.py:98-118), [0] = step, [1] = run
  int32_t mb_corr_count[2];
  double mb_corr_abs_sum[2], pop_delta_abs_sum[2], flow_delta_abs_sum[2];
  double flow_err_filtered_run, flow_gain_effective_step;
  // plane-flux controller (fluid.py:119-146)
  double target_flux, measured_flux, fluid_area, true_outlet_flux, near_flux[3];
  double flux_err_filtered, u_feedback, rho_feedback, guard_reference;
  int32_t guard_active_step, guard_count_run, ctl_update[2], ctl_saturation[2];
  double mn_mass_current, mn_reference, mn_error, mn_rho_feedback;
  int32_t mn_initialized, mn_update[2], mn_saturation[2], pad_mn;
};

struct OrcMpmParams {
  int32_t n_grid;
  int32_t n_particles;
  int32_t bound;
  int32_t damping_enabled;
  int32_t lock_z;
  int32_t pad;
  double dx, inv_dx, dt, mu, la;
  double gravity[3];
  double damping;
};

struct OrcMpmStats {
  double min_x[3], max_x[3];
  double max_speed, min_J, max_J, total_mass;
};

struct OrcCouplingParams {
  int32_t n_grid;          // MPM grid edge (solid.inside_grid)
  int32_t pad;
  double inv_dx_norm;      // 1/dx_norm
  double cell_volume_norm; // dx_norm^3
  double vel_scale;        // lbm_dt_phys / dx_norm (projection.py:11)
  double eps_mass;         // 1e-12 (projection.py:12)
  double phi_min;
  double beta_lbm;
  double force_cap;        // force_cap_lbm (penalty) or force_cap_norm (moving boundary)
  double reaction_scale;
  double force_density_scale;  // dx_norm / lbm_dt_phys^2
  double area_scale;       // link-area transfer only (1 for engineering)
};

struct OrcCouplingStats {
  double projected_mass, projected_volume_raw, projected_volume_clamped, max_phi_raw;
  int32_t active_cell_count;
  int32_t active_force_cell_count;
  double max_cell_force_norm, max_hydro_force_norm;
  double net_cell_force[3], net_hydro_force[3];
  double max_reaction_grid_force_norm;
  double net_reaction_grid_force[3];
  int32_t active_reaction_particle_count;
  int32_t pad;
  double max_particle_reaction_norm;
  double max_grid_reaction_norm;
  double net_particle_reaction_force[3];
  double net_grid_reaction_force[3];
};

}  // extern "C"

namespace {

template <typename R>
struct Grid {
  int nx, ny, nz;
  inline int64_t id(int i, int j, int k) const { return ((int64_t)i * ny + j) * nz + k; }
  inline int64_t n() const { return (int64_t)nx * ny * nz; }
};

// fluid.py:320-326
template <typename R>
inline R feq(int s, R rho, const R u[3]) {
  R eu = (R)E[s][0] * u[0] + (R)E[s][1] * u[1] + (R)E[s][2] * u[2];
  R uv = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  return (R)W[s] * rho * ((R)1 + (R)3 * eu + (R)4.5 * eu * eu - (R)1.5 * uv);
}

template <typename R>
void lbm_init(const OrcLbmParams& p, R* f, R* F, R* rho, R* v) {
  // fluid.py:328-344 (both branches write the same values)
  Grid<R> g{p.nx, p.ny, p.nz};
  const R zero[3] = {0, 0, 0};
  for (int64_t c = 0; c < g.n(); ++c) {
    rho[c] = (R)p.rho0;
    v[c * 3 + 0] = v[c * 3 + 1] = v[c * 3 + 2] = 0;
    for (int s = 0; s < 19; ++s) {
      R q = feq<R>(s, (R)p.rho0, zero);
      f[c * 19 + s] = q;
      F[c * 19 + s] = q;
    }
  }
}

// fluid.py:398-413 (colission) with meq_vec 385-391 and cal_local_force 393-396
template <typename R>
void lbm_collide(const OrcLbmParams& p, const R* F, const R* rho, const R* v, const R* cell_force,
                 const int8_t* solid, R* f, int threads) {
  Grid<R> g{p.nx, p.ny, p.nz};
  R invM[19][19], S[19];
  for (int a = 0; a < 19; ++a) {
    S[a] = (R)p.S[a];
    for (int b = 0; b < 19; ++b) invM[a][b] = (R)p.inv_M[a * 19 + b];
  }
  const int64_t n = g.n();
#pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
  for (int64_t c = 0; c < n; ++c) {
    if (solid[c] != 0) continue;
    const R* Fc = F + c * 19;
    R m[19];
    for (int a = 0; a < 19; ++a) {
      R acc = (R)MM[a][0] * Fc[0];
      for (int b = 1; b < 19; ++b) acc += (R)MM[a][b] * Fc[b];
      m[a] = acc;
    }
    const R u[3] = {v[c * 3 + 0], v[c * 3 + 1], v[c * 3 + 2]};
    R meq[19] = {0};
    meq[0] = rho[c];
    meq[3] = u[0];
    meq[5] = u[1];
    meq[7] = u[2];
    meq[1] = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    meq[9] = (R)2 * u[0] * u[0] - u[1] * u[1] - u[2] * u[2];
    meq[11] = u[1] * u[1] - u[2] * u[2];
    meq[13] = u[0] * u[1];
    meq[14] = u[1] * u[2];
    meq[15] = u[0] * u[2];
    for (int a = 0; a < 19; ++a) m[a] -= S[a] * (m[a] - meq[a]);
    const R fo[3] = {(R)p.force[0] + cell_force[c * 3 + 0], (R)p.force[1] + cell_force[c * 3 + 1],
                     (R)p.force[2] + cell_force[c * 3 + 2]};
    R guo[19];
    for (int l = 0; l < 19; ++l) {
      R d0 = (R)E[l][0] - u[0], d1 = (R)E[l][1] - u[1], d2 = (R)E[l][2] - u[2];
      R a1 = d0 * fo[0] + d1 * fo[1] + d2 * fo[2];
      R eu = (R)E[l][0] * u[0] + (R)E[l][1] * u[1] + (R)E[l][2] * u[2];
      R ef = (R)E[l][0] * fo[0] + (R)E[l][1] * fo[1] + (R)E[l][2] * fo[2];
      guo[l] = (R)W[l] * (a1 / (R)3 + (eu * ef) / (R)9);
    }
    for (int a = 0; a < 19; ++a) {
      R acc = (R)MM[a][0] * guo[0];
      for (int b = 1; b < 19; ++b) acc += (R)MM[a][b] * guo[b];
      m[a] += ((R)1 - (R)0.5 * S[a]) * acc;
    }
    R* fc = f + c * 19;
    for (int a = 0; a < 19; ++a) {
      R acc = invM[a][0] * m[0];
      for (int b = 1; b < 19; ++b) acc += invM[a][b] * m[b];
      fc[a] = (R)0 + acc;
    }
  }
}

inline int wrap(int i, int n) { return i < 0 ? n - 1 : (i > n - 1 ? 0 : i); }  // fluid.py:419-429

// fluid.py:431-440 (streaming1, moving=0) and 488-519 (streaming_moving_bounceback, moving=1),
// including clear_moving_boundary_diagnostics 443-458 and finalize 521-536 when moving.
template <typename R>
void lbm_stream_mt(const OrcLbmParams& p, int moving, const R* f, R* F, const int8_t* solid, const R* rho,
                   const R* solid_vel, R* hydro_force, OrcLbmDiag* d, int threads);

template <typename R>
void lbm_stream(const OrcLbmParams& p, int moving, const R* f, R* F, const int8_t* solid, const R* rho,
                const R* solid_vel, R* hydro_force, OrcLbmDiag* d, int threads = 1) {
  if (threads > 1) {
    lbm_stream_mt<R>(p, moving, f, F, solid, rho, solid_vel, hydro_force, d, threads);
    return;
  }
  Grid<R> g{p.nx, p.ny, p.nz};
  R link_fluid[19][3], link_solid[19][3], corr_sum[19], corr_max[19], max_corr = 0;
  R net_fluid[3] = {0, 0, 0}, net_solid[3] = {0, 0, 0};
  int count[19];
  if (moving) {
    for (int s = 0; s < 19; ++s) {
      count[s] = 0;
      corr_sum[s] = corr_max[s] = 0;
      for (int a = 0; a < 3; ++a) link_fluid[s][a] = link_solid[s][a] = 0;
    }
    std::memset(hydro_force, 0, sizeof(R) * 3 * g.n());
  }
  int total = 0;
  for (int i = 0; i < p.nx; ++i)
    for (int j = 0; j < p.ny; ++j)
      for (int k = 0; k < p.nz; ++k) {
        const int64_t c = g.id(i, j, k);
        if (solid[c] != 0) continue;
        for (int s = 0; s < 19; ++s) {
          const int ii = wrap(i + E[s][0], p.nx), jj = wrap(j + E[s][1], p.ny), kk = wrap(k + E[s][2], p.nz);
          const int64_t ip = g.id(ii, jj, kk);
          if (solid[ip] == 0) {
            F[ip * 19 + s] = f[c * 19 + s];
          } else if (!moving) {
            F[c * 19 + LR[s]] = f[c * 19 + s];
          } else {
            const R rl = rho[c];
            const R* uw = solid_vel + ip * 3;
            const R eu = (R)E[s][0] * uw[0] + (R)E[s][1] * uw[1] + (R)E[s][2] * uw[2];
            const R correction = (R)-6.0 * (R)W[s] * rl * eu;
            const R bounced = f[c * 19 + s] + correction;
            F[c * 19 + LR[s]] = bounced;
            R fi[3], sf[3];
            for (int a = 0; a < 3; ++a) {
              const R inc = (R)E[s][a] * f[c * 19 + s];
              const R out = (R)E[LR[s]][a] * bounced;
              fi[a] = out - inc;
              sf[a] = -fi[a];
            }
            const R ac = std::fabs(correction);
            total += 1;
            max_corr = std::max(max_corr, ac);
            count[s] += 1;
            corr_sum[s] += ac;
            corr_max[s] = std::max(corr_max[s], ac);
            for (int a = 0; a < 3; ++a) {
              net_fluid[a] += fi[a];
              net_solid[a] += sf[a];
              hydro_force[ip * 3 + a] += sf[a];
              link_fluid[s][a] += fi[a];
              link_solid[s][a] += sf[a];
            }
          }
        }
      }
  if (!moving) return;
  // finalize_moving_boundary_diagnostics (fluid.py:521-536)
  int lc = 0;
  R fluid_sum[3] = {0, 0, 0}, solid_sum[3] = {0, 0, 0}, mc = 0;
  for (int s = 0; s < 19; ++s) {
    lc += count[s];
    for (int a = 0; a < 3; ++a) {
      fluid_sum[a] += link_fluid[s][a];
      solid_sum[a] += link_solid[s][a];
    }
    mc = std::max(mc, corr_max[s]);
  }
  (void)total;
  (void)max_corr;
  (void)net_fluid;
  (void)net_solid;
  d->bb_link_count = lc;
  d->bb_max_correction = (double)mc;
  for (int a = 0; a < 3; ++a) {
    d->bb_net_fluid_impulse[a] = (double)fluid_sum[a];
    d->bb_net_solid_force[a] = (double)solid_sum[a];
  }
  for (int s = 0; s < 19; ++s) {
    d->bb_link_count_by_dir[s] = count[s];
    d->bb_correction_abs_sum_by_dir[s] = (double)corr_sum[s];
    d->bb_correction_abs_max_by_dir[s] = (double)corr_max[s];
    for (int a = 0; a < 3; ++a) {
      d->bb_fluid_impulse_by_dir[s][a] = (double)link_fluid[s][a];
      d->bb_solid_force_by_dir[s][a] = (double)link_solid[s][a];
    }
  }
}

// Same as lbm_stream, parallel over x-slices for the timed CPU baseline; the
// diagnostic sums use per-thread partials and hydro_force uses atomics, so
// their summation order differs from the single-thread restatement.
template <typename R>
void lbm_stream_mt(const OrcLbmParams& p, int moving, const R* f, R* F, const int8_t* solid, const R* rho,
                   const R* solid_vel, R* hydro_force, OrcLbmDiag* d, int threads) {
  Grid<R> g{p.nx, p.ny, p.nz};
  if (moving) std::memset(hydro_force, 0, sizeof(R) * 3 * g.n());
  int count[19] = {0};
  R csum[19] = {0}, cmax[19] = {0}, imp[19][3] = {{0}};
#pragma omp parallel num_threads(threads)
  {
    int lcount[19] = {0};
    R lsum[19] = {0}, lmax[19] = {0}, limp[19][3] = {{0}};
#pragma omp for schedule(static)
    for (int i = 0; i < p.nx; ++i)
      for (int j = 0; j < p.ny; ++j)
        for (int k = 0; k < p.nz; ++k) {
          const int64_t c = g.id(i, j, k);
          if (solid[c] != 0) continue;
          for (int s = 0; s < 19; ++s) {
            const int64_t ip = g.id(wrap(i + E[s][0], p.nx), wrap(j + E[s][1], p.ny), wrap(k + E[s][2], p.nz));
            if (solid[ip] == 0) {
              F[ip * 19 + s] = f[c * 19 + s];
            } else if (!moving) {
              F[c * 19 + LR[s]] = f[c * 19 + s];
            } else {
              const R* uw = solid_vel + ip * 3;
              const R eu = (R)E[s][0] * uw[0] + (R)E[s][1] * uw[1] + (R)E[s][2] * uw[2];
              const R corr = (R)-6.0 * (R)W[s] * rho[c] * eu;
              const R b = f[c * 19 + s] + corr;
              F[c * 19 + LR[s]] = b;
              const R ac = std::fabs(corr);
              lcount[s] += 1;
              lsum[s] += ac;
              lmax[s] = std::max(lmax[s], ac);
              for (int a = 0; a < 3; ++a) {
                const R fi = (R)E[LR[s]][a] * b - (R)E[s][a] * f[c * 19 + s];
                limp[s][a] += fi;
#pragma omp atomic
                hydro_force[ip * 3 + a] += -fi;
              }
            }
          }
        }
#pragma omp critical
    for (int s = 0; s < 19; ++s) {
      count[s] += lcount[s];
      csum[s] += lsum[s];
      cmax[s] = std::max(cmax[s], lmax[s]);
      for (int a = 0; a < 3; ++a) imp[s][a] += limp[s][a];
    }
  }
  if (!moving) return;
  int lc = 0;
  R fsum[3] = {0, 0, 0}, mc = 0;
  for (int s = 0; s < 19; ++s) {
    lc += count[s];
    mc = std::max(mc, cmax[s]);
    d->bb_link_count_by_dir[s] = count[s];
    d->bb_correction_abs_sum_by_dir[s] = (double)csum[s];
    d->bb_correction_abs_max_by_dir[s] = (double)cmax[s];
    for (int a = 0; a < 3; ++a) {
      fsum[a] += imp[s][a];
      d->bb_fluid_impulse_by_dir[s][a] = (double)imp[s][a];
      d->bb_solid_force_by_dir[s][a] = -(double)imp[s][a];
    }
  }
  d->bb_link_count = lc;
  d->bb_max_correction = (double)mc;
  for (int a = 0; a < 3; ++a) {
    d->bb_net_fluid_impulse[a] = (double)fsum[a];
    d->bb_net_solid_force[a] = -(double)fsum[a];
  }
}

// fluid.py:1026-1029
template <typename R>
inline R regularized_population(const OrcLbmParams&, int s, R target_rho, const R tu[3], const R* F, const R* rho,
                                const R* v, int64_t n) {
  const R nu[3] = {v[n * 3 + 0], v[n * 3 + 1], v[n * 3 + 2]};
  const R noneq = F[n * 19 + s] - feq<R>(s, rho[n], nu);
  return feq<R>(s, target_rho, tu) + noneq;
}

// fluid.py:1059-1096
template <typename R>
inline R limited_regularized_population(const OrcLbmParams& p, int s, R target_rho, const R tu[3], const R* F,
                                        const R* rho, const R* v, int64_t n, OrcLbmDiag* d) {
  R rl = target_rho;
  R ul[3] = {tu[0], tu[1], tu[2]};
  if (p.limiter_enabled) {
    d->ob_reconstructed[0]++;
    d->ob_reconstructed[1]++;
    if (rl < (R)p.ob_rho_min) {
      rl = (R)p.ob_rho_min;
      d->ob_rho_clip[0]++;
      d->ob_rho_clip[1]++;
    }
    if (rl > (R)p.ob_rho_max) {
      rl = (R)p.ob_rho_max;
      d->ob_rho_clip[0]++;
      d->ob_rho_clip[1]++;
    }
    const R norm = std::sqrt(ul[0] * ul[0] + ul[1] * ul[1] + ul[2] * ul[2]);
    if (norm > (R)p.ob_u_max) {
      const R sc = (R)p.ob_u_max / norm;
      ul[0] *= sc;
      ul[1] *= sc;
      ul[2] *= sc;
      d->ob_velocity_clip[0]++;
      d->ob_velocity_clip[1]++;
    }
  }
  const R nu[3] = {v[n * 3 + 0], v[n * 3 + 1], v[n * 3 + 2]};
  R noneq = F[n * 19 + s] - feq<R>(s, rho[n], nu);
  if (p.limiter_enabled) {
    if (noneq > (R)p.ob_noneq_cap) {
      noneq = (R)p.ob_noneq_cap;
      d->ob_noneq_clip[0]++;
      d->ob_noneq_clip[1]++;
    }
    if (noneq < -(R)p.ob_noneq_cap) {
      noneq = -(R)p.ob_noneq_cap;
      d->ob_noneq_clip[0]++;
      d->ob_noneq_clip[1]++;
    }
  }
  R out = feq<R>(s, rl, ul) + noneq;
  if (p.limiter_enabled && p.floor_enabled) {
    if (out < (R)p.ob_floor) {
      out = (R)p.ob_floor;
      d->ob_floor_count[0]++;
      d->ob_floor_count[1]++;
    }
  }
  return out;
}

// fluid.py:1050-1057 and 1098-1103
template <typename R>
inline R convective_outlet_population(const OrcLbmParams& p, int s, int64_t n1, int64_t n2, const R* F,
                                      const int8_t* solid) {
  R ex = F[n1 * 19 + s];
  if (solid[n2] == 0) ex = (R)2 * F[n1 * 19 + s] - F[n2 * 19 + s];
  if (p.limiter_enabled && p.floor_enabled && ex < (R)p.ob_floor) ex = (R)p.ob_floor;
  return ex;
}

// fluid.py:1105-1112
template <typename R>
inline R bounded_scalar(R value, R limit) {
  R out = value;
  if (out > limit) out = limit;
  if (out < -limit) out = -limit;
  return out;
}

// _limit_open_boundary_population (fluid.py:1043-1049)
template <typename R>
inline R limit_population(const OrcLbmParams& p, R value) {
  if (p.limiter_enabled && p.floor_enabled && value < (R)p.ob_floor) return (R)p.ob_floor;
  return value;
}

// The repair and flow-correction fields one Boundary_condition call updates,
// held in R (the reference's ti.f32 fields take each record in order).
template <typename R>
struct RepairRec {
  int count[2];
  R corr[2], delta[2], flow_delta[2], filtered, gain_step;
};

// fluid.py:1114-1120
template <typename R>
inline void record_repair(RepairRec<R>& r, R corr, R delta) {
  for (int a = 0; a < 2; ++a) {
    r.count[a] += 1;
    r.corr[a] += corr;
    r.delta[a] += delta;
  }
}

// fluid.py:1122-1131
template <typename R>
inline void record_flow(const OrcLbmParams& p, RepairRec<R>& r, R corr, R err) {
  r.flow_delta[0] += corr;
  r.flow_delta[1] += corr;
  r.filtered = ((R)1 - (R)p.flux_filter_alpha) * r.filtered + (R)p.flux_filter_alpha * err;
  r.gain_step = (R)p.flux_gain_u;
}

// fluid.py:1133-1138
template <typename R>
inline void record_plane(const OrcLbmParams& p, RepairRec<R>& r, R corr, R delta) {
  record_repair(r, corr, delta);
  r.flow_delta[0] += corr;
  r.flow_delta[1] += corr;
  r.gain_step = (R)p.flux_gain_u;
}

// The regularized outlet population of semantics 4, 6, 8 (fluid.py:1265-1274,
// 1286-1304, 1318-1335): target density rho_bcxr and velocity v[ni] repaired
// by the semantics' feedback, the neighbour's non-equilibrium part kept.
template <typename R>
R repaired_regularized(const OrcLbmParams& p, int kind, RepairRec<R>& r, int s, const R* F, const R* rho,
                       const R* v, int64_t n, const OrcLbmDiag* d) {
  const R target_rho = (R)p.rho_bc[1];
  const R tu[3] = {v[n * 3], v[n * 3 + 1], v[n * 3 + 2]};
  const R vx_in = (R)p.vel_bc[0][0];
  R rho_fb, vel_fb, extra = 0;
  if (kind == ORC_OB_REG_MASS_BALANCED) {
    rho_fb = bounded_scalar<R>((R)0.02 * ((R)p.rho0 - rho[n]), (R)0.01);
    vel_fb = bounded_scalar<R>((R)0.05 * (vx_in - tu[0]), (R)0.02);
  } else if (kind == ORC_OB_REG_FLUX_MATCHED) {
    rho_fb = bounded_scalar<R>((R)p.flux_gain_rho * ((R)p.rho0 - rho[n]), (R)0.01);
    vel_fb = bounded_scalar<R>((R)p.flux_gain_u * (vx_in - tu[0]), (R)p.flux_cap_u);
  } else {
    rho_fb = (R)d->rho_feedback;
    if (p.ob_semantics == ORC_OB_REG_PLANE_FLUX && p.mass_neutral) extra = (R)d->mn_rho_feedback;
    vel_fb = (R)d->u_feedback;
  }
  const R ru[3] = {tu[0] + vel_fb, tu[1], tu[2]};
  const R before = regularized_population<R>(p, s, target_rho, tu, F, rho, v, n);
  const R after = regularized_population<R>(p, s, target_rho + rho_fb + extra, ru, F, rho, v, n);
  if (kind == ORC_OB_REG_MASS_BALANCED) {
    record_repair<R>(r, std::fabs(rho_fb) + std::fabs(vel_fb), std::fabs(after - before));
  } else if (kind == ORC_OB_REG_FLUX_MATCHED) {
    record_repair<R>(r, std::fabs(rho_fb) + std::fabs(vel_fb), std::fabs(after - before));
    record_flow<R>(p, r, std::fabs(vel_fb), vx_in - tu[0]);
  } else {
    record_plane<R>(p, r, std::fabs(rho_fb) + std::fabs(extra) + std::fabs(vel_fb), std::fabs(after - before));
  }
  return limit_population<R>(p, after);
}

// One unknown population of a pressure-outlet face cell under semantics 4-9
// (fluid.py:1265-1346); the convective variants blend the extrapolation of
// fluid.py:1098-1103 toward the regularized repair.
template <typename R>
R repaired_outlet_population(const OrcLbmParams& p, RepairRec<R>& r, int s, int64_t n, int64_t n2, const R* F,
                             const R* rho, const R* v, const int8_t* solid, const OrcLbmDiag* d) {
  const int sem = p.ob_semantics;
  const int kind = sem == ORC_OB_CONV_MASS_BALANCED ? ORC_OB_REG_MASS_BALANCED
                   : sem == ORC_OB_CONV_FLUX_MATCHED ? ORC_OB_REG_FLUX_MATCHED
                   : sem == ORC_OB_CONV_PLANE_FLUX  ? ORC_OB_REG_PLANE_FLUX
                                                    : sem;
  if (kind == sem) return repaired_regularized<R>(p, kind, r, s, F, rho, v, n, d);
  const R convective = convective_outlet_population<R>(p, s, n, n2, F, solid);
  const R regularized = repaired_regularized<R>(p, kind, r, s, F, rho, v, n, d);
  const R blend = sem == ORC_OB_CONV_MASS_BALANCED ? (R)0.15 : (R)p.convective_blend;
  const R repaired = convective + blend * (regularized - convective);
  const R dd = std::fabs(repaired - convective);
  if (sem == ORC_OB_CONV_MASS_BALANCED) {
    record_repair<R>(r, (R)0, dd);
  } else if (sem == ORC_OB_CONV_FLUX_MATCHED) {
    record_repair<R>(r, (R)0, dd);
    record_flow<R>(p, r, dd, (R)p.vel_bc[0][0] - v[n * 3]);
  } else {
    record_plane<R>(p, r, dd, dd);
  }
  return limit_population<R>(p, repaired);
}

// update_open_boundary_plane_flux_controller (fluid.py:1141-1263), in the
// reference's loop order with R accumulators.
template <typename R>
void plane_flux_controller(const OrcLbmParams& p, const R* rho, const R* v, const int8_t* solid, OrcLbmDiag* d) {
  Grid<R> g{p.nx, p.ny, p.nz};
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  R target = 0, measured = 0, area = 0, near1 = 0, near2 = 0, near3 = 0, true_out = 0;
  d->guard_active_step = 0;
  d->guard_reference = 0;
  const int mi = std::max(0, nx - 1 - p.measure_plane_offset);
  const int i1 = std::max(0, nx - 2), i2 = std::max(0, nx - 3), i3 = std::max(0, nx - 4);
  auto flux = [&](int i, int j, int k) {
    const int64_t c = g.id(i, j, k);
    return rho[c] * v[c * 3];
  };
  for (int j = 0; j < ny; ++j)
    for (int k = 0; k < nz; ++k) {
      if (solid[g.id(0, j, k)] == 0) target += flux(0, j, k);
      if (solid[g.id(mi, j, k)] == 0) {
        measured += flux(mi, j, k);
        area += (R)1;
      }
      if (solid[g.id(nx - 1, j, k)] == 0) true_out += flux(nx - 1, j, k);
      if (solid[g.id(i1, j, k)] == 0) near1 += flux(i1, j, k);
      if (solid[g.id(i2, j, k)] == 0) near2 += flux(i2, j, k);
      if (solid[g.id(i3, j, k)] == 0) near3 += flux(i3, j, k);
    }
  target = (R)p.flux_target_scale * target;
  if (area <= (R)0) area = (R)1;
  d->target_flux = (double)target;
  d->measured_flux = (double)measured;
  d->fluid_area = (double)area;
  d->true_outlet_flux = (double)true_out;
  d->near_flux[0] = (double)near1;
  d->near_flux[1] = (double)near2;
  d->near_flux[2] = (double)near3;
  const R raw = target - measured;
  const R filtered = ((R)1 - (R)p.flux_filter_alpha) * (R)d->flux_err_filtered + (R)p.flux_filter_alpha * raw;
  d->flux_err_filtered = (double)filtered;
  d->flow_err_filtered_run = (double)filtered;
  const R requested = (R)p.flux_gain_u * filtered / area;
  const R bounded = bounded_scalar<R>(requested, (R)p.flux_cap_u);
  const R previous = (R)d->u_feedback;
  R limited = bounded;
  if ((R)p.flux_delta_cap_u > (R)0) limited = previous + bounded_scalar<R>(bounded - previous, (R)p.flux_delta_cap_u);
  R next = previous + (R)p.flux_slew_alpha * (limited - previous);
  if (p.drop_guard_enabled) {
    const R reference = std::max(std::fabs(target), std::fabs(measured));
    d->guard_reference = (double)reference;
    const R outlet = std::fabs(true_out);
    if (reference > (R)1.0e-12 && outlet < (R)p.drop_guard_min_ratio * reference && next < previous) {
      next = previous;
      d->guard_active_step = 1;
      d->guard_count_run += 1;
    }
  }
  d->u_feedback = (double)next;
  d->rho_feedback = (double)bounded_scalar<R>((R)p.flux_gain_rho * filtered / area, (R)0.01);
  if (p.mass_neutral) {
    // the fluid mass in FP64 (the reference's f32 atomic sum depends on the
    // order of its parallel loop; FP64 makes the sum order-independent), then
    // rounded to R like the reference's field
    double mass_d = 0.0;
    for (int64_t c = 0; c < g.n(); ++c)
      if (solid[c] == 0) mass_d += (double)rho[c];
    const R mass = (R)mass_d;
    d->mn_mass_current = (double)mass;
    if (d->mn_initialized == 0) {
      R reference = mass;
      if (std::fabs(reference) <= (R)1.0e-12) reference = (R)1;
      d->mn_reference = (double)reference;
      d->mn_initialized = 1;
    }
    R reference = (R)d->mn_reference;
    if (std::fabs(reference) <= (R)1.0e-12) {
      reference = (R)1;
      d->mn_reference = 1.0;
    }
    const R err = (mass - reference) / reference;
    const R raw_fb = -(R)p.mn_gain * err;
    const R bounded_fb = bounded_scalar<R>(raw_fb, (R)p.mn_cap);
    d->mn_error = (double)err;
    d->mn_rho_feedback = (double)((R)p.mn_blend * bounded_fb);
    d->mn_update[0] = 1;
    d->mn_update[1] += 1;
    if (std::fabs(raw_fb - bounded_fb) > (R)1.0e-12) {
      d->mn_saturation[0] = 1;
      d->mn_saturation[1] += 1;
    }
  }
  d->flow_gain_effective_step = (double)(R)p.flux_gain_u;
  d->ctl_update[0] = 1;
  d->ctl_update[1] += 1;
  if (std::fabs(requested - bounded) > (R)1.0e-12) {
    d->ctl_saturation[0] = 1;
    d->ctl_saturation[1] += 1;
  }
}

// Boundary_condition dispatch (fluid.py:538-569): legacy 926-1024,
// regularized 1348-1394, regularized-limited 1396-1442, convective 1444-1493,
// and the outlet repairs of 1495-1792 (inlets and velocity outlets are the
// plain regularized ones there).
template <typename R>
void lbm_boundary(const OrcLbmParams& p, R* F, const R* rho, const R* v, const int8_t* solid, OrcLbmDiag* d) {
  Grid<R> g{p.nx, p.ny, p.nz};
  // clear_open_boundary_limiter_step_counters (fluid.py:571-587)
  d->ob_rho_clip[0] = d->ob_velocity_clip[0] = d->ob_noneq_clip[0] = d->ob_floor_count[0] = 0;
  d->ob_reconstructed[0] = 0;
  d->mb_corr_count[0] = 0;
  d->mb_corr_abs_sum[0] = d->pop_delta_abs_sum[0] = d->flow_delta_abs_sum[0] = 0;
  d->flow_gain_effective_step = 0;
  d->ctl_saturation[0] = d->ctl_update[0] = d->mn_saturation[0] = d->mn_update[0] = 0;
  d->guard_active_step = 0;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  if (p.ob_semantics >= ORC_OB_REG_PLANE_FLUX) plane_flux_controller<R>(p, rho, v, solid, d);
  if (p.ob_semantics == ORC_OB_EQUILIBRIUM_RESET) {
    // x faces
    if (p.bc[0] == 1)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int64_t c = g.id(0, j, k);
          if (solid[c] != 0) continue;
          const int64_t src = solid[g.id(1, j, k)] > 0 ? g.id(1, j, k) : c;
          const R u[3] = {v[src * 3], v[src * 3 + 1], v[src * 3 + 2]};
          for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)p.rho_bc[0], u);
        }
    if (p.bc[0] == 2)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int64_t c = g.id(0, j, k);
          if (solid[c] != 0) continue;
          const R u[3] = {(R)p.vel_bc[0][0], (R)p.vel_bc[0][1], (R)p.vel_bc[0][2]};
          for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)1, u);
        }
    if (p.bc[1] == 1)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int64_t c = g.id(nx - 1, j, k);
          if (solid[c] != 0) continue;
          const int64_t src = g.id(nx - 2, j, k);  // both branches of fluid.py:947-951 use v[nx-2]
          const R u[3] = {v[src * 3], v[src * 3 + 1], v[src * 3 + 2]};
          for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)p.rho_bc[1], u);
        }
    if (p.bc[1] == 2)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          const int64_t c = g.id(nx - 1, j, k);
          if (solid[c] != 0) continue;
          const R u[3] = {(R)p.vel_bc[1][0], (R)p.vel_bc[1][1], (R)p.vel_bc[1][2]};
          for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)1, u);
        }
    // y faces (fluid.py:961-991)
    if (p.bc[2] == 1 || p.bc[2] == 2 || p.bc[3] == 1 || p.bc[3] == 2 || p.bc[4] == 1 || p.bc[4] == 2 ||
        p.bc[5] == 1 || p.bc[5] == 2) {
      for (int face = 2; face < 6; ++face) {
        if (p.bc[face] != 1 && p.bc[face] != 2) continue;
        const int axis = face / 2;
        const bool hi = face % 2;
        const int na = axis == 1 ? ny : nz;
        const int nb1 = axis == 1 ? nx : nx;
        const int nb2 = axis == 1 ? nz : ny;
        for (int a = 0; a < nb1; ++a)
          for (int b = 0; b < nb2; ++b) {
            int ijk[3], in1[3];
            ijk[0] = a;
            ijk[axis] = hi ? na - 1 : 0;
            ijk[axis == 1 ? 2 : 1] = b;
            in1[0] = ijk[0];
            in1[1] = ijk[1];
            in1[2] = ijk[2];
            in1[axis] = hi ? na - 2 : 1;
            const int64_t c = g.id(ijk[0], ijk[1], ijk[2]);
            if (solid[c] != 0) continue;
            if (p.bc[face] == 1) {
              const int64_t src = solid[g.id(in1[0], in1[1], in1[2])] > 0 ? g.id(in1[0], in1[1], in1[2]) : c;
              const R u[3] = {v[src * 3], v[src * 3 + 1], v[src * 3 + 2]};
              for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)p.rho_bc[face], u);
            } else {
              const R u[3] = {(R)p.vel_bc[face][0], (R)p.vel_bc[face][1], (R)p.vel_bc[face][2]};
              for (int s = 0; s < 19; ++s) F[c * 19 + s] = feq<R>(s, (R)1, u);
            }
          }
      }
    }
    return;
  }
  // x-axis open boundaries reconstructing only the unknown populations
  const bool limited = p.ob_semantics == ORC_OB_REGULARIZED_LIMITED;
  const bool convective = p.ob_semantics == ORC_OB_CONVECTIVE;
  const bool repaired = p.ob_semantics >= ORC_OB_REG_MASS_BALANCED;
  RepairRec<R> rec;
  for (int a = 0; a < 2; ++a) {
    rec.count[a] = d->mb_corr_count[a];
    rec.corr[a] = (R)d->mb_corr_abs_sum[a];
    rec.delta[a] = (R)d->pop_delta_abs_sum[a];
    rec.flow_delta[a] = (R)d->flow_delta_abs_sum[a];
  }
  rec.filtered = (R)d->flow_err_filtered_run;
  rec.gain_step = (R)d->flow_gain_effective_step;
  for (int side = 0; side < 2; ++side) {
    const int bc = p.bc[side];
    if (bc != 1 && bc != 2) continue;
    const int bi = side == 0 ? 0 : nx - 1;
    const int* unknown = side == 0 ? UNKNOWN_XMIN : UNKNOWN_XMAX;
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const int64_t c = g.id(bi, j, k);
        if (solid[c] != 0) continue;
        int ni = side == 0 ? 1 : nx - 2;
        int n2i = nx - 3;
        if (solid[g.id(ni, j, k)] > 0) {
          ni = bi;
          n2i = bi;
        }
        const int64_t n = g.id(ni, j, k);
        if (repaired && side == 1 && bc == 1) {
          const int64_t n2 = g.id(n2i, j, k);
          for (int q = 0; q < 5; ++q)
            F[c * 19 + unknown[q]] = repaired_outlet_population<R>(p, rec, unknown[q], n, n2, F, rho, v, solid, d);
          continue;
        }
        if (convective && side == 1 && bc == 1) {
          const int64_t n2 = g.id(n2i, j, k);
          for (int q = 0; q < 5; ++q) F[c * 19 + unknown[q]] = convective_outlet_population<R>(p, unknown[q], n, n2, F, solid);
          continue;
        }
        R target_rho;
        R tu[3];
        if (bc == 1) {
          target_rho = (R)p.rho_bc[side];
          tu[0] = v[n * 3];
          tu[1] = v[n * 3 + 1];
          tu[2] = v[n * 3 + 2];
        } else {
          target_rho = rho[n];
          if (target_rho <= (R)1.0e-6) target_rho = (R)p.rho0;
          tu[0] = (R)p.vel_bc[side][0];
          tu[1] = (R)p.vel_bc[side][1];
          tu[2] = (R)p.vel_bc[side][2];
        }
        for (int q = 0; q < 5; ++q) {
          const int s = unknown[q];
          F[c * 19 + s] = limited ? limited_regularized_population<R>(p, s, target_rho, tu, F, rho, v, n, d)
                                  : regularized_population<R>(p, s, target_rho, tu, F, rho, v, n);
        }
      }
  }
  for (int a = 0; a < 2; ++a) {
    d->mb_corr_count[a] = rec.count[a];
    d->mb_corr_abs_sum[a] = (double)rec.corr[a];
    d->pop_delta_abs_sum[a] = (double)rec.delta[a];
    d->flow_delta_abs_sum[a] = (double)rec.flow_delta[a];
  }
  d->flow_err_filtered_run = (double)rec.filtered;
  d->flow_gain_effective_step = (double)rec.gain_step;
}

// fluid.py:1794-1814
template <typename R>
void lbm_macros(const OrcLbmParams& p, R* f, const R* F, R* rho, R* v, const int8_t* solid, const R* cell_force,
                int threads) {
  Grid<R> g{p.nx, p.ny, p.nz};
  const int64_t n = g.n();
#pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
  for (int64_t c = 0; c < n; ++c) {
    if (solid[c] == 0) {
      R sum = 0;
      for (int s = 0; s < 19; ++s) {
        f[c * 19 + s] = F[c * 19 + s];
        sum += F[c * 19 + s];
      }
      const R r = (R)0 + sum;
      R u[3] = {0, 0, 0};
      for (int s = 0; s < 19; ++s)
        for (int a = 0; a < 3; ++a) u[a] += (R)E[s][a] * F[c * 19 + s];
      for (int a = 0; a < 3; ++a) {
        const R fo = (R)p.force[a] + cell_force[c * 3 + a];
        u[a] /= r;
        u[a] += (fo / (R)2) / r;
        v[c * 3 + a] = u[a];
      }
      rho[c] = r;
    } else {
      rho[c] = (R)p.rho0;
      v[c * 3] = v[c * 3 + 1] = v[c * 3 + 2] = 0;
    }
  }
}

// fluid.py:1847-1861
template <typename R>
void lbm_update_dynamic_solid(const OrcLbmParams& p, double threshold, int8_t* solid, const int8_t* static_solid,
                              int8_t* old_solid, const R* solid_phi, int8_t* reinit) {
  Grid<R> g{p.nx, p.ny, p.nz};
  const R thr = (R)threshold;
  for (int64_t c = 0; c < g.n(); ++c) {
    const int8_t prev = solid[c];
    old_solid[c] = prev;
    const bool dyn = solid_phi[c] >= thr;
    const int8_t ns = (static_solid[c] != 0 || dyn) ? 1 : 0;
    solid[c] = ns;
    reinit[c] = (prev != 0 && ns == 0) ? 1 : 0;
  }
}

// fluid.py:1863-1877
template <typename R>
void lbm_reinit(const OrcLbmParams& p, int8_t* reinit, const R* solid_vel, R* rho, R* v, R* f, R* F) {
  Grid<R> g{p.nx, p.ny, p.nz};
  for (int64_t c = 0; c < g.n(); ++c) {
    if (reinit[c] != 1) continue;
    R u[3] = {0, 0, 0};
    const R* sv = solid_vel + c * 3;
    if (std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]) > (R)0) {
      u[0] = sv[0];
      u[1] = sv[1];
      u[2] = sv[2];
    }
    rho[c] = (R)p.rho0;
    v[c * 3] = u[0];
    v[c * 3 + 1] = u[1];
    v[c * 3 + 2] = u[2];
    for (int s = 0; s < 19; ++s) {
      const R q = feq<R>(s, (R)p.rho0, u);
      f[c * 19 + s] = q;
      F[c * 19 + s] = q;
    }
    reinit[c] = 0;
  }
}

// fluid.py:460-486.  op: 0 clear, 1 accumulate, 2 finalize
template <typename R>
void lbm_force_accumulator(const OrcLbmParams& p, int op, R* hydro_force, R* accum, OrcLbmDiag* d) {
  Grid<R> g{p.nx, p.ny, p.nz};
  const int64_t n = g.n();
  if (op == 0) {
    d->mb_sample_count = 0;
    d->mb_accum_norm_max = 0;
    d->mb_mean_norm_max = 0;
    std::memset(accum, 0, sizeof(R) * 3 * n);
  } else if (op == 1) {
    d->mb_sample_count += 1;
    R mx = (R)d->mb_accum_norm_max;
    for (int64_t c = 0; c < n; ++c) {
      for (int a = 0; a < 3; ++a) accum[c * 3 + a] += hydro_force[c * 3 + a];
      const R* q = accum + c * 3;
      mx = std::max(mx, (R)std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
    }
    d->mb_accum_norm_max = (double)mx;
  } else {
    d->mb_mean_norm_max = 0;
    const int cnt = d->mb_sample_count;
    R inv = 0;
    if (cnt > 0) inv = (R)1 / (R)cnt;
    R mx = 0;
    for (int64_t c = 0; c < n; ++c) {
      if (cnt > 0) {
        R m[3];
        for (int a = 0; a < 3; ++a) {
          m[a] = accum[c * 3 + a] * inv;
          hydro_force[c * 3 + a] = m[a];
        }
        mx = std::max(mx, (R)std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]));
      }
    }
    d->mb_mean_norm_max = (double)mx;
  }
}

// ---------------------------------------------------------------- MPM ----
// 3x3 helpers in double (the polar rotation is computed in FP64).
struct M3 {
  double a[3][3];
};
inline M3 mul(const M3& A, const M3& B) {
  M3 C;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C.a[i][j] = A.a[i][0] * B.a[0][j] + A.a[i][1] * B.a[1][j] + A.a[i][2] * B.a[2][j];
  return C;
}
inline M3 transpose(const M3& A) {
  M3 T;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T.a[i][j] = A.a[j][i];
  return T;
}
inline double det(const M3& A) {
  return A.a[0][0] * (A.a[1][1] * A.a[2][2] - A.a[1][2] * A.a[2][1]) -
         A.a[0][1] * (A.a[1][0] * A.a[2][2] - A.a[1][2] * A.a[2][0]) +
         A.a[0][2] * (A.a[1][0] * A.a[2][1] - A.a[1][1] * A.a[2][0]);
}

// Proper rotation of the polar decomposition F = R S (R = U V^T with det U =
// det V = +1; the smallest singular value carries the sign of det F), the
// quantity the reference takes from ti.svd (mpm/solid.py:233-234).  Method:
// cyclic Jacobi eigen-decomposition of F^T F for V (Golub & Van Loan, 8.5),
// then Givens QR of F V for U (the structure of McAdams et al. 2011,
// "Computing the SVD of 3x3 matrices with minimal branching").
M3 polar_rotation(const M3& F) {
  M3 A = mul(transpose(F), F);
  M3 V{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
  for (int sweep = 0; sweep < 40; ++sweep) {
    const double off = A.a[0][1] * A.a[0][1] + A.a[0][2] * A.a[0][2] + A.a[1][2] * A.a[1][2];
    const double diag = A.a[0][0] * A.a[0][0] + A.a[1][1] * A.a[1][1] + A.a[2][2] * A.a[2][2];
    if (off <= 1e-30 * diag || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A.a[p][q];
        if (apq == 0.0) continue;
        const double theta = (A.a[q][q] - A.a[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- J^T A J
          const double akp = A.a[k][p], akq = A.a[k][q];
          A.a[k][p] = c * akp - s * akq;
          A.a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A.a[p][k], aqk = A.a[q][k];
          A.a[p][k] = c * apk - s * aqk;
          A.a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = V.a[k][p], vkq = V.a[k][q];
          V.a[k][p] = c * vkp - s * vkq;
          V.a[k][q] = s * vkp + c * vkq;
        }
      }
  }
  // sort eigenvalues descending (columns of V follow)
  double ev[3] = {A.a[0][0], A.a[1][1], A.a[2][2]};
  int order[3] = {0, 1, 2};
  std::sort(order, order + 3, [&](int x, int y) { return ev[x] > ev[y]; });
  M3 Vs;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Vs.a[i][j] = V.a[i][order[j]];
  if (det(Vs) < 0)
    for (int i = 0; i < 3; ++i) Vs.a[i][2] = -Vs.a[i][2];
  M3 B = mul(F, Vs);
  // Givens QR: zero B(1,0), B(2,0), B(2,1); accumulate U = G1^T G2^T G3^T
  M3 U{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
  auto givens = [&](int r1, int r2, int col) {
    const double a = B.a[r1][col], b = B.a[r2][col];
    const double h = std::sqrt(a * a + b * b);
    double c = 1.0, s = 0.0;
    if (h > 1e-300) {
      c = a / h;
      s = b / h;
    }
    for (int k = 0; k < 3; ++k) {
      const double x = B.a[r1][k], y = B.a[r2][k];
      B.a[r1][k] = c * x + s * y;
      B.a[r2][k] = -s * x + c * y;
    }
    for (int k = 0; k < 3; ++k) {
      const double x = U.a[k][r1], y = U.a[k][r2];
      U.a[k][r1] = c * x + s * y;
      U.a[k][r2] = -s * x + c * y;
    }
  };
  givens(0, 1, 0);
  givens(0, 2, 0);
  givens(1, 2, 1);
  // B is now upper triangular with B(0,0), B(1,1) >= 0; keep det(U) = +1
  return mul(U, transpose(Vs));
}

inline void bspline_weights(double fx, double w[3]) {
  w[0] = 0.5 * (1.5 - fx) * (1.5 - fx);
  w[1] = 0.75 - (fx - 1.0) * (fx - 1.0);
  w[2] = 0.5 * (fx - 0.5) * (fx - 0.5);
}

template <typename R>
inline void bspline_weights_r(R fx, R w[3]) {
  w[0] = (R)0.5 * ((R)1.5 - fx) * ((R)1.5 - fx);
  w[1] = (R)0.75 - (fx - (R)1.0) * (fx - (R)1.0);
  w[2] = (R)0.5 * (fx - (R)0.5) * (fx - (R)0.5);
}

// mpm/solid.py:219-249
template <typename R>
void mpm_p2g(const OrcMpmParams& p, const R* x, const R* v, const R* C, R* F, R* Jp, const R* mass, const R* vol0,
             R* grid_v, R* grid_m) {
  const int ng = p.n_grid;
  const R inv_dx = (R)p.inv_dx, dx = (R)p.dx;
  for (int q = 0; q < p.n_particles; ++q) {
    R Xp[3], fx[3], w[3][3];
    int base[3];
    for (int a = 0; a < 3; ++a) {
      Xp[a] = x[q * 3 + a] * inv_dx;
      base[a] = (int)(Xp[a] - (R)0.5);
      fx[a] = Xp[a] - (R)base[a];
      bspline_weights_r<R>(fx[a], w[a]);
    }
    // weights are indexed w[offset][axis] in the reference; here w[axis][offset]
    M3 Fd;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Fd.a[i][j] = (double)F[q * 9 + i * 3 + j];
    const M3 Rr = polar_rotation(Fd);
    R Fp[3][3], Rp[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Fp[i][j] = F[q * 9 + i * 3 + j];
        Rp[i][j] = (R)Rr.a[i][j];
      }
    const R J = Fp[0][0] * (Fp[1][1] * Fp[2][2] - Fp[1][2] * Fp[2][1]) - Fp[0][1] * (Fp[1][0] * Fp[2][2] - Fp[1][2] * Fp[2][0]) +
                Fp[0][2] * (Fp[1][0] * Fp[2][1] - Fp[1][1] * Fp[2][0]);
    Jp[q] = J;
    // inverse transpose of Fp via cofactors: (F^-1)^T = cof(F) / det
    R FinvT[3][3];
    FinvT[0][0] = (Fp[1][1] * Fp[2][2] - Fp[1][2] * Fp[2][1]) / J;
    FinvT[0][1] = -(Fp[1][0] * Fp[2][2] - Fp[1][2] * Fp[2][0]) / J;
    FinvT[0][2] = (Fp[1][0] * Fp[2][1] - Fp[1][1] * Fp[2][0]) / J;
    FinvT[1][0] = -(Fp[0][1] * Fp[2][2] - Fp[0][2] * Fp[2][1]) / J;
    FinvT[1][1] = (Fp[0][0] * Fp[2][2] - Fp[0][2] * Fp[2][0]) / J;
    FinvT[1][2] = -(Fp[0][0] * Fp[2][1] - Fp[0][1] * Fp[2][0]) / J;
    FinvT[2][0] = (Fp[0][1] * Fp[1][2] - Fp[0][2] * Fp[1][1]) / J;
    FinvT[2][1] = -(Fp[0][0] * Fp[1][2] - Fp[0][2] * Fp[1][0]) / J;
    FinvT[2][2] = (Fp[0][0] * Fp[1][1] - Fp[0][1] * Fp[1][0]) / J;
    R P[3][3];
    const R mu2 = (R)2 * (R)p.mu, lam = (R)p.la * (J - (R)1) * J;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) P[i][j] = mu2 * (Fp[i][j] - Rp[i][j]) + lam * FinvT[i][j];
    // stress = -dt * vol0 * P @ F^T * inv_dx^2 (no factor 4: solid.py:239)
    const R pre = -(R)p.dt * vol0[q];
    R aff[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        R pf = 0;
        for (int k = 0; k < 3; ++k) pf += (pre * P[i][k]) * Fp[j][k];
        aff[i][j] = pf * inv_dx * inv_dx + mass[q] * C[q * 9 + i * 3 + j];
      }
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
          if (I[0] < 0 || I[0] >= ng || I[1] < 0 || I[1] >= ng || I[2] < 0 || I[2] >= ng) continue;
          const R dpos[3] = {((R)ox - fx[0]) * dx, ((R)oy - fx[1]) * dx, ((R)oz - fx[2]) * dx};
          const R weight = w[0][ox] * w[1][oy] * w[2][oz];
          const int64_t node = ((int64_t)I[0] * ng + I[1]) * ng + I[2];
          for (int a = 0; a < 3; ++a) {
            const R mom = mass[q] * v[q * 3 + a] + (aff[a][0] * dpos[0] + aff[a][1] * dpos[1] + aff[a][2] * dpos[2]);
            grid_v[node * 3 + a] += weight * mom;
          }
          grid_m[node] += weight * mass[q];
        }
  }
}

// mpm/solid.py:251-259 with apply_boundary_at_node 97-111
template <typename R>
void mpm_grid_update(const OrcMpmParams& p, R* grid_v, const R* grid_m, const R* grid_f_ext) {
  const int ng = p.n_grid;
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j)
      for (int k = 0; k < ng; ++k) {
        const int64_t n = ((int64_t)i * ng + j) * ng + k;
        const R m = grid_m[n];
        if (!(m > (R)0)) continue;
        R* gv = grid_v + n * 3;
        for (int a = 0; a < 3; ++a) {
          gv[a] = gv[a] / m;
          gv[a] += (R)p.dt * (R)p.gravity[a];
          gv[a] += (R)p.dt * grid_f_ext[n * 3 + a] / m;
        }
        const int I[3] = {i, j, k};
        for (int a = 0; a < 3; ++a) {
          if (I[a] < p.bound && gv[a] < (R)0) gv[a] = 0;
          if (I[a] > ng - p.bound && gv[a] > (R)0) gv[a] = 0;
        }
      }
}

// mpm/solid.py:261-315
template <typename R>
void mpm_g2p(const OrcMpmParams& p, R* x, R* v, R* C, R* F, R* Jp, const int8_t* fixed_mask, const R* fixed_x,
             const R* grid_v) {
  const int ng = p.n_grid;
  const R inv_dx = (R)p.inv_dx, dx = (R)p.dx, dt = (R)p.dt;
  for (int q = 0; q < p.n_particles; ++q) {
    R Xp[3], fx[3], w[3][3];
    int base[3];
    for (int a = 0; a < 3; ++a) {
      Xp[a] = x[q * 3 + a] * inv_dx;
      base[a] = (int)(Xp[a] - (R)0.5);
      fx[a] = Xp[a] - (R)base[a];
      bspline_weights_r<R>(fx[a], w[a]);
    }
    R nv[3] = {0, 0, 0}, nC[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
          if (I[0] < 0 || I[0] >= ng || I[1] < 0 || I[1] >= ng || I[2] < 0 || I[2] >= ng) continue;
          const R dpos[3] = {((R)ox - fx[0]) * dx, ((R)oy - fx[1]) * dx, ((R)oz - fx[2]) * dx};
          const R weight = w[0][ox] * w[1][oy] * w[2][oz];
          const int64_t node = ((int64_t)I[0] * ng + I[1]) * ng + I[2];
          const R* gv = grid_v + node * 3;
          for (int a = 0; a < 3; ++a) nv[a] += weight * gv[a];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) nC[a][b] += (R)4 * weight * gv[a] * dpos[b] * inv_dx * inv_dx;
        }
    for (int a = 0; a < 3; ++a) {
      v[q * 3 + a] = nv[a];
      x[q * 3 + a] += dt * nv[a];
    }
    // clamp_particle_to_domain (solid.py:114-124)
    for (int a = 0; a < 3; ++a) {
      if (x[q * 3 + a] < dx) {
        x[q * 3 + a] = dx;
        if (v[q * 3 + a] < (R)0) v[q * 3 + a] = 0;
      }
      if (x[q * 3 + a] > (R)1.0 - dx) {
        x[q * 3 + a] = (R)1.0 - dx;
        if (v[q * 3 + a] > (R)0) v[q * 3 + a] = 0;
      }
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) C[q * 9 + a * 3 + b] = nC[a][b];
    R Fn[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        R acc = 0;
        for (int k = 0; k < 3; ++k) acc += (((a == k) ? (R)1 : (R)0) + dt * nC[a][k]) * F[q * 9 + k * 3 + b];
        Fn[a][b] = acc;
      }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) F[q * 9 + a * 3 + b] = Fn[a][b];
    auto det3 = [&](const R* M) {
      return M[0] * (M[4] * M[8] - M[5] * M[7]) - M[1] * (M[3] * M[8] - M[5] * M[6]) + M[2] * (M[3] * M[7] - M[4] * M[6]);
    };
    Jp[q] = det3(F + q * 9);
    // apply_step112_dynamics_controls (solid.py:301-315)
    if (p.damping_enabled) {
      const R damp = std::max((R)0, (R)1 - (R)p.damping * dt);
      for (int a = 0; a < 3; ++a) v[q * 3 + a] *= damp;
    }
    if (p.lock_z) {
      x[q * 3 + 2] = fixed_x[q * 3 + 2];
      v[q * 3 + 2] = 0;
      for (int d = 0; d < 3; ++d) {
        C[q * 9 + 2 * 3 + d] = 0;
        C[q * 9 + d * 3 + 2] = 0;
        F[q * 9 + 2 * 3 + d] = 0;
        F[q * 9 + d * 3 + 2] = 0;
      }
      F[q * 9 + 8] = 1;
      Jp[q] = det3(F + q * 9);
    }
    if (fixed_mask[q] != 0) {
      for (int a = 0; a < 3; ++a) {
        x[q * 3 + a] = fixed_x[q * 3 + a];
        v[q * 3 + a] = 0;
      }
      for (int a = 0; a < 9; ++a) C[q * 9 + a] = 0;
      for (int a = 0; a < 9; ++a) F[q * 9 + a] = (a % 4 == 0) ? (R)1 : (R)0;
      Jp[q] = 1;
    }
  }
}

// mpm/solid.py:341-357
template <typename R>
void mpm_stats(const OrcMpmParams& p, const R* x, const R* v, const R* Jp, const R* mass, OrcMpmStats* st) {
  R mn[3] = {(R)1e9, (R)1e9, (R)1e9}, mx[3] = {(R)-1e9, (R)-1e9, (R)-1e9}, ms = 0, mnJ = (R)1e9, mxJ = (R)-1e9, tm = 0;
  for (int q = 0; q < p.n_particles; ++q) {
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], x[q * 3 + a]);
      mx[a] = std::max(mx[a], x[q * 3 + a]);
    }
    const R* vv = v + q * 3;
    ms = std::max(ms, (R)std::sqrt(vv[0] * vv[0] + vv[1] * vv[1] + vv[2] * vv[2]));
    mnJ = std::min(mnJ, Jp[q]);
    mxJ = std::max(mxJ, Jp[q]);
    tm += mass[q];
  }
  for (int a = 0; a < 3; ++a) {
    st->min_x[a] = mn[a];
    st->max_x[a] = mx[a];
  }
  st->max_speed = ms;
  st->min_J = mnJ;
  st->max_J = mxJ;
  st->total_mass = tm;
}

// ----------------------------------------------------------- coupling ----
// coupling/projection.py:21-91
template <typename R>
void couple_project(const OrcCouplingParams& cp, const OrcLbmParams& lp, int n_particles, const R* x, const R* v,
                    const R* Jp, const R* vol0, const R* mass, R* solid_phi, R* solid_mass, R* solid_vel,
                    OrcCouplingStats* st) {
  Grid<R> g{lp.nx, lp.ny, lp.nz};
  const int64_t n = g.n();
  std::memset(solid_phi, 0, sizeof(R) * n);
  std::memset(solid_mass, 0, sizeof(R) * n);
  std::memset(solid_vel, 0, sizeof(R) * 3 * n);
  const R inv_dx = (R)cp.inv_dx_norm, cellv = (R)cp.cell_volume_norm, vs = (R)cp.vel_scale;
  for (int q = 0; q < n_particles; ++q) {
    R Xp[3], fx[3], w[3][3];
    int base[3];
    for (int a = 0; a < 3; ++a) {
      Xp[a] = x[q * 3 + a] * inv_dx;
      base[a] = (int)(Xp[a] - (R)0.5);
      fx[a] = Xp[a] - (R)base[a];
      bspline_weights_r<R>(fx[a], w[a]);
    }
    const R J = std::max(Jp[q], (R)0);
    const R cur_vol = vol0[q] * J;
    const R vl[3] = {v[q * 3] * vs, v[q * 3 + 1] * vs, v[q * 3 + 2] * vs};
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
          if (I[0] < 0 || I[0] >= lp.nx || I[1] < 0 || I[1] >= lp.ny || I[2] < 0 || I[2] >= lp.nz) continue;
          const R weight = w[0][ox] * w[1][oy] * w[2][oz];
          const R mc = weight * mass[q];
          const R vfc = weight * cur_vol / cellv;
          const int64_t c = g.id(I[0], I[1], I[2]);
          solid_phi[c] += vfc;
          solid_mass[c] += mc;
          for (int a = 0; a < 3; ++a) solid_vel[c * 3 + a] += mc * vl[a];
        }
  }
  // normalize_projection (projection.py:67-91)
  R pm = 0, pvr = 0, pvc = 0, mphi = 0;
  int active = 0;
  for (int64_t c = 0; c < n; ++c) {
    const R raw = solid_phi[c];
    mphi = std::max(mphi, raw);
    if (solid_mass[c] > (R)cp.eps_mass) {
      for (int a = 0; a < 3; ++a) solid_vel[c * 3 + a] = solid_vel[c * 3 + a] / solid_mass[c];
    } else {
      for (int a = 0; a < 3; ++a) solid_vel[c * 3 + a] = 0;
    }
    const R cl = std::min((R)1, std::max((R)0, raw));
    solid_phi[c] = cl;
    if (cl > (R)1.0e-8) active += 1;
    pm += solid_mass[c];
    pvr += raw * cellv;
    pvc += cl * cellv;
  }
  st->projected_mass = pm;
  st->projected_volume_raw = pvr;
  st->projected_volume_clamped = pvc;
  st->max_phi_raw = mphi;
  st->active_cell_count = active;
}

// coupling/penalty.py:42-88 (clear_force_fields + build_penalty_force)
template <typename R>
void couple_penalty_force(const OrcCouplingParams& cp, const OrcLbmParams& lp, const int8_t* solid, const R* solid_phi,
                          const R* rho, const R* v, const R* solid_vel, R* cell_force, R* hydro_force,
                          OrcCouplingStats* st) {
  Grid<R> g{lp.nx, lp.ny, lp.nz};
  int active = 0;
  R mcf = 0, mhf = 0, ncf[3] = {0, 0, 0}, nhf[3] = {0, 0, 0};
  for (int64_t c = 0; c < g.n(); ++c) {
    R force[3] = {0, 0, 0};
    if (solid[c] == 0) {
      const R phi = solid_phi[c];
      if (phi > (R)cp.phi_min) {
        for (int a = 0; a < 3; ++a)
          force[a] = (R)cp.beta_lbm * phi * rho[c] * (solid_vel[c * 3 + a] - v[c * 3 + a]);
        const R nrm = std::sqrt(force[0] * force[0] + force[1] * force[1] + force[2] * force[2]);
        if (nrm > (R)cp.force_cap) {
          const R sc = (R)cp.force_cap / nrm;
          for (int a = 0; a < 3; ++a) force[a] = force[a] * sc;
        }
        active += 1;
      }
    }
    for (int a = 0; a < 3; ++a) {
      cell_force[c * 3 + a] = force[a];
      hydro_force[c * 3 + a] = -force[a];
      ncf[a] += force[a];
      nhf[a] += -force[a];
    }
    const R nrm = std::sqrt(force[0] * force[0] + force[1] * force[1] + force[2] * force[2]);
    mcf = std::max(mcf, nrm);
    mhf = std::max(mhf, nrm);
  }
  st->active_force_cell_count = active;
  st->max_cell_force_norm = mcf;
  st->max_hydro_force_norm = mhf;
  for (int a = 0; a < 3; ++a) {
    st->net_cell_force[a] = ncf[a];
    st->net_hydro_force[a] = nhf[a];
  }
}

// Reaction transfer LBM -> MPM grid.
//   kind 0: penalty (coupling/penalty.py:90-129)
//   kind 1: engineering moving boundary (coupling/moving_boundary.py:58-110)
//   kind 2: link-area (coupling/link_area.py:139-193; area_scale from cp)
template <typename R>
void couple_reaction(int kind, const OrcCouplingParams& cp, const OrcLbmParams& lp, int n_particles, const R* x,
                     const R* Jp, const R* vol0, const R* hydro_force, const R* solid_phi, R* grid_f_ext,
                     OrcCouplingStats* st) {
  Grid<R> g{lp.nx, lp.ny, lp.nz};
  const int ng = cp.n_grid;
  const R inv_dx = (R)cp.inv_dx_norm;
  R max_grid = 0, net_grid[3] = {0, 0, 0}, max_part = 0, net_part[3] = {0, 0, 0};
  int active = 0;
  for (int q = 0; q < n_particles; ++q) {
    R Xp[3], fx[3], w[3][3];
    int base[3];
    for (int a = 0; a < 3; ++a) {
      Xp[a] = x[q * 3 + a] * inv_dx;
      base[a] = (int)(Xp[a] - (R)0.5);
      fx[a] = Xp[a] - (R)base[a];
      bspline_weights_r<R>(fx[a], w[a]);
    }
    R hs[3] = {0, 0, 0}, ps = 0;
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
          if (I[0] < 0 || I[0] >= lp.nx || I[1] < 0 || I[1] >= lp.ny || I[2] < 0 || I[2] >= lp.nz) continue;
          const R weight = w[0][ox] * w[1][oy] * w[2][oz];
          const int64_t c = g.id(I[0], I[1], I[2]);
          for (int a = 0; a < 3; ++a) hs[a] += weight * hydro_force[c * 3 + a];
          if (kind != 0) ps += weight * solid_phi[c];
        }
    R pf[3];
    const R J = std::max(Jp[q], (R)0);
    const R pv = vol0[q] * J;
    if (kind == 0) {
      for (int a = 0; a < 3; ++a) pf[a] = hs[a] * (R)cp.force_density_scale * pv * (R)cp.reaction_scale;
    } else {
      if (!(ps > (R)cp.phi_min)) continue;
      for (int a = 0; a < 3; ++a) {
        pf[a] = hs[a] * (R)cp.force_density_scale * pv * (R)cp.reaction_scale;
        if (kind == 2) pf[a] = pf[a] * (R)cp.area_scale;
      }
      R nrm = std::sqrt(pf[0] * pf[0] + pf[1] * pf[1] + pf[2] * pf[2]);
      if (nrm > (R)cp.force_cap) {
        const R sc = (R)cp.force_cap / nrm;
        for (int a = 0; a < 3; ++a) pf[a] = pf[a] * sc;
        nrm = (R)cp.force_cap;
      }
      if (nrm > (R)0) active += 1;
      max_part = std::max(max_part, nrm);
      for (int a = 0; a < 3; ++a) net_part[a] += pf[a];
    }
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I[3] = {base[0] + ox, base[1] + oy, base[2] + oz};
          if (I[0] < 0 || I[0] >= ng || I[1] < 0 || I[1] >= ng || I[2] < 0 || I[2] >= ng) continue;
          const R weight = w[0][ox] * w[1][oy] * w[2][oz];
          const int64_t node = ((int64_t)I[0] * ng + I[1]) * ng + I[2];
          R con[3];
          for (int a = 0; a < 3; ++a) {
            con[a] = weight * pf[a];
            grid_f_ext[node * 3 + a] += con[a];
            net_grid[a] += con[a];
          }
          max_grid = std::max(max_grid, (R)std::sqrt(con[0] * con[0] + con[1] * con[1] + con[2] * con[2]));
        }
  }
  if (kind == 0) {
    st->max_reaction_grid_force_norm = max_grid;
    for (int a = 0; a < 3; ++a) st->net_reaction_grid_force[a] = net_grid[a];
  } else {
    st->active_reaction_particle_count = active;
    st->max_particle_reaction_norm = max_part;
    st->max_grid_reaction_norm = max_grid;
    for (int a = 0; a < 3; ++a) {
      st->net_particle_reaction_force[a] = net_part[a];
      st->net_grid_reaction_force[a] = net_grid[a];
    }
  }
}

}  // namespace

// ------------------------------------------------------------ C ABI ----
#define ORC_EXPORT(SUF, R)                                                                                          \
  extern "C" void orc##SUF##_lbm_init(const OrcLbmParams* p, R* f, R* F, R* rho, R* v) { lbm_init<R>(*p, f, F, rho, v); } \
  extern "C" void orc##SUF##_lbm_collide(const OrcLbmParams* p, const R* F, const R* rho, const R* v,               \
                                         const R* cf, const int8_t* solid, R* f, int threads) {                   \
    lbm_collide<R>(*p, F, rho, v, cf, solid, f, threads);                                                          \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_stream(const OrcLbmParams* p, int moving, const R* f, R* F, const int8_t* solid,  \
                                        const R* rho, const R* sv, R* hydro, OrcLbmDiag* d, int threads) {        \
    lbm_stream<R>(*p, moving, f, F, solid, rho, sv, hydro, d, threads);                                            \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_boundary(const OrcLbmParams* p, R* F, const R* rho, const R* v,                   \
                                          const int8_t* solid, OrcLbmDiag* d) {                                   \
    lbm_boundary<R>(*p, F, rho, v, solid, d);                                                                      \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_plane_flux_controller(const OrcLbmParams* p, const R* rho, const R* v,            \
                                                       const int8_t* solid, OrcLbmDiag* d) {                    \
    plane_flux_controller<R>(*p, rho, v, solid, d);                                                                \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_macros(const OrcLbmParams* p, R* f, const R* F, R* rho, R* v,                     \
                                        const int8_t* solid, const R* cf, int threads) {                          \
    lbm_macros<R>(*p, f, F, rho, v, solid, cf, threads);                                                           \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_update_dynamic_solid(const OrcLbmParams* p, double thr, int8_t* solid,            \
                                                      const int8_t* st, int8_t* old, const R* phi,                \
                                                      int8_t* reinit) {                                           \
    lbm_update_dynamic_solid<R>(*p, thr, solid, st, old, phi, reinit);                                             \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_reinit(const OrcLbmParams* p, int8_t* reinit, const R* sv, R* rho, R* v, R* f,    \
                                        R* F) {                                                                   \
    lbm_reinit<R>(*p, reinit, sv, rho, v, f, F);                                                                   \
  }                                                                                                                \
  extern "C" void orc##SUF##_lbm_force_accumulator(const OrcLbmParams* p, int op, R* hydro, R* accum,              \
                                                   OrcLbmDiag* d) {                                               \
    lbm_force_accumulator<R>(*p, op, hydro, accum, d);                                                             \
  }                                                                                                                \
  extern "C" void orc##SUF##_mpm_p2g(const OrcMpmParams* p, const R* x, const R* v, const R* C, R* F, R* Jp,        \
                                     const R* mass, const R* vol0, R* gv, R* gm) {                                \
    mpm_p2g<R>(*p, x, v, C, F, Jp, mass, vol0, gv, gm);                                                            \
  }                                                                                                                \
  extern "C" void orc##SUF##_mpm_grid_update(const OrcMpmParams* p, R* gv, const R* gm, const R* gf) {             \
    mpm_grid_update<R>(*p, gv, gm, gf);                                                                            \
  }                                                                                                                \
  extern "C" void orc##SUF##_mpm_g2p(const OrcMpmParams* p, R* x, R* v, R* C, R* F, R* Jp, const int8_t* fm,        \
                                     const R* fxp, const R* gv) {                                                 \
    mpm_g2p<R>(*p, x, v, C, F, Jp, fm, fxp, gv);                                                                   \
  }                                                                                                                \
  extern "C" void orc##SUF##_mpm_stats(const OrcMpmParams* p, const R* x, const R* v, const R* Jp, const R* m,     \
                                       OrcMpmStats* st) {                                                         \
    mpm_stats<R>(*p, x, v, Jp, m, st);                                                                             \
  }                                                                                                                \
  extern "C" void orc##SUF##_couple_project(const OrcCouplingParams* cp, const OrcLbmParams* lp, int np_,          \
                                            const R* x, const R* v, const R* Jp, const R* vol0, const R* mass,    \
                                            R* phi, R* smass, R* svel, OrcCouplingStats* st) {                    \
    couple_project<R>(*cp, *lp, np_, x, v, Jp, vol0, mass, phi, smass, svel, st);                                  \
  }                                                                                                                \
  extern "C" void orc##SUF##_couple_penalty_force(const OrcCouplingParams* cp, const OrcLbmParams* lp,             \
                                                  const int8_t* solid, const R* phi, const R* rho, const R* v,    \
                                                  const R* sv, R* cf, R* hf, OrcCouplingStats* st) {              \
    couple_penalty_force<R>(*cp, *lp, solid, phi, rho, v, sv, cf, hf, st);                                         \
  }                                                                                                                \
  extern "C" void orc##SUF##_couple_reaction(int kind, const OrcCouplingParams* cp, const OrcLbmParams* lp,         \
                                             int np_, const R* x, const R* Jp, const R* vol0, const R* hf,        \
                                             const R* phi, R* gfe, OrcCouplingStats* st) {                        \
    couple_reaction<R>(kind, *cp, *lp, np_, x, Jp, vol0, hf, phi, gfe, st);                                        \
  }

ORC_EXPORT(32, float)
ORC_EXPORT(64, double)

extern "C" void orc_polar_rotation(const double* F, double* R) {
  M3 A;
  for (int i = 0; i < 9; ++i) A.a[i / 3][i % 3] = F[i];
  const M3 Q = polar_rotation(A);
  for (int i = 0; i < 9; ++i) R[i] = Q.a[i / 3][i % 3];
}

extern "C" int orc_abi_version() { return 2; }

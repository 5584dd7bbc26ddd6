// Particle-side kernels of the coupled FSI step: MPM -> LBM projection,
// LBM -> MPM reaction transfer and the MLS-MPM substep.
//
// Reference semantics:
//   projection      src/mpm_lbm/sim/coupling/projection.py:21-97
//   penalty react.  src/mpm_lbm/sim/coupling/penalty.py:90-129
//   engineering     src/mpm_lbm/sim/coupling/moving_boundary.py:58-110
//   link-area       src/mpm_lbm/sim/coupling/link_area.py:84-193
//                   (+ link_area_accounting.py:42-148 for the area scale)
//   MPM substep     src/mpm_lbm/sim/mpm/solid.py:212-315
// Particle fields are planar ([comp][n]); the MPM grid and the lattice are
// x-fastest: node = (k * n + j) * n + i, cell = (k * ny + j) * nx + i.

#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "polar3.cuh"

namespace fsi {

struct BSpline {
  int base[3];
  float fx[3];
  float w[3][3];  // [axis][offset]
};

// quadratic B-spline weights exactly as the reference builds them (solid.py:222-230)
__device__ __forceinline__ void bspline(const float* X, float inv_dx, BSpline& b) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float Xp = X[a] * inv_dx;
    b.base[a] = (int)(Xp - 0.5f);  // truncation, as ti.cast(.., ti.i32)
    const float f = Xp - (float)b.base[a];
    b.fx[a] = f;
    b.w[a][0] = 0.5f * (1.5f - f) * (1.5f - f);
    b.w[a][1] = 0.75f - (f - 1.0f) * (f - 1.0f);
    b.w[a][2] = 0.5f * (f - 0.5f) * (f - 0.5f);
  }
}

struct LatView {
  int nx, ny, nz;
  int64_t pitch;
};

__device__ __forceinline__ int64_t lat_cell(const LatView& L, int i, int j, int k) {
  return ((int64_t)k * L.ny + j) * L.nx + i;
}

// ---------------------------------------------------------- projection ----
__global__ void k_project_scatter(LatView L, FsiParticles pt, FsiCouplingParams cp, float* phi, float* smass,
                                  float* svel) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pt.n) return;
  const int n = pt.n;
  const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
  BSpline b;
  bspline(X, cp.inv_dx_norm, b);
  const float J = fmaxf(pt.Jp[p], 0.0f);
  const float cur_vol = pt.vol0[p] * J;
  const float m = pt.mass[p];
  const float vl[3] = {pt.v[p] * cp.vel_scale, pt.v[n + p] * cp.vel_scale, pt.v[2 * n + p] * cp.vel_scale};
  for (int ox = 0; ox < 3; ++ox)
    for (int oy = 0; oy < 3; ++oy)
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (I < 0 || I >= L.nx || Jj < 0 || Jj >= L.ny || K < 0 || K >= L.nz) continue;
        const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
        const float mc = w * m;
        const int64_t c = lat_cell(L, I, Jj, K);
        atomicAdd(phi + c, w * cur_vol / cp.cell_volume_norm);
        atomicAdd(smass + c, mc);
        atomicAdd(svel + c, mc * vl[0]);
        atomicAdd(svel + L.pitch + c, mc * vl[1]);
        atomicAdd(svel + 2 * L.pitch + c, mc * vl[2]);
      }
}

__global__ void k_project_normalize(LatView L, FsiCouplingParams cp, float* phi, float* smass, float* svel,
                                    FsiCouplingStats* st) {
  const int64_t n = (int64_t)L.nx * L.ny * L.nz;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double pm = 0.0, pvr = 0.0, pvc = 0.0;
  float mx = 0.f;
  int active = 0;
  if (c < n) {
    const float raw = phi[c];
    const float m = smass[c];
    mx = raw;
    if (m > cp.eps_mass) {
      for (int a = 0; a < 3; ++a) svel[a * L.pitch + c] = svel[a * L.pitch + c] / m;
    } else {
      for (int a = 0; a < 3; ++a) svel[a * L.pitch + c] = 0.f;
    }
    const float cl = fminf(1.0f, fmaxf(0.0f, raw));
    phi[c] = cl;
    active = cl > 1.0e-8f;
    pm = m;
    pvr = (double)raw * cp.cell_volume_norm;
    pvc = (double)cl * cp.cell_volume_norm;
  }
  pm = warp_sum_d(pm);
  pvr = warp_sum_d(pvr);
  pvc = warp_sum_d(pvc);
  mx = warp_max(fmaxf(mx, 0.f));
  const int na = __popc(__ballot_sync(0xffffffffu, active));
  if ((threadIdx.x & 31) == 0) {
    if (pm != 0.0) atomicAdd(&st->projected_mass, pm);
    if (pvr != 0.0) atomicAdd(&st->projected_volume_raw, pvr);
    if (pvc != 0.0) atomicAdd(&st->projected_volume_clamped, pvc);
    if (mx > 0.f) atomic_max_nonneg(&st->max_phi_raw, mx);
    if (na) atomicAdd(&st->active_cell_count, na);
  }
}

// ------------------------------------------------------------ reaction ----
__device__ float link_area_scale(const FsiLbmDiag* d, const FsiCouplingParams& cp, float* raw_out) {
  // link_area_accounting.py:42-60 weights; link_area.py:84-100 scale
  double num = 0.0, den = 0.0;
  for (int s = 1; s < 19; ++s) {
    const double sfx = -(double)d->fluid_impulse[s][0];
    const double len = s <= 6 ? 1.0 : 1.4142135623730951;
    double w = 1.0;
    if (cp.area_policy == 1) w = 1.0 / len;
    if (cp.area_policy == 2) w = len;
    num += w * sfx;
    den += sfx;
  }
  const double raw = fabs(num) / (fabs((double)(float)den) + 1.0e-12);
  double sc = fmin(fmax(raw, (double)cp.area_scale_min), (double)cp.area_scale_max);
  if (!isfinite(sc)) sc = cp.area_scale_min;
  *raw_out = (float)raw;
  return (float)sc;
}

__global__ void k_reaction(LatView L, const float* hydro, const float* phi, FsiParticles pt, FsiGrid g,
                           FsiCouplingParams cp, FsiCouplingStats* st, const FsiLbmDiag* diag) {
  __shared__ float s_scale;
  if (threadIdx.x == 0) {
    float raw = 1.f;
    s_scale = cp.kind == 2 ? link_area_scale(diag, cp, &raw) : 1.0f;
    if (blockIdx.x == 0 && cp.kind == 2) {
      st->area_scale = s_scale;
      st->raw_area_scale = raw;
    }
  }
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = pt.n;
  bool act = false, gated = false;
  float pf[3] = {0.f, 0.f, 0.f}, pnorm = 0.f, gmax = 0.f;
  double gnet[3] = {0.0, 0.0, 0.0};
  if (p < n) {
    const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
    BSpline b;
    bspline(X, cp.inv_dx_norm, b);
    float hs[3] = {0.f, 0.f, 0.f}, ps = 0.f;
    for (int ox = 0; ox < 3; ++ox)
      for (int oy = 0; oy < 3; ++oy)
        for (int oz = 0; oz < 3; ++oz) {
          const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
          if (I < 0 || I >= L.nx || Jj < 0 || Jj >= L.ny || K < 0 || K >= L.nz) continue;
          const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
          const int64_t c = lat_cell(L, I, Jj, K);
          hs[0] += w * hydro[c];
          hs[1] += w * hydro[L.pitch + c];
          hs[2] += w * hydro[2 * L.pitch + c];
          if (cp.kind != 0) ps += w * phi[c];
        }
    const float J = fmaxf(pt.Jp[p], 0.0f);
    const float pv = pt.vol0[p] * J;
    bool scatter = true;
    if (cp.kind == 0) {
      for (int a = 0; a < 3; ++a) pf[a] = hs[a] * cp.force_density_scale * pv * cp.reaction_scale;
    } else if (ps > cp.phi_min) {
      for (int a = 0; a < 3; ++a) {
        pf[a] = hs[a] * cp.force_density_scale * pv * cp.reaction_scale;
        if (cp.kind == 2) pf[a] = pf[a] * s_scale;
      }
      float nrm = sqrtf(pf[0] * pf[0] + pf[1] * pf[1] + pf[2] * pf[2]);
      if (nrm > cp.force_cap) {
        const float r = cp.force_cap / nrm;
        for (int a = 0; a < 3; ++a) pf[a] = pf[a] * r;
        nrm = cp.force_cap;
      }
      act = nrm > 0.f;
      gated = true;
      pnorm = nrm;
    } else {
      scatter = false;
      pf[0] = pf[1] = pf[2] = 0.f;
    }
    if (scatter) {
      const int64_t N = (int64_t)g.n * g.n * g.n;
      for (int ox = 0; ox < 3; ++ox)
        for (int oy = 0; oy < 3; ++oy)
          for (int oz = 0; oz < 3; ++oz) {
            const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
            if (I < 0 || I >= g.n || Jj < 0 || Jj >= g.n || K < 0 || K >= g.n) continue;
            const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
            const int64_t node = ((int64_t)K * g.n + Jj) * g.n + I;
            const float c0 = w * pf[0], c1 = w * pf[1], c2 = w * pf[2];
            atomicAdd(g.f_ext + node, c0);
            atomicAdd(g.f_ext + N + node, c1);
            atomicAdd(g.f_ext + 2 * N + node, c2);
            gnet[0] += c0;
            gnet[1] += c1;
            gnet[2] += c2;
            gmax = fmaxf(gmax, sqrtf(c0 * c0 + c1 * c1 + c2 * c2));
          }
    }
  }
  // diagnostics reductions (penalty.py:202-240, moving_boundary.py:312-374)
  const int na = __popc(__ballot_sync(0xffffffffu, act));
  const float pm = warp_max(pnorm), gm = warp_max(gmax);
  double pn[3], gn[3];
  for (int a = 0; a < 3; ++a) {
    pn[a] = warp_sum_d(gated ? (double)pf[a] : 0.0);
    gn[a] = warp_sum_d(gnet[a]);
  }
  if ((threadIdx.x & 31) == 0) {
    if (na) atomicAdd(&st->active_reaction_particle_count, na);
    if (pm > 0.f) atomic_max_nonneg(&st->max_particle_reaction_norm, pm);
    if (gm > 0.f) atomic_max_nonneg(&st->max_grid_reaction_norm, gm);
    for (int a = 0; a < 3; ++a) {
      if (pn[a] != 0.0) atomicAdd(&st->net_particle_reaction[a], pn[a]);
      if (gn[a] != 0.0) atomicAdd(&st->net_grid_reaction[a], gn[a]);
    }
  }
}

// ----------------------------------------------------------------- MPM ----
__global__ void k_p2g(FsiParticles pt, FsiGrid g, FsiMpmParams mp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pt.n) return;
  const int n = pt.n;
  const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
  BSpline b;
  bspline(X, mp.inv_dx, b);
  float Fp[9], Cp[9];
  double Fd[9], Rd[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    Fp[a] = pt.F[(int64_t)a * n + p];
    Cp[a] = pt.C[(int64_t)a * n + p];
    Fd[a] = (double)Fp[a];
  }
  polar_rotation_d(Fd, Rd);
  const float c00 = Fp[4] * Fp[8] - Fp[5] * Fp[7];
  const float c01 = Fp[3] * Fp[8] - Fp[5] * Fp[6];
  const float c02 = Fp[3] * Fp[7] - Fp[4] * Fp[6];
  const float J = Fp[0] * c00 - Fp[1] * c01 + Fp[2] * c02;
  pt.Jp[p] = J;
  // (F^-1)^T = cof(F) / det
  float FinvT[9];
  FinvT[0] = c00 / J;
  FinvT[1] = -c01 / J;
  FinvT[2] = c02 / J;
  FinvT[3] = -(Fp[1] * Fp[8] - Fp[2] * Fp[7]) / J;
  FinvT[4] = (Fp[0] * Fp[8] - Fp[2] * Fp[6]) / J;
  FinvT[5] = -(Fp[0] * Fp[7] - Fp[1] * Fp[6]) / J;
  FinvT[6] = (Fp[1] * Fp[5] - Fp[2] * Fp[4]) / J;
  FinvT[7] = -(Fp[0] * Fp[5] - Fp[2] * Fp[3]) / J;
  FinvT[8] = (Fp[0] * Fp[4] - Fp[1] * Fp[3]) / J;
  const float mu2 = 2.0f * mp.mu, lam = mp.la * (J - 1.0f) * J;
  float P[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) P[a] = mu2 * (Fp[a] - (float)Rd[a]) + lam * FinvT[a];
  // stress = -dt vol0 P F^T inv_dx^2 (solid.py:239: no factor 4), affine = stress + m C
  const float pre = -mp.dt * pt.vol0[p];
  const float mass = pt.mass[p];
  float aff[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float pf = (pre * P[i * 3 + 0]) * Fp[j * 3 + 0] + (pre * P[i * 3 + 1]) * Fp[j * 3 + 1] + (pre * P[i * 3 + 2]) * Fp[j * 3 + 2];
      aff[i * 3 + j] = pf * mp.inv_dx * mp.inv_dx + mass * Cp[i * 3 + j];
    }
  const float mv[3] = {mass * pt.v[p], mass * pt.v[n + p], mass * pt.v[2 * n + p]};
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  for (int ox = 0; ox < 3; ++ox)
    for (int oy = 0; oy < 3; ++oy)
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
        const float dpos[3] = {((float)ox - b.fx[0]) * mp.dx, ((float)oy - b.fx[1]) * mp.dx, ((float)oz - b.fx[2]) * mp.dx};
        const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
        const int64_t node = ((int64_t)K * G + Jj) * G + I;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float mom = mv[a] + (aff[a * 3 + 0] * dpos[0] + aff[a * 3 + 1] * dpos[1] + aff[a * 3 + 2] * dpos[2]);
          atomicAdd(g.v + a * N + node, w * mom);
        }
        atomicAdd(g.m + node, w * mass);
      }
}

__global__ void k_grid_update(FsiGrid g, FsiMpmParams mp) {
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N) return;
  const float m = g.m[node];
  if (!(m > 0.0f)) return;
  const int idx[3] = {(int)(node % G), (int)((node / G) % G), (int)(node / ((int64_t)G * G))};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float v = g.v[a * N + node] / m;
    v += mp.dt * mp.gravity[a];
    v += mp.dt * g.f_ext[a * N + node] / m;
    // apply_boundary_at_node (solid.py:97-111)
    if (idx[a] < mp.bound && v < 0.0f) v = 0.0f;
    if (idx[a] > G - mp.bound && v > 0.0f) v = 0.0f;
    g.v[a * N + node] = v;
  }
}

__global__ void k_g2p(FsiParticles pt, FsiGrid g, FsiMpmParams mp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pt.n) return;
  const int n = pt.n;
  float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
  BSpline b;
  bspline(X, mp.inv_dx, b);
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  float nv[3] = {0.f, 0.f, 0.f}, nC[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const float s4 = 4.0f * mp.inv_dx * mp.inv_dx;
  for (int ox = 0; ox < 3; ++ox)
    for (int oy = 0; oy < 3; ++oy)
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
        const float dpos[3] = {((float)ox - b.fx[0]) * mp.dx, ((float)oy - b.fx[1]) * mp.dx, ((float)oz - b.fx[2]) * mp.dx};
        const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
        const int64_t node = ((int64_t)K * G + Jj) * G + I;
        const float gv[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          nv[a] += w * gv[a];
#pragma unroll
          for (int c = 0; c < 3; ++c) nC[a * 3 + c] += (w * gv[a]) * dpos[c] * s4;
        }
      }
  float v[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v[a] = nv[a];
    X[a] += mp.dt * nv[a];
  }
  // clamp_particle_to_domain (solid.py:114-124)
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (X[a] < mp.dx) {
      X[a] = mp.dx;
      if (v[a] < 0.f) v[a] = 0.f;
    }
    if (X[a] > 1.0f - mp.dx) {
      X[a] = 1.0f - mp.dx;
      if (v[a] > 0.f) v[a] = 0.f;
    }
  }
  float Fo[9], Fn[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) Fo[a] = pt.F[(int64_t)a * n + p];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc += ((a == k ? 1.0f : 0.0f) + mp.dt * nC[a * 3 + k]) * Fo[k * 3 + c];
      Fn[a * 3 + c] = acc;
    }
  auto det3 = [](const float* M) {
    return M[0] * (M[4] * M[8] - M[5] * M[7]) - M[1] * (M[3] * M[8] - M[5] * M[6]) + M[2] * (M[3] * M[7] - M[4] * M[6]);
  };
  float J = det3(Fn);
  // apply_step112_dynamics_controls (solid.py:301-315)
  if (mp.damping > 0.f) {
    const float d = fmaxf(0.0f, 1.0f - mp.damping * mp.dt);
    for (int a = 0; a < 3; ++a) v[a] *= d;
  }
  if (mp.lock_z) {
    X[2] = pt.fixed_x[2 * n + p];
    v[2] = 0.f;
    for (int d = 0; d < 3; ++d) {
      nC[2 * 3 + d] = 0.f;
      nC[d * 3 + 2] = 0.f;
      Fn[2 * 3 + d] = 0.f;
      Fn[d * 3 + 2] = 0.f;
    }
    Fn[8] = 1.0f;
    J = det3(Fn);
  }
  if (pt.fixed[p]) {
    for (int a = 0; a < 3; ++a) {
      X[a] = pt.fixed_x[a * n + p];
      v[a] = 0.f;
    }
    for (int a = 0; a < 9; ++a) {
      nC[a] = 0.f;
      Fn[a] = (a % 4 == 0) ? 1.0f : 0.0f;
    }
    J = 1.0f;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    pt.x[a * n + p] = X[a];
    pt.v[a * n + p] = v[a];
  }
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    pt.C[(int64_t)a * n + p] = nC[a];
    pt.F[(int64_t)a * n + p] = Fn[a];
  }
  pt.Jp[p] = J;
}

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

static int check_particles(const FsiParticles* pt) {
  if (!pt) return invalid("null particles");
  if (pt->n <= 0) return invalid("n_particles must be positive");
  if (!pt->x || !pt->v || !pt->C || !pt->F || !pt->Jp || !pt->mass || !pt->vol0) return invalid("null particle field");
  return FSI_OK;
}

}  // namespace fsi

using namespace fsi;

extern "C" int fsi_project(const FsiLbmState* s, const FsiParticles* pt, const FsiCouplingParams* cp,
                           FsiCouplingStats* stats, void* stream) {
  if (!s || !cp || !stats) return invalid("null argument");
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!s->phi || !s->smass || !s->svel) return invalid("projection needs phi, smass, svel");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t P = s->pitch;
  if ((rc = cuda_check(cudaMemsetAsync(s->phi, 0, sizeof(float) * P, st), "clear phi"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(s->smass, 0, sizeof(float) * P, st), "clear smass"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(s->svel, 0, sizeof(float) * 3 * P, st), "clear svel"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(stats, 0, offsetof(FsiCouplingStats, active_reaction_particle_count), st),
                       "clear projection stats")))
    return rc;
  const LatView L{s->nx, s->ny, s->nz, P};
  k_project_scatter<<<nblk(pt->n, 128), 128, 0, st>>>(L, *pt, *cp, s->phi, s->smass, s->svel);
  if ((rc = launch_check("k_project_scatter"))) return rc;
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_project_normalize<<<nblk(n, 256), 256, 0, st>>>(L, *cp, s->phi, s->smass, s->svel, stats);
  return launch_check("k_project_normalize");
}

extern "C" int fsi_reaction_to_grid(const FsiLbmState* s, const float* hydro, const FsiParticles* pt, const FsiGrid* g,
                                    const FsiCouplingParams* cp, FsiCouplingStats* stats, void* stream) {
  if (!s || !hydro || !g || !cp || !stats) return invalid("null argument");
  int rc = check_particles(pt);
  if (rc) return rc;
  if (cp->kind < 0 || cp->kind > 2) return invalid("reaction kind must be 0 (penalty), 1 (engineering), 2 (link-area)");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t off = offsetof(FsiCouplingStats, active_reaction_particle_count);
  if ((rc = cuda_check(cudaMemsetAsync(reinterpret_cast<char*>(stats) + off, 0, sizeof(FsiCouplingStats) - off, st),
                       "clear reaction stats")))
    return rc;
  const LatView L{s->nx, s->ny, s->nz, s->pitch};
  k_reaction<<<nblk(pt->n, 128), 128, 0, st>>>(L, hydro, s->phi, *pt, *g, *cp, stats, s->diag);
  return launch_check("k_reaction");
}

extern "C" int fsi_mpm_p2g(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, void* stream) {
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!g || !mp || g->n <= 0) return invalid("bad grid or params");
  k_p2g<<<nblk(pt->n, 128), 128, 0, (cudaStream_t)stream>>>(*pt, *g, *mp);
  return launch_check("k_p2g");
}

extern "C" int fsi_mpm_grid_update(const FsiGrid* g, const FsiMpmParams* mp, void* stream) {
  if (!g || !mp || g->n <= 0) return invalid("bad grid or params");
  const int64_t N = (int64_t)g->n * g->n * g->n;
  k_grid_update<<<nblk(N, 256), 256, 0, (cudaStream_t)stream>>>(*g, *mp);
  return launch_check("k_grid_update");
}

extern "C" int fsi_mpm_g2p(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, void* stream) {
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!g || !mp || g->n <= 0) return invalid("bad grid or params");
  if (!pt->fixed || !pt->fixed_x) return invalid("null fixed-particle fields");
  k_g2p<<<nblk(pt->n, 128), 128, 0, (cudaStream_t)stream>>>(*pt, *g, *mp);
  return launch_check("k_g2p");
}

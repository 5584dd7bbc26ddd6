// Per-particle and per-node pieces of the MPM substep and of the reaction
// transfer, shared by the one-phase-per-launch kernels (mpm_kernels.cu) and
// the binned, shared-memory-staged substep (mpm_binned.cu) so that both paths
// perform the same arithmetic.
//
// Reference semantics:
//   B-spline weights     src/mpm_lbm/sim/mpm/solid.py:222-230
//   P2G stress/affine    src/mpm_lbm/sim/mpm/solid.py:231-249
//   grid update + walls  src/mpm_lbm/sim/mpm/solid.py:97-111, 251-259
//   G2P + controls       src/mpm_lbm/sim/mpm/solid.py:114-124, 261-315
//   reaction transfer    src/mpm_lbm/sim/coupling/penalty.py:90-129,
//                        moving_boundary.py:58-110, link_area.py:84-193
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/fsi_b200.h"
#include "polar3.cuh"

namespace fsi {

struct BSpline {
  int base[3];
  float fx[3];
  float w[3][3];  // [axis][offset]
};

// quadratic B-spline weights as the reference builds them (solid.py:222-230).
// Xp is rounded before the subtraction so that the base cell (which also keys
// the particle bins) does not depend on FMA contraction.
__device__ __forceinline__ void bspline(const float* X, float inv_dx, BSpline& b) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float Xp = __fmul_rn(X[a], inv_dx);
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

// global area scale of the link-area transfer from the last LBM step's
// per-direction fluid impulse (link_area_accounting.py:42-60, link_area.py:84-100)
__device__ inline float link_area_scale(const FsiLbmDiag* d, const FsiCouplingParams& cp, float* raw_out) {
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

// ---------------------------------------------------------------- P2G ----
struct P2GParticle {
  float mass, J;
  float mv[3];
  float aff[9];  // -dt vol0 P F^T inv_dx^2 + m C (solid.py:239: no factor 4)
};

// the particle's state read from rows of stride `ld` (global SoA fields with
// ld = n, or a shared-memory stage with ld = chunk size), column `col`
__device__ __forceinline__ void p2g_particle_rows(const float* __restrict__ Frow, const float* __restrict__ Crow,
                                                  const float* __restrict__ vrow, int64_t ld, int col, float mass,
                                                  float vol0, const FsiMpmParams& mp, P2GParticle& q) {
  float Fp[9], Cp[9];
  double Fd[9], Rd[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    Fp[a] = Frow[a * ld + col];
    Cp[a] = Crow[a * ld + col];
    Fd[a] = (double)Fp[a];
  }
  polar_rotation_d(Fd, Rd);
  const float c00 = Fp[4] * Fp[8] - Fp[5] * Fp[7];
  const float c01 = Fp[3] * Fp[8] - Fp[5] * Fp[6];
  const float c02 = Fp[3] * Fp[7] - Fp[4] * Fp[6];
  const float J = Fp[0] * c00 - Fp[1] * c01 + Fp[2] * c02;
  q.J = J;
  // (F^-1)^T = cof(F) / det, as one correctly rounded reciprocal and nine products
  const float iJ = __frcp_rn(J);
  float FinvT[9];
  FinvT[0] = c00 * iJ;
  FinvT[1] = -c01 * iJ;
  FinvT[2] = c02 * iJ;
  FinvT[3] = -(Fp[1] * Fp[8] - Fp[2] * Fp[7]) * iJ;
  FinvT[4] = (Fp[0] * Fp[8] - Fp[2] * Fp[6]) * iJ;
  FinvT[5] = -(Fp[0] * Fp[7] - Fp[1] * Fp[6]) * iJ;
  FinvT[6] = (Fp[1] * Fp[5] - Fp[2] * Fp[4]) * iJ;
  FinvT[7] = -(Fp[0] * Fp[5] - Fp[2] * Fp[3]) * iJ;
  FinvT[8] = (Fp[0] * Fp[4] - Fp[1] * Fp[3]) * iJ;
  const float mu2 = 2.0f * mp.mu, lam = mp.la * (J - 1.0f) * J;
  float P[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) P[a] = mu2 * (Fp[a] - (float)Rd[a]) + lam * FinvT[a];
  const float pre = -mp.dt * vol0;
  q.mass = mass;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float pf = (pre * P[i * 3 + 0]) * Fp[j * 3 + 0] + (pre * P[i * 3 + 1]) * Fp[j * 3 + 1] +
                       (pre * P[i * 3 + 2]) * Fp[j * 3 + 2];
      q.aff[i * 3 + j] = pf * mp.inv_dx * mp.inv_dx + mass * Cp[i * 3 + j];
    }
#pragma unroll
  for (int a = 0; a < 3; ++a) q.mv[a] = mass * vrow[a * ld + col];
}

__device__ __forceinline__ void p2g_particle(const FsiParticles& pt, int p, const FsiMpmParams& mp, P2GParticle& q) {
  p2g_particle_rows(pt.F, pt.C, pt.v, pt.n, p, pt.mass[p], pt.vol0[p], mp, q);
}

// momentum carried to the node at stencil offset (ox, oy, oz)
__device__ __forceinline__ void p2g_node(const P2GParticle& q, const BSpline& b, int ox, int oy, int oz, float dx,
                                         float& w, float mom[3]) {
  const float dpos[3] = {((float)ox - b.fx[0]) * dx, ((float)oy - b.fx[1]) * dx, ((float)oz - b.fx[2]) * dx};
  w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
#pragma unroll
  for (int a = 0; a < 3; ++a) mom[a] = q.mv[a] + (q.aff[a * 3 + 0] * dpos[0] + q.aff[a * 3 + 1] * dpos[1] + q.aff[a * 3 + 2] * dpos[2]);
}

// ---------------------------------------------------------- reaction ----
struct ReactParticle {
  float pf[3];
  float pnorm;
  bool scatter, act, gated;
};

// Per-particle reaction force from the interpolated LBM force density hs and
// solid fraction ps (kind 0: penalty, 1: engineering moving boundary,
// 2: link-area).
__device__ __forceinline__ void reaction_from_sums(const FsiCouplingParams& cp, const float hs[3], float ps, float Jp,
                                                   float vol0, float scale, ReactParticle& r) {
  const float J = fmaxf(Jp, 0.0f);
  const float pv = vol0 * J;
  r.scatter = true;
  r.act = r.gated = false;
  r.pnorm = 0.f;
  if (cp.kind == 0) {
    for (int a = 0; a < 3; ++a) r.pf[a] = hs[a] * cp.force_density_scale * pv * cp.reaction_scale;
  } else if (ps > cp.phi_min) {
    for (int a = 0; a < 3; ++a) {
      r.pf[a] = hs[a] * cp.force_density_scale * pv * cp.reaction_scale;
      if (cp.kind == 2) r.pf[a] = r.pf[a] * scale;
    }
    float nrm = sqrtf(r.pf[0] * r.pf[0] + r.pf[1] * r.pf[1] + r.pf[2] * r.pf[2]);
    if (nrm > cp.force_cap) {
      const float k = cp.force_cap / nrm;
      for (int a = 0; a < 3; ++a) r.pf[a] = r.pf[a] * k;
      nrm = cp.force_cap;
    }
    r.act = nrm > 0.f;
    r.gated = true;
    r.pnorm = nrm;
  } else {
    r.scatter = false;
    r.pf[0] = r.pf[1] = r.pf[2] = 0.f;
  }
}

// the same with the interpolation from the lattice fields in global memory
__device__ __forceinline__ void reaction_particle(const LatView& L, const float* __restrict__ hydro,
                                                  const float* __restrict__ phi, const FsiCouplingParams& cp,
                                                  const BSpline& b, float Jp, float vol0, float scale,
                                                  ReactParticle& r) {
  float hs[3] = {0.f, 0.f, 0.f}, ps = 0.f;
  // stencils wholly inside the lattice (the common case) skip the per-node checks
  const bool inside = b.base[0] >= 0 && b.base[1] >= 0 && b.base[2] >= 0 && b.base[0] + 2 < L.nx &&
                      b.base[1] + 2 < L.ny && b.base[2] + 2 < L.nz;
  const int64_t c000 = inside ? lat_cell(L, b.base[0], b.base[1], b.base[2]) : 0;
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (!inside && (I < 0 || I >= L.nx || Jj < 0 || Jj >= L.ny || K < 0 || K >= L.nz)) continue;
        const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
        const int64_t c = inside ? c000 + ((int64_t)oz * L.ny + oy) * L.nx + ox : lat_cell(L, I, Jj, K);
        hs[0] += w * hydro[c];
        hs[1] += w * hydro[L.pitch + c];
        hs[2] += w * hydro[2 * L.pitch + c];
        if (cp.kind != 0) ps += w * phi[c];
      }
  reaction_from_sums(cp, hs, ps, Jp, vol0, scale, r);
}

// ------------------------------------------------------- grid update ----
// velocity of one node from its momentum, mass and external force, with the
// sticky-wall condition (solid.py:97-111, 251-259); m > 0
__device__ __forceinline__ void grid_node_velocity(const float P[3], float m, const float f[3], int i, int j, int k,
                                                   int G, const FsiMpmParams& mp, float v[3]) {
  const int idx[3] = {i, j, k};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float u = P[a] / m;
    u += mp.dt * mp.gravity[a];
    u += mp.dt * f[a] / m;
    if (idx[a] < mp.bound && u < 0.0f) u = 0.0f;
    if (idx[a] > G - mp.bound && u > 0.0f) u = 0.0f;
    v[a] = u;
  }
}

// ---------------------------------------------------------------- G2P ----
__device__ __forceinline__ float det3(const float (&M)[9]) {
  return M[0] * (M[4] * M[8] - M[5] * M[7]) - M[1] * (M[3] * M[8] - M[5] * M[6]) + M[2] * (M[3] * M[7] - M[4] * M[6]);
}

// advect, clamp, update F and apply the step-112 controls, then store
// (solid.py:261-315); nv and nC are the gathered velocity and affine matrix.
// With a stage (rows x 3, v 3, C 9, F 9 of stride ld, column col) the new
// state is also written there.  fixed_pre / fx_pre: the particle's fixed flag
// and fixed position when the caller loaded them ahead (-1 / null: loaded
// here).
// Fo: the particle's deformation gradient before the substep
__device__ __forceinline__ void g2p_finish_f(const FsiParticles& pt, int p, const FsiMpmParams& mp, float X[3],
                                             const float nv[3], float nC[9], const float Fo[9],
                                             float* stage = nullptr, int ld = 0, int col = 0, int fixed_pre = -1,
                                             const float* fx_pre = nullptr) {
  const int n = pt.n;
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
  float Fn[9];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float acc = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) acc += ((a == k ? 1.0f : 0.0f) + mp.dt * nC[a * 3 + k]) * Fo[k * 3 + c];
      Fn[a * 3 + c] = acc;
    }
  float J = det3(Fn);
  // apply_step112_dynamics_controls (solid.py:301-315)
  if (mp.damping > 0.f) {
    const float d = fmaxf(0.0f, 1.0f - mp.damping * mp.dt);
#pragma unroll
    for (int a = 0; a < 3; ++a) v[a] *= d;
  }
  if (mp.lock_z) {
    X[2] = fx_pre ? fx_pre[2] : pt.fixed_x[2 * n + p];
    v[2] = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      nC[2 * 3 + d] = 0.f;
      nC[d * 3 + 2] = 0.f;
      Fn[2 * 3 + d] = 0.f;
      Fn[d * 3 + 2] = 0.f;
    }
    Fn[8] = 1.0f;
    J = det3(Fn);
  }
  if (fixed_pre >= 0 ? fixed_pre != 0 : pt.fixed[p] != 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      X[a] = fx_pre ? fx_pre[a] : pt.fixed_x[a * n + p];
      v[a] = 0.f;
    }
#pragma unroll
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
  if (stage) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      stage[a * ld + col] = X[a];
      stage[(3 + a) * ld + col] = v[a];
    }
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      stage[(6 + a) * ld + col] = nC[a];
      stage[(15 + a) * ld + col] = Fn[a];
    }
  }
}

__device__ __forceinline__ void g2p_finish(const FsiParticles& pt, int p, const FsiMpmParams& mp, float X[3],
                                           const float nv[3], float nC[9]) {
  float Fo[9];
#pragma unroll
  for (int a = 0; a < 9; ++a) Fo[a] = pt.F[(int64_t)a * pt.n + p];
  g2p_finish_f(pt, p, mp, X, nv, nC, Fo);
}

// one gathered node's contribution to the particle velocity and affine matrix
__device__ __forceinline__ void g2p_node(const BSpline& b, int ox, int oy, int oz, float dx, float s4, const float gv[3],
                                         float nv[3], float nC[9]) {
  const float dpos[3] = {((float)ox - b.fx[0]) * dx, ((float)oy - b.fx[1]) * dx, ((float)oz - b.fx[2]) * dx};
  const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    nv[a] += w * gv[a];
#pragma unroll
    for (int c = 0; c < 3; ++c) nC[a * 3 + c] += (w * gv[a]) * dpos[c] * s4;
  }
}

}  // namespace fsi

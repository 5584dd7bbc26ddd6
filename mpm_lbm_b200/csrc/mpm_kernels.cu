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

#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "mpm_common.cuh"

namespace fsi {

// ---------------------------------------------------------- projection ----
__device__ __forceinline__ void project_particle(const LatView& L, const FsiParticles& pt, const FsiCouplingParams& cp,
                                                 float* phi, float* smass, float* svel, int p) {
  const int n = pt.n;
  const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
  BSpline b;
  bspline(X, cp.inv_dx_norm, b);
  const float J = fmaxf(pt.Jp[p], 0.0f);
  const float cur_vol = pt.vol0[p] * J;
  const float m = pt.mass[p];
  const float vl[3] = {pt.v[p] * cp.vel_scale, pt.v[n + p] * cp.vel_scale, pt.v[2 * n + p] * cp.vel_scale};
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
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

__global__ void k_project_scatter(LatView L, FsiParticles pt, FsiCouplingParams cp, float* phi, float* smass,
                                  float* svel) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < pt.n) project_particle(L, pt, cp, phi, smass, svel, p);
}

// cells base + lane of one warp (base warp-uniform: the reductions need the
// whole warp)
__device__ __forceinline__ void project_normalize_warp(const LatView& L, const FsiCouplingParams& cp, float* phi,
                                                       float* smass, float* svel, FsiCouplingStats* st,
                                                       int64_t base) {
  const int64_t n = (int64_t)L.nx * L.ny * L.nz;
  const int64_t c = base + (threadIdx.x & 31);
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

__global__ void k_project_normalize(LatView L, FsiCouplingParams cp, float* phi, float* smass, float* svel,
                                    FsiCouplingStats* st) {
  project_normalize_warp(L, cp, phi, smass, svel, st,
                         (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31));
}

// ------------------------------------------------------------ reaction ----
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
    ReactParticle r;
    reaction_particle(L, hydro, phi, cp, b, pt.Jp[p], pt.vol0[p], s_scale, r);
    for (int a = 0; a < 3; ++a) pf[a] = r.pf[a];
    act = r.act;
    gated = r.gated;
    pnorm = r.pnorm;
    const bool scatter = r.scatter;
    if (scatter) {
      const int64_t N = (int64_t)g.n * g.n * g.n;
#pragma unroll
      for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
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
  P2GParticle q;
  p2g_particle(pt, p, mp, q);
  pt.Jp[p] = q.J;
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
        float w, mom[3];
        p2g_node(q, b, ox, oy, oz, mp.dx, w, mom);
        const int64_t node = ((int64_t)K * G + Jj) * G + I;
#pragma unroll
        for (int a = 0; a < 3; ++a) atomicAdd(g.v + a * N + node, w * mom[a]);
        atomicAdd(g.m + node, w * q.mass);
      }
}

__global__ void k_grid_update(FsiGrid g, FsiMpmParams mp) {
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N) return;
  const float m = g.m[node];
  if (!(m > 0.0f)) return;
  const float P[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
  const float f[3] = {g.f_ext[node], g.f_ext[N + node], g.f_ext[2 * N + node]};
  float v[3];
  grid_node_velocity(P, m, f, (int)(node % G), (int)((node / G) % G), (int)(node / ((int64_t)G * G)), G, mp, v);
#pragma unroll
  for (int a = 0; a < 3; ++a) g.v[a * N + node] = v[a];
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
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
        const int64_t node = ((int64_t)K * G + Jj) * G + I;
        const float gv[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
        g2p_node(b, ox, oy, oz, mp.dx, s4, gv, nv, nC);
      }
  g2p_finish(pt, p, mp, X, nv, nC);
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

// ---- batched cases: projection (grid.y = case slot) -------------------------
namespace fsi {
namespace {

__device__ __forceinline__ LatView lat_of(const FsiBatchCase& bc) {
  return LatView{bc.lbm.nx, bc.lbm.ny, bc.lbm.nz, bc.lbm.pitch};
}

// fsi_project's clears: solid_phi, solid_mass, solid_vel and the projection
// reductions
__global__ void k_batch_project_clear(FsiBatchCase* cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const int64_t P = bc.lbm.pitch;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P; i += stride) {
    bc.lbm.phi[i] = 0.f;
    bc.lbm.smass[i] = 0.f;
    bc.lbm.svel[i] = 0.f;
    bc.lbm.svel[P + i] = 0.f;
    bc.lbm.svel[2 * P + i] = 0.f;
  }
  if (blockIdx.x == 0) {
    int* w = reinterpret_cast<int*>(bc.proj_stats);
    for (int i = threadIdx.x; i < (int)(offsetof(FsiCouplingStats, active_reaction_particle_count) / 4);
         i += blockDim.x)
      w[i] = 0;
  }
}

__global__ void k_batch_project_scatter(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const LatView L = lat_of(bc);
  const FsiParticles pt = bc.pt;
  const FsiCouplingParams cp = bc.cp;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < pt.n; p += gridDim.x * blockDim.x)
    project_particle(L, pt, cp, bc.lbm.phi, bc.lbm.smass, bc.lbm.svel, p);
}

__global__ void k_batch_project_normalize(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const LatView L = lat_of(bc);
  const FsiCouplingParams cp = bc.cp;
  const int64_t n = (int64_t)L.nx * L.ny * L.nz;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride)
    project_normalize_warp(L, cp, bc.lbm.phi, bc.lbm.smass, bc.lbm.svel, bc.proj_stats, base);
}

}  // namespace
}  // namespace fsi

extern "C" int fsi_batch_project(FsiBatchCase* cases, const FsiBatchDims* d, void* stream) {
  if (!cases || !d || d->n_cases <= 0 || d->n_cases > 65535 || d->max_cells <= 0 || d->max_particles <= 0)
    return invalid("bad batch arguments");
  cudaStream_t st = (cudaStream_t)stream;
  // one CTA per 256 cells / 128 particles of the largest case (smaller cases' extra CTAs exit at once)
  const int64_t cap = 1 << 20;
  const unsigned gc = (unsigned)std::min<int64_t>((d->max_cells + 255) / 256, cap);
  k_batch_project_clear<<<dim3(gc, d->n_cases), 256, 0, st>>>(cases);
  int rc = launch_check("k_batch_project_clear");
  if (rc) return rc;
  const unsigned gp = (unsigned)std::min<int64_t>((d->max_particles + 127) / 128, cap);
  k_batch_project_scatter<<<dim3(gp, d->n_cases), 128, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_project_scatter"))) return rc;
  k_batch_project_normalize<<<dim3(gc, d->n_cases), 256, 0, st>>>(cases);
  return launch_check("k_batch_project_normalize");
}

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
#include <climits>
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

// normalize_projection (projection.py:67-91) of one cell, with the cell's
// share of the projection statistics accumulated in a
struct ProjAcc {
  double pm = 0.0, pvr = 0.0, pvc = 0.0;
  float mx = 0.f;
  int na = 0;
};

__device__ __forceinline__ void project_normalize_cell(const LatView& L, const FsiCouplingParams& cp, float* phi,
                                                       float* smass, float* svel, int64_t c, ProjAcc& a) {
  const float raw = phi[c];
  const float m = smass[c];
  a.mx = fmaxf(a.mx, raw);
  if (m > cp.eps_mass) {
    for (int q = 0; q < 3; ++q) svel[q * L.pitch + c] = svel[q * L.pitch + c] / m;
  } else {
    for (int q = 0; q < 3; ++q) svel[q * L.pitch + c] = 0.f;
  }
  const float cl = fminf(1.0f, fmaxf(0.0f, raw));
  phi[c] = cl;
  a.na += cl > 1.0e-8f;
  a.pm += m;
  a.pvr += (double)raw * cp.cell_volume_norm;
  a.pvc += (double)cl * cp.cell_volume_norm;
}

// the CTA's statistics into st: warp sums, then the CTA's warps in shared
// memory, then one atomic per CTA and value (an atomic per warp serialised
// tens of thousands of FP64 adds on five addresses)
__device__ __forceinline__ void project_stats_flush(ProjAcc a, FsiCouplingStats* st) {
  __shared__ double s_d[32][3];
  __shared__ float s_m[32];
  __shared__ int s_n[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a.pm = warp_sum_d(a.pm);
  a.pvr = warp_sum_d(a.pvr);
  a.pvc = warp_sum_d(a.pvc);
  a.mx = warp_max(fmaxf(a.mx, 0.f));
  a.na = __reduce_add_sync(0xffffffffu, (unsigned)a.na);
  if (lane == 0) {
    s_d[wid][0] = a.pm;
    s_d[wid][1] = a.pvr;
    s_d[wid][2] = a.pvc;
    s_m[wid] = a.mx;
    s_n[wid] = a.na;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    ProjAcc t;
    for (int w = 0; w < nw; ++w) {
      t.pm += s_d[w][0];
      t.pvr += s_d[w][1];
      t.pvc += s_d[w][2];
      t.mx = fmaxf(t.mx, s_m[w]);
      t.na += s_n[w];
    }
    if (t.pm != 0.0) atomicAdd(&st->projected_mass, t.pm);
    if (t.pvr != 0.0) atomicAdd(&st->projected_volume_raw, t.pvr);
    if (t.pvc != 0.0) atomicAdd(&st->projected_volume_clamped, t.pvc);
    if (t.mx > 0.f) atomic_max_nonneg(&st->max_phi_raw, t.mx);
    if (t.na) atomicAdd(&st->active_cell_count, t.na);
  }
}

// grid-stride over the cells (every thread of the CTA reaches the flush)
__global__ void k_project_normalize(LatView L, FsiCouplingParams cp, float* phi, float* smass, float* svel,
                                    FsiCouplingStats* st) {
  const int64_t n = (int64_t)L.nx * L.ny * L.nz;
  ProjAcc a;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    project_normalize_cell(L, cp, phi, smass, svel, c, a);
  project_stats_flush(a, st);
}

// ------------------------------------- projection in particle order ----
// projection.py:39-65 adds, for particle p = 0, 1, ... and its 27 stencil
// offsets, w * vol / cell_volume, w * m and w * m * v to the cells; a serial
// run sums every cell's terms in ascending p.  Here particles are sorted by
// B-spline base cell (a counting sort over the bounding box of the base cells,
// each base cell's list then ordered by p), and one warp per cell collects the
// contributors of its <= 27 base cells, ranks them by p and sums the terms in
// that order with IEEE FP32 adds.  The term arithmetic is written with
// explicit round-to-nearest operations, so no multiply-add is contracted and
// every term is the one a serial FP32 run computes.
//
// scratch->box: [0..2] max(-base), [3..5] max(base) over the particles whose
// base cell touches the lattice (base in [-2, dim - 1] on each axis); a memset
// of 0x80 bytes (INT_MIN-like) is the empty box.

struct OrdBase {
  int b[3];
  float fx[3];
};

__device__ __forceinline__ OrdBase ordered_base(const FsiParticles& pt, int p, float inv_dx) {
  OrdBase o;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float Xp = __fmul_rn(pt.x[a * pt.n + p], inv_dx);
    o.b[a] = (int)__fsub_rn(Xp, 0.5f);
    o.fx[a] = __fsub_rn(Xp, (float)o.b[a]);
  }
  return o;
}

__device__ __forceinline__ bool ordered_base_touches(const LatView& L, const OrdBase& o) {
  return o.b[0] >= -2 && o.b[0] < L.nx && o.b[1] >= -2 && o.b[1] < L.ny && o.b[2] >= -2 && o.b[2] < L.nz;
}

// quadratic B-spline weight of offset d for fractional position f, in the
// reference's evaluation order (solid.py:222-230 / projection.py:45-47)
__device__ __forceinline__ float ordered_w(float f, int d) {
  if (d == 0) {
    const float t = __fsub_rn(1.5f, f);
    return __fmul_rn(__fmul_rn(0.5f, t), t);
  }
  if (d == 1) {
    const float t = __fsub_rn(f, 1.0f);
    return __fsub_rn(0.75f, __fmul_rn(t, t));
  }
  const float t = __fsub_rn(f, 0.5f);
  return __fmul_rn(__fmul_rn(0.5f, t), t);
}

struct OrdBox {
  int lo[3], hi[3], ext[3];
  int64_t keys;
};

__device__ __forceinline__ OrdBox ordered_box(const int32_t* box) {
  OrdBox B;
  int64_t k = 1;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    B.lo[a] = -box[a];
    B.hi[a] = box[3 + a];
    B.ext[a] = B.hi[a] >= B.lo[a] ? B.hi[a] - B.lo[a] + 1 : 0;
    k *= B.ext[a];
  }
  B.keys = k;
  return B;
}

__global__ void k_po_box(LatView L, FsiParticles pt, float inv_dx, int32_t* __restrict__ box) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  int v[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) v[a] = INT_MIN;
  if (p < pt.n) {
    const OrdBase o = ordered_base(pt, p, inv_dx);
    if (ordered_base_touches(L, o)) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        v[a] = -o.b[a];
        v[3 + a] = o.b[a];
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v[a] = max(v[a], __shfl_xor_sync(0xffffffffu, v[a], s));
  }
  if ((threadIdx.x & 31) == 0 && v[3] != INT_MIN) {
#pragma unroll
    for (int a = 0; a < 6; ++a) atomicMax(box + a, v[a]);
  }
}

__device__ __forceinline__ int ordered_key(const OrdBox& B, const int b[3]) {
  return ((b[2] - B.lo[2]) * B.ext[1] + (b[1] - B.lo[1])) * B.ext[0] + (b[0] - B.lo[0]);
}

__global__ void k_po_count(LatView L, FsiParticles pt, float inv_dx, const int32_t* __restrict__ box,
                           int32_t* __restrict__ key, int32_t* __restrict__ count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pt.n) return;
  const OrdBox B = ordered_box(box);
  const OrdBase o = ordered_base(pt, p, inv_dx);
  int k = -1;
  if (ordered_base_touches(L, o)) {
    k = ordered_key(B, o.b);
    atomicAdd(count + k, 1);
  }
  key[p] = k;
}

// one CTA: exclusive scan of count[0, keys) into start[0, keys], count zeroed
constexpr int kPoScanT = 1024;
__global__ __launch_bounds__(kPoScanT) void k_po_scan(const int32_t* __restrict__ box, int32_t* __restrict__ count,
                                                      int32_t* __restrict__ start) {
  __shared__ int s_w[kPoScanT / 32];
  const OrdBox B = ordered_box(box);
  const int nk = (int)B.keys;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int per = (nk + kPoScanT - 1) / kPoScanT;
  const int k0 = min(t * per, nk), k1 = min(k0 + per, nk);
  int sum = 0;
  for (int k = k0; k < k1; ++k) sum += count[k];
  int inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_w[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const int a0 = s_w[lane];
    int a = a0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, a, o);
      if (lane >= o) a += y;
    }
    s_w[lane] = a - a0;
  }
  __syncthreads();
  int off = s_w[wid] + inc - sum;
  for (int k = k0; k < k1; ++k) {
    const int c = count[k];
    start[k] = off;
    count[k] = 0;
    off += c;
  }
  if (t == kPoScanT - 1) start[nk] = off;
}

__global__ void k_po_fill(int n, const int32_t* __restrict__ key, const int32_t* __restrict__ start,
                          int32_t* __restrict__ cursor, int32_t* __restrict__ list) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = key[p];
  if (k >= 0) list[start[k] + atomicAdd(cursor + k, 1)] = p;
}

// orders each base cell's list by particle id and leaves count zero
__global__ void k_po_sort(const int32_t* __restrict__ box, const int32_t* __restrict__ start,
                          int32_t* __restrict__ count, int32_t* __restrict__ list) {
  const int64_t nk = ordered_box(box).keys;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += (int64_t)gridDim.x * blockDim.x) {
    const int s = start[k], e = start[k + 1];
    if (e - s > 1) {
      for (int i = s + 1; i < e; ++i) {
        const int v = list[i];
        int j = i - 1;
        while (j >= s && list[j] > v) {
          list[j + 1] = list[j];
          --j;
        }
        list[j + 1] = v;
      }
    }
    if (e > s) count[k] = 0;
  }
}

// the five terms particle p adds to the cell at offset d from its base cell
__device__ __forceinline__ void ordered_terms(const FsiParticles& pt, const FsiCouplingParams& cp, int p,
                                              const OrdBase& o, const int d[3], float t[5]) {
  const int n = pt.n;
  const float w = __fmul_rn(__fmul_rn(ordered_w(o.fx[0], d[0]), ordered_w(o.fx[1], d[1])), ordered_w(o.fx[2], d[2]));
  const float J = fmaxf(pt.Jp[p], 0.0f);
  const float cur_vol = __fmul_rn(pt.vol0[p], J);
  const float mc = __fmul_rn(w, pt.mass[p]);
  t[0] = __fdiv_rn(__fmul_rn(w, cur_vol), cp.cell_volume_norm);
  t[1] = mc;
#pragma unroll
  for (int a = 0; a < 3; ++a) t[2 + a] = __fmul_rn(mc, __fmul_rn(pt.v[a * n + p], cp.vel_scale));
}

constexpr int kPoWarps = 4;
constexpr int kPoCap = 504;             // contributors per cell ranked in shared memory
constexpr int kPoStride = kPoCap + 1;   // term rows on distinct banks

__global__ __launch_bounds__(32 * kPoWarps) void k_po_gather(LatView L, FsiParticles pt, FsiCouplingParams cp,
                                                             const int32_t* __restrict__ box,
                                                             const int32_t* __restrict__ start,
                                                             const int32_t* __restrict__ list, float* __restrict__ phi,
                                                             float* __restrict__ smass, float* __restrict__ svel) {
  __shared__ int s_cand[kPoWarps][kPoCap];
  __shared__ float s_term[kPoWarps][5 * kPoStride];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int* cand = s_cand[wid];
  float* term = s_term[wid];
  const OrdBox B = ordered_box(box);
  if (B.keys == 0) return;
  // cells reached from the box: [lo, hi + 2] clipped to the lattice
  int clo[3], cext[3];
  const int dims[3] = {L.nx, L.ny, L.nz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    clo[a] = max(B.lo[a], 0);
    cext[a] = max(min(B.hi[a] + 2, dims[a] - 1) - clo[a] + 1, 0);
  }
  const int64_t ncell = (int64_t)cext[0] * cext[1] * cext[2];
  // lane l < 27 owns stencil offset d = (l / 9, l / 3 % 3, l % 3): base cell = cell - d
  const int d[3] = {lane / 9, (lane / 3) % 3, lane % 3};
  for (int64_t q = (int64_t)blockIdx.x * kPoWarps + wid; q < ncell; q += (int64_t)gridDim.x * kPoWarps) {
    const int ci = clo[0] + (int)(q % cext[0]);
    const int cj = clo[1] + (int)((q / cext[0]) % cext[1]);
    const int ck = clo[2] + (int)(q / ((int64_t)cext[0] * cext[1]));
    const int b[3] = {ci - d[0], cj - d[1], ck - d[2]};
    int s = 0, len = 0;
    if (lane < 27 && b[0] >= B.lo[0] && b[0] <= B.hi[0] && b[1] >= B.lo[1] && b[1] <= B.hi[1] && b[2] >= B.lo[2] &&
        b[2] <= B.hi[2]) {
      const int k = ordered_key(B, b);
      s = start[k];
      len = start[k + 1] - s;
    }
    int off = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, off, o);
      if (lane >= o) off += y;
    }
    const int K = __shfl_sync(0xffffffffu, off, 31);
    off -= len;
    if (K == 0) continue;
    const int64_t c = lat_cell(L, ci, cj, ck);
    float acc = 0.f;  // lane v < 5: running sum of term v
    if (K <= kPoCap) {
      for (int i = 0; i < len; ++i) cand[off + i] = list[s + i];
      __syncwarp();
      for (int i = lane; i < K; i += 32) {
        const int p = cand[i];
        int rank = 0;
        for (int j = 0; j < K; ++j) rank += cand[j] < p;
        const OrdBase o = ordered_base(pt, p, cp.inv_dx_norm);
        const int dd[3] = {ci - o.b[0], cj - o.b[1], ck - o.b[2]};
        float t[5];
        ordered_terms(pt, cp, p, o, dd, t);
#pragma unroll
        for (int v = 0; v < 5; ++v) term[v * kPoStride + rank] = t[v];
      }
      __syncwarp();
      if (lane < 5)
        for (int r = 0; r < K; ++r) acc = __fadd_rn(acc, term[lane * kPoStride + r]);
      __syncwarp();
    } else {
      // more contributors than the shared ranking holds: lane 0 merges the 27
      // sorted base-cell lists (heads and ends staged in cand), kPoCap terms at
      // a time, and lanes 0-4 continue their sums over each batch
      if (lane < 27) {
        cand[lane] = s;
        cand[27 + lane] = s + len;
      }
      __syncwarp();
      for (int done = 0; done < K; done += kPoCap) {
        const int m = min(kPoCap, K - done);
        if (lane == 0) {
          for (int r = 0; r < m; ++r) {
            int best = INT_MAX, bl = 0;
            for (int l = 0; l < 27; ++l) {
              const int h = cand[l];
              if (h < cand[27 + l]) {
                const int v = list[h];
                if (v < best) {
                  best = v;
                  bl = l;
                }
              }
            }
            cand[bl] += 1;
            const OrdBase o = ordered_base(pt, best, cp.inv_dx_norm);
            const int dd[3] = {ci - o.b[0], cj - o.b[1], ck - o.b[2]};
            float t[5];
            ordered_terms(pt, cp, best, o, dd, t);
#pragma unroll
            for (int v = 0; v < 5; ++v) term[v * kPoStride + r] = t[v];
          }
        }
        __syncwarp();
        if (lane < 5)
          for (int r = 0; r < m; ++r) acc = __fadd_rn(acc, term[lane * kPoStride + r]);
        __syncwarp();
      }
    }
    if (lane < 5) {
      float* dst = lane == 0 ? phi + c : (lane == 1 ? smass + c : svel + (int64_t)(lane - 2) * L.pitch + c);
      *dst = acc;
    }
  }
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
  k_project_normalize<<<(unsigned)std::min<int64_t>(nblk(n, 256), 8LL * device_sm_count()), 256, 0, st>>>(
      L, *cp, s->phi, s->smass, s->svel, stats);
  return launch_check("k_project_normalize");
}

extern "C" int fsi_project_ordered(const FsiLbmState* s, const FsiParticles* pt, const FsiCouplingParams* cp,
                                   const FsiProjectScratch* sc, FsiCouplingStats* stats, void* stream) {
  if (!s || !cp || !sc || !stats) return invalid("null argument");
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!s->phi || !s->smass || !s->svel) return invalid("projection needs phi, smass, svel");
  if (!sc->count || !sc->start || !sc->list || !sc->key || !sc->box) return invalid("null projection scratch array");
  const int64_t keys = (int64_t)(s->nx + 2) * (s->ny + 2) * (s->nz + 2);
  if (keys > INT_MAX - 1) return invalid("lattice too large for the ordered projection");
  if (sc->key_capacity < keys) return invalid("scratch key_capacity below (nx + 2) * (ny + 2) * (nz + 2)");
  if (sc->particle_capacity < pt->n) return invalid("scratch particle_capacity below the particle count");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t P = s->pitch;
  if ((rc = cuda_check(cudaMemsetAsync(s->phi, 0, sizeof(float) * P, st), "clear phi"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(s->smass, 0, sizeof(float) * P, st), "clear smass"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(s->svel, 0, sizeof(float) * 3 * P, st), "clear svel"))) return rc;
  if ((rc = cuda_check(cudaMemsetAsync(stats, 0, offsetof(FsiCouplingStats, active_reaction_particle_count), st),
                       "clear projection stats")))
    return rc;
  if ((rc = cuda_check(cudaMemsetAsync(sc->box, 0x80, 6 * sizeof(int32_t), st), "clear projection box"))) return rc;
  const LatView L{s->nx, s->ny, s->nz, P};
  const float inv_dx = cp->inv_dx_norm;
  const int sms = device_sm_count();
  k_po_box<<<nblk(pt->n, 256), 256, 0, st>>>(L, *pt, inv_dx, sc->box);
  if ((rc = launch_check("k_po_box"))) return rc;
  k_po_count<<<nblk(pt->n, 256), 256, 0, st>>>(L, *pt, inv_dx, sc->box, sc->key, sc->count);
  if ((rc = launch_check("k_po_count"))) return rc;
  k_po_scan<<<1, kPoScanT, 0, st>>>(sc->box, sc->count, sc->start);
  if ((rc = launch_check("k_po_scan"))) return rc;
  k_po_fill<<<nblk(pt->n, 256), 256, 0, st>>>(pt->n, sc->key, sc->start, sc->count, sc->list);
  if ((rc = launch_check("k_po_fill"))) return rc;
  k_po_sort<<<sms * 2, 256, 0, st>>>(sc->box, sc->start, sc->count, sc->list);
  if ((rc = launch_check("k_po_sort"))) return rc;
  k_po_gather<<<sms * 8, 32 * kPoWarps, 0, st>>>(L, *pt, *cp, sc->box, sc->start, sc->list, s->phi, s->smass,
                                                 s->svel);
  if ((rc = launch_check("k_po_gather"))) return rc;
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_project_normalize<<<(unsigned)std::min<int64_t>(nblk(n, 256), 8LL * device_sm_count()), 256, 0, st>>>(
      L, *cp, s->phi, s->smass, s->svel, stats);
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
  ProjAcc a;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x)
    project_normalize_cell(L, cp, bc.lbm.phi, bc.lbm.smass, bc.lbm.svel, c, a);
  project_stats_flush(a, bc.proj_stats);
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

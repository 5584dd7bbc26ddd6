// Binned MPM substep: particles sorted by 4x4x4-cell block, P2G (+ reaction
// transfer) staged in a shared-memory tile per chunk of a bin, G2P with the
// grid update evaluated while staging the chunk's node box, and two grid
// buffers so that only the boxes touched one substep earlier are zeroed.
//
// The per-particle and per-node arithmetic is the one of the one-phase
// kernels (mpm_common.cuh): solid.py:212-315 and the reaction transfers of
// penalty.py:90-129, moving_boundary.py:58-110, link_area.py:84-193.  Only
// the summation order of the grid sums differs (shared-memory atomics, then
// one global atomic per chunk and touched node value).

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "common.cuh"
#include "mpm_common.cuh"

namespace fsi {
namespace {

constexpr int kChunk = FSI_BIN_CHUNK;  // particles per chunk
constexpr int kEdge = FSI_BIN_EDGE;
// nodes staged per CTA: a chunk of one bin spans (4 + 3)^3 = 343 nodes; the
// rest absorbs drift since the last binning (a 10^3 box).  7 floats per node
// in P2G = 28 KB.
constexpr int kTileCap = 1000;

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// bin of a particle: the cell block of its B-spline base cell (solid.py:222-223)
__device__ __forceinline__ int particle_bin(const float X[3], float inv_dx, int G, int nb) {
  int c[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float Xp = __fmul_rn(X[a], inv_dx);
    c[a] = clampi((int)(Xp - 0.5f), 0, G - 1) / kEdge;
  }
  return (c[2] * nb + c[1]) * nb + c[0];
}

__device__ __forceinline__ void bin_count_body(const FsiParticles& pt, float inv_dx, int G, int nb,
                                               int32_t* __restrict__ key, int32_t* __restrict__ count, int vb, int vg) {
  const int p = vb * blockDim.x + threadIdx.x;
  if (p >= pt.n) return;
  const int n = pt.n;
  const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
  const int k = particle_bin(X, inv_dx, G, nb);
  key[p] = k;
  atomicAdd(count + k, 1);
}

__global__ void k_bin_count(FsiParticles pt, float inv_dx, int G, int nb, int32_t* __restrict__ key,
                            int32_t* __restrict__ count) {
  bin_count_body(pt, inv_dx, G, nb, key, count, blockIdx.x, gridDim.x);
}

// One CTA: exclusive scan of the bin counts and of the chunks per bin, the
// chunk table, and the counts reset to zero for the next binning.  Each
// thread owns a contiguous, 4-aligned range of bins and reads it with 16-byte
// loads, so the pass costs a few memory latencies rather than one per bin.
__device__ __forceinline__ int4 ld_bins4(const int32_t* p, int b, int b1) {
  if (b + 4 <= b1) return *reinterpret_cast<const int4*>(p + b);
  int4 v = make_int4(0, 0, 0, 0);
  if (b < b1) v.x = p[b];
  if (b + 1 < b1) v.y = p[b + 1];
  if (b + 2 < b1) v.z = p[b + 2];
  return v;
}

__device__ __forceinline__ void bin_scan_body(int nbins, int32_t* __restrict__ count, int32_t* __restrict__ start,
                                              int2* __restrict__ chunk, int32_t* __restrict__ meta) {
  __shared__ int s_p[32], s_c[32];
  const int T = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int per = ((nbins + T - 1) / T + 3) & ~3;
  const int b0 = min(tid * per, nbins), b1 = min(b0 + per, nbins);
  int ps = 0, cs = 0;
  for (int b = b0; b < b1; b += 4) {
    const int4 c = ld_bins4(count, b, b1);
    ps += c.x + c.y + c.z + c.w;
    cs += (c.x + kChunk - 1) / kChunk + (c.y + kChunk - 1) / kChunk + (c.z + kChunk - 1) / kChunk +
          (c.w + kChunk - 1) / kChunk;
  }
  int pi = ps, ci = cs;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int a = __shfl_up_sync(0xffffffffu, pi, o), c = __shfl_up_sync(0xffffffffu, ci, o);
    if (lane >= o) {
      pi += a;
      ci += c;
    }
  }
  if (lane == 31) {
    s_p[wid] = pi;
    s_c[wid] = ci;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = T >> 5;
    const int a0 = lane < nw ? s_p[lane] : 0, c0 = lane < nw ? s_c[lane] : 0;
    int a = a0, c = c0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, a, o), y = __shfl_up_sync(0xffffffffu, c, o);
      if (lane >= o) {
        a += x;
        c += y;
      }
    }
    if (lane < nw) {
      s_p[lane] = a - a0;
      s_c[lane] = c - c0;
    }
  }
  __syncthreads();
  int po = s_p[wid] + pi - ps, co = s_c[wid] + ci - cs;
  for (int b = b0; b < b1; b += 4) {
    const int4 c4 = ld_bins4(count, b, b1);
    const int cv[4] = {c4.x, c4.y, c4.z, c4.w};
    int st[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      st[q] = po;
      for (int j = 0; j < cv[q]; j += kChunk) chunk[co++] = make_int2(po + j, min(kChunk, cv[q] - j));
      po += cv[q];
    }
    if (b + 4 <= b1) {
      *reinterpret_cast<int4*>(start + b) = make_int4(st[0], st[1], st[2], st[3]);
      *reinterpret_cast<int4*>(count + b) = make_int4(0, 0, 0, 0);
    } else {
      for (int q = 0; q < 4 && b + q < b1; ++q) {
        start[b + q] = st[q];
        count[b + q] = 0;
      }
    }
  }
  if (tid == T - 1) meta[0] = co;
}

__global__ __launch_bounds__(1024) void k_bin_scan(int nbins, int32_t* __restrict__ count,
                                                   int32_t* __restrict__ start, int2* __restrict__ chunk,
                                                   int32_t* __restrict__ meta) {
  bin_scan_body(nbins, count, start, chunk, meta);
}

__device__ __forceinline__ void bin_scatter_body(int n, const int32_t* __restrict__ key,
                                                 int32_t* __restrict__ cursor, int32_t* __restrict__ perm, int vb,
                                                 int vg) {
  const int p = vb * blockDim.x + threadIdx.x;
  if (p >= n) return;
  perm[atomicAdd(cursor + key[p], 1)] = p;
}

__global__ void k_bin_scatter(int n, const int32_t* __restrict__ key, int32_t* __restrict__ cursor,
                              int32_t* __restrict__ perm) {
  bin_scatter_body(n, key, cursor, perm, blockIdx.x, gridDim.x);
}

struct Box {
  int lo[3], ext[3];
  int vol;
};

__device__ __forceinline__ Box load_box(const int32_t* r) {
  Box b;
  long long v = 1;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = r[a];
    b.ext[a] = max(r[3 + a] - r[a] + 1, 0);
    v *= b.ext[a];
  }
  b.vol = v > INT_MAX ? INT_MAX : (int)v;
  return b;
}

__device__ __forceinline__ int64_t box_node(const Box& b, int li, int G) {
  const int i = b.lo[0] + li % b.ext[0];
  const int j = b.lo[1] + (li / b.ext[0]) % b.ext[1];
  const int k = b.lo[2] + li / (b.ext[0] * b.ext[1]);
  return ((int64_t)k * G + j) * G + i;
}

// quadratic B-spline weight of offset o for the fractional position f (the
// expressions of bspline())
__device__ __forceinline__ float bspline_w(float f, int o) {
  return o == 0 ? 0.5f * (1.5f - f) * (1.5f - f) : (o == 1 ? 0.75f - (f - 1.0f) * (f - 1.0f) : 0.5f * (f - 0.5f) * (f - 0.5f));
}

// Fallbacks for chunks whose node box does not fit the shared-memory tile
// (bins gone stale): rolled loops, so that the staged path stays compact.
__device__ __forceinline__ void g2p_gather_global(const FsiGrid& g, const FsiMpmParams& mp, const BSpline& b,
                                                  float nvl[3], float nC[9]) {
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const float s4 = 4.0f * mp.inv_dx * mp.inv_dx;
#pragma unroll 1
  for (int o = 0; o < 27; ++o) {
    const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
    const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
    if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
    const int64_t node = ((int64_t)K * G + Jj) * G + I;
    const float m = g.m[node];
    const float P[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
    float gv[3] = {P[0], P[1], P[2]};
    if (m > 0.0f) {
      const float f[3] = {g.f_ext[node], g.f_ext[N + node], g.f_ext[2 * N + node]};
      grid_node_velocity(P, m, f, I, Jj, K, G, mp, gv);
    }
    const float dpos[3] = {((float)ox - b.fx[0]) * mp.dx, ((float)oy - b.fx[1]) * mp.dx, ((float)oz - b.fx[2]) * mp.dx};
    const float w = bspline_w(b.fx[0], ox) * bspline_w(b.fx[1], oy) * bspline_w(b.fx[2], oz);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      nvl[a] += w * gv[a];
#pragma unroll
      for (int c = 0; c < 3; ++c) nC[a * 3 + c] += (w * gv[a]) * dpos[c] * s4;
    }
  }
}

// Per-particle P2G payload, one row per quantity, one column per particle slot
// (the particle's position in the bin order perm): fractional position, base
// node, momentum, affine matrix, mass, reaction force, and the B-spline
// weights [axis][offset].
enum { kPfx = 0, kPbase = 3, kPmv = 6, kPaff = 9, kPmass = 18, kPpf = 19, kPw = 22, kPn = 31 };
static_assert(kPn <= FSI_MPM_PAYLOAD_ROWS, "payload rows exceed the caller's buffer");

// P2G, per particle (one thread per slot): fixed-corotated stress and affine
// momentum with the FP64 polar rotation (solid.py:231-249), the reaction force
// gathered from the lattice hydro force (penalty.py:90-129,
// moving_boundary.py:58-110, link_area.py:139-193) and its reductions, and the
// particle's B-spline data -- written to the payload for the scatter kernel.
template <bool REACT>
__device__ __forceinline__ void p2g_payload_body(const FsiParticles& pt, const FsiMpmParams& mp,
                                                 const int32_t* __restrict__ perm, float* __restrict__ payload,
                                                 const LatView& L, const float* __restrict__ hydro,
                                                 const float* __restrict__ phi, const FsiCouplingParams& cp,
                                                 FsiCouplingStats* st, const FsiLbmDiag* diag, int vb, int vg) {
  __shared__ float s_scale;
  const int n = pt.n;
  if (REACT) {
    if (threadIdx.x == 0) {
      float raw = 1.f;
      s_scale = cp.kind == 2 ? link_area_scale(diag, cp, &raw) : 1.0f;
      if (vb == 0 && cp.kind == 2) {
        st->area_scale = s_scale;
        st->raw_area_scale = raw;
      }
    }
    __syncthreads();
  }
  int n_act = 0;
  float pmax = 0.f;
  double pn[3] = {0.0, 0.0, 0.0};
  // two lanes per particle slot, in different warps of the CTA so that the two
  // halves of the work run side by side instead of one after the other:
  // warps of role 0 the stress and affine momentum (FP64 polar rotation),
  // warps of role 1 the B-spline data and the reaction force (with its own
  // det F for the volume).  Warp w of the CTA covers slots
  // (vb * blockDim.x / 2) + (w / 2) * 32 + lane with role w % 2.
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pslot = vb * (blockDim.x >> 1) + (wid >> 1) * 32 + lane, role = wid & 1;
  if (pslot < n) {
    const int p = perm[pslot];
    float* const col = payload + pslot;
    if (role == 0) {
      P2GParticle q;
      p2g_particle(pt, p, mp, q);
      pt.Jp[p] = q.J;
#pragma unroll
      for (int a = 0; a < 3; ++a) col[(int64_t)(kPmv + a) * n] = q.mv[a];
#pragma unroll
      for (int a = 0; a < 9; ++a) col[(int64_t)(kPaff + a) * n] = q.aff[a];
      col[(int64_t)kPmass * n] = q.mass;
    } else {
      const float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
      BSpline b;
      bspline(X, mp.inv_dx, b);
      float pf[3] = {0.f, 0.f, 0.f};
      if (REACT) {
        float Fp[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) Fp[a] = pt.F[(int64_t)a * n + p];
        const float J = det3(Fp);
        ReactParticle r;
        reaction_particle(L, hydro, phi, cp, b, J, pt.vol0[p], s_scale, r);
        n_act = r.act ? 1 : 0;
        pmax = r.pnorm;
        if (r.gated)
          for (int a = 0; a < 3; ++a) pn[a] = (double)r.pf[a];
        if (r.scatter)
          for (int a = 0; a < 3; ++a) pf[a] = r.pf[a];
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        col[(int64_t)(kPfx + a) * n] = b.fx[a];
        col[(int64_t)(kPbase + a) * n] = __int_as_float(b.base[a]);
        col[(int64_t)(kPpf + a) * n] = pf[a];
#pragma unroll
        for (int o = 0; o < 3; ++o) col[(int64_t)(kPw + 3 * a + o) * n] = b.w[a][o];
      }
    }
  }
  if (REACT) {
    // diagnostics reductions (penalty.py:202-240, moving_boundary.py:312-374)
    const int na = __reduce_add_sync(0xffffffffu, (unsigned)n_act);
    const float pm = warp_max(pmax);
    double sp3[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) sp3[a] = warp_sum_d(pn[a]);
    if ((threadIdx.x & 31) == 0) {
      if (na) atomicAdd(&st->active_reaction_particle_count, na);
      if (pm > 0.f) atomic_max_nonneg(&st->max_particle_reaction_norm, pm);
      for (int a = 0; a < 3; ++a)
        if (sp3[a] != 0.0) atomicAdd(&st->net_particle_reaction[a], sp3[a]);
    }
  }
}

template <bool REACT>
__global__ __launch_bounds__(128) void k_p2g_payload(FsiParticles pt, FsiMpmParams mp,
                                                     const int32_t* __restrict__ perm, float* __restrict__ payload,
                                                     LatView L, const float* __restrict__ hydro,
                                                     const float* __restrict__ phi, FsiCouplingParams cp,
                                                     FsiCouplingStats* st, const FsiLbmDiag* diag) {
  griddep_wait();
  griddep_launch();
  p2g_payload_body<REACT>(pt, mp, perm, payload, L, hydro, phi, cp, st, diag, blockIdx.x, gridDim.x);
}

// P2G scatter of the chunks of this CTA into grid buffer g, from the payload:
//  stage the chunk's payload columns and find its node box;
//  each warp scatters one particle at a time, lane o on stencil node o, so
//  that the lanes of one shared-memory atomic touch distinct nodes (float
//  atomics to one shared address serialise);
//  one global atomic per touched node value.
// Chunks whose box exceeds the tile (bins gone stale) scatter with global
// atomics directly.
template <bool REACT, int T>
__device__ __forceinline__ void p2g_scatter_body(const FsiGrid& g, const FsiMpmParams& mp,
                                                 const float* __restrict__ payload, int n,
                                                 const int2* __restrict__ chunks, int32_t* meta, int32_t* box, int buf,
                                                 FsiCouplingStats* st, int vb, int vg) {
  __shared__ float tile[7 * kTileCap];
  __shared__ float sp[kPn][kChunk];
  __shared__ int s_lo[3], s_hi[3];
  const int tid = threadIdx.x;
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const int nch = meta[0];
  if (vb == 0 && tid == 0) meta[1 + buf] = nch;
  float* const dst[7] = {g.v, g.v + N, g.v + 2 * N, g.m, g.f_ext, g.f_ext + N, g.f_ext + 2 * N};
  float gmax = 0.f;
  double gn[3] = {0.0, 0.0, 0.0};
  for (int c = vb; c < nch; c += vg) {
    __syncthreads();  // the previous chunk's flush has read the tile and sp
    if (tid < 3) {
      s_lo[tid] = INT_MAX;
      s_hi[tid] = INT_MIN;
    }
    const int2 ch = chunks[c];
    for (int i = tid; i < kPn * ch.y; i += T) {
      const int r = i / ch.y, k = i - r * ch.y;
      sp[r][k] = payload[(int64_t)r * n + ch.x + k];
    }
    __syncthreads();
    if (tid < 32 * ((ch.y + 31) / 32)) {
      const bool live = tid < ch.y;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int bs = live ? __float_as_int(sp[kPbase + a][tid]) : 0;
        const int lo = __reduce_min_sync(0xffffffffu, live ? bs : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, live ? bs : INT_MIN);
        if ((tid & 31) == 0) {
          atomicMin(&s_lo[a], lo);
          atomicMax(&s_hi[a], hi);
        }
      }
    }
    __syncthreads();
    int32_t rec[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      rec[a] = max(s_lo[a], 0);
      rec[3 + a] = s_hi[a] == INT_MIN ? -1 : min(min(s_hi[a], G) + 2, G - 1);
    }
    const Box bx = load_box(rec);
    const bool staged = bx.vol <= kTileCap;
    if (tid == 0) {
#pragma unroll
      for (int a = 0; a < 6; ++a) box[6 * c + a] = rec[a];
      if (!staged) atomicAdd(meta + 3, 1);
    }
    const int nv = staged ? bx.vol : 0;
    for (int i = tid; i < 7 * nv; i += T) tile[i] = 0.f;
    __syncthreads();
    // one warp per particle, lane o < 27 on stencil node o (ox, oy, oz = o / 9,
    // o / 3 % 3, o % 3): the particle's payload is a broadcast read and the
    // warp's shared-memory atomics land on 27 distinct nodes
    const int lane = tid & 31, warp = tid >> 5;
    const int ox = lane / 9, oy = (lane / 3) % 3, oz = lane % 3;
    const float dox = (float)ox, doy = (float)oy, doz = (float)oz;
    float gsum[3] = {0.f, 0.f, 0.f}, gm2 = 0.f;
    for (int lp = warp; lp < ch.y; lp += T / 32) {
      if (lane >= 27) continue;
      const int I = __float_as_int(sp[kPbase][lp]) + ox, Jj = __float_as_int(sp[kPbase + 1][lp]) + oy,
                K = __float_as_int(sp[kPbase + 2][lp]) + oz;
      if (I < 0 || I >= G || Jj < 0 || Jj >= G || K < 0 || K >= G) continue;
      // weights of bspline() (staged by the payload) and offsets as in p2g_node()
      const float w = sp[kPw + ox][lp] * sp[kPw + 3 + oy][lp] * sp[kPw + 6 + oz][lp];
      const float dpos[3] = {(dox - sp[kPfx][lp]) * mp.dx, (doy - sp[kPfx + 1][lp]) * mp.dx,
                             (doz - sp[kPfx + 2][lp]) * mp.dx};
      float val[7];
#pragma unroll
      for (int q = 0; q < 3; ++q)
        val[q] = w * (sp[kPmv + q][lp] + (sp[kPaff + 3 * q][lp] * dpos[0] + sp[kPaff + 3 * q + 1][lp] * dpos[1] +
                                          sp[kPaff + 3 * q + 2][lp] * dpos[2]));
      val[3] = w * sp[kPmass][lp];
      bool react = false;
      if (REACT) {
        const float f0 = sp[kPpf][lp], f1 = sp[kPpf + 1][lp], f2 = sp[kPpf + 2][lp];
        react = f0 != 0.f || f1 != 0.f || f2 != 0.f;
        if (react) {
          val[4] = w * f0;
          val[5] = w * f1;
          val[6] = w * f2;
#pragma unroll
          for (int q = 0; q < 3; ++q) gsum[q] += val[4 + q];
          gm2 = fmaxf(gm2, val[4] * val[4] + val[5] * val[5] + val[6] * val[6]);
        }
      }
      const int nq = react ? 7 : 4;
      if (staged) {
        const int li = ((K - bx.lo[2]) * bx.ext[1] + (Jj - bx.lo[1])) * bx.ext[0] + (I - bx.lo[0]);
#pragma unroll
        for (int q = 0; q < 7; ++q)
          if (q < nq) atomicAdd(&tile[q * nv + li], val[q]);
      } else {
        const int64_t node = ((int64_t)K * G + Jj) * G + I;
#pragma unroll
        for (int q = 0; q < 7; ++q)
          if (q < nq) atomicAdd(dst[q] + node, val[q]);
      }
    }
    if (REACT) {
#pragma unroll
      for (int q = 0; q < 3; ++q) gn[q] += (double)gsum[q];
      gmax = fmaxf(gmax, sqrtf(gm2));
    }
    __syncthreads();
    for (int li = tid; li < nv; li += T) {
      const int64_t node = box_node(bx, li, G);
#pragma unroll
      for (int q = 0; q < 7; ++q) {
        const float v = tile[q * nv + li];
        if (v != 0.f) atomicAdd(dst[q] + node, v);
      }
    }
  }
  if (REACT) {
    const float gm = warp_max(gmax);
    double sg[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) sg[a] = warp_sum_d(gn[a]);
    if ((tid & 31) == 0) {
      if (gm > 0.f) atomic_max_nonneg(&st->max_grid_reaction_norm, gm);
      for (int a = 0; a < 3; ++a)
        if (sg[a] != 0.0) atomicAdd(&st->net_grid_reaction[a], sg[a]);
    }
  }
}

// register budget: 128-thread CTAs keep 4 per SM, 384-thread CTAs 1
template <bool REACT, int T>
__global__ __launch_bounds__(T, T == 384 ? 1 : 4) void k_p2g_scatter(FsiGrid g, FsiMpmParams mp, const float* __restrict__ payload,
                                                   int n, const int2* __restrict__ chunks, int32_t* meta,
                                                   int32_t* box, int buf, FsiCouplingStats* st) {
  griddep_wait();
  griddep_launch();
  p2g_scatter_body<REACT, T>(g, mp, payload, n, chunks, meta, box, buf, st, blockIdx.x, gridDim.x);
}

// G2P of the chunks of this CTA from grid buffer g; zeroes the boxes the
// previous substep recorded in the other buffer go.  T threads per CTA: each
// particle's 27 nodes are split over T / kChunk adjacent lanes (offsets o =
// sub, sub + T/kChunk, ...), whose partial sums are combined with shuffles
// before the first of them finishes the particle.
template <int T>
__device__ __forceinline__ void g2p_binned_body(const FsiParticles& pt, const FsiGrid& g, const FsiGrid& go,
                                                const FsiMpmParams& mp, const int32_t* __restrict__ perm,
                                                const int2* __restrict__ chunks, const int32_t* meta,
                                                const int32_t* __restrict__ box_b, const int32_t* __restrict__ box_o,
                                                int buf, FsiCouplingStats* st_other, int vb, int vg) {
  constexpr int GP = T / kChunk;  // lanes per particle: 1, 2 or 4
  static_assert(GP == 1 || GP == 2 || GP == 4, "T must be 128, 256 or 512");
  __shared__ float vt[3 * kTileCap];
  const int tid = threadIdx.x;
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const int nrec = meta[1 + (1 - buf)];
  for (int r = vb; r < nrec; r += vg) {
    const Box bx = load_box(box_o + 6 * r);
    for (int li = tid; li < bx.vol; li += T) {
      const int64_t node = box_node(bx, li, G);
      go.v[node] = 0.f;
      go.v[N + node] = 0.f;
      go.v[2 * N + node] = 0.f;
      go.m[node] = 0.f;
      go.f_ext[node] = 0.f;
      go.f_ext[N + node] = 0.f;
      go.f_ext[2 * N + node] = 0.f;
    }
  }
  if (st_other && vb == 0 && tid == 0) {
    st_other->active_reaction_particle_count = 0;
    st_other->max_particle_reaction_norm = 0.f;
    st_other->max_grid_reaction_norm = 0.f;
    st_other->area_scale = 0.f;
    st_other->raw_area_scale = 0.f;
    for (int a = 0; a < 3; ++a) {
      st_other->net_particle_reaction[a] = 0.0;
      st_other->net_grid_reaction[a] = 0.0;
    }
  }
  const int nch = meta[0];
  const float s4 = 4.0f * mp.inv_dx * mp.inv_dx;
  const int lp = tid / GP, sub = tid % GP;
  for (int c = vb; c < nch; c += vg) {
    __syncthreads();  // the previous chunk's gathers are done
    const Box bx = load_box(box_b + 6 * c);
    const bool staged = bx.vol <= kTileCap;
    const int nv = staged ? bx.vol : 0;
    for (int li = tid; li < nv; li += T) {
      const int64_t node = box_node(bx, li, G);
      const float m = g.m[node];
      const float P[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
      float v[3] = {P[0], P[1], P[2]};
      if (m > 0.0f) {
        const float f[3] = {g.f_ext[node], g.f_ext[N + node], g.f_ext[2 * N + node]};
        const int i = (int)(node % G), j = (int)((node / G) % G), k = (int)(node / ((int64_t)G * G));
        grid_node_velocity(P, m, f, i, j, k, G, mp, v);
      }
      vt[li] = v[0];
      vt[nv + li] = v[1];
      vt[2 * nv + li] = v[2];
    }
    __syncthreads();
    const int2 ch = chunks[c];
    // all GP lanes of a particle take the same branch (lp < ch.y is uniform
    // over them), so the shuffles below see all their partners
    if (lp < ch.y) {
      const int p = perm[ch.x + lp];
      const int n = pt.n;
      float X[3] = {pt.x[p], pt.x[n + p], pt.x[2 * n + p]};
      BSpline b;
      bspline(X, mp.inv_dx, b);
      float nvl[3] = {0.f, 0.f, 0.f}, nC[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (!staged) {
        if (sub == 0) g2p_gather_global(g, mp, b, nvl, nC);
      } else {
#pragma unroll
        for (int o0 = 0; o0 < 27; o0 += GP) {
          const int o = o0 + sub;
          if (o < 27) {
            const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
            const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
            if (I >= 0 && I < G && Jj >= 0 && Jj < G && K >= 0 && K < G) {
              const int li = ((K - bx.lo[2]) * bx.ext[1] + (Jj - bx.lo[1])) * bx.ext[0] + (I - bx.lo[0]);
              const float gv[3] = {vt[li], vt[nv + li], vt[2 * nv + li]};
              if (GP == 1) {
                g2p_node(b, ox, oy, oz, mp.dx, s4, gv, nvl, nC);
              } else {
                // the offsets of this lane are not compile-time constants: weights by
                // value instead of indexing b.w (g2p_node's arithmetic otherwise)
                const float dpos[3] = {((float)ox - b.fx[0]) * mp.dx, ((float)oy - b.fx[1]) * mp.dx,
                                       ((float)oz - b.fx[2]) * mp.dx};
                const float w = bspline_w(b.fx[0], ox) * bspline_w(b.fx[1], oy) * bspline_w(b.fx[2], oz);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                  nvl[a] += w * gv[a];
#pragma unroll
                  for (int cc = 0; cc < 3; ++cc) nC[a * 3 + cc] += (w * gv[a]) * dpos[cc] * s4;
                }
              }
            }
          }
        }
      }
      if (GP > 1) {
        // partners of a particle are adjacent lanes, aligned to GP
        const unsigned grp = ((1u << GP) - 1u) << ((tid & 31) & ~(GP - 1));
#pragma unroll
        for (int w = 1; w < GP; w <<= 1) {
#pragma unroll
          for (int a = 0; a < 3; ++a) nvl[a] += __shfl_xor_sync(grp, nvl[a], w, GP);
#pragma unroll
          for (int a = 0; a < 9; ++a) nC[a] += __shfl_xor_sync(grp, nC[a], w, GP);
        }
      }
      if (sub == 0) g2p_finish(pt, p, mp, X, nvl, nC);
    }
  }
}

template <int T>
__global__ __launch_bounds__(T) void k_g2p_binned(FsiParticles pt, FsiGrid g, FsiGrid go, FsiMpmParams mp,
                                                  const int32_t* __restrict__ perm,
                                                  const int2* __restrict__ chunks, const int32_t* meta,
                                                  const int32_t* __restrict__ box_b,
                                                  const int32_t* __restrict__ box_o, int buf,
                                                  FsiCouplingStats* st_other) {
  griddep_wait();
  griddep_launch();
  g2p_binned_body<T>(pt, g, go, mp, perm, chunks, meta, box_b, box_o, buf, st_other, blockIdx.x, gridDim.x);
}

__global__ void k_grid_velocity(FsiGrid g, FsiMpmParams mp, float* __restrict__ out) {
  const int G = g.n;
  const int64_t N = (int64_t)G * G * G;
  const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N) return;
  const float m = g.m[node];
  const float P[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
  float v[3] = {P[0], P[1], P[2]};
  if (m > 0.0f) {
    const float f[3] = {g.f_ext[node], g.f_ext[N + node], g.f_ext[2 * N + node]};
    grid_node_velocity(P, m, f, (int)(node % G), (int)((node / G) % G), (int)(node / ((int64_t)G * G)), G, mp, v);
  }
  out[node] = v[0];
  out[N + node] = v[1];
  out[2 * N + node] = v[2];
}

int layout(int32_t n_particles, int32_t n_grid, int32_t* n_bins, int32_t* max_chunks) {
  if (n_particles <= 0 || n_grid <= 0) return invalid("n_particles and n_grid must be positive");
  const int64_t nb = (n_grid + kEdge - 1) / kEdge;
  const int64_t bins = nb * nb * nb;
  const int64_t mc = ((int64_t)n_particles + kChunk - 1) / kChunk + std::min<int64_t>(n_particles, bins);
  if (bins > INT_MAX || mc > INT_MAX / 12) return invalid("grid or particle count too large for binning");
  *n_bins = (int32_t)bins;
  *max_chunks = (int32_t)mc;
  return FSI_OK;
}

int check_bins(const FsiMpmBins* bins, int32_t n_particles, int32_t n_grid) {
  if (!bins) return invalid("null bins");
  if (!bins->key || !bins->count || !bins->start || !bins->perm || !bins->chunk || !bins->box || !bins->meta ||
      !bins->payload)
    return invalid("null bins array");
  int32_t nb = 0, mc = 0;
  const int rc = layout(n_particles, n_grid, &nb, &mc);
  if (rc) return rc;
  if (bins->n_bins != nb) return invalid("bins->n_bins does not match the grid (see fsi_mpm_bins_layout)");
  if (bins->max_chunks < mc) return invalid("bins->max_chunks below fsi_mpm_bins_layout's capacity");
  if (((uintptr_t)bins->count | (uintptr_t)bins->start | (uintptr_t)bins->chunk) & 15)
    return invalid("bins->count, start and chunk must be 16-byte aligned");
  return FSI_OK;
}

int check_particles(const FsiParticles* pt) {
  if (!pt) return invalid("null particles");
  if (pt->n <= 0) return invalid("n_particles must be positive");
  if (!pt->x || !pt->v || !pt->C || !pt->F || !pt->Jp || !pt->mass || !pt->vol0 || !pt->fixed || !pt->fixed_x)
    return invalid("null particle field");
  return FSI_OK;
}

int check_grid(const FsiGrid* g) {
  if (!g || g->n <= 0 || !g->v || !g->m || !g->f_ext) return invalid("bad grid");
  return FSI_OK;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace
}  // namespace fsi

using namespace fsi;

extern "C" int fsi_mpm_bins_layout(int32_t n_particles, int32_t n_grid, int32_t* n_bins, int32_t* max_chunks) {
  if (!n_bins || !max_chunks) return invalid("null output");
  return layout(n_particles, n_grid, n_bins, max_chunks);
}

extern "C" int fsi_mpm_bin(const FsiParticles* pt, const FsiGrid* g, const FsiMpmParams* mp, const FsiMpmBins* bins,
                           void* stream) {
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!g || g->n <= 0 || !mp) return invalid("bad grid or params");
  if ((rc = check_bins(bins, pt->n, g->n))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (g->n + kEdge - 1) / kEdge;
  k_bin_count<<<nblk(pt->n, 256), 256, 0, st>>>(*pt, mp->inv_dx, g->n, nb, bins->key, bins->count);
  if ((rc = launch_check("k_bin_count"))) return rc;
  k_bin_scan<<<1, 1024, 0, st>>>(bins->n_bins, bins->count, bins->start, reinterpret_cast<int2*>(bins->chunk),
                                 bins->meta);
  if ((rc = launch_check("k_bin_scan"))) return rc;
  k_bin_scatter<<<nblk(pt->n, 256), 256, 0, st>>>(pt->n, bins->key, bins->start, bins->perm);
  return launch_check("k_bin_scatter");
}

extern "C" int fsi_mpm_substep_binned(const FsiParticles* pt, const FsiGrid grid[2], const FsiMpmBins* bins,
                                      const FsiMpmParams* mp, int32_t buffer, const FsiLbmState* s,
                                      const float* hydro, const FsiCouplingParams* cp, FsiCouplingStats stats[2],
                                      void* stream) {
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!grid || !mp) return invalid("null grid or params");
  if ((rc = check_grid(&grid[0])) || (rc = check_grid(&grid[1]))) return rc;
  if (grid[0].n != grid[1].n) return invalid("the two grid buffers differ in size");
  if (buffer != 0 && buffer != 1) return invalid("buffer must be 0 or 1");
  if (mp->tune < 0 || mp->tune > 15 || (mp->tune & 3) > 1 || ((mp->tune >> 2) & 3) == 3)
    return invalid("unknown FsiMpmParams.tune");
  if ((rc = check_bins(bins, pt->n, grid[0].n))) return rc;
  if (cp) {
    if (!s || !hydro || !stats) return invalid("reaction transfer needs the lattice state, hydro and stats");
    if (cp->kind < 0 || cp->kind > 2) return invalid("reaction kind must be 0 (penalty), 1 (engineering), 2 (link-area)");
    if (cp->kind != 0 && !s->phi) return invalid("moving-boundary reaction needs phi");
    if (cp->kind == 2 && !s->diag) return invalid("link-area reaction needs the directional reductions");
    if (cp->inv_dx_norm != mp->inv_dx)
      return invalid("binned substep needs the coupling and MPM grids to share dx (inv_dx_norm == inv_dx)");
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int grid_ctas = (int)std::min<int64_t>(bins->max_chunks, (int64_t)sm_count() * 4);
  int32_t* box_b = bins->box + (int64_t)6 * bins->max_chunks * buffer;
  int32_t* box_o = bins->box + (int64_t)6 * bins->max_chunks * (1 - buffer);
  const int2* chunks = reinterpret_cast<const int2*>(bins->chunk);
  const FsiGrid g = grid[buffer], go = grid[1 - buffer];
  const int tsc = mp->tune & 3, tg = (mp->tune >> 2) & 3;
  const int T = tsc == FSI_TUNE_P2G_T384 ? 384 : 128;
  const int TG = tg == FSI_TUNE_MPM_T512 ? 512 : (tg == FSI_TUNE_MPM_T256 ? 256 : 128);
  const LatView L = cp ? LatView{s->nx, s->ny, s->nz, s->pitch} : LatView{0, 0, 0, 0};
  const float* hy = cp ? hydro : nullptr;
  const float* ph = cp ? s->phi : nullptr;
  const FsiCouplingParams cpv = cp ? *cp : FsiCouplingParams{};
  FsiCouplingStats* stb = cp ? &stats[buffer] : nullptr;
  const FsiLbmDiag* dg = cp ? s->diag : nullptr;
  // the three kernels of a substep, and the substeps, follow each other with
  // programmatic dependent launch (each waits for its predecessor's writes)
  const unsigned gp = nblk(2 * (int64_t)pt->n, 128);
  cudaError_t lerr;
  if (cp)
    lerr = launch_pdl(k_p2g_payload<true>, dim3(gp), dim3(128), 0, st, *pt, *mp, (const int32_t*)bins->perm,
                      bins->payload, L, hy, ph, cpv, stb, dg);
  else
    lerr = launch_pdl(k_p2g_payload<false>, dim3(gp), dim3(128), 0, st, *pt, *mp, (const int32_t*)bins->perm,
                      bins->payload, L, hy, ph, cpv, stb, dg);
  if ((rc = cuda_check(lerr, "k_p2g_payload (launch)")) || (rc = launch_check("k_p2g_payload"))) return rc;
#define FSI_P2G(R, TT)                                                                                        \
  lerr = launch_pdl(k_p2g_scatter<R, TT>, dim3(grid_ctas), dim3(TT), 0, st, g, *mp,                         \
                    (const float*)bins->payload, pt->n, chunks, bins->meta, box_b, buffer, stb)
  if (cp) {
    if (T == 384) FSI_P2G(true, 384); else FSI_P2G(true, 128);
  } else {
    if (T == 384) FSI_P2G(false, 384); else FSI_P2G(false, 128);
  }
#undef FSI_P2G
  if ((rc = cuda_check(lerr, "k_p2g_scatter (launch)")) || (rc = launch_check("k_p2g_scatter"))) return rc;
  FsiCouplingStats* sto = cp ? &stats[1 - buffer] : nullptr;
#define FSI_G2P(TT)                                                                                       \
  lerr = launch_pdl(k_g2p_binned<TT>, dim3(grid_ctas), dim3(TT), 0, st, *pt, g, go, *mp,                   \
                    (const int32_t*)bins->perm, chunks, (const int32_t*)bins->meta, (const int32_t*)box_b, \
                    (const int32_t*)box_o, buffer, sto)
  if (TG == 512) FSI_G2P(512); else if (TG == 256) FSI_G2P(256); else FSI_G2P(128);
#undef FSI_G2P
  if ((rc = cuda_check(lerr, "k_g2p_binned (launch)"))) return rc;
  return launch_check("k_g2p_binned");
}

extern "C" int fsi_mpm_grid_velocity(const FsiGrid* g, const FsiMpmParams* mp, float* out, void* stream) {
  int rc = check_grid(g);
  if (rc) return rc;
  if (!mp || !out) return invalid("null params or output");
  const int64_t N = (int64_t)g->n * g->n * g->n;
  k_grid_velocity<<<nblk(N, 256), 256, 0, (cudaStream_t)stream>>>(*g, *mp, out);
  return launch_check("k_grid_velocity");
}

// ---- batched cases: MPM (grid.y = case slot) --------------------------------
namespace fsi {
namespace {

// the force field the reaction transfer samples: the last LBM step's link
// forces (moving boundary, one LBM step per FSI step: the ping-pong slot the
// step wrote, now pp ^ 1) or the penalty hydro force
__device__ __forceinline__ const float* batch_hydro(const FsiBatchCase& bc) {
  if (bc.mode == FSI_BATCH_MOVING) return bc.lbm.hpp + (int64_t)(bc.ctl.pp ^ 1) * 3 * bc.lbm.pitch;
  return bc.lbm.hydro;
}

__global__ void k_batch_bin_count(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const int G = bc.grid[0].n, nb = (G + kEdge - 1) / kEdge;
  const int nvb = (bc.pt.n + blockDim.x - 1) / blockDim.x;
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
    bin_count_body(bc.pt, bc.mp.inv_dx, G, nb, bc.bins.key, bc.bins.count, vb, nvb);
}

__global__ __launch_bounds__(1024) void k_batch_bin_scan(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  bin_scan_body(bc.bins.n_bins, bc.bins.count, bc.bins.start, reinterpret_cast<int2*>(bc.bins.chunk), bc.bins.meta);
}

__global__ void k_batch_bin_scatter(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const int nvb = (bc.pt.n + blockDim.x - 1) / blockDim.x;
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
    bin_scatter_body(bc.pt.n, bc.bins.key, bc.bins.start, bc.bins.perm, vb, nvb);
}

__global__ __launch_bounds__(128) void k_batch_p2g_payload(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const LatView L{bc.lbm.nx, bc.lbm.ny, bc.lbm.nz, bc.lbm.pitch};
  const int nvb = (2 * bc.pt.n + blockDim.x - 1) / blockDim.x;  // two lanes per particle
  const float* hydro = batch_hydro(bc);
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
    p2g_payload_body<true>(bc.pt, bc.mp, bc.bins.perm, bc.bins.payload, L, hydro, bc.lbm.phi, bc.cp,
                           &bc.react_stats[bc.buf], bc.lbm.diag, vb, nvb);
}

template <int T>
__global__ __launch_bounds__(T, T == 384 ? 1 : 4) void k_batch_p2g_scatter(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const int b = bc.buf;
  int32_t* box_b = bc.bins.box + (int64_t)6 * bc.bins.max_chunks * b;
  p2g_scatter_body<true, T>(bc.grid[b], bc.mp, bc.bins.payload, bc.pt.n, reinterpret_cast<const int2*>(bc.bins.chunk),
                            bc.bins.meta, box_b, b, &bc.react_stats[b], blockIdx.x, gridDim.x);
}

template <int T>
__global__ __launch_bounds__(T) void k_batch_g2p(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  const int b = bc.buf;
  const int32_t* box_b = bc.bins.box + (int64_t)6 * bc.bins.max_chunks * b;
  const int32_t* box_o = bc.bins.box + (int64_t)6 * bc.bins.max_chunks * (1 - b);
  g2p_binned_body<T>(bc.pt, bc.grid[b], bc.grid[1 - b], bc.mp, bc.bins.perm,
                     reinterpret_cast<const int2*>(bc.bins.chunk), bc.bins.meta, box_b, box_o, b,
                     &bc.react_stats[1 - b], blockIdx.x, gridDim.x);
}

__global__ void k_batch_mpm_post(FsiBatchCase* cases) {
  FsiBatchCase& bc = cases[blockIdx.x];
  if (bc.active && threadIdx.x == 0) bc.buf ^= 1;
}

int check_batch_mpm(const FsiBatchCase* cases, const FsiBatchDims* d) {
  if (!cases || !d) return invalid("null batch argument");
  if (d->n_cases <= 0 || d->n_cases > 65535) return invalid("n_cases must be in 1..65535");
  if (d->max_particles <= 0 || d->max_chunks <= 0 || d->max_bins <= 0) return invalid("batch MPM dims must be positive");
  if (d->mpm_tune < 0 || d->mpm_tune > 15 || (d->mpm_tune & 3) > 1 || ((d->mpm_tune >> 2) & 3) == 3)
    return invalid("unknown FsiBatchDims.mpm_tune");
  return FSI_OK;
}

}  // namespace
}  // namespace fsi

extern "C" int fsi_batch_mpm_bin(FsiBatchCase* cases, const FsiBatchDims* d, void* stream) {
  int rc = check_batch_mpm(cases, d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 g(nblk(d->max_particles, 256), d->n_cases);
  k_batch_bin_count<<<g, 256, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_bin_count"))) return rc;
  k_batch_bin_scan<<<dim3(1, d->n_cases), 1024, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_bin_scan"))) return rc;
  k_batch_bin_scatter<<<g, 256, 0, st>>>(cases);
  return launch_check("k_batch_bin_scatter");
}

extern "C" int fsi_batch_mpm_substep(FsiBatchCase* cases, const FsiBatchDims* d, void* stream) {
  int rc = check_batch_mpm(cases, d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 gp(nblk(2 * (int64_t)d->max_particles, 128), d->n_cases);
  k_batch_p2g_payload<<<gp, 128, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_p2g_payload"))) return rc;
  // about one CTA per chunk of the largest case (a bin's chunks hold <= 128 particles each; bins
  // partly filled add chunks): CTAs stride over the case's chunk table
  const dim3 gc((unsigned)std::min<int64_t>(d->max_chunks, 2 * nblk(d->max_particles, kChunk) + 8), d->n_cases);
  const int tsc = d->mpm_tune & 3, tg = (d->mpm_tune >> 2) & 3;
  if (tsc == FSI_TUNE_P2G_T384)
    k_batch_p2g_scatter<384><<<gc, 384, 0, st>>>(cases);
  else
    k_batch_p2g_scatter<128><<<gc, 128, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_p2g_scatter"))) return rc;
  if (tg == FSI_TUNE_MPM_T512)
    k_batch_g2p<512><<<gc, 512, 0, st>>>(cases);
  else if (tg == FSI_TUNE_MPM_T256)
    k_batch_g2p<256><<<gc, 256, 0, st>>>(cases);
  else
    k_batch_g2p<128><<<gc, 128, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_g2p"))) return rc;
  k_batch_mpm_post<<<d->n_cases, 32, 0, st>>>(cases);
  return launch_check("k_batch_mpm_post");
}

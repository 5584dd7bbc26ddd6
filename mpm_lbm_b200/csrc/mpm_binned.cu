// Binned MPM substeps: particles sorted by 4x4x4-cell block and cut into
// chunks; one launch per substep, in which each CTA takes whole chunks
// through the G2P gather of the previous substep (grid update evaluated while
// the chunk's node box is staged), the P2G stress / reaction payload and the
// P2G scatter staged in a shared-memory tile, flushed with one global atomic
// per touched node value.  Three grid buffers rotate so that only the boxes
// touched two substeps earlier are zeroed, by the launch after their last
// reader.
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
// nodes staged per CTA: the stencils of a chunk of one bin span at most
// (8 + 2)^3 = 1000 nodes; the rest absorbs a node of drift since the last
// binning (an 11^3 box).  Two regions of shared memory: the scatter tile (7
// floats per node, 37 KB) and the stage of the gather's node velocities and of
// the reaction's lattice box (4 floats per node), so that the tile can be
// zeroed while the payload is built.
constexpr int kTileCap = 1331;

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
//
// Chunks: a bin of c particles is cut into ceil(c / kChunk) chunks of equal
// size (sizes differ by at most one), so that no chunk of a few particles
// follows a full one.
__device__ __forceinline__ int4 ld_bins4(const int32_t* p, int b, int b1) {
  if (b + 4 <= b1) return *reinterpret_cast<const int4*>(p + b);
  int4 v = make_int4(0, 0, 0, 0);
  if (b < b1) v.x = p[b];
  if (b + 1 < b1) v.y = p[b + 1];
  if (b + 2 < b1) v.z = p[b + 2];
  return v;
}

__device__ __forceinline__ int chunks_of(int c) { return (c + kChunk - 1) / kChunk; }

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
    cs += chunks_of(c.x) + chunks_of(c.y) + chunks_of(c.z) + chunks_of(c.w);
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
      const int nc = chunks_of(cv[q]);
      if (nc > 0) {
        const int sz = cv[q] / nc, rem = cv[q] - sz * nc;  // rem chunks of sz + 1, then sz
        int off = po;
        for (int i = 0; i < nc; ++i) {
          const int n = sz + (i < rem ? 1 : 0);
          chunk[co++] = make_int2(off, n);
          off += n;
        }
      }
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

// Orders the particles of each bin by B-spline base node (counting sort over
// the bin's kEdge^3 base cells; order within a cell unspecified), so that the
// chunks cut from a bin are compact slabs and particles sharing a stencil are
// adjacent.  One CTA per bin (grid-stride); the bin's range of perm is sorted
// through the same range of `tmp`.  After fsi_mpm_bin's scatter, end[b] is the
// end offset of bin b in perm (its start is end[b - 1]).
constexpr int kBinCells = kEdge * kEdge * kEdge;
constexpr int kSortT = 256;

__device__ __forceinline__ int local_base_cell(const FsiParticles& pt, int p, float inv_dx, int G) {
  int l = 0;
  for (int a = 2; a >= 0; --a) {
    const float Xp = __fmul_rn(pt.x[a * pt.n + p], inv_dx);
    l = l * kEdge + clampi((int)(Xp - 0.5f), 0, G - 1) % kEdge;
  }
  return l;
}

__device__ __forceinline__ void bin_sort_body(const FsiParticles& pt, float inv_dx, int G, int nbins,
                                              const int32_t* __restrict__ end, int32_t* __restrict__ perm,
                                              int32_t* __restrict__ tmp, int vb, int vg) {
  __shared__ int cnt[kBinCells];
  __shared__ int wsum[kSortT / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  constexpr int PER = kBinCells / kSortT;  // counters per thread
  static_assert(kBinCells % kSortT == 0, "bin cells must be a multiple of the sort CTA");
  for (int b = vb; b < nbins; b += vg) {
    const int lo = b ? end[b - 1] : 0, hi = end[b];
    if (hi - lo < 2) continue;  // uniform over the CTA
    for (int i = t; i < kBinCells; i += kSortT) cnt[i] = 0;
    __syncthreads();
    for (int i = lo + t; i < hi; i += kSortT) atomicAdd(&cnt[local_base_cell(pt, perm[i], inv_dx, G)], 1);
    __syncthreads();
    // exclusive scan of the counters: PER per thread, then warps, then CTA
    int v[PER], sum = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      v[q] = cnt[t * PER + q];
      sum += v[q];
    }
    int inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[wid] = inc;
    __syncthreads();
    int off = inc - sum;
    for (int w = 0; w < wid; ++w) off += wsum[w];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      cnt[t * PER + q] = off;  // becomes the cell's cursor
      off += v[q];
    }
    __syncthreads();
    for (int i = lo + t; i < hi; i += kSortT) {
      const int p = perm[i];
      tmp[lo + atomicAdd(&cnt[local_base_cell(pt, p, inv_dx, G)], 1)] = p;
    }
    __syncthreads();
    for (int i = lo + t; i < hi; i += kSortT) perm[i] = tmp[i];
    __syncthreads();
  }
}

__global__ __launch_bounds__(kSortT) void k_bin_sort(FsiParticles pt, float inv_dx, int G, int nbins,
                                                      const int32_t* __restrict__ end, int32_t* __restrict__ perm,
                                                      int32_t* __restrict__ tmp) {
  bin_sort_body(pt, inv_dx, G, nbins, end, perm, tmp, blockIdx.x, gridDim.x);
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

// P2G payload of a particle (shared memory), one record of kQn floats per
// particle of the chunk, in float4 groups so that the scatter reads the
// values every lane needs as 128-bit broadcasts:
//   [0]  mv0 mv1 mv2 mass      [4]  aff0..3      [8]  aff4..7     [12] aff8
//   [16] base0 base1 base2 fx0 [20] fx1 fx2 pf0 pf1
//   [24] w[0][0..2] pf2        [28] w[1][0..2]   [32] w[2][0..2]
// (base as int bits; w the B-spline weights [axis][offset]).  A record of 36
// floats keeps the 128-bit stores of 8 consecutive particles on distinct banks.
enum { kQmv = 0, kQaff = 4, kQbase = 16, kQfx1 = 20, kQwx = 24, kQwy = 28, kQwz = 32, kQn = 36 };

// ---- fused substep sequence --------------------------------------------------
// M substeps in M + 1 launches (after a prologue).  Launch s, for each chunk of
// its CTA: the gather of substep s - 1 (G2P from grid buffer (s - 1) % 3, the
// new particle state written to the particle fields and kept in shared
// memory), then the P2G payload of substep s from that state and its scatter
// into buffer s % 3.  A chunk's particles belong to one CTA for the launch, so
// gather, payload and scatter of a chunk follow each other without any
// grid-wide synchronisation; the launch boundary is the one grid-wide step
// (every scatter of substep s is complete before any gather of it).  The
// launch also zeroes the boxes substep s - 2 recorded in buffer (s + 1) % 3,
// whose last reader (the gather of substep s - 2) ran in the launch before:
// three buffers, so that no launch zeroes a buffer that another CTA of the
// same launch still reads or writes.  The arithmetic is the one of the
// three-kernel substep above (p2g_particle, reaction_particle, g2p_node and
// g2p_finish on the same values).

enum { kSx = 0, kSv = 3, kSC = 6, kSF = 15, kSn = 24 };  // staged particle state rows
// bins->meta: [0] chunks, [1 + b] records in box[b], [4] chunks scattered
// without the tile, [5 + b] buffer b holds recorded boxes not yet zeroed
enum { kMetaChunks = 0, kMetaRec = 1, kMetaOverflow = 4, kMetaDirty = 5 };
constexpr int kSeqT = 256;
constexpr int kTileFloats = (7 * kTileCap + 3) & ~3;  // keeps the next region 16-byte aligned
// G2P: the staged node velocities use 3 * nv <= 3 * kTileCap floats of the
// stage; the two stencil halves of a particle meet behind them (12 sums per
// particle).  The reaction's lattice box uses 4 * nv.
constexpr int kXchOffset = (3 * kTileCap + 3) & ~3;
constexpr int kStageFloats = ((kXchOffset + 12 * kChunk > 4 * kTileCap ? kXchOffset + 12 * kChunk : 4 * kTileCap) + 3) & ~3;
constexpr size_t kSeqSmem = sizeof(float) * (kTileFloats + kStageFloats + (kQn + kSn) * kChunk);

struct SeqArgs {
  FsiParticles pt;
  FsiGrid grid[3];
  FsiMpmParams mp;
  const int32_t* perm;
  const int2* chunks;
  int32_t* meta;
  int32_t* box;        // [3][max_chunks][6]
  int64_t box_stride;  // 6 * max_chunks
  LatView L;
  const float* hydro;
  const float* phi;
  FsiCouplingParams cp;
  FsiCouplingStats* stats;  // [3]; null without the reaction transfer
  const FsiLbmDiag* diag;
  int32_t s, M;             // launch index (0..M) and substeps in the sequence
};

// lattice coordinates of entry li of a box (two divisions)
__device__ __forceinline__ void box_ijk(const Box& b, int li, int& i, int& j, int& k) {
  const int e0 = b.ext[0], e01 = b.ext[0] * b.ext[1];
  k = li / e01;
  const int r = li - k * e01;
  j = r / e0;
  i = r - j * e0 + b.lo[0];
  j += b.lo[1];
  k += b.lo[2];
}

__device__ __forceinline__ void zero_boxes(const FsiGrid& go, const int32_t* __restrict__ rec, int nrec, int vb,
                                           int vg) {
  const int G = go.n;
  const int64_t N = (int64_t)G * G * G;
  for (int r = vb; r < nrec; r += vg) {
    const Box bx = load_box(rec + 6 * r);
    for (int li = threadIdx.x; li < bx.vol; li += blockDim.x) {
      int i, j, k;
      box_ijk(bx, li, i, j, k);
      const int64_t node = ((int64_t)k * G + j) * G + i;
      go.v[node] = 0.f;
      go.v[N + node] = 0.f;
      go.v[2 * N + node] = 0.f;
      go.m[node] = 0.f;
      go.f_ext[node] = 0.f;
      go.f_ext[N + node] = 0.f;
      go.f_ext[2 * N + node] = 0.f;
    }
  }
}

__device__ __forceinline__ void zero_reaction_stats(FsiCouplingStats* st) {
  st->active_reaction_particle_count = 0;
  st->max_particle_reaction_norm = 0.f;
  st->max_grid_reaction_norm = 0.f;
  st->area_scale = 0.f;
  st->raw_area_scale = 0.f;
  for (int a = 0; a < 3; ++a) {
    st->net_particle_reaction[a] = 0.0;
    st->net_grid_reaction[a] = 0.0;
  }
}

// grid buffer b by value (a select, not an indexed access, so that a
// SeqArgs held in registers needs no local memory)
__device__ __forceinline__ FsiGrid grid_of(const SeqArgs& A, int b) {
  return b == 0 ? A.grid[0] : (b == 1 ? A.grid[1] : A.grid[2]);
}

// zeroes every buffer with boxes left from an earlier sequence, and the
// reaction record of the first substep
__device__ __forceinline__ void seq_prologue_body(const SeqArgs& A, int vb, int vg) {
  for (int b = 0; b < 3; ++b)
    if (A.meta[kMetaDirty + b]) zero_boxes(grid_of(A, b), A.box + b * A.box_stride, A.meta[kMetaRec + b], vb, vg);
  if (A.stats && vb == 0 && threadIdx.x == 0) zero_reaction_stats(A.stats);
}

// reaction_particle() from the chunk's lattice box staged in shared memory
// (lat[q * nv + li], q = 0..2 the force field, 3 phi; li the index in the box
// bx, which holds every stencil node of the chunk inside the grid): the same
// nodes, weights and summation order
__device__ __forceinline__ void reaction_particle_staged(const float* __restrict__ lat, const Box& bx, int nv,
                                                         const LatView& L, const FsiCouplingParams& cp,
                                                         const BSpline& b, float Jp, float vol0, float scale,
                                                         ReactParticle& r) {
  float hs[3] = {0.f, 0.f, 0.f}, ps = 0.f;
  const bool inside = b.base[0] >= 0 && b.base[1] >= 0 && b.base[2] >= 0 && b.base[0] + 2 < L.nx &&
                      b.base[1] + 2 < L.ny && b.base[2] + 2 < L.nz;
  const int l000 = ((b.base[2] - bx.lo[2]) * bx.ext[1] + (b.base[1] - bx.lo[1])) * bx.ext[0] + (b.base[0] - bx.lo[0]);
#pragma unroll
  for (int ox = 0; ox < 3; ++ox)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
      for (int oz = 0; oz < 3; ++oz) {
        const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
        if (!inside && (I < 0 || I >= L.nx || Jj < 0 || Jj >= L.ny || K < 0 || K >= L.nz)) continue;
        const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
        const int li = l000 + (oz * bx.ext[1] + oy) * bx.ext[0] + ox;
        hs[0] += w * lat[li];
        hs[1] += w * lat[nv + li];
        hs[2] += w * lat[2 * nv + li];
        if (cp.kind != 0) ps += w * lat[3 * nv + li];
      }
  reaction_from_sums(cp, hs, ps, Jp, vol0, scale, r);
}

__device__ __forceinline__ int base_of(float x, float inv_dx) { return (int)(__fmul_rn(x, inv_dx) - 0.5f); }

// the chunk's node box: min / max base node over the live threads (every
// thread of the CTA calls this, live or not)
__device__ __forceinline__ void box_reduce(bool live, const int nb[3], int* s_lo, int* s_hi) {
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int lo = __reduce_min_sync(0xffffffffu, live ? nb[r] : INT_MAX);
    const int hi = __reduce_max_sync(0xffffffffu, live ? nb[r] : INT_MIN);
    if ((threadIdx.x & 31) == 0) {
      if (lo != INT_MAX) atomicMin(&s_lo[r], lo);
      if (hi != INT_MIN) atomicMax(&s_hi[r], hi);
    }
  }
}

constexpr int kRun = kChunk / (kSeqT / 32);  // particles per warp in the scatter

// G2P gather of one particle over the stencil offsets o = SUB, SUB + 2, ...
// (the two halves of the 27 nodes, one per warp of a pair) from the node
// velocities staged in tile (box bx, nv nodes): the arithmetic of the
// one-phase g2p_node, with the offsets, weights and offset distances known
// per offset at compile time and the grid-range test skipped for particles
// whose whole stencil lies inside the grid.
template <int SUB>
__device__ __forceinline__ void g2p_gather_half(const float* tile, int nv, const Box& bx, int G, const BSpline& b,
                                                float dx, float s4, float* nvl, float* nC) {
  float dp[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int o = 0; o < 3; ++o) dp[a][o] = ((float)o - b.fx[a]) * dx;
  const int e0 = bx.ext[0], e01 = bx.ext[0] * bx.ext[1];
  const int li0 = ((b.base[2] - bx.lo[2]) * bx.ext[1] + (b.base[1] - bx.lo[1])) * bx.ext[0] + (b.base[0] - bx.lo[0]);
  const bool inside = b.base[0] >= 0 && b.base[0] + 2 < G && b.base[1] >= 0 && b.base[1] + 2 < G &&
                      b.base[2] >= 0 && b.base[2] + 2 < G;
#pragma unroll
  for (int o = SUB; o < 27; o += 2) {
    const int ox = o / 9, oy = (o / 3) % 3, oz = o % 3;
    const int I = b.base[0] + ox, Jj = b.base[1] + oy, K = b.base[2] + oz;
    if (inside || (I >= 0 && I < G && Jj >= 0 && Jj < G && K >= 0 && K < G)) {
      const int li = li0 + oz * e01 + oy * e0 + ox;
      const float gv[3] = {tile[li], tile[nv + li], tile[2 * nv + li]};
      const float dpos[3] = {dp[0][ox], dp[1][oy], dp[2][oz]};
      const float w = b.w[0][ox] * b.w[1][oy] * b.w[2][oz];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        nvl[q] += w * gv[q];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) nC[q * 3 + cc] += (w * gv[q]) * dpos[cc] * s4;
      }
    }
  }
}

// launch A.s of the sequence for the chunks vb, vb + vg, ... (kSeqT threads,
// kSeqSmem bytes of dynamic shared memory)
template <bool REACT>
__device__ __forceinline__ void mpm_seq_body(const SeqArgs& A, int vb, int vg) {
  constexpr int T = kSeqT, NW = T / 32;
  static_assert(kSeqT == 2 * kChunk, "G2P: two warps per 32 particles, one per stencil half");
  extern __shared__ float4 seq_smem4[];
  // G2P: [3][nv] node velocities; payload: [4][nv] lattice box; scatter: [7][nv] tile
  float* const tile = reinterpret_cast<float*>(seq_smem4);  // [7][nv] scatter tile
  float* const stg = tile + kTileFloats;                      // [3][nv] node velocities / [4][nv] lattice box
  float* const sp = stg + kStageFloats;  // [kChunk][kQn] P2G payload
  float* const ss = sp + kQn * kChunk;   // [kSn][kChunk] particle state
  __shared__ int s_lo[3], s_hi[3];
  __shared__ float s_scale;
  __shared__ int s_cnt[NW];
  __shared__ float s_fmax[NW][2];
  __shared__ double s_dsum[NW][6];
  const FsiParticles& pt = A.pt;
  const FsiMpmParams& mp = A.mp;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int s = A.s;
  const bool do_g2p = s > 0, do_p2g = s < A.M;
  const int bg = (s + 2) % 3, bs = s % 3, bz = (s + 1) % 3;
  const int G = A.grid[0].n;
  const int64_t N = (int64_t)G * G * G;
  const int nch = A.meta[kMetaChunks];
  FsiCouplingStats* const st = REACT ? A.stats + bs : nullptr;
  if (vb == 0 && tid == 0) {
    if (s == 0) {  // the prologue zeroed every buffer
      A.meta[kMetaDirty + 1] = 0;
      A.meta[kMetaDirty + 2] = 0;
    }
    if (s >= 2) A.meta[kMetaDirty + bz] = 0;
    if (do_p2g) {
      A.meta[kMetaRec + bs] = nch;
      A.meta[kMetaDirty + bs] = 1;
    }
    if (REACT) zero_reaction_stats(A.stats + bz);  // the record of substep s + 1
  }
  if (REACT && do_p2g && tid == 0) {
    float raw = 1.f;
    s_scale = A.cp.kind == 2 ? link_area_scale(A.diag, A.cp, &raw) : 1.0f;
    if (vb == 0 && A.cp.kind == 2) {
      st->area_scale = s_scale;
      st->raw_area_scale = raw;
    }
  }
  if (s >= 2) {
    // the boxes of substep s - 2: CTAs left without a chunk (fewer chunks than
    // CTAs) zero them, off the path of the CTAs that have one; with no idle
    // CTA every CTA takes a share
    const int nrec = A.meta[kMetaRec + bz], idle = vg - nch;
    if (idle <= 0)
      zero_boxes(grid_of(A, bz), A.box + bz * A.box_stride, nrec, vb, vg);
    else if (vb >= nch)
      zero_boxes(grid_of(A, bz), A.box + bz * A.box_stride, nrec, vb - nch, idle);
  }

  const float s4 = 4.0f * mp.inv_dx * mp.inv_dx;
  const int n = pt.n;
  int n_act = 0;
  float pmax = 0.f, gmax = 0.f;
  double pn[3] = {0.0, 0.0, 0.0}, gn[3] = {0.0, 0.0, 0.0};
  for (int c = vb; c < nch; c += vg) {
    __syncthreads();  // the previous chunk is done with the tile, the stages and the box
    if (tid < 3) {
      s_lo[tid] = INT_MAX;
      s_hi[tid] = INT_MIN;
    }
    const int2 ch = A.chunks[c];
    int nb[3] = {0, 0, 0};  // base node of this thread's particle after the gather
    bool nb_live = false;
    // particle reads of the payload, issued ahead of the gather
    const int pslot = (wid >> 1) * 32 + lane;
    int pq = 0;
    float pmass = 0.f, pvol0 = 0.f;
    if (do_p2g && pslot < ch.y) {
      pq = A.perm[ch.x + pslot];
      pmass = pt.mass[pq];
      pvol0 = pt.vol0[pq];
    }
    if (do_g2p) {
      // ---- G2P of substep s - 1 from buffer bg
      const FsiGrid g = grid_of(A, bg);
      const Box bx = load_box(A.box + bg * A.box_stride + 6 * c);
      const bool staged = bx.vol <= kTileCap;
      const int nv = staged ? bx.vol : 0;
      // this lane's particle, read ahead of the staging barrier: warps 2 i and
      // 2 i + 1 take particles 32 i .. 32 i + 31, each one half of the stencil
      const int lp = (wid >> 1) * 32 + lane, sub = wid & 1;
      int p = 0;
      float X[3] = {0.f, 0.f, 0.f}, Fo[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) Fo[a] = 0.f;
      // the fixed flag and position, loaded with the state so that the
      // finish does not wait on them
      int pfixed = 0;
      float pfx[3] = {0.f, 0.f, 0.f};
      if (lp < ch.y) {
        p = A.perm[ch.x + lp];
#pragma unroll
        for (int a = 0; a < 3; ++a) X[a] = pt.x[a * n + p];
        if (sub == 0) {
#pragma unroll
          for (int a = 0; a < 9; ++a) Fo[a] = pt.F[(int64_t)a * n + p];
          pfixed = pt.fixed[p];
#pragma unroll
          for (int a = 0; a < 3; ++a) pfx[a] = pt.fixed_x[a * n + p];
        }
      }
      for (int li = tid; li < nv; li += T) {
        int i, j, k;
        box_ijk(bx, li, i, j, k);
        const int64_t node = ((int64_t)k * G + j) * G + i;
        const float m = g.m[node];
        const float P[3] = {g.v[node], g.v[N + node], g.v[2 * N + node]};
        float v[3] = {P[0], P[1], P[2]};
        if (m > 0.0f) {
          const float f[3] = {g.f_ext[node], g.f_ext[N + node], g.f_ext[2 * N + node]};
          grid_node_velocity(P, m, f, i, j, k, G, mp, v);
        }
        stg[li] = v[0];
        stg[nv + li] = v[1];
        stg[2 * nv + li] = v[2];
      }
      __syncthreads();  // also publishes the s_lo / s_hi reset
      float nvl[3] = {0.f, 0.f, 0.f}, nC[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      BSpline b;
      if (lp < ch.y) {
        bspline(X, mp.inv_dx, b);
        if (!staged) {
          if (sub == 0) g2p_gather_global(g, mp, b, nvl, nC);
        } else if (sub == 0) {
          g2p_gather_half<0>(stg, nv, bx, G, b, mp.dx, s4, nvl, nC);
        } else {
          g2p_gather_half<1>(stg, nv, bx, G, b, mp.dx, s4, nvl, nC);
        }
      }
      // the odd half's sums to the even half's lanes, through the part of
      // the tile the staged velocities leave free
      float* const xch = stg + kXchOffset;
      if (sub == 1 && lp < ch.y) {
#pragma unroll
        for (int q = 0; q < 3; ++q) xch[q * kChunk + lp] = nvl[q];
#pragma unroll
        for (int q = 0; q < 9; ++q) xch[(3 + q) * kChunk + lp] = nC[q];
      }
      __syncthreads();
      if (sub == 0 && lp < ch.y) {
#pragma unroll
        for (int q = 0; q < 3; ++q) nvl[q] += xch[q * kChunk + lp];
#pragma unroll
        for (int q = 0; q < 9; ++q) nC[q] += xch[(3 + q) * kChunk + lp];
        g2p_finish_f(pt, p, mp, X, nvl, nC, Fo, do_p2g ? ss : nullptr, kChunk, lp, pfixed, pfx);
#pragma unroll
        for (int r = 0; r < 3; ++r) nb[r] = base_of(X[r], mp.inv_dx);
        nb_live = true;
      }
    } else {
      __syncthreads();  // publishes the s_lo / s_hi reset
      if (tid < ch.y) {
        // ---- first launch: stage the state from the particle fields
        const int p = A.perm[ch.x + tid];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float x = pt.x[q * n + p];
          ss[(kSx + q) * kChunk + tid] = x;
          ss[(kSv + q) * kChunk + tid] = pt.v[q * n + p];
          nb[q] = base_of(x, mp.inv_dx);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          ss[(kSC + q) * kChunk + tid] = pt.C[(int64_t)q * n + p];
          ss[(kSF + q) * kChunk + tid] = pt.F[(int64_t)q * n + p];
        }
        nb_live = true;
      }
    }
    if (!do_p2g) continue;
    box_reduce(nb_live, nb, s_lo, s_hi);
    __syncthreads();  // the state stage and the box of substep s are complete
    int32_t rec[6];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      rec[r] = max(s_lo[r], 0);
      rec[3 + r] = s_hi[r] == INT_MIN ? -1 : min(min(s_hi[r], G) + 2, G - 1);
    }
    const Box bx = load_box(rec);
    const bool staged = bx.vol <= kTileCap;
    const int nv = staged ? bx.vol : 0;
    if (tid == 0) {
      int32_t* const out = A.box + bs * A.box_stride + 6 * c;
#pragma unroll
      for (int r = 0; r < 6; ++r) out[r] = rec[r];
      if (!staged) atomicAdd(A.meta + kMetaOverflow, 1);
    }
    // ---- P2G payload of substep s: warps of role 0 the stress and affine
    // momentum, warps of role 1 the B-spline data and the reaction force
    {
      const int role = wid & 1, slot = pslot;
      if (role == 0) {
        if (slot < ch.y) {
          const int p = pq;
          P2GParticle q;
          p2g_particle_rows(ss + kSF * kChunk, ss + kSC * kChunk, ss + kSv * kChunk, kChunk, slot, pmass, pvol0, mp,
                            q);
          pt.Jp[p] = q.J;
          float* const rq = sp + slot * kQn;
          *reinterpret_cast<float4*>(rq + kQmv) = make_float4(q.mv[0], q.mv[1], q.mv[2], q.mass);
          *reinterpret_cast<float4*>(rq + kQaff) = make_float4(q.aff[0], q.aff[1], q.aff[2], q.aff[3]);
          *reinterpret_cast<float4*>(rq + kQaff + 4) = make_float4(q.aff[4], q.aff[5], q.aff[6], q.aff[7]);
          rq[kQaff + 8] = q.aff[8];
        }
      } else {
        if (REACT && staged) {
          // the chunk's lattice box (force field, phi) into shared memory, by
          // the role-1 warps only (named barrier 1)
          for (int li = slot; li < nv; li += T / 2) {
            int i, j, k;
            box_ijk(bx, li, i, j, k);
            float h0 = 0.f, h1 = 0.f, h2 = 0.f, ph = 0.f;
            if (i < A.L.nx && j < A.L.ny && k < A.L.nz) {
              const int64_t cl = lat_cell(A.L, i, j, k);
              h0 = A.hydro[cl];
              h1 = A.hydro[A.L.pitch + cl];
              h2 = A.hydro[2 * A.L.pitch + cl];
              if (A.cp.kind != 0) ph = A.phi[cl];
            }
            stg[li] = h0;
            stg[nv + li] = h1;
            stg[2 * nv + li] = h2;
            stg[3 * nv + li] = ph;
          }
          asm volatile("bar.sync 1, %0;" ::"n"(kSeqT / 2) : "memory");
        }
        if (slot < ch.y) {
          const float X[3] = {ss[kSx * kChunk + slot], ss[(kSx + 1) * kChunk + slot], ss[(kSx + 2) * kChunk + slot]};
          BSpline b;
          bspline(X, mp.inv_dx, b);
          float pf[3] = {0.f, 0.f, 0.f};
          if (REACT) {
            float Fp[9];
#pragma unroll
            for (int r = 0; r < 9; ++r) Fp[r] = ss[(kSF + r) * kChunk + slot];
            const float J = det3(Fp);
            ReactParticle rp;
            if (staged)
              reaction_particle_staged(stg, bx, nv, A.L, A.cp, b, J, pvol0, s_scale, rp);
            else
              reaction_particle(A.L, A.hydro, A.phi, A.cp, b, J, pvol0, s_scale, rp);
            if (rp.act) ++n_act;
            pmax = fmaxf(pmax, rp.pnorm);
            if (rp.gated)
              for (int r = 0; r < 3; ++r) pn[r] += (double)rp.pf[r];
            if (rp.scatter)
              for (int r = 0; r < 3; ++r) pf[r] = rp.pf[r];
          }
          float* const rq = sp + slot * kQn;
          *reinterpret_cast<float4*>(rq + kQbase) =
              make_float4(__int_as_float(b.base[0]), __int_as_float(b.base[1]), __int_as_float(b.base[2]), b.fx[0]);
          *reinterpret_cast<float4*>(rq + kQfx1) = make_float4(b.fx[1], b.fx[2], pf[0], pf[1]);
          *reinterpret_cast<float4*>(rq + kQwx) = make_float4(b.w[0][0], b.w[0][1], b.w[0][2], pf[2]);
          *reinterpret_cast<float4*>(rq + kQwy) = make_float4(b.w[1][0], b.w[1][1], b.w[1][2], 0.f);
          *reinterpret_cast<float4*>(rq + kQwz) = make_float4(b.w[2][0], b.w[2][1], b.w[2][2], 0.f);
        }
        // the scatter tile, free since the last flush, zeroed by the role-1
        // warps while the role-0 warps finish the polar rotation
        for (int i = slot; i < 7 * nv; i += T / 2) tile[i] = 0.f;
      }
    }
    __syncthreads();  // payload complete, tile zeroed
    // ---- P2G scatter of substep s into buffer bs.  Warp w takes kRun
    // consecutive particles of the chunk, one at a time, lane o on stencil node
    // o; particles are sorted by base node within the chunk (fsi_mpm_bin), so
    // a run of particles with the same base is summed in registers and added
    // to the tile with one shared-memory atomic per node value.
    const FsiGrid g = grid_of(A, bs);
    float* const dst[7] = {g.v, g.v + N, g.v + 2 * N, g.m, g.f_ext, g.f_ext + N, g.f_ext + 2 * N};
    {
      constexpr int NQ = REACT ? 7 : 4;
      const int ox = lane / 9, oy = (lane / 3) % 3, oz = lane % 3;
      const float dox = (float)ox, doy = (float)oy, doz = (float)oz;
      float gsum[3] = {0.f, 0.f, 0.f}, gm2 = 0.f;
      float acc[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) acc[q] = 0.f;
      int cb0 = INT_MIN, cb1 = 0, cb2 = 0;  // base of the run (warp-uniform)
      // adds the run's sums of this lane's node to the tile (or the grid)
      auto flush_run = [&]() {
        const int I = cb0 + ox, Jj = cb1 + oy, K = cb2 + oz;
        if (lane < 27 && I >= 0 && I < G && Jj >= 0 && Jj < G && K >= 0 && K < G) {
          if (staged) {
            const int li = ((K - bx.lo[2]) * bx.ext[1] + (Jj - bx.lo[1])) * bx.ext[0] + (I - bx.lo[0]);
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              if (acc[q] != 0.f) atomicAdd(&tile[q * nv + li], acc[q]);
          } else {
            const int64_t node = ((int64_t)K * G + Jj) * G + I;
#pragma unroll
            for (int q = 0; q < NQ; ++q)
              if (acc[q] != 0.f) atomicAdd(dst[q] + node, acc[q]);
          }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = 0.f;
      };
      const int p1 = min(wid * kRun + kRun, ch.y);
      for (int lp = wid * kRun; lp < p1; ++lp) {
        const float* const rq = sp + lp * kQn;
        const float4 q4 = *reinterpret_cast<const float4*>(rq + kQbase);
        const int b0 = __float_as_int(q4.x), b1 = __float_as_int(q4.y), b2 = __float_as_int(q4.z);
        if (b0 != cb0 || b1 != cb1 || b2 != cb2) {
          if (cb0 != INT_MIN) flush_run();
          cb0 = b0;
          cb1 = b1;
          cb2 = b2;
        }
        if (lane < 27) {
          // weights of bspline() (staged by the payload) and offsets as in p2g_node()
          const float4 q5 = *reinterpret_cast<const float4*>(rq + kQfx1);
          const float w = rq[kQwx + ox] * rq[kQwy + oy] * rq[kQwz + oz];
          const float dpos[3] = {(dox - q4.w) * mp.dx, (doy - q5.x) * mp.dx, (doz - q5.y) * mp.dx};
          const float4 m4 = *reinterpret_cast<const float4*>(rq + kQmv);
          const float4 a0 = *reinterpret_cast<const float4*>(rq + kQaff);
          const float4 a1 = *reinterpret_cast<const float4*>(rq + kQaff + 4);
          const float a8 = rq[kQaff + 8];
          const float mv[3] = {m4.x, m4.y, m4.z};
          const float aff[9] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a8};
#pragma unroll
          for (int q = 0; q < 3; ++q)
            acc[q] += w * (mv[q] + (aff[3 * q] * dpos[0] + aff[3 * q + 1] * dpos[1] + aff[3 * q + 2] * dpos[2]));
          acc[3] += w * m4.w;
          if (REACT) {
            const float f0 = q5.z, f1 = q5.w, f2 = rq[kQwx + 3];
            if (f0 != 0.f || f1 != 0.f || f2 != 0.f) {
              const float v4 = w * f0, v5 = w * f1, v6 = w * f2;
              acc[NQ - 3] += v4;
              acc[NQ - 2] += v5;
              acc[NQ - 1] += v6;
              gsum[0] += v4;
              gsum[1] += v5;
              gsum[2] += v6;
              gm2 = fmaxf(gm2, v4 * v4 + v5 * v5 + v6 * v6);
            }
          }
        }
      }
      if (cb0 != INT_MIN) flush_run();
      if (REACT) {
#pragma unroll
        for (int q = 0; q < 3; ++q) gn[q] += (double)gsum[q];
        gmax = fmaxf(gmax, sqrtf(gm2));
      }
    }
    __syncthreads();
    for (int li = tid; li < nv; li += T) {
      int i, j, k;
      box_ijk(bx, li, i, j, k);
      const int64_t node = ((int64_t)k * G + j) * G + i;
#pragma unroll
      for (int q = 0; q < 7; ++q) {
        const float v = tile[q * nv + li];
        if (v != 0.f) atomicAdd(dst[q] + node, v);
      }
    }
  }
  if (REACT && do_p2g) {
    // diagnostics reductions (penalty.py:202-240, moving_boundary.py:312-374):
    // warp, then CTA, then one global atomic per CTA and quantity
    const int na = __reduce_add_sync(0xffffffffu, (unsigned)n_act);
    const float pm = warp_max(pmax), gm = warp_max(gmax);
    double r6[6];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      r6[r] = warp_sum_d(pn[r]);
      r6[3 + r] = warp_sum_d(gn[r]);
    }
    if (lane == 0) {
      s_cnt[wid] = na;
      s_fmax[wid][0] = pm;
      s_fmax[wid][1] = gm;
#pragma unroll
      for (int r = 0; r < 6; ++r) s_dsum[wid][r] = r6[r];
    }
    __syncthreads();
    if (tid == 0) {
      int ca = 0;
      float m0 = 0.f, m1 = 0.f;
      double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      for (int w = 0; w < NW; ++w) {
        ca += s_cnt[w];
        m0 = fmaxf(m0, s_fmax[w][0]);
        m1 = fmaxf(m1, s_fmax[w][1]);
        for (int r = 0; r < 6; ++r) d[r] += s_dsum[w][r];
      }
      if (ca) atomicAdd(&st->active_reaction_particle_count, ca);
      if (m0 > 0.f) atomic_max_nonneg(&st->max_particle_reaction_norm, m0);
      if (m1 > 0.f) atomic_max_nonneg(&st->max_grid_reaction_norm, m1);
      for (int r = 0; r < 3; ++r) {
        if (d[r] != 0.0) atomicAdd(&st->net_particle_reaction[r], d[r]);
        if (d[3 + r] != 0.0) atomicAdd(&st->net_grid_reaction[r], d[3 + r]);
      }
    }
  }
}

__global__ __launch_bounds__(kSeqT) void k_mpm_seq_prologue(const __grid_constant__ SeqArgs A) {
  griddep_wait();
  griddep_launch();
  seq_prologue_body(A, blockIdx.x, gridDim.x);
}

template <bool REACT>
__global__ __launch_bounds__(kSeqT, 2) void k_mpm_seq(const __grid_constant__ SeqArgs A) {
  griddep_wait();
  griddep_launch();
  mpm_seq_body<REACT>(A, blockIdx.x, gridDim.x);
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
  if (n_grid > 1600) return invalid("n_grid above 1600 is not supported by the binned substeps");
  const int64_t nb = (n_grid + kEdge - 1) / kEdge;
  const int64_t bins = nb * nb * nb;
  const int64_t mc = ((int64_t)n_particles + kChunk - 1) / kChunk + std::min<int64_t>(n_particles, bins);
  if (bins > INT_MAX || mc > INT_MAX / 18) return invalid("grid or particle count too large for binning");
  *n_bins = (int32_t)bins;
  *max_chunks = (int32_t)mc;
  return FSI_OK;
}

int check_bins(const FsiMpmBins* bins, int32_t n_particles, int32_t n_grid) {
  if (!bins) return invalid("null bins");
  if (!bins->key || !bins->count || !bins->start || !bins->perm || !bins->chunk || !bins->box || !bins->meta)
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

int sm_count() { return device_sm_count(); }

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// CTAs of a fused-sequence launch: one resident wave (at most one CTA per chunk)
int seq_ctas(bool react, int max_chunks, int* ctas) {
  static int occ[64][2] = {};
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return invalid("device ordinal out of range");
  int& o = occ[dev][react ? 1 : 0];
  if (!o) {
    void (*k)(const SeqArgs) = react ? k_mpm_seq<true> : k_mpm_seq<false>;
    if ((rc = cuda_check(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSeqSmem),
                         "k_mpm_seq shared memory")))
      return rc;
    int b = 0;
    if ((rc = cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kSeqT, kSeqSmem), "k_mpm_seq occupancy")))
      return rc;
    o = b > 0 ? b : 1;
  }
  *ctas = std::max(1, std::min(max_chunks, sm_count() * o));
  return FSI_OK;
}

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
  if ((rc = launch_check("k_bin_scatter"))) return rc;
  // the bin keys are no longer needed: key[] is the sort's scratch
  k_bin_sort<<<(unsigned)std::min(bins->n_bins, sm_count() * 8), kSortT, 0, st>>>(
      *pt, mp->inv_dx, g->n, bins->n_bins, bins->start, bins->perm, bins->key);
  return launch_check("k_bin_sort");
}

extern "C" int fsi_mpm_substeps_binned(const FsiParticles* pt, const FsiGrid grid[3], const FsiMpmBins* bins,
                                       const FsiMpmParams* mp, int32_t n_substeps, const FsiLbmState* s,
                                       const float* hydro, const FsiCouplingParams* cp, FsiCouplingStats stats[3],
                                       void* stream) {
  int rc = check_particles(pt);
  if (rc) return rc;
  if (!grid || !mp) return invalid("null grid or params");
  for (int b = 0; b < 3; ++b)
    if ((rc = check_grid(&grid[b]))) return rc;
  if (grid[0].n != grid[1].n || grid[0].n != grid[2].n) return invalid("the three grid buffers differ in size");
  if (n_substeps < 0) return invalid("n_substeps must be >= 0");
  if ((rc = check_bins(bins, pt->n, grid[0].n))) return rc;
  if (cp) {
    if (!s || !hydro || !stats) return invalid("reaction transfer needs the lattice state, hydro and stats");
    if (cp->kind < 0 || cp->kind > 2) return invalid("reaction kind must be 0 (penalty), 1 (engineering), 2 (link-area)");
    if (cp->kind != 0 && !s->phi) return invalid("moving-boundary reaction needs phi");
    if (cp->kind == 2 && !s->diag) return invalid("link-area reaction needs the directional reductions");
    if (cp->inv_dx_norm != mp->inv_dx)
      return invalid("binned substep needs the coupling and MPM grids to share dx (inv_dx_norm == inv_dx)");
  }
  if (n_substeps == 0) return FSI_OK;
  SeqArgs A{};
  A.pt = *pt;
  for (int b = 0; b < 3; ++b) A.grid[b] = grid[b];
  A.mp = *mp;
  A.perm = bins->perm;
  A.chunks = reinterpret_cast<const int2*>(bins->chunk);
  A.meta = bins->meta;
  A.box = bins->box;
  A.box_stride = (int64_t)6 * bins->max_chunks;
  if (cp) {
    A.L = LatView{s->nx, s->ny, s->nz, s->pitch};
    A.hydro = hydro;
    A.phi = s->phi;
    A.cp = *cp;
    A.stats = stats;
    A.diag = s->diag;
  }
  A.M = n_substeps;
  int ctas = 0;
  if ((rc = seq_ctas(cp != nullptr, bins->max_chunks, &ctas))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t lerr = launch_pdl(k_mpm_seq_prologue, dim3(ctas), dim3(kSeqT), 0, st, A);
  if ((rc = cuda_check(lerr, "k_mpm_seq_prologue (launch)")) || (rc = launch_check("k_mpm_seq_prologue"))) return rc;
  for (int i = 0; i <= n_substeps; ++i) {
    A.s = i;
    lerr = cp ? launch_pdl(k_mpm_seq<true>, dim3(ctas), dim3(kSeqT), kSeqSmem, st, A)
              : launch_pdl(k_mpm_seq<false>, dim3(ctas), dim3(kSeqT), kSeqSmem, st, A);
    if ((rc = cuda_check(lerr, "k_mpm_seq (launch)")) || (rc = launch_check("k_mpm_seq"))) return rc;
  }
  return FSI_OK;
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

// the sequence arguments of a batched case (one thread, into shared memory)
__device__ __forceinline__ void load_batch_seq(const FsiBatchCase& bc, int s, int M, SeqArgs* A) {
  A->pt = bc.pt;
#pragma unroll
  for (int b = 0; b < 3; ++b) A->grid[b] = bc.grid[b];
  A->mp = bc.mp;
  A->perm = bc.bins.perm;
  A->chunks = reinterpret_cast<const int2*>(bc.bins.chunk);
  A->meta = bc.bins.meta;
  A->box = bc.bins.box;
  A->box_stride = (int64_t)6 * bc.bins.max_chunks;
  A->L = LatView{bc.lbm.nx, bc.lbm.ny, bc.lbm.nz, bc.lbm.pitch};
  A->hydro = batch_hydro(bc);
  A->phi = bc.lbm.phi;
  A->cp = bc.cp;
  A->stats = bc.react_stats;
  A->diag = bc.lbm.diag;
  A->s = s;
  A->M = M;
}

__global__ __launch_bounds__(kSeqT) void k_batch_mpm_seq_prologue(const FsiBatchCase* __restrict__ cases) {
  __shared__ SeqArgs A;
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  if (threadIdx.x == 0) load_batch_seq(bc, 0, 1, &A);
  __syncthreads();
  seq_prologue_body(A, blockIdx.x, gridDim.x);
}

__global__ __launch_bounds__(kSeqT, 2) void k_batch_mpm_seq(const FsiBatchCase* __restrict__ cases, int s, int M) {
  __shared__ SeqArgs A;
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  if (threadIdx.x == 0) load_batch_seq(bc, s, M, &A);
  __syncthreads();
  mpm_seq_body<true>(A, blockIdx.x, gridDim.x);
}

__global__ __launch_bounds__(kSortT) void k_batch_bin_sort(const FsiBatchCase* __restrict__ cases) {
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (!bc.active) return;
  bin_sort_body(bc.pt, bc.mp.inv_dx, bc.grid[0].n, bc.bins.n_bins, bc.bins.start, bc.bins.perm, bc.bins.key,
                blockIdx.x, gridDim.x);
}

int check_batch_mpm(const FsiBatchCase* cases, const FsiBatchDims* d) {
  if (!cases || !d) return invalid("null batch argument");
  if (d->n_cases <= 0 || d->n_cases > 65535) return invalid("n_cases must be in 1..65535");
  if (d->max_particles <= 0 || d->max_chunks <= 0 || d->max_bins <= 0) return invalid("batch MPM dims must be positive");
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
  if ((rc = launch_check("k_batch_bin_scatter"))) return rc;
  k_batch_bin_sort<<<dim3((unsigned)std::min(d->max_bins, 64), d->n_cases), kSortT, 0, st>>>(cases);
  return launch_check("k_batch_bin_sort");
}

extern "C" int fsi_batch_mpm_substeps(FsiBatchCase* cases, const FsiBatchDims* d, int32_t n_substeps,
                                      void* stream) {
  int rc = check_batch_mpm(cases, d);
  if (rc) return rc;
  if (n_substeps < 0) return invalid("n_substeps must be >= 0");
  if (n_substeps == 0) return FSI_OK;
  cudaStream_t st = (cudaStream_t)stream;
  {
    // once per device (not during stream capture of a later call)
    static bool attr_set[64] = {};
    int dev = 0;
    if ((rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
    if (dev < 0 || dev >= 64) return invalid("device ordinal out of range");
    if (!attr_set[dev]) {
      if ((rc = cuda_check(cudaFuncSetAttribute(k_batch_mpm_seq, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kSeqSmem),
                           "k_batch_mpm_seq shared memory")))
        return rc;
      attr_set[dev] = true;
    }
  }
  // about one CTA per chunk of the largest case (a bin's chunks hold <= 128 particles each; bins
  // partly filled add chunks): CTAs stride over the case's chunk table
  if (d->mpm_ctas < 0 || d->mpm_ctas > 65535) return invalid("FsiBatchDims.mpm_ctas must be in 0..65535");
  const unsigned gx = d->mpm_ctas > 0 ? (unsigned)d->mpm_ctas
                                      : (unsigned)std::min<int64_t>(d->max_chunks, 2 * nblk(d->max_particles, kChunk) + 8);
  const dim3 gc(gx, d->n_cases);
  k_batch_mpm_seq_prologue<<<gc, kSeqT, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_mpm_seq_prologue"))) return rc;
  for (int i = 0; i <= n_substeps; ++i) {
    k_batch_mpm_seq<<<gc, kSeqT, kSeqSmem, st>>>(cases, i, n_substeps);
    if ((rc = launch_check("k_batch_mpm_seq"))) return rc;
  }
  return FSI_OK;
}

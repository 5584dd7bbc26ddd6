// LBM kernels of the coupled FSI step (D3Q19 MRT, AA-pattern, SoA).
//
// Reference semantics (src/mpm_lbm/sim/lbm/fluid.py):
//   step_moving_bounceback 2105-2111 = clear diag 443 -> colission 398 ->
//   streaming_moving_bounceback 488 -> finalize diag 521 -> Boundary_condition
//   538 -> streaming3 1794.
// One launch of k_lbm_step performs, per cell, the previous step's open
// boundary (pending) and macroscopic update, then this step's collision and
// streaming, so a step costs one read and one write of the 19 populations.
//
// Thread layout: blockDim = (32, 8); a warp covers 32 consecutive x cells of
// one (j, k) row, so the x-face open boundaries (which read the populations of
// x = 1, nx-2, nx-3 of the same row) resolve with warp shuffles.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "d3q19.cuh"

namespace fsi {

constexpr uint8_t kSolid = FSI_CELL_SOLID, kNear = FSI_CELL_NEAR, kLink = FSI_CELL_LINK,
                  kOverride = FSI_CELL_OVERRIDE, kCF = FSI_CELL_CF;

// unknown populations of the x faces (fluid.py:26-27): {1,7,9,11,13} / {2,8,10,12,14}
__host__ __device__ constexpr int kUnknownL(int q) { return q == 0 ? 1 : 2 * q + 5; }
__host__ __device__ constexpr int kUnknownR(int q) { return kUnknownL(q) + 1; }

struct Case {
  FsiLbmState s;
  FsiLbmParams p;
  FsiStepCtl c;
  MrtK K;
  int pf_dist;  // tiles between a CTA's tile and the one it prefetches into L2 (0: none)
  int aligned;  // nx % 32 == 0: every row starts a 32-cell block of the population storage
};

// ------------------------------------------------------------ storage ----
template <bool H>
struct Pop;

// Element index of population s of a cell.  Populations are stored in
// blocks of 32 cells: block b = cell / 32 holds the 19 populations of its
// cells as 19 runs of 32 values, element (s, cell) at b * 608 + s * 32 +
// cell % 32.  A warp of 32 aligned cells still reads 128 contiguous bytes
// per population, and the 19 accesses of one cell differ by the constant
// s * 128 bytes, which the compiler folds into the load / store immediate
// (one address computation per cell instead of one per population).  The
// block base is computed in 32 bits (the host checks 19 * pitch < 2^32).
__device__ __forceinline__ int64_t pop_index(const Case&, int s, int64_t cell) {
  const uint32_t i = (uint32_t)cell;
  return (int64_t)(i + (i >> 5) * 576u) + 32 * s;
}

template <>
struct Pop<false> {
  static __device__ __forceinline__ float ld(const Case& c, int s, int64_t cell) {
    return __ldg(static_cast<const float*>(c.s.pop) + pop_index(c, s, cell));
  }
  static __device__ __forceinline__ float ld_rw(const Case& c, int s, int64_t cell) {
    return static_cast<const float*>(c.s.pop)[pop_index(c, s, cell)];
  }
  static __device__ __forceinline__ void st(const Case& c, int s, int64_t cell, float v) {
    static_cast<float*>(c.s.pop)[pop_index(c, s, cell)] = v;
  }
  // by block-layout index b (pop_index without the 32 s term)
  static __device__ __forceinline__ float ldb(const Case& c, int s, int64_t b) {
    return __ldg(static_cast<const float*>(c.s.pop) + b + 32 * s);
  }
  static __device__ __forceinline__ void stb(const Case& c, int s, int64_t b, float v) {
    static_cast<float*>(c.s.pop)[b + 32 * s] = v;
  }
};

// half storage of the scaled deviation from rest equilibrium: h = f / w - rho0
template <>
struct Pop<true> {
  static __device__ __forceinline__ float ld(const Case& c, int s, int64_t cell) {
    const __half h = static_cast<const __half*>(c.s.pop)[pop_index(c, s, cell)];
    return lattice_w(s) * (c.p.rho0 + __half2float(h));
  }
  static __device__ __forceinline__ float ld_rw(const Case& c, int s, int64_t cell) { return ld(c, s, cell); }
  static __device__ __forceinline__ void st(const Case& c, int s, int64_t cell, float v) {
    const float inv_w = s == 0 ? 3.0f : (s <= 6 ? 18.0f : 36.0f);
    static_cast<__half*>(c.s.pop)[pop_index(c, s, cell)] = __float2half_rn(__fmaf_rn(v, inv_w, -c.p.rho0));
  }
  static __device__ __forceinline__ float ldb(const Case& c, int s, int64_t b) {
    const __half h = static_cast<const __half*>(c.s.pop)[b + 32 * s];
    return lattice_w(s) * (c.p.rho0 + __half2float(h));
  }
  static __device__ __forceinline__ void stb(const Case& c, int s, int64_t b, float v) {
    const float inv_w = s == 0 ? 3.0f : (s <= 6 ? 18.0f : 36.0f);
    static_cast<__half*>(c.s.pop)[b + 32 * s] = __float2half_rn(__fmaf_rn(v, inv_w, -c.p.rho0));
  }
};

struct Coord {
  int x, j, k;
};

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ int64_t cell_of(const Case& c, int x, int j, int k) {
  return ((int64_t)k * c.s.ny + j) * c.s.nx + x;
}

__device__ __forceinline__ int64_t nb_cell(const Case& c, const Coord& q, int dx, int dy, int dz) {
  return cell_of(c, wrapi(q.x + dx, c.s.nx), wrapi(q.j + dy, c.s.ny), wrapi(q.k + dz, c.s.nz));
}

// Location of population s of fluid cell q in the current AA layout.
__device__ __forceinline__ void pop_slot(const Case& c, const Coord& q, int64_t cell, uint8_t fl, uint32_t nb, int s,
                                         int& slot_s, int64_t& slot_cell) {
  if (c.c.parity == 0 || s == 0 || (fl & kSolid)) {
    slot_s = s;
    slot_cell = cell;
    return;
  }
  const bool src_solid = (fl & kNear) && ((nb >> kOpp(s)) & 1u);
  if (src_solid) {
    slot_s = s;
    slot_cell = cell;
  } else {
    slot_s = kOpp(s);
    slot_cell = nb_cell(c, q, -kEx(s), -kEy(s), -kEz(s));
  }
}

template <bool H>
__device__ __forceinline__ float decode_pop(const Case& c, const Coord& q, int s) {
  const int64_t cell = cell_of(c, q.x, q.j, q.k);
  const uint8_t fl = c.s.flags[cell];
  const uint32_t nb = (fl & kNear) ? c.s.nbr[cell] : 0u;
  int ss;
  int64_t sc;
  pop_slot(c, q, cell, fl, nb, s, ss, sc);
  return Pop<H>::ld_rw(c, ss, sc);
}

// ------------------------------------------------------- open boundary ----
struct FaceIn {
  float Fni[5];      // populations of ni in the unknown directions
  float Fn2[5];      // populations of n2i (convective outlet)
  bool n1_solid;     // solid[1] (left face) / solid[nx-2] (right face)
  bool n2_fluid;     // solid[n2i] == 0
  float mac_n[4];    // rho, ux, uy, uz of ni from the previous macroscopic update
  float mac_leg[4];  // legacy pressure face: v[1] or v[0] (left), v[nx-2] (right)
};

// fluid.py:1059-1096 (limited) and 1026-1029 (plain) for one unknown population
__device__ __forceinline__ float regularized_pop(const FsiLbmParams& p, bool limited, int s, float trho, float tu0,
                                                 float tu1, float tu2, float Fn, const float* mac, int* cnt) {
  float rl = trho, u0 = tu0, u1 = tu1, u2 = tu2;
  if (limited && p.limiter) {
    cnt[4] += 1;
    if (rl < p.ob_rho_min) {
      rl = p.ob_rho_min;
      cnt[0] += 1;
    }
    if (rl > p.ob_rho_max) {
      rl = p.ob_rho_max;
      cnt[0] += 1;
    }
    const float nrm = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    if (nrm > p.ob_u_max) {
      const float sc = p.ob_u_max / nrm;
      u0 *= sc;
      u1 *= sc;
      u2 *= sc;
      cnt[1] += 1;
    }
  }
  float noneq = Fn - feq(s, mac[0], mac[1], mac[2], mac[3]);
  if (limited && p.limiter) {
    if (noneq > p.ob_noneq_cap) {
      noneq = p.ob_noneq_cap;
      cnt[2] += 1;
    }
    if (noneq < -p.ob_noneq_cap) {
      noneq = -p.ob_noneq_cap;
      cnt[2] += 1;
    }
  }
  float out = feq(s, rl, u0, u1, u2) + noneq;
  if (limited && p.limiter && p.floor_enabled && out < p.ob_floor) {
    out = p.ob_floor;
    cnt[3] += 1;
  }
  return out;
}

// ---- pressure-outlet repair of semantics 4-9 (fluid.py:1106-1346) ----------
__device__ __forceinline__ float ob_bounded(float v, float lim) { return v > lim ? lim : (v < -lim ? -lim : v); }

// _limit_open_boundary_population (fluid.py:1043-1049)
__device__ __forceinline__ float ob_floor_limit(const FsiLbmParams& p, float v) {
  return (p.limiter && p.floor_enabled && v < p.ob_floor) ? p.ob_floor : v;
}

// The repair records of the populations a thread evaluates.  Each record of
// the flow filter (flow_outlet_flux_error_filtered_run <- (1 - a) f + a e,
// fluid.py:1127-1131) is an affine map of f; fd, fb hold the composite of the
// thread's records in order as f -> (1 - fd) f + fb (zero: no record).
struct ObRepair {
  int count;
  float corr, delta, fdelta;
  bool gain;
  float fd, fb;
};

__device__ __forceinline__ void ob_filter_add(ObRepair& r, float alpha, float err) {
  r.fb = (1.0f - alpha) * r.fb + alpha * err;
  r.fd = r.fd + alpha * (1.0f - r.fd);
}

// composite of map (d1, b1) followed by map (d2, b2)
__device__ __forceinline__ void ob_filter_then(float& d1, float& b1, float d2, float b2) {
  b1 = (1.0f - d2) * b1 + b2;
  d1 = d1 + d2 - d1 * d2;
}

// Slot of outlet row (j, k) for its filter composite: plane 4 of the plane
// array, in the reference's loop order over the face (j outer, k inner).
__device__ __forceinline__ float* ob_filter_slot(const FsiLbmState& st, int j, int k) {
  const int64_t n = (int64_t)st.ny * st.nz;
  return st.plane + 16 * n + 2 * ((int64_t)j * st.nz + k);
}

// One unknown population s of a right-face pressure-outlet cell (bc_right == 1)
// under semantics 4-9: trho = rho_bc_right, tu = v[ni] (mac_n: rho, v of ni
// from the last macroscopic update), Fn / Fn2 = F[ni] / F[n2i]; dc holds the
// controller feedback.  Records go to r.
__device__ float repaired_outlet_pop(const FsiLbmParams& p, const FsiLbmDiag* dc, int s, float trho,
                                     float tu0, float tu1, float tu2, float Fn, float Fn2, bool n2_fluid,
                                     const float* mac_n, ObRepair& r) {
  const int sem = p.ob_semantics;
  const float vx_in = p.vel_bc_left[0];  // vx_bcxl
  const float noneq = Fn - feq(s, mac_n[0], mac_n[1], mac_n[2], mac_n[3]);
  const float before = feq(s, trho, tu0, tu1, tu2) + noneq;  // _regularized_population (fluid.py:1032-1035)
  float inner;
  if (sem == FSI_OB_REG_MASS_BALANCED || sem == FSI_OB_CONV_MASS_BALANCED) {  // fluid.py:1266-1276
    const float rho_fb = ob_bounded(0.02f * (p.rho0 - mac_n[0]), 0.01f);
    const float vel_fb = ob_bounded(0.05f * (vx_in - tu0), 0.02f);
    const float after = feq(s, trho + rho_fb, tu0 + vel_fb, tu1, tu2) + noneq;
    r.count += 1;
    r.corr += fabsf(rho_fb) + fabsf(vel_fb);
    r.delta += fabsf(after - before);
    inner = ob_floor_limit(p, after);
  } else if (sem == FSI_OB_REG_FLUX_MATCHED || sem == FSI_OB_CONV_FLUX_MATCHED) {  // fluid.py:1287-1306
    const float rho_fb = ob_bounded(p.ob_gain_rho * (p.rho0 - mac_n[0]), 0.01f);
    const float verr = vx_in - tu0;
    const float vel_fb = ob_bounded(p.ob_gain_u * verr, p.ob_cap_u);
    const float after = feq(s, trho + rho_fb, tu0 + vel_fb, tu1, tu2) + noneq;
    r.count += 1;
    r.corr += fabsf(rho_fb) + fabsf(vel_fb);
    r.delta += fabsf(after - before);
    r.fdelta += fabsf(vel_fb);
    r.gain = true;
    ob_filter_add(r, p.ob_filter_alpha, verr);
    inner = ob_floor_limit(p, after);
  } else {  // plane-flux controlled, fluid.py:1319-1337
    const float rho_fb = dc->pc_rho_fb;
    const float mn = (sem == FSI_OB_REG_PLANE_FLUX && p.ob_mass_neutral) ? dc->mn_rho_fb : 0.0f;
    const float vel_fb = dc->pc_u_fb;
    const float after = feq(s, trho + rho_fb + mn, tu0 + vel_fb, tu1, tu2) + noneq;
    const float corr = fabsf(rho_fb) + fabsf(mn) + fabsf(vel_fb);
    r.count += 1;
    r.corr += corr;
    r.delta += fabsf(after - before);
    r.fdelta += corr;
    r.gain = true;
    inner = ob_floor_limit(p, after);
  }
  if (sem == FSI_OB_REG_MASS_BALANCED || sem == FSI_OB_REG_FLUX_MATCHED || sem == FSI_OB_REG_PLANE_FLUX) return inner;
  // convective blend (fluid.py:1278-1285, 1308-1317, 1339-1346)
  const float conv = ob_floor_limit(p, n2_fluid ? 2.0f * Fn - Fn2 : Fn);
  const float blend = sem == FSI_OB_CONV_MASS_BALANCED ? 0.15f : p.ob_blend;
  const float repaired = conv + blend * (inner - conv);
  const float dd = fabsf(repaired - conv);
  r.count += 1;
  r.delta += dd;
  if (sem == FSI_OB_CONV_FLUX_MATCHED) {
    r.fdelta += dd;
    ob_filter_add(r, p.ob_filter_alpha, vx_in - tu0);
  } else if (sem == FSI_OB_CONV_PLANE_FLUX) {
    r.corr += dd;
    r.fdelta += dd;
  }
  return ob_floor_limit(p, repaired);
}

// one thread's repair records into the diagnostics (step and run)
__device__ __forceinline__ void ob_repair_flush(const FsiLbmParams& p, FsiLbmDiag* d, const ObRepair& r) {
  if (r.count) {
    atomicAdd(&d->obr_count_step, r.count);
    atomicAdd(&d->obr_count_run, r.count);
  }
  if (r.corr != 0.f) {
    atomicAdd(&d->obr_corr_step, r.corr);
    atomicAdd(&d->obr_corr_run, r.corr);
  }
  if (r.delta != 0.f) {
    atomicAdd(&d->obr_delta_step, r.delta);
    atomicAdd(&d->obr_delta_run, r.delta);
  }
  if (r.fdelta != 0.f) {
    atomicAdd(&d->obf_delta_step, r.fdelta);
    atomicAdd(&d->obf_delta_run, r.fdelta);
  }
  if (r.gain) d->obf_gain_step = p.ob_gain_u;
}

// Boundary_condition for one fluid face cell (fluid.py:926-1024, 1348-1493).
// rec: diagnostics the repair records go to (null: none, a readout);
// ctl: controller state; slot: the row's filter composite (with rec).
__device__ void apply_face_bc(const FsiLbmParams& p, const float* vdyn, int side, const FaceIn& in, float* F,
                              int* cnt, FsiLbmDiag* rec = nullptr, const FsiLbmDiag* ctl = nullptr,
                              float* slot = nullptr) {
  const int bc = side == 0 ? p.bc_left : p.bc_right;
  
  if (p.ob_semantics == FSI_OB_EQUILIBRIUM_RESET) {
    if (bc == 2) {
      const float* vb = side == 0 ? (vdyn ? vdyn : p.vel_bc_left) : p.vel_bc_right;
#pragma unroll
      for (int s = 0; s < 19; ++s) F[s] = feq(s, 1.0f, vb[0], vb[1], vb[2]);
    } else if (bc == 1) {
      const float rb = side == 0 ? p.rho_bc_left : p.rho_bc_right;
#pragma unroll
      for (int s = 0; s < 19; ++s) F[s] = feq(s, rb, in.mac_leg[1], in.mac_leg[2], in.mac_leg[3]);
    }
    return;
  }
  if (p.ob_semantics == FSI_OB_CONVECTIVE && side == 1 && bc == 1) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      float ex = in.Fni[q];
      if (in.n2_fluid) ex = 2.0f * in.Fni[q] - in.Fn2[q];
      if (p.limiter && p.floor_enabled && ex < p.ob_floor) ex = p.ob_floor;
      F[(side == 0 ? kUnknownL(q) : kUnknownR(q))] = ex;
    }
    return;
  }
  if (p.ob_semantics >= FSI_OB_REG_MASS_BALANCED && side == 1 && bc == 1) {
    ObRepair r{0, 0.f, 0.f, 0.f, false, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 5; ++q)
      F[kUnknownR(q)] = repaired_outlet_pop(p, ctl, kUnknownR(q), p.rho_bc_right, in.mac_n[1], in.mac_n[2],
                                            in.mac_n[3], in.Fni[q], in.Fn2[q], in.n2_fluid, in.mac_n, r);
    if (rec) {
      ob_repair_flush(p, rec, r);
      if (slot && r.fd != 0.f) {
        slot[0] = r.fd;
        slot[1] = r.fb;
      }
    }
    return;
  }
  const bool limited = p.ob_semantics == FSI_OB_REGULARIZED_LIMITED;
  float trho, t0, t1, t2;
  if (bc == 1) {
    trho = side == 0 ? p.rho_bc_left : p.rho_bc_right;
    t0 = in.mac_n[1];
    t1 = in.mac_n[2];
    t2 = in.mac_n[3];
  } else {
    trho = in.mac_n[0];
    if (trho <= 1.0e-6f) trho = p.rho0;
    const float* vb = side == 0 ? (vdyn ? vdyn : p.vel_bc_left) : p.vel_bc_right;
    t0 = vb[0];
    t1 = vb[1];
    t2 = vb[2];
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) F[(side == 0 ? kUnknownL(q) : kUnknownR(q))] = regularized_pop(p, limited, (side == 0 ? kUnknownL(q) : kUnknownR(q)), trho, t0, t1, t2, in.Fni[q], in.mac_n, cnt);
}

__device__ __forceinline__ const float* plane_ptr(const Case& c, int plane) {
  return c.s.plane + (int64_t)plane * 4 * c.s.ny * c.s.nz;
}

__device__ __forceinline__ void load_plane(const Case& c, int plane, int row, float* m) {
  const float* pp = plane_ptr(c, plane);
  const int64_t n = (int64_t)c.s.ny * c.s.nz;
#pragma unroll
  for (int a = 0; a < 4; ++a) m[a] = pp[a * n + row];
}

constexpr unsigned kFull = 0xffffffffu;

// Limiter counters of one warp (rho, velocity, noneq, floor, reconstructed).
__device__ __forceinline__ void flush_counts(const Case& c, const int* cnt) {
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const int v = (int)__reduce_add_sync(kFull, (unsigned)cnt[a]);
    if ((threadIdx.x & 31) == 0 && v) {
      atomicAdd(&c.s.diag->ob_step[a], v);
      atomicAdd(&c.s.diag->ob_run[a], v);
    }
  }
}

// One population of a face cell, evaluated by lane `lane` (population index
// lane for the equilibrium reset, unknown population number lane otherwise).
struct FaceVal {
  float val;
  int packed;  // five 6-bit limiter counters
  ObRepair rep;
};

__device__ __forceinline__ FaceVal face_population(const FsiLbmParams& p, const float* vdyn, int side, int lane,
                                                   float Fn, float Fn2, bool n2_fluid, const float* mac_n,
                                                   const float* mac_l, FsiLbmDiag* d) {
  FaceVal r{0.f, 0, ObRepair{0, 0.f, 0.f, 0.f, false, 0.f, 0.f}};
  const int bc = side == 0 ? p.bc_left : p.bc_right;
  const float* vb = side == 0 ? (vdyn ? vdyn : p.vel_bc_left) : p.vel_bc_right;
  if (p.ob_semantics == FSI_OB_EQUILIBRIUM_RESET) {  // fluid.py:926-1024
    if (lane < 19) {
      if (bc == 2) r.val = feq(lane, 1.0f, vb[0], vb[1], vb[2]);
      else r.val = feq(lane, side == 0 ? p.rho_bc_left : p.rho_bc_right, mac_l[1], mac_l[2], mac_l[3]);
    }
    return r;
  }
  if (lane >= 5) return r;
  const int s = side == 0 ? kUnknownL(lane) : kUnknownR(lane);
  if (p.ob_semantics >= FSI_OB_REG_MASS_BALANCED && side == 1 && bc == 1) {
    r.val = repaired_outlet_pop(p, d, s, p.rho_bc_right, mac_n[1], mac_n[2], mac_n[3], Fn, Fn2, n2_fluid, mac_n,
                                r.rep);
    return r;
  }
  if (p.ob_semantics == FSI_OB_CONVECTIVE && side == 1 && bc == 1) {  // fluid.py:1098-1103
    float ex = n2_fluid ? 2.0f * Fn - Fn2 : Fn;
    if (p.limiter && p.floor_enabled && ex < p.ob_floor) ex = p.ob_floor;
    r.val = ex;
    return r;
  }
  float trho, t0, t1, t2;
  if (bc == 1) {
    trho = side == 0 ? p.rho_bc_left : p.rho_bc_right;
    t0 = mac_n[1];
    t1 = mac_n[2];
    t2 = mac_n[3];
  } else {
    trho = mac_n[0];
    if (trho <= 1.0e-6f) trho = p.rho0;
    t0 = vb[0];
    t1 = vb[1];
    t2 = vb[2];
  }
  int cnt[5] = {0, 0, 0, 0, 0};
  r.val = regularized_pop(p, p.ob_semantics == FSI_OB_REGULARIZED_LIMITED, s, trho, t0, t1, t2, Fn, mac_n, cnt);
  r.packed = cnt[0] | (cnt[1] << 6) | (cnt[2] << 12) | (cnt[3] << 18) | (cnt[4] << 24);
  return r;
}

// the repair records of a face warp's lanes (lane q: unknown population q of
// the face cell of face row `row`), one set of atomics per warp, and the
// row's filter composite in population order
__device__ __forceinline__ void ob_repair_warp(const Case& c, int lane, int row, const ObRepair& r) {
  ObRepair w;
  w.count = (int)__reduce_add_sync(kFull, (unsigned)r.count);
  w.corr = warp_sum(r.corr);
  w.delta = warp_sum(r.delta);
  w.fdelta = warp_sum(r.fdelta);
  w.gain = __any_sync(kFull, r.gain);
  float fd = 0.f, fb = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) ob_filter_then(fd, fb, __shfl_sync(kFull, r.fd, q), __shfl_sync(kFull, r.fb, q));
  if (lane == 0) {
    ob_repair_flush(c.p, c.s.diag, w);
    if (fd != 0.f) {
      float* slot = ob_filter_slot(c.s, row % c.s.ny, row / c.s.ny);
      slot[0] = fd;
      slot[1] = fb;
    }
  }
}

// Open boundary of one x face for the warp holding that face cell: the five
// (or nineteen) face populations are computed by different lanes and gathered
// into the face lane with shuffles.
template <int SIDE>
__device__ __forceinline__ void bc_face_warp(const Case& c, int lane, int row, uint8_t fl, float* F) {
  const int nx = c.s.nx;
  const int lf = SIDE == 0 ? 0 : ((nx - 1) & 31);
  const int l1 = SIDE == 0 ? 1 : ((nx - 2) & 31);
  const int l2 = SIDE == 0 ? 1 : ((nx - 3) & 31);
  const unsigned solid_bits = __ballot_sync(kFull, (fl & kSolid) != 0);
  if ((solid_bits >> lf) & 1u) return;
  const bool n1_solid = (solid_bits >> l1) & 1u;
  const bool n2_fluid = n1_solid ? true : !((solid_bits >> l2) & 1u);
  float mac_n[4], mac_l[4] = {0.f, 0.f, 0.f, 0.f};
  // an equilibrium-reset velocity face (bc 2) reads no plane either
  if (!(c.p.ob_semantics == FSI_OB_EQUILIBRIUM_RESET && (SIDE == 0 ? c.p.bc_left : c.p.bc_right) == 2))
    load_plane(c, SIDE == 0 ? (n1_solid ? 1 : 0) : 2, row, mac_l);
  if (c.p.ob_semantics == FSI_OB_EQUILIBRIUM_RESET) {
    // the equilibrium reset reads neither the neighbours' unknown
    // populations nor the neighbour plane (face_population)
    const FaceVal r = face_population(c.p, c.s.vel_left_dyn, SIDE, lane, 0.f, 0.f, n2_fluid, mac_l, mac_l, c.s.diag);
#pragma unroll
    for (int s = 0; s < 19; ++s) {
      const float v = __shfl_sync(kFull, r.val, s);
      if (lane == lf) F[s] = v;
    }
  } else {
    const int src1 = n1_solid ? lf : l1, src2 = n1_solid ? lf : l2;
    float Fn = 0.f, Fn2 = 0.f;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const int s = SIDE == 0 ? kUnknownL(q) : kUnknownR(q);
      const float a = __shfl_sync(kFull, F[s], src1);
      const float b = __shfl_sync(kFull, F[s], src2);
      if (lane == q) {
        Fn = a;
        Fn2 = b;
      }
    }
    load_plane(c, SIDE == 0 ? (n1_solid ? 0 : 1) : (n1_solid ? 3 : 2), row, mac_n);
    const FaceVal r = face_population(c.p, c.s.vel_left_dyn, SIDE, lane, Fn, Fn2, n2_fluid, mac_n, mac_l, c.s.diag);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float v = __shfl_sync(kFull, r.val, q);
      if (lane == lf) F[SIDE == 0 ? kUnknownL(q) : kUnknownR(q)] = v;
    }
    if (c.p.limiter) {
      const int cnt[5] = {r.packed & 63, (r.packed >> 6) & 63, (r.packed >> 12) & 63, (r.packed >> 18) & 63,
                          (r.packed >> 24) & 63};
      flush_counts(c, cnt);
    }
    if (SIDE == 1 && c.p.ob_semantics >= FSI_OB_REG_MASS_BALANCED && c.p.bc_right == 1)
      ob_repair_warp(c, lane, row, r.rep);
  }
}

// ---- plane sums of the outlet flux controller (fluid.py:1152-1187, 1225-1229)
// From the macroscopic state the collision uses, which is the rho, v the
// reference's controller reads at the open boundary of the same step:
// t[0] rho u_x over the fluid cells of x = 0, t[1] over the measure plane
// (x = nx - 1 - offset, at least 0), t[2] the measure plane's fluid cell
// count, t[3..6] rho u_x over x = nx-1, nx-2, nx-3, nx-4 (each at least 0),
// t[7] the fluid mass (mass-neutral feedback only).
__device__ __forceinline__ void plane_flux_add(const Case& c, int x, bool fluid, float rho, float ux, float* t) {
  const int nx = c.s.nx;
  const int mi = max(0, nx - 1 - c.p.ob_measure_offset);
  const float q = fluid ? rho * ux : 0.f;
  t[0] += x == 0 ? q : 0.f;
  t[1] += x == mi ? q : 0.f;
  t[2] += (fluid && x == mi) ? 1.f : 0.f;
  t[3] += x == nx - 1 ? q : 0.f;
  t[4] += x == max(0, nx - 2) ? q : 0.f;
  t[5] += x == max(0, nx - 3) ? q : 0.f;
  t[6] += x == max(0, nx - 4) ? q : 0.f;
  t[7] += fluid ? rho : 0.f;
}

// one warp's sums into pc_acc (the fluid mass in FP64 into mn_mass_acc, so
// that its value does not depend on the order of the atomics); x0 .. x0 + w - 1
// is the warp's x range
__device__ __forceinline__ void plane_flux_flush(const Case& c, int lane, int x0, int w, const float* t) {
  const int nx = c.s.nx;
  const int mi = max(0, nx - 1 - c.p.ob_measure_offset);
  const bool planes = x0 == 0 || (mi >= x0 && mi < x0 + w) || x0 + w > nx - 4;
  if (planes) {
#pragma unroll
    for (int a = 0; a < 7; ++a) {
      const float v = warp_sum(t[a]);
      if (lane == 0 && v != 0.f) atomicAdd(&c.s.diag->pc_acc[a], v);
    }
  }
  if (c.p.ob_mass_neutral) {
    const double m = warp_sum_d((double)t[7]);
    if (lane == 0 && m != 0.0) atomicAdd(&c.s.diag->mn_mass_acc, m);
  }
}

// --------------------------------------------------------- step kernel ----
struct DirAcc {
  int cnt[19];
  float csum[19];
  float cmax[19];
  float imp[19][3];
  int any;
};

// wrapped neighbourhood of a cell: row bases for dy, dz in {-1, 0, 1} and x +- 1
struct Nbh {
  int rb[3][3];
  int xm, xp, x;
  int bxm, bxp, bx;  // block-layout indices of xm, xp, x (row 0)
  __device__ __forceinline__ int at(int dx, int dy, int dz) const {
    return rb[dz + 1][dy + 1] + (dx < 0 ? xm : (dx > 0 ? xp : x));
  }
  // block-layout index of a neighbour when every row starts a 32-cell block
  // (Case::aligned): row part 19 * rb plus x part, one multiply-add
  __device__ __forceinline__ int64_t blk(int dx, int dy, int dz) const {
    // unsigned arithmetic: 19 * row base reaches 2^32 (the host bounds 19 * pitch by 2^32)
    return (int64_t)((uint32_t)rb[dz + 1][dy + 1] * 19u + (uint32_t)(dx < 0 ? bxm : (dx > 0 ? bxp : bx)));
  }
};

__device__ __forceinline__ int block_index(int i) { return i + (int)((uint32_t)i >> 5) * 576; }

__device__ __forceinline__ void make_nbh(const Case& c, int x, int j, int k, Nbh& n) {
  const int nx = c.s.nx, ny = c.s.ny, nz = c.s.nz;
  const int jj[3] = {j == 0 ? ny - 1 : j - 1, j, j == ny - 1 ? 0 : j + 1};
  const int kk[3] = {k == 0 ? nz - 1 : k - 1, k, k == nz - 1 ? 0 : k + 1};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) n.rb[a][b] = (kk[a] * ny + jj[b]) * nx;
  n.xm = x == 0 ? nx - 1 : x - 1;
  n.xp = x == nx - 1 ? 0 : x + 1;
  n.x = x;
  n.bxm = block_index(n.xm);
  n.bxp = block_index(n.xp);
  n.bx = block_index(x);
}

template <bool H>
__device__ __forceinline__ float ldp(const Case& c, int s, int idx) {
  return Pop<H>::ld(c, s, (int64_t)idx);
}

template <bool H>
__device__ __forceinline__ void stp(const Case& c, int s, int idx, float v) {
  Pop<H>::st(c, s, (int64_t)idx, v);
}

// mb_subcycle_force_accum_norm_max over the lanes of a warp that reach this
// point (the LINK cells of the warp): one redux and one atomic per warp
// instead of one contended atomic per cell (norms are non-negative, so their
// bit patterns order as unsigned integers)
__device__ __forceinline__ void accum_max_warp(const Case& c, float nrm) {
  const unsigned am = __activemask();
  const unsigned mx = __reduce_max_sync(am, __float_as_uint(nrm));
  if ((int)(threadIdx.x & 31) == __ffs(am) - 1) atomic_max_nonneg(&c.s.diag->accum_norm_max, __uint_as_float(mx));
}

// Streaming of a cell next to a solid: half-way bounce-back, with the
// moving-wall correction and momentum-exchange link force when MOVING
// (fluid.py:431-440, 488-519).
template <bool ODD, bool H, bool MOVING>
__device__ __forceinline__ void store_near_solid(const Case& c, const Nbh& n, int cell, uint32_t nb, float rho,
                                              const float* out) {
  float* hpp = c.s.hpp + (int64_t)c.c.pp * 3 * c.s.pitch;
  const int64_t P = c.s.pitch;
#pragma unroll
  for (int s = 0; s < 19; ++s) {
    float val = out[s];
    const bool bb = (nb >> s) & 1u;
    if (MOVING && bb) {
      const int ip = n.at(kEx(s), kEy(s), kEz(s));
      const float ew = (float)kEx(s) * c.s.svel[ip] + (float)kEy(s) * c.s.svel[P + ip] + (float)kEz(s) * c.s.svel[2 * P + ip];
      const float corr = -6.0f * lattice_w(s) * rho * ew;
      const float f0 = val;
      val = f0 + corr;
      const float tot = val + f0;  // solid force = e_s (bounced + f)
      if (kEx(s)) atomicAdd(hpp + ip, (float)kEx(s) * tot);
      if (kEy(s)) atomicAdd(hpp + P + ip, (float)kEy(s) * tot);
      if (kEz(s)) atomicAdd(hpp + 2 * P + ip, (float)kEz(s) * tot);
    }
    if (!ODD || s == 0 || bb)
      stp<H>(c, kOpp(s), cell, val);
    else
      stp<H>(c, s, n.at(kEx(s), kEy(s), kEz(s)), val);
  }
}

// Per-direction bounce-back reductions of one step (fluid.py:488-536: link
// counts, |correction| sum and max, fluid impulse), called by every lane of
// the warp together after the streaming stores: per direction the warp's link
// contributions are combined with shuffles and one lane adds them to the CTA's
// shared accumulator (float atomics to one shared address serialise, so that
// each direction sees at most one per warp).  nb: the lane's cell's solid
// neighbour mask (0 for no cell, solid or plain fluid); out: the cell's
// post-collision populations; rho: its density.
__device__ __forceinline__ void dirstats_warp(const Case& c, const Nbh& n, uint32_t nb, float rho, const float* out,
                                              DirAcc& acc) {
  // warps without a link cell (most of the lattice) skip the 18 ballots
  if (!__any_sync(kFull, nb != 0u)) return;
  const int64_t P = c.s.pitch;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 1; s < 19; ++s) {
    const bool link = (nb >> s) & 1u;
    const unsigned m = __ballot_sync(kFull, link);
    if (m == 0u) continue;
    float ac = 0.f, tot = 0.f;
    if (link) {
      const int ip = n.at(kEx(s), kEy(s), kEz(s));
      const float ew = (float)kEx(s) * c.s.svel[ip] + (float)kEy(s) * c.s.svel[P + ip] + (float)kEz(s) * c.s.svel[2 * P + ip];
      const float corr = -6.0f * lattice_w(s) * rho * ew;
      const float f0 = out[s];
      tot = (f0 + corr) + f0;  // solid force = e_s (bounced + f)
      ac = fabsf(corr);
    }
    const float sum = warp_sum(ac), mx = warp_max(ac), ts = warp_sum(tot);
    if (lane == 0) {
      atomicAdd(&acc.cnt[s], __popc(m));
      atomicAdd(&acc.csum[s], sum);
      atomic_max_nonneg(&acc.cmax[s], mx);
      if (kEx(s)) atomicAdd(&acc.imp[s][0], -(float)kEx(s) * ts);
      if (kEy(s)) atomicAdd(&acc.imp[s][1], -(float)kEy(s) * ts);
      if (kEz(s)) atomicAdd(&acc.imp[s][2], -(float)kEz(s) * ts);
      acc.any = 1;
    }
  }
}

// One cell of the fused step, read before its collision: position, flags,
// solid-neighbour mask and post-streaming populations.  The step of a cell is
// step_cell_load followed by step_cell_finish, so that a thread can issue the
// loads of several cells before it collides the first.
struct StepCell {
  int x, jr, k;
  uint8_t fl;
  uint32_t nb;
  float F[19];
};

template <bool ODD, bool H>
__device__ __forceinline__ void step_cell_load(const Case& c, int x, int jr, int bz, StepCell& q) {
  const int nx = c.s.nx, ny = c.s.ny;
  const bool inrow = jr < ny;
  const bool valid = inrow && x < nx;
  const int j = inrow ? jr : 0, k = bz;
  const int row = k * ny + j;
  const int cell = row * nx + x;
  q.x = x;
  q.jr = jr;
  q.k = bz;
  const uint8_t fl = valid ? c.s.flags[cell] : kSolid;
  const bool fluid = !(fl & kSolid);
  const uint32_t nb = (fluid && (fl & kNear)) ? c.s.nbr[cell] : 0u;
  q.fl = fl;
  q.nb = nb;
  Nbh n;
  if (ODD || nb) make_nbh(c, x < nx ? x : 0, j, k, n);
  float* const F = q.F;

  // ---- post-streaming populations of this cell (AA layout, fluid.py:431-440)
  if (fluid) {
    if (!ODD) {
#pragma unroll
      for (int s = 0; s < 19; ++s) F[s] = ldp<H>(c, s, cell);
    } else if (nb == 0) {
      F[0] = ldp<H>(c, 0, cell);
      if (c.aligned) {
#pragma unroll
        for (int s = 1; s < 19; ++s) F[s] = Pop<H>::ldb(c, kOpp(s), n.blk(-kEx(s), -kEy(s), -kEz(s)));
      } else {
#pragma unroll
        for (int s = 1; s < 19; ++s) F[s] = ldp<H>(c, kOpp(s), n.at(-kEx(s), -kEy(s), -kEz(s)));
      }
    } else {
      F[0] = ldp<H>(c, 0, cell);
#pragma unroll
      for (int s = 1; s < 19; ++s) {
        const bool src_solid = (nb >> kOpp(s)) & 1u;
        F[s] = src_solid ? ldp<H>(c, s, cell) : ldp<H>(c, kOpp(s), n.at(-kEx(s), -kEy(s), -kEz(s)));
      }
    }
  } else {
#pragma unroll
    for (int s = 0; s < 19; ++s) F[s] = 0.f;
  }

}

// The rest of the step of one cell (everything after its loads) for the warp's
// 32 cells x = 32 bx + lane of one row; ends with the cell's part of the
// per-direction link statistics (the caller synchronises the CTA and flushes
// them).
template <bool ODD, bool H, bool MOVING, bool BCW, bool PEN>
__device__ __forceinline__ void step_cell_finish(const Case& c, int bx, StepCell& q, DirAcc& acc) {
  const int lane = threadIdx.x;
  const int nx = c.s.nx, ny = c.s.ny, nz = c.s.nz;
  const int x = q.x;
  const bool inrow = q.jr < ny;
  const bool valid = inrow && x < nx;
  const int j = inrow ? q.jr : 0, k = q.k;
  const int row = k * ny + j;
  const int cell = row * nx + x;
  const bool dirstats = MOVING && (c.c.mode & FSI_MODE_DIRSTATS);
  const uint8_t fl = q.fl;
  const bool fluid = !(fl & kSolid);
  const uint32_t nb = q.nb;
  Nbh n;
  if (ODD || nb) make_nbh(c, x < nx ? x : 0, j, k, n);
  float* const F = q.F;

  // ---- pending open boundary of the previous step (fluid.py:538-569)
  if (BCW && c.c.bc_pending && inrow) {
    if (c.p.bc_left != 0 && bx == 0) bc_face_warp<0>(c, lane, row, fl, F);
    if (c.p.bc_right != 0 && bx == ((nx - 1) >> 5)) bc_face_warp<1>(c, lane, row, fl, F);
  }

  // ---- macroscopic state the collision uses (streaming3 of the previous step, fluid.py:1794-1814)
  float rho = c.p.rho0, ux = 0.f, uy = 0.f, uz = 0.f;
  float cf0 = 0.f, cf1 = 0.f, cf2 = 0.f;
  const int64_t P = c.s.pitch;
  if (fluid && (fl & kCF)) {
    cf0 = c.s.cell_force[cell];
    cf1 = c.s.cell_force[P + cell];
    cf2 = c.s.cell_force[2 * P + cell];
  }
  if (valid && (fl & kOverride)) {
    rho = c.s.rho[cell];
    ux = c.s.vel[cell];
    uy = c.s.vel[P + cell];
    uz = c.s.vel[2 * P + cell];
  } else if (fluid) {
    float jx, jy, jz;
    moments0(F, rho, jx, jy, jz);
    const float inv = __frcp_rn(rho);
    ux = (jx + 0.5f * (c.p.force[0] + cf0)) * inv;
    uy = (jy + 0.5f * (c.p.force[1] + cf1)) * inv;
    uz = (jz + 0.5f * (c.p.force[2] + cf2)) * inv;
  }
  if (BCW) {
    __syncwarp();
    // planes x = 0, 1, nx - 2, nx - 1 lie in the first and last 32-cell tiles
    // of a row (nx >= 4 with open faces), so other warps skip the test
    const bool edge_tile = bx == 0 || bx >= ((nx - 2) >> 5);
    const int plane = !edge_tile ? -1 : (x == 0 ? 0 : (x == 1 ? 1 : (x == nx - 2 ? 2 : (x == nx - 1 ? 3 : -1))));
    if (valid && plane >= 0) {
      float* pp = c.s.plane + (int64_t)plane * 4 * ny * nz;
      const int64_t m = (int64_t)ny * nz;
      pp[row] = rho;
      pp[m + row] = ux;
      pp[2 * m + row] = uy;
      pp[3 * m + row] = uz;
    }
    if (c.p.ob_semantics >= FSI_OB_REG_PLANE_FLUX) {
      float t[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      plane_flux_add(c, x, fluid, rho, ux, t);
      plane_flux_flush(c, lane, bx * 32, 32, t);
    }
  }

  // ---- penalty force built from this state (coupling/penalty.py:59-88)
  float Ax = c.p.force[0] + cf0, Ay = c.p.force[1] + cf1, Az = c.p.force[2] + cf2;
  uint8_t nfl = fl & (uint8_t)~kOverride;
  if (PEN) {
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;
    bool active = false;
    if (fluid) {
      const float phi = c.s.phi[cell];
      if (phi > c.p.penalty_phi_min) {
        const float sc = c.p.penalty_beta * phi * rho;
        f0 = sc * (c.s.svel[cell] - ux);
        f1 = sc * (c.s.svel[P + cell] - uy);
        f2 = sc * (c.s.svel[2 * P + cell] - uz);
        const float nrm = sqrtf(f0 * f0 + f1 * f1 + f2 * f2);
        if (nrm > c.p.penalty_cap) {
          const float r = c.p.penalty_cap / nrm;
          f0 *= r;
          f1 *= r;
          f2 *= r;
        }
        active = true;
      }
    }
    if (active || (valid && (fl & kCF))) {
      c.s.cell_force[cell] = f0;
      c.s.cell_force[P + cell] = f1;
      c.s.cell_force[2 * P + cell] = f2;
      c.s.hydro[cell] = -f0;
      c.s.hydro[P + cell] = -f1;
      c.s.hydro[2 * P + cell] = -f2;
    }
    nfl = active ? (nfl | kCF) : (nfl & (uint8_t)~kCF);
    Ax = c.p.force[0] + f0;
    Ay = c.p.force[1] + f1;
    Az = c.p.force[2] + f2;
    if (__any_sync(kFull, active)) {
      const int na = __popc(__ballot_sync(kFull, active));
      const float mx = warp_max(sqrtf(f0 * f0 + f1 * f1 + f2 * f2));
      const float s0 = warp_sum(f0), s1 = warp_sum(f1), s2 = warp_sum(f2);
      if (lane == 0) {
        atomicAdd(&c.s.diag->penalty_active, na);
        atomic_max_nonneg(&c.s.diag->penalty_max_norm, mx);
        atomicAdd(&c.s.diag->penalty_net[0], s0);
        atomicAdd(&c.s.diag->penalty_net[1], s1);
        atomicAdd(&c.s.diag->penalty_net[2], s2);
      }
    }
  }
  if (valid && nfl != fl) c.s.flags[cell] = nfl;

  // ---- collision (fluid.py:398-413) and AA streaming
  // the Guo term only where some fluid cell of the warp is forced (body force,
  // penalty or cell force); with no force it vanishes exactly
  const bool forced = __any_sync(kFull, fluid && (Ax != 0.f || Ay != 0.f || Az != 0.f));
  if (fluid) {
    if (forced)
      mrt_collide<true>(F, rho, ux, uy, uz, Ax, Ay, Az, c.K, F);
    else
      mrt_collide<false>(F, rho, ux, uy, uz, Ax, Ay, Az, c.K, F);
    if (nb == 0) {
      if (!ODD) {
#pragma unroll
        for (int s = 0; s < 19; ++s) stp<H>(c, kOpp(s), cell, F[s]);
      } else {
        stp<H>(c, 0, cell, F[0]);
        if (c.aligned) {
#pragma unroll
          for (int s = 1; s < 19; ++s) Pop<H>::stb(c, s, n.blk(kEx(s), kEy(s), kEz(s)), F[s]);
        } else {
#pragma unroll
          for (int s = 1; s < 19; ++s) stp<H>(c, s, n.at(kEx(s), kEy(s), kEz(s)), F[s]);
        }
      }
    } else {
      store_near_solid<ODD, H, MOVING>(c, n, cell, nb, rho, F);
    }
  } else if (MOVING && valid && (fl & kLink)) {
    // solid cell receiving link forces: recycle last step's ping-pong slot
    float* prev = c.s.hpp + (int64_t)(c.c.pp ^ 1) * 3 * P;
    if (c.c.mode & FSI_MODE_SUBCYCLED) {
      float a[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        a[d] = c.s.accum[d * P + cell] + prev[d * P + cell];
        c.s.accum[d * P + cell] = a[d];
        prev[d * P + cell] = 0.f;
      }
      accum_max_warp(c, sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d) prev[d * P + cell] = 0.f;
    }
  }

  if (dirstats) dirstats_warp(c, n, fluid ? nb : 0u, rho, F, acc);
}

// the CTA's per-direction link statistics of one step: zeroed before the
// tile's cells, flushed to FsiLbmDiag after them (one atomic per direction)
__device__ __forceinline__ void dirstats_begin(DirAcc& acc, int nthreads) {
  const int tid = threadIdx.y * 32 + threadIdx.x;
  for (int i = tid; i < 19; i += nthreads) {
    acc.cnt[i] = 0;
    acc.csum[i] = 0.f;
    acc.cmax[i] = 0.f;
    acc.imp[i][0] = acc.imp[i][1] = acc.imp[i][2] = 0.f;
  }
  if (tid == 0) acc.any = 0;
  __syncthreads();
}

__device__ __forceinline__ void dirstats_end(const Case& c, DirAcc& acc, int nthreads) {
  __syncthreads();
  if (acc.any) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int i = tid; i < 19; i += nthreads) {
      if (acc.cnt[i]) {
        atomicAdd(&c.s.diag->link_count[i], acc.cnt[i]);
        atomicAdd(&c.s.diag->corr_abs_sum[i], acc.csum[i]);
        atomic_max_nonneg(&c.s.diag->corr_abs_max[i], acc.cmax[i]);
        atomicAdd(&c.s.diag->fluid_impulse[i][0], acc.imp[i][0]);
        atomicAdd(&c.s.diag->fluid_impulse[i][1], acc.imp[i][1]);
        atomicAdd(&c.s.diag->fluid_impulse[i][2], acc.imp[i][2]);
      }
    }
  }
}

// One tile of the fused step: the 32 x 8 cells (x, row = k * ny + j) of tile
// (bx, by).  Called by the single-case kernel (c in the parameter bank) and by
// the batched kernel (c staged in shared memory); acc: the CTA's shared
// per-direction accumulator.
template <bool ODD, bool H, bool MOVING, bool BCW, bool PEN>
__device__ __forceinline__ void lbm_step_tile(const Case& c, int bx, int by, int bz, DirAcc& acc) {
  const bool dirstats = MOVING && (c.c.mode & FSI_MODE_DIRSTATS);
  if (dirstats) dirstats_begin(acc, 256);
  StepCell q;
  step_cell_load<ODD, H>(c, bx * 32 + (int)threadIdx.x, by * 8 + (int)threadIdx.y, bz, q);
  step_cell_finish<ODD, H, MOVING, BCW, PEN>(c, bx, q, acc);
  if (dirstats) dirstats_end(c, acc, 256);
}

// L2 prefetch of the populations of tile (bx, by, bz) of a 32 x 8 x 1 tiling:
// its 8 rows of 32 cells in the 19 planes, one 128-byte line per thread.
template <bool H>
__device__ __forceinline__ void prefetch_tile_l2(const Case& c, int bx, int by, int bz) {
  const int tid = threadIdx.y * 32 + threadIdx.x;
  if (tid >= 19 * 8) return;
  const int s = tid >> 3, j = by * 8 + (tid & 7);
  if (j >= c.s.ny) return;
  const int64_t idx = pop_index(c, s, (int64_t)(bz * c.s.ny + j) * c.s.nx + bx * 32);
  const void* ptr = H ? static_cast<const void*>(static_cast<const __half*>(c.s.pop) + idx)
                      : static_cast<const void*>(static_cast<const float*>(c.s.pop) + idx);
  asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr));
}

// MINB: resident CTAs per SM the register allocation must allow (3: no
// spills; 4: 64 registers with a few spilled words).  PF: each CTA first
// prefetches into L2 the tile c.pf_dist tiles after its own in launch order
// (about one resident wave later), so that the populations of the next wave
// are read from L2.  The host picks both from FsiLbmParams.tune (chosen by the
// autotuner of the Python layer).  Grid: (ceil(nx / 32), ceil(ny / 8), nz).
template <bool ODD, bool H, bool MOVING, bool BCW, bool PEN, int MINB, bool PF>
__global__ void __launch_bounds__(256, MINB) k_lbm_step(const Case c) {
  __shared__ DirAcc acc;
  griddep_wait();
  griddep_launch();
  if (PF) {
    const unsigned gx = gridDim.x, gy = gridDim.y;
    const unsigned t = blockIdx.x + gx * (blockIdx.y + gy * blockIdx.z) + (unsigned)c.pf_dist;
    if (t < gx * gy * gridDim.z) {
      const unsigned r = t / gx;
      prefetch_tile_l2<H>(c, (int)(t - r * gx), (int)(r % gy), (int)(r / gy));
    }
  }
  lbm_step_tile<ODD, H, MOVING, BCW, PEN>(c, blockIdx.x, blockIdx.y, blockIdx.z, acc);
}

// ------------------------------------------- paired step (2 cells/thread) ----
// The same step as lbm_step_tile for the two adjacent cells (x0, x0 + 1) of
// each thread (x0 even; nx even, so that the pair is 8-byte aligned): a warp
// covers 64 cells of a row, a tile 64 x 4 cells.  Populations of a pair move
// as float2 / half2 where the AA layout keeps them adjacent (every direction
// on even steps; directions without an x component on odd steps), and the
// collision runs on the paired FP32 pipe (mrt_collide2).  Cells next to a
// solid, penalty forces and open boundaries take the per-cell paths of the
// one-cell kernel.
template <bool H>
struct Pop2;

template <>
struct Pop2<false> {
  static __device__ __forceinline__ float2 ld(const Case& c, int s, int64_t cell) {
    return __ldg(reinterpret_cast<const float2*>(static_cast<const float*>(c.s.pop) + pop_index(c, s, cell)));
  }
  static __device__ __forceinline__ void st(const Case& c, int s, int64_t cell, float2 v) {
    *reinterpret_cast<float2*>(static_cast<float*>(c.s.pop) + pop_index(c, s, cell)) = v;
  }
  // by block-layout index b of the pair's first cell (b even)
  static __device__ __forceinline__ float2 ldb(const Case& c, int s, int64_t b) {
    return __ldg(reinterpret_cast<const float2*>(static_cast<const float*>(c.s.pop) + b + 32 * s));
  }
  static __device__ __forceinline__ void stb(const Case& c, int s, int64_t b, float2 v) {
    *reinterpret_cast<float2*>(static_cast<float*>(c.s.pop) + b + 32 * s) = v;
  }
};

template <>
struct Pop2<true> {
  static __device__ __forceinline__ float2 ld(const Case& c, int s, int64_t cell) {
    return ldb(c, s, pop_index(c, 0, cell));
  }
  static __device__ __forceinline__ void st(const Case& c, int s, int64_t cell, float2 v) {
    stb(c, s, pop_index(c, 0, cell), v);
  }
  // the decode and encode of Pop<true> on both cells at once (paired FP32
  // instructions, the same roundings)
  static __device__ __forceinline__ float2 ldb(const Case& c, int s, int64_t b) {
    const __half2 h = *reinterpret_cast<const __half2*>(static_cast<const __half*>(c.s.pop) + b + 32 * s);
    return __fmul2_rn(make_float2(lattice_w(s), lattice_w(s)), __fadd2_rn(make_float2(c.p.rho0, c.p.rho0), __half22float2(h)));
  }
  static __device__ __forceinline__ void stb(const Case& c, int s, int64_t b, float2 v) {
    const float inv_w = s == 0 ? 3.0f : (s <= 6 ? 18.0f : 36.0f);
    const float2 e = __ffma2_rn(v, make_float2(inv_w, inv_w), make_float2(-c.p.rho0, -c.p.rho0));
    *reinterpret_cast<__half2*>(static_cast<__half*>(c.s.pop) + b + 32 * s) = __floats2half2_rn(e.x, e.y);
  }
};

__device__ __forceinline__ float comp(const float2& v, int i) { return i ? v.y : v.x; }
__device__ __forceinline__ void set_comp(float2& v, int i, float a) {
  if (i)
    v.y = a;
  else
    v.x = a;
}

// Open boundary of one x face for the warp holding that face cell, pairs
// layout: face cell, first and second neighbour by (lane, component).
template <int SIDE>
__device__ __forceinline__ void bc_face_warp2(const Case& c, int lane, int row, uint8_t fl0, uint8_t fl1,
                                              float2* F) {
  const int nx = c.s.nx;
  const unsigned sb0 = __ballot_sync(kFull, (fl0 & kSolid) != 0), sb1 = __ballot_sync(kFull, (fl1 & kSolid) != 0);
  const int lr = ((nx - 1) & 63) >> 1;  // lane of x = nx - 1 (component 1) and x = nx - 2 (component 0)
  const int lf = SIDE == 0 ? 0 : lr, cf = SIDE == 0 ? 0 : 1;
  const int l1 = SIDE == 0 ? 0 : lr, c1 = SIDE == 0 ? 1 : 0;
  const int l2 = SIDE == 0 ? 1 : lr - 1, c2 = SIDE == 0 ? 0 : 1;
  const bool face_solid = ((cf ? sb1 : sb0) >> lf) & 1u;
  if (face_solid) return;
  const bool n1_solid = ((c1 ? sb1 : sb0) >> l1) & 1u;
  const bool n2_fluid = n1_solid ? true : !(((c2 ? sb1 : sb0) >> l2) & 1u);
  const int src1 = n1_solid ? lf : l1, cs1 = n1_solid ? cf : c1;
  const int src2 = n1_solid ? lf : l2, cs2 = n1_solid ? cf : c2;
  float Fn = 0.f, Fn2 = 0.f;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const int s = SIDE == 0 ? kUnknownL(q) : kUnknownR(q);
    const float a = __shfl_sync(kFull, comp(F[s], cs1), src1);
    const float b = __shfl_sync(kFull, comp(F[s], cs2), src2);
    if (lane == q) {
      Fn = a;
      Fn2 = b;
    }
  }
  float mac_n[4], mac_l[4];
  load_plane(c, SIDE == 0 ? (n1_solid ? 0 : 1) : (n1_solid ? 3 : 2), row, mac_n);
  load_plane(c, SIDE == 0 ? (n1_solid ? 1 : 0) : 2, row, mac_l);
  const FaceVal r = face_population(c.p, c.s.vel_left_dyn, SIDE, lane, Fn, Fn2, n2_fluid, mac_n, mac_l, c.s.diag);
  if (c.p.ob_semantics == FSI_OB_EQUILIBRIUM_RESET) {
#pragma unroll
    for (int s = 0; s < 19; ++s) {
      const float v = __shfl_sync(kFull, r.val, s);
      if (lane == lf) set_comp(F[s], cf, v);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float v = __shfl_sync(kFull, r.val, q);
      if (lane == lf) set_comp(F[SIDE == 0 ? kUnknownL(q) : kUnknownR(q)], cf, v);
    }
    if (c.p.limiter) {
      const int cnt[5] = {r.packed & 63, (r.packed >> 6) & 63, (r.packed >> 12) & 63, (r.packed >> 18) & 63,
                          (r.packed >> 24) & 63};
      flush_counts(c, cnt);
    }
    if (SIDE == 1 && c.p.ob_semantics >= FSI_OB_REG_MASS_BALANCED && c.p.bc_right == 1)
      ob_repair_warp(c, lane, row, r.rep);
  }
}

// Neighbourhood of the cell pair (x0, x0 + 1) of a thread (x0 even): the
// nine wrapped row bases (rows j + dy, k + dz) and the x coordinates x0 - 1,
// x0, x0 + 1, x0 + 2 (wrapped), with their block-layout indices for lattices
// whose rows start 32-cell blocks (Case::aligned).  One structure serves both
// members, so that a thread holds one set of row bases.
struct PairNbh {
  int rb[3][3];
  int xs[4];
  uint32_t bxs[4];
  // cell index of the neighbour (dx, dy, dz) of member m (0: x0, 1: x0 + 1)
  __device__ __forceinline__ int cell(int m, int dx, int dy, int dz) const {
    return rb[dz + 1][dy + 1] + xs[m + dx + 1];
  }
  // block-layout index of population 0 of that neighbour (pop_index without
  // the 32 s term); aligned: 19 * row base + block index of x, one multiply-add
  __device__ __forceinline__ int64_t blk(bool aligned, int m, int dx, int dy, int dz) const {
    if (aligned) return (int64_t)((uint32_t)rb[dz + 1][dy + 1] * 19u + bxs[m + dx + 1]);
    const uint32_t i = (uint32_t)cell(m, dx, dy, dz);
    return (int64_t)(i + (i >> 5) * 576u);
  }
};

__device__ __forceinline__ void make_pair_nbh(const Case& c, int x0, int j, int k, PairNbh& q) {
  const int nx = c.s.nx, ny = c.s.ny, nz = c.s.nz;
  const int jj[3] = {j == 0 ? ny - 1 : j - 1, j, j == ny - 1 ? 0 : j + 1};
  const int kk[3] = {k == 0 ? nz - 1 : k - 1, k, k == nz - 1 ? 0 : k + 1};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) q.rb[a][b] = (kk[a] * ny + jj[b]) * nx;
  q.xs[0] = x0 == 0 ? nx - 1 : x0 - 1;
  q.xs[1] = x0;
  q.xs[2] = x0 + 1;  // x0 even and nx even: x0 + 1 < nx
  q.xs[3] = x0 + 2 >= nx ? x0 + 2 - nx : x0 + 2;
  q.bxs[0] = (uint32_t)block_index(q.xs[0]);
  q.bxs[1] = (uint32_t)block_index(x0);
  q.bxs[2] = q.bxs[1] + 1u;  // x0 even: x0 + 1 lies in the same 32-cell block
  q.bxs[3] = (uint32_t)block_index(q.xs[3]);
}

template <int M>
__device__ __forceinline__ float cm(const float2& v) {
  return M ? v.y : v.x;
}
template <int M>
__device__ __forceinline__ void set_cm(float2& v, float a) {
  if (M)
    v.y = a;
  else
    v.x = a;
}

// post-streaming populations of member M of a pair when it is a fluid cell
// next to a solid (per-cell path, written into component M of F)
template <bool ODD, bool H, int M>
__device__ __forceinline__ void near_solid_loads2(const Case& c, const PairNbh& q, int cell, uint32_t nb, float2* F) {
  set_cm<M>(F[0], ldp<H>(c, 0, cell));
#pragma unroll
  for (int s = 1; s < 19; ++s) {
    float v;
    if (!ODD || ((nb >> kOpp(s)) & 1u))
      v = ldp<H>(c, s, cell);
    else
      v = Pop<H>::ldb(c, kOpp(s), q.blk(c.aligned, M, -kEx(s), -kEy(s), -kEz(s)));
    set_cm<M>(F[s], v);
  }
}

// streaming of member M next to a solid: store_near_solid for component M of
// the pair's post-collision populations
template <bool ODD, bool H, bool MOVING, int M>
__device__ __forceinline__ void near_solid_stores2(const Case& c, const PairNbh& q, int cell, uint32_t nb, float rho,
                                                   const float2* F) {
  float* hpp = c.s.hpp + (int64_t)c.c.pp * 3 * c.s.pitch;
  const int64_t P = c.s.pitch;
#pragma unroll
  for (int s = 0; s < 19; ++s) {
    float val = cm<M>(F[s]);
    const bool bb = (nb >> s) & 1u;
    if (MOVING && bb) {
      const int ip = q.cell(M, kEx(s), kEy(s), kEz(s));
      const float ew = (float)kEx(s) * c.s.svel[ip] + (float)kEy(s) * c.s.svel[P + ip] + (float)kEz(s) * c.s.svel[2 * P + ip];
      const float corr = -6.0f * lattice_w(s) * rho * ew;
      const float f0 = val;
      val = f0 + corr;
      const float tot = val + f0;  // solid force = e_s (bounced + f)
      if (kEx(s)) atomicAdd(hpp + ip, (float)kEx(s) * tot);
      if (kEy(s)) atomicAdd(hpp + P + ip, (float)kEy(s) * tot);
      if (kEz(s)) atomicAdd(hpp + 2 * P + ip, (float)kEz(s) * tot);
    }
    if (!ODD || s == 0 || bb)
      stp<H>(c, kOpp(s), cell, val);
    else
      Pop<H>::stb(c, s, q.blk(c.aligned, M, kEx(s), kEy(s), kEz(s)), val);
  }
}

// dirstats_warp for member M of every lane's pair
template <int M>
__device__ __forceinline__ void dirstats_warp2(const Case& c, const PairNbh& q, uint32_t nb, float rho, const float2* F,
                                               DirAcc& acc) {
  if (!__any_sync(kFull, nb != 0u)) return;
  const int64_t P = c.s.pitch;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int s = 1; s < 19; ++s) {
    const bool link = (nb >> s) & 1u;
    const unsigned m = __ballot_sync(kFull, link);
    if (m == 0u) continue;
    float ac = 0.f, tot = 0.f;
    if (link) {
      const int ip = q.cell(M, kEx(s), kEy(s), kEz(s));
      const float ew = (float)kEx(s) * c.s.svel[ip] + (float)kEy(s) * c.s.svel[P + ip] + (float)kEz(s) * c.s.svel[2 * P + ip];
      const float corr = -6.0f * lattice_w(s) * rho * ew;
      const float f0 = cm<M>(F[s]);
      tot = (f0 + corr) + f0;
      ac = fabsf(corr);
    }
    const float sum = warp_sum(ac), mx = warp_max(ac), ts = warp_sum(tot);
    if (lane == 0) {
      atomicAdd(&acc.cnt[s], __popc(m));
      atomicAdd(&acc.csum[s], sum);
      atomic_max_nonneg(&acc.cmax[s], mx);
      if (kEx(s)) atomicAdd(&acc.imp[s][0], -(float)kEx(s) * ts);
      if (kEy(s)) atomicAdd(&acc.imp[s][1], -(float)kEy(s) * ts);
      if (kEz(s)) atomicAdd(&acc.imp[s][2], -(float)kEz(s) * ts);
      acc.any = 1;
    }
  }
}

// penalty force of one cell (coupling/penalty.py:59-88); returns whether active
__device__ __forceinline__ bool penalty_cell(const Case& c, int cell, bool fluid, float rho, float ux, float uy,
                                             float uz, float& f0, float& f1, float& f2) {
  const int64_t P = c.s.pitch;
  f0 = f1 = f2 = 0.f;
  if (!fluid) return false;
  const float phi = c.s.phi[cell];
  if (!(phi > c.p.penalty_phi_min)) return false;
  const float sc = c.p.penalty_beta * phi * rho;
  f0 = sc * (c.s.svel[cell] - ux);
  f1 = sc * (c.s.svel[P + cell] - uy);
  f2 = sc * (c.s.svel[2 * P + cell] - uz);
  const float nrm = sqrtf(f0 * f0 + f1 * f1 + f2 * f2);
  if (nrm > c.p.penalty_cap) {
    const float r = c.p.penalty_cap / nrm;
    f0 *= r;
    f1 *= r;
    f2 *= r;
  }
  return true;
}

template <bool ODD, bool H, bool MOVING, bool BCW, bool PEN>
__device__ __forceinline__ void lbm_step_tile2(const Case& c, int bx, int by, DirAcc& acc) {
  const int lane = threadIdx.x;
  const int nx = c.s.nx, ny = c.s.ny, nz = c.s.nz;
  const int x0 = bx * 64 + 2 * lane;
  const int row = by * 4 + threadIdx.y;
  const bool inrow = row < ny * nz;
  const bool valid = inrow && x0 < nx;  // nx even: x0 + 1 < nx as well
  const int j = inrow ? row % ny : 0, k = inrow ? row / ny : 0;
  const int cell0 = valid ? row * nx + x0 : 0;
  const int64_t P = c.s.pitch;
  const bool dirstats = MOVING && (c.c.mode & FSI_MODE_DIRSTATS);
  if (dirstats) {
    const int tid = threadIdx.y * 32 + lane;
    for (int i = tid; i < 19; i += 128) {
      acc.cnt[i] = 0;
      acc.csum[i] = 0.f;
      acc.cmax[i] = 0.f;
      acc.imp[i][0] = acc.imp[i][1] = acc.imp[i][2] = 0.f;
    }
    if (tid == 0) acc.any = 0;
    __syncthreads();
  }
  uint8_t fl[2];
  if (valid) {
    const uint16_t f2 = *reinterpret_cast<const uint16_t*>(c.s.flags + cell0);
    fl[0] = (uint8_t)(f2 & 0xff);
    fl[1] = (uint8_t)(f2 >> 8);
  } else {
    fl[0] = fl[1] = kSolid;
  }
  const bool fluid0 = !(fl[0] & kSolid), fluid1 = !(fl[1] & kSolid);
  const uint32_t nb0 = (fluid0 && (fl[0] & kNear)) ? c.s.nbr[cell0] : 0u;
  const uint32_t nb1 = (fluid1 && (fl[1] & kNear)) ? c.s.nbr[cell0 + 1] : 0u;
  const bool plain = (nb0 | nb1) == 0u;
  PairNbh q;
  if (ODD || !plain) make_pair_nbh(c, valid ? x0 : 0, j, k, q);

  // ---- post-streaming populations (AA layout, fluid.py:431-440): a pair
  // moves as one float2 / half2 where the layout keeps it adjacent (every
  // direction on even steps, directions without an x component on odd steps)
  float2 F[19];
  if (fluid0 || fluid1) {
    if (plain) {
      if (!ODD) {
#pragma unroll
        for (int s = 0; s < 19; ++s) F[s] = Pop2<H>::ld(c, s, cell0);
      } else {
        F[0] = Pop2<H>::ld(c, 0, cell0);
        const bool al = c.aligned;
#pragma unroll
        for (int s = 1; s < 19; ++s) {
          if (kEx(s) == 0) {
            F[s] = Pop2<H>::ldb(c, kOpp(s), q.blk(al, 0, 0, -kEy(s), -kEz(s)));
          } else {
            F[s].x = Pop<H>::ldb(c, kOpp(s), q.blk(al, 0, -kEx(s), -kEy(s), -kEz(s)));
            F[s].y = Pop<H>::ldb(c, kOpp(s), q.blk(al, 1, -kEx(s), -kEy(s), -kEz(s)));
          }
        }
      }
    } else {
#pragma unroll
      for (int s = 0; s < 19; ++s) F[s] = make_float2(0.f, 0.f);
      if (fluid0) near_solid_loads2<ODD, H, 0>(c, q, cell0, nb0, F);
      if (fluid1) near_solid_loads2<ODD, H, 1>(c, q, cell0 + 1, nb1, F);
    }
  } else {
#pragma unroll
    for (int s = 0; s < 19; ++s) F[s] = make_float2(0.f, 0.f);
  }

  // ---- pending open boundary of the previous step (fluid.py:538-569)
  if (BCW && c.c.bc_pending && inrow) {
    if (c.p.bc_left != 0 && bx == 0) bc_face_warp2<0>(c, lane, row, fl[0], fl[1], F);
    if (c.p.bc_right != 0 && bx == ((nx - 1) >> 6)) bc_face_warp2<1>(c, lane, row, fl[0], fl[1], F);
  }

  // ---- macroscopic state the collision uses (streaming3, fluid.py:1794-1814)
  float2 cf0 = p2(0.f), cf1 = p2(0.f), cf2 = p2(0.f);
  if (fluid0 && (fl[0] & kCF)) {
    cf0.x = c.s.cell_force[cell0];
    cf1.x = c.s.cell_force[P + cell0];
    cf2.x = c.s.cell_force[2 * P + cell0];
  }
  if (fluid1 && (fl[1] & kCF)) {
    cf0.y = c.s.cell_force[cell0 + 1];
    cf1.y = c.s.cell_force[P + cell0 + 1];
    cf2.y = c.s.cell_force[2 * P + cell0 + 1];
  }
  float2 rho, ux, uy, uz;
  {
    float2 jx, jy, jz;
    moments0_2(F, rho, jx, jy, jz);
    const float2 inv = make_float2(__frcp_rn(rho.x), __frcp_rn(rho.y));
    ux = mul2(fma2(p2(0.5f), add2(p2(c.p.force[0]), cf0), jx), inv);
    uy = mul2(fma2(p2(0.5f), add2(p2(c.p.force[1]), cf1), jy), inv);
    uz = mul2(fma2(p2(0.5f), add2(p2(c.p.force[2]), cf2), jz), inv);
  }
  if (valid && ((fl[0] | fl[1]) & kOverride)) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (fl[i] & kOverride) {
        set_comp(rho, i, c.s.rho[cell0 + i]);
        set_comp(ux, i, c.s.vel[cell0 + i]);
        set_comp(uy, i, c.s.vel[P + cell0 + i]);
        set_comp(uz, i, c.s.vel[2 * P + cell0 + i]);
      }
    }
  }
  if (!fluid0 && !(valid && (fl[0] & kOverride))) {
    rho.x = c.p.rho0;
    ux.x = uy.x = uz.x = 0.f;
  }
  if (!fluid1 && !(valid && (fl[1] & kOverride))) {
    rho.y = c.p.rho0;
    ux.y = uy.y = uz.y = 0.f;
  }
  if (BCW) {
    __syncwarp();
    if (valid) {
      const int64_t m = (int64_t)ny * nz;
      const int pl0 = x0 == 0 ? 0 : (x0 == nx - 2 ? 2 : -1);
      const int pl1 = x0 + 1 == 1 ? 1 : (x0 + 1 == nx - 1 ? 3 : -1);
      if (pl0 >= 0) {
        float* pp = c.s.plane + (int64_t)pl0 * 4 * m;
        pp[row] = rho.x;
        pp[m + row] = ux.x;
        pp[2 * m + row] = uy.x;
        pp[3 * m + row] = uz.x;
      }
      if (pl1 >= 0) {
        float* pp = c.s.plane + (int64_t)pl1 * 4 * m;
        pp[row] = rho.y;
        pp[m + row] = ux.y;
        pp[2 * m + row] = uy.y;
        pp[3 * m + row] = uz.y;
      }
    }
    if (c.p.ob_semantics >= FSI_OB_REG_PLANE_FLUX) {
      float t[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      plane_flux_add(c, x0, fluid0, rho.x, ux.x, t);
      plane_flux_add(c, x0 + 1, fluid1, rho.y, ux.y, t);
      plane_flux_flush(c, lane, bx * 64, 64, t);
    }
  }

  // ---- penalty force built from this state (coupling/penalty.py:59-88)
  float2 Ax = add2(p2(c.p.force[0]), cf0), Ay = add2(p2(c.p.force[1]), cf1), Az = add2(p2(c.p.force[2]), cf2);
  uint8_t nfl[2] = {(uint8_t)(fl[0] & (uint8_t)~kOverride), (uint8_t)(fl[1] & (uint8_t)~kOverride)};
  if (PEN) {
    int na = 0;
    float mx = 0.f, s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int cell = cell0 + i;
      float f0, f1, f2;
      const bool active = penalty_cell(c, cell, i ? fluid1 : fluid0, comp(rho, i), comp(ux, i), comp(uy, i),
                                       comp(uz, i), f0, f1, f2);
      if (active || (valid && (fl[i] & kCF))) {
        c.s.cell_force[cell] = f0;
        c.s.cell_force[P + cell] = f1;
        c.s.cell_force[2 * P + cell] = f2;
        c.s.hydro[cell] = -f0;
        c.s.hydro[P + cell] = -f1;
        c.s.hydro[2 * P + cell] = -f2;
      }
      nfl[i] = active ? (nfl[i] | kCF) : (nfl[i] & (uint8_t)~kCF);
      set_comp(Ax, i, c.p.force[0] + f0);
      set_comp(Ay, i, c.p.force[1] + f1);
      set_comp(Az, i, c.p.force[2] + f2);
      if (active) {
        ++na;
        mx = fmaxf(mx, sqrtf(f0 * f0 + f1 * f1 + f2 * f2));
        s0 += f0;
        s1 += f1;
        s2 += f2;
      }
    }
    if (__any_sync(kFull, na > 0)) {
      const int nat = (int)__reduce_add_sync(kFull, (unsigned)na);
      const float wmx = warp_max(mx);
      const float w0 = warp_sum(s0), w1 = warp_sum(s1), w2 = warp_sum(s2);
      if (lane == 0) {
        atomicAdd(&c.s.diag->penalty_active, nat);
        atomic_max_nonneg(&c.s.diag->penalty_max_norm, wmx);
        atomicAdd(&c.s.diag->penalty_net[0], w0);
        atomicAdd(&c.s.diag->penalty_net[1], w1);
        atomicAdd(&c.s.diag->penalty_net[2], w2);
      }
    }
  }
  if (valid && (nfl[0] != fl[0] || nfl[1] != fl[1]))
    *reinterpret_cast<uint16_t*>(c.s.flags + cell0) = (uint16_t)(nfl[0] | (nfl[1] << 8));

  // ---- collision (fluid.py:398-413) and AA streaming
  const bool forced = __any_sync(kFull, (fluid0 && (Ax.x != 0.f || Ay.x != 0.f || Az.x != 0.f)) ||
                                           (fluid1 && (Ax.y != 0.f || Ay.y != 0.f || Az.y != 0.f)));
  if (fluid0 || fluid1) {
    if (forced)
      mrt_collide2<true>(F, rho, ux, uy, uz, Ax, Ay, Az, c.K, F);
    else
      mrt_collide2<false>(F, rho, ux, uy, uz, Ax, Ay, Az, c.K, F);
    if (plain) {
      // a solid member of the pair keeps its slots: write the fluid member alone
      const bool both = fluid0 && fluid1;
      if (!ODD) {
#pragma unroll
        for (int s = 0; s < 19; ++s) {
          if (both) {
            Pop2<H>::st(c, kOpp(s), cell0, F[s]);
          } else {
            if (fluid0) stp<H>(c, kOpp(s), cell0, F[s].x);
            if (fluid1) stp<H>(c, kOpp(s), cell0 + 1, F[s].y);
          }
        }
      } else {
        const bool al = c.aligned;
        if (both) {
          Pop2<H>::st(c, 0, cell0, F[0]);
        } else {
          if (fluid0) stp<H>(c, 0, cell0, F[0].x);
          if (fluid1) stp<H>(c, 0, cell0 + 1, F[0].y);
        }
#pragma unroll
        for (int s = 1; s < 19; ++s) {
          if (both && kEx(s) == 0) {
            Pop2<H>::stb(c, s, q.blk(al, 0, 0, kEy(s), kEz(s)), F[s]);
          } else {
            if (fluid0) Pop<H>::stb(c, s, q.blk(al, 0, kEx(s), kEy(s), kEz(s)), F[s].x);
            if (fluid1) Pop<H>::stb(c, s, q.blk(al, 1, kEx(s), kEy(s), kEz(s)), F[s].y);
          }
        }
      }
    } else {
      if (fluid0) {
        if (nb0)
          near_solid_stores2<ODD, H, MOVING, 0>(c, q, cell0, nb0, rho.x, F);
        else if (!ODD) {
#pragma unroll
          for (int s = 0; s < 19; ++s) stp<H>(c, kOpp(s), cell0, F[s].x);
        } else {
          stp<H>(c, 0, cell0, F[0].x);
#pragma unroll
          for (int s = 1; s < 19; ++s) Pop<H>::stb(c, s, q.blk(c.aligned, 0, kEx(s), kEy(s), kEz(s)), F[s].x);
        }
      }
      if (fluid1) {
        if (nb1)
          near_solid_stores2<ODD, H, MOVING, 1>(c, q, cell0 + 1, nb1, rho.y, F);
        else if (!ODD) {
#pragma unroll
          for (int s = 0; s < 19; ++s) stp<H>(c, kOpp(s), cell0 + 1, F[s].y);
        } else {
          stp<H>(c, 0, cell0 + 1, F[0].y);
#pragma unroll
          for (int s = 1; s < 19; ++s) Pop<H>::stb(c, s, q.blk(c.aligned, 1, kEx(s), kEy(s), kEz(s)), F[s].y);
        }
      }
    }
  }
  if (MOVING && valid) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if ((i ? fluid1 : fluid0) || !(fl[i] & kLink)) continue;
      // solid cell receiving link forces: recycle last step's ping-pong slot
      const int cell = cell0 + i;
      float* prev = c.s.hpp + (int64_t)(c.c.pp ^ 1) * 3 * P;
      if (c.c.mode & FSI_MODE_SUBCYCLED) {
        float a[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          a[d] = c.s.accum[d * P + cell] + prev[d * P + cell];
          c.s.accum[d * P + cell] = a[d];
          prev[d * P + cell] = 0.f;
        }
        accum_max_warp(c, sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
      } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) prev[d * P + cell] = 0.f;
      }
    }
  }

  if (dirstats) {
    dirstats_warp2<0>(c, q, fluid0 ? nb0 : 0u, rho.x, F, acc);
    dirstats_warp2<1>(c, q, fluid1 ? nb1 : 0u, rho.y, F, acc);
    __syncthreads();
    if (acc.any) {
      const int tid = threadIdx.y * 32 + lane;
      for (int i = tid; i < 19; i += 128) {
        if (acc.cnt[i]) {
          atomicAdd(&c.s.diag->link_count[i], acc.cnt[i]);
          atomicAdd(&c.s.diag->corr_abs_sum[i], acc.csum[i]);
          atomic_max_nonneg(&c.s.diag->corr_abs_max[i], acc.cmax[i]);
          atomicAdd(&c.s.diag->fluid_impulse[i][0], acc.imp[i][0]);
          atomicAdd(&c.s.diag->fluid_impulse[i][1], acc.imp[i][1]);
          atomicAdd(&c.s.diag->fluid_impulse[i][2], acc.imp[i][2]);
        }
      }
    }
  }
}

template <bool ODD, bool H, bool MOVING, bool BCW, bool PEN>
__global__ void __launch_bounds__(128, 4) k_lbm_step2(const __grid_constant__ Case c) {
  __shared__ DirAcc acc;
  griddep_wait();
  griddep_launch();
  lbm_step_tile2<ODD, H, MOVING, BCW, PEN>(c, blockIdx.x, blockIdx.y, acc);
}

// ------------------------------------------------- init / neighbours ----
__global__ void k_init(const Case c) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t st = c.s.static_solid[i] ? kSolid : 0;
  c.s.flags[i] = st | kOverride;
  c.s.old_solid[i] = st ? 1 : 0;
  c.s.reinit_flag[i] = 0;
  c.s.rho[i] = c.p.rho0;
  for (int a = 0; a < 3; ++a) c.s.vel[(int64_t)a * c.s.pitch + i] = 0.f;
  for (int s = 0; s < 19; ++s) {
    const float fe = feq(s, c.p.rho0, 0.f, 0.f, 0.f);
    if (c.s.store_fp16)
      Pop<true>::st(c, s, i, fe);
    else
      Pop<false>::st(c, s, i, fe);
  }
}

__device__ __forceinline__ void neighbour_data(const Case& c, const Coord& q, uint32_t& mask, bool& any_fluid) {
  mask = 0u;
  any_fluid = false;
#pragma unroll
  for (int s = 1; s < 19; ++s) {
    const int64_t m = nb_cell(c, q, kEx(s), kEy(s), kEz(s));
    if (c.s.flags[m] & kSolid)
      mask |= 1u << s;
    else
      any_fluid = true;
  }
}

__global__ void k_neighbours_all(const Case c) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Coord q{(int)(i % c.s.nx), (int)((i / c.s.nx) % c.s.ny), (int)(i / ((int64_t)c.s.nx * c.s.ny))};
  uint32_t mask;
  bool anyf;
  neighbour_data(c, q, mask, anyf);
  const uint8_t fl = c.s.flags[i];
  const bool solid = fl & kSolid;
  uint8_t nfl = fl & (uint8_t)~(kNear | kLink);
  if (!solid && mask) nfl |= kNear;
  if (solid && anyf) nfl |= kLink;
  c.s.flags[i] = nfl;
  c.s.nbr[i] = mask;
}

__global__ void k_set_solid(const Case c, const uint8_t* solid) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t s = solid[i] ? 1 : 0;
  c.s.flags[i] = (c.s.flags[i] & (uint8_t)~kSolid) | (s ? kSolid : 0);
  c.s.static_solid[i] = s;
  c.s.old_solid[i] = s;
}

// parity 1 -> parity 0: swap the two slots of every fluid-fluid link
template <bool H>
__global__ void k_to_natural(const Case c) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (c.s.flags[i] & kSolid) return;
  const Coord q{(int)(i % c.s.nx), (int)((i / c.s.nx) % c.s.ny), (int)(i / ((int64_t)c.s.nx * c.s.ny))};
#pragma unroll
  for (int s = 1; s < 19; s += 2) {
    const int64_t z = nb_cell(c, q, kEx(s), kEy(s), kEz(s));
    if (c.s.flags[z] & kSolid) continue;
    const float a = Pop<H>::ld_rw(c, s, z);
    const float b = Pop<H>::ld_rw(c, kOpp(s), i);
    Pop<H>::st(c, s, z, b);
    Pop<H>::st(c, kOpp(s), i, a);
  }
}

// ------------------------------------------------------- mask rebuild ----
// update_dynamic_solid (fluid.py:1847-1861) for cell i
__device__ __forceinline__ void mask_update_cell(const Case& c, float thr, int64_t i) {
  const uint8_t fl = c.s.flags[i];
  const uint8_t prev = (fl & kSolid) ? 1 : 0;
  c.s.old_solid[i] = prev;
  const bool dyn = c.s.phi[i] >= thr;
  const uint8_t nw = (c.s.static_solid[i] != 0 || dyn) ? 1 : 0;
  c.s.reinit_flag[i] = (prev && !nw) ? 1 : 0;
  if (nw != prev) {
    c.s.flags[i] = (fl & (uint8_t)~kSolid) | (nw ? kSolid : 0);
    const int slot = atomicAdd(&c.s.diag->change_count, 1);
    c.s.change_list[slot] = (int32_t)i;
  }
}

__global__ void k_mask_update(const Case c, float thr) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mask_update_cell(c, thr, i);
}

__device__ __forceinline__ void flag_bits(uint8_t* flags, int64_t i, uint8_t set, uint8_t clear) {
  uintptr_t addr = reinterpret_cast<uintptr_t>(flags + i);
  unsigned int* word = reinterpret_cast<unsigned int*>(addr & ~(uintptr_t)3);
  const int sh = (int)(addr & 3) * 8;
  if (clear) atomicAnd(word, ~((unsigned int)clear << sh));
  if (set) atomicOr(word, (unsigned int)set << sh);
}

__device__ __forceinline__ Coord coord_of(const Case& c, int64_t i) {
  return Coord{(int)(i % c.s.nx), (int)((i / c.s.nx) % c.s.ny), (int)(i / ((int64_t)c.s.nx * c.s.ny))};
}

__device__ __forceinline__ void reset_velocity(const Case& c, int64_t i, float* u) {
  // reinitialize_new_fluid_cells (fluid.py:1867-1869)
  const int64_t P = c.s.pitch;
  const float a = c.s.svel[i], b = c.s.svel[P + i], d = c.s.svel[2 * P + i];
  if (sqrtf(a * a + b * b + d * d) > 0.f) {
    u[0] = a;
    u[1] = b;
    u[2] = d;
  } else {
    u[0] = u[1] = u[2] = 0.f;
  }
}

__device__ __forceinline__ bool is_changed(const Case& c, int64_t i) {
  return ((c.s.flags[i] & kSolid) ? 1 : 0) != c.s.old_solid[i];
}

// reinitialize_new_fluid_cells (fluid.py:1863-1877) and AA re-pairing of the
// changed cells widx0, widx0 + wstride, ... of the change list, one warp per
// changed cell: lane t < 19 rebuilds the neighbour data of the cell's
// neighbour t (t = 0: the cell), lane s in 1..18 re-pairs the cell's link s
// (the links of one cell hold distinct population slots; a link shared by two
// changed cells is handled by the lower index), lane 0 resets the cell itself.
// The neighbour rebuild only touches NEAR / LINK bits and nbr, which the link
// step does not read, so the lanes need no ordering between the two.
template <bool H>
__device__ __forceinline__ void relink_cells(const Case& c, int widx0, int wstride) {
  const int count = c.s.diag->change_count;
  const int lane = threadIdx.x & 31;
  for (int idx = widx0; idx < count; idx += wstride) {
    const int64_t ci = c.s.change_list[idx];
    const Coord q = coord_of(c, ci);
    if (lane < 19) {
      // neighbour-derived data of ci (lane 0) and its 18 neighbours
      const int t = lane;
      const int64_t m = t == 0 ? ci : nb_cell(c, q, kEx(t), kEy(t), kEz(t));
      const Coord qm = coord_of(c, m);
      uint32_t mask;
      bool anyf;
      neighbour_data(c, qm, mask, anyf);
      const uint8_t fl = c.s.flags[m];
      const bool solid = fl & kSolid;
      const uint8_t want = (uint8_t)((!solid && mask) ? kNear : 0) | (uint8_t)((solid && anyf) ? kLink : 0);
      c.s.nbr[m] = mask;
      const bool link_now = want & kLink;
      if (!link_now || !(fl & kLink)) {
        const int64_t P = c.s.pitch;
        for (int a = 0; a < 6; ++a) c.s.hpp[(int64_t)a * P + m] = 0.f;
      }
      flag_bits(c.s.flags, m, want, (uint8_t)((kNear | kLink) & ~want));
    }
    const bool reinit_c = c.s.reinit_flag[ci] != 0;
    const int s = lane;
    if ((c.c.parity != 0 || reinit_c) && s >= 1 && s < 19) {
      const int64_t z = nb_cell(c, q, kEx(s), kEy(s), kEz(s));
      // a link to another changed cell with a lower index belongs to that cell
      if (!(z != ci && is_changed(c, z) && z < ci)) {
        // canonical orientation: link (y, zz = y + e_sd) with sd odd
        int64_t y, zz;
        int sd;
        if (s & 1) {
          y = ci;
          zz = z;
          sd = s;
        } else {
          y = z;
          zz = ci;
          sd = kOpp(s);
        }
        const bool yf = !(c.s.flags[y] & kSolid), zf = !(c.s.flags[zz] & kSolid);
        if (c.c.parity == 1) {
          const bool old_ff = !c.s.old_solid[y] && !c.s.old_solid[zz];
          const bool new_ff = yf && zf;
          if (old_ff != new_ff) {
            const float a = Pop<H>::ld_rw(c, sd, zz);
            const float b = Pop<H>::ld_rw(c, kOpp(sd), y);
            Pop<H>::st(c, sd, zz, b);
            Pop<H>::st(c, kOpp(sd), y, a);
          }
        }
        if (c.s.reinit_flag[zz]) {
          float u[3];
          reset_velocity(c, zz, u);
          const float v = feq(sd, c.p.rho0, u[0], u[1], u[2]);
          if (c.c.parity == 1 && yf)
            Pop<H>::st(c, kOpp(sd), y, v);
          else
            Pop<H>::st(c, sd, zz, v);
        }
        if (c.s.reinit_flag[y]) {
          float u[3];
          reset_velocity(c, y, u);
          const float v = feq(kOpp(sd), c.p.rho0, u[0], u[1], u[2]);
          if (c.c.parity == 1 && zf)
            Pop<H>::st(c, sd, zz, v);
          else
            Pop<H>::st(c, kOpp(sd), y, v);
        }
      }
    }
    if (reinit_c && lane == 0) {
      float u[3];
      reset_velocity(c, ci, u);
      Pop<H>::st(c, 0, ci, feq(0, c.p.rho0, u[0], u[1], u[2]));
      c.s.rho[ci] = c.p.rho0;
      c.s.vel[ci] = u[0];
      c.s.vel[c.s.pitch + ci] = u[1];
      c.s.vel[2 * c.s.pitch + ci] = u[2];
      flag_bits(c.s.flags, ci, kOverride, 0);
    }
  }
}

template <bool H>
__global__ void k_relink(const Case c) {
  relink_cells<H>(c, (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), (int)((gridDim.x * blockDim.x) >> 5));
}

// reinit flags are consumed only after every link of every changed cell is done
__device__ __forceinline__ void clear_reinit_cells(const Case& c, int idx0, int stride) {
  const int count = c.s.diag->change_count;
  for (int idx = idx0; idx < count; idx += stride) c.s.reinit_flag[c.s.change_list[idx]] = 0;
}

__global__ void k_clear_reinit(const Case c) {
  clear_reinit_cells(c, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------ BC flush and readout ----
template <bool H>
__device__ void face_inputs(const Case& c, int side, int j, int k, FaceIn& in, int& face_x) {
  const int nx = c.s.nx;
  const int row = k * c.s.ny + j;
  
  face_x = side == 0 ? 0 : nx - 1;
  const int x1 = side == 0 ? 1 : nx - 2;
  in.n1_solid = c.s.flags[cell_of(c, x1, j, k)] & kSolid;
  const int ni = in.n1_solid ? face_x : x1;
  const int n2i = in.n1_solid ? face_x : nx - 3;
  in.n2_fluid = !(c.s.flags[cell_of(c, n2i, j, k)] & kSolid);
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    in.Fni[t] = decode_pop<H>(c, Coord{ni, j, k}, (side == 0 ? kUnknownL(t) : kUnknownR(t)));
    in.Fn2[t] = side == 1 ? decode_pop<H>(c, Coord{n2i, j, k}, (side == 0 ? kUnknownL(t) : kUnknownR(t))) : 0.f;
  }
  if (side == 0) {
    load_plane(c, in.n1_solid ? 0 : 1, row, in.mac_n);
    load_plane(c, in.n1_solid ? 1 : 0, row, in.mac_leg);
  } else {
    load_plane(c, in.n1_solid ? 3 : 2, row, in.mac_n);
    load_plane(c, 2, row, in.mac_leg);
  }
}

// applies a pending open-boundary step into the state
template <bool H>
__global__ void k_flush_bc(const Case c) {
  const int nrow = c.s.ny * c.s.nz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  int cnt[5] = {0, 0, 0, 0, 0};
  if (t < 2 * nrow) {
    const int side = t / nrow, row = t % nrow;
    const int bc = side == 0 ? c.p.bc_left : c.p.bc_right;
    const int j = row % c.s.ny, k = row / c.s.ny;
    const int fx = side == 0 ? 0 : c.s.nx - 1;
    const int64_t cell = cell_of(c, fx, j, k);
    const uint8_t fl = c.s.flags[cell];
    if (bc != 0 && !(fl & kSolid)) {
      FaceIn in;
      int face_x;
      face_inputs<H>(c, side, j, k, in, face_x);
      const Coord q{fx, j, k};
      const uint32_t nb = (fl & kNear) ? c.s.nbr[cell] : 0u;
      float F[19];
      int ss[19];
      int64_t sc[19];
#pragma unroll
      for (int s = 0; s < 19; ++s) {
        pop_slot(c, q, cell, fl, nb, s, ss[s], sc[s]);
        F[s] = Pop<H>::ld_rw(c, ss[s], sc[s]);
      }
      apply_face_bc(c.p, c.s.vel_left_dyn, side, in, F, cnt, c.s.diag, c.s.diag, ob_filter_slot(c.s, j, k));
#pragma unroll
      for (int s = 0; s < 19; ++s) Pop<H>::st(c, ss[s], sc[s], F[s]);
    }
  }
  if (c.p.limiter) flush_counts(c, cnt);
}

// The readout state of cell i (what F, rho, v .to_numpy() return): the 19
// populations in natural order with a pending open boundary applied, and the
// macroscopic fields of streaming3 (fluid.py:1794-1814), or the stored ones
// for cells whose collision uses them.  Returns the cell's flags.
template <bool H>
__device__ __forceinline__ uint8_t readout_cell(const Case& c, int64_t i, float F[19], float& rho, float u[3]) {
  const Coord q = coord_of(c, i);
  const uint8_t fl = c.s.flags[i];
  const uint32_t nb = (fl & kNear) ? c.s.nbr[i] : 0u;
#pragma unroll
  for (int s = 0; s < 19; ++s) {
    int ss;
    int64_t sc;
    pop_slot(c, q, i, fl, nb, s, ss, sc);
    F[s] = Pop<H>::ld_rw(c, ss, sc);
  }
  const bool fluid = !(fl & kSolid);
  if (fluid && c.c.bc_pending) {
    int cnt[5] = {0, 0, 0, 0, 0};
    for (int side = 0; side < 2; ++side) {
      const int bc = side == 0 ? c.p.bc_left : c.p.bc_right;
      const int fx = side == 0 ? 0 : c.s.nx - 1;
      if (bc == 0 || q.x != fx) continue;
      FaceIn in;
      int face_x;
      face_inputs<H>(c, side, q.j, q.k, in, face_x);
      apply_face_bc(c.p, c.s.vel_left_dyn, side, in, F, cnt, nullptr, c.s.diag);  // a readout records nothing
    }
  }
  const int64_t P = c.s.pitch;
  rho = c.p.rho0;
  u[0] = u[1] = u[2] = 0.f;
  if (!fluid && (fl & kOverride)) {
    rho = c.s.rho[i];
    for (int a = 0; a < 3; ++a) u[a] = c.s.vel[a * P + i];
  }
  if (fluid) {
    if (fl & kOverride) {
      rho = c.s.rho[i];
      for (int a = 0; a < 3; ++a) u[a] = c.s.vel[a * P + i];
    } else {
      float j[3];
      moments0(F, rho, j[0], j[1], j[2]);
      const float inv = 1.0f / rho;
      for (int a = 0; a < 3; ++a) {
        const float cf = (fl & kCF) ? c.s.cell_force[a * P + i] : 0.f;
        u[a] = j[a] * inv + (0.5f * (c.p.force[a] + cf)) * inv;
      }
    }
  }
  return fl;
}

template <bool H>
__global__ void k_readout(const Case c, float* out_pop, float* out_rho, float* out_vel) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float F[19], rho, u[3];
  readout_cell<H>(c, i, F, rho, u);
  const int64_t P = c.s.pitch;
  for (int s = 0; s < 19; ++s) out_pop[(int64_t)s * P + i] = F[s];
  out_rho[i] = rho;
  for (int a = 0; a < 3; ++a) out_vel[a * P + i] = u[a];
}

// Reductions of the subcycled-flow campaign over the readout state, one pass
// (official_subcycled_flow_solver.py:443-515 computes them in FP64 on host
// copies of rho, v, f and solid): over fluid cells the mass sum(rho), the
// cell count and the counts of cells with a non-finite rho, v or population;
// over the cells of region r (bit r of regions[i], any solid state) the flux
// sum(rho * u_x).  Products and sums in FP64; one atomic per CTA and value.
// The cells come from the lattice state (ARR false: readout of the AA
// layout) or from plain fields in lattice order (ARR true: a snapshot).
struct CampaignArrays {
  const float* rho;       // [n]
  const float* vel;       // [3][n]
  const float* pop;       // [19][n] or null (no population check)
  const uint8_t* solid;   // [n] non-zero: solid
};

template <bool H, bool ARR>
__global__ void __launch_bounds__(256) k_campaign_sums(const Case c, const CampaignArrays a,
                                                       const uint8_t* __restrict__ regions, FsiCampaignSums* out) {
  __shared__ double s_d[8][1 + FSI_CAMPAIGN_REGIONS];
  __shared__ int s_i[8][4];
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  double mass = 0.0, flux[FSI_CAMPAIGN_REGIONS];
#pragma unroll
  for (int r = 0; r < FSI_CAMPAIGN_REGIONS; ++r) flux[r] = 0.0;
  int cells = 0, bad_rho = 0, bad_vel = 0, bad_pop = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float rho, u[3];
    bool solid, pf = true;
    if (ARR) {
      rho = a.rho[i];
      u[0] = a.vel[i];
      u[1] = a.vel[n + i];
      u[2] = a.vel[2 * n + i];
      solid = a.solid[i] != 0;
      if (!solid && a.pop) {
#pragma unroll
        for (int s = 0; s < 19; ++s) pf = pf && isfinite(a.pop[(int64_t)s * n + i]);
      }
    } else {
      float F[19];
      const uint8_t fl = readout_cell<H>(c, i, F, rho, u);
      solid = (fl & kSolid) != 0;
#pragma unroll
      for (int s = 0; s < 19; ++s) pf = pf && isfinite(F[s]);
    }
    if (!solid) {
      ++cells;
      mass += (double)rho;
      bad_rho += isfinite(rho) ? 0 : 1;
      bad_vel += (isfinite(u[0]) && isfinite(u[1]) && isfinite(u[2])) ? 0 : 1;
      bad_pop += pf ? 0 : 1;
    }
    const unsigned rg = regions ? regions[i] : 0u;
    if (rg) {
      const double jx = (double)rho * (double)u[0];
#pragma unroll
      for (int r = 0; r < FSI_CAMPAIGN_REGIONS; ++r)
        if ((rg >> r) & 1u) flux[r] += jx;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  mass = warp_sum_d(mass);
#pragma unroll
  for (int r = 0; r < FSI_CAMPAIGN_REGIONS; ++r) flux[r] = warp_sum_d(flux[r]);
  cells = __reduce_add_sync(0xffffffffu, (unsigned)cells);
  bad_rho = __reduce_add_sync(0xffffffffu, (unsigned)bad_rho);
  bad_vel = __reduce_add_sync(0xffffffffu, (unsigned)bad_vel);
  bad_pop = __reduce_add_sync(0xffffffffu, (unsigned)bad_pop);
  if (lane == 0) {
    s_d[wid][0] = mass;
#pragma unroll
    for (int r = 0; r < FSI_CAMPAIGN_REGIONS; ++r) s_d[wid][1 + r] = flux[r];
    s_i[wid][0] = cells;
    s_i[wid][1] = bad_rho;
    s_i[wid][2] = bad_vel;
    s_i[wid][3] = bad_pop;
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (threadIdx.x < 1 + FSI_CAMPAIGN_REGIONS) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += s_d[w][threadIdx.x];
    double* dst = threadIdx.x == 0 ? &out->fluid_mass : &out->region_flux[threadIdx.x - 1];
    if (v != 0.0) atomicAdd(dst, v);
  } else if (threadIdx.x >= 32 && threadIdx.x < 36) {
    const int k = threadIdx.x - 32;
    int v = 0;
    for (int w = 0; w < nw; ++w) v += s_i[w][k];
    int32_t* dst = k == 0 ? &out->fluid_cells : (k == 1 ? &out->nonfinite_rho : (k == 2 ? &out->nonfinite_vel : &out->nonfinite_pop));
    if (v) atomicAdd(dst, v);
  }
}

// ---- per-x-plane field statistics (sim/diagnostics/lbm_*_diagnostics.py) --
__device__ __forceinline__ uint32_t order_key(float v) {
  const uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// one thread's statistics of the cells of its x plane it visits
struct PlaneAcc {
  double flux, uxs, uxq, rs, rq, spd;
  int fluid, neg, rnan, rnf, vnan, vnf, cnf, rlow, rhigh, vhigh, rlow_first, rhigh_first, vhigh_first, uxnan;
  uint32_t uxmin, uxmax, rmin, rmax, pmin[2], pmax[2];
  int pneg[2], pnf[2];
  float cux;
  int cfl;
};

__device__ __forceinline__ void plane_acc_init(PlaneAcc& a) {
  a.flux = a.uxs = a.uxq = a.rs = a.rq = a.spd = 0.0;
  a.fluid = a.neg = a.rnan = a.rnf = a.vnan = a.vnf = a.cnf = a.rlow = a.rhigh = a.vhigh = a.uxnan = 0;
  a.rlow_first = a.rhigh_first = a.vhigh_first = INT32_MAX;
  a.uxmin = a.rmin = a.pmin[0] = a.pmin[1] = 0xffffffffu;
  a.uxmax = a.rmax = a.pmax[0] = a.pmax[1] = 0u;
  a.pneg[0] = a.pneg[1] = a.pnf[0] = a.pnf[1] = 0;
  a.cux = 0.f;
  a.cfl = -1;
}

__device__ __forceinline__ void plane_acc_pops(PlaneAcc& a, int w, const float* F) {
#pragma unroll
  for (int s = 0; s < 19; ++s) {
    const float v = F[s];
    if (!isnan(v)) {
      a.pmin[w] = min(a.pmin[w], order_key(v));
      a.pmax[w] = max(a.pmax[w], order_key(v));
    }
    a.pneg[w] += v < 0.f ? 1 : 0;
    a.pnf[w] += isfinite(v) ? 0 : 1;
  }
}

// cell (in-plane index jk = j * nz + k) with its rho, v and solid state
__device__ __forceinline__ void plane_acc_cell(PlaneAcc& a, const FsiFieldStatsArgs& g, int jk, bool fluid, float rho,
                                               const float* u) {
  const bool rho_ok = isfinite(rho), vel_ok = isfinite(u[0]) && isfinite(u[1]) && isfinite(u[2]);
  a.cnf += (rho_ok && vel_ok) ? 0 : 1;
  if (!fluid) return;
  ++a.fluid;
  const double r = rho, ux = u[0];
  a.flux += r * ux;
  a.uxs += ux;
  a.uxq += ux * ux;
  a.rs += r;
  a.rq += (r - 1.0) * (r - 1.0);
  a.neg += u[0] < 0.f ? 1 : 0;
  if (!isnan(u[0])) {
    a.uxmin = min(a.uxmin, order_key(u[0]));
    a.uxmax = max(a.uxmax, order_key(u[0]));
  } else {
    ++a.uxnan;
  }
  if (!isnan(rho)) {
    a.rmin = min(a.rmin, order_key(rho));
    a.rmax = max(a.rmax, order_key(rho));
  }
  a.rnan += isnan(rho) ? 1 : 0;
  a.rnf += rho_ok ? 0 : 1;
  const bool vnan = isnan(u[0]) || isnan(u[1]) || isnan(u[2]);
  a.vnan += vnan ? 1 : 0;
  a.vnf += vel_ok ? 0 : 1;
  const double sp = sqrt((double)u[0] * u[0] + (double)u[1] * u[1] + (double)u[2] * u[2]);
  if (!vnan) a.spd = fmax(a.spd, sp);
  if (rho < g.rho_low) {
    ++a.rlow;
    a.rlow_first = min(a.rlow_first, jk);
  }
  if (rho > g.rho_high) {
    ++a.rhigh;
    a.rhigh_first = min(a.rhigh_first, jk);
  }
  if (sp > (double)g.vel_high) {
    ++a.vhigh;
    a.vhigh_first = min(a.vhigh_first, jk);
  }
}

// SRC 0: the state's readout; 1: plain fields in g.  Block (32, 8): lane
// -> x = blockIdx.x * 32 + lane, warps and blockIdx.y stride over the rows
// (j, k); one set of atomics per plane and block.
template <int SRC, bool H>
__global__ void __launch_bounds__(256) k_plane_stats(const Case c, const FsiFieldStatsArgs g, FsiPlaneStats* out) {
  __shared__ PlaneAcc sacc[8][32];
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int nx = c.s.nx, ny = c.s.ny, nz = c.s.nz;
  const int x = blockIdx.x * 32 + lane;
  const int64_t n = (int64_t)nx * ny * nz;
  PlaneAcc a;
  plane_acc_init(a);
  if (x < nx) {
    for (int r = blockIdx.y * 8 + wy; r < ny * nz; r += gridDim.y * 8) {
      const int j = r % ny, k = r / ny;
      const int64_t i = (int64_t)r * nx + x;
      float F[19], rho, u[3];
      bool fluid;
      if (SRC == 0) {
        fluid = !(readout_cell<H>(c, i, F, rho, u) & kSolid);
        plane_acc_pops(a, 0, F);
      } else {
        fluid = g.solid[i] == 0;
        rho = g.rho[i];
#pragma unroll
        for (int d = 0; d < 3; ++d) u[d] = g.vel[d * n + i];
#pragma unroll
        for (int w = 0; w < 2; ++w) {
          const float* src = w ? g.pop_F : g.pop_f;
#pragma unroll
          for (int s = 0; s < 19; ++s) F[s] = src ? src[s * n + i] : 0.f;
          plane_acc_pops(a, w, F);
        }
      }
      plane_acc_cell(a, g, j * nz + k, fluid, rho, u);
      if (j == g.cy && k == g.cz) {
        a.cux = u[0];
        a.cfl = fluid ? 1 : 0;
      }
    }
  }
  sacc[wy][lane] = a;
  __syncthreads();
  if (wy != 0 || x >= nx) return;
  for (int w = 1; w < 8; ++w) {
    const PlaneAcc& b = sacc[w][lane];
    a.flux += b.flux;
    a.uxs += b.uxs;
    a.uxq += b.uxq;
    a.rs += b.rs;
    a.rq += b.rq;
    a.spd = fmax(a.spd, b.spd);
    a.fluid += b.fluid;
    a.neg += b.neg;
    a.rnan += b.rnan;
    a.rnf += b.rnf;
    a.vnan += b.vnan;
    a.vnf += b.vnf;
    a.cnf += b.cnf;
    a.rlow += b.rlow;
    a.rhigh += b.rhigh;
    a.vhigh += b.vhigh;
    a.uxnan += b.uxnan;
    a.rlow_first = min(a.rlow_first, b.rlow_first);
    a.rhigh_first = min(a.rhigh_first, b.rhigh_first);
    a.vhigh_first = min(a.vhigh_first, b.vhigh_first);
    a.uxmin = min(a.uxmin, b.uxmin);
    a.uxmax = max(a.uxmax, b.uxmax);
    a.rmin = min(a.rmin, b.rmin);
    a.rmax = max(a.rmax, b.rmax);
    for (int q = 0; q < 2; ++q) {
      a.pmin[q] = min(a.pmin[q], b.pmin[q]);
      a.pmax[q] = max(a.pmax[q], b.pmax[q]);
      a.pneg[q] += b.pneg[q];
      a.pnf[q] += b.pnf[q];
    }
    if (b.cfl >= 0) {
      a.cux = b.cux;
      a.cfl = b.cfl;
    }
  }
  if (SRC == 0) {  // f and F are one array in the readout
    a.pmin[1] = a.pmin[0];
    a.pmax[1] = a.pmax[0];
    a.pneg[1] = a.pneg[0];
    a.pnf[1] = a.pnf[0];
  }
  FsiPlaneStats* o = out + x;
  auto addd = [](double* p, double v) {
    if (v != 0.0) atomicAdd(p, v);
  };
  auto addi = [](int32_t* p, int v) {
    if (v) atomicAdd(p, v);
  };
  addd(&o->flux, a.flux);
  addd(&o->ux_sum, a.uxs);
  addd(&o->ux_sq, a.uxq);
  addd(&o->rho_sum, a.rs);
  addd(&o->rho_sq, a.rq);
  if (a.spd > 0.0) atomicMax(reinterpret_cast<unsigned long long*>(&o->speed_max), (unsigned long long)__double_as_longlong(a.spd));
  addi(&o->fluid_cells, a.fluid);
  addi(&o->ux_negative, a.neg);
  addi(&o->rho_nan, a.rnan);
  addi(&o->rho_nonfinite, a.rnf);
  addi(&o->vel_nan, a.vnan);
  addi(&o->vel_nonfinite, a.vnf);
  addi(&o->cell_nonfinite, a.cnf);
  addi(&o->rho_low, a.rlow);
  addi(&o->rho_high, a.rhigh);
  addi(&o->vel_high, a.vhigh);
  addi(&o->ux_nan, a.uxnan);
  if (a.rlow_first != INT32_MAX) atomicMin(&o->rho_low_first, a.rlow_first);
  if (a.rhigh_first != INT32_MAX) atomicMin(&o->rho_high_first, a.rhigh_first);
  if (a.vhigh_first != INT32_MAX) atomicMin(&o->vel_high_first, a.vhigh_first);
  if (a.uxmin != 0xffffffffu) atomicMin(&o->ux_min, a.uxmin);
  if (a.uxmax) atomicMax(&o->ux_max, a.uxmax);
  if (a.rmin != 0xffffffffu) atomicMin(&o->rho_min, a.rmin);
  if (a.rmax) atomicMax(&o->rho_max, a.rmax);
  for (int q = 0; q < 2; ++q) {
    if (a.pmin[q] != 0xffffffffu) atomicMin(&o->pop_min[q], a.pmin[q]);
    if (a.pmax[q]) atomicMax(&o->pop_max[q], a.pmax[q]);
    addi(&o->pop_negative[q], a.pneg[q]);
    addi(&o->pop_nonfinite[q], a.pnf[q]);
  }
  if (a.cfl >= 0) {  // the one block holding (cy, cz) of this plane
    o->center_ux = a.cux;
    o->center_fluid = a.cfl;
  }
}

__global__ void k_plane_stats_init(FsiPlaneStats* out, int nx) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nx) return;
  FsiPlaneStats z{};
  z.ux_min = z.rho_min = z.pop_min[0] = z.pop_min[1] = 0xffffffffu;
  z.rho_low_first = z.rho_high_first = z.vel_high_first = INT32_MAX;
  out[x] = z;
}

// ---- wall velocity application to solid_vel (wall_velocity/application.py:118-158)
__device__ __forceinline__ void atomic_max_dnonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// |a| as numpy's norm computes it: products and sums rounded one by one (no
// fused multiply-add), so caps and norms match the reference bit for bit
__device__ __forceinline__ double norm3_rn(const double* a) {
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(a[0], a[0]), __dmul_rn(a[1], a[1])), __dmul_rn(a[2], a[2])));
}

__global__ void __launch_bounds__(256) k_wall_velocity(const Case c, const double* __restrict__ grid, int additive,
                                                       double cap, FsiWallVelocityStats* out) {
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz, P = c.s.pitch;
  double dmax = 0.0, dsum = 0.0, bmax = 0.0, amax = 0.0, aamax = 0.0, aasum = 0.0;
  int applied = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double b[3], g[3], a[3], e[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      b[d] = (double)c.s.svel[d * P + i];
      g[d] = grid[d * P + i];
      a[d] = b[d];
    }
    const double bn = norm3_rn(b);
    bmax = fmax(bmax, bn);
    if (norm3_rn(g) > 0.0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) a[d] = additive ? __dadd_rn(b[d], g[d]) : g[d];
      const double an = norm3_rn(a);
      if (an > cap) {
        const double sc = __ddiv_rn(cap, an);
#pragma unroll
        for (int d = 0; d < 3; ++d) a[d] = __dmul_rn(a[d], sc);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        c.s.svel[d * P + i] = (float)a[d];
        e[d] = __dsub_rn(a[d], b[d]);
      }
      const double dn = norm3_rn(e), an2 = norm3_rn(a);
      ++applied;
      dmax = fmax(dmax, dn);
      dsum += dn;
      aamax = fmax(aamax, an2);
      aasum += an2;
      amax = fmax(amax, an2);
    } else {
      amax = fmax(amax, bn);
    }
  }
  dsum = warp_sum_d(dsum);
  aasum = warp_sum_d(aasum);
  applied = (int)__reduce_add_sync(0xffffffffu, (unsigned)applied);
  for (int o = 16; o > 0; o >>= 1) {
    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    aamax = fmax(aamax, __shfl_xor_sync(0xffffffffu, aamax, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (applied) {
      atomicAdd(&out->applied_cells, applied);
      atomicAdd(&out->delta_norm_sum, dsum);
      atomicAdd(&out->after_norm_sum_active, aasum);
      atomic_max_dnonneg(&out->delta_norm_max, dmax);
      atomic_max_dnonneg(&out->after_norm_max_active, aamax);
    }
    atomic_max_dnonneg(&out->before_norm_max, bmax);
    atomic_max_dnonneg(&out->after_norm_max, amax);
  }
}

// finalize_moving_boundary_force_accumulator (fluid.py:475-486), grid-stride
// over the cells; the two norm maxima are reduced over the CTA and added with
// one atomic each per CTA (one per warp contended on the two addresses)
__global__ void k_accum_finalize(const Case c, int32_t sample_count) {
  __shared__ float s_max[2][32];
  const int64_t n = (int64_t)c.s.nx * c.s.ny * c.s.nz;
  const int64_t P = c.s.pitch;
  float mean_max = 0.f, acc_max = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float a[3];
    for (int d = 0; d < 3; ++d) a[d] = c.s.accum[d * P + i];
    if ((c.c.mode & FSI_MODE_SUBCYCLED) && (c.s.flags[i] & kLink)) {
      float* last = c.s.hpp + (int64_t)c.c.pp * 3 * P;
      for (int d = 0; d < 3; ++d) {
        a[d] += last[d * P + i];
        last[d * P + i] = 0.f;
        c.s.accum[d * P + i] = a[d];
      }
      acc_max = fmaxf(acc_max, sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]));
    }
    if (sample_count > 0) {
      const float inv = 1.0f / (float)sample_count;
      float m[3];
      for (int d = 0; d < 3; ++d) {
        m[d] = a[d] * inv;
        c.s.hydro[d * P + i] = m[d];
      }
      mean_max = fmaxf(mean_max, sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]));
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  mean_max = warp_max(mean_max);
  acc_max = warp_max(acc_max);
  if (lane == 0) {
    s_max[0][wid] = mean_max;
    s_max[1][wid] = acc_max;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float m0 = 0.f, m1 = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      m0 = fmaxf(m0, s_max[0][w]);
      m1 = fmaxf(m1, s_max[1][w]);
    }
    if (m0 > 0.f) atomic_max_nonneg(&c.s.diag->mean_norm_max, m0);
    if (m1 > 0.f) atomic_max_nonneg(&c.s.diag->accum_norm_max, m1);
  }
}

// ------------------------------------------------------------- host ABI ----
static int check_state(const FsiLbmState* s, const FsiLbmParams* p) {
  if (!s || !p) return invalid("null state or params");
  if (s->nx < 3 || s->ny < 1 || s->nz < 1) return invalid("lattice must have nx >= 3, ny >= 1, nz >= 1");
  if (s->pitch < (int64_t)s->nx * s->ny * s->nz || (s->pitch % 32) != 0)
    return invalid("pitch must cover nx*ny*nz and be a multiple of 32");
  if (19 * s->pitch > (int64_t)UINT32_MAX) return invalid("lattice too large: 19 * pitch must be below 2^32");
  if (p->tune < FSI_TUNE_LBM_OCC3 || p->tune > FSI_TUNE_LBM_OCC4_PF) return invalid("unknown FsiLbmParams.tune");
  if (p->ob_semantics < FSI_OB_EQUILIBRIUM_RESET || p->ob_semantics > FSI_OB_CONV_PLANE_FLUX)
    return invalid("unknown FsiLbmParams.ob_semantics");
  if (p->ob_measure_offset < 0) return invalid("ob_measure_offset must be >= 0");
  if ((p->bc_left || p->bc_right) && (s->nx < 4 || (s->nx % 32 == 1) || (s->nx % 32 == 2)))
    return invalid("x open boundaries need nx >= 4 and nx % 32 not in {1, 2}");
  if (!s->pop || !s->flags || !s->nbr || !s->diag) return invalid("null device pointer in FsiLbmState");
  if ((p->bc_left || p->bc_right || p->ob_semantics >= FSI_OB_REG_PLANE_FLUX) && !s->plane)
    return invalid("open boundaries and the outlet flux controller need FsiLbmState.plane");
  return FSI_OK;
}

// the paired kernel needs x-adjacent cell pairs aligned (nx even) and, with
// open boundaries, the three cells next to the x = nx - 1 face in one warp
static bool pair_ok(const FsiLbmState* s, const FsiLbmParams* p) {
  if (s->nx % 2) return false;
  if ((p->bc_left || p->bc_right) && (s->nx % 64 == 2 || s->nx < 4)) return false;
  return true;
}

static Case make_case(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl) {
  Case c;
  c.s = *s;
  c.p = *p;
  if (ctl)
    c.c = *ctl;
  else
    c.c = FsiStepCtl{0, 0, 0, 0};
  c.K = make_mrt_k(p->s_v, p->s_o);
  c.pf_dist = 0;
  c.aligned = (s->nx % 32) == 0;
  return c;
}

static int lbm_sm_count() { return device_sm_count(); }

static inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace fsi

using namespace fsi;

extern "C" int fsi_lbm_init_equilibrium(const FsiLbmState* s, const FsiLbmParams* p, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const Case c = make_case(s, p, nullptr);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_init<<<blocks_for(n, 256), 256, 0, st>>>(c);
  if ((rc = launch_check("k_init"))) return rc;
  k_neighbours_all<<<blocks_for(n, 256), 256, 0, st>>>(c);
  return launch_check("k_neighbours_all");
}

extern "C" int fsi_lbm_set_solid(const FsiLbmState* s, const uint8_t* solid, void* stream) {
  if (!s || !solid) return invalid("null argument");
  cudaStream_t st = (cudaStream_t)stream;
  FsiLbmParams p{};
  p.rho0 = 1.f;
  p.s_v = p.s_o = 1.f;
  const Case c = make_case(s, &p, nullptr);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_set_solid<<<blocks_for(n, 256), 256, 0, st>>>(c, solid);
  int rc = launch_check("k_set_solid");
  if (rc) return rc;
  k_neighbours_all<<<blocks_for(n, 256), 256, 0, st>>>(c);
  return launch_check("k_neighbours_all");
}

extern "C" int fsi_lbm_to_natural(const FsiLbmState* s, void* stream) {
  if (!s) return invalid("null state");
  if (19 * s->pitch > (int64_t)UINT32_MAX) return invalid("lattice too large: 19 * pitch must be below 2^32");
  FsiLbmParams p{};
  p.rho0 = 1.f;
  p.s_v = p.s_o = 1.f;
  const Case c = make_case(s, &p, nullptr);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  if (s->store_fp16)
    k_to_natural<true><<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(c);
  else
    k_to_natural<false><<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(c);
  return launch_check("k_to_natural");
}

// After each step, before its (pending) open boundary is applied: the clear
// of the repair step counters (clear_open_boundary_limiter_step_counters,
// fluid.py:571-586) and, under semantics 8 and 9, the outlet flux controller
// update_open_boundary_plane_flux_controller (fluid.py:1141-1263) from the
// plane sums the step accumulated in pc_acc, which it then zeroes.
// step_clear = 0, run = 1: a controller update on its own (the reference's
// kernel called directly), which clears no step counter of its own.
// compose: first fold the flow-filter composites the last open-boundary
// application left in the outlet row slots (semantics 6, 7) into
// flow_outlet_flux_error_filtered_run, in row order, and clear the slots.
// One block of kObThreads threads.
constexpr int kObThreads = 1024;

__global__ void __launch_bounds__(kObThreads) k_ob_controller(const FsiLbmState st, const FsiLbmParams p,
                                                              int step_clear, int run, int compose) {
  FsiLbmDiag* d = st.diag;
  if (compose) {
    __shared__ float sd[kObThreads], sb[kObThreads];
    const int n = st.ny * st.nz;
    const int per = (n + kObThreads - 1) / kObThreads;
    const int t = threadIdx.x;
    float* slots = ob_filter_slot(st, 0, 0);
    float cd = 0.f, cb = 0.f;
    for (int i = t * per; i < min(n, (t + 1) * per); ++i) {
      ob_filter_then(cd, cb, slots[2 * i], slots[2 * i + 1]);
      slots[2 * i] = 0.f;
      slots[2 * i + 1] = 0.f;
    }
    sd[t] = cd;
    sb[t] = cb;
    __syncthreads();
    for (int w = 1; w < kObThreads; w *= 2) {  // ordered tree: left part first
      if ((t % (2 * w)) == 0) {
        float ld = sd[t], lb = sb[t];
        ob_filter_then(ld, lb, sd[t + w], sb[t + w]);
        sd[t] = ld;
        sb[t] = lb;
      }
      __syncthreads();
    }
    if (t == 0 && sd[0] != 0.f) d->obf_err_filtered_run = (1.0f - sd[0]) * d->obf_err_filtered_run + sb[0];
  }
  if (threadIdx.x != 0) return;
  if (step_clear) {
    d->obr_count_step = 0;
    d->obr_corr_step = 0.f;
    d->obr_delta_step = 0.f;
    d->obf_delta_step = 0.f;
    d->obf_gain_step = 0.f;
    d->pc_update_step = d->pc_sat_step = 0;
    d->mn_update_step = d->mn_sat_step = 0;
  }
  if (!run) return;
  d->pc_guard_step = 0;
  d->pc_guard_ref = 0.f;
  const float target = p.ob_target_scale * d->pc_acc[0];
  const float measured = d->pc_acc[1];
  float area = d->pc_acc[2];
  if (area <= 0.f) area = 1.f;
  d->pc_target = target;
  d->pc_measured = measured;
  d->pc_area = area;
  d->pc_true_outlet = d->pc_acc[3];
  d->pc_near[0] = d->pc_acc[4];
  d->pc_near[1] = d->pc_acc[5];
  d->pc_near[2] = d->pc_acc[6];
  const float filtered = (1.0f - p.ob_filter_alpha) * d->pc_err_filtered + p.ob_filter_alpha * (target - measured);
  d->pc_err_filtered = filtered;
  d->obf_err_filtered_run = filtered;
  const float requested = p.ob_gain_u * filtered / area;
  const float bounded = ob_bounded(requested, p.ob_cap_u);
  const float previous = d->pc_u_fb;
  float limited = bounded;
  if (p.ob_delta_cap_u > 0.f) limited = previous + ob_bounded(bounded - previous, p.ob_delta_cap_u);
  float next = previous + p.ob_slew_alpha * (limited - previous);
  if (p.ob_guard) {  // outlet flux drop guard
    const float reference = fmaxf(fabsf(target), fabsf(measured));
    d->pc_guard_ref = reference;
    if (reference > 1.0e-12f && fabsf(d->pc_true_outlet) < p.ob_guard_min_ratio * reference && next < previous) {
      next = previous;
      d->pc_guard_step = 1;
      d->pc_guard_run += 1;
    }
  }
  d->pc_u_fb = next;
  d->pc_rho_fb = ob_bounded(p.ob_gain_rho * filtered / area, 0.01f);
  if (p.ob_mass_neutral) {  // global_mass_error_density_offset
    const float mass = (float)d->mn_mass_acc;
    d->mn_mass_acc = 0.0;
    d->mn_mass = mass;
    if (d->mn_initialized == 0) {
      d->mn_reference = fabsf(mass) <= 1.0e-12f ? 1.0f : mass;
      d->mn_initialized = 1;
    }
    float reference = d->mn_reference;
    if (fabsf(reference) <= 1.0e-12f) {
      reference = 1.0f;
      d->mn_reference = reference;
    }
    const float err = (mass - reference) / reference;
    const float raw = -p.ob_mn_gain * err;
    const float bm = ob_bounded(raw, p.ob_mn_cap);
    d->mn_error = err;
    d->mn_rho_fb = p.ob_mn_blend * bm;
    d->mn_update_step = 1;
    d->mn_update_run += 1;
    if (fabsf(raw - bm) > 1.0e-12f) {
      d->mn_sat_step = 1;
      d->mn_sat_run += 1;
    }
  }
  d->obf_gain_step = p.ob_gain_u;
  d->pc_update_step = 1;
  d->pc_update_run += 1;
  if (fabsf(requested - bounded) > 1.0e-12f) {
    d->pc_sat_step = 1;
    d->pc_sat_run += 1;
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) d->pc_acc[a] = 0.f;
}

// plane sums of the controller from given macroscopic fields (lattice order,
// vel as three planes of pitch entries), for a controller update on its own
__global__ void __launch_bounds__(256) k_plane_flux_sums(const Case c, const float* __restrict__ rho,
                                                         const float* __restrict__ vel) {
  const int nx = c.s.nx;
  const int64_t n = (int64_t)nx * c.s.ny * c.s.nz;
  float t[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  double mass = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool fluid = !(c.s.flags[i] & kSolid);
    t[7] = 0.f;
    plane_flux_add(c, (int)(i % nx), fluid, rho[i], vel[i], t);
    mass += (double)t[7];
  }
#pragma unroll
  for (int a = 0; a < 7; ++a) {
    const float v = warp_sum(t[a]);
    if ((threadIdx.x & 31) == 0 && v != 0.f) atomicAdd(&c.s.diag->pc_acc[a], v);
  }
  mass = warp_sum_d(mass);
  if ((threadIdx.x & 31) == 0 && mass != 0.0) atomicAdd(&c.s.diag->mn_mass_acc, mass);
}

extern "C" int fsi_ob_controller_update(const FsiLbmState* s, const FsiLbmParams* p, const float* rho,
                                        const float* vel, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!rho || !vel) return invalid("null rho or vel");
  cudaStream_t st = (cudaStream_t)stream;
  const Case c = make_case(s, p, nullptr);
  if ((rc = cuda_check(cudaMemsetAsync(s->diag->pc_acc, 0, sizeof(s->diag->pc_acc), st), "memset pc_acc")))
    return rc;
  if ((rc = cuda_check(cudaMemsetAsync(&s->diag->mn_mass_acc, 0, sizeof(double), st), "memset mn_mass_acc")))
    return rc;
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  const int blocks = (int)std::min<int64_t>(blocks_for(n, 256), 4LL * lbm_sm_count());
  k_plane_flux_sums<<<blocks, 256, 0, st>>>(c, rho, vel);
  if ((rc = launch_check("k_plane_flux_sums"))) return rc;
  k_ob_controller<<<1, 32, 0, st>>>(*s, *p, 0, 1, 0);
  return launch_check("k_ob_controller");
}

extern "C" int fsi_lbm_substep(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl) return invalid("null step control");
  cudaStream_t st = (cudaStream_t)stream;
  bool memset_before = false;
  if (ctl->bc_pending && p->limiter) {
    rc = cuda_check(cudaMemsetAsync(s->diag->ob_step, 0, sizeof(s->diag->ob_step), st), "memset ob_step");
    if (rc) return rc;
    memset_before = true;
  }
  if ((ctl->mode & FSI_MODE_DIRSTATS) && (ctl->mode & FSI_MODE_MOVING_BB)) {
    rc = cuda_check(cudaMemsetAsync(s->diag, 0, offsetof(FsiLbmDiag, accum_norm_max), st), "memset dirstats");
    if (rc) return rc;
    memset_before = true;
  }
  if (ctl->mode & FSI_MODE_PENALTY) {
    memset_before = true;
    rc = cuda_check(cudaMemsetAsync(&s->diag->penalty_active, 0,
                                    offsetof(FsiLbmDiag, change_count) - offsetof(FsiLbmDiag, penalty_active), st),
                    "memset penalty stats");
    if (rc) return rc;
  }
  Case c = make_case(s, p, ctl);
  dim3 block(32, 8);
  dim3 grid((unsigned)((s->nx + 31) / 32), (unsigned)((s->ny + 7) / 8), (unsigned)s->nz);
  if (p->tune == FSI_TUNE_LBM_OCC3_PF || p->tune == FSI_TUNE_LBM_OCC4_PF)
    c.pf_dist = lbm_sm_count() * (p->tune == FSI_TUNE_LBM_OCC4_PF ? 4 : 3);
  const bool odd = ctl->parity != 0, h = s->store_fp16 != 0;
  const bool moving = ctl->mode & FSI_MODE_MOVING_BB, pen = ctl->mode & FSI_MODE_PENALTY;
  const bool bcw = p->bc_left != 0 || p->bc_right != 0 || p->ob_semantics >= FSI_OB_REG_PLANE_FLUX;
  if (moving && pen) return invalid("penalty steps use static bounce-back (fluid.py:2099-2103)");
  const dim3 grid2((unsigned)((s->nx + 63) / 64), (unsigned)((s->ny * s->nz + 3) / 4));
  const dim3 block2(32, 4);
  if (p->tune == FSI_TUNE_LBM_PAIR && !pair_ok(s, p)) return invalid("FSI_TUNE_LBM_PAIR needs an even nx (and nx % 64 != 2 with open boundaries)");
  // back-to-back steps overlap the launch of the next with the tail of the
  // previous (programmatic dependent launch) unless a memset came in between
  const bool pdl = !memset_before;
  cudaError_t lerr = cudaSuccess;
#define FSI_KLAUNCH(K, G, BL)                          \
  if (pdl)                                             \
    lerr = launch_pdl(K, G, BL, 0, st, c);             \
  else                                                 \
    K<<<G, BL, 0, st>>>(c)
#define FSI_LAUNCH(O, HH, M, B, PN)                                        \
  if (p->tune == FSI_TUNE_LBM_PAIR) {                                      \
    FSI_KLAUNCH((k_lbm_step2<O, HH, M, B, PN>), grid2, block2);            \
  } else if (p->tune == FSI_TUNE_LBM_OCC4) {                               \
    FSI_KLAUNCH((k_lbm_step<O, HH, M, B, PN, 4, false>), grid, block);     \
  } else if (p->tune == FSI_TUNE_LBM_OCC4_PF) {                            \
    FSI_KLAUNCH((k_lbm_step<O, HH, M, B, PN, 4, true>), grid, block);      \
  } else if (p->tune == FSI_TUNE_LBM_OCC3_PF) {                            \
    FSI_KLAUNCH((k_lbm_step<O, HH, M, B, PN, 3, true>), grid, block);      \
  } else {                                                                 \
    FSI_KLAUNCH((k_lbm_step<O, HH, M, B, PN, 3, false>), grid, block);     \
  }
#define FSI_BY_H(O, M, B, PN) \
  if (h) { FSI_LAUNCH(O, true, M, B, PN); } else { FSI_LAUNCH(O, false, M, B, PN); }
#define FSI_BY_O(M, B, PN) \
  if (odd) { FSI_BY_H(true, M, B, PN); } else { FSI_BY_H(false, M, B, PN); }
  if (moving) {
    if (bcw) { FSI_BY_O(true, true, false) } else { FSI_BY_O(true, false, false) }
  } else if (pen) {
    if (bcw) { FSI_BY_O(false, true, true) } else { FSI_BY_O(false, false, true) }
  } else {
    if (bcw) { FSI_BY_O(false, true, false) } else { FSI_BY_O(false, false, false) }
  }
#undef FSI_BY_O
#undef FSI_BY_H
#undef FSI_LAUNCH
#undef FSI_KLAUNCH
  if ((rc = cuda_check(lerr, "k_lbm_step (launch)"))) return rc;
  if ((rc = launch_check("k_lbm_step"))) return rc;
  if (p->ob_semantics >= FSI_OB_REG_MASS_BALANCED) {
    const int compose = p->ob_semantics == FSI_OB_REG_FLUX_MATCHED || p->ob_semantics == FSI_OB_CONV_FLUX_MATCHED;
    k_ob_controller<<<1, compose ? kObThreads : 32, 0, st>>>(*s, *p, 1, p->ob_semantics >= FSI_OB_REG_PLANE_FLUX,
                                                            compose);
    return launch_check("k_ob_controller");
  }
  return FSI_OK;
}

extern "C" int fsi_lbm_flush_bc(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl) return invalid("null step control");
  if (!ctl->bc_pending || (!p->bc_left && !p->bc_right)) return FSI_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (p->limiter) {
    rc = cuda_check(cudaMemsetAsync(s->diag->ob_step, 0, sizeof(s->diag->ob_step), st), "memset ob_step");
    if (rc) return rc;
  }
  const Case c = make_case(s, p, ctl);
  const int64_t n = 2LL * s->ny * s->nz;
  if (s->store_fp16)
    k_flush_bc<true><<<blocks_for(n, 128), 128, 0, st>>>(c);
  else
    k_flush_bc<false><<<blocks_for(n, 128), 128, 0, st>>>(c);
  if ((rc = launch_check("k_flush_bc"))) return rc;
  if (p->ob_semantics == FSI_OB_REG_FLUX_MATCHED || p->ob_semantics == FSI_OB_CONV_FLUX_MATCHED) {
    k_ob_controller<<<1, kObThreads, 0, st>>>(*s, *p, 0, 0, 1);
    return launch_check("k_ob_controller");
  }
  return FSI_OK;
}

extern "C" int fsi_mask_rebuild(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, float threshold,
                                void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl) return invalid("null step control");
  if (!s->change_list || !s->phi || !s->static_solid || !s->old_solid || !s->reinit_flag)
    return invalid("mask rebuild needs phi, static_solid, old_solid, reinit_flag and change_list");
  cudaStream_t st = (cudaStream_t)stream;
  rc = cuda_check(cudaMemsetAsync(&s->diag->change_count, 0, sizeof(int32_t), st), "memset change_count");
  if (rc) return rc;
  const Case c = make_case(s, p, ctl);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_mask_update<<<blocks_for(n, 256), 256, 0, st>>>(c, threshold);
  if ((rc = launch_check("k_mask_update"))) return rc;
  const unsigned g = (unsigned)lbm_sm_count() * 4;
  if (s->store_fp16)
    k_relink<true><<<g, 128, 0, st>>>(c);
  else
    k_relink<false><<<g, 128, 0, st>>>(c);
  if ((rc = launch_check("k_relink"))) return rc;
  k_clear_reinit<<<g, 128, 0, st>>>(c);
  return launch_check("k_clear_reinit");
}

extern "C" int fsi_force_accum_finalize(const FsiLbmState* s, const FsiStepCtl* ctl, int32_t sample_count,
                                        void* stream) {
  if (!s || !ctl) return invalid("null argument");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = cuda_check(cudaMemsetAsync(&s->diag->mean_norm_max, 0, sizeof(float), st), "memset mean_norm_max");
  if (rc) return rc;
  FsiLbmParams p{};
  p.rho0 = 1.f;
  p.s_v = p.s_o = 1.f;
  const Case c = make_case(s, &p, ctl);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  k_accum_finalize<<<(unsigned)std::min<int64_t>(blocks_for(n, 256), (int64_t)lbm_sm_count() * 8), 256, 0, st>>>(
      c, sample_count);
  return launch_check("k_accum_finalize");
}

extern "C" int fsi_lbm_readout(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl, float* out_pop,
                               float* out_rho, float* out_vel, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl || !out_pop || !out_rho || !out_vel) return invalid("null argument");
  const Case c = make_case(s, p, ctl);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  if (s->store_fp16)
    k_readout<true><<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(c, out_pop, out_rho, out_vel);
  else
    k_readout<false><<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(c, out_pop, out_rho, out_vel);
  return launch_check("k_readout");
}

extern "C" int fsi_campaign_sums(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl,
                                 const uint8_t* regions, FsiCampaignSums* out, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl || !out) return invalid("null step control or output");
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = cuda_check(cudaMemsetAsync(out, 0, sizeof(FsiCampaignSums), st), "memset campaign sums"))) return rc;
  const Case c = make_case(s, p, ctl);
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  const unsigned blocks = (unsigned)std::min<int64_t>(blocks_for(n, 256), (int64_t)lbm_sm_count() * 8);
  if (s->store_fp16)
    k_campaign_sums<true, false><<<blocks, 256, 0, st>>>(c, CampaignArrays{}, regions, out);
  else
    k_campaign_sums<false, false><<<blocks, 256, 0, st>>>(c, CampaignArrays{}, regions, out);
  return launch_check("k_campaign_sums");
}

extern "C" int fsi_campaign_sums_arrays(int32_t nx, int32_t ny, int32_t nz, const float* rho, const float* vel,
                                        const float* pop, const uint8_t* solid, const uint8_t* regions,
                                        FsiCampaignSums* out, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0) return invalid("lattice dimensions must be positive");
  if (!rho || !vel || !solid || !out) return invalid("null field or output");
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if ((rc = cuda_check(cudaMemsetAsync(out, 0, sizeof(FsiCampaignSums), st), "memset campaign sums"))) return rc;
  Case c{};
  c.s.nx = nx;
  c.s.ny = ny;
  c.s.nz = nz;
  const int64_t n = (int64_t)nx * ny * nz;
  const unsigned blocks = (unsigned)std::min<int64_t>(blocks_for(n, 256), (int64_t)lbm_sm_count() * 8);
  k_campaign_sums<false, true><<<blocks, 256, 0, st>>>(c, CampaignArrays{rho, vel, pop, solid}, regions, out);
  return launch_check("k_campaign_sums");
}

static int plane_stats_launch(const Case& c, const FsiFieldStatsArgs* a, FsiPlaneStats* planes, bool arrays,
                              cudaStream_t st) {
  const int nx = c.s.nx, rows = c.s.ny * c.s.nz;
  if (a->cy < 0 || a->cy >= c.s.ny || a->cz < 0 || a->cz >= c.s.nz) return invalid("centerline cell out of range");
  k_plane_stats_init<<<(nx + 127) / 128, 128, 0, st>>>(planes, nx);
  int rc = launch_check("k_plane_stats_init");
  if (rc) return rc;
  const int xt = (nx + 31) / 32;
  const int gy = std::max(1, std::min((rows + 7) / 8, 2 * lbm_sm_count() / xt));
  const dim3 grid((unsigned)xt, (unsigned)gy), block(32, 8);
  if (arrays)
    k_plane_stats<1, false><<<grid, block, 0, st>>>(c, *a, planes);
  else if (c.s.store_fp16)
    k_plane_stats<0, true><<<grid, block, 0, st>>>(c, *a, planes);
  else
    k_plane_stats<0, false><<<grid, block, 0, st>>>(c, *a, planes);
  return launch_check("k_plane_stats");
}

extern "C" int fsi_lbm_field_stats(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl,
                                   const FsiFieldStatsArgs* a, FsiPlaneStats* planes, void* stream) {
  int rc = check_state(s, p);
  if (rc) return rc;
  if (!ctl || !a || !planes) return invalid("null step control, arguments or output");
  return plane_stats_launch(make_case(s, p, ctl), a, planes, false, (cudaStream_t)stream);
}

extern "C" int fsi_field_stats_arrays(int32_t nx, int32_t ny, int32_t nz, const FsiFieldStatsArgs* a,
                                      FsiPlaneStats* planes, void* stream) {
  if (nx < 1 || ny < 1 || nz < 1) return invalid("lattice extents must be positive");
  if ((int64_t)ny * nz > INT32_MAX / 2 || 19 * (int64_t)nx * ny * nz > INT64_MAX / 4) return invalid("lattice too large");
  if (!a || !planes || !a->rho || !a->vel || !a->solid) return invalid("null rho, vel, solid or output");
  Case c{};
  c.s.nx = nx;
  c.s.ny = ny;
  c.s.nz = nz;
  return plane_stats_launch(c, a, planes, true, (cudaStream_t)stream);
}

extern "C" int fsi_apply_wall_velocity(const FsiLbmState* s, const double* grid, int32_t policy, double cap,
                                       FsiWallVelocityStats* out, void* stream) {
  if (!s || !grid || !out || !s->svel) return invalid("null state, grid, solid_vel or output");
  if (policy != FSI_WALL_REPLACE && policy != FSI_WALL_ADDITIVE) return invalid("unknown wall velocity policy");
  if (!(cap > 0.0)) return invalid("wall velocity cap must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = cuda_check(cudaMemsetAsync(out, 0, sizeof(FsiWallVelocityStats), st), "memset wall velocity stats");
  if (rc) return rc;
  Case c{};
  c.s = *s;
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  const unsigned blocks = (unsigned)std::min<int64_t>(blocks_for(n, 256), (int64_t)lbm_sm_count() * 8);
  k_wall_velocity<<<blocks, 256, 0, st>>>(c, grid, policy == FSI_WALL_ADDITIVE, cap, out);
  return launch_check("k_wall_velocity");
}

// ---- mask rebuild with a built-in change list ----------------------------
// fsi_mask_rebuild needs a pitch-sized int32 scratch (FsiLbmState.change_list)
// to list the cells whose solid bit flipped.  Some callers hold the lattice
// state but have no way to hand over another device buffer: a foreign-language
// host that received the state's buffers from elsewhere and owns no device
// allocator, or code running where allocating is not allowed.  For them the
// list lives in this file-scope array, sized for lattices of up to
// kStaticChangeCap cells (4 MiB of device memory per device that loads the
// library).  Its contents need no initial value: the count of listed cells is
// diag->change_count, which every call zeroes before use.
namespace fsi {
constexpr int64_t kStaticChangeCap = int64_t(1) << 20;
constexpr int kStaticScratchDevices = 64;
static __device__ __align__(256) int32_t g_change_scratch[kStaticChangeCap];

// address of g_change_scratch on the current device, looked up once per device
static int static_change_scratch(int32_t** out) {
  static std::mutex mu;
  static int32_t* addr[kStaticScratchDevices] = {};
  int dev = 0;
  int rc = cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= kStaticScratchDevices) return invalid("device ordinal out of range for the built-in scratch");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    rc = cuda_check(cudaGetSymbolAddress(&p, g_change_scratch), "cudaGetSymbolAddress(change-list scratch)");
    if (rc) return rc;
    addr[dev] = static_cast<int32_t*>(p);
  }
  *out = addr[dev];
  return FSI_OK;
}
}  // namespace fsi

extern "C" int fsi_mask_rebuild_static_scratch(const FsiLbmState* s, const FsiLbmParams* p, const FsiStepCtl* ctl,
                                               float threshold, void* stream) {
  if (!s) return invalid("null state");
  const int64_t n = (int64_t)s->nx * s->ny * s->nz;
  if (n > kStaticChangeCap)
    return invalid("lattice of " + std::to_string(n) + " cells exceeds the built-in change list of " +
                   std::to_string(kStaticChangeCap) + " cells; use fsi_mask_rebuild with a caller-provided change_list");
  int32_t* scratch = nullptr;
  const int rc = static_change_scratch(&scratch);
  if (rc) return rc;
  FsiLbmState local = *s;
  local.change_list = scratch;
  return fsi_mask_rebuild(&local, p, ctl, threshold, stream);
}

// ---- batched cases ---------------------------------------------------------
// grid.y = case slot; grid.x strides over the case's work.  Each CTA stages
// its case's lattice descriptors in shared memory once.
namespace fsi {

__device__ __forceinline__ void copy_words(void* dst, const void* src, int bytes, int tid, int nt) {
  const int* s = static_cast<const int*>(src);
  int* d = static_cast<int*>(dst);
  for (int i = tid; i < bytes / 4; i += nt) d[i] = s[i];
}

// stage the lattice part of a batch case (state, params, step control, and the
// MRT rates when with_k) in shared memory; returns false for an inactive slot
__device__ __forceinline__ bool stage_case(const FsiBatchCase& bc, Case& sc, bool with_k) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x, nt = blockDim.x * blockDim.y;
  if (!bc.active) return false;  // same value for every thread of the CTA
  copy_words(&sc.s, &bc.lbm, (int)sizeof(FsiLbmState), tid, nt);
  copy_words(&sc.p, &bc.lp, (int)sizeof(FsiLbmParams), tid, nt);
  copy_words(&sc.c, &bc.ctl, (int)sizeof(FsiStepCtl), tid, nt);
  if (with_k && tid == 0) {
    sc.K = make_mrt_k(bc.lp.s_v, bc.lp.s_o);
    sc.pf_dist = 0;
  }
  if (tid == 0) sc.aligned = (bc.lbm.nx % 32) == 0;
  __syncthreads();
  return true;
}

template <bool H>
__global__ void __launch_bounds__(256, 3) k_batch_lbm_step(const FsiBatchCase* __restrict__ cases) {
  __shared__ Case sc;
  __shared__ DirAcc acc;
  const FsiBatchCase& bc = cases[blockIdx.y];
  const int gx = (bc.lbm.nx + 31) / 32, gy = (bc.lbm.ny + 7) / 8, nt = gx * gy * bc.lbm.nz;
  if ((int)blockIdx.x >= nt || !stage_case(bc, sc, true)) return;
  const bool moving = sc.c.mode & FSI_MODE_MOVING_BB;
  const bool odd = sc.c.parity != 0;
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    const int r = t / gx, bx = t - r * gx, by = r % gy, bz = r / gy;
    if (moving) {
      if (odd)
        lbm_step_tile<true, H, true, false, false>(sc, bx, by, bz, acc);
      else
        lbm_step_tile<false, H, true, false, false>(sc, bx, by, bz, acc);
    } else {
      if (odd)
        lbm_step_tile<true, H, false, false, true>(sc, bx, by, bz, acc);
      else
        lbm_step_tile<false, H, false, false, true>(sc, bx, by, bz, acc);
    }
    __syncthreads();  // acc is reused by the next tile
  }
}

// the same with two cells per thread (lbm_step_tile2): tiles of 64 x 4 cells
template <bool H>
__global__ void __launch_bounds__(128, 4) k_batch_lbm_step2(const FsiBatchCase* __restrict__ cases) {
  __shared__ Case sc;
  __shared__ DirAcc acc;
  const FsiBatchCase& bc = cases[blockIdx.y];
  const int gx = (bc.lbm.nx + 63) / 64, nt = gx * ((bc.lbm.ny * bc.lbm.nz + 3) / 4);
  if ((int)blockIdx.x >= nt || !stage_case(bc, sc, true)) return;
  const bool moving = sc.c.mode & FSI_MODE_MOVING_BB;
  const bool odd = sc.c.parity != 0;
  for (int t = blockIdx.x; t < nt; t += gridDim.x) {
    const int bx = t % gx, by = t / gx;
    if (moving) {
      if (odd)
        lbm_step_tile2<true, H, true, false, false>(sc, bx, by, acc);
      else
        lbm_step_tile2<false, H, true, false, false>(sc, bx, by, acc);
    } else {
      if (odd)
        lbm_step_tile2<true, H, false, false, true>(sc, bx, by, acc);
      else
        lbm_step_tile2<false, H, false, false, true>(sc, bx, by, acc);
    }
    __syncthreads();  // acc is reused by the next tile
  }
}

__global__ void k_batch_mask_update(const FsiBatchCase* __restrict__ cases) {
  __shared__ Case sc;
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (bc.mode != FSI_BATCH_MOVING) return;
  const int64_t n = (int64_t)bc.lbm.nx * bc.lbm.ny * bc.lbm.nz;
  if ((int64_t)blockIdx.x * blockDim.x >= n || !stage_case(bc, sc, false)) return;
  const float thr = bc.mask_threshold;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    mask_update_cell(sc, thr, i);
}

template <bool H>
__global__ void k_batch_relink(const FsiBatchCase* __restrict__ cases) {
  __shared__ Case sc;
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (bc.mode != FSI_BATCH_MOVING || !stage_case(bc, sc, false)) return;
  relink_cells<H>(sc, (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), (int)((gridDim.x * blockDim.x) >> 5));
}

__global__ void k_batch_clear_reinit(const FsiBatchCase* __restrict__ cases) {
  __shared__ Case sc;
  const FsiBatchCase& bc = cases[blockIdx.y];
  if (bc.mode != FSI_BATCH_MOVING || !stage_case(bc, sc, false)) return;
  clear_reinit_cells(sc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// per-case bookkeeping between phases (one CTA of 32 threads per case)
enum { kBatchLbmPre = 1, kBatchLbmPost = 2, kBatchMaskPre = 3 };

__global__ void k_batch_ctl(FsiBatchCase* cases, int op) {
  FsiBatchCase& bc = cases[blockIdx.x];
  if (!bc.active) return;
  const int tid = threadIdx.x;
  FsiLbmDiag* d = bc.lbm.diag;
  if (op == kBatchLbmPre) {
    // the reductions fsi_lbm_substep zeroes before a step of this mode
    int* w = reinterpret_cast<int*>(d);
    if (bc.ctl.mode & FSI_MODE_MOVING_BB) {
      for (int i = tid; i < (int)(offsetof(FsiLbmDiag, accum_norm_max) / 4); i += blockDim.x) w[i] = 0;
    } else if (bc.ctl.mode & FSI_MODE_PENALTY) {
      const int a = (int)(offsetof(FsiLbmDiag, penalty_active) / 4), b = (int)(offsetof(FsiLbmDiag, change_count) / 4);
      for (int i = a + tid; i < b; i += blockDim.x) w[i] = 0;
    }
  } else if (op == kBatchLbmPost && tid == 0) {
    bc.ctl.parity ^= 1;
    bc.ctl.pp ^= 1;
  } else if (op == kBatchMaskPre && tid == 0) {
    d->change_count = 0;
  }
}

int check_batch(const FsiBatchCase* cases, const FsiBatchDims* d) {
  if (!cases || !d) return invalid("null batch argument");
  if (d->n_cases <= 0 || d->n_cases > 65535) return invalid("n_cases must be in 1..65535");
  if (d->max_lbm_tiles <= 0 || d->max_cells <= 0) return invalid("batch dims must be positive");
  if (d->lbm_tune != FSI_TUNE_LBM_OCC3 && d->lbm_tune != FSI_TUNE_LBM_PAIR)
    return invalid("FsiBatchDims.lbm_tune must be FSI_TUNE_LBM_OCC3 or FSI_TUNE_LBM_PAIR (every case nx even)");
  return FSI_OK;
}

static inline unsigned batch_x(int64_t work, int threads, int cap) {
  const int64_t b = (work + threads - 1) / threads;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

}  // namespace fsi

extern "C" int fsi_batch_lbm_substep(FsiBatchCase* cases, const FsiBatchDims* d, void* stream) {
  int rc = check_batch(cases, d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  k_batch_ctl<<<d->n_cases, 32, 0, st>>>(cases, kBatchLbmPre);
  if ((rc = launch_check("k_batch_ctl"))) return rc;
  // one CTA per tile of the largest case; CTAs past a smaller case's tiles exit at once
  if (d->lbm_tune == FSI_TUNE_LBM_PAIR) {
    // max_lbm_tiles counts 32 x 8 x 1 tiles; a 64 x 4 tile covers as many cells
    const dim3 grid(batch_x((int64_t)d->max_lbm_tiles + 64, 1, 1 << 20), d->n_cases);
    if (d->store_fp16)
      k_batch_lbm_step2<true><<<grid, dim3(32, 4), 0, st>>>(cases);
    else
      k_batch_lbm_step2<false><<<grid, dim3(32, 4), 0, st>>>(cases);
  } else {
    const dim3 grid(batch_x(d->max_lbm_tiles, 1, 1 << 20), d->n_cases);
    if (d->store_fp16)
      k_batch_lbm_step<true><<<grid, dim3(32, 8), 0, st>>>(cases);
    else
      k_batch_lbm_step<false><<<grid, dim3(32, 8), 0, st>>>(cases);
  }
  if ((rc = launch_check("k_batch_lbm_step"))) return rc;
  k_batch_ctl<<<d->n_cases, 32, 0, st>>>(cases, kBatchLbmPost);
  return launch_check("k_batch_ctl");
}

extern "C" int fsi_batch_mask_rebuild(FsiBatchCase* cases, const FsiBatchDims* d, void* stream) {
  int rc = check_batch(cases, d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  k_batch_ctl<<<d->n_cases, 32, 0, st>>>(cases, kBatchMaskPre);
  if ((rc = launch_check("k_batch_ctl"))) return rc;
  k_batch_mask_update<<<dim3(batch_x(d->max_cells, 256, 1 << 20), d->n_cases), 256, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_mask_update"))) return rc;
  const dim3 g2(std::max(1, lbm_sm_count() * 4 / std::max(1, d->n_cases)), d->n_cases);
  if (d->store_fp16)
    k_batch_relink<true><<<g2, 128, 0, st>>>(cases);
  else
    k_batch_relink<false><<<g2, 128, 0, st>>>(cases);
  if ((rc = launch_check("k_batch_relink"))) return rc;
  k_batch_clear_reinit<<<g2, 128, 0, st>>>(cases);
  return launch_check("k_batch_clear_reinit");
}

// D3Q19 lattice and the reference's MRT collision, restructured for few flops.
//
// The reference collides with dense 19x19 products (src/mpm_lbm/sim/lbm/
// fluid.py:398-413):
//     m  = M F;  m -= S (m - meq(rho,u));  m += (1 - S/2) M g;  f = M^-1 m
// with the integer moment matrix M (fluid.py:257-275), relaxation rates S
// (fluid.py:301-304), the reference's own moment equilibrium meq
// (fluid.py:385-391) and Guo forcing g (fluid.py:405-410, including its /3 and
// /9 factors).  Algebraically the same operator is
//     f = F + g - M^T K (M h - meq),   h = F + g/2,   K = (M M^T)^-1 S,
// because M^-1 = M^T (M M^T)^-1 and the Gram matrix M M^T of this M is block
// diagonal (one 3x3 block {0,1,2}, 2x2 blocks {3,4} {5,6} {7,8} {9,10}
// {11,12}, scalars 13..18).  With opposite directions paired, M h and M^T y
// become short add chains: ~330 flops per cell instead of ~2000.
//
// The header compiles as CUDA and as host C++ (tests check the host build of
// these exact functions against the CPU oracle).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define FSI_HD __host__ __device__ __forceinline__
#else
#define FSI_HD inline
#endif

namespace fsi {

// velocity set in the reference's order (fluid.py:359-363); direction 2p-1 and
// 2p are opposite for p = 1..9.
constexpr int kQ = 19;
// velocity components of direction s as bit masks (+1 set, -1 set), so that
// the same constexpr lookup works in host and device code
FSI_HD constexpr int kEx(int s) { return ((0x2a82 >> s) & 1) - ((0x5504 >> s) & 1); }
FSI_HD constexpr int kEy(int s) { return ((0x28488 >> s) & 1) - ((0x50310 >> s) & 1); }
FSI_HD constexpr int kEz(int s) { return ((0x4c820 >> s) & 1) - ((0x33040 >> s) & 1); }
FSI_HD constexpr int kOpp(int s) { return s == 0 ? 0 : ((s & 1) ? s + 1 : s - 1); }

FSI_HD float lattice_w(int s) { return s == 0 ? (1.0f / 3.0f) : (s <= 6 ? (1.0f / 18.0f) : (1.0f / 36.0f)); }

// Non-zero entries of K = (M M^T)^-1 S.  Column 0/3/5/7 of K vanish (S = 0 on
// the conserved moments), so only these remain.
struct MrtK {
  float k01, k02, k11, k12, k21, k22;  // block {0,1,2}, columns 1 and 2
  float kq0, kq1;                      // blocks {3,4} {5,6} {7,8}: column 4/6/8
  float ka, kb;                        // block {9,10}
  float kc, kd;                        // block {11,12}
  float ke;                            // 13, 14, 15
  float kf;                            // 16, 17, 18
};

FSI_HD MrtK make_mrt_k(float s_v, float s_o) {
  // K = (M M^T)^-1 S on the non-zero blocks (see d3q19.cuh); Gram blocks of the
  // reference's M (fluid.py:257-275): {0,1,2}: [[19,11,1],[11,13,11],[1,11,37]],
  // {3,4}: [[10,4],[4,16]], {9,10}: [[36,12],[12,36]], {11,12}: [[12,4],[4,12]],
  // 13..15: 4, 16..18: 8.
  const double G[3][3] = {{19, 11, 1}, {11, 13, 11}, {1, 11, 37}};
  double inv[3][3];
  const double det = G[0][0] * (G[1][1] * G[2][2] - G[1][2] * G[2][1]) - G[0][1] * (G[1][0] * G[2][2] - G[1][2] * G[2][0]) +
                     G[0][2] * (G[1][0] * G[2][1] - G[1][1] * G[2][0]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
      inv[i][j] = (G[r0][c0] * G[r1][c1] - G[r0][c1] * G[r1][c0]) / det;
    }
  MrtK K;
  K.k01 = (float)(inv[0][1] * s_v);
  K.k02 = (float)(inv[0][2] * s_v);
  K.k11 = (float)(inv[1][1] * s_v);
  K.k12 = (float)(inv[1][2] * s_v);
  K.k21 = (float)(inv[2][1] * s_v);
  K.k22 = (float)(inv[2][2] * s_v);
  const double dq = 10.0 * 16.0 - 16.0;  // det [[10,4],[4,16]]
  K.kq0 = (float)((-4.0 / dq) * s_o);
  K.kq1 = (float)((10.0 / dq) * s_o);
  const double d9 = 36.0 * 36.0 - 144.0;
  K.ka = (float)((36.0 / d9) * s_v);
  K.kb = (float)((-12.0 / d9) * s_v);
  const double d11 = 144.0 - 16.0;
  K.kc = (float)((12.0 / d11) * s_v);
  K.kd = (float)((-4.0 / d11) * s_v);
  K.ke = (float)(s_v / 4.0);
  K.kf = (float)(s_o / 8.0);
  return K;
}

// Reference equilibrium (fluid.py:320-326); w * rho * (1 + 3 eu + 4.5 eu^2 - 1.5 u.u)
FSI_HD float feq(int s, float rho, float ux, float uy, float uz) {
  const float eu = (float)kEx(s) * ux + (float)kEy(s) * uy + (float)kEz(s) * uz;
  const float uv = ux * ux + uy * uy + uz * uz;
  return lattice_w(s) * rho * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * uv);
}

// Density and raw momentum of 19 populations.
FSI_HD void moments0(const float* F, float& rho, float& jx, float& jy, float& jz) {
  float s[10], d[10];
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    s[p] = F[2 * p - 1] + F[2 * p];
    d[p] = F[2 * p - 1] - F[2 * p];
  }
  rho = F[0] + ((s[1] + s[2]) + (s[3] + s[4])) + ((s[5] + s[6]) + (s[7] + s[8])) + s[9];
  jx = d[1] + (d[4] + d[5]) + (d[6] + d[7]);
  jy = d[2] + (d[4] - d[5]) + (d[8] + d[9]);
  jz = d[3] + (d[6] - d[7]) + (d[8] - d[9]);
}

// One MRT collision with Guo forcing.  F: post-streaming populations; (rho,u):
// the macroscopic state the reference collides with (streaming3 output,
// fluid.py:1799-1810); (Ax,Ay,Az): body force + cell force (fluid.py:393-396).
// Writes the post-collision populations to out (may alias F).
// FORCED = false: the caller knows Ax = Ay = Az = 0, so the Guo term vanishes
// (g = 0, h = F) and is not evaluated.
template <bool FORCED = true>
FSI_HD void mrt_collide(const float* F, float rho, float ux, float uy, float uz, float Ax, float Ay, float Az,
                        const MrtK& K, float* out) {
  // Guo term, paired: g_a = P + Q, g_b = P - Q
  float g[19];
  if (FORCED) {
    const float uA = ux * Ax + uy * Ay + uz * Az;
    const float eA[10] = {0.f, Ax, Ay, Az, Ax + Ay, Ax - Ay, Ax + Az, Ax - Az, Ay + Az, Ay - Az};
    const float eU[10] = {0.f, ux, uy, uz, ux + uy, ux - uy, ux + uz, ux - uz, uy + uz, uy - uz};
    g[0] = (-1.0f / 9.0f) * uA;  // w0 * (-uA/3)
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      const float w = p <= 3 ? (1.0f / 18.0f) : (1.0f / 36.0f);
      const float P = w * ((eU[p] * eA[p]) * (1.0f / 9.0f) - uA * (1.0f / 3.0f));
      const float Q = w * (1.0f / 3.0f) * eA[p];
      g[2 * p - 1] = P + Q;
      g[2 * p] = P - Q;
    }
  }
  // h = F + g/2 and its non-conserved moments
  float h[19];
#pragma unroll
  for (int s = 0; s < 19; ++s) h[s] = FORCED ? F[s] + 0.5f * g[s] : F[s];
  float sg[10], dl[10];
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    sg[p] = h[2 * p - 1] + h[2 * p];
    dl[p] = h[2 * p - 1] - h[2 * p];
  }
  const float Sa = sg[1] + sg[2] + sg[3];
  const float Sxy = sg[4] + sg[5], Sxz = sg[6] + sg[7], Syz = sg[8] + sg[9];
  const float Sd = Sxy + Sxz + Syz;
  const float uu = ux * ux + uy * uy + uz * uz;
  const float r1 = (Sd - h[0]) - uu;
  const float r2 = h[0] - 2.0f * Sa + Sd;
  const float r4 = (dl[4] + dl[5] + dl[6] + dl[7]) - 2.0f * dl[1];
  const float r6 = (dl[4] - dl[5] + dl[8] + dl[9]) - 2.0f * dl[2];
  const float r8 = (dl[6] - dl[7] + dl[8] - dl[9]) - 2.0f * dl[3];
  const float U = 2.0f * sg[1] - sg[2] - sg[3];
  const float T = Sxy + Sxz - 2.0f * Syz;
  const float r9 = (U + T) - (2.0f * ux * ux - uy * uy - uz * uz);
  const float r10 = T - U;
  const float V = sg[2] - sg[3], Wq = Sxy - Sxz;
  const float r11 = (V + Wq) - (uy * uy - uz * uz);
  const float r12 = Wq - V;
  const float r13 = (sg[4] - sg[5]) - ux * uy;
  const float r14 = (sg[8] - sg[9]) - uy * uz;
  const float r15 = (sg[6] - sg[7]) - ux * uz;
  const float r16 = dl[4] + dl[5] - dl[6] - dl[7];
  const float r17 = dl[5] - dl[4] + dl[8] + dl[9];
  const float r18 = dl[6] - dl[7] - dl[8] + dl[9];
  // y = K r
  const float y0 = K.k01 * r1 + K.k02 * r2;
  const float y1 = K.k11 * r1 + K.k12 * r2;
  const float y2 = K.k21 * r1 + K.k22 * r2;
  const float y3 = K.kq0 * r4, y4 = K.kq1 * r4;
  const float y5 = K.kq0 * r6, y6 = K.kq1 * r6;
  const float y7 = K.kq0 * r8, y8 = K.kq1 * r8;
  const float y9 = K.ka * r9 + K.kb * r10, y10 = K.kb * r9 + K.ka * r10;
  const float y11 = K.kc * r11 + K.kd * r12, y12 = K.kd * r11 + K.kc * r12;
  const float y13 = K.ke * r13, y14 = K.ke * r14, y15 = K.ke * r15;
  const float y16 = K.kf * r16, y17 = K.kf * r17, y18 = K.kf * r18;
  // f = F + g - M^T y, paired: f_a = F_a + g_a - (E + O), f_b = F_b + g_b - (E - O)
  const float Y012 = y0 + y1 + y2, B = y0 - 2.0f * y2;
  const float d910 = y9 - y10, s910 = y9 + y10, d1112 = y11 - y12, s1112 = y11 + y12;
  const float q34 = y3 + y4, q56 = y5 + y6, q78 = y7 + y8;
  float Ev[10], Ov[10];
  Ev[1] = B + 2.0f * d910;
  Ov[1] = y3 - 2.0f * y4;
  Ev[2] = B - d910 + d1112;
  Ov[2] = y5 - 2.0f * y6;
  Ev[3] = B - d910 - d1112;
  Ov[3] = y7 - 2.0f * y8;
  const float P45 = Y012 + s910 + s1112, P67 = Y012 + s910 - s1112, P89 = Y012 - 2.0f * s910;
  Ev[4] = P45 + y13;
  Ov[4] = q34 + q56 + y16 - y17;
  Ev[5] = P45 - y13;
  Ov[5] = q34 - q56 + y16 + y17;
  Ev[6] = P67 + y15;
  Ov[6] = q34 + q78 - y16 + y18;
  Ev[7] = P67 - y15;
  Ov[7] = q34 - q78 - y16 - y18;
  Ev[8] = P89 + y14;
  Ov[8] = q56 + q78 + y17 - y18;
  Ev[9] = P89 - y14;
  Ov[9] = q56 - q78 + y17 + y18;
  out[0] = (FORCED ? F[0] + g[0] : F[0]) - (y0 - y1 + y2);
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    const float a = FORCED ? F[2 * p - 1] + g[2 * p - 1] : F[2 * p - 1];
    const float b = FORCED ? F[2 * p] + g[2 * p] : F[2 * p];
    out[2 * p - 1] = a - (Ev[p] + Ov[p]);
    out[2 * p] = b - (Ev[p] - Ov[p]);
  }
}

}  // namespace fsi

#if defined(__CUDACC__)
#include <cuda_runtime.h>
namespace fsi {

// ---- paired form: two cells per thread on the sm_100 paired FP32 pipe ----
// The same operator as mrt_collide, for the populations of two cells held as
// (cell 0, cell 1) pairs, each operation one paired FP32 instruction.
__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b, exact as a subtraction: fma(b, -1, a) rounds once
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

__device__ __forceinline__ void moments0_2(const float2* F, float2& rho, float2& jx, float2& jy, float2& jz) {
  float2 s[10], d[10];
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    s[p] = add2(F[2 * p - 1], F[2 * p]);
    d[p] = sub2(F[2 * p - 1], F[2 * p]);
  }
  rho = add2(add2(F[0], add2(add2(s[1], s[2]), add2(s[3], s[4]))), add2(add2(add2(s[5], s[6]), add2(s[7], s[8])), s[9]));
  jx = add2(add2(d[1], add2(d[4], d[5])), add2(d[6], d[7]));
  jy = add2(add2(d[2], sub2(d[4], d[5])), add2(d[8], d[9]));
  jz = add2(add2(d[3], sub2(d[6], d[7])), sub2(d[8], d[9]));
}

// FORCED = false: the caller knows the force vanishes for both cells (g = 0)
template <bool FORCED = true>
__device__ __forceinline__ void mrt_collide2(const float2* F, float2 rho, float2 ux, float2 uy, float2 uz, float2 Ax,
                                             float2 Ay, float2 Az, const MrtK& K, float2* out) {
  (void)rho;
  // Fg = F + g (kept), and h = F + g/2 reduced at once to its pair sums / differences
  float2 Fg[19];
  float2 sg[10], dl[10];
  float2 h0;
  if (FORCED) {
    // Guo term, paired over directions: g_a = P + Q, g_b = P - Q
    const float2 uA = fma2(uz, Az, fma2(uy, Ay, mul2(ux, Ax)));
    const float2 eA[10] = {p2(0.f), Ax, Ay, Az, add2(Ax, Ay), sub2(Ax, Ay), add2(Ax, Az), sub2(Ax, Az), add2(Ay, Az),
                           sub2(Ay, Az)};
    const float2 eU[10] = {p2(0.f), ux, uy, uz, add2(ux, uy), sub2(ux, uy), add2(ux, uz), sub2(ux, uz), add2(uy, uz),
                           sub2(uy, uz)};
    const float2 uA3 = mul2(uA, p2(1.0f / 3.0f));
    Fg[0] = add2(F[0], mul2(p2(-1.0f / 9.0f), uA));
    h0 = fma2(p2(-1.0f / 18.0f), uA, F[0]);
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      const float w = p <= 3 ? (1.0f / 18.0f) : (1.0f / 36.0f);
      const float2 P = mul2(p2(w), sub2(mul2(mul2(eU[p], eA[p]), p2(1.0f / 9.0f)), uA3));
      const float2 Q = mul2(p2(w * (1.0f / 3.0f)), eA[p]);
      const float2 ga = add2(P, Q), gb = sub2(P, Q);
      Fg[2 * p - 1] = add2(F[2 * p - 1], ga);
      Fg[2 * p] = add2(F[2 * p], gb);
      const float2 ha = fma2(p2(0.5f), ga, F[2 * p - 1]);
      const float2 hb = fma2(p2(0.5f), gb, F[2 * p]);
      sg[p] = add2(ha, hb);
      dl[p] = sub2(ha, hb);
    }
  } else {
    Fg[0] = F[0];
    h0 = F[0];
#pragma unroll
    for (int p = 1; p <= 9; ++p) {
      Fg[2 * p - 1] = F[2 * p - 1];
      Fg[2 * p] = F[2 * p];
      sg[p] = add2(F[2 * p - 1], F[2 * p]);
      dl[p] = sub2(F[2 * p - 1], F[2 * p]);
    }
  }
  const float2 Sa = add2(add2(sg[1], sg[2]), sg[3]);
  const float2 Sxy = add2(sg[4], sg[5]), Sxz = add2(sg[6], sg[7]), Syz = add2(sg[8], sg[9]);
  const float2 Sd = add2(add2(Sxy, Sxz), Syz);
  const float2 uu = fma2(uz, uz, fma2(uy, uy, mul2(ux, ux)));
  const float2 r1 = sub2(sub2(Sd, h0), uu);
  const float2 r2 = add2(fma2(p2(-2.0f), Sa, h0), Sd);
  const float2 r4 = fma2(p2(-2.0f), dl[1], add2(add2(dl[4], dl[5]), add2(dl[6], dl[7])));
  const float2 r6 = fma2(p2(-2.0f), dl[2], add2(sub2(dl[4], dl[5]), add2(dl[8], dl[9])));
  const float2 r8 = fma2(p2(-2.0f), dl[3], add2(sub2(dl[6], dl[7]), sub2(dl[8], dl[9])));
  const float2 U = sub2(sub2(mul2(p2(2.0f), sg[1]), sg[2]), sg[3]);
  const float2 T = fma2(p2(-2.0f), Syz, add2(Sxy, Sxz));
  const float2 r9 = sub2(add2(U, T), sub2(sub2(mul2(p2(2.0f), mul2(ux, ux)), mul2(uy, uy)), mul2(uz, uz)));
  const float2 r10 = sub2(T, U);
  const float2 V = sub2(sg[2], sg[3]), Wq = sub2(Sxy, Sxz);
  const float2 r11 = sub2(add2(V, Wq), sub2(mul2(uy, uy), mul2(uz, uz)));
  const float2 r12 = sub2(Wq, V);
  const float2 r13 = sub2(sub2(sg[4], sg[5]), mul2(ux, uy));
  const float2 r14 = sub2(sub2(sg[8], sg[9]), mul2(uy, uz));
  const float2 r15 = sub2(sub2(sg[6], sg[7]), mul2(ux, uz));
  const float2 r16 = sub2(sub2(add2(dl[4], dl[5]), dl[6]), dl[7]);
  const float2 r17 = add2(add2(sub2(dl[5], dl[4]), dl[8]), dl[9]);
  const float2 r18 = add2(sub2(sub2(dl[6], dl[7]), dl[8]), dl[9]);
  // y = K r
  const float2 y0 = fma2(p2(K.k02), r2, mul2(p2(K.k01), r1));
  const float2 y1 = fma2(p2(K.k12), r2, mul2(p2(K.k11), r1));
  const float2 y2 = fma2(p2(K.k22), r2, mul2(p2(K.k21), r1));
  const float2 y3 = mul2(p2(K.kq0), r4), y4 = mul2(p2(K.kq1), r4);
  const float2 y5 = mul2(p2(K.kq0), r6), y6 = mul2(p2(K.kq1), r6);
  const float2 y7 = mul2(p2(K.kq0), r8), y8 = mul2(p2(K.kq1), r8);
  const float2 y9 = fma2(p2(K.kb), r10, mul2(p2(K.ka), r9)), y10 = fma2(p2(K.ka), r10, mul2(p2(K.kb), r9));
  const float2 y11 = fma2(p2(K.kd), r12, mul2(p2(K.kc), r11)), y12 = fma2(p2(K.kc), r12, mul2(p2(K.kd), r11));
  const float2 y13 = mul2(p2(K.ke), r13), y14 = mul2(p2(K.ke), r14), y15 = mul2(p2(K.ke), r15);
  const float2 y16 = mul2(p2(K.kf), r16), y17 = mul2(p2(K.kf), r17), y18 = mul2(p2(K.kf), r18);
  // f = F + g - M^T y, paired: f_a = Fg_a - (E + O), f_b = Fg_b - (E - O)
  const float2 Y012 = add2(add2(y0, y1), y2), B = fma2(p2(-2.0f), y2, y0);
  const float2 d910 = sub2(y9, y10), s910 = add2(y9, y10), d1112 = sub2(y11, y12), s1112 = add2(y11, y12);
  const float2 q34 = add2(y3, y4), q56 = add2(y5, y6), q78 = add2(y7, y8);
  float2 Ev[10], Ov[10];
  Ev[1] = fma2(p2(2.0f), d910, B);
  Ov[1] = fma2(p2(-2.0f), y4, y3);
  Ev[2] = add2(sub2(B, d910), d1112);
  Ov[2] = fma2(p2(-2.0f), y6, y5);
  Ev[3] = sub2(sub2(B, d910), d1112);
  Ov[3] = fma2(p2(-2.0f), y8, y7);
  const float2 P45 = add2(add2(Y012, s910), s1112), P67 = sub2(add2(Y012, s910), s1112);
  const float2 P89 = fma2(p2(-2.0f), s910, Y012);
  Ev[4] = add2(P45, y13);
  Ov[4] = sub2(add2(add2(q34, q56), y16), y17);
  Ev[5] = sub2(P45, y13);
  Ov[5] = add2(add2(sub2(q34, q56), y16), y17);
  Ev[6] = add2(P67, y15);
  Ov[6] = add2(sub2(add2(q34, q78), y16), y18);
  Ev[7] = sub2(P67, y15);
  Ov[7] = sub2(sub2(sub2(q34, q78), y16), y18);
  Ev[8] = add2(P89, y14);
  Ov[8] = sub2(add2(add2(q56, q78), y17), y18);
  Ev[9] = sub2(P89, y14);
  Ov[9] = add2(add2(sub2(q56, q78), y17), y18);
  out[0] = sub2(Fg[0], add2(sub2(y0, y1), y2));
#pragma unroll
  for (int p = 1; p <= 9; ++p) {
    out[2 * p - 1] = sub2(Fg[2 * p - 1], add2(Ev[p], Ov[p]));
    out[2 * p] = sub2(Fg[2 * p], sub2(Ev[p], Ov[p]));
  }
}

}  // namespace fsi
#endif

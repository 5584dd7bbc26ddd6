// FP64 polar rotation of a 3x3 deformation gradient (host + device).
//
// The reference takes R = U V^T from ti.svd (src/mpm_lbm/sim/mpm/solid.py:
// 233-234), with U, V proper rotations and the sign of det F carried by the
// smallest singular value.  R is unique for any SVD with that convention, so
// it is computed here from a cyclic Jacobi eigen-decomposition of F^T F (V)
// followed by a Givens QR of F V (U) -- the structure of McAdams et al. 2011,
// "Computing the Singular Value Decomposition of 3x3 matrices with minimal
// branching and elementary floating point operations" -- all in double.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define FSI_HD2 __host__ __device__ __forceinline__
#else
#define FSI_HD2 inline
#endif

namespace fsi {

FSI_HD2 void polar_rotation_jacobi_d(const double F[9], double R[9]) {
  // A = F^T F (symmetric)
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = F[0 * 3 + i] * F[0 * 3 + j] + F[1 * 3 + i] * F[1 * 3 + j] + F[2 * 3 + i] * F[2 * 3 + j];
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dg = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (off <= 1e-30 * dg || off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        const double apq = A[p][q];
        if (apq == 0.0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  // order eigenvalues descending
  double ev[3] = {A[0][0], A[1][1], A[2][2]};
  int o[3] = {0, 1, 2};
  if (ev[o[0]] < ev[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  if (ev[o[1]] < ev[o[2]]) { int t = o[1]; o[1] = o[2]; o[2] = t; }
  if (ev[o[0]] < ev[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  double Vs[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Vs[i][j] = V[i][o[j]];
  const double dv = Vs[0][0] * (Vs[1][1] * Vs[2][2] - Vs[1][2] * Vs[2][1]) - Vs[0][1] * (Vs[1][0] * Vs[2][2] - Vs[1][2] * Vs[2][0]) +
                    Vs[0][2] * (Vs[1][0] * Vs[2][1] - Vs[1][1] * Vs[2][0]);
  if (dv < 0)
    for (int i = 0; i < 3; ++i) Vs[i][2] = -Vs[i][2];
  // B = F Vs
  double B[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) B[i][j] = F[i * 3 + 0] * Vs[0][j] + F[i * 3 + 1] * Vs[1][j] + F[i * 3 + 2] * Vs[2][j];
  double U[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const int rr[3][3] = {{0, 1, 0}, {0, 2, 0}, {1, 2, 1}};  // (row1, row2, column) of each Givens step
  for (int g = 0; g < 3; ++g) {
    const int r1 = rr[g][0], r2 = rr[g][1], col = rr[g][2];
    const double a = B[r1][col], b = B[r2][col];
    const double h = sqrt(a * a + b * b);
    double c = 1.0, s = 0.0;
    if (h > 1e-300) {
      c = a / h;
      s = b / h;
    }
    for (int k = 0; k < 3; ++k) {
      const double x = B[r1][k], y = B[r2][k];
      B[r1][k] = c * x + s * y;
      B[r2][k] = -s * x + c * y;
    }
    for (int k = 0; k < 3; ++k) {
      const double x = U[k][r1], y = U[k][r2];
      U[k][r1] = c * x + s * y;
      U[k][r2] = -s * x + c * y;
    }
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i * 3 + j] = U[i][0] * Vs[j][0] + U[i][1] * Vs[j][1] + U[i][2] * Vs[j][2];
}

// Scaled Newton iteration X <- a X + b X^-T (X^-T = cof(X) / det X); returns
// false (R untouched) when det F <= 0 or the iteration has not converged, so
// that the caller falls back to Jacobi.  With X = R S, a X + b X^-T =
// R (a S + b S^-1): the polar factor R is kept exactly for any positive a, b,
// which only steer the convergence.  So the matrix arithmetic is FP64 while the
// scaling a = g/2, b = 1/(2 g det) with g = (|X^-1|_F / |X|_F)^(1/2) is formed
// in FP32 (square roots and division on the fast FP32 path); once the steps are
// small the iteration switches to the unscaled a = 1/2, b = 1/(2 det) in FP64,
// which drives S to I quadratically (and removes the FP32 rounding of the
// scalars from the scale of X).
FSI_HD2 bool polar_rotation_newton_d(const double F[9], double R[9]) {
  double X[9];
  for (int a = 0; a < 9; ++a) X[a] = F[a];
  bool scaled = true;
  for (int it = 0; it < 20; ++it) {
    // cofactor matrix C = det(X) X^-T
    const double C0 = X[4] * X[8] - X[5] * X[7], C1 = X[5] * X[6] - X[3] * X[8], C2 = X[3] * X[7] - X[4] * X[6];
    const double C3 = X[2] * X[7] - X[1] * X[8], C4 = X[0] * X[8] - X[2] * X[6], C5 = X[1] * X[6] - X[0] * X[7];
    const double C6 = X[1] * X[5] - X[2] * X[4], C7 = X[2] * X[3] - X[0] * X[5], C8 = X[0] * X[4] - X[1] * X[3];
    const double det = X[0] * C0 + X[1] * C1 + X[2] * C2;
    if (!(det > 0.0)) return false;
    const double C[9] = {C0, C1, C2, C3, C4, C5, C6, C7, C8};
    double a0, b0;
    if (scaled) {
      double nx = 0.0, nc = 0.0;
      for (int a = 0; a < 9; ++a) {
        nx += X[a] * X[a];
        nc += C[a] * C[a];
      }
      const float detf = (float)det;
      const float g = sqrtf(sqrtf((float)nc / ((float)nx * detf * detf)));
      if (!(g > 0.0f) || !(g < 3.0e38f)) return false;
      a0 = (double)(0.5f * g);
      b0 = (double)(0.5f / (g * detf));
    } else {
      a0 = 0.5;
      b0 = 0.5 / det;
    }
    double d2 = 0.0;
    for (int a = 0; a < 9; ++a) {
      const double xn = a0 * X[a] + b0 * C[a];
      const double d = xn - X[a];
      d2 += d * d;
      X[a] = xn;
    }
    // near convergence the scale factor is 1 to first order: drop it
    if (d2 < 1e-6) scaled = false;
    // quadratic convergence of the unscaled steps: a step of size e leaves an error of order e^2
    if (!scaled && d2 < 1e-18) {
      const double tr = X[0] + X[4] + X[8];
      if (!(tr - tr == 0.0)) return false;  // inf or NaN
      for (int a = 0; a < 9; ++a) R[a] = X[a];
      return true;
    }
  }
  return false;
}

FSI_HD2 void polar_rotation_d(const double F[9], double R[9]) {
  if (!polar_rotation_newton_d(F, R)) polar_rotation_jacobi_d(F, R);
}

}  // namespace fsi

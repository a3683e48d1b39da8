// FP64 6x6 normal-equation solve and SE(3) update, callable on host and device.
//
// The reference solves x = pinv(JtJ) Jtr with TooN::GR_SVD::backsub(b, 1e6)
// (apps/kfusion/include/commons.h:689-696): singular values below
// sigma_max / 1e6 are dropped.  Here the well-conditioned case (all LDL^T
// pivots within 1e-5 of the largest) is solved by Gauss-Jordan elimination;
// otherwise the symmetric matrix is diagonalised by cyclic Jacobi rotations
// and the same truncated pseudo-inverse is applied.  The update exponentiates the twist
// (v, w) (translation first, as TooN::SE3 does) and left-multiplies the pose
// (tracking.cpp:333-334).
#pragma once
#include <cmath>
#include "mf_common.cuh"

namespace mf {

// makeJTJ, commons.h:673-687: 21 upper-triangle terms (row-major) -> 6x6.
MF_HD void make_jtj(const double* v21, double A[6][6]) {
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int j = i; j < 6; ++j) {
      const int q = i * 6 - i * (i - 1) / 2 + (j - i);
      A[i][j] = v21[q];
      A[j][i] = v21[q];
    }
}

// Not inlined: the rare ill-conditioned path.
__host__ __device__ __noinline__ inline void solve6_eigen(const double Ain[6][6],
                                                          const double b[6], double condition,
                                                          double x[6]) {
  double A[6][6], V[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) { A[i][j] = Ain[i][j]; V[i][j] = i == j ? 1.0 : 0.0; }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) off += A[p][q] * A[p][q];
    if (off < 1e-300) break;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) {
        if (A[p][q] == 0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        const double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 6; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq; A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk; A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 6; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq; V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  double smax = 0;
  for (int i = 0; i < 6; ++i) smax = fmax(smax, fabs(A[i][i]));
  for (int i = 0; i < 6; ++i) x[i] = 0;
  for (int k = 0; k < 6; ++k) {
    const double sk = fabs(A[k][k]);
    if (!(sk > smax / condition) || sk == 0) continue;
    double vb = 0;
    for (int i = 0; i < 6; ++i) vb += V[i][k] * b[i];
    const double coef = vb / A[k][k];
    for (int i = 0; i < 6; ++i) x[i] += coef * V[i][k];
  }
}

// Returns true when the truncated eigen solve was needed.  Gauss-Jordan
// elimination without pivoting (the matrix is symmetric positive definite
// when the solve is used): at step j every other row i subtracts
// (a_ij / a_jj) times row j from its columns j..5 and from its right-hand
// side, so after six steps x_i = b_i / a_ii.  The pivots a_jj are the LDL^T
// pivots; all within 1e-5 of the largest, else the truncated eigen solve.
// Each row's operations depend on the pivot row only, so the device runs the
// rows on six lanes of a warp (gn_step_warp) with the same operations in the
// same order.  All loops have compile-time bounds and are unrolled.
MF_HD bool solve6(const double A[6][6], const double b[6], double x[6]) {
  double a[6][6], c[6], piv[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    c[i] = b[i];
#pragma unroll
    for (int k = 0; k < 6; ++k) a[i][k] = A[i][k];
  }
  double pmax = 0;
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    piv[j] = a[j][j];
    pmax = fmax(pmax, a[j][j]);
    ok = ok && (a[j][j] > 0);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (i == j) continue;
      const double f = a[i][j] / a[j][j];
#pragma unroll
      for (int k = j; k < 6; ++k) a[i][k] -= f * a[j][k];
      c[i] -= f * c[j];
    }
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) ok = ok && (piv[j] > 1e-5 * pmax);
  if (!ok) {
    solve6_eigen(A, b, 1e6, x);
    return true;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) x[i] = c[i] / a[i][i];
  return false;
}

// SE(3) exponential of (v, w), translation first: R = I + A W + B W^2,
// t = (I + B W + C W^2) v with A = sin(t)/t, B = (1 - cos t)/t^2, C = (1 - A)/t^2.
MF_HD void se3_exp(const double xi[6], double T[16]) {
  const double w0 = xi[3], w1 = xi[4], w2 = xi[5];
  const double th2 = w0 * w0 + w1 * w1 + w2 * w2;
  double A, B, C;
  if (th2 < 1e-10) {
    A = 1 - th2 / 6; B = 0.5 - th2 / 24; C = 1.0 / 6 - th2 / 120;
  } else {
    const double th = sqrt(th2);
    double sn, cs;
    sincos(th, &sn, &cs);
    A = sn / th; B = (1 - cs) / th2; C = (1 - A) / th2;
  }
  const double W[3][3] = {{0, -w2, w1}, {w2, 0, -w0}, {-w1, w0, 0}};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double t = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double W2 = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
      const double I = i == j ? 1.0 : 0.0;
      T[4 * i + j] = I + A * W[i][j] + B * W2;
      t += (I + B * W[i][j] + C * W2) * xi[j];
    }
    T[4 * i + 3] = t;
  }
  T[12] = T[13] = T[14] = 0; T[15] = 1;
}

MF_HD void mul4d(const double* A, const double* B, double* R) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) s += A[4 * i + k] * B[4 * k + j];
      R[4 * i + j] = s;
    }
}

MF_HD M4 to_m4f(const double* T) {
  M4 m;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    m.r[i].x = (float)T[4 * i]; m.r[i].y = (float)T[4 * i + 1];
    m.r[i].z = (float)T[4 * i + 2]; m.r[i].w = (float)T[4 * i + 3];
  }
  return m;
}

}  // namespace mf

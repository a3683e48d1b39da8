// TEST INFRASTRUCTURE ONLY.  The SVD solve of the TooN stand-in (see TooN.h):
// GR_SVD<R, C>(M).backsub(b, condition) returns the pseudo-inverse solution
// x = V diag(s_i^-1) U^T b in double, where a singular value s_i with
// s_i * condition <= s_max contributes 0.  The decomposition here is a
// one-sided Jacobi SVD (Hestenes), not TooN's Golub-Reinsch code; both give
// the same singular vectors to rounding for the well-separated 6x6 normal
// equations the tracker solves.
#pragma once
#include "TooN.h"

namespace TooN {

template <int R, int C = R, typename P = double>
class GR_SVD {
  P U_[R][C];   // columns: left singular vectors (scaled columns of M V)
  P V_[C][C];
  P s_[C];

 public:
  template <typename P2, typename L2>
  explicit GR_SVD(const Matrix<R, C, P2, L2>& m) {
    P a[R][C];
    for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) a[i][j] = m(i, j);
    for (int i = 0; i < C; ++i) for (int j = 0; j < C; ++j) V_[i][j] = (i == j);
    for (int sweep = 0; sweep < 60; ++sweep) {
      P off = 0;
      for (int p = 0; p < C - 1; ++p)
        for (int q = p + 1; q < C; ++q) {
          P alpha = 0, beta = 0, gamma = 0;
          for (int i = 0; i < R; ++i) {
            alpha += a[i][p] * a[i][p];
            beta += a[i][q] * a[i][q];
            gamma += a[i][p] * a[i][q];
          }
          if (gamma == 0) continue;
          const P rel = std::fabs(gamma) / std::sqrt(alpha * beta);
          if (rel > off) off = rel;
          if (rel < P(1e-17)) continue;
          const P zeta = (beta - alpha) / (2 * gamma);
          const P tt = (zeta >= 0 ? 1 : -1) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
          const P c = 1 / std::sqrt(1 + tt * tt), s = c * tt;
          for (int i = 0; i < R; ++i) {
            const P x = a[i][p], y = a[i][q];
            a[i][p] = c * x - s * y;
            a[i][q] = s * x + c * y;
          }
          for (int i = 0; i < C; ++i) {
            const P x = V_[i][p], y = V_[i][q];
            V_[i][p] = c * x - s * y;
            V_[i][q] = s * x + c * y;
          }
        }
      if (off < P(1e-16)) break;
    }
    for (int j = 0; j < C; ++j) {
      P n = 0;
      for (int i = 0; i < R; ++i) n += a[i][j] * a[i][j];
      s_[j] = std::sqrt(n);
      for (int i = 0; i < R; ++i) U_[i][j] = (s_[j] > 0) ? a[i][j] / s_[j] : 0;
    }
  }

  P get_largest_singular_value() const {
    P m = 0;
    for (int j = 0; j < C; ++j) if (s_[j] > m) m = s_[j];
    return m;
  }

  template <typename P2, typename B2>
  Vector<C, double> backsub(const Vector<R, P2, B2>& b, const P condition = P(1e9)) const {
    const P smax = get_largest_singular_value();
    P y[C];
    for (int j = 0; j < C; ++j) {
      P d = 0;
      for (int i = 0; i < R; ++i) d += U_[i][j] * P(b[i]);
      y[j] = (s_[j] * condition <= smax) ? P(0) : d / s_[j];
    }
    Vector<C, double> x;
    for (int i = 0; i < C; ++i) {
      P acc = 0;
      for (int j = 0; j < C; ++j) acc += V_[i][j] * y[j];
      x[i] = acc;
    }
    return x;
  }
};

}  // namespace TooN

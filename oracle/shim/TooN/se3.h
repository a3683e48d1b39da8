// TEST INFRASTRUCTURE ONLY.  SE(3) for the TooN stand-in (see TooN.h): the
// group element built from a twist by the exponential map, with TooN's twist
// order (translation part first, rotation part last), and its action on a
// 4-row matrix.  Written from the mathematics (Rodrigues' formula and the
// left Jacobian of SO(3)), not from TooN source.
#pragma once
#include "TooN.h"

namespace TooN {

template <typename P = double>
class SE3 {
 public:
  P R[3][3];
  P t[3];

  SE3() { for (int i = 0; i < 3; ++i) { t[i] = 0; for (int j = 0; j < 3; ++j) R[i][j] = (i == j); } }
  template <int N, typename P2, typename B2>
  explicit SE3(const Vector<N, P2, B2>& mu) { set_exp(mu); }

  // exp of the twist mu = (v, w):
  //   R = I + A [w]x + B [w]x^2,  t = (I + B [w]x + C [w]x^2) v
  //   A = sin(th)/th, B = (1 - cos(th))/th^2, C = (1 - A)/th^2,  th = |w|,
  // with the series of A, B, C where th^2 is too small for the closed forms.
  template <int N, typename P2, typename B2>
  void set_exp(const Vector<N, P2, B2>& mu) {
    const P v[3] = {P(mu[0]), P(mu[1]), P(mu[2])};
    const P w[3] = {P(mu[3]), P(mu[4]), P(mu[5])};
    const P th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    P A, B, C;
    if (th2 < P(1e-8)) {
      A = 1 - th2 / 6;
      B = P(0.5) - th2 / 24;
      C = P(1) / 6 - th2 / 120;
    } else {
      const P th = std::sqrt(th2);
      A = std::sin(th) / th;
      B = (1 - std::cos(th)) / th2;
      C = (1 - A) / th2;
    }
    // [w]x and [w]x^2
    const P W[3][3] = {{0, -w[2], w[1]}, {w[2], 0, -w[0]}, {-w[1], w[0], 0}};
    P W2[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) W2[i][j] = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
    P V[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const P I = (i == j) ? 1 : 0;
        R[i][j] = I + A * W[i][j] + B * W2[i][j];
        V[i][j] = I + B * W[i][j] + C * W2[i][j];
      }
    for (int i = 0; i < 3; ++i) t[i] = V[i][0] * v[0] + V[i][1] * v[1] + V[i][2] * v[2];
  }
};

// SE3 * M for a 4-row matrix M: rows 0-2 become R * M(0..2, :) + t * M(3, :),
// row 3 is copied; computed in double.
template <typename P, int C, typename PM, typename LM>
inline Matrix<4, C, double> operator*(const SE3<P>& g, const Matrix<4, C, PM, LM>& m) {
  Matrix<4, C, double> r;
  for (int j = 0; j < C; ++j) {
    for (int i = 0; i < 3; ++i)
      r(i, j) = double(g.R[i][0]) * m(0, j) + double(g.R[i][1]) * m(1, j) + double(g.R[i][2]) * m(2, j) +
                double(g.t[i]) * m(3, j);
    r(3, j) = m(3, j);
  }
  return r;
}

}  // namespace TooN

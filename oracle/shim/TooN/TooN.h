// TEST INFRASTRUCTURE ONLY.  A minimal stand-in for the part of TooN
// (https://github.com/edrosten/TooN, commit 92241416d2a4874fd2334e08a5d417dfea6a1a3f,
// which the reference pins in apps/kfusion/Makefile:31-35 and does not vendor)
// that the reference's tracking and its helpers in apps/kfusion/include/commons.h
// call: fixed-size vectors and matrices, borrowed row-major views, slices, the
// Zeros / Identity initialisers, a 4x4 Gauss-Jordan solve, the SE(3)
// exponential (se3.h) and the SVD pseudo-inverse solve (GR_SVD.h).  It is
// written for this project from the published mathematics and the call sites'
// use of it; it is not TooN source.  Used only to compile the reference's own
// tracking.cpp / preprocessing.cpp / object.cpp into oracle/_ref.
#pragma once
#include <cmath>
#include <cstddef>

namespace TooN {

struct ZerosT {};
struct IdentityT {};
static const ZerosT Zeros = ZerosT();
static const IdentityT Identity = IdentityT();

struct Internal {};                    // storage owned by the object
struct Reference { struct RowMajor {}; };  // borrowed storage (a vector, or a row-major matrix)
struct RowMajor {};
template <int Stride> struct Strided {};   // a borrowed vector with an element stride

template <int N, typename P = double, typename B = Internal> class Vector;

// ---- owned vector --------------------------------------------------------
template <int N, typename P>
class Vector<N, P, Internal> {
  P d_[N];

 public:
  Vector() {}
  Vector(ZerosT) { for (int i = 0; i < N; ++i) d_[i] = 0; }
  template <typename P2, typename B2>
  Vector(const Vector<N, P2, B2>& o) { for (int i = 0; i < N; ++i) d_[i] = o[i]; }
  template <typename P2, typename B2>
  Vector& operator=(const Vector<N, P2, B2>& o) { for (int i = 0; i < N; ++i) d_[i] = o[i]; return *this; }
  P& operator[](int i) { return d_[i]; }
  const P& operator[](int i) const { return d_[i]; }
  int size() const { return N; }
  template <int S, int L> Vector<L, P, Strided<1>> slice() { return Vector<L, P, Strided<1>>(d_ + S); }
  template <int S, int L> Vector<L, const P, Strided<1>> slice() const {
    return Vector<L, const P, Strided<1>>(d_ + S);
  }
};

// ---- borrowed vector (a row of a matrix, a slice, or a wrapped pointer) ---
template <int N, typename P, int St>
class Vector<N, P, Strided<St>> {
  P* p_;

 public:
  explicit Vector(P* p) : p_(p) {}
  Vector(const Vector& o) : p_(o.p_) {}
  // assignment writes through to the borrowed elements
  Vector& operator=(const Vector& o) { for (int i = 0; i < N; ++i) p_[i * St] = o[i]; return *this; }
  template <typename P2, typename B2>
  Vector& operator=(const Vector<N, P2, B2>& o) { for (int i = 0; i < N; ++i) p_[i * St] = o[i]; return *this; }
  template <typename P2, typename B2>
  Vector& operator+=(const Vector<N, P2, B2>& o) { for (int i = 0; i < N; ++i) p_[i * St] += o[i]; return *this; }
  P& operator[](int i) const { return p_[i * St]; }
  int size() const { return N; }
  template <int S, int L> Vector<L, P, Strided<St>> slice() const { return Vector<L, P, Strided<St>>(p_ + S * St); }
};

// Vector<N, P, Reference>(ptr): a borrowed contiguous vector
template <int N, typename P>
class Vector<N, P, Reference> : public Vector<N, P, Strided<1>> {
 public:
  explicit Vector(P* p) : Vector<N, P, Strided<1>>(p) {}
};

template <int N, typename P, typename B>
inline double norm_sq(const Vector<N, P, B>& v) {
  double s = 0;
  for (int i = 0; i < N; ++i) s += double(v[i]) * double(v[i]);
  return s;
}
template <int N, typename P, typename B>
inline double norm(const Vector<N, P, B>& v) { return std::sqrt(norm_sq(v)); }

template <int N, typename P, typename B>
inline Vector<N, double> operator*(double s, const Vector<N, P, B>& v) {
  Vector<N, double> r; for (int i = 0; i < N; ++i) r[i] = s * v[i]; return r;
}

// ---- matrices --------------------------------------------------------------
template <int R, int C = R, typename P = double, typename L = RowMajor> class Matrix;

template <int R, int C, typename P>
class Matrix<R, C, P, RowMajor> {
  P d_[R * C];

 public:
  Matrix() {}
  Matrix(ZerosT) { for (int i = 0; i < R * C; ++i) d_[i] = 0; }
  Matrix(IdentityT) { for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) d_[i * C + j] = (i == j) ? 1 : 0; }
  template <typename P2, typename L2>
  Matrix(const Matrix<R, C, P2, L2>& o) { for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) d_[i * C + j] = o(i, j); }
  P& operator()(int i, int j) { return d_[i * C + j]; }
  const P& operator()(int i, int j) const { return d_[i * C + j]; }
  Vector<C, P, Strided<1>> operator[](int i) { return Vector<C, P, Strided<1>>(d_ + i * C); }
  Vector<C, const P, Strided<1>> operator[](int i) const { return Vector<C, const P, Strided<1>>(d_ + i * C); }
  int num_rows() const { return R; }
  int num_cols() const { return C; }
};

// a borrowed row-major matrix over caller storage (TooN's Reference::RowMajor)
template <int R, int C, typename P>
class Matrix<R, C, P, Reference::RowMajor> {
  P* d_;

 public:
  explicit Matrix(P* p) : d_(p) {}
  template <typename P2, typename L2>
  const Matrix& operator=(const Matrix<R, C, P2, L2>& o) const {
    for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) d_[i * C + j] = o(i, j);
    return *this;
  }
  P& operator()(int i, int j) const { return d_[i * C + j]; }
  Vector<C, P, Strided<1>> operator[](int i) const { return Vector<C, P, Strided<1>>(d_ + i * C); }
  int num_rows() const { return R; }
  int num_cols() const { return C; }
};

template <int R, int C, typename P>
inline Matrix<R, C, P, Reference::RowMajor> wrapMatrix(P* p) { return Matrix<R, C, P, Reference::RowMajor>(p); }

template <typename A, typename B> struct Promote { typedef double type; };
template <> struct Promote<float, float> { typedef float type; };

template <typename T> struct Plain { typedef T type; };
template <typename T> struct Plain<const T> { typedef T type; };

// Matrix product: every element is the dot product of a row and a column,
// accumulated from k = 0 upwards in the promoted precision.
template <int R, int K, int C, typename P1, typename L1, typename P2, typename L2>
inline Matrix<R, C, typename Promote<typename Plain<P1>::type, typename Plain<P2>::type>::type>
operator*(const Matrix<R, K, P1, L1>& a, const Matrix<K, C, P2, L2>& b) {
  typedef typename Promote<typename Plain<P1>::type, typename Plain<P2>::type>::type T;
  Matrix<R, C, T> r;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < C; ++j) {
      T s = T(a(i, 0)) * T(b(0, j));
      for (int k = 1; k < K; ++k) s += T(a(i, k)) * T(b(k, j));
      r(i, j) = s;
    }
  return r;
}

// gaussian_elimination(A, B) solves A X = B.  Restated as elimination with
// partial pivoting on [A | B] in the matrices' precision, then back
// substitution; the arithmetic equals the oracle's 4x4 inverse
// (oracle/or_math.hpp orc::inverse), so both checkers invert poses identically.
template <int N, int M, typename P>
inline Matrix<N, M, P> gaussian_elimination(Matrix<N, N, P> a, Matrix<N, M, P> b) {
  for (int c = 0; c < N; ++c) {
    int p = c; P best = std::fabs(a(c, c));
    for (int r = c + 1; r < N; ++r) if (std::fabs(a(r, c)) > best) { best = std::fabs(a(r, c)); p = r; }
    if (p != c)
      for (int j = 0; j < N; ++j) { P t = a(c, j); a(c, j) = a(p, j); a(p, j) = t; }
    if (p != c)
      for (int j = 0; j < M; ++j) { P t = b(c, j); b(c, j) = b(p, j); b(p, j) = t; }
    for (int r = c + 1; r < N; ++r) {
      const P f = a(r, c) / a(c, c);
      for (int j = c; j < N; ++j) a(r, j) -= f * a(c, j);
      for (int j = 0; j < M; ++j) b(r, j) -= f * b(c, j);
    }
  }
  Matrix<N, M, P> x;
  for (int j = 0; j < M; ++j)
    for (int r = N - 1; r >= 0; --r) {
      P s = b(r, j);
      for (int k = r + 1; k < N; ++k) s -= a(r, k) * x(k, j);
      x(r, j) = s / a(r, r);
    }
  return x;
}

}  // namespace TooN

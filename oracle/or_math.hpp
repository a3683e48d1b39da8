// TEST INFRASTRUCTURE ONLY — part of the CPU oracle.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference leg
// may load or call anything under oracle/.  The product path never does.
//
// Scalar and small-vector arithmetic with the exact evaluation order of the
// reference's host math (utils/cutil_math.h, utils/math_utils.h,
// apps/kfusion/include/commons.h).  Compile with -ffp-contract=off so that no
// multiply-add is fused: parity is defined on IEEE single-precision evaluation
// in source order.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace orc {

struct F2 { float x, y; };
struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
struct I3 { int x, y, z; };
struct M4 { F4 r[4]; };  // row-major, r[i] = row i (Matrix4::data[i])

// utils/cutil_math.h:43-49 host fminf/fmaxf: plain comparisons (not IEEE 754
// minNum): fminf(NaN, b) == b, fminf(a, NaN) == NaN.
inline float fmn(float a, float b) { return a < b ? a : b; }
inline float fmx(float a, float b) { return a > b ? a : b; }
inline int imin(int a, int b) { return a < b ? a : b; }
inline int imax(int a, int b) { return a > b ? a : b; }
// utils/cutil_math.h:981-983
inline float clampf(float f, float a, float b) { return fmx(a, fmn(f, b)); }
inline float sq(float r) { return r * r; }   // utils/math_utils.h:96

inline F3 mk3(float x, float y, float z) { F3 v{x, y, z}; return v; }
inline F3 mk3(float s) { return mk3(s, s, s); }
inline F3 operator+(F3 a, F3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 operator-(F3 a, F3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 operator*(F3 a, F3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline F3 operator*(F3 a, float b) { return mk3(a.x * b, a.y * b, a.z * b); }
inline F3 operator*(float b, F3 a) { return mk3(b * a.x, b * a.y, b * a.z); }
inline F3 operator/(F3 a, F3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline F3 operator/(F3 a, float b) { return mk3(a.x / b, a.y / b, a.z / b); }
inline F3 operator+(F3 a, float b) { return mk3(a.x + b, a.y + b, a.z + b); }
inline F3 operator-(float b, F3 a) { return mk3(b - a.x, b - a.y, b - a.z); }
inline F3& operator+=(F3& a, F3 b) { a = a + b; return a; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot4(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline F3 cross(F3 a, F3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(F3 v) { return sqrtf(dot(v, v)); }
// cutil_math.h:1156-1160 with the host rsqrtf of :59-61 (1/sqrtf).
inline F3 normalize(F3 v) { float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
inline F3 floor3(F3 v) { return mk3(floorf(v.x), floorf(v.y), floorf(v.z)); }
inline F3 frac3(F3 v) { return mk3(v.x - floorf(v.x), v.y - floorf(v.y), v.z - floorf(v.z)); }
inline F3 fmn3(F3 a, F3 b) { return mk3(fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z)); }
inline F3 fmx3(F3 a, F3 b) { return mk3(fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)); }
inline F3 xyz(F4 a) { return mk3(a.x, a.y, a.z); }
inline I3 to_i3(F3 a) { I3 r{int(a.x), int(a.y), int(a.z)}; return r; }  // truncation
inline F3 to_f3(I3 a) { return mk3(float(a.x), float(a.y), float(a.z)); }

// utils/math_utils.h:50-52
inline F3 get_translation(const M4& m) { return mk3(m.r[0].w, m.r[1].w, m.r[2].w); }
// utils/math_utils.h:105-110
inline F3 operator*(const M4& M, F3 v) {
  return mk3(dot(xyz(M.r[0]), v) + M.r[0].w, dot(xyz(M.r[1]), v) + M.r[1].w,
             dot(xyz(M.r[2]), v) + M.r[2].w);
}
// utils/math_utils.h:112-115
inline F3 rotate(const M4& M, F3 v) {
  return mk3(dot(xyz(M.r[0]), v), dot(xyz(M.r[1]), v), dot(xyz(M.r[2]), v));
}
// utils/math_utils.h:117-121  (v^T M: dot with the columns)
inline F3 rotate_t(F3 v, const M4& M) {
  return mk3(dot(mk3(M.r[0].x, M.r[1].x, M.r[2].x), v),
             dot(mk3(M.r[0].y, M.r[1].y, M.r[2].y), v),
             dot(mk3(M.r[0].z, M.r[1].z, M.r[2].z), v));
}
inline float& at(M4& m, int i, int j) { return (&m.r[i].x)[j]; }
inline float at(const M4& m, int i, int j) { return (&m.r[i].x)[j]; }
inline M4 transpose(const M4& M) {
  M4 t; for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) at(t, i, j) = at(M, j, i);
  return t;
}
// commons.h:657-662 (TooN float product; each element accumulated k = 0..3).
inline M4 mul(const M4& A, const M4& B) {
  M4 R;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      float s = at(A, i, 0) * at(B, 0, j);
      for (int k = 1; k < 4; ++k) s += at(A, i, k) * at(B, k, j);
      at(R, i, j) = s;
    }
  return R;
}
// commons.h:649-655 wraps TooN::gaussian_elimination (TooN is not vendored).
// Restated as Gaussian elimination with partial pivoting on [A | I] in float,
// then back substitution.  Parity with TooN for this 4x4 inverse is unpinned.
inline M4 inverse(const M4& A) {
  float a[4][4], b[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) { a[i][j] = at(A, i, j); b[i][j] = (i == j) ? 1.f : 0.f; }
  for (int c = 0; c < 4; ++c) {
    int p = c; float best = fabsf(a[c][c]);
    for (int r = c + 1; r < 4; ++r) if (fabsf(a[r][c]) > best) { best = fabsf(a[r][c]); p = r; }
    if (p != c) for (int j = 0; j < 4; ++j) { float t = a[c][j]; a[c][j] = a[p][j]; a[p][j] = t;
                                               t = b[c][j]; b[c][j] = b[p][j]; b[p][j] = t; }
    for (int r = c + 1; r < 4; ++r) {
      const float f = a[r][c] / a[c][c];
      for (int j = c; j < 4; ++j) a[r][j] -= f * a[c][j];
      for (int j = 0; j < 4; ++j) b[r][j] -= f * b[c][j];
    }
  }
  M4 R;
  for (int j = 0; j < 4; ++j)
    for (int r = 3; r >= 0; --r) {
      float s = b[r][j];
      for (int k = r + 1; k < 4; ++k) s -= a[r][k] * at(R, k, j);
      at(R, r, j) = s / a[r][r];
    }
  return R;
}
// commons.h:631-647
inline M4 camera_matrix(F4 k) {
  M4 K; std::memset(&K, 0, sizeof(K));
  K.r[0] = F4{k.x, 0, k.z, 0}; K.r[1] = F4{0, k.y, k.w, 0};
  K.r[2] = F4{0, 0, 1, 0}; K.r[3] = F4{0, 0, 0, 1};
  return K;
}
inline M4 inverse_camera_matrix(F4 k) {
  M4 K; std::memset(&K, 0, sizeof(K));
  K.r[0] = F4{1.0f / k.x, 0, -k.z / k.x, 0}; K.r[1] = F4{0, 1.0f / k.y, -k.w / k.y, 0};
  K.r[2] = F4{0, 0, 1, 0}; K.r[3] = F4{0, 0, 0, 1};
  return K;
}
inline F4 kdiv(F4 k, float d) { return F4{k.x / d, k.y / d, k.z / d, k.w / d}; }
inline M4 load_m4(const float* p) { M4 m; std::memcpy(&m, p, sizeof(M4)); return m; }
inline void store_m4(float* p, const M4& m) { std::memcpy(p, &m, sizeof(M4)); }

// utils/math_utils.h:149-166: bilinear interpolation, same term order.
template <typename T> struct Bil;
template <> struct Bil<float> {
  static float mix(const float* v, float fx, float fy) {
    return v[0] * (1.f - fx) * (1.f - fy) + v[1] * (1.f - fy) * fx +
           v[2] * (1.f - fx) * fy + v[3] * fx * fy;
  }
};
inline float bilinear(const float* img, int w, F2 pos) {
  const int bx = int(floorf(pos.x)), by = int(floorf(pos.y));
  const float fx = pos.x - floorf(pos.x), fy = pos.y - floorf(pos.y);
  float v[4] = {img[bx + by * w], img[bx + 1 + by * w], img[bx + (by + 1) * w],
                img[bx + 1 + (by + 1) * w]};
  return Bil<float>::mix(v, fx, fy);
}
inline F3 bilinear3(const F3* img, int w, F2 pos) {
  const int bx = int(floorf(pos.x)), by = int(floorf(pos.y));
  const float fx = pos.x - floorf(pos.x), fy = pos.y - floorf(pos.y);
  const F3 v0 = img[bx + by * w], v1 = img[bx + 1 + by * w], v2 = img[bx + (by + 1) * w],
           v3 = img[bx + 1 + (by + 1) * w];
  // float3 * float is component-wise, so the scalar expression applies per axis.
  const float a = (1.f - fx), b = (1.f - fy);
  F3 r;
  r.x = v0.x * a * b + v1.x * b * fx + v2.x * a * fy + v3.x * fx * fy;
  r.y = v0.y * a * b + v1.y * b * fx + v2.y * a * fy + v3.y * fx * fy;
  r.z = v0.z * a * b + v1.z * b * fx + v2.z * a * fy + v3.z * fx * fy;
  return r;
}

}  // namespace orc

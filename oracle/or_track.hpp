// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
//
// Restatement of the reference's tracking path, templated on the scalar type:
// T = float follows the reference's single-precision arithmetic (the reduction
// in float, row blocks summed in order), T = double is the all-FP64 precision
// oracle.  Sources:
//   apps/kfusion/src/cpp/tracking/tracking.cpp   (Tracking, GN drivers, kernels)
//   apps/kfusion/src/cpp/preprocessing/*         (pyramid kernels)
//   apps/kfusion/include/commons.h:673-704       (makeJTJ, solve, toMatrix4)
// The 6x6 solve of commons.h uses TooN::GR_SVD::backsub(b, 1e6) and the update
// TooN::SE3::exp; TooN is not vendored, so both are restated from their
// mathematics (pseudo-inverse with singular values below sigma_max / 1e6
// dropped; the SE(3) exponential with translation-first twists).  Parity with
// TooN itself is unpinned.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace ort {

template <typename T> struct V3 { T x, y, z; };
template <typename T> struct M4 { T m[4][4]; };

template <typename T> inline V3<T> v3(T x, T y, T z) { V3<T> r{x, y, z}; return r; }
template <typename T> inline V3<T> operator+(V3<T> a, V3<T> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> inline V3<T> operator-(V3<T> a, V3<T> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> inline V3<T> operator*(T s, V3<T> a) { return v3(s * a.x, s * a.y, s * a.z); }
template <typename T> inline V3<T> operator*(V3<T> a, T s) { return v3(a.x * s, a.y * s, a.z * s); }
template <typename T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline V3<T> cross(V3<T> a, V3<T> b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T> inline T length(V3<T> v) { return std::sqrt(dot(v, v)); }
template <typename T> inline V3<T> normalize(V3<T> v) { T inv = T(1) / std::sqrt(dot(v, v)); return v * inv; }
template <typename T> inline V3<T> xform(const M4<T>& M, V3<T> v) {
  return v3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z + M.m[0][3],
            M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z + M.m[1][3],
            M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z + M.m[2][3]);
}
template <typename T> inline V3<T> rotate(const M4<T>& M, V3<T> v) {
  return v3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z,
            M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z,
            M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z);
}
template <typename T> M4<T> mul(const M4<T>& A, const M4<T>& B) {
  M4<T> R;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      T s = A.m[i][0] * B.m[0][j];
      for (int k = 1; k < 4; ++k) s += A.m[i][k] * B.m[k][j];
      R.m[i][j] = s;
    }
  return R;
}
template <typename T> M4<T> inverse(const M4<T>& A) {  // partial-pivot elimination
  T a[4][4], b[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) { a[i][j] = A.m[i][j]; b[i][j] = i == j ? T(1) : T(0); }
  for (int c = 0; c < 4; ++c) {
    int p = c; T best = std::fabs(a[c][c]);
    for (int r = c + 1; r < 4; ++r) if (std::fabs(a[r][c]) > best) { best = std::fabs(a[r][c]); p = r; }
    if (p != c) for (int j = 0; j < 4; ++j) { std::swap(a[c][j], a[p][j]); std::swap(b[c][j], b[p][j]); }
    for (int r = c + 1; r < 4; ++r) {
      const T f = a[r][c] / a[c][c];
      for (int j = c; j < 4; ++j) a[r][j] -= f * a[c][j];
      for (int j = 0; j < 4; ++j) b[r][j] -= f * b[c][j];
    }
  }
  M4<T> R;
  for (int j = 0; j < 4; ++j)
    for (int r = 3; r >= 0; --r) {
      T s = b[r][j];
      for (int k = r + 1; k < 4; ++k) s -= a[r][k] * R.m[k][j];
      R.m[r][j] = s / a[r][r];
    }
  return R;
}
template <typename T> M4<T> camera_matrix(T fx, T fy, T cx, T cy) {
  M4<T> K = {{{fx, 0, cx, 0}, {0, fy, cy, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  return K;
}
template <typename T> M4<T> inverse_camera_matrix(T fx, T fy, T cx, T cy) {
  M4<T> K = {{{T(1) / fx, 0, -cx / fx, 0}, {0, T(1) / fy, -cy / fy, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}};
  return K;
}

// GR_SVD<6,6>::backsub(b, 1e6) restated: symmetric eigen-decomposition of the
// PSD normal matrix by cyclic Jacobi rotations (its singular values), then the
// pseudo-inverse with singular values below sigma_max / condition dropped.
void solve6_pinv(const double A[6][6], const double b[6], double condition, double x[6]);
// SE(3) exponential of (v, w), translation first (TooN SE3 convention).
void se3_exp(const double xi[6], double T[4][4]);

struct TrackParams {
  int W, H;
  float k[4];
  int levels;
  int iters[4];
  int robust;       // 0 none, 1 huber, 2 tukey, 3 cauchy
  bool use_icp, use_rgb;
};

// Tracking state of one camera stream (apps/kfusion/src/cpp/tracking/tracking.h:34-409).
template <typename T>
struct Tracker {
  TrackParams p;
  std::vector<int> lw, lh;
  std::vector<std::vector<T>> l_D, l_I, r_I, gx, gy;
  std::vector<std::vector<V3<T>>> l_vertex, l_normal, cov, r_vertex_live, r_vertex_render;
  std::vector<std::vector<T>> r_D_render;
  std::vector<std::vector<uint8_t>> icp_mask;  // outlier mask per level (0 = keep)
  T gaussian[5];
  T sigma_bright;
  // last reduction per level (for tests), 32 values
  std::vector<std::vector<double>> last_sums;
  int last_iterations[4];
  std::vector<int8_t> last_result;  // level-0 row codes of the last evaluation

  void init(const TrackParams& prm);
  void set_frame(const uint8_t* rgb, const float* depth);   // rgb2intensity + set_params_frame
  void set_ref_from_current();                               // setRefImgFromCurr
  void set_outlier_mask(const uint8_t* mask);                // trackLiveFrame(..., mask)
  void render_reference(const float* model_vertex, const M4<T>& T_w_r, const int* labels,
                        int label);
  // trackLiveFrame: T_w_l in/out
  void track_camera(M4<T>& T_w_l, const M4<T>& T_w_r, const float* model_vertex,
                    const float* model_normal);
  void camera_sums(int level, const M4<T>& T_w_l, const M4<T>& T_w_r,
                   const std::vector<V3<T>>& MV, const std::vector<V3<T>>& MN,
                   std::vector<double>& s);
  void object_maps(const float* vtx, const float* nrm, const int* labels, int label,
                   std::vector<V3<T>>& MV, std::vector<V3<T>>& MN);
  void object_sums(int level, const M4<T>& T_c2_o2, const M4<T>& T_c1_o1, const M4<T>& T_wo1,
                   const std::vector<V3<T>>& MV, const std::vector<V3<T>>& MN,
                   std::vector<double>& s);
  // trackEachObject: returns the new volume pose T_w_o2
  M4<T> track_object(const M4<T>& T_w_o1, const M4<T>& T_w_c2, const M4<T>& T_w_c1,
                     const float* vertex, const float* normal, const int* labels, int label);
  // Tracking::compute_residuals at level 0 (tracking.cpp:1535-1747): result
  // codes and errors of the ICP rows (first W*H) and photometric rows (next
  // W*H).  model_*: the model maps raycast at T_w_r; live_render_vertex: the
  // model vertices raycast at T_w_l.  Rows that are not computed keep result
  // 0 and error 0.
  void motion_residuals(const M4<T>& T_w_l, const M4<T>& T_w_r, const float* model_vertex,
                        const float* model_normal, const float* live_render_vertex,
                        float threshold, int8_t* result, float* error) const;
};

// check_static_state (rendering.cpp:907-947) and the inlier ratio of
// kfusion.cpp:312-320 for the pixels of `labels` equal to `label`: -1 when
// the label holds no pixel (the reference computes no ratio then).
float inlier_ratio(const int8_t* result, const int* labels, int label, int n, bool use_icp,
                   bool use_rgb);
// Object::refine_mask_use_motion (object.cpp:255-315), outliers not absorbed.
void refine_mask_use_motion(float* mask, const int8_t* result, int n, bool use_icp,
                            bool use_rgb);

}  // namespace ort

// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
// Restatement of the reference tracking path; see or_track.hpp.
#include "or_track.hpp"
#include <algorithm>
#include <cstring>
#include <limits>

namespace ort {

static const float INVALID = -2;

// ----------------------------------------------------------------- solve / exp
void solve6_pinv(const double Ain[6][6], const double b[6], double condition, double x[6]) {
  double A[6][6], V[6][6];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) { A[i][j] = Ain[i][j]; V[i][j] = i == j ? 1.0 : 0.0; }
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int p = 0; p < 6; ++p) for (int q = p + 1; q < 6; ++q) off += A[p][q] * A[p][q];
    if (off < 1e-300) break;
    for (int p = 0; p < 6; ++p)
      for (int q = p + 1; q < 6; ++q) {
        if (A[p][q] == 0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 6; ++k) {  // A <- A J
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq; A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 6; ++k) {  // A <- J^T A
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
  for (int i = 0; i < 6; ++i) smax = std::max(smax, std::fabs(A[i][i]));
  for (int i = 0; i < 6; ++i) x[i] = 0;
  for (int k = 0; k < 6; ++k) {
    const double sk = std::fabs(A[k][k]);
    if (!(sk > smax / condition) || sk == 0) continue;
    double vb = 0;
    for (int i = 0; i < 6; ++i) vb += V[i][k] * b[i];
    const double coef = vb / A[k][k];
    for (int i = 0; i < 6; ++i) x[i] += coef * V[i][k];
  }
}

void se3_exp(const double xi[6], double T[4][4]) {
  const double v[3] = {xi[0], xi[1], xi[2]}, w[3] = {xi[3], xi[4], xi[5]};
  const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double A, B, C;
  if (th2 < 1e-10) {
    A = 1 - th2 / 6; B = 0.5 - th2 / 24; C = 1.0 / 6 - th2 / 120;
  } else {
    const double th = std::sqrt(th2);
    A = std::sin(th) / th; B = (1 - std::cos(th)) / th2; C = (1 - A) / th2;
  }
  const double W[3][3] = {{0, -w[2], w[1]}, {w[2], 0, -w[0]}, {-w[1], w[0], 0}};
  double W2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) W2[i][j] = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
  for (int i = 0; i < 3; ++i) {
    double t = 0;
    for (int j = 0; j < 3; ++j) {
      const double I = i == j ? 1.0 : 0.0;
      T[i][j] = I + A * W[i][j] + B * W2[i][j];
      t += (I + B * W[i][j] + C * W2[i][j]) * v[j];
    }
    T[i][3] = t;
  }
  T[3][0] = T[3][1] = T[3][2] = 0; T[3][3] = 1;
}

// ----------------------------------------------------------------- helpers
// The reference squares through math_utils.h:92 `float sq(float)`: its Tukey
// and Cauchy terms round r / b (a double) and 1 - r^2 / b^2 to float and
// square them in float.  The FP32 oracle (T = float) keeps those roundings;
// the FP64 oracle squares in double.
template <typename T> static double sq_ref(double x) {
  if (sizeof(T) == sizeof(float)) { const float f = (float)x; return (double)(f * f); }
  return x * x;
}
template <typename T> static T robust_weight(T e, int kind) {  // tracking.cpp:1504-1532
  double w = 1.0;
  const double r = e;
  switch (kind) {
    case 1: w = std::fabs(r) <= 1.345 ? 1.0 : 1.345 / std::fabs(r); break;
    case 2:
      if (std::fabs(r) <= 4.6851) {
        // sq(1.0 - sq(residual) / sq(tukey_b)): float quotient of float squares
        const double q = sizeof(T) == sizeof(float)
                             ? (double)((float)sq_ref<T>(r) / (float)sq_ref<T>(4.6851))
                             : r * r / (4.6851 * 4.6851);
        w = sq_ref<T>(1.0 - q);
      } else {
        w = 0.0;
      }
      break;
    case 3:
      // 1 / (1 + sq(residual / cauchy_k)): int + float and the quotient in float
      w = sizeof(T) == sizeof(float) ? (double)(1.f / (1.f + (float)sq_ref<T>(r / 2.3849)))
                                     : 1 / (1 + sq_ref<T>(r / 2.3849));
      break;
    default: break;
  }
  return (T)w;
}
template <typename T> static T robust_loss(T e, int kind) {  // tracking.cpp:1474-1502
  double l = 0;
  const double r = e;
  switch (kind) {
    case 1: l = std::fabs(r) <= 1.345 ? 0.5 * r * r : 1.345 * (std::fabs(r) - 0.5 * 1.345); break;
    case 2: {
      const double b = 4.6851;
      l = std::fabs(r) <= b ? b * b / 6.0 * (1.0 - std::pow(1.0 - sq_ref<T>(r / b), 3)) : b * b / 6.0;
      break;
    }
    case 3: l = 0.5 * 2.3849 * 2.3849 * std::log(1.0 + sq_ref<T>(r / 2.3849)); break;
    default: l = 0.5 * r * r;
  }
  return (T)l;
}

template <typename T> static T bil(const T* img, int w, T px, T py) {
  const int bx = (int)std::floor(px), by = (int)std::floor(py);
  const T fx = px - std::floor(px), fy = py - std::floor(py);
  return img[bx + by * w] * (T(1) - fx) * (T(1) - fy) + img[bx + 1 + by * w] * (T(1) - fy) * fx +
         img[bx + (by + 1) * w] * (T(1) - fx) * fy + img[bx + 1 + (by + 1) * w] * fx * fy;
}
template <typename T> static V3<T> bil3(const V3<T>* img, int w, T px, T py) {
  const int bx = (int)std::floor(px), by = (int)std::floor(py);
  const T fx = px - std::floor(px), fy = py - std::floor(py);
  const T a = T(1) - fx, b = T(1) - fy;
  const V3<T> v0 = img[bx + by * w], v1 = img[bx + 1 + by * w], v2 = img[bx + (by + 1) * w],
              v3_ = img[bx + 1 + (by + 1) * w];
  return v3(v0.x * a * b + v1.x * b * fx + v2.x * a * fy + v3_.x * fx * fy,
            v0.y * a * b + v1.y * b * fx + v2.y * a * fy + v3_.y * fx * fy,
            v0.z * a * b + v1.z * b * fx + v2.z * a * fy + v3_.z * fx * fy);
}

template <typename T> static T kexp(T v);
template <> float kexp<float>(float v) { return expf(v); }
template <> double kexp<double>(double v) { return std::exp(v); }

// preprocessing.cpp:11-50
template <typename T>
static void bilateral(std::vector<T>& out, const std::vector<T>& in, int W, int H,
                      const T* gaussian, T e_d, int r) {
  const T e2 = e_d * e_d * 2;
  out.assign((size_t)W * H, T(0));
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int pos = x + y * W;
      if (in[pos] == 0) { out[pos] = 0; continue; }
      T sum = 0, t = 0;
      const T center = in[pos];
      for (int i = -r; i <= r; ++i)
        for (int j = -r; j <= r; ++j) {
          const int cx = std::min(std::max(x + i, 0), W - 1), cy = std::min(std::max(y + j, 0), H - 1);
          const T cur = in[cx + cy * W];
          if (cur > 0) {
            const T mod = (cur - center) * (cur - center);
            const T factor = gaussian[i + r] * gaussian[j + r] * kexp<T>(-mod / e2);
            t += factor * cur;
            sum += factor;
          }
        }
      out[pos] = t / sum;
    }
}
// preprocessing.cpp:161-196
template <typename T>
static void half_sample(std::vector<T>& out, const std::vector<T>& in, int iw, int ih, T e_d, int r) {
  const int ow = iw / 2, oh = ih / 2;
  out.assign((size_t)ow * oh, T(0));
  for (int y = 0; y < oh; ++y)
    for (int x = 0; x < ow; ++x) {
      const int cx = 2 * x, cy = 2 * y;
      T sum = 0, t = 0;
      const T center = in[cx + cy * iw];
      for (int i = -r + 1; i <= r; ++i)
        for (int j = -r + 1; j <= r; ++j) {
          const int ux = std::min(std::max(cx + j, 0), 2 * ow - 1);
          const int uy = std::min(std::max(cy + i, 0), 2 * oh - 1);
          const T cur = in[ux + uy * iw];
          if (std::fabs(cur - center) < e_d) { sum += 1; t += cur; }
        }
      out[x + y * ow] = t / sum;
    }
}
// preprocessing.cpp:52-71
template <typename T>
static void depth2vertex(std::vector<V3<T>>& v, const std::vector<T>& d, int W, int H,
                         const M4<T>& invK) {
  v.assign((size_t)W * H, v3<T>(0, 0, 0));
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const T dd = d[x + y * W];
      v[x + y * W] = dd > 0 ? dd * rotate(invK, v3<T>((T)x, (T)y, T(1))) : v3<T>(0, 0, 0);
    }
}
// preprocessing.h:39-81 (SDF field): only .x is set on invalid pixels; the
// others keep the previous frame's values in the reference buffer.  NegY (a
// negative fy, the ICL-NUIM convention, tracking.cpp:805-810) swaps the rows
// taken as up and down.
template <typename T>
static void vertex2normal(std::vector<V3<T>>& out, const std::vector<V3<T>>& in, int W, int H,
                          bool negy) {
  if (out.size() != (size_t)W * H) out.assign((size_t)W * H, v3<T>(0, 0, 0));
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const V3<T> left = in[std::max(x - 1, 0) + W * y], right = in[std::min(x + 1, W - 1) + W * y];
      const int ylo = std::max(y - 1, 0), yhi = std::min(y + 1, H - 1);
      const V3<T> down = in[x + W * (negy ? yhi : ylo)], up = in[x + W * (negy ? ylo : yhi)];
      if (left.z == 0 || right.z == 0 || up.z == 0 || down.z == 0) {
        out[x + y * W].x = INVALID;
        continue;
      }
      out[x + y * W] = normalize(cross(up - down, right - left));
    }
}
// preprocessing.cpp:235-246 (borders stay 0)
template <typename T>
static void gradients(std::vector<T>& gx, std::vector<T>& gy, const std::vector<T>& in, int W, int H) {
  gx.assign((size_t)W * H, T(0));
  gy.assign((size_t)W * H, T(0));
  for (int y = 1; y < H - 1; ++y)
    for (int x = 1; x < W - 1; ++x) {
      gx[x + W * y] = (in[x + 1 + W * y] - in[x - 1 + W * y]) * T(0.5);
      gy[x + W * y] = (in[x + W * (y + 1)] - in[x + W * (y - 1)]) * T(0.5);
    }
}

template <typename T> static M4<T> from_f(const float* p) {
  M4<T> m; for (int i = 0; i < 16; ++i) m.m[i / 4][i % 4] = (T)p[i]; return m;
}

// ----------------------------------------------------------------- Tracker
template <typename T> void Tracker<T>::init(const TrackParams& prm) {
  p = prm;
  lw.clear(); lh.clear();
  for (int l = 0; l < p.levels; ++l) { lw.push_back(p.W >> l); lh.push_back(p.H >> l); }
  const size_t L = p.levels;
  l_D.assign(L, {}); l_I.assign(L, {}); r_I.assign(L, {}); gx.assign(L, {}); gy.assign(L, {});
  l_vertex.assign(L, {}); l_normal.assign(L, {}); cov.assign(L, {}); r_vertex_live.assign(L, {});
  r_vertex_render.assign(L, {}); r_D_render.assign(L, {}); icp_mask.assign(L, {});
  for (size_t l = 0; l < L; ++l) {
    const size_t n = (size_t)lw[l] * lh[l];
    r_I[l].assign(n, T(0)); r_vertex_live[l].assign(n, v3<T>(0, 0, 0)); icp_mask[l].assign(n, 0);
  }
  // tracking.cpp:77-84: x = i - 2, delta = 4
  for (int i = 0; i < 5; ++i) {
    const int x = i - 2;
    gaussian[i] = kexp<T>(-(T)(x * x) / (T)(2 * 4.0f * 4.0f));
  }
  // obtainErrorParameters (TUM branch), tracking.cpp:766-772: float member
  sigma_bright = (T)(float)(sqrtf(100.0) / 255.0);
  if (sizeof(T) == 8) sigma_bright = (T)(10.0 / 255.0);
  last_sums.assign(L, std::vector<double>(32, 0.0));
}

template <typename T> void Tracker<T>::set_frame(const uint8_t* rgb, const float* depth) {
  const int W = p.W, H = p.H;
  std::vector<T> grey((size_t)W * H), dep((size_t)W * H);
  for (int i = 0; i < W * H; ++i) {
    const T r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
    grey[i] = (T(0.299f) * r + T(0.587f) * g + T(0.114f) * b) / T(255.f);  // commons.h:150-154
    dep[i] = depth[i];
  }
  const T e_delta = T(0.1f);
  for (int l = 0; l < p.levels; ++l) {
    if (l == 0) {
      bilateral(l_I[0], grey, W, H, gaussian, T(0.1f), 2);
      bilateral(l_D[0], dep, W, H, gaussian, T(0.1f), 2);
    } else {
      half_sample(l_D[l], l_D[l - 1], lw[l - 1], lh[l - 1], T(e_delta * 3), 1);
      half_sample(l_I[l], l_I[l - 1], lw[l - 1], lh[l - 1], T(e_delta * 3), 1);
    }
    const T d = T(1 << l);
    const M4<T> invK = inverse_camera_matrix<T>(T(p.k[0]) / d, T(p.k[1]) / d, T(p.k[2]) / d, T(p.k[3]) / d);
    depth2vertex(l_vertex[l], l_D[l], lw[l], lh[l], invK);
    vertex2normal(l_normal[l], l_vertex[l], lw[l], lh[l], p.k[1] < 0);
    gradients(gx[l], gy[l], l_I[l], lw[l], lh[l]);
    // calc_icp_cov, tracking.cpp:845-871 (sigma_xy = sigma_disp = 1, baseline 0.075)
    const T focal = T(p.k[0]) / d, baseline = T(0.075f);
    cov[l].assign((size_t)lw[l] * lh[l], v3<T>(0, 0, 0));
    for (size_t i = 0; i < cov[l].size(); ++i) {
      const T z = l_D[l][i];
      V3<T> c;
      c.x = (z / focal) * T(1); c.y = (z / focal) * T(1);
      c.z = (z * z * T(1)) / (focal * baseline);
      c.x = c.x * c.x; c.y = c.y * c.y; c.z = c.z * c.z;
      cov[l][i] = c;
    }
    std::fill(icp_mask[l].begin(), icp_mask[l].end(), 0);
  }
}

template <typename T> void Tracker<T>::set_ref_from_current() {
  for (int l = 0; l < p.levels; ++l) { r_I[l] = l_I[l]; r_vertex_live[l] = l_vertex[l]; }
}

template <typename T> void Tracker<T>::set_outlier_mask(const uint8_t* mask) {
  // cv::resize(mask, size / 2^l): level 1 is INTER_AREA over 2x2 (any nonzero
  // stays nonzero), level l >= 2 is INTER_LINEAR, whose two taps per axis sit at
  // 2^l x + 2^(l-1) - 1 and 2^l x + 2^(l-1).
  for (int l = 0; l < p.levels; ++l)
    for (int y = 0; y < lh[l]; ++y)
      for (int x = 0; x < lw[l]; ++x) {
        uint8_t v;
        if (l == 0) v = mask[x + y * p.W];
        else {
          const int o = l == 1 ? 0 : (1 << (l - 1)) - 1, s = 1 << l;
          v = 0;
          for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
              v |= mask[(s * x + o + dx) + (s * y + o + dy) * p.W];
        }
        icp_mask[l][x + y * lw[l]] = v ? 1 : 0;
      }
}

template <typename T>
void Tracker<T>::render_reference(const float* model_vertex, const M4<T>& T_w_r,
                                  const int* labels, int label) {
  // tracking.cpp:218-238 / :608-627: vertex2depth + depth2vertex, then robust
  // half-sampling of the rendered depth.
  const int W = p.W, H = p.H;
  r_D_render[0].assign((size_t)W * H, T(0));
  const M4<T> inv = inverse(T_w_r);
  for (int i = 0; i < W * H; ++i) {
    V3<T> v = v3<T>(model_vertex[3 * i], model_vertex[3 * i + 1], model_vertex[3 * i + 2]);
    if (labels && labels[i] != label) v = v3<T>(0, 0, 0);  // per-object model map
    r_D_render[0][i] = v.z > 0.0 ? xform(inv, v).z : T(0);  // preprocessing.cpp:292-309
  }
  for (int l = 0; l < p.levels; ++l) {
    if (l > 0) half_sample(r_D_render[l], r_D_render[l - 1], lw[l - 1], lh[l - 1], T(T(0.1f) * 3), 1);
    const T d = T(1 << l);
    depth2vertex(r_vertex_render[l], r_D_render[l], lw[l], lh[l],
                 inverse_camera_matrix<T>(T(p.k[0]) / d, T(p.k[1]) / d, T(p.k[2]) / d, T(p.k[3]) / d));
  }
}

struct Row { int result; double error; double J[6]; };

// tracking.cpp:1191-1352 (8 row blocks; then values[0] += values[j]).
template <typename T>
static void reduce(std::vector<double>& out, const std::vector<Row>& icp, const std::vector<Row>& rgb,
                   int w, int h, int robust, bool use_icp, bool use_rgb) {
  T blocks[8][32];
  for (int b = 0; b < 8; ++b) {
    T s[32];
    for (int i = 0; i < 32; ++i) s[i] = 0;
    for (int y = b; y < h; y += 8)
      for (int x = 0; x < w; ++x)
        for (int k = 0; k < 2; ++k) {
          if ((k == 0 && !use_icp) || (k == 1 && !use_rgb)) continue;
          const Row& r = (k == 0 ? icp : rgb)[x + y * w];
          if (r.result < 1) {
            s[29] += r.result == -4 ? 1 : 0;
            s[30] += r.result == -5 ? 1 : 0;
            s[31] += r.result > -4 ? 1 : 0;
            continue;
          }
          const T e = (T)r.error;
          T J[6];
          for (int i = 0; i < 6; ++i) J[i] = (T)r.J[i];
          const T wgt = robust_weight<T>(e, robust);
          s[0] += robust_loss<T>(e, robust);
          for (int i = 0; i < 6; ++i) s[1 + i] += wgt * e * J[i];
          int q = 7;
          for (int i = 0; i < 6; ++i)
            for (int j = i; j < 6; ++j) s[q++] += wgt * J[i] * J[j];
          s[28] += 1;
        }
    for (int i = 0; i < 32; ++i) blocks[b][i] = s[i];
  }
  for (int j = 1; j < 8; ++j)
    for (int i = 0; i < 32; ++i) blocks[0][i] += blocks[j][i];
  out.assign(32, 0.0);
  for (int i = 0; i < 32; ++i) out[i] = blocks[0][i];
}

// commons.h:673-696 (makeJTJ + solve) and tracking.cpp:1354-1374.
template <typename T>
static bool solve_pose(const std::vector<double>& s, M4<T>& update) {
  double A[6][6], b[6], x[6];
  for (int i = 0; i < 6; ++i) b[i] = (T)s[1 + i];
  int q = 7;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) { A[i][j] = A[j][i] = (T)s[q]; ++q; }
  solve6_pinv(A, b, 1e6, x);
  double E[4][4];
  se3_exp(x, E);
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) update.m[i][j] = (T)E[i][j];
  double nx = 0;
  for (int i = 0; i < 6; ++i) nx += x[i] * x[i];
  nx = std::sqrt(nx);
  const T ratio = (T)s[0] / (T)s[28];
  return nx < (double)1e-05f && (double)std::sqrt(ratio) < 2e-3;
}

// trackingResult_[0] after the last level-0 evaluation: the codes of the
// ICP rows, then of the photometric rows (0 for a term that is off)
static void keep_codes(std::vector<int8_t>& out, const std::vector<Row>& icp,
                       const std::vector<Row>& rgb, bool use_icp, bool use_rgb) {
  const size_t n = icp.size();
  out.assign(2 * n, 0);
  for (size_t i = 0; i < n; ++i) {
    out[i] = use_icp ? (int8_t)icp[i].result : 0;
    out[n + i] = use_rgb ? (int8_t)rgb[i].result : 0;
  }
}

template <typename T>
void Tracker<T>::camera_sums(int level, const M4<T>& T_w_l, const M4<T>& T_w_r,
                             const std::vector<V3<T>>& MV, const std::vector<V3<T>>& MN,
                             std::vector<double>& s) {
  const int W = p.W;
  const M4<T> K = camera_matrix<T>(p.k[0], p.k[1], p.k[2], p.k[3]);
  const M4<T> view = mul(K, inverse(T_w_r));
  const T inv_cov_rgb = sizeof(T) == 4 ? (T)(float)(1.0 / (double)sigma_bright) : T(1) / sigma_bright;
  const int w = lw[level], h = lh[level];
  const T dl = T(1 << level);
  const M4<T> KL = camera_matrix<T>(T(p.k[0]) / dl, T(p.k[1]) / dl, T(p.k[2]) / dl, T(p.k[3]) / dl);
  std::vector<Row> icp((size_t)w * h), rgb((size_t)w * h);
  const M4<T> inv_l = inverse(T_w_l);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const int i = x + y * w;
      Row& r = icp[i];
      r.result = 0;
      // track_ICP_Kernel, tracking.cpp:923-1020
      if (icp_mask[level][i]) { r.result = -6; }
      else if (l_normal[level][i].x == INVALID) { r.result = -1; }
      else {
        const V3<T> pv = xform(T_w_l, l_vertex[level][i]);
        const V3<T> pp = xform(view, pv);
        const T px = pp.x / pp.z, py = pp.y / pp.z;
        if (px < 1 || px > (T)(unsigned)(W - 2) || py < 1 || py > (T)(unsigned)(p.H - 2) ||
            std::isnan(px) || std::isnan(py)) { r.result = -2; }
        else {
          const unsigned rx = (unsigned)px, ry = (unsigned)py;
          const V3<T> rn = MN[rx + ry * W];
          if (rn.x == INVALID) { r.result = -3; }
          else {
            const V3<T> diff = MV[rx + ry * W] - pv;
            const V3<T> pn = rotate(T_w_l, l_normal[level][i]);
            if (length(diff) > T(0.1f)) r.result = -4;
            else if (dot(pn, rn) < T(0.8f)) r.result = -5;
            else {
              r.result = 1;
              const V3<T> P = cov[level][i];
              const T sig = rn.x * rn.x * P.x + rn.y * rn.y * P.y + rn.z * rn.z * P.z;
              const T ic = sizeof(T) == 4 ? (T)sqrtf((float)(1.0 / (double)sig)) : std::sqrt(T(1) / sig);
              r.error = ic * dot(rn, diff);
              const V3<T> j1 = ic * cross(pv, rn);
              r.J[0] = ic * rn.x; r.J[1] = ic * rn.y; r.J[2] = ic * rn.z;
              r.J[3] = j1.x; r.J[4] = j1.y; r.J[5] = j1.z;
            }
          }
        }
      }
      // trackRGB, tracking.cpp:1023-1111
      Row& g = rgb[i];
      g.result = 0;
      const V3<T> rv = r_vertex_render[level][i], rl = r_vertex_live[level][i];
      if (rv.z <= 0 || rv.z == INVALID) { g.result = -1; continue; }
      if (length(rv - rl) > T(0.1f) && rl.z > 0) { g.result = -3; continue; }
      const V3<T> wv = xform(T_w_r, rv);
      const V3<T> lv = xform(inv_l, wv);
      const V3<T> pr = rotate(KL, lv);
      const T px = pr.x / pr.z, py = pr.y / pr.z;
      if (px < 1 || px > (T)(unsigned)(w - 2) || py < 1 || py > (T)(unsigned)(h - 2) ||
          std::isnan(px) || std::isnan(py)) { g.result = -2; continue; }
      const T residual = r_I[level][i] - bil(l_I[level].data(), w, px, py);
      const T gxv = bil(gx[level].data(), w, px, py), gyv = bil(gy[level].data(), w, px, py);
      const T fx = KL.m[0][0], fy = KL.m[1][1];
      V3<T> Jt = (T(1) / lv.z) * v3<T>(gxv * fx, gyv * fy, -(gxv * lv.x * fx + gyv * lv.y * fy) / lv.z);
      Jt = T(-1) * rotate(T_w_l, Jt);
      const V3<T> Jr = cross(wv, Jt);
      g.J[0] = inv_cov_rgb * Jt.x; g.J[1] = inv_cov_rgb * Jt.y; g.J[2] = inv_cov_rgb * Jt.z;
      g.J[3] = inv_cov_rgb * Jr.x; g.J[4] = inv_cov_rgb * Jr.y; g.J[5] = inv_cov_rgb * Jr.z;
      g.error = inv_cov_rgb * residual;
      g.result = 1;
    }
  if (level == 0) keep_codes(last_result, icp, rgb, p.use_icp, p.use_rgb);
  reduce<T>(s, icp, rgb, w, h, p.robust, p.use_icp, p.use_rgb);
}

template <typename T>
void Tracker<T>::track_camera(M4<T>& T_w_l, const M4<T>& T_w_r, const float* mv,
                              const float* mn) {
  std::vector<V3<T>> MV((size_t)p.W * p.H), MN((size_t)p.W * p.H);
  for (size_t i = 0; i < MV.size(); ++i) {
    MV[i] = v3<T>(mv[3 * i], mv[3 * i + 1], mv[3 * i + 2]);
    MN[i] = v3<T>(mn[3 * i], mn[3 * i + 1], mn[3 * i + 2]);
  }
  M4<T> previous_pose = T_w_l, update;
  for (int level = p.levels - 1; level >= 0; --level) {
    double previous_error = std::numeric_limits<double>::infinity();
    last_iterations[level] = 0;
    for (int it = 0; it < p.iters[level]; ++it) {
      last_iterations[level] = it + 1;
      std::vector<double> s;
      camera_sums(level, T_w_l, T_w_r, MV, MN, s);
      last_sums[level] = s;
      const T current_error = (T)s[0] / (T)s[28];
      if ((double)current_error > previous_error) { T_w_l = previous_pose; break; }
      previous_error = current_error;
      if (solve_pose<T>(s, update)) break;
      previous_pose = T_w_l;
      T_w_l = mul(update, previous_pose);
    }
  }
}

template <typename T>
void Tracker<T>::object_maps(const float* vtx, const float* nrm, const int* labels, int label,
                             std::vector<V3<T>>& MV, std::vector<V3<T>>& MN) {
  const int n = p.W * p.H;
  MV.resize(n); MN.resize(n);
  for (int i = 0; i < n; ++i) {  // Object::m_vertex / m_normal, rendering.cpp:153-178
    if (labels[i] == label) {
      MV[i] = v3<T>(vtx[3 * i], vtx[3 * i + 1], vtx[3 * i + 2]);
      MN[i] = v3<T>(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    } else {
      MV[i] = v3<T>(0, 0, 0);
      MN[i] = v3<T>(INVALID, 0, 0);
    }
  }
}

template <typename T>
void Tracker<T>::object_sums(int level, const M4<T>& T_c2_o2, const M4<T>& T_c1_o1,
                             const M4<T>& T_wo1, const std::vector<V3<T>>& MV,
                             const std::vector<V3<T>>& MN, std::vector<double>& s) {
  const int W = p.W, H = p.H;
  const M4<T> K = camera_matrix<T>(p.k[0], p.k[1], p.k[2], p.k[3]);
  const M4<T> inv_wo1 = inverse(T_wo1), inv_c1o1 = inverse(T_c1_o1);
  const T inv_cov_rgb = sizeof(T) == 4 ? (T)(float)(1.0 / (double)sigma_bright) : T(1) / sigma_bright;
  const int w = lw[level], h = lh[level];
  const T dl = T(1 << level);
  const M4<T> KL = camera_matrix<T>(T(p.k[0]) / dl, T(p.k[1]) / dl, T(p.k[2]) / dl, T(p.k[3]) / dl);
  std::vector<Row> icp((size_t)w * h), rgb((size_t)w * h);
  const M4<T> inv_c2o2 = inverse(T_c2_o2);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const int i = x + y * w;
      // track_Obj_ICP_Kernel, tracking.cpp:392-486 (outlier mask: all zero)
      Row& r = icp[i];
      r.result = 0;
      const V3<T> cn = l_normal[level][i], cv = l_vertex[level][i];
      if (cn.x == INVALID) r.result = -1;
      else if (cv.x == 0 && cv.y == 0 && cv.z == 0) r.result = -1;
      else {
        const V3<T> o2v = xform(inv_c2o2, cv);
        const V3<T> c1v = xform(T_c1_o1, o2v);
        const V3<T> pr = rotate(K, c1v);
        const T px = pr.x / pr.z, py = pr.y / pr.z;
        if (px < 1 || px > (T)(unsigned)(W - 2) || py < 1 || py > (T)(unsigned)(H - 2) ||
            std::isnan(px) || std::isnan(py)) r.result = -2;
        else {
          const V3<T> o2n = rotate(inv_c2o2, cn);
          const V3<T> wrv = bil3(MV.data(), W, px, py), wrn = bil3(MN.data(), W, px, py);
          if (wrn.x == INVALID) r.result = -3;
          else {
            const V3<T> o1rv = xform(inv_wo1, wrv);
            const V3<T> o1rn = rotate(inv_wo1, wrn);
            const V3<T> diff = o2v - o1rv;
            const T residual = dot(o1rn, diff);
            if (length(diff) > T(0.1f)) r.result = -4;
            else if (dot(o2n, o1rn) < T(0.8f)) r.result = -5;
            else {
              const V3<T> P = cov[level][i];
              const T sig = o1rn.x * o1rn.x * P.x + o1rn.y * o1rn.y * P.y + o1rn.z * o1rn.z * P.z;
              const T ic = sizeof(T) == 4 ? (T)sqrtf((float)(1.0 / (double)sig)) : std::sqrt(T(1) / sig);
              r.error = ic * residual;
              const V3<T> Jt = rotate(T_c2_o2, o1rn);
              const T c0 = T(-1) * ic * T(-1);
              const V3<T> j1 = ic * cross(cv, Jt);
              r.J[0] = c0 * Jt.x; r.J[1] = c0 * Jt.y; r.J[2] = c0 * Jt.z;
              r.J[3] = j1.x; r.J[4] = j1.y; r.J[5] = j1.z;
              r.result = 1;
            }
          }
        }
      }
      // track_obj_RGB_kernel, tracking.cpp:491-578
      Row& g = rgb[i];
      g.result = 0;
      const V3<T> rv = r_vertex_render[level][i], rl = r_vertex_live[level][i];
      if (rv.z <= 0 || rv.z == INVALID) { g.result = -1; continue; }
      if (length(rv - rl) > T(0.1f) && rl.z > 0) { g.result = -3; continue; }
      const V3<T> o1v = xform(inv_c1o1, rv);
      const V3<T> c2v = xform(T_c2_o2, o1v);
      const V3<T> pr = rotate(KL, c2v);
      const T px = pr.x / pr.z, py = pr.y / pr.z;
      if (px < 1 || px > (T)(unsigned)(w - 2) || py < 1 || py > (T)(unsigned)(h - 2) ||
          std::isnan(px) || std::isnan(py)) { g.result = -2; continue; }
      const T residual = r_I[level][i] - bil(l_I[level].data(), w, px, py);
      const T gxv = bil(gx[level].data(), w, px, py), gyv = bil(gy[level].data(), w, px, py);
      const T fx = KL.m[0][0], fy = KL.m[1][1];
      const V3<T> Jt = (T(1) / c2v.z) * v3<T>(gxv * fx, gyv * fy, -(gxv * c2v.x * fx + gyv * c2v.y * fy) / c2v.z);
      const V3<T> Jr = cross(c2v, Jt);
      g.J[0] = inv_cov_rgb * Jt.x; g.J[1] = inv_cov_rgb * Jt.y; g.J[2] = inv_cov_rgb * Jt.z;
      g.J[3] = inv_cov_rgb * Jr.x; g.J[4] = inv_cov_rgb * Jr.y; g.J[5] = inv_cov_rgb * Jr.z;
      g.error = inv_cov_rgb * residual;
      g.result = 1;
    }
  if (level == 0) keep_codes(last_result, icp, rgb, p.use_icp, p.use_rgb);
  reduce<T>(s, icp, rgb, w, h, p.robust, p.use_icp, p.use_rgb);
}

template <typename T>
M4<T> Tracker<T>::track_object(const M4<T>& T_wo1, const M4<T>& T_w_c2, const M4<T>& T_w_c1,
                               const float* vtx, const float* nrm, const int* labels, int label) {
  std::vector<V3<T>> MV, MN;
  object_maps(vtx, nrm, labels, label, MV, MN);
  render_reference(vtx, T_w_c1, labels, label);
  const M4<T> T_c1_o1 = mul(inverse(T_w_c1), T_wo1);
  M4<T> T_c2_o2 = mul(inverse(T_w_c2), T_wo1);
  M4<T> previous_pose = T_c2_o2, update;
  for (int level = p.levels - 1; level >= 0; --level) {
    double previous_error = std::numeric_limits<double>::infinity();
    last_iterations[level] = 0;
    for (int it = 0; it < p.iters[level]; ++it) {
      last_iterations[level] = it + 1;
      std::vector<double> s;
      object_sums(level, T_c2_o2, T_c1_o1, T_wo1, MV, MN, s);
      last_sums[level] = s;
      const T current_error = (T)s[0] / (T)s[28];
      if (s[28] == 0) break;
      if ((double)current_error > previous_error) { T_c2_o2 = previous_pose; break; }
      previous_error = current_error;
      if (solve_pose<T>(s, update)) break;
      previous_pose = T_c2_o2;
      T_c2_o2 = mul(update, previous_pose);
    }
  }
  return mul(T_w_c2, T_c2_o2);
}

template <typename T>
void Tracker<T>::motion_residuals(const M4<T>& T_w_l, const M4<T>& T_w_r,
                                  const float* model_vertex, const float* model_normal,
                                  const float* live_render_vertex, float threshold,
                                  int8_t* result, float* error) const {
  const int W = p.W, H = p.H, n = W * H;
  const M4<T> K = camera_matrix<T>(p.k[0], p.k[1], p.k[2], p.k[3]);
  const M4<T> invK = inverse_camera_matrix<T>(p.k[0], p.k[1], p.k[2], p.k[3]);
  const M4<T> inv_r = inverse(T_w_r);
  auto at = [](const float* a, int q) { return v3<T>(a[3 * q], a[3 * q + 1], a[3 * q + 2]); };
  // warp (tracking.cpp:1114-1121) with T_w_l for the world transform and
  // inverse(T_w_r) for the reference frame; false for pixels outside
  // [1, W-2] x [1, H-2] (and, where the reference's conversion of a NaN
  // coordinate to a pixel index is undefined, for NaN)
  auto warp = [&](V3<T> v, V3<T>& w, T& px, T& py) {
    w = xform(T_w_l, v);
    const V3<T> pr = rotate(K, xform(inv_r, w));
    px = pr.x / pr.z; py = pr.y / pr.z;
    return !(px < 1 || px > (T)(unsigned)(W - 2) || py < 1 || py > (T)(unsigned)(H - 2) ||
             std::isnan(px) || std::isnan(py));
  };
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int i = x + y * W;
      int8_t ri = 0, rr = 0;
      float ei = 0.f, er = 0.f;
      // no row is -6: the reference's outlier_mask_ stays the all-zero mask of
      // set_params_frame (tracking.cpp:170); the mask variant of
      // trackLiveFrame keeps its mask pyramid local (:1781-1787)
      {
        if (p.use_icp) {  // compute_icp_residual_kernel, tracking.cpp:1615-1677
          V3<T> w;
          T px, py;
          if (l_normal[0][i].x == INVALID) ri = -1;
          else if (!warp(l_vertex[0][i], w, px, py)) ri = -2;
          else {
            const int q = (int)((unsigned)px + (unsigned)py * W);
            const V3<T> rn = at(model_normal, q), rv = at(model_vertex, q);
            if (rn.x == INVALID) ri = -3;
            else {
              const V3<T> diff = rv - w;
              const V3<T> wn = rotate(T_w_l, l_normal[0][i]);
              if (length(diff) > T(0.1f)) ri = -4;
              else if (dot(wn, rn) < T(0.8f)) ri = -5;
              else {
                const V3<T> P = cov[0][i];
                const double sig = rn.x * rn.x * P.x + rn.y * rn.y * P.y + rn.z * rn.z * P.z;
                const double e = std::sqrt(1.0 / sig) * dot(rn, diff);
                if (std::fabs(e) > threshold) ri = -4;
                else { ri = 1; ei = (float)e; }
              }
            }
          }
        }
        if (p.use_rgb) {  // compute_rgb_residual_kernel, tracking.cpp:1680-1747
          // vertex2depth with T_w_r (preprocessing.cpp:292-309), depth2vertexKernel
          const V3<T> vl = at(live_render_vertex, i);
          const T d = vl.z > 0.0 ? xform(inv_r, vl).z : T(0);
          const V3<T> ref = d > 0 ? d * rotate(invK, v3<T>((T)x, (T)y, T(1))) : v3<T>(0, 0, 0);
          const V3<T> live = l_vertex[0][i];
          V3<T> w;
          T px, py;
          if (ref.z <= 0 || ref.z == INVALID) rr = -1;
          else if (length(ref - live) > T(0.1f) && live.z > 0) rr = -5;
          else if (!warp(ref, w, px, py)) rr = -2;
          else {
            const T residual = l_I[0][i] - bil(r_I[0].data(), W, px, py);
            const double e = (1.0 / (double)sigma_bright) * residual;
            if (std::fabs(e) > threshold) rr = -4;
            else { rr = 1; er = (float)e; }
          }
        }
      }
      result[i] = ri; result[n + i] = rr;
      error[i] = ei; error[n + i] = er;
    }
}

float inlier_ratio(const int8_t* result, const int* labels, int label, int n, bool use_icp,
                   bool use_rgb) {
  int all = 0, inl = 0;
  for (int i = 0; i < n; ++i) {
    if (labels[i] != label) continue;
    ++all;
    bool ok = false;
    if (use_icp && use_rgb) ok = result[i] > -3 && result[n + i] > -3;
    else if (use_icp) ok = result[i] > -3;
    else if (use_rgb) ok = result[n + i] > -3;
    inl += ok;
  }
  return all ? static_cast<float>(inl) / all : -1.f;
}

void refine_mask_use_motion(float* mask, const int8_t* result, int n, bool use_icp,
                            bool use_rgb) {
  for (int i = 0; i < n; ++i) {
    if (!(mask[i] >= 0)) continue;
    if (use_icp && (result[i] == -4 || result[i] == -6)) { mask[i] = -1; continue; }
    if (use_rgb && result[n + i] < -3) mask[i] = -1;
  }
}

template struct Tracker<float>;
template struct Tracker<double>;

}  // namespace ort

// TEST INFRASTRUCTURE ONLY — C ABI of the CPU tracking oracle.
#include <cstring>
#include "or_track.hpp"

using namespace ort;

namespace {
struct Handle {
  bool fp64;
  Tracker<float> f;
  Tracker<double> d;
};
template <typename T> M4<T> ld(const float* p) {
  M4<T> m; for (int i = 0; i < 16; ++i) m.m[i / 4][i % 4] = (T)p[i]; return m;
}
template <typename T> void st(float* p, const M4<T>& m) {
  for (int i = 0; i < 16; ++i) p[i] = (float)m.m[i / 4][i % 4];
}
template <typename T> void std_(double* p, const M4<T>& m) {
  for (int i = 0; i < 16; ++i) p[i] = (double)m.m[i / 4][i % 4];
}
}  // namespace

extern "C" {

void* ot_create(int W, int H, const float* k, int levels, const int* iters, int robust,
                int use_icp, int use_rgb, int fp64) {
  Handle* h = new Handle;
  h->fp64 = fp64 != 0;
  TrackParams p;
  p.W = W; p.H = H;
  for (int i = 0; i < 4; ++i) p.k[i] = k[i];
  p.levels = levels;
  for (int i = 0; i < 4; ++i) p.iters[i] = i < levels ? iters[i] : 0;
  p.robust = robust; p.use_icp = use_icp; p.use_rgb = use_rgb;
  if (h->fp64) h->d.init(p); else h->f.init(p);
  return h;
}
void ot_destroy(void* h) { delete (Handle*)h; }

void ot_set_frame(void* hh, const unsigned char* rgb, const float* depth) {
  Handle* h = (Handle*)hh;
  if (h->fp64) h->d.set_frame(rgb, depth); else h->f.set_frame(rgb, depth);
}
void ot_set_ref_from_current(void* hh) {
  Handle* h = (Handle*)hh;
  if (h->fp64) h->d.set_ref_from_current(); else h->f.set_ref_from_current();
}
void ot_set_outlier_mask(void* hh, const unsigned char* mask) {
  Handle* h = (Handle*)hh;
  if (h->fp64) h->d.set_outlier_mask(mask); else h->f.set_outlier_mask(mask);
}
// trackLiveFrame (with the reference depth rendered from the model first).
// T_in: initial live pose, T_out: result; both float 4x4 (T_out64 optional).
void ot_track_camera(void* hh, const float* T_in, const float* T_w_r, const float* vertex,
                     const float* normal, float* T_out, double* T_out64) {
  Handle* h = (Handle*)hh;
  if (h->fp64) {
    M4<double> T = ld<double>(T_in);
    h->d.render_reference(vertex, ld<double>(T_w_r), nullptr, 0);
    h->d.track_camera(T, ld<double>(T_w_r), vertex, normal);
    st(T_out, T);
    if (T_out64) std_(T_out64, T);
  } else {
    M4<float> T = ld<float>(T_in);
    h->f.render_reference(vertex, ld<float>(T_w_r), nullptr, 0);
    h->f.track_camera(T, ld<float>(T_w_r), vertex, normal);
    st(T_out, T);
    if (T_out64) std_(T_out64, T);
  }
}
// trackEachObject: new volume pose for the object with `label`.
void ot_track_object(void* hh, const float* T_wo1, const float* T_w_c2, const float* T_w_c1,
                     const float* vertex, const float* normal, const int* labels, int label,
                     float* T_out, double* T_out64) {
  Handle* h = (Handle*)hh;
  if (h->fp64) {
    M4<double> r = h->d.track_object(ld<double>(T_wo1), ld<double>(T_w_c2), ld<double>(T_w_c1),
                                     vertex, normal, labels, label);
    st(T_out, r);
    if (T_out64) std_(T_out64, r);
  } else {
    M4<float> r = h->f.track_object(ld<float>(T_wo1), ld<float>(T_w_c2), ld<float>(T_w_c1),
                                    vertex, normal, labels, label);
    st(T_out, r);
    if (T_out64) std_(T_out64, r);
  }
}
// The 32 sums of the normal equations at one level for a given pose, after
// render_reference has been run for the problem (camera: T_w_r; object: T_w_c1).
void ot_camera_sums(void* hh, int level, const float* T_w_l, const float* T_w_r,
                    const float* vertex, const float* normal, double* out) {
  Handle* h = (Handle*)hh;
  auto run = [&](auto& t, auto zero) {
    using T = decltype(zero);
    const int n = t.p.W * t.p.H;
    std::vector<V3<T>> MV(n), MN(n);
    for (int i = 0; i < n; ++i) {
      MV[i] = v3<T>(vertex[3 * i], vertex[3 * i + 1], vertex[3 * i + 2]);
      MN[i] = v3<T>(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
    }
    t.render_reference(vertex, ld<T>(T_w_r), nullptr, 0);
    std::vector<double> s;
    t.camera_sums(level, ld<T>(T_w_l), ld<T>(T_w_r), MV, MN, s);
    for (int i = 0; i < 32; ++i) out[i] = s[i];
  };
  if (h->fp64) run(h->d, 0.0); else run(h->f, 0.0f);
}
void ot_object_sums(void* hh, int level, const float* T_c2_o2, const float* T_wo1,
                    const float* T_w_c1, const float* vertex, const float* normal,
                    const int* labels, int label, double* out) {
  Handle* h = (Handle*)hh;
  auto run = [&](auto& t, auto zero) {
    using T = decltype(zero);
    std::vector<V3<T>> MV, MN;
    t.object_maps(vertex, normal, labels, label, MV, MN);
    t.render_reference(vertex, ld<T>(T_w_c1), labels, label);
    const M4<T> T_c1_o1 = mul(inverse(ld<T>(T_w_c1)), ld<T>(T_wo1));
    std::vector<double> s;
    t.object_sums(level, ld<T>(T_c2_o2), T_c1_o1, ld<T>(T_wo1), MV, MN, s);
    for (int i = 0; i < 32; ++i) out[i] = s[i];
  };
  if (h->fp64) run(h->d, 0.0); else run(h->f, 0.0f);
}
void ot_last_sums(void* hh, int level, double* out) {
  Handle* h = (Handle*)hh;
  const std::vector<double>& s = h->fp64 ? h->d.last_sums[level] : h->f.last_sums[level];
  for (int i = 0; i < 32; ++i) out[i] = s[i];
}
int ot_last_iterations(void* hh, int level) {
  Handle* h = (Handle*)hh;
  return h->fp64 ? h->d.last_iterations[level] : h->f.last_iterations[level];
}
// Pyramid planes for tests: which 0 depth, 1 intensity, 2 vertex, 3 normal, 4 gradx,
// 5 grady, 6 icp covariance, 7 rendered reference vertex.
int ot_get_level(void* hh, int level, int which, float* out) {
  Handle* h = (Handle*)hh;
  auto get = [&](auto& t) {
    const size_t n = (size_t)t.lw[level] * t.lh[level];
    switch (which) {
      case 0: for (size_t i = 0; i < n; ++i) out[i] = (float)t.l_D[level][i]; break;
      case 1: for (size_t i = 0; i < n; ++i) out[i] = (float)t.l_I[level][i]; break;
      case 4: for (size_t i = 0; i < n; ++i) out[i] = (float)t.gx[level][i]; break;
      case 5: for (size_t i = 0; i < n; ++i) out[i] = (float)t.gy[level][i]; break;
      default: {
        const auto& v = which == 2 ? t.l_vertex[level] : which == 3 ? t.l_normal[level]
                        : which == 6 ? t.cov[level] : t.r_vertex_render[level];
        if (v.size() < n) return -1;  // not computed yet (the rendered reference: a track)
        for (size_t i = 0; i < n; ++i) {
          out[3 * i] = (float)v[i].x; out[3 * i + 1] = (float)v[i].y; out[3 * i + 2] = (float)v[i].z;
        }
      }
    }
    return (int)n;
  };
  return h->fp64 ? get(h->d) : get(h->f);
}

// Tracking::compute_residuals at level 0 with the single-precision tracker
// (the reference's arithmetic); -1 for an all-FP64 tracker.
int ot_motion_residuals(void* hh, const float* T_w_l, const float* T_w_r, const float* vertex,
                        const float* normal, const float* live_render_vertex, float threshold,
                        signed char* result, float* error) {
  Handle* h = (Handle*)hh;
  if (h->fp64) return -1;
  h->f.motion_residuals(ld<float>(T_w_l), ld<float>(T_w_r), vertex, normal, live_render_vertex,
                        threshold, (int8_t*)result, error);
  return 0;
}
float ot_inlier_ratio(const signed char* result, const int* labels, int label, int n, int use_icp,
                      int use_rgb) {
  return inlier_ratio((const int8_t*)result, labels, label, n, use_icp != 0, use_rgb != 0);
}
void ot_refine_mask_use_motion(float* mask, const signed char* result, int n, int use_icp,
                               int use_rgb) {
  refine_mask_use_motion(mask, (const int8_t*)result, n, use_icp != 0, use_rgb != 0);
}

// The level-0 row result codes of the last camera or object evaluation
// (2 * W * H int8); returns the count written (0 before any evaluation).
int ot_last_results(void* hh, signed char* out) {
  Handle* h = (Handle*)hh;
  const std::vector<int8_t>& r = h->fp64 ? h->d.last_result : h->f.last_result;
  std::memcpy(out, r.data(), r.size());
  return (int)r.size();
}

// Overwrites one plane of a pyramid level (test input injection): `which` as
// in ot_get_level for the live frame, 8 = reference intensity, 9 = reference
// (live) vertex.
int ot_set_level(void* hh, int level, int which, const float* in) {
  Handle* h = (Handle*)hh;
  auto set = [&](auto& t, auto zero) {
    using T = decltype(zero);
    const size_t n = (size_t)t.lw[level] * t.lh[level];
    auto plane = [&](std::vector<T>& d) { for (size_t i = 0; i < n; ++i) d[i] = (T)in[i]; };
    auto vec = [&](std::vector<V3<T>>& d) {
      for (size_t i = 0; i < n; ++i) d[i] = v3<T>(in[3 * i], in[3 * i + 1], in[3 * i + 2]);
    };
    switch (which) {
      case 0: plane(t.l_D[level]); break;
      case 1: plane(t.l_I[level]); break;
      case 2: vec(t.l_vertex[level]); break;
      case 3: vec(t.l_normal[level]); break;
      case 4: plane(t.gx[level]); break;
      case 5: plane(t.gy[level]); break;
      case 6: vec(t.cov[level]); break;
      case 8: plane(t.r_I[level]); break;
      case 9: vec(t.r_vertex_live[level]); break;
      default: return -1;
    }
    return (int)n;
  };
  return h->fp64 ? set(h->d, 0.0) : set(h->f, 0.0f);
}

}  // extern "C"

// TEST INFRASTRUCTURE ONLY.  Builds oracle/_ref/libmf_ref_track*.so: the
// reference's own tracking, preprocessing and object sources
// (apps/kfusion/src/cpp/tracking/tracking.cpp, preprocessing/preprocessing.cpp,
// object/object.cpp, rendering/rendering.cpp) compiled unmodified where they lie, against the project's
// stand-ins for TooN, Eigen and OpenCV under oracle/shim/, with a C ABI for the
// tests and the CPU baseline.  The sources are included into this one
// translation unit so that the tests can read the tracker's pyramids and
// per-level sums through member pointers taken in explicit template
// instantiations (where access checks do not apply), which leaves the
// reference's classes as they are.  Nothing here is shipped or measured as the
// product.
#include <algorithm>
#include <array>
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dirent.h>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <iterator>
#include <limits>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <omp.h>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <time.h>
#include <tuple>
#include <type_traits>
#include <typeinfo>
#include <unordered_map>
#include <utility>
#include <vector>
#include <zlib.h>

#include <Eigen/Dense>
#include <TooN/GR_SVD.h>
#include <TooN/TooN.h>
#include <TooN/se3.h>
#include <opencv2/imgproc/imgproc.hpp>
#include <opencv2/opencv.hpp>
#include "cnpy.h"
#include "tiny_obj_loader.h"
#include "perfstats.h"

#include "tracking/tracking.cpp"
#include "preprocessing/preprocessing.cpp"
#include "object/object.cpp"
#include "rendering/rendering.cpp"

// utils/timings.h declares these for the reference's drivers.
PerfStats Stats;
void synchroniseDevices() {}

// ---- read access to the tracker's private state -----------------------------
template <typename Tag, typename Tag::type M>
struct Grant { friend typename Tag::type get(Tag) { return M; } };
#define REF_MEMBER(name, T)                                        \
  struct Tag_##name { typedef T Tracking::*type; friend type get(Tag_##name); }; \
  template struct Grant<Tag_##name, &Tracking::name>;
REF_MEMBER(reductionoutput_, float**)
REF_MEMBER(trackingResult_, TrackData**)
REF_MEMBER(l_D_, float**)
REF_MEMBER(r_D_render_, float**)
REF_MEMBER(r_D_live_, float**)
REF_MEMBER(l_I_, float**)
REF_MEMBER(r_I_, float**)
REF_MEMBER(l_vertex_, float3**)
REF_MEMBER(r_Vertex_live_, float3**)
REF_MEMBER(r_Vertex_render_, float3**)
REF_MEMBER(l_normal_, float3**)
REF_MEMBER(l_gradx_, float**)
REF_MEMBER(l_grady_, float**)
REF_MEMBER(icp_cov_pyramid_, float3**)
REF_MEMBER(localImgSize_, std::vector<uint2>)
REF_MEMBER(outlier_mask_, std::vector<cv::Mat>)
REF_MEMBER(prev_outlier_mask_, std::vector<cv::Mat>)
REF_MEMBER(sigma_bright_, float)
#define REF_GET(t, name) ((t)->*get(Tag_##name()))

// ---- C ABI for the tests and the CPU baseline --------------------------------
namespace {
Matrix4 m4(const float* p) { Matrix4 m; std::memcpy(&m, p, 64); return m; }
void put(float* p, const Matrix4& m) { std::memcpy(p, &m, 64); }
float4 k4(const float* k) { return make_float4(k[0], k[1], k[2], k[3]); }
uint2 img_size(Tracking* t) { return REF_GET(t, localImgSize_)[0]; }
}  // namespace

extern "C" {

// A tracker as Kfusion builds it (kfusion.cpp:96-103): ICP and photometric
// rows, the reference depth rendered from the model (use_live_depth_only
// false).  robust: 0 none, 1 Huber, 2 Tukey, 3 Cauchy (RobustW order).
void* rt_create(int W, int H, int levels, const int* iters, int robust, int use_icp,
                int use_rgb) {
  std::vector<int> it(iters, iters + levels);
  Tracking* t = new Tracking(make_uint2(W, H), it, false, use_icp != 0, use_rgb != 0);
  t->robustWeight_ = static_cast<RobustW>(robust);
  return t;
}
void rt_destroy(void* h) { delete (Tracking*)h; }

// Tracking::calc_robust_weight / calc_robust_residual (tracking.cpp:1474-1532)
// of n residuals; robust in RobustW order.
void rt_robust(void* h, int robust, const float* e, int n, float* w, float* loss) {
  Tracking* t = (Tracking*)h;
  const RobustW k = static_cast<RobustW>(robust);
  for (int i = 0; i < n; ++i) {
    w[i] = t->calc_robust_weight(e[i], k);
    loss[i] = t->calc_robust_residual(e[i], k);
  }
}

// preprocessing.cpp:73-102: grey intensity and float RGB of an 8-bit frame (ratio 1).
void rt_rgb2intensity(const unsigned char* rgb, int W, int H, float* grey, float* rgb3) {
  rgb2intensity(grey, (float3*)rgb3, make_uint2(W, H), (const uchar3*)rgb, make_uint2(W, H));
}

// Tracking::set_params_frame (tracking.cpp:142-206); human_mask (8-bit, W x H)
// selects the masked overload when given.
void rt_set_frame(void* h, const float* k, const float* grey, const float* depth,
                  const unsigned char* human_mask) {
  Tracking* t = (Tracking*)h;
  if (human_mask) {
    const uint2 s = img_size(t);
    cv::Mat m((int)s.y, (int)s.x, CV_8UC1, (void*)human_mask);
    t->set_params_frame(k4(k), grey, depth, m);
  } else {
    t->set_params_frame(k4(k), grey, depth);
  }
}
void rt_set_ref_from_current(void* h) { ((Tracking*)h)->setRefImgFromCurr(); }

// Tracking::trackLiveFrame (tracking.cpp:208-357), or its masked overload
// (:1750-1879) when mask (8-bit, W x H, nonzero = excluded) is given.
// T_w_l is read and written (row-major 4x4).
int rt_track_live(void* h, float* T_w_l, const float* T_w_r, const float* k, const float* vertex,
                  const float* normal, const unsigned char* mask) {
  Tracking* t = (Tracking*)h;
  Matrix4 T = m4(T_w_l);
  bool ok;
  if (mask) {
    const uint2 s = img_size(t);
    cv::Mat m((int)s.y, (int)s.x, CV_8UC1, (void*)mask);
    ok = t->trackLiveFrame(T, m4(T_w_r), k4(k), (const float3*)vertex, (const float3*)normal, m);
  } else {
    ok = t->trackLiveFrame(T, m4(T_w_r), k4(k), (const float3*)vertex, (const float3*)normal);
  }
  put(T_w_l, T);
  return ok ? 1 : 0;
}

// The 32 sums of the last reduction at a level (row 0 of reductionoutput_).
void rt_reduction(void* h, int level, float* out) {
  std::memcpy(out, REF_GET((Tracking*)h, reductionoutput_)[level], 32 * sizeof(float));
}

// Pyramid planes: which 0 depth, 1 intensity, 2 vertex, 3 normal, 4 gradx,
// 5 grady, 6 ICP covariance, 7 rendered reference vertex, 8 reference
// intensity, 9 reference (live) vertex, 10 rendered reference depth.
// Returns the element count of the level (3 floats per element for vertex planes).
int rt_get_level(void* h, int level, int which, float* out) {
  Tracking* t = (Tracking*)h;
  const uint2 s = REF_GET(t, localImgSize_)[level];
  const size_t n = (size_t)s.x * s.y;
  const float* src = nullptr;
  size_t comp = 1;
  switch (which) {
    case 0: src = REF_GET(t, l_D_)[level]; break;
    case 1: src = REF_GET(t, l_I_)[level]; break;
    case 2: src = (const float*)REF_GET(t, l_vertex_)[level]; comp = 3; break;
    case 3: src = (const float*)REF_GET(t, l_normal_)[level]; comp = 3; break;
    case 4: src = REF_GET(t, l_gradx_)[level]; break;
    case 5: src = REF_GET(t, l_grady_)[level]; break;
    case 6: src = (const float*)REF_GET(t, icp_cov_pyramid_)[level]; comp = 3; break;
    case 7: src = (const float*)REF_GET(t, r_Vertex_render_)[level]; comp = 3; break;
    case 8: src = REF_GET(t, r_I_)[level]; break;
    case 9: src = (const float*)REF_GET(t, r_Vertex_live_)[level]; comp = 3; break;
    case 10: src = REF_GET(t, r_D_render_)[level]; break;
    default: return -1;
  }
  std::memcpy(out, src, n * comp * sizeof(float));
  return (int)n;
}

// The rows of the last evaluation at a level: 2 x W x H TrackData (ICP rows,
// then photometric rows, both with the full-resolution stride).
void rt_track_data(void* h, int level, int* result, float* error, float* J) {
  Tracking* t = (Tracking*)h;
  const uint2 s = img_size(t);
  const size_t n = 2 * (size_t)s.x * s.y;
  const TrackData* d = REF_GET(t, trackingResult_)[level];
  for (size_t i = 0; i < n; ++i) {
    result[i] = d[i].result;
    error[i] = d[i].error;
    for (int j = 0; j < 6; ++j) J[6 * i + j] = d[i].J[j];
  }
}

// Tracking::compute_residuals (tracking.cpp:1535-1554): level-0 residual rows
// into the tracker's level-0 result buffer (read with rt_track_data).
void rt_compute_residuals(void* h, const float* T_w_l, const float* T_w_r, const float* vertex,
                          const float* normal, const float* vertex_l, int use_icp, int use_rgb,
                          float threshold) {
  ((Tracking*)h)->compute_residuals(m4(T_w_l), m4(T_w_r), (const float3*)vertex,
                                    (const float3*)normal, (const float3*)vertex_l,
                                    use_icp != 0, use_rgb != 0, threshold);
}

// An Object (object.cpp:19-45) with a small volume: the tracker reads only its
// pose and model maps.
void* rt_object_create(int W, int H, const float* T_w_o, int volume_resol, float volume_size,
                       int class_id) {
  All_Prob_Vect p = All_Prob_Vect::Zero();
  return new Object(8, make_float3(volume_size), make_uint3(volume_resol), m4(T_w_o), m4(T_w_o),
                    class_id, p, make_uint2(W, H));
}
void rt_object_destroy(void* o) { delete (Object*)o; }
void rt_object_set_maps(void* o, int W, int H, const float* vertex, const float* normal,
                        const float* vertex_bef_integ) {
  Object* ob = (Object*)o;
  const size_t n = (size_t)W * H * sizeof(float3);
  if (vertex) std::memcpy(ob->m_vertex, vertex, n);
  if (normal) std::memcpy(ob->m_normal, normal, n);
  if (vertex_bef_integ) std::memcpy(ob->m_vertex_bef_integ, vertex_bef_integ, n);
}
void rt_object_set_pose(void* o, const float* T_w_o, const float* T_virtual) {
  Object* ob = (Object*)o;
  if (T_w_o) ob->volume_pose_ = m4(T_w_o);
  if (T_virtual) ob->virtual_camera_pose_ = m4(T_virtual);
}
void rt_object_pose(void* o, float* T_w_o, float* T_virtual) {
  Object* ob = (Object*)o;
  if (T_w_o) put(T_w_o, ob->volume_pose_);
  if (T_virtual) put(T_virtual, ob->virtual_camera_pose_);
}

// Tracking::trackEachObject (tracking.cpp:580-708): the object's new volume
// pose and virtual camera pose.
void rt_track_object(void* h, void* o, const float* k, const float* T_w_c2, const float* T_w_c1,
                     const float* grey, const float* depth) {
  ObjectPointer op((Object*)o, [](Object*) {});  // borrowed: the caller owns the object
  ((Tracking*)h)->trackEachObject(op, k4(k), m4(T_w_c2), m4(T_w_c1), grey, depth);
}

// The tracker's result rows into the object's (kfusion.cpp:283-284, 396-397).
void rt_object_take_results(void* o, void* h) {
  Tracking* t = (Tracking*)h;
  const uint2 s = img_size(t);
  std::memcpy(((Object*)o)->trackresult_, t->getTrackingResult(),
              sizeof(TrackData) * s.x * s.y * 2);
}
// Object::refine_mask_use_motion (object.cpp:255-315) on a float mask (H x W).
void rt_refine_mask_use_motion(void* o, float* mask, int W, int H, int use_icp, int use_rgb) {
  cv::Mat m(H, W, CV_32FC1, (void*)mask);
  ((Object*)o)->refine_mask_use_motion(m, use_icp != 0, use_rgb != 0);
}
// Object::set_static_state (object.cpp:317-320); returns is_static().
int rt_object_set_static_state(void* o, int state) {
  Object* ob = (Object*)o;
  ob->set_static_state(state != 0);
  return ob->is_static() ? 1 : 0;
}
// Object::fuseSemanticLabel (object.cpp:222-252) with an 80-class vector;
// returns the fused class id and the fused vector.
int rt_object_fuse_semantics(void* o, const float* prob80, int recog_time, float* fused80) {
  Object* ob = (Object*)o;
  All_Prob_Vect p;
  for (int i = 0; i < 80; ++i) p[i] = prob80[i];
  cv::Mat empty;
  instance_seg seg(1, cv::Mat::zeros(1, 1, CV_8UC1), p);
  seg.recog_time_ = recog_time;
  ob->fuseSemanticLabel(seg);
  for (int i = 0; i < 80; ++i) fused80[i] = ob->semanticfusion_[i];
  return ob->class_id_;
}

// The ray iterator keeps its direction epsilon in a function-local static set by
// the first iterator the library builds (lib/octree.hpp:931); this pins it.
void rt_pin_epsilon(int size) {
  Octree<SDF> o;
  o.init(size, 1.f);
  ray_iterator<SDF> it(o, make_float3(0.5f), make_float3(0.f, 0.f, 1.f), 0.1f, 1.f);
  (void)it;
}

void rt_object_set_label(void* o, int label) { ((Object*)o)->instance_label_ = label; }

// Object::integrate_volume_kernel (object.cpp:128-195): allocation, block and
// node integration of the object's volume from one frame; mask is the
// generalised float mask (H x W), rgb3 the float RGB frame.
void rt_object_integrate(void* o, const float* depth, const float* rgb3, const float* mask, int W,
                         int H, const float* T_w_c, const float* k, float mu, int frame) {
  cv::Mat m(H, W, CV_32FC1, (void*)mask);
  ((Object*)o)->integrate_volume_kernel(depth, (const float3*)rgb3, m, make_uint2(W, H),
                                        m4(T_w_c), mu, k4(k), (uint)frame);
}

namespace {
ObjectList borrowed_list(void** objs, int n) {
  ObjectList l;
  for (int i = 0; i < n; ++i) l.push_back(ObjectPointer((Object*)objs[i], [](Object*) {}));
  return l;
}
TrackData* track_rows(const int* res, const float* err, size_t n) {
  TrackData* d = (TrackData*)calloc(n, sizeof(TrackData));
  for (size_t i = 0; i < n; ++i) { d[i].result = res[i]; d[i].error = err ? err[i] : 0.f; }
  return d;
}
}  // namespace

// raycastObjectList (rendering.cpp:9-181) over every object, after
// integration (the model maps and each object's m_vertex / m_normal).
void rt_raycast_objects(void** objs, int n, const float* T_w_c, const float* k, int W, int H,
                        float near_plane, float far_plane, float mu, float* vertex, float* normal,
                        int* label) {
  ObjectList l = borrowed_list(objs, n);
  cv::Mat lab(H, W, CV_32SC1, (void*)label);
  std::set<int> in_view;
  raycastObjectList(l, (float3*)vertex, (float3*)normal, lab, in_view, m4(T_w_c), k4(k),
                    make_uint2(W, H), near_plane, far_plane, mu, true);
}

// renderVolume_many_Kernel (rendering.cpp:489-646); out is W x H uchar4.
void rt_render_volume(void** objs, int n, unsigned char* out, int W, int H, const float* T_w_c,
                      const float* k, float near_plane, float far_plane, float mu, float largestep,
                      const float* ambient, int doraycast, int render_color, const float* vertex,
                      const float* normal, const int* label, const unsigned char* colors,
                      int ncolors) {
  ObjectList l = borrowed_list(objs, n);
  cv::Mat lab(H, W, CV_32SC1, (void*)label);
  std::vector<uchar4> col((size_t)ncolors);
  std::memcpy(col.data(), colors, 4 * (size_t)ncolors);
  renderVolume_many_Kernel(l, (uchar4*)out, make_uint2(W, H), m4(T_w_c), k4(k), near_plane,
                           far_plane, mu, largestep, make_float3(ambient[0], ambient[1], ambient[2]),
                           doraycast != 0, render_color != 0, (const float3*)vertex,
                           (const float3*)normal, lab, col);
}

// renderDepthKernel / renderIntensityKernel / renderNormalKernel
// (rendering.cpp:346-393, 648-664).
void rt_render_depth(unsigned char* out, const float* depth, int W, int H, float near_plane,
                     float far_plane) {
  renderDepthKernel((uchar4*)out, (float*)depth, make_uint2(W, H), near_plane, far_plane);
}
void rt_render_intensity(unsigned char* out, const float* grey, int W, int H) {
  renderIntensityKernel((uchar4*)out, (float*)grey, make_uint2(W, H));
}
void rt_render_normal(unsigned char* out3, const float* normal, int W, int H) {
  renderNormalKernel((uchar3*)out3, (const float3*)normal, make_uint2(W, H));
}

// renderTrackKernel (mode 0, ICP rows), renderRGBTrackKernel (mode 1,
// photometric rows), render_RGBD_TrackKernel (mode 2, both); res / err hold
// 2 x W x H rows (ICP, then photometric).
void rt_render_track(unsigned char* out, const int* res, const float* err, int W, int H, int mode) {
  const size_t n = (size_t)W * H;
  TrackData* d = track_rows(res, err, 2 * n);
  if (mode == 0) renderTrackKernel((uchar4*)out, d, make_uint2(W, H));
  else if (mode == 1) renderRGBTrackKernel((uchar4*)out, d + n, make_uint2(W, H));
  else render_RGBD_TrackKernel((uchar4*)out, d, d + n, make_uint2(W, H));
  free(d);
}

// renderInstanceMaskKernel (mode 0, rendering.cpp:797-820),
// renderMaskWithImageKernel (1, :679-723) and renderMaskMotionWithImageKernel
// (2, :725-795) of a label image; mode 2 reads objs[label]'s trackresult_.
void rt_render_mask(unsigned char* out, const float* rgb3, const int* label, int W, int H,
                    int mode, const unsigned char* colors, int ncolors, void** objs, int nobjs) {
  SegmentationResult seg(make_uint2(W, H));
  seg.labelImg = cv::Mat(H, W, CV_32SC1, (void*)label);
  std::vector<uchar4> col((size_t)ncolors);
  std::memcpy(col.data(), colors, 4 * (size_t)ncolors);
  if (mode == 0) {
    renderInstanceMaskKernel((uchar4*)out, make_uint2(W, H), seg, col);
  } else if (mode == 1) {
    renderMaskWithImageKernel((uchar4*)out, make_uint2(W, H), (const float3*)rgb3, seg, col);
  } else {
    ObjectList l = borrowed_list(objs, nobjs);
    renderMaskMotionWithImageKernel((uchar4*)out, make_uint2(W, H), (const float3*)rgb3, seg, l,
                                    col);
  }
}

// An object's trackresult_ result codes (2 x W x H: ICP rows, then photometric).
void rt_object_set_results(void* o, const int* res, int W, int H) {
  Object* ob = (Object*)o;
  for (size_t i = 0; i < 2 * (size_t)W * H; ++i) ob->trackresult_[i].result = res[i];
}

// check_static_state (rendering.cpp:907-947): the inlier mask (255 / 0) of an
// 8-bit object mask under the camera's residual rows (2 x W x H codes).
void rt_check_static_state(unsigned char* inlier, const unsigned char* object_mask,
                           const int* res, int W, int H, int use_icp, int use_rgb) {
  const size_t n = (size_t)W * H;
  TrackData* d = track_rows(res, nullptr, 2 * n);
  cv::Mat in(H, W, CV_8UC1, (void*)inlier), om(H, W, CV_8UC1, (void*)object_mask);
  check_static_state(in, om, d, make_uint2(W, H), use_icp != 0, use_rgb != 0);
  free(d);
}

}  // extern "C"

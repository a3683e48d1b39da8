// ICP + photometric Gauss-Newton tracking on the device.
//
// Reference: apps/kfusion/src/cpp/tracking/tracking.cpp (Tracking) and
// apps/kfusion/src/cpp/preprocessing/*.  Per GN iteration one kernel evaluates
// the ICP row and the photometric row of every pixel of the level for every
// problem of the stage (the camera, or all moving objects at once), weights
// them (IRLS), and reduces the 29 sums of the normal equations plus the three
// outlier counts:
//   - per thread in FP32 over at most GN_PIX_MAX pixels (2 rows each), so no
//     FP32 sum runs over more than 2 * GN_PIX_MAX terms,
//   - per warp / block / grid in FP64 (block partials, fixed summation order,
//     so results are bitwise reproducible run to run),
// and the block that finishes last for a problem runs that problem's GN step
// on the device (cost test, step back, FP64 6x6 solve, SE(3) update,
// convergence test).  The host only launches: the whole coarse-to-fine loop is
// a fixed sequence of launches, and problems that stopped skip their work.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include "mf_internal.h"
#include "mf_robust.cuh"
#include "mf_solve.cuh"

namespace mf {

constexpr float INVALIDF = -2.f;
constexpr int GN_THREADS = 256;
#ifndef MF_GN_PIX0
#define MF_GN_PIX0 3
#endif
#ifndef MF_GN_MINB
#define MF_GN_MINB 3
#endif
// pixels per thread per iteration at level 0 (1 above): 3 makes the 640x480
// level one wave of 400 CTAs on 148 SMs x 3 resident (2: 600 CTAs in two
// waves, 30.9 us per launch against 24.8 us)
constexpr int GN_PIX_MAX = MF_GN_PIX0;
__host__ __device__ constexpr int gn_pix(int L) { return L == 0 ? GN_PIX_MAX : 1; }

struct GNState {
  double T[16], prevT[16];
  double prev_err;
  int done;
  int kind;          // 0 camera, 1 object
  int label;
  int inst;
  int iters[MAX_PYR];
  int fallback;
  int ticket;
  int pad_;
  // objects: bounding box (x0, y0, x1, y1) of the object's pixels in the
  // full-resolution model label map; empty when x1 < x0
  int box[4];
  M4 Tf, invTf;      // float pose (and inverse) seen by the per-pixel kernels
  M4 evalTf;         // the pose of the last GN evaluation (Tf when gn_step ran)
  M4 T_w_r, inv_T_w_r, view;               // camera: reference pose, K * inverse(T_w_r)
  M4 T_c1_o1, inv_T_c1_o1, inv_T_w_o1, T_w_c2;  // object constants
  M4 T_w_o1;         // object: the volume pose before this frame's tracking
  M4 T_virtual;      // object: virtual camera pose T_w_o1 inverse(T_c2_o2) after tracking
  double sums[MAX_PYR][32];
};

struct PyrPtrs {
  int w[MAX_PYR], h[MAX_PYR];
  float* D[MAX_PYR];
  float* I[2][MAX_PYR];
  F3* V[2][MAX_PYR];
  F3* N[MAX_PYR];
  float* GX[MAX_PYR];
  float* GY[MAX_PYR];
  F3* COV[MAX_PYR];
  uint8_t* MASK[MAX_PYR];
};

struct TrackState {
  int levels = 0;
  PyrPtrs pyr{};
  int cur = 0;                      // live set; 1 - cur holds the reference frame
  bool have_ref = false;
  bool tracked = false;             // the reference pose of this frame is saved
  float* rD[MAX_INSTANCES][MAX_PYR] = {};
  F3* rV[MAX_INSTANCES][MAX_PYR] = {};
  GNState* d_state = nullptr;       // MAX_INSTANCES (slot 0: camera, slot i: object i)
  int slot_kind[MAX_INSTANCES];     // per slot: -1 never set up, else the GNState kind
  unsigned* d_gnbar = nullptr;      // 2 x MAX_PYR grid-barrier counters (camera, objects)
  int coop_blocks[2] = {0, 0};      // co-resident CTAs of gn_level_kernel<0> / <1>
  double* d_partials = nullptr;     // MAX_INSTANCES x max_tiles x 32
  int max_tiles = 0;
  float2* d_zr = nullptr;           // MAX_PYR x max_tiles live depth range per CTA tile
  float* d_Twc_prev = nullptr;      // camera pose of the previous frame
  uint8_t* d_mask0 = nullptr;       // full-resolution ICP outlier mask
  float gaussian[5];
  std::vector<void*> allocs;
  // camera cost and adjoint (allocated on first use)
  double* d_gmodel = nullptr;       // 2 x 3 x W x H: dE/d model vertex, dE/d model normal
  double* d_cost_part = nullptr;    // per-CTA partials of the cost rows, 8 each
  double* d_cost = nullptr;         // 8: cost, dE/d twist (6), rows
  int cost_blocks = 0;
  // motion residuals (allocated on first use)
  int8_t* d_mres = nullptr;         // 2 x W x H result codes: ICP rows, then photometric
  float* d_merr = nullptr;          // 2 x W x H errors
  F3* d_lvert = nullptr;            // model raycast at the live pose: vertex, normal, label
  F3* d_lnorm = nullptr;
  int* d_llabel = nullptr;
  int* d_mcount = nullptr;          // 2 x MAX_INSTANCES: object pixels, inliers
};

// ------------------------------------------------------------------ preprocessing
struct Gauss5 { float g[5]; };

// exp of a float argument, rounded to the nearest float (what the host's expf
// returns in all but rare cases): the double-precision exp rounded to float.
// (A degree-6 Taylor polynomial for small arguments, which rounds alike, was
// slower: the lanes of a warp split between the two paths.)
__device__ __forceinline__ float exp_nearest(float x) { return (float)exp((double)x); }

// bilateralFilterKernel, preprocessing.cpp:11-50 (e_d = 0.1, r = 2) on the
// intensity (z = 0) and the depth (z = 1).  Neighbour coordinates clamp to the
// image (the reference's host clamp on unsigned values goes through int min/max,
// utils/cutil_math.h:51-57, 987-989).  The range weight is the reference's
// expf of the same float argument, rounded to the nearest float
// (exp_nearest), as the host's expf is in all but rare cases (measured on a
// 640x480 frame: 99.94 % of the filtered pixels equal the reference's bit for
// bit, against 72 % with the single-precision expf, whose results differ from
// the nearest float by up to 2 ulp); every later stage inherits the
// difference.
__global__ void bilateral_kernel(const float* __restrict__ grey, const float* __restrict__ depth,
                                 float* __restrict__ out_i, float* __restrict__ out_d, int W,
                                 int H, Gauss5 gs) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= W * H) return;
  const float* in = blockIdx.z == 0 ? grey : depth;
  float* out = blockIdx.z == 0 ? out_i : out_d;
  const int x = p % W, y = p / W;
  const float center = in[p];
  if (center == 0) { out[p] = 0; return; }
  const float e_d = 0.1f;
  const float e2 = e_d * e_d * 2;
  float sum = 0.0f, t = 0.0f;
  for (int i = -2; i <= 2; ++i)
    for (int j = -2; j <= 2; ++j) {
      const int cx = imn(imx(x + i, 0), W - 1), cy = imn(imx(y + j, 0), H - 1);
      const float cur = in[cx + cy * W];
      if (cur > 0) {
        const float mod = sq(cur - center);
        const float factor = gs.g[i + 2] * gs.g[j + 2] * exp_nearest(-mod / e2);
        t += factor * cur;
        sum += factor;
      }
    }
  out[p] = t / sum;
}

// halfSampleRobustImageKernel, preprocessing.cpp:161-196 (e_d = 0.3, r = 1).
__global__ void half_sample_kernel(const float* __restrict__ in0, float* __restrict__ out0,
                                   const float* __restrict__ in1, float* __restrict__ out1,
                                   int iw, int ih, float e_d) {
  const int ow = iw / 2, oh = ih / 2;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ow * oh) return;
  const float* in = blockIdx.z == 0 ? in0 : in1;
  float* out = blockIdx.z == 0 ? out0 : out1;
  if (!in) return;
  const int x = p % ow, y = p / ow;
  const int cx = 2 * x, cy = 2 * y;
  const float center = in[cx + cy * iw];
  float sum = 0.0f, t = 0.0f;
  for (int i = 0; i <= 1; ++i)
    for (int j = 0; j <= 1; ++j) {
      const int ux = imn(imx(cx + j, 0), 2 * ow - 1), uy = imn(imx(cy + i, 0), 2 * oh - 1);
      const float cur = in[ux + uy * iw];
      if (fabsf(cur - center) < e_d) { sum += 1.0f; t += cur; }
    }
  out[p] = t / sum;
}

// depth2vertexKernel, preprocessing.cpp:52-71.
__device__ __forceinline__ void depth2vertex_px(const float* __restrict__ depth,
                                                F3* __restrict__ vertex, int w, int p,
                                                const M4& invK) {
  const int x = p % w, y = p / w;
  const float d = depth[p];
  vertex[p] = d > 0 ? d * rotate(invK, mk3((float)x, (float)y, 1.f)) : mk3(0.f);
}

// The planes of every level of the live pyramid; the level kernels below take
// the level from blockIdx.y, so one launch covers all levels.
struct LevelMaps {
  const float* D[MAX_PYR];
  F3* V[MAX_PYR];
  const float* I[MAX_PYR];
  F3* N[MAX_PYR];
  float* GX[MAX_PYR];
  float* GY[MAX_PYR];
  F3* COV[MAX_PYR];
  uint8_t* MASK[MAX_PYR];
  int w[MAX_PYR], h[MAX_PYR];
  M4 invK[MAX_PYR];
  float focal[MAX_PYR];
  int negy;             // fy < 0 (the ICL-NUIM convention): up and down swap
};

__global__ void depth2vertex_levels_kernel(LevelMaps m) {
  const int l = blockIdx.y;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.w[l] * m.h[l]) return;
  depth2vertex_px(m.D[l], m.V[l], m.w[l], p, m.invK[l]);
}

// vertex2normalKernel<SDF, NegY> (preprocessing.h:39-81; NegY when fy < 0,
// tracking.cpp:805-810), gradientsKernel (preprocessing.cpp:235-246, borders
// untouched) and calc_icp_cov (tracking.cpp:845-871, sigma_xy = sigma_disp = 1,
// baseline 0.075).
__device__ __forceinline__ void normal_grad_cov_px(const F3* __restrict__ V,
                                                   const float* __restrict__ I,
                                                   const float* __restrict__ D,
                                                   F3* __restrict__ N, float* __restrict__ GX,
                                                   float* __restrict__ GY, F3* __restrict__ COV,
                                                   int w, int h, float focal, int negy,
                                                   int p) {
  const int x = p % w, y = p / w;
  const F3 left = V[imx(x - 1, 0) + w * y], right = V[imn(x + 1, w - 1) + w * y];
  const int ylo = imx(y - 1, 0), yhi = imn(y + 1, h - 1);
  const F3 down = V[x + w * (negy ? yhi : ylo)], up = V[x + w * (negy ? ylo : yhi)];
  if (left.z == 0 || right.z == 0 || up.z == 0 || down.z == 0) {
    N[p].x = INVALIDF;  // the other components keep their previous values
  } else {
    N[p] = normalize(cross(up - down, right - left));
  }
  if (x >= 1 && y >= 1 && x < w - 1 && y < h - 1) {
    GX[p] = (I[p + 1] - I[p - 1]) * 0.5f;
    GY[p] = (I[p + w] - I[p - w]) * 0.5f;
  }
  const float d = D[p];
  F3 c;
  c.x = (d / focal) * 1.0f;
  c.y = (d / focal) * 1.0f;
  c.z = (d * d * 1.0f) / (focal * 0.075f);
  c.x = c.x * c.x; c.y = c.y * c.y; c.z = c.z * c.z;
  COV[p] = c;
}

// normal_grad_cov_px on every level; it also clears the level's ICP outlier
// mask (no pixel is masked until the camera track sets one) unless MASK is
// null (the mask is then written whole by the camera's mask kernel).
__global__ void normal_grad_cov_levels_kernel(LevelMaps m) {
  const int l = blockIdx.y;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m.w[l] * m.h[l]) return;
  normal_grad_cov_px(m.V[l], m.I[l], m.D[l], m.N[l], m.GX[l], m.GY[l], m.COV[l], m.w[l],
                     m.h[l], m.focal[l], m.negy, p);
  if (m.MASK[l]) m.MASK[l][p] = 0;
}

struct SlotPtrs {
  float* D[MAX_INSTANCES];
  F3* V[MAX_INSTANCES];
  const float* Din[MAX_INSTANCES];
};

// vertex2depth (preprocessing.cpp:292-309) of the model vertex map -- for an
// object, its own map: the composite where label == object, 0 elsewhere
// (rendering.cpp:153-178) -- seen from the reference camera (T_w_r for the
// camera problem, T_w_c1 for an object; its inverse is kept in inv_T_w_r).
// For an object it also gathers the bounding box of the object's pixels in the
// label map (warp-reduced atomics); the object rows use it to skip gathers that
// can only find other labels.
__global__ void render_depth_kernel(const F3* __restrict__ vertex, const int* __restrict__ label,
                                    GNState* __restrict__ st, IdList slots, SlotPtrs sp,
                                    int W, int WH) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  GNState& S = st[slots.v[blockIdx.y]];
  bool mine = false;
  if (p < WH) {
    F3 v = vertex[p];
    if (S.kind == 1) {
      mine = label[p] == S.label;
      if (!mine) v = mk3(0.f);
    }
    sp.D[blockIdx.y][p] = v.z > 0.0 ? xform(S.inv_T_w_r, v).z : 0.f;
  }
  if (S.kind != 1) return;
  const int x = mine ? p % W : INT_MAX, y = mine ? p / W : INT_MAX;
  const int x0 = __reduce_min_sync(0xffffffffu, x), y0 = __reduce_min_sync(0xffffffffu, y);
  const int x1 = __reduce_max_sync(0xffffffffu, mine ? x : -1);
  const int y1 = __reduce_max_sync(0xffffffffu, mine ? y : -1);
  if ((threadIdx.x & 31) == 0 && x1 >= 0) {
    atomicMin(&S.box[0], x0); atomicMin(&S.box[1], y0);
    atomicMax(&S.box[2], x1); atomicMax(&S.box[3], y1);
  }
}

__global__ void half_sample_slots_kernel(SlotPtrs sp, int iw, int ih, float e_d) {
  const int ow = iw / 2, oh = ih / 2;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= ow * oh) return;
  const float* in = sp.Din[blockIdx.y];
  float* out = sp.D[blockIdx.y];
  const int x = p % ow, y = p / ow;
  const int cx = 2 * x, cy = 2 * y;
  const float center = in[cx + cy * iw];
  float sum = 0.0f, t = 0.0f;
  for (int i = 0; i <= 1; ++i)
    for (int j = 0; j <= 1; ++j) {
      const int ux = imn(imx(cx + j, 0), 2 * ow - 1), uy = imn(imx(cy + i, 0), 2 * oh - 1);
      const float cur = in[ux + uy * iw];
      if (fabsf(cur - center) < e_d) { sum += 1.0f; t += cur; }
    }
  out[p] = t / sum;
}

// The rendered reference depth and vertex planes of every slot at every level.
struct SlotLevels {
  const float* D[MAX_PYR][MAX_INSTANCES];
  F3* V[MAX_PYR][MAX_INSTANCES];
  int w[MAX_PYR], h[MAX_PYR];
  M4 invK[MAX_PYR];
};

// depth2vertex of every slot (blockIdx.y) at every level (blockIdx.z).
__global__ void depth2vertex_slots_kernel(SlotLevels sl) {
  const int l = blockIdx.z;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sl.w[l] * sl.h[l]) return;
  depth2vertex_px(sl.D[l][blockIdx.y], sl.V[l][blockIdx.y], sl.w[l], p, sl.invK[l]);
}

// ------------------------------------------------------------------ GN setup
// retrack: the second trackLiveFrame of a frame (kfusion.cpp:370-373), from
// the tracked pose against the same reference pose, which stays saved.
__global__ void setup_camera_kernel(GNState* st, const float* __restrict__ Twc,
                                    float* __restrict__ Twc_prev, F4 k, int retrack) {
  GNState& S = st[0];
  const M4 T = load_m4(Twc);
  const M4 Tr = retrack ? load_m4(Twc_prev) : T;
  if (!retrack) store_m4(Twc_prev, T);
  for (int i = 0; i < 16; ++i) {
    S.T[i] = (double)Twc[i];
    S.prevT[i] = S.T[i];
  }
  S.kind = 0; S.label = 0; S.inst = 0; S.done = 0; S.ticket = 0; S.fallback = 0;
  for (int l = 0; l < MAX_PYR; ++l) S.iters[l] = 0;
  S.T_w_r = Tr;
  S.inv_T_w_r = inverse(Tr);
  S.view = mul(camera_matrix(k), S.inv_T_w_r);  // tracking.cpp:258
  S.Tf = T;
  S.invTf = inverse(T);
  S.evalTf = T;
}

// trackEachObject setup, tracking.cpp:586-593: T_c1_o1 = inverse(T_w_c1) T_wo1,
// T_c2_o2 = inverse(T_w_c2) T_wo1 with T_w_c2 the freshly tracked camera.
// The part that does not need T_w_c2 (the previous camera pose, the object's
// last pose, the rendered reference's label box) and the part that does.
__device__ void setup_object_pre(GNState& S, int s, const M4& T_w_c1, const M4& T_wo1,
                                 int label) {
  S.kind = 1; S.inst = s; S.label = label; S.done = 0; S.ticket = 0; S.fallback = 0;
  for (int l = 0; l < MAX_PYR; ++l) S.iters[l] = 0;
  S.box[0] = S.box[1] = INT_MAX;
  S.box[2] = S.box[3] = -1;
  S.inv_T_w_r = inverse(T_w_c1);
  S.T_c1_o1 = mul(S.inv_T_w_r, T_wo1);
  S.inv_T_c1_o1 = inverse(S.T_c1_o1);
  S.inv_T_w_o1 = inverse(T_wo1);
  S.T_w_o1 = T_wo1;
}
__device__ void setup_object_post(GNState& S, const M4& T_w_c2) {
  S.T_w_c2 = T_w_c2;
  const M4 T0 = mul(inverse(T_w_c2), S.T_w_o1);
  for (int i = 0; i < 16; ++i) {
    S.T[i] = (double)m_at(T0, i / 4, i % 4);
    S.prevT[i] = S.T[i];
  }
  S.Tf = T0;
  S.invTf = inverse(T0);
  S.evalTf = T0;
}

__global__ void setup_objects_kernel(GNState* st, IdList slots, const float* __restrict__ Twc2,
                                     const float* __restrict__ Twc1, const float* __restrict__ Two,
                                     const int* __restrict__ inst_label) {
  const int t = threadIdx.x;
  if (t >= slots.n) return;
  const int s = slots.v[t];
  setup_object_pre(st[s], s, load_m4(Twc1), load_m4(Two + 16 * s), inst_label[s]);
  setup_object_post(st[s], load_m4(Twc2));
}
__global__ void setup_objects_pre_kernel(GNState* st, IdList slots, const float* __restrict__ Twc1,
                                         const float* __restrict__ Two,
                                         const int* __restrict__ inst_label) {
  const int t = threadIdx.x;
  if (t >= slots.n) return;
  const int s = slots.v[t];
  setup_object_pre(st[s], s, load_m4(Twc1), load_m4(Two + 16 * s), inst_label[s]);
}
__global__ void setup_objects_post_kernel(GNState* st, IdList slots, const float* __restrict__ Twc2) {
  const int t = threadIdx.x;
  if (t >= slots.n) return;
  setup_object_post(st[slots.v[t]], load_m4(Twc2));
}

__global__ void finalize_camera_kernel(const GNState* st, float* __restrict__ Twc) {
  store_m4(Twc, to_m4f(st[0].T));
}

// volume_pose_ = T_w_c2 * T_c2_o2, tracking.cpp:695.
// trackEachObject's outputs, tracking.cpp:695-696: the volume pose
// T_w_c2 T_c2_o2 and the virtual camera pose T_w_o1 inverse(T_c2_o2).
__global__ void finalize_objects_kernel(GNState* st, IdList slots, float* __restrict__ Two) {
  const int t = threadIdx.x;
  if (t >= slots.n) return;
  const int s = slots.v[t];
  const M4 Tco = to_m4f(st[s].T);
  store_m4(Two + 16 * s, mul(st[s].T_w_c2, Tco));
  st[s].T_virtual = mul(st[s].T_w_o1, inverse(Tco));
}

// ------------------------------------------------------------------ GN step
// One GN iteration's decision logic (tracking.cpp:287-335, objects :657-686):
// cost test with step back, solve, convergence test, left-multiplied update.
MF_HD void gn_step(GNState& S, const double* s, int level) {
  // work on register copies; one copy-out at the end
  double T[16], P[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) { T[i] = S.T[i]; P[i] = S.prevT[i]; }
  S.evalTf = S.Tf;   // the rows just summed were evaluated here
  const double prev_err = S.prev_err;
  const double err = s[0] / s[28];
  int done = 0, fallback = 0;
  if (S.kind == 1 && s[28] == 0) {  // no valid row: the object loop stops (:674-676)
    S.done = 1;
    S.iters[level] += 1;
    return;
  }
  if (err > prev_err) {
#pragma unroll
    for (int i = 0; i < 16; ++i) T[i] = P[i];
    done = 1;
  } else {
    S.prev_err = err;
    double A[6][6], b[6], x[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) b[i] = s[1 + i];
    make_jtj(s + 7, A);
    if (solve6(A, b, x)) fallback = 1;
    double nx = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) nx += x[i] * x[i];
    if (sqrt(nx) < (double)1e-05f && sqrt(s[0] / s[28]) < 2e-3) {
      done = 1;
    } else {
      double E[16], R[16];
      se3_exp(x, E);
      mul4d(E, T, R);
#pragma unroll
      for (int i = 0; i < 16; ++i) { P[i] = T[i]; T[i] = R[i]; }
    }
  }
#pragma unroll
  for (int i = 0; i < 16; ++i) { S.T[i] = T[i]; S.prevT[i] = P[i]; }
  S.done = done;
  if (fallback) S.fallback = 1;
  S.iters[level] += 1;
  const M4 Tf = to_m4f(T);
  S.Tf = Tf;
  S.invTf = inverse(Tf);
}

// gn_step by one whole warp (every lane of the calling warp, converged), with
// the same operations in the same order on every value, so the results equal
// the serial gn_step's bit for bit.  The serial step holds the 6x6 system, the
// poses and the update in one thread and spills at the GN kernels' register
// budget; here lane i < 6 holds row i of the system, lane l < 16 element l of
// the poses, and values move by shuffles.
// first: the level's first iteration (prev_err starts at infinity).
constexpr unsigned FULL_MASK = 0xffffffffu;

// A[i][j] of the symmetric normal matrix from the 21 packed sums (makeJTJ).
__device__ __forceinline__ double jtj_at(const double* v21, int i, int j) {
  const int a = i < j ? i : j, b = i < j ? j : i;
  return v21[a * 6 - a * (a - 1) / 2 + (b - a)];
}

// solve6 with row i of the eliminated system on lane i < 6 (lanes 6..31
// repeat row 5): the pivot row reaches every lane by shuffles; x (all lanes)
// and the fallback flag as solve6 gives them.
__device__ __forceinline__ bool solve6_warp(const double* s, int lane, double x[6]) {
  const double* v21 = s + 7;
  const int r = lane < 6 ? lane : 5;
  double a[6], c = s[1 + r];
#pragma unroll
  for (int k = 0; k < 6; ++k) a[k] = jtj_at(v21, r, k);
  double piv[6], pmax = 0;
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double pr[6];
#pragma unroll
    for (int k = j; k < 6; ++k) pr[k] = __shfl_sync(FULL_MASK, a[k], j);
    const double pc = __shfl_sync(FULL_MASK, c, j);
    piv[j] = pr[j];
    pmax = fmax(pmax, pr[j]);
    ok = ok && (pr[j] > 0);
    if (r != j) {
      const double f = a[j] / pr[j];
#pragma unroll
      for (int k = j; k < 6; ++k) a[k] -= f * pr[k];
      c -= f * pc;
    }
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) ok = ok && (piv[j] > 1e-5 * pmax);
  if (!ok) {  // the rare truncated eigen solve, serially on lane 0
    if (lane == 0) {
      double A[6][6], b[6];
      make_jtj(v21, A);
      for (int i = 0; i < 6; ++i) b[i] = s[1 + i];
      solve6_eigen(A, b, 1e6, x);
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) x[i] = __shfl_sync(FULL_MASK, x[i], 0);
    return true;
  }
  const double xr = c / a[r];
#pragma unroll
  for (int i = 0; i < 6; ++i) x[i] = __shfl_sync(FULL_MASK, xr, i);
  return false;
}

// inverse(M4) by the lanes of one warp, the same operations on the same values
// (so the same bits): lane j < 8 holds column j of [A | I] and the elimination
// updates every column at once; the pivot column is broadcast by shuffles.
// m_e: element (lane & 15) of A, row-major; returns element (lane & 15) of the
// inverse.
__device__ __forceinline__ float inverse_warp(float m_e, int lane) {
  const int col = lane & 7;
  float c[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float v = __shfl_sync(FULL_MASK, m_e, 4 * r + (col & 3));
    c[r] = col < 4 ? v : (r == col - 4 ? 1.f : 0.f);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float ac[4];
#pragma unroll
    for (int r = k; r < 4; ++r) ac[r] = __shfl_sync(FULL_MASK, c[r], k);
    int p = k;
    float best = fabsf(ac[k]);
#pragma unroll
    for (int r = k + 1; r < 4; ++r)
      if (fabsf(ac[r]) > best) { best = fabsf(ac[r]); p = r; }
#pragma unroll
    for (int r = k + 1; r < 4; ++r) {
      if (p == r) {
        float t = c[k]; c[k] = c[r]; c[r] = t;
        t = ac[k]; ac[k] = ac[r]; ac[r] = t;
      }
    }
    // the columns of A left of k are not updated (inverse() starts at j = k)
#pragma unroll
    for (int r = k + 1; r < 4; ++r) {
      const float f = ac[r] / ac[k];
      if (col >= k) c[r] -= f * c[k];
    }
  }
  // back substitution on the identity's columns (lanes 4..7), with the upper
  // triangle of the eliminated A from lanes 0..3
  float U[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int k = r; k < 4; ++k) U[r][k] = __shfl_sync(FULL_MASK, c[r], k);
  float R[4];
#pragma unroll
  for (int r = 3; r >= 0; --r) {
    float s = c[r];
#pragma unroll
    for (int k = r + 1; k < 4; ++k) s -= U[r][k] * R[k];
    R[r] = s / U[r][r];
  }
  const int i = (lane >> 2) & 3;
  float out = 0.f;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const float v = __shfl_sync(FULL_MASK, R[r], 4 + (lane & 3));
    if (r == i) out = v;
  }
  return out;
}

__device__ __noinline__ void gn_step_warp(GNState* Sp, const double* s, int level, int first) {
  GNState& S = *Sp;
  const int lane = threadIdx.x & 31;
  const int e = lane & 15;                 // pose element of this lane
  const int kind = S.kind;
  const double prev_err = first ? INFINITY : S.prev_err;
  const double err = s[0] / s[28];
  const float tf_old = reinterpret_cast<const float*>(&S.Tf)[e];
  double Tl = S.T[e], Pl = S.prevT[e];
  __syncwarp();
  if (lane < 16) reinterpret_cast<float*>(&S.evalTf)[e] = tf_old;
  if (kind == 1 && s[28] == 0) {  // no valid row: the object loop stops (:674-676)
    if (lane == 0) {
      S.prev_err = prev_err;
      S.done = 1;
      S.iters[level] += 1;
    }
    __syncwarp();
    return;
  }
  int done = 0, fallback = 0;
  double new_err = prev_err;
  if (err > prev_err) {
    Tl = Pl;
    done = 1;
  } else {
    new_err = err;
    double x[6];
    if (solve6_warp(s, lane, x)) fallback = 1;
    double nx = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) nx += x[i] * x[i];
    if (sqrt(nx) < (double)1e-05f && sqrt(s[0] / s[28]) < 2e-3) {
      done = 1;
    } else {
      // se3_exp(x): element (i, j) of the update on lane 4 i + j
      const double w0 = x[3], w1 = x[4], w2 = x[5];
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
      // every lane evaluates se3_exp's elements in its order (no divergence)
      // and keeps element (i, j)
      const int i = e >> 2, j = e & 3;
      const double W[3][3] = {{0, -w2, w1}, {w2, 0, -w0}, {-w1, w0, 0}};
      double El = (i == 3 && j == 3) ? 1.0 : 0.0;
#pragma unroll
      for (int ii = 0; ii < 3; ++ii) {
        double t = 0;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
          const double W2 = W[ii][0] * W[0][jj] + W[ii][1] * W[1][jj] + W[ii][2] * W[2][jj];
          const double I = ii == jj ? 1.0 : 0.0;
          const double v = I + A * W[ii][jj] + B * W2;
          if (ii == i && jj == j) El = v;
          t += (I + B * W[ii][jj] + C * W2) * x[jj];
        }
        if (ii == i && j == 3) El = t;
      }
      // R = E T (mul4d)
      double R = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k)
        R += __shfl_sync(FULL_MASK, El, 4 * i + k) * __shfl_sync(FULL_MASK, Tl, 4 * k + j);
      Pl = Tl;
      Tl = R;
    }
  }
  const float tf = (float)Tl;
  const float itf = inverse_warp(tf, lane);
  if (lane < 16) {
    S.T[e] = Tl;
    S.prevT[e] = Pl;
    reinterpret_cast<float*>(&S.Tf)[e] = tf;
    reinterpret_cast<float*>(&S.invTf)[e] = itf;
  }
  if (lane == 0) {
    S.prev_err = new_err;
    S.done = done;
    if (fallback) S.fallback = 1;
    S.iters[level] += 1;
  }
  __syncwarp();
}

// ------------------------------------------------------------------ residuals
struct GNArgs {
  PyrPtrs pyr;
  int cur;              // live set index
  int W, H;             // full-resolution model maps
  const F3* mvertex; const F3* mnormal; const int* mlabel;  // composite model maps
  F3* rV[MAX_INSTANCES];   // rendered reference vertex of each slot at this level
  GNState* st;
  double* partials;
  int max_tiles;
  const float2* zr;     // live depth range of each CTA tile, [level][tile]
  F4 kL;                // intrinsics at this level
  F4 k0;                // full resolution
  float inv_cov_rgb;
  int robust;
  int use_icp, use_rgb;
  int device_step;      // 1: the last block runs gn_step; 0: only the sums
  int first_iter;       // 1: the first iteration of a level in the batched loop:
                        // a stopped problem runs again and the step starts
                        // from prev_err = infinity (trackLiveFrame's per-level
                        // reset, tracking.cpp:247-249, 624-627)
};

struct Row { int result; float e; float J[6]; };

__device__ __forceinline__ float bil(const float* img, int w, float px, float py) {
  const float fx0 = floorf(px), fy0 = floorf(py);
  const int bx = (int)fx0, by = (int)fy0;
  const float fx = px - fx0, fy = py - fy0;
  return img[bx + by * w] * (1.f - fx) * (1.f - fy) + img[bx + 1 + by * w] * (1.f - fy) * fx +
         img[bx + (by + 1) * w] * (1.f - fx) * fy + img[bx + 1 + (by + 1) * w] * fx * fy;
}

// Object model maps derived from the composite maps and labels.
__device__ __forceinline__ void obj_maps(const GNArgs& a, int idx, int label, F3& v, F3& n) {
  if (a.mlabel[idx] == label) { v = a.mvertex[idx]; n = a.mnormal[idx]; }
  else { v = mk3(0.f); n = mk3(INVALIDF, 0.f, 0.f); }
}
// A 2x2 cell outside the object's label box holds only other labels: its four
// taps are (0, INVALID normal) without reading the maps (same arithmetic).
__device__ __forceinline__ void bil_obj(const GNArgs& a, const GNState& S, float px, float py,
                                        F3& v, F3& n) {
  const float fx0 = floorf(px), fy0 = floorf(py);
  const int bx = (int)fx0, by = (int)fy0;
  const float fx = px - fx0, fy = py - fy0;
  F3 v0, v1, v2, v3, n0, n1, n2, n3;
  if (bx + 1 < S.box[0] || bx > S.box[2] || by + 1 < S.box[1] || by > S.box[3]) {
    v0 = v1 = v2 = v3 = mk3(0.f);
    n0 = n1 = n2 = n3 = mk3(INVALIDF, 0.f, 0.f);
  } else {
    obj_maps(a, bx + by * a.W, S.label, v0, n0);
    obj_maps(a, bx + 1 + by * a.W, S.label, v1, n1);
    obj_maps(a, bx + (by + 1) * a.W, S.label, v2, n2);
    obj_maps(a, bx + 1 + (by + 1) * a.W, S.label, v3, n3);
  }
  const float A = 1.f - fx, B = 1.f - fy;
  v = mk3(v0.x * A * B + v1.x * B * fx + v2.x * A * fy + v3.x * fx * fy,
          v0.y * A * B + v1.y * B * fx + v2.y * A * fy + v3.y * fx * fy,
          v0.z * A * B + v1.z * B * fx + v2.z * A * fy + v3.z * fx * fy);
  n = mk3(n0.x * A * B + n1.x * B * fx + n2.x * A * fy + n3.x * fx * fy,
          n0.y * A * B + n1.y * B * fx + n2.y * A * fy + n3.y * fx * fy,
          n0.z * A * B + n1.z * B * fx + n2.z * A * fy + n3.z * fx * fy);
}

// track_ICP_Kernel, tracking.cpp:923-1020.
__device__ void icp_camera(const GNArgs& a, const GNState& S, int L, int p, Row& r) {
  if (a.pyr.MASK[L][p]) { r.result = -6; return; }
  const F3 n = a.pyr.N[L][p];
  if (n.x == INVALIDF) { r.result = -1; return; }
  const F3 pv = xform(S.Tf, a.pyr.V[a.cur][L][p]);
  const F3 pp = xform(S.view, pv);
  const float px = pp.x / pp.z, py = pp.y / pp.z;
  if (px < 1 || px > (float)(unsigned)(a.W - 2) || py < 1 || py > (float)(unsigned)(a.H - 2) ||
      isnan(px) || isnan(py)) { r.result = -2; return; }
  const unsigned rx = (unsigned)px, ry = (unsigned)py;
  const F3 rn = a.mnormal[rx + ry * a.W];
  if (rn.x == INVALIDF) { r.result = -3; return; }
  const F3 diff = a.mvertex[rx + ry * a.W] - pv;
  const F3 pn = rotate(S.Tf, n);
  if (length(diff) > 0.1f) { r.result = -4; return; }
  if (dot(pn, rn) < 0.8f) { r.result = -5; return; }
  r.result = 1;
  const F3 P = a.pyr.COV[L][p];
  const float sig = rn.x * rn.x * P.x + rn.y * rn.y * P.y + rn.z * rn.z * P.z;
  const float ic = sqrtf((float)(1.0 / (double)sig));
  r.e = ic * dot(rn, diff);
  const F3 j1 = ic * cross(pv, rn);
  r.J[0] = ic * rn.x; r.J[1] = ic * rn.y; r.J[2] = ic * rn.z;
  r.J[3] = j1.x; r.J[4] = j1.y; r.J[5] = j1.z;
}

// track_Obj_ICP_Kernel, tracking.cpp:392-486 (object outlier mask is all zero).
__device__ void icp_object(const GNArgs& a, const GNState& S, int L, int p, Row& r) {
  const F3 cn = a.pyr.N[L][p];
  if (cn.x == INVALIDF) { r.result = -1; return; }
  const F3 cv = a.pyr.V[a.cur][L][p];
  if (cv.x == 0 && cv.y == 0 && cv.z == 0) { r.result = -1; return; }
  const F3 o2v = xform(S.invTf, cv);
  const F3 c1v = xform(S.T_c1_o1, o2v);
  const F3 pr = rotate(camera_matrix(a.k0), c1v);
  const float px = pr.x / pr.z, py = pr.y / pr.z;
  if (px < 1 || px > (float)(unsigned)(a.W - 2) || py < 1 || py > (float)(unsigned)(a.H - 2) ||
      isnan(px) || isnan(py)) { r.result = -2; return; }
  const F3 o2n = rotate(S.invTf, cn);
  F3 wrv, wrn;
  bil_obj(a, S, px, py, wrv, wrn);
  if (wrn.x == INVALIDF) { r.result = -3; return; }
  const F3 o1rv = xform(S.inv_T_w_o1, wrv);
  const F3 o1rn = rotate(S.inv_T_w_o1, wrn);
  const F3 diff = o2v - o1rv;
  const float residual = dot(o1rn, diff);
  if (length(diff) > 0.1f) { r.result = -4; return; }
  if (dot(o2n, o1rn) < 0.8f) { r.result = -5; return; }
  const F3 P = a.pyr.COV[L][p];
  const float sig = o1rn.x * o1rn.x * P.x + o1rn.y * o1rn.y * P.y + o1rn.z * o1rn.z * P.z;
  const float ic = sqrtf((float)(1.0 / (double)sig));
  r.e = ic * residual;
  const F3 Jt = rotate(S.Tf, o1rn);
  const float c0 = -1.0f * ic * -1.0f;
  const F3 j1 = ic * cross(cv, Jt);
  r.J[0] = c0 * Jt.x; r.J[1] = c0 * Jt.y; r.J[2] = c0 * Jt.z;
  r.J[3] = j1.x; r.J[4] = j1.y; r.J[5] = j1.z;
  r.result = 1;
}

// trackRGB (tracking.cpp:1023-1111, warp :1114-1121, rgb_jacobian :1123-1150)
// and track_obj_RGB_kernel (:491-578, obj_warp :359-367, obj_rgb_jacobian
// :1152-1178).  The photometric outlier mask of the reference is all zero.
__device__ void rgb_row(const GNArgs& a, const GNState& S, const F3* rV, int L, int p, int w,
                        int h, Row& r) {
  if (S.kind == 1) {
    // an object's rendered reference is valid only inside its label box,
    // halved per pyramid level (half-sampling never widens it)
    const int x = p % w, y = p / w;
    if (x < (S.box[0] >> L) || x > (S.box[2] >> L) || y < (S.box[1] >> L) ||
        y > (S.box[3] >> L)) {
      r.result = -1;
      return;
    }
  }
  const F3 rv = rV[p];
  const F3 rl = a.pyr.V[1 - a.cur][L][p];
  if (rv.z <= 0.f || rv.z == INVALIDF) { r.result = -1; return; }
  if (length(rv - rl) > 0.1f && rl.z > 0.f) { r.result = -3; return; }
  const M4 KL = camera_matrix(a.kL);
  F3 lv, wv;
  if (S.kind == 0) {
    wv = xform(S.T_w_r, rv);
    lv = xform(S.invTf, wv);
  } else {
    const F3 o1v = xform(S.inv_T_c1_o1, rv);
    lv = xform(S.Tf, o1v);
  }
  const F3 pr = rotate(KL, lv);
  const float px = pr.x / pr.z, py = pr.y / pr.z;
  if (px < 1 || px > (float)(unsigned)(w - 2) || py < 1 || py > (float)(unsigned)(h - 2) ||
      isnan(px) || isnan(py)) { r.result = -2; return; }
  const float residual = a.pyr.I[1 - a.cur][L][p] - bil(a.pyr.I[a.cur][L], w, px, py);
  const float gx = bil(a.pyr.GX[L], w, px, py), gy = bil(a.pyr.GY[L], w, px, py);
  const float fx = KL.r[0].x, fy = KL.r[1].y;
  F3 Jt = (1.f / lv.z) * mk3(gx * fx, gy * fy, -(gx * lv.x * fx + gy * lv.y * fy) / lv.z);
  F3 Jr;
  if (S.kind == 0) {
    Jt = -1.f * rotate(S.Tf, Jt);  // rotate(Jtrans, transpose(T_w_l))
    Jr = cross(wv, Jt);
  } else {
    Jr = cross(lv, Jt);
  }
  const float ic = a.inv_cov_rgb;
  r.J[0] = ic * Jt.x; r.J[1] = ic * Jt.y; r.J[2] = ic * Jt.z;
  r.J[3] = ic * Jr.x; r.J[4] = ic * Jr.y; r.J[5] = ic * Jr.z;
  r.e = ic * residual;
  r.result = 1;
}

// Index of J_i J_j (i <= j) among the 21 upper-triangle terms, row-major
// (reduce, tracking.cpp:1279-1311).
__host__ __device__ constexpr int jtj_index(int i, int j) { return 7 + i * 6 - i * (i - 1) / 2 + (j - i); }

__device__ __forceinline__ void accumulate(float* acc, int* cnt, const Row& r, int kind) {
  if (r.result < 1) {
    cnt[0] += r.result == -4;
    cnt[1] += r.result == -5;
    cnt[2] += r.result > -4;
    return;
  }
  float w, loss;
  robust(r.e, kind, w, loss);
  acc[0] += loss;
  const float we = w * r.e;
#pragma unroll
  for (int i = 0; i < 6; ++i) acc[1 + i] += we * r.J[i];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const float wj = w * r.J[i];
#pragma unroll
    for (int j = i; j < 6; ++j) acc[jtj_index(i, j)] += wj * r.J[j];
  }
  acc[28] += 1.f;
}

// Range of live depths over the pixels of each GN tile (CTA) and level whose
// ICP row gets past the validity checks (valid normal, nonzero vertex).
__global__ void tile_depth_range_kernel(PyrPtrs pyr, int cur, float2* __restrict__ zr,
                                        int max_tiles) {
  const int L = blockIdx.y;
  const int w = pyr.w[L], n = w * pyr.h[L];
  const int ppt = gn_pix(L);
  const int p0 = blockIdx.x * GN_THREADS * ppt;
  if (p0 >= n) return;
  float lo = INFINITY, hi = -INFINITY;
  for (int k = 0; k < ppt; ++k) {
    const int p = p0 + k * GN_THREADS + threadIdx.x;
    if (p < n && pyr.N[L][p].x != INVALIDF) {
      const F3 v = pyr.V[cur][L][p];
      if (!(v.x == 0 && v.y == 0 && v.z == 0)) { lo = fminf(lo, v.z); hi = fmaxf(hi, v.z); }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  __shared__ float2 sw[GN_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = make_float2(lo, hi);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < GN_THREADS / 32; ++i) { lo = fminf(lo, sw[i].x); hi = fmaxf(hi, sw[i].y); }
    zr[L * max_tiles + blockIdx.x] = make_float2(lo, hi);
  }
}

// Can any pixel of tile `tile` at level L give an object problem a valid row?
// A `false` answer is exact for the 29 normal-equation sums (the tile's pixels
// all end in a negative result code); only the diagnostic outlier counts
// (sums 29-31, which the reference computes and never reads) then leave the
// tile out.
//  - photometric rows need the object's rendered reference: inside its label
//    box, halved per level;
//  - an ICP row needs a model tap with the object's label, i.e. a projection
//    into the label box: the tile's live points lie in the frustum spanned by
//    its pixel rectangle and depth range, whose projection lies in the hull
//    of its 8 projected corners (2 px of slack for rounding);
//  - or, with no such tap, the blended model vertex is 0, the world origin:
//    rows then need a live point within 0.1 m of it (in object coordinates).
// Called by a whole warp: lane l projects frustum corner l & 7 and the warp
// combines the corners with shuffles (every lane gets the answer).  A corner
// behind camera 1 or a NaN projection makes the answer true, as the first such
// corner did in a sequential loop; otherwise no NaN reaches the minima and
// maxima, so their order does not matter.
__device__ bool object_tile_live(const GNArgs& a, const GNState& S, int L, int tile, int w,
                                 int n) {
  const int ppt = gn_pix(L);
  const int p0 = tile * GN_THREADS * ppt, p1 = min(n, p0 + GN_THREADS * ppt);
  const int ya = p0 / w, yb = (p1 - 1) / w;
  const int xa = ya == yb ? p0 % w : 0, xb = ya == yb ? (p1 - 1) % w : w - 1;
  const bool has_box = S.box[2] >= S.box[0];
  if (a.use_rgb && has_box &&
      !(xb < (S.box[0] >> L) || xa > (S.box[2] >> L) || yb < (S.box[1] >> L) ||
        ya > (S.box[3] >> L)))
    return true;
  if (!a.use_icp) return false;
  const float2 zr = a.zr[L * a.max_tiles + tile];
  if (!(zr.x <= zr.y)) return false;  // no pixel of the tile reaches the projection
  const M4 iK = inverse_camera_matrix(a.kL), K0 = camera_matrix(a.k0);
  const int c = threadIdx.x & 7;
  const float x = (float)((c & 1) ? xb : xa), y = (float)((c & 2) ? yb : ya);
  const float z = (c & 4) ? zr.y : zr.x;
  const F3 o2v = xform(S.invTf, z * rotate(iK, mk3(x, y, 1.f)));
  F3 lo = o2v, hi = o2v;
  const F3 c1v = xform(S.T_c1_o1, o2v);
  bool unbounded = !(c1v.z > 0.f);  // the frustum reaches behind camera 1: no bound
  float qx0 = 0.f, qy0 = 0.f;
  if (!unbounded) {
    const F3 pr = rotate(K0, c1v);
    qx0 = pr.x / pr.z;
    qy0 = pr.y / pr.z;
    unbounded = isnan(qx0) || isnan(qy0);
  }
  if (__any_sync(0xffffffffu, unbounded)) return true;
  float qx1 = qx0, qy1 = qy0;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    qx0 = fminf(qx0, __shfl_xor_sync(0xffffffffu, qx0, o));
    qx1 = fmaxf(qx1, __shfl_xor_sync(0xffffffffu, qx1, o));
    qy0 = fminf(qy0, __shfl_xor_sync(0xffffffffu, qy0, o));
    qy1 = fmaxf(qy1, __shfl_xor_sync(0xffffffffu, qy1, o));
    lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
  }
  if (has_box && floorf(qx1) + 3.f >= (float)S.box[0] && floorf(qx0) - 2.f <= (float)S.box[2] &&
      floorf(qy1) + 3.f >= (float)S.box[1] && floorf(qy0) - 2.f <= (float)S.box[3])
    return true;
  const F3 o = get_translation(S.inv_T_w_o1);
  const float dx = fmaxf(fmaxf(lo.x - o.x, o.x - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - o.y, o.y - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - o.z, o.z - hi.z), 0.f);
  return dx * dx + dy * dy + dz * dz <= 0.101f * 0.101f;
}

// The warp's sum of value `lane` (29 sums, then the 3 counts) in FP64: every
// lane stores its FP32 partials in shared memory (rows padded to 33 words, so
// the column reads hit 32 banks) and lane i adds column i over the 32 lanes in
// lane order.  A shuffle tree would take 10 shuffles per double and 320 per
// warp; with one problem per grid row and many problems per launch that tree
// dominated the launch.
__device__ __forceinline__ double warp_sum_fp64(const float* acc, const int* cnt,
                                                float (*red)[33], int lane) {
#pragma unroll
  for (int i = 0; i < 29; ++i) red[lane][i] = acc[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) red[lane][29 + i] = (float)cnt[i];  // small, exact
  __syncwarp();
  double v = 0;
#pragma unroll 8
  for (int j = 0; j < 32; ++j) v += (double)red[j][lane];
  return v;
}

// The FP64 sums of one tile (CTA) of a problem at level L: every thread
// evaluates the ICP and photometric rows of its pixels, weights them and
// accumulates in FP32 (at most 6 rows per thread); the sums are FP64 from the
// warp level up, in a fixed order.  Thread i < 32 returns sum i (29 sums, then
// the 3 counts).  Object problems skip a tile that cannot hold a valid row.
template <int KIND>
__device__ __forceinline__ double gn_tile_sums(const GNArgs& a, const GNState& S, int s, int L,
                                               int tile, double (*sh)[32],
                                               float (*red)[32][33]) {
  const int w = a.pyr.w[L], h = a.pyr.h[L];
  const int n = w * h;
  bool live = true;
  if (KIND == 1) {
    __shared__ int s_live;
    if (threadIdx.x < 32) {
      const bool lv = object_tile_live(a, S, L, tile, w, n);
      if (threadIdx.x == 0) s_live = lv ? 1 : 0;
    }
    __syncthreads();
    live = s_live != 0;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (live) {
    float acc[29];
#pragma unroll
    for (int i = 0; i < 29; ++i) acc[i] = 0.f;
    int cnt[3] = {0, 0, 0};
    const F3* rV = a.rV[s];
    const int ppt = gn_pix(L);
#pragma unroll 1
    for (int k = 0; k < ppt; ++k) {
      const int p = tile * (GN_THREADS * ppt) + k * GN_THREADS + threadIdx.x;
      if (p >= n) break;
      Row r;
      if (a.use_icp) {
        r.result = 0;
        if (KIND == 0) icp_camera(a, S, L, p, r);
        else icp_object(a, S, L, p, r);
        accumulate(acc, cnt, r, a.robust);
      }
      if (a.use_rgb) {
        r.result = 0;
        rgb_row(a, S, rV, L, p, w, h, r);
        accumulate(acc, cnt, r, a.robust);
      }
    }
    sh[warp][lane] = warp_sum_fp64(acc, cnt, red[warp], lane);
  } else {
    sh[warp][lane] = 0.0;
  }
  __syncthreads();
  double v = 0;
  if (threadIdx.x < 32) {
#pragma unroll
    for (int wi = 0; wi < GN_THREADS / 32; ++wi) v += sh[wi][threadIdx.x];
  }
  return v;
}

// The 32 sums of a problem over its `ntiles` tile partials, in a fixed order,
// by the whole CTA (the last CTA of the problem): tot[i] = sum i.  The loads
// of 16 tiles are issued before their in-order additions, so the tail waits on
// about ntiles / 128 L2 round trips instead of ntiles / 64.
__device__ __forceinline__ void gn_tail_sums(const GNArgs& a, int s, int ntiles,
                                             double (*sh)[32], double* tot) {
  constexpr int G = GN_THREADS / 32, U = 16;
  {
    const int i = threadIdx.x & 31, g = threadIdx.x >> 5;  // 8 groups of tiles
    const double* col = a.partials + (size_t)s * a.max_tiles * 32 + i;
    double v = 0;
    int b = g;
    for (; b + (U - 1) * G < ntiles; b += U * G) {
      double t[U];
#pragma unroll
      for (int u = 0; u < U; ++u) t[u] = __ldcg(col + (size_t)(b + u * G) * 32);
#pragma unroll
      for (int u = 0; u < U; ++u) v += t[u];
    }
    for (; b < ntiles; b += G) v += __ldcg(col + (size_t)b * 32);
    sh[g][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) v += sh[g][threadIdx.x];
    tot[threadIdx.x] = v;
  }
  __syncthreads();
}

// One GN iteration of every problem in `slots` (grid.y = problem): the rows of
// every tile, the tile partials, and in the CTA that finishes last for a
// problem (ticket counter) the sum over the tiles and, with device_step, the
// problem's GN step on the device.
// KIND 0: the camera problem; KIND 1: object problems (one instantiation each
// keeps the kernel's code small).
// Programmatic dependent launch: the iterations of a level are chained so that
// the next launch's CTAs start while the previous one finishes (its tail and
// step), issue the prefetch of their pose-independent pixel data, and wait
// (griddepcontrol.wait) before they read anything the previous launch writes
// (the problem states, the partials).  Without the launch attribute the wait
// returns at once.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.L1 [%0];" :: "l"(p));
}

// The pixel data of a tile that does not depend on the pose (live vertex,
// normal, covariance and mask; rendered and live reference vertex, reference
// intensity) into L1.  Written before the GN launches of a frame start.
__device__ __forceinline__ void gn_prefetch(const GNArgs& a, int s, int L, int tile) {
  const int n = a.pyr.w[L] * a.pyr.h[L];
  const int ppt = gn_pix(L);
#pragma unroll 1
  for (int k = 0; k < ppt; ++k) {
    const int p = tile * (GN_THREADS * ppt) + k * GN_THREADS + threadIdx.x;
    if (p >= n) break;
    if (a.use_icp) {
      prefetch_l1(a.pyr.N[L] + p);
      prefetch_l1(a.pyr.V[a.cur][L] + p);
      prefetch_l1(a.pyr.COV[L] + p);
      prefetch_l1(a.pyr.MASK[L] + p);
    }
    if (a.use_rgb) {
      prefetch_l1(a.rV[s] + p);
      prefetch_l1(a.pyr.V[1 - a.cur][L] + p);
      prefetch_l1(a.pyr.I[1 - a.cur][L] + p);
    }
  }
}

template <int KIND>
__global__ void __launch_bounds__(GN_THREADS, MF_GN_MINB)
gn_iter_kernel(GNArgs a, IdList slots, int L) {
  const int s = slots.v[blockIdx.y];
  gn_prefetch(a, s, L, blockIdx.x);
  griddep_wait();
  GNState& S = a.st[s];
  if (S.done && !a.first_iter) return;
  // every CTA of this launch is resident: the next iteration may start
  griddep_launch_dependents();
  __shared__ double sh[GN_THREADS / 32][32];
  __shared__ float red[GN_THREADS / 32][32][33];
  const double v = gn_tile_sums<KIND>(a, S, s, L, blockIdx.x, sh, red);
  __shared__ bool last;
  if (threadIdx.x < 32) {
    a.partials[((size_t)s * a.max_tiles + blockIdx.x) * 32 + threadIdx.x] = v;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(&S.ticket, 1);
    last = (t == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double tot[32];
  gn_tail_sums(a, s, (int)gridDim.x, sh, tot);
  if (threadIdx.x < 32) {
    S.sums[L][threadIdx.x] = tot[threadIdx.x];
    if (threadIdx.x == 0) S.ticket = 0;
    if (a.device_step) gn_step_warp(&S, tot, L, a.first_iter);
  }
}

// ------------------------------------------------------------------ persistent level
// All GN iterations of one pyramid level for every problem in `slots`, in one
// cooperative launch (every CTA resident): the (problem, tile) items of an
// iteration are spread over the grid, the CTA that finishes a problem's last
// tile sums its partials and runs its step (as gn_iter_kernel does), and a
// grid barrier separates the iterations.  After each barrier the CTAs read the
// problems' `done` flags; when every problem has stopped, the level ends
// without launching the remaining iterations.  The per-pixel rows, the tile
// partials, their sum and the step are gn_iter_kernel's, so the poses equal
// the per-iteration launches' bit for bit.
// Every wait is bounded: a barrier that does not complete within
// GN_BAR_SPINS polls sets MF_STATUS_GN_TIMEOUT and the CTA returns.
constexpr unsigned GN_BAR_SPINS = 1u << 22;   // x >= 64 ns sleeps: about 0.3 s

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// GNState copied between global memory (through L2: other SMs write it within
// the launch) and shared memory, by the whole CTA.
__device__ __forceinline__ void state_load(const GNState* g, GNState* sm) {
  static_assert(sizeof(GNState) % 4 == 0, "GNState is copied as words");
  const int* src = reinterpret_cast<const int*>(g);
  int* dst = reinterpret_cast<int*>(sm);
  for (int i = threadIdx.x; i < (int)(sizeof(GNState) / 4); i += blockDim.x) dst[i] = __ldcg(src + i);
  __syncthreads();
}
__device__ __forceinline__ void state_store(const GNState* sm, GNState* g) {
  const int* src = reinterpret_cast<const int*>(sm);
  int* dst = reinterpret_cast<int*>(g);
  for (int i = threadIdx.x; i < (int)(sizeof(GNState) / 4); i += blockDim.x) __stcg(dst + i, src[i]);
  __threadfence();
  __syncthreads();
}

template <int KIND>
__global__ void __launch_bounds__(GN_THREADS, MF_GN_MINB)
gn_level_kernel(GNArgs a, IdList slots, int L, int iters, int ntiles, unsigned* __restrict__ bar,
                int* __restrict__ status) {
  __shared__ GNState sS;
  __shared__ double sh[GN_THREADS / 32][32];
  __shared__ float red[GN_THREADS / 32][32][33];
  __shared__ double tot[32];
  __shared__ int s_flag, s_done;
  const int items = slots.n * ntiles;
  for (int it = 0; it < iters; ++it) {
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
      const int pi = item / ntiles, tile = item - pi * ntiles;
      const int s = slots.v[pi];
      state_load(a.st + s, &sS);
      // a stopped problem runs again in the level's first iteration (the
      // level's reset, tracking.cpp:247-249, 624-627)
      if (sS.done && it > 0) continue;
      const double v = gn_tile_sums<KIND>(a, sS, s, L, tile, sh, red);
      if (threadIdx.x < 32) {
        a.partials[((size_t)s * a.max_tiles + tile) * 32 + threadIdx.x] = v;
        __threadfence();
      }
      __syncthreads();
      if (threadIdx.x == 0) s_flag = atomicAdd(&a.st[s].ticket, 1) == ntiles - 1;
      __syncthreads();
      if (!s_flag) continue;
      __threadfence();
      gn_tail_sums(a, s, ntiles, sh, tot);
      if (threadIdx.x < 32) sS.sums[L][threadIdx.x] = tot[threadIdx.x];
      __syncthreads();
      if (threadIdx.x < 32) {
        if (threadIdx.x == 0) sS.ticket = 0;
        gn_step_warp(&sS, tot, L, it == 0);
      }
      __syncthreads();
      state_store(&sS, a.st + s);
    }
    // grid barrier; then every CTA reads the same `done` flags
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(bar, 1u);
      const unsigned target = (unsigned)(it + 1) * gridDim.x;
      int flag = 0;
      for (unsigned spins = 0; ld_acquire_u32(bar) < target; ++spins) {
        if (spins >= GN_BAR_SPINS) {
          atomicOr(status, MF_STATUS_GN_TIMEOUT);
          flag = -1;
          break;
        }
        __nanosleep(64);
      }
      s_flag = flag;
    }
    __syncthreads();
    if (s_flag != 0) return;
    // the problems' done flags, one lane per problem
    if (threadIdx.x < 32) {
      int all = 1;
      for (int i = threadIdx.x; i < slots.n; i += 32) all &= __ldcg(&a.st[slots.v[i]].done) != 0;
      all = __all_sync(FULL_MASK, all);
      if (threadIdx.x == 0) s_done = all;
    }
    __syncthreads();
    if (s_done) return;
  }
}

// ------------------------------------------------------------------ host side
static int div_up(long long a, int b) { return (int)((a + b - 1) / b); }

template <typename T>
static int talloc(Context* ctx, T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
    ctx->last_error = "tracking buffer allocation failed";
    return MF_E_CUDA;
  }
  ctx->track->allocs.push_back(*p);
  MF_CUDA(cudaMemsetAsync(*p, 0, sizeof(T) * (n ? n : 1), ctx->stream));
  return MF_OK;
}

int track_init(Context* ctx) {
  if (ctx->track) return MF_OK;
  TrackState* ts = new TrackState;
  ctx->track = ts;
  for (int i = 0; i < MAX_INSTANCES; ++i) ts->slot_kind[i] = -1;
  ts->levels = std::max(1, std::min(ctx->cfg.pyramid_levels, MAX_PYR));
  PyrPtrs& P = ts->pyr;
  for (int l = 0; l < ts->levels; ++l) {
    P.w[l] = ctx->W >> l;
    P.h[l] = ctx->H >> l;
    const size_t n = (size_t)P.w[l] * P.h[l];
    int rc = 0;
    rc |= talloc(ctx, &P.D[l], n);
    rc |= talloc(ctx, &P.I[0][l], n);
    rc |= talloc(ctx, &P.I[1][l], n);
    rc |= talloc(ctx, &P.V[0][l], n);
    rc |= talloc(ctx, &P.V[1][l], n);
    rc |= talloc(ctx, &P.N[l], n);
    rc |= talloc(ctx, &P.GX[l], n);
    rc |= talloc(ctx, &P.GY[l], n);
    rc |= talloc(ctx, &P.COV[l], n);
    rc |= talloc(ctx, &P.MASK[l], n);
    for (int s = 0; s < ctx->cfg.max_instances; ++s) {
      rc |= talloc(ctx, &ts->rD[s][l], n);
      rc |= talloc(ctx, &ts->rV[s][l], n);
    }
    if (rc) return MF_E_CUDA;
  }
  ts->max_tiles = 0;
  for (int l = 0; l < ts->levels; ++l)
    ts->max_tiles = std::max(ts->max_tiles, div_up((long long)P.w[l] * P.h[l], GN_THREADS * gn_pix(l)));
  if (talloc(ctx, &ts->d_state, MAX_INSTANCES)) return MF_E_CUDA;
  if (talloc(ctx, &ts->d_partials, (size_t)MAX_INSTANCES * ts->max_tiles * 32)) return MF_E_CUDA;
  if (talloc(ctx, &ts->d_zr, (size_t)MAX_PYR * ts->max_tiles)) return MF_E_CUDA;
  if (talloc(ctx, &ts->d_Twc_prev, 16)) return MF_E_CUDA;
  if (talloc(ctx, &ts->d_mask0, (size_t)ctx->W * ctx->H)) return MF_E_CUDA;
  if (talloc(ctx, &ts->d_gnbar, 2 * MAX_PYR)) return MF_E_CUDA;
  // the persistent GN launch needs every CTA resident: its grid is at most
  // the SM count times the CTAs one SM holds
  {
    int sms = 0, b0 = 0, b1 = 0;
    MF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    MF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, gn_level_kernel<0>, GN_THREADS, 0));
    MF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, gn_level_kernel<1>, GN_THREADS, 0));
    ts->coop_blocks[0] = sms * b0;
    ts->coop_blocks[1] = sms * b1;
  }
  // Tracking::Tracking, tracking.cpp:77-84: gaussian[i] = expf(-(x*x) / (2 delta^2)),
  // x = i - 2, delta = 4 (computed on the host exactly as the reference does).
  for (int i = 0; i < 5; ++i) {
    const int x = i - 2;
    ts->gaussian[i] = expf(-(x * x) / (2 * 4.0f * 4.0f));
  }
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

void track_free(Context* ctx) {
  if (!ctx->track) return;
  for (void* p : ctx->track->allocs) cudaFree(p);
  delete ctx->track;
  ctx->track = nullptr;
}

static F4 kdiv(const mf_config& c, int l) {
  const float d = float(1 << l);
  return F4{c.k[0] / d, c.k[1] / d, c.k[2] / d, c.k[3] / d};
}

// Tracking::set_params_frame, tracking.cpp:142-171 (buildPyramid :776-818).
int track_preprocess(Context* ctx, bool clear_mask) {
  if (int rc = track_init(ctx)) return rc;
  TrackState& T = *ctx->track;
  PyrPtrs& P = T.pyr;
  const int W = ctx->W, H = ctx->H;
  Gauss5 g;
  for (int i = 0; i < 5; ++i) g.g[i] = T.gaussian[i];
  bilateral_kernel<<<dim3(div_up((long long)W * H, 256), 1, 2), 256, 0, ctx->stream>>>(
      ctx->d_grey, ctx->d_depth, P.I[T.cur][0], P.D[0], W, H, g);
  MF_CUDA(cudaGetLastError());
  const float e_d = 0.1f * 3;
  for (int l = 1; l < T.levels; ++l) {
    half_sample_kernel<<<dim3(div_up((long long)P.w[l] * P.h[l], 256), 1, 2), 256, 0, ctx->stream>>>(
        P.D[l - 1], P.D[l], P.I[T.cur][l - 1], P.I[T.cur][l], P.w[l - 1], P.h[l - 1], e_d);
    MF_CUDA(cudaGetLastError());
  }
  // vertex maps of every level, then normals, gradients, covariances and the
  // cleared outlier masks of every level: two launches
  LevelMaps m{};
  for (int l = 0; l < T.levels; ++l) {
    const F4 kl = kdiv(ctx->cfg, l);
    m.D[l] = P.D[l];
    m.V[l] = P.V[T.cur][l];
    m.I[l] = P.I[T.cur][l];
    m.N[l] = P.N[l];
    m.GX[l] = P.GX[l];
    m.GY[l] = P.GY[l];
    m.COV[l] = P.COV[l];
    m.MASK[l] = clear_mask ? P.MASK[l] : nullptr;
    m.w[l] = P.w[l];
    m.h[l] = P.h[l];
    m.invK[l] = inverse_camera_matrix(kl);
    m.focal[l] = kl.x;
  }
  m.negy = ctx->cfg.k[1] < 0.f;
  const dim3 grid(div_up((long long)P.w[0] * P.h[0], 256), T.levels);
  depth2vertex_levels_kernel<<<grid, 256, 0, ctx->stream>>>(m);
  normal_grad_cov_levels_kernel<<<grid, 256, 0, ctx->stream>>>(m);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// Tracking::setRefImgFromCurr, tracking.cpp:1400-1413: the live intensity and
// vertex pyramids become the reference (a buffer swap instead of a copy).
int track_set_ref(Context* ctx) {
  if (int rc = track_init(ctx)) return rc;
  ctx->track->cur = 1 - ctx->track->cur;
  ctx->track->have_ref = true;
  ctx->track->tracked = false;
  return MF_OK;
}

// The camera's ICP outlier mask, trackLiveFrame(..., mask): cv::resize to each
// level: 2x (INTER_AREA) keeps any nonzero of a 2x2 cell, 4x (INTER_LINEAR)
// samples taps 4x+1 and 4x+2 per axis.
struct MaskLevels {
  uint8_t* out[MAX_PYR];
  int w[MAX_PYR], h[MAX_PYR];
};

// One launch for every level (level = blockIdx.y); each level reads m0 only.
__global__ void mask_pyramid_kernel(const uint8_t* __restrict__ m0, MaskLevels ml, int W) {
  const int l = blockIdx.y;
  const int w = ml.w[l], h = ml.h[l];
  uint8_t* __restrict__ out = ml.out[l];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= w * h) return;
  const int x = p % w, y = p / w;
  uint8_t v;
  if (l == 0) {
    v = m0[p];
  } else {
    const int o = l == 1 ? 0 : (1 << (l - 1)) - 1, s = 1 << l;
    v = 0;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) v |= m0[(s * x + o + dx) + (s * y + o + dy) * W];
  }
  out[p] = v ? 1 : 0;
}

// Mask of the pixels whose composite label belongs to a moving object
// (the dynamic-object mask of Kfusion::tracking, kfusion.cpp:358-393).
__global__ void label_mask_kernel(const int* __restrict__ label, uint32_t moving,
                                  uint8_t* __restrict__ out, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int l = label[p];
  out[p] = (l >= 0 && l < 32 && ((moving >> l) & 1u)) ? 255 : 0;
}

int track_set_mask(Context* ctx, const uint8_t* d_mask0) {
  TrackState& T = *ctx->track;
  PyrPtrs& P = T.pyr;
  MaskLevels ml{};
  for (int l = 0; l < T.levels; ++l) {
    ml.out[l] = P.MASK[l];
    ml.w[l] = P.w[l];
    ml.h[l] = P.h[l];
  }
  mask_pyramid_kernel<<<dim3(div_up((long long)P.w[0] * P.h[0], 256), T.levels), 256, 0,
                        ctx->stream>>>(d_mask0, ml, ctx->W);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

static int render_reference(Context* ctx, const IdList& slots) {
  TrackState& T = *ctx->track;
  PyrPtrs& P = T.pyr;
  const int WH = ctx->W * ctx->H;
  SlotPtrs sp{};
  for (int i = 0; i < slots.n; ++i) sp.D[i] = T.rD[slots.v[i]][0];
  render_depth_kernel<<<dim3(div_up(WH, 256), slots.n), 256, 0, ctx->stream>>>(
      ctx->d_vertex, ctx->d_label, T.d_state, slots, sp, ctx->W, WH);
  MF_CUDA(cudaGetLastError());
  // the depth pyramid level by level, then the vertex maps of every level in
  // one launch
  SlotLevels sl{};
  for (int l = 0; l < T.levels; ++l) {
    SlotPtrs q{};
    for (int i = 0; i < slots.n; ++i) {
      q.D[i] = T.rD[slots.v[i]][l];
      q.V[i] = T.rV[slots.v[i]][l];
      q.Din[i] = l > 0 ? T.rD[slots.v[i]][l - 1] : nullptr;
      sl.D[l][i] = q.D[i];
      sl.V[l][i] = q.V[i];
    }
    sl.w[l] = P.w[l];
    sl.h[l] = P.h[l];
    sl.invK[l] = inverse_camera_matrix(kdiv(ctx->cfg, l));
    const int n = P.w[l] * P.h[l];
    if (l > 0) {
      half_sample_slots_kernel<<<dim3(div_up(n, 256), slots.n), 256, 0, ctx->stream>>>(
          q, P.w[l - 1], P.h[l - 1], 0.1f * 3);
      MF_CUDA(cudaGetLastError());
    }
  }
  depth2vertex_slots_kernel<<<dim3(div_up(WH, 256), slots.n, T.levels), 256, 0,
                              ctx->stream>>>(sl);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

static const void* sums_ptr(const TrackState& T, int slot, int L) {
  return (const char*)(T.d_state + slot) + offsetof(GNState, sums) + sizeof(double) * 32 * L;
}

static GNArgs make_args(Context* ctx, int L, int device_step) {
  TrackState& T = *ctx->track;
  GNArgs a;
  std::memset(&a, 0, sizeof(a));
  a.pyr = T.pyr;
  a.cur = T.cur;
  a.W = ctx->W; a.H = ctx->H;
  a.mvertex = ctx->d_vertex; a.mnormal = ctx->d_normal; a.mlabel = ctx->d_label;
  for (int s = 0; s < ctx->cfg.max_instances; ++s) a.rV[s] = T.rV[s][L];
  a.st = T.d_state;
  a.partials = T.d_partials;
  a.max_tiles = T.max_tiles;
  a.zr = T.d_zr;
  a.kL = kdiv(ctx->cfg, L);
  a.k0 = kdiv(ctx->cfg, 0);
  // obtainErrorParameters (TUM branch, tracking.cpp:766-772) keeps sigma_bright
  // in a float member; trackRGB uses 1.0 / sigma_bright (double) as a float.
  const float sigma_bright = (float)(sqrtf(100.0f) / 255.0);
  a.inv_cov_rgb = (float)(1.0 / (double)sigma_bright);
  a.robust = ctx->cfg.robust_kernel;
  a.use_icp = ctx->cfg.use_icp;
  a.use_rgb = ctx->cfg.use_rgb;
  a.device_step = device_step;
  return a;
}

// Live depth range of every GN tile at every level (object problems read it to
// skip tiles that cannot hold a valid row).  Recomputed before each object
// evaluation, so it always matches the live vertex and normal maps.
static int tile_depth_range(Context* ctx) {
  TrackState& T = *ctx->track;
  const int tiles = div_up((long long)T.pyr.w[0] * T.pyr.h[0], GN_THREADS * gn_pix(0));
  tile_depth_range_kernel<<<dim3(tiles, T.levels), GN_THREADS, 0, ctx->stream>>>(
      T.pyr, T.cur, T.d_zr, T.max_tiles);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// Coarse-to-fine GN of every problem in `slots`, all on the device
// (trackLiveFrame :240-335 / trackEachObject :629-694): one cooperative
// launch per level (gn_level_kernel), or, with gn_persistent off, one launch
// per iteration (gn_iter_kernel); both give the same poses bit for bit.
template <int KIND>
static cudaError_t launch_gn_level(const GNArgs& a, const IdList& slots, int L, int iters,
                                   int ntiles, unsigned* bar, int* status, int grid,
                                   cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(GN_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, gn_level_kernel<KIND>, a, slots, L, iters, ntiles, bar,
                            status);
}

template <int KIND>
static cudaError_t launch_gn_iter(const GNArgs& a, const IdList& slots, int L, int tiles,
                                  bool overlap, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles, slots.n);
  cfg.blockDim = dim3(GN_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = overlap ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, gn_iter_kernel<KIND>, a, slots, L);
}

static int gn_device(Context* ctx, const IdList& slots, int kind) {
  TrackState& T = *ctx->track;
  bool chained = false;
  const bool persistent = ctx->gn_persistent && T.coop_blocks[kind] > 0;
  unsigned* bar = T.d_gnbar + kind * MAX_PYR;
  if (persistent) MF_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned) * MAX_PYR, ctx->stream));
  for (int L = T.levels - 1; L >= 0; --L) {
    GNArgs a = make_args(ctx, L, 1);
    const int tiles = div_up((long long)T.pyr.w[L] * T.pyr.h[L], GN_THREADS * gn_pix(L));
    const int iters = ctx->cfg.gn_iterations[L];
    if (persistent) {
      if (iters <= 0) continue;
      const int grid = std::min(tiles * slots.n, T.coop_blocks[kind]);
      const cudaError_t e =
          kind == 0 ? launch_gn_level<0>(a, slots, L, iters, tiles, bar + L, ctx->d_status, grid,
                                         ctx->stream)
                    : launch_gn_level<1>(a, slots, L, iters, tiles, bar + L, ctx->d_status, grid,
                                         ctx->stream);
      if (e != cudaSuccess) {
        ctx->last_error = std::string("persistent GN launch: ") + cudaGetErrorString(e);
        return MF_E_CUDA;
      }
      continue;
    }
    for (int it = 0; it < iters; ++it) {
      a.first_iter = it == 0;  // the level's reset happens in its first iteration
      // every launch but the first of the chain overlaps its predecessor, a
      // GN launch (which writes only problem states and partials)
      const bool overlap = chained;
      chained = true;
      const cudaError_t e = kind == 0 ? launch_gn_iter<0>(a, slots, L, tiles, overlap, ctx->stream)
                                      : launch_gn_iter<1>(a, slots, L, tiles, overlap, ctx->stream);
      if (e != cudaSuccess) {
        ctx->last_error = std::string("GN launch: ") + cudaGetErrorString(e);
        return MF_E_CUDA;
      }
    }
  }
  return MF_OK;
}

// Host-driven GN of one problem: the sums come back to the host every
// iteration and the step runs there (the reference's structure on a GPU).
static int gn_host(Context* ctx, int slot) {
  TrackState& T = *ctx->track;
  IdList one;
  one.n = 1;
  one.v[0] = slot;
  GNState S;
  MF_CUDA(cudaMemcpyAsync(&S, T.d_state + slot, sizeof(GNState), cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int L = T.levels - 1; L >= 0; --L) {
    S.prev_err = INFINITY;
    S.done = 0;
    S.ticket = 0;
    const GNArgs a = make_args(ctx, L, 0);
    const int tiles = div_up((long long)T.pyr.w[L] * T.pyr.h[L], GN_THREADS * gn_pix(L));
    for (int it = 0; it < ctx->cfg.gn_iterations[L] && !S.done; ++it) {
      MF_CUDA(cudaMemcpyAsync(T.d_state + slot, &S, sizeof(GNState), cudaMemcpyHostToDevice,
                              ctx->stream));
      if (S.kind == 0) gn_iter_kernel<0><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, L);
      else gn_iter_kernel<1><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, L);
      MF_CUDA(cudaGetLastError());
      MF_CUDA(cudaMemcpyAsync(S.sums[L], sums_ptr(T, slot, L), sizeof(double) * 32,
                              cudaMemcpyDeviceToHost, ctx->stream));
      MF_CUDA(cudaStreamSynchronize(ctx->stream));
      gn_step(S, S.sums[L], L);
    }
  }
  MF_CUDA(cudaMemcpyAsync(T.d_state + slot, &S, sizeof(GNState), cudaMemcpyHostToDevice,
                          ctx->stream));
  return MF_OK;
}

// Tracking::trackLiveFrame with the current model maps; the camera pose is read
// from and written back to the device.  `moving` (bit per label) selects the
// pixels excluded from ICP (trackLiveFrame(..., mask)); 0 = no mask.
// The parts of trackLiveFrame before its GN that read neither the live
// pyramid nor the ICP outlier mask: the problem's setup from the current
// (pre-tracking) camera pose and the rendered reference of the model maps.
int track_camera_pre(Context* ctx, int retrack) {
  if (int rc = track_init(ctx)) return rc;
  TrackState& T = *ctx->track;
  const mf_config& c = ctx->cfg;
  if (retrack && !T.tracked) {
    ctx->last_error = "mf_retrack_camera: no mf_track_camera on this frame";
    return MF_E_STATE;
  }
  T.tracked = true;
  T.slot_kind[0] = 0;
  setup_camera_kernel<<<1, 1, 0, ctx->stream>>>(T.d_state, ctx->d_Twc, T.d_Twc_prev,
                                                F4{c.k[0], c.k[1], c.k[2], c.k[3]}, retrack);
  MF_CUDA(cudaGetLastError());
  IdList cam;
  cam.n = 1;
  cam.v[0] = 0;
  return render_reference(ctx, cam);
}

// The ICP outlier mask of the moving objects' pixels (after the pyramid,
// whose normals kernel clears the mask planes).
int track_camera_mask(Context* ctx, uint32_t moving) {
  if (!moving) return MF_OK;
  TrackState& T = *ctx->track;
  label_mask_kernel<<<div_up((long long)ctx->W * ctx->H, 256), 256, 0, ctx->stream>>>(
      ctx->d_label, moving, T.d_mask0, ctx->W * ctx->H);
  return track_set_mask(ctx, T.d_mask0);
}

int track_camera_gn(Context* ctx) {
  TrackState& T = *ctx->track;
  IdList cam;
  cam.n = 1;
  cam.v[0] = 0;
  if (ctx->cfg.batched) {
    if (int rc = gn_device(ctx, cam, 0)) return rc;
  } else {
    if (int rc = gn_host(ctx, 0)) return rc;
  }
  finalize_camera_kernel<<<1, 1, 0, ctx->stream>>>(T.d_state, ctx->d_Twc);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

int track_camera(Context* ctx, uint32_t moving, int retrack) {
  if (int rc = track_camera_pre(ctx, retrack)) return rc;
  if (int rc = track_camera_mask(ctx, moving)) return rc;
  return track_camera_gn(ctx);
}

// Tracking::trackEachObject for every id (instance ids >= 1), against the
// model maps of the last raycast, from the previous camera pose (saved by
// track_camera) to the current one.
static int track_objects_run(Context* ctx, const IdList& ids);

// The parts of trackEachObject before its GN that need neither the freshly
// tracked camera pose nor the live pyramid: the problems' setup from the
// previous camera pose (saved by track_camera_pre) and the objects' last
// poses, and their rendered references.
int track_objects_pre(Context* ctx, const IdList& ids) {
  if (int rc = track_init(ctx)) return rc;
  if (ids.n == 0) return MF_OK;
  TrackState& T = *ctx->track;
  for (int i = 0; i < ids.n; ++i) T.slot_kind[ids.v[i]] = 1;
  setup_objects_pre_kernel<<<1, 32, 0, ctx->stream>>>(T.d_state, ids, T.d_Twc_prev, ctx->d_Two,
                                                      ctx->d_inst_label);
  MF_CUDA(cudaGetLastError());
  return render_reference(ctx, ids);
}

// After track_objects_pre: the rest of the setup with the tracked camera pose,
// then the GN.
int track_objects_gn(Context* ctx, const IdList& ids) {
  if (ids.n == 0) return MF_OK;
  TrackState& T = *ctx->track;
  setup_objects_post_kernel<<<1, 32, 0, ctx->stream>>>(T.d_state, ids, ctx->d_Twc);
  MF_CUDA(cudaGetLastError());
  return track_objects_run(ctx, ids);
}

int track_objects(Context* ctx, const IdList& ids) {
  if (int rc = track_init(ctx)) return rc;
  if (ids.n == 0) return MF_OK;
  TrackState& T = *ctx->track;
  for (int i = 0; i < ids.n; ++i) T.slot_kind[ids.v[i]] = 1;
  setup_objects_kernel<<<1, 32, 0, ctx->stream>>>(T.d_state, ids, ctx->d_Twc, T.d_Twc_prev,
                                                  ctx->d_Two, ctx->d_inst_label);
  MF_CUDA(cudaGetLastError());
  if (int rc = render_reference(ctx, ids)) return rc;
  return track_objects_run(ctx, ids);
}

// The objects' GN once their problems are set up and their references rendered.
static int track_objects_run(Context* ctx, const IdList& ids) {
  TrackState& T = *ctx->track;
  if (int rc = tile_depth_range(ctx)) return rc;
  if (ctx->cfg.batched) {
    if (int rc = gn_device(ctx, ids, 1)) return rc;
  } else {
    for (int i = 0; i < ids.n; ++i)
      if (int rc = gn_host(ctx, ids.v[i])) return rc;
  }
  finalize_objects_kernel<<<1, 32, 0, ctx->stream>>>(T.d_state, ids, ctx->d_Two);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

bool track_has_ref(Context* ctx) { return ctx->track && ctx->track->have_ref; }
int track_parity(Context* ctx) { return ctx->track->cur; }
void track_set_parity(Context* ctx, int parity) { ctx->track->cur = parity; }

void track_save_prev_camera(Context* ctx) {
  cudaMemcpyAsync(ctx->track->d_Twc_prev, ctx->d_Twc, 64, cudaMemcpyDeviceToDevice, ctx->stream);
}

int track_info(Context* ctx, int slot, int* iters, double* sums, double* T64) {
  if (!ctx->track) return MF_E_STATE;
  GNState S;
  MF_CUDA(cudaMemcpyAsync(&S, ctx->track->d_state + slot, sizeof(GNState),
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int l = 0; l < MAX_PYR; ++l) {
    if (iters) iters[l] = S.iters[l];
    if (sums) for (int i = 0; i < 32; ++i) sums[32 * l + i] = S.sums[l][i];
  }
  if (T64) for (int i = 0; i < 16; ++i) T64[i] = S.T[i];
  return S.fallback ? 1 : 0;
}

// One evaluation of the normal equations at a given level for one problem at
// its current pose, without a step (parity checks of residuals + reduction).
int track_eval(Context* ctx, int slot, int L, const float* pose16, double* sums) {
  if (!ctx->track) return MF_E_STATE;
  TrackState& T = *ctx->track;
  if (T.slot_kind[slot] < 0) {
    ctx->last_error = "mf_track_eval: slot " + std::to_string(slot) + " has no tracking problem";
    return MF_E_STATE;
  }
  GNState S;
  MF_CUDA(cudaMemcpyAsync(&S, T.d_state + slot, sizeof(GNState), cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  if (pose16) {
    std::memcpy(&S.Tf, pose16, 64);
    S.invTf = inverse(S.Tf);
    for (int i = 0; i < 16; ++i) S.T[i] = pose16[i];
  }
  S.done = 0;
  S.ticket = 0;
  MF_CUDA(cudaMemcpyAsync(T.d_state + slot, &S, sizeof(GNState), cudaMemcpyHostToDevice,
                          ctx->stream));
  IdList one;
  one.n = 1;
  one.v[0] = slot;
  const GNArgs a = make_args(ctx, L, 0);
  const int tiles = div_up((long long)T.pyr.w[L] * T.pyr.h[L], GN_THREADS * gn_pix(L));
  if (S.kind == 1)
    if (int rc = tile_depth_range(ctx)) return rc;
  if (S.kind == 0) gn_iter_kernel<0><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, L);
  else gn_iter_kernel<1><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, L);
  MF_CUDA(cudaGetLastError());
  MF_CUDA(cudaMemcpyAsync(sums, sums_ptr(T, slot, L), sizeof(double) * 32,
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

// Timing and algorithmic bytes of one camera GN evaluation at level 0 on the
// current frame (used after the timed region).  Bytes per pixel: ICP live
// vertex, normal, covariance and the model vertex and normal (5 x 12 B), RGB
// rendered and live reference vertex (2 x 12 B), reference intensity (4 B), the
// 4-tap intensity and gradient gathers (16 + 32 B) and the outlier mask (2 B).
int profile_gn(Context* ctx, int reps, double* us, double* bytes) {
  if (!ctx->track) return MF_E_STATE;
  TrackState& T = *ctx->track;
  IdList one;
  one.n = 1;
  one.v[0] = 0;
  GNState S;
  MF_CUDA(cudaMemcpyAsync(&S, T.d_state, sizeof(GNState), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  S.done = 0;
  S.ticket = 0;
  MF_CUDA(cudaMemcpyAsync(T.d_state, &S, sizeof(GNState), cudaMemcpyHostToDevice, ctx->stream));
  const GNArgs a = make_args(ctx, 0, 0);
  const int tiles = div_up((long long)T.pyr.w[0] * T.pyr.h[0], GN_THREADS * gn_pix(0));
  gn_iter_kernel<0><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, 0);  // warm
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx->stream);
  for (int r = 0; r < reps; ++r)
    gn_iter_kernel<0><<<dim3(tiles, 1), GN_THREADS, 0, ctx->stream>>>(a, one, 0);
  cudaEventRecord(e1, ctx->stream);
  MF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MF_CUDA(cudaGetLastError());
  *us = 1e3 * ms / reps;
  *bytes = 138.0 * T.pyr.w[0] * T.pyr.h[0];
  return MF_OK;
}

int track_download_level(Context* ctx, int L, int which, float* out) {
  if (!ctx->track) return MF_E_STATE;
  TrackState& T = *ctx->track;
  const PyrPtrs& P = T.pyr;
  const size_t n = (size_t)P.w[L] * P.h[L];
  const void* src = nullptr;
  size_t bytes = 4 * n;
  switch (which) {
    case 0: src = P.D[L]; break;
    case 1: src = P.I[T.cur][L]; break;
    case 2: src = P.V[T.cur][L]; bytes = 12 * n; break;
    case 3: src = P.N[L]; bytes = 12 * n; break;
    case 4: src = P.GX[L]; break;
    case 5: src = P.GY[L]; break;
    case 6: src = P.COV[L]; bytes = 12 * n; break;
    case 7: src = T.rV[0][L]; bytes = 12 * n; break;
    default: return MF_E_ARG;
  }
  MF_CUDA(cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

// ------------------------------------------------------------------------
// Normal-equation evaluation that allocates nothing (mf_track_eval_static).
//
// Same sums as track_eval (the per-pixel rows and the FP64 reduction of
// gn_iter_kernel, in the same order, so the two agree bit for bit), but the
// scratch -- the per-CTA FP64 partials, the 32 result sums and the CTA ticket
// -- is the file-scope array below, not a cudaMalloc'd buffer, and the pose is
// a kernel argument, so the context's GN state is not touched either.
// Layout of the array (bytes):
//   [0, EVAL_PARTIALS_BYTES)        double partials[EVAL_MAX_TILES][32]
//   [EVAL_SUMS_OFF, +256)           double sums[32]
//   [EVAL_TICKET_OFF, +4)           unsigned ticket (zeroed before each launch)
// EVAL_MAX_TILES bounds the level's pixel count: 4096 CTAs x 768 pixels at
// level 0 (3 145 728 px, e.g. 2048x1536) and 4096 x 256 above it.
constexpr int EVAL_MAX_TILES = 4096;
constexpr size_t EVAL_PARTIALS_BYTES = (size_t)EVAL_MAX_TILES * 32 * sizeof(double);
constexpr size_t EVAL_SUMS_OFF = EVAL_PARTIALS_BYTES;
constexpr size_t EVAL_TICKET_OFF = EVAL_SUMS_OFF + 32 * sizeof(double);
constexpr size_t EVAL_SCRATCH_BYTES = EVAL_TICKET_OFF + 256;
static __device__ __align__(256) unsigned char g_eval_scratch[EVAL_SCRATCH_BYTES];

template <int KIND>
__global__ void __launch_bounds__(GN_THREADS, 2)
gn_eval_static_kernel(GNArgs a, int s, int L, int set_pose, M4 Tf, M4 invTf,
                      unsigned char* scratch) {
  // the problem's constants, with the pose to evaluate at, in shared memory
  __shared__ GNState S;
  {
    static_assert(sizeof(GNState) % 4 == 0, "GNState is copied as words");
    const int* src = reinterpret_cast<const int*>(&a.st[s]);
    int* dst = reinterpret_cast<int*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(GNState) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  if (threadIdx.x == 0 && set_pose) {
    S.Tf = Tf;
    S.invTf = invTf;
  }
  __syncthreads();
  double* partials = reinterpret_cast<double*>(scratch);
  double* out = reinterpret_cast<double*>(scratch + EVAL_SUMS_OFF);
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + EVAL_TICKET_OFF);

  const int w = a.pyr.w[L], h = a.pyr.h[L];
  const int n = w * h;
  // object problems: a tile that cannot hold a valid row skips its pixels
  bool live = true;
  if (KIND == 1) {
    __shared__ int s_live;
    if (threadIdx.x < 32) {
      const bool lv = object_tile_live(a, S, L, blockIdx.x, w, n);
      if (threadIdx.x == 0) s_live = lv ? 1 : 0;
    }
    __syncthreads();
    live = s_live != 0;
  }
  // FP64 from the warp level up
  __shared__ double sh[GN_THREADS / 32][32];
  __shared__ float red[GN_THREADS / 32][32][33];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (live) {
    float acc[29];
#pragma unroll
    for (int i = 0; i < 29; ++i) acc[i] = 0.f;
    int cnt[3] = {0, 0, 0};
    const F3* rV = a.rV[s];
    const int ppt = gn_pix(L);
#pragma unroll 1
    for (int k = 0; k < ppt; ++k) {
      const int p = blockIdx.x * (GN_THREADS * ppt) + k * GN_THREADS + threadIdx.x;
      if (p >= n) break;
      Row r;
      if (a.use_icp) {
        r.result = 0;
        if (KIND == 0) icp_camera(a, S, L, p, r);
        else icp_object(a, S, L, p, r);
        accumulate(acc, cnt, r, a.robust);
      }
      if (a.use_rgb) {
        r.result = 0;
        rgb_row(a, S, rV, L, p, w, h, r);
        accumulate(acc, cnt, r, a.robust);
      }
    }
    sh[warp][lane] = warp_sum_fp64(acc, cnt, red[warp], lane);
  } else {
    sh[warp][lane] = 0.0;
  }
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x < 32) {
    double v = 0;
#pragma unroll
    for (int wi = 0; wi < GN_THREADS / 32; ++wi) v += sh[wi][threadIdx.x];
    partials[(size_t)blockIdx.x * 32 + threadIdx.x] = v;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  {
    const int i = threadIdx.x & 31, g = threadIdx.x >> 5;
    double v = 0;
    for (int b = g; b < (int)gridDim.x; b += GN_THREADS / 32)
      v += __ldcg(&partials[(size_t)b * 32 + i]);
    sh[g][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = 0;
#pragma unroll
    for (int g = 0; g < GN_THREADS / 32; ++g) v += sh[g][threadIdx.x];
    out[threadIdx.x] = v;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// Device address of g_eval_scratch for each device, looked up once per device
// with that device current, on the first call (host code cannot use the
// address of a __device__ variable directly).
static std::mutex g_eval_mutex;
static unsigned char* g_eval_ptr[64] = {};

static int eval_scratch_setup(Context* ctx, unsigned char** out) {
  int dev = -1;
  MF_CUDA(cudaGetDevice(&dev));
  if (dev != ctx->device) {
    ctx->last_error = "mf_track_eval_static: the context's device is not the current device";
    return MF_E_STATE;
  }
  if (dev < 0 || dev >= 64) {
    ctx->last_error = "mf_track_eval_static: device ordinal above 63";
    return MF_E_ARG;
  }
  std::lock_guard<std::mutex> lock(g_eval_mutex);
  if (!g_eval_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_eval_scratch);
    if (e != cudaSuccess || !p) {
      ctx->last_error = std::string("cudaGetSymbolAddress(g_eval_scratch): ") +
                        cudaGetErrorString(e);
      return MF_E_CUDA;
    }
    g_eval_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_eval_ptr[dev];
  return MF_OK;
}

int track_eval_static(Context* ctx, int slot, int L, const float* pose16, double* sums) {
  const int tiles = div_up((long long)(ctx->W >> L) * (ctx->H >> L), GN_THREADS * gn_pix(L));
  if (tiles > EVAL_MAX_TILES) {
    ctx->last_error = "mf_track_eval_static: level has more than 4096 x " +
                      std::to_string(GN_THREADS * gn_pix(L)) +
                      " pixels (the static scratch holds 4096 CTA partials)";
    return MF_E_ARG;
  }
  if (!ctx->track) return MF_E_STATE;
  const int kind = ctx->track->slot_kind[slot];
  if (kind < 0) {
    ctx->last_error = "mf_track_eval_static: slot " + std::to_string(slot) +
                      " has no tracking problem";
    return MF_E_STATE;
  }
  unsigned char* scratch = nullptr;
  if (int rc = eval_scratch_setup(ctx, &scratch)) return rc;
  M4 Tf{}, invTf{};
  const int set_pose = pose16 ? 1 : 0;
  if (pose16) {
    std::memcpy(&Tf, pose16, 64);
    invTf = inverse(Tf);
  }
  const GNArgs a = make_args(ctx, L, 0);
  if (kind == 1)
    if (int rc = tile_depth_range(ctx)) return rc;
  // the ticket must be zero when the launch starts (the last CTA also resets it)
  MF_CUDA(cudaMemsetAsync(scratch + EVAL_TICKET_OFF, 0, sizeof(unsigned), ctx->stream));
  if (kind == 0)
    gn_eval_static_kernel<0><<<tiles, GN_THREADS, 0, ctx->stream>>>(a, slot, L, set_pose, Tf,
                                                                     invTf, scratch);
  else
    gn_eval_static_kernel<1><<<tiles, GN_THREADS, 0, ctx->stream>>>(a, slot, L, set_pose, Tf,
                                                                     invTf, scratch);
  MF_CUDA(cudaGetLastError());
  MF_CUDA(cudaMemcpyAsync(sums, scratch + EVAL_SUMS_OFF, 32 * sizeof(double),
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

// ------------------------------------------------------------------------
// The GN step on given inputs, on the device (gn_step_warp, one warp per
// problem) and on the host (gn_step), for checking that the two agree.
// state: n x 36 doubles: T[16], prevT[16], prev_err, kind, first, level;
// sums: n x 32.  out_dev / out_host: n x 68 doubles: T[16], prevT[16],
// prev_err, done, fallback, iterations at the level, Tf[16], invTf[16].
__global__ void gn_step_check_kernel(GNState* st, const double* __restrict__ sums,
                                     const int* __restrict__ first, const int* __restrict__ level) {
  const int i = blockIdx.x;
  gn_step_warp(st + i, sums + 32 * i, level[i], first[i]);
}

static void gn_step_out(const GNState& S, int level, double* o) {
  for (int k = 0; k < 16; ++k) { o[k] = S.T[k]; o[16 + k] = S.prevT[k]; }
  o[32] = S.prev_err;
  o[33] = S.done;
  o[34] = S.fallback;
  o[35] = S.iters[level];
  for (int k = 0; k < 16; ++k) {
    o[36 + k] = m_at(S.Tf, k / 4, k % 4);
    o[52 + k] = m_at(S.invTf, k / 4, k % 4);
  }
}

int gn_step_check(Context* ctx, int n, const double* state, const double* sums, double* out_dev,
                  double* out_host) {
  std::vector<GNState> hs(n);
  std::vector<int> first(n), level(n);
  for (int i = 0; i < n; ++i) {
    GNState& S = hs[i];
    std::memset(&S, 0, sizeof(GNState));
    const double* q = state + 36 * i;
    for (int k = 0; k < 16; ++k) { S.T[k] = q[k]; S.prevT[k] = q[16 + k]; }
    S.prev_err = q[32];
    S.kind = (int)q[33];
    first[i] = (int)q[34];
    level[i] = (int)q[35];
    if (level[i] < 0 || level[i] >= MAX_PYR || (S.kind != 0 && S.kind != 1)) {
      ctx->last_error = "mf_debug_gn_step: level or kind out of range";
      return MF_E_ARG;
    }
    S.Tf = to_m4f(S.T);
    S.invTf = inverse(S.Tf);
  }
  GNState* d_st = nullptr;
  double* d_sums = nullptr;
  int* d_int = nullptr;
  int rc = MF_OK;
  if (cudaMalloc(&d_st, sizeof(GNState) * n) != cudaSuccess ||
      cudaMalloc(&d_sums, sizeof(double) * 32 * n) != cudaSuccess ||
      cudaMalloc(&d_int, sizeof(int) * 2 * n) != cudaSuccess) {
    ctx->last_error = "mf_debug_gn_step: allocation failed";
    rc = MF_E_CUDA;
  }
  std::vector<GNState> ds(n);
  if (rc == MF_OK) {
    cudaMemcpyAsync(d_st, hs.data(), sizeof(GNState) * n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_sums, sums, sizeof(double) * 32 * n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_int, first.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(d_int + n, level.data(), sizeof(int) * n, cudaMemcpyHostToDevice,
                    ctx->stream);
    gn_step_check_kernel<<<n, 32, 0, ctx->stream>>>(d_st, d_sums, d_int, d_int + n);
    cudaMemcpyAsync(ds.data(), d_st, sizeof(GNState) * n, cudaMemcpyDeviceToHost, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      ctx->last_error = std::string("mf_debug_gn_step: ") + cudaGetErrorString(e);
      rc = MF_E_CUDA;
    }
  }
  if (d_st) cudaFree(d_st);
  if (d_sums) cudaFree(d_sums);
  if (d_int) cudaFree(d_int);
  if (rc) return rc;
  for (int i = 0; i < n; ++i) {
    GNState& S = hs[i];
    if (first[i]) S.prev_err = INFINITY;
    gn_step(S, sums + 32 * i, level[i]);
    gn_step_out(S, level[i], out_host + 68 * i);
    gn_step_out(ds[i], level[i], out_dev + 68 * i);
  }
  return MF_OK;
}

// ------------------------------------------------------------------------
// Camera cost at level 0 and its adjoint (no reference counterpart).
//
//   E(T_live, tsdf) = sum_p rho(e_icp(p)) + rho(e_rgb(p))
//
// with the camera rows of gn_iter_kernel (the same validity tests, residuals,
// whitening and robust kernel) at level 0.  Per valid row the kernel adds
// rho'(e) de/d(twist) -- the exact derivative for a left perturbation
// T <- exp(twist) T_live, with the bilinear image gradient of the photometric
// lookup -- and, when asked, rho'(e) de/d(model vertex, normal) into per
// model-pixel FP64 buffers, which the raycast adjoint then carries back to the
// TSDF voxels.  ICP: e = ic n.(v_m - T v) with ic = (n^T P n)^(-1/2).
// Photometric: e = ic_rgb (I_ref(p) - I_live(pi(K T^-1 T_w_r rv(p)))), where
// the reference vertex rv(p) = d(p) K^-1 (x, y, 1) and d(p) is the depth of the
// model vertex at p in the reference camera.
struct CostOut {
  double* partials;  // 8 per CTA: loss, dE/d twist (6), rows
  double* gV;        // 3 per model pixel (may be null)
  double* gN;
  int want_grad;
};

__device__ __forceinline__ void atomic_add3(double* p, F3 v) {
  atomicAdd(p, (double)v.x);
  atomicAdd(p + 1, (double)v.y);
  atomicAdd(p + 2, (double)v.z);
}

__global__ void __launch_bounds__(256)
camera_cost_kernel(GNArgs a, CostOut c) {
  const GNState& S = a.st[0];
  const int w = a.pyr.w[0], h = a.pyr.h[0];
  const int p = blockIdx.x * 256 + threadIdx.x;
  float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // loss, grad[6], rows
  if (p < w * h) {
    // ---- ICP (icp_camera)
    if (a.use_icp && !a.pyr.MASK[0][p]) {
      const F3 nl = a.pyr.N[0][p];
      if (nl.x != INVALIDF) {
        const F3 pv = xform(S.Tf, a.pyr.V[a.cur][0][p]);
        const F3 pp = xform(S.view, pv);
        const float px = pp.x / pp.z, py = pp.y / pp.z;
        if (!(px < 1 || px > (float)(unsigned)(a.W - 2) || py < 1 ||
              py > (float)(unsigned)(a.H - 2) || isnan(px) || isnan(py))) {
          const int q = (int)((unsigned)px + (unsigned)py * a.W);
          const F3 rn = a.mnormal[q];
          if (rn.x != INVALIDF) {
            const F3 diff = a.mvertex[q] - pv;
            const F3 pn = rotate(S.Tf, nl);
            if (!(length(diff) > 0.1f) && !(dot(pn, rn) < 0.8f)) {
              const F3 P = a.pyr.COV[0][p];
              const float sig = rn.x * rn.x * P.x + rn.y * rn.y * P.y + rn.z * rn.z * P.z;
              const float ic = sqrtf((float)(1.0 / (double)sig));
              const float e = ic * dot(rn, diff);
              float wt, loss;
              robust(e, a.robust, wt, loss);
              const float de = wt * e;  // rho'(e)
              v[0] += loss;
              v[7] += 1.f;
              // de/d(v, w) = -ic (n, pv x n)
              const F3 j1 = cross(pv, rn);
              v[1] -= de * ic * rn.x; v[2] -= de * ic * rn.y; v[3] -= de * ic * rn.z;
              v[4] -= de * ic * j1.x; v[5] -= de * ic * j1.y; v[6] -= de * ic * j1.z;
              if (c.want_grad) {
                atomic_add3(c.gV + 3 * (size_t)q, (de * ic) * rn);
                // d ic / d n = -ic^3 (n * P)
                const float ic3 = ic * ic * ic;
                const F3 dic = mk3(-ic3 * rn.x * P.x, -ic3 * rn.y * P.y, -ic3 * rn.z * P.z);
                atomic_add3(c.gN + 3 * (size_t)q, de * (ic * diff + dot(rn, diff) * dic));
              }
            }
          }
        }
      }
    }
    // ---- photometric (rgb_row, camera, level 0)
    if (a.use_rgb) {
      const F3 rv = a.rV[0][p];
      const F3 rl = a.pyr.V[1 - a.cur][0][p];
      if (!(rv.z <= 0.f || rv.z == INVALIDF) && !(length(rv - rl) > 0.1f && rl.z > 0.f)) {
        const M4 KL = camera_matrix(a.kL);
        const F3 wv = xform(S.T_w_r, rv);
        const F3 lv = xform(S.invTf, wv);
        const F3 pr = rotate(KL, lv);
        const float px = pr.x / pr.z, py = pr.y / pr.z;
        if (!(px < 1 || px > (float)(unsigned)(w - 2) || py < 1 || py > (float)(unsigned)(h - 2) ||
              isnan(px) || isnan(py))) {
          const float* IL = a.pyr.I[a.cur][0];
          const float fx0 = floorf(px), fy0 = floorf(py);
          const int bx = (int)fx0, by = (int)fy0;
          const float ax = px - fx0, ay = py - fy0;
          const float i00 = IL[bx + by * w], i10 = IL[bx + 1 + by * w];
          const float i01 = IL[bx + (by + 1) * w], i11 = IL[bx + 1 + (by + 1) * w];
          const float residual = a.pyr.I[1 - a.cur][0][p] - bil(IL, w, px, py);
          const float ic = a.inv_cov_rgb;
          const float e = ic * residual;
          float wt, loss;
          robust(e, a.robust, wt, loss);
          const float de = wt * e;
          v[0] += loss;
          v[7] += 1.f;
          // d bil / d(px, py) of the bilinear interpolation itself
          const float gx = (i10 - i00) * (1.f - ay) + (i11 - i01) * ay;
          const float gy = (i01 - i00) * (1.f - ax) + (i11 - i10) * ax;
          const float fxk = KL.r[0].x, fyk = KL.r[1].y, iz = 1.f / lv.z;
          // de/d lv = -ic (gx dpx/dlv + gy dpy/dlv)
          const F3 g_lv = -ic * mk3(gx * fxk * iz, gy * fyk * iz,
                                     -(gx * fxk * lv.x + gy * fyk * lv.y) * iz * iz);
          const F3 g3 = rotate_t(g_lv, S.invTf);  // in world coordinates
          const F3 j1 = cross(wv, g3);
          // lv = T^-1 exp(-twist) wv: de/d(v, w) = -(g3, wv x g3)
          v[1] -= de * g3.x; v[2] -= de * g3.y; v[3] -= de * g3.z;
          v[4] -= de * j1.x; v[5] -= de * j1.y; v[6] -= de * j1.z;
          if (c.want_grad) {
            // rv = d K^-1 (x, y, 1), d = (T_w_r^-1 v_m).z
            const int x = p % w, y = p / w;
            const F3 ray = rotate(inverse_camera_matrix(a.kL), mk3((float)x, (float)y, 1.f));
            const float g_d = dot(rotate_t(g3, S.T_w_r), ray);
            atomic_add3(c.gV + 3 * (size_t)p, (de * g_d) * xyz(S.inv_T_w_r.r[2]));
          }
        }
      }
    }
  }
  // FP64 block sums, fixed order
  __shared__ double sh[8][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    double d = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if (lane == 0) sh[warp][i] = d;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double d = 0;
    for (int i = 0; i < 8; ++i) d += sh[i][threadIdx.x];
    c.partials[(size_t)blockIdx.x * 8 + threadIdx.x] = d;
  }
}

__global__ void cost_sum_kernel(const double* __restrict__ partials, int n, double* out) {
  if (threadIdx.x >= 8) return;
  double d = 0;
#pragma unroll 8
  for (int b = 0; b < n; ++b) d += partials[(size_t)b * 8 + threadIdx.x];
  out[threadIdx.x] = d;
}

// Camera problem (slot 0) for a cost evaluation: reference pose = the current
// camera pose, live pose = T_live.
__global__ void cost_setup_kernel(GNState* st, const float* __restrict__ Twc, F4 k, M4 Tl,
                                  M4 iTl) {
  GNState& S = st[0];
  const M4 T = load_m4(Twc);
  S.kind = 0; S.label = 0; S.inst = 0; S.done = 0; S.ticket = 0;
  S.T_w_r = T;
  S.inv_T_w_r = inverse(T);
  S.view = mul(camera_matrix(k), S.inv_T_w_r);
  S.Tf = Tl;
  S.invTf = iTl;
}

int camera_cost(Context* ctx, const float* T_live16, int want_grad, double* out8,
                float* d_grad) {
  if (!ctx->track || !ctx->track->have_ref) {
    ctx->last_error = "mf_camera_cost: needs a reference frame (mf_set_ref_from_current) "
                      "and a preprocessed live frame";
    return MF_E_STATE;
  }
  TrackState& T = *ctx->track;
  const size_t WH = (size_t)ctx->W * ctx->H;
  const int nb = (int)((WH + 255) / 256);
  if (!T.d_cost) {
    MF_CUDA(cudaMalloc(&T.d_gmodel, sizeof(double) * 6 * WH));
    MF_CUDA(cudaMalloc(&T.d_cost_part, sizeof(double) * 8 * nb));
    MF_CUDA(cudaMalloc(&T.d_cost, sizeof(double) * 8));
    T.allocs.push_back(T.d_gmodel);
    T.allocs.push_back(T.d_cost_part);
    T.allocs.push_back(T.d_cost);
    T.cost_blocks = nb;
  }
  // the model maps of the current TSDF at the current (reference) camera pose
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  if (int rc = stage_prepare(ctx, all)) return rc;
  if (int rc = stage_raycast(ctx, all, ctx->ray_epsilon)) return rc;
  M4 Tl;
  std::memcpy(&Tl, T_live16, 64);
  const mf_config& c = ctx->cfg;
  T.slot_kind[0] = 0;
  cost_setup_kernel<<<1, 1, 0, ctx->stream>>>(T.d_state, ctx->d_Twc,
                                              F4{c.k[0], c.k[1], c.k[2], c.k[3]}, Tl,
                                              inverse(Tl));
  MF_CUDA(cudaGetLastError());
  IdList cam;
  cam.n = 1;
  cam.v[0] = 0;
  if (int rc = render_reference(ctx, cam)) return rc;
  double* gV = want_grad ? T.d_gmodel : nullptr;
  double* gN = want_grad ? T.d_gmodel + 3 * WH : nullptr;
  if (want_grad) MF_CUDA(cudaMemsetAsync(T.d_gmodel, 0, sizeof(double) * 6 * WH, ctx->stream));
  const GNArgs a = make_args(ctx, 0, 0);
  camera_cost_kernel<<<nb, 256, 0, ctx->stream>>>(a, CostOut{T.d_cost_part, gV, gN, want_grad});
  cost_sum_kernel<<<1, 32, 0, ctx->stream>>>(T.d_cost_part, nb, T.d_cost);
  MF_CUDA(cudaGetLastError());
  if (want_grad && d_grad)
    if (int rc = stage_raycast_adjoint(ctx, all, gV, gN, d_grad)) return rc;
  MF_CUDA(cudaMemcpyAsync(out8, T.d_cost, sizeof(double) * 8, cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}


// ------------------------------------------------------------------------
// Motion residuals (Tracking::compute_residuals, tracking.cpp:1535-1553,
// compute_residual_kernel :1555-1612, compute_icp_residual_kernel :1615-1677,
// compute_rgb_residual_kernel :1680-1747) and the moving-object test
// (check_static_state, rendering/rendering.cpp:907-947, and the inlier ratio
// of kfusion.cpp:312-341).  T_w_l is the freshly tracked camera pose, T_w_r
// the reference pose of the model maps; the photometric reference vertices
// come from the model raycast at T_w_l with the objects at their last poses,
// turned into depth relative to T_w_r (vertex2depth with T_w_r, as the
// reference passes it, preprocessing.cpp:292-309) and back into vertices.
struct MotionArgs {
  PyrPtrs pyr;
  int cur, W, H;
  const F3* mvertex; const F3* mnormal;   // model maps at T_w_r
  const int* mlabel;
  const F3* lvert;                          // model vertices raycast at T_w_l
  const int* llabel;
  int obj_label;    // >= 0: one object's maps (its pixels of the composite maps,
                    // m_vertex / m_normal, and of the live raycast,
                    // m_vertex_bef_integ, rendering.cpp:152-176), no counts
  M4 T_w_l, T_w_r, inv_T_w_r, K, invK;
  float sigma_bright, threshold;
  int use_icp, use_rgb;
  int8_t* res; float* err;
  int* count;                               // [label]: object pixels, [32 + label]: inliers
};

__global__ void motion_residual_kernel(MotionArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = a.W * a.H;
  if (p >= n) return;
  const int x = p % a.W, y = p / a.W;
  int8_t ri = 0, rr = 0;
  float ei = 0.f, er = 0.f;
  // the outlier-mask test of :1586-1590 never fires: the reference's
  // outlier_mask_ stays the all-zero mask of set_params_frame (:170), since
  // the mask variant of trackLiveFrame keeps its pyramid local (:1781-1787)
  {
    if (a.use_icp) {
      const F3 ln = a.pyr.N[0][p];
      if (ln.x == INVALIDF) {
        ri = -1;
      } else {
        const F3 w_vertex = xform(a.T_w_l, a.pyr.V[a.cur][0][p]);
        const F3 r_vertex = xform(a.inv_T_w_r, w_vertex);
        const F3 proj = rotate(a.K, r_vertex);
        const float px = proj.x / proj.z, py = proj.y / proj.z;
        if (px < 1 || px > (float)(unsigned)(a.W - 2) || py < 1 || py > (float)(unsigned)(a.H - 2) ||
            isnan(px) || isnan(py)) {
          ri = -2;
        } else {
          const int q = (int)((unsigned)px + (unsigned)py * a.W);
          const bool own = a.obj_label < 0 || a.mlabel[q] == a.obj_label;
          const F3 rn = own ? a.mnormal[q] : mk3(INVALIDF, 0.f, 0.f);
          const F3 rv = own ? a.mvertex[q] : mk3(0.f);
          if (rn.x == INVALIDF) {
            ri = -3;
          } else {
            const F3 diff = rv - w_vertex;
            const F3 wn = rotate(a.T_w_l, ln);
            if (length(diff) > 0.1f) ri = -4;
            else if (dot(wn, rn) < 0.8f) ri = -5;
            else {
              const F3 P = a.pyr.COV[0][p];
              const double sig = rn.x * rn.x * P.x + rn.y * rn.y * P.y + rn.z * rn.z * P.z;
              const double e = sqrt(1.0 / sig) * dot(rn, diff);
              if (fabs(e) > a.threshold) ri = -4;
              else { ri = 1; ei = (float)e; }
            }
          }
        }
      }
    }
    if (a.use_rgb) {
      // rendered live vertex -> depth relative to T_w_r -> vertex
      const F3 vl = (a.obj_label < 0 || a.llabel[p] == a.obj_label) ? a.lvert[p] : mk3(0.f);
      const float d = vl.z > 0.0 ? xform(a.inv_T_w_r, vl).z : 0.f;
      const F3 ref = d > 0 ? d * rotate(a.invK, mk3((float)x, (float)y, 1.f)) : mk3(0.f);
      const F3 live = a.pyr.V[a.cur][0][p];
      if (ref.z <= 0.f || ref.z == INVALIDF) {
        rr = -1;
      } else if (length(ref - live) > 0.1f && live.z > 0.f) {
        rr = -5;
      } else {
        const F3 w_vertex = xform(a.T_w_l, ref);
        const F3 r_vertex = xform(a.inv_T_w_r, w_vertex);
        const F3 proj = rotate(a.K, r_vertex);
        const float px = proj.x / proj.z, py = proj.y / proj.z;
        if (px < 1 || px > (float)(unsigned)(a.W - 2) || py < 1 || py > (float)(unsigned)(a.H - 2) ||
            isnan(px) || isnan(py)) {
          rr = -2;
        } else {
          const float residual = a.pyr.I[a.cur][0][p] - bil(a.pyr.I[1 - a.cur][0], a.W, px, py);
          const double e = (1.0 / a.sigma_bright) * residual;
          if (fabs(e) > a.threshold) rr = -4;
          else { rr = 1; er = (float)e; }
        }
      }
    }
  }
  a.res[p] = ri; a.res[n + p] = rr;
  if (a.err) { a.err[p] = ei; a.err[n + p] = er; }
  if (a.obj_label >= 0) return;
  // check_static_state: an object pixel of the live render is an inlier when
  // its rows' results are > -3
  const int l = a.llabel[p];
  if (l >= 1 && l < 32) {
    bool inl;
    if (a.use_icp && a.use_rgb) inl = ri > -3 && rr > -3;
    else if (a.use_icp) inl = ri > -3;
    else inl = a.use_rgb && rr > -3;
    atomicAdd(a.count + l, 1);
    if (inl) atomicAdd(a.count + 32 + l, 1);
  }
}

// Object::refine_mask_use_motion (object/object.cpp:255-315, outliers not
// absorbed into the background): inside the band, pixels whose ICP row is -4
// or -6, or whose photometric row is below -3, leave the object's mask.
__global__ void refine_mask_kernel(float* __restrict__ mask, const int8_t* __restrict__ res,
                                   int n, int use_icp, int use_rgb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || !(mask[p] >= 0)) return;
  if (use_icp && (res[p] == -4 || res[p] == -6)) { mask[p] = -1; return; }
  if (use_rgb && res[n + p] < -3) mask[p] = -1;
}

// Object::static_object, object.cpp:326: classes that never move (tv 63,
// and 69, 70)
static bool never_moving_class(int c) { return c == 63 || c == 69 || c == 70; }

int motion_residuals(Context* ctx, float threshold, float moved, float* ratio,
                     uint32_t* moving) {
  if (!ctx->track || !ctx->track->have_ref) {
    ctx->last_error = "mf_motion_residuals: needs a reference frame and a tracked live frame";
    return MF_E_STATE;
  }
  TrackState& T = *ctx->track;
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (!T.d_mres) {
    MF_CUDA(cudaMalloc(&T.d_mres, 2 * WH));
    T.allocs.push_back(T.d_mres);
    MF_CUDA(cudaMalloc(&T.d_merr, sizeof(float) * 2 * WH));
    T.allocs.push_back(T.d_merr);
    MF_CUDA(cudaMalloc(&T.d_lvert, sizeof(F3) * WH));
    T.allocs.push_back(T.d_lvert);
    MF_CUDA(cudaMalloc(&T.d_lnorm, sizeof(F3) * WH));
    T.allocs.push_back(T.d_lnorm);
    MF_CUDA(cudaMalloc(&T.d_llabel, sizeof(int) * WH));
    T.allocs.push_back(T.d_llabel);
    MF_CUDA(cudaMalloc(&T.d_mcount, sizeof(int) * 64));
    T.allocs.push_back(T.d_mcount);
    // like the reference's persistent render buffers, the maps start zeroed
    // and keep what a later raycast does not overwrite
    MF_CUDA(cudaMemsetAsync(T.d_lvert, 0, sizeof(F3) * WH, ctx->stream));
    MF_CUDA(cudaMemsetAsync(T.d_lnorm, 0, sizeof(F3) * WH, ctx->stream));
    MF_CUDA(cudaMemsetAsync(T.d_llabel, 0, sizeof(int) * WH, ctx->stream));
  }
  // the model raycast at the live pose, objects at their last poses
  // (kfusion.cpp:291-296)
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  if (int rc = stage_prepare(ctx, all)) return rc;
  if (int rc = stage_raycast_to(ctx, all, ctx->ray_epsilon, T.d_lvert, T.d_lnorm, T.d_llabel))
    return rc;
  float Tl[16], Tr[16];
  MF_CUDA(cudaMemcpyAsync(Tl, ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(Tr, T.d_Twc_prev, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemsetAsync(T.d_mcount, 0, sizeof(int) * 64, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  const mf_config& c = ctx->cfg;
  const F4 k{c.k[0], c.k[1], c.k[2], c.k[3]};
  MotionArgs a;
  a.pyr = T.pyr;
  a.cur = T.cur;
  a.W = ctx->W;
  a.H = ctx->H;
  a.mvertex = ctx->d_vertex;
  a.mnormal = ctx->d_normal;
  a.mlabel = ctx->d_label;
  a.lvert = T.d_lvert;
  a.llabel = T.d_llabel;
  a.obj_label = -1;
  a.T_w_l = load_m4(Tl);
  a.T_w_r = load_m4(Tr);
  a.inv_T_w_r = inverse(a.T_w_r);
  a.K = camera_matrix(k);
  a.invK = inverse_camera_matrix(k);
  a.sigma_bright = (float)(sqrtf(100.0f) / 255.0);  // tracking.cpp:766-772
  a.threshold = threshold;
  a.use_icp = c.use_icp;
  a.use_rgb = c.use_rgb;
  a.res = T.d_mres;
  a.err = T.d_merr;
  a.count = T.d_mcount;
  motion_residual_kernel<<<div_up((long long)WH, 256), 256, 0, ctx->stream>>>(a);
  MF_CUDA(cudaGetLastError());
  int cnt[64];
  MF_CUDA(cudaMemcpyAsync(cnt, T.d_mcount, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  // kfusion.cpp:312-338: an object in view (with pixels in the live render)
  // moves when move-out threshold 0.05 < inliers / pixels < `moved` and its
  // class is not one of the never-moving classes (Object::static_object)
  uint32_t mv = 0;
  for (int i = 0; i < (int)ctx->inst.size(); ++i) {
    const int l = ctx->inst[i].label;
    float r = -1.f;
    if (i >= 1 && l >= 1 && l < 32 && cnt[l] > 0) {
      r = static_cast<float>(cnt[32 + l]) / (cnt[l]);
      if (r < moved && r > 0.05f && !never_moving_class(ctx->inst[i].class_id)) mv |= 1u << l;
    }
    if (ratio) ratio[i] = r;
  }
  if (moving) *moving = mv;
  return MF_OK;
}

// kfusion.cpp:446-466: a moving object's result rows recomputed after its
// tracking, Tracking::compute_residuals at the object's virtual camera pose
// (tracking.cpp:696) against its own model maps (m_vertex / m_normal: its
// pixels of the last frame's composite maps) and its pixels of the live
// raycast (m_vertex_bef_integ, the raycast at the current camera pose and the
// objects' new poses, i.e. the last mf_motion_residuals).  Rows (2 x W*H
// int8) to d_rows; the virtual pose (16 floats) to T_virtual when given.
int object_residuals(Context* ctx, int i, float threshold, int8_t* d_rows, float* T_virtual) {
  TrackState* T = ctx->track;
  if (!T || !T->have_ref || !T->d_mres || T->slot_kind[i] != 1) {
    ctx->last_error = "mf_object_residuals: needs the object tracked (mf_track_objects) and "
                      "the live raycast of mf_motion_residuals";
    return MF_E_STATE;
  }
  GNState S;
  MF_CUDA(cudaMemcpyAsync(&S, T->d_state + i, sizeof(GNState), cudaMemcpyDeviceToHost,
                          ctx->stream));
  float Tr[16];
  MF_CUDA(cudaMemcpyAsync(Tr, T->d_Twc_prev, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  const mf_config& c = ctx->cfg;
  const F4 k{c.k[0], c.k[1], c.k[2], c.k[3]};
  MotionArgs a;
  a.pyr = T->pyr;
  a.cur = T->cur;
  a.W = ctx->W;
  a.H = ctx->H;
  a.mvertex = ctx->d_vertex;
  a.mnormal = ctx->d_normal;
  a.mlabel = ctx->d_label;
  a.lvert = T->d_lvert;
  a.llabel = T->d_llabel;
  a.obj_label = ctx->inst[i].label;
  a.T_w_l = S.T_virtual;
  a.T_w_r = load_m4(Tr);
  a.inv_T_w_r = inverse(a.T_w_r);
  a.K = camera_matrix(k);
  a.invK = inverse_camera_matrix(k);
  a.sigma_bright = (float)(sqrtf(100.0f) / 255.0);  // tracking.cpp:766-772
  a.threshold = threshold;
  a.use_icp = c.use_icp;
  a.use_rgb = c.use_rgb;
  a.res = d_rows;
  a.err = nullptr;
  a.count = nullptr;
  const size_t WH = (size_t)ctx->W * ctx->H;
  motion_residual_kernel<<<div_up((long long)WH, 256), 256, 0, ctx->stream>>>(a);
  MF_CUDA(cudaGetLastError());
  if (T_virtual) store_m4(T_virtual, S.T_virtual);
  return MF_OK;
}

int motion_download(Context* ctx, int8_t* res, float* err, float* lvert, int32_t* llabel) {
  TrackState* T = ctx->track;
  if (!T || !T->d_mres) {
    ctx->last_error = "mf_motion_download: no motion residuals yet";
    return MF_E_STATE;
  }
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (res) MF_CUDA(cudaMemcpyAsync(res, T->d_mres, 2 * WH, cudaMemcpyDeviceToHost, ctx->stream));
  if (err)
    MF_CUDA(cudaMemcpyAsync(err, T->d_merr, sizeof(float) * 2 * WH, cudaMemcpyDeviceToHost,
                            ctx->stream));
  if (lvert)
    MF_CUDA(cudaMemcpyAsync(lvert, T->d_lvert, sizeof(F3) * WH, cudaMemcpyDeviceToHost,
                            ctx->stream));
  if (llabel)
    MF_CUDA(cudaMemcpyAsync(llabel, T->d_llabel, sizeof(int) * WH, cudaMemcpyDeviceToHost,
                            ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

// The result codes of problem `slot`'s rows at level 0, evaluated at the pose
// of its last level-0 GN iteration: Tracking::trackingResult_[0] after
// trackLiveFrame / trackEachObject, which kfusion.cpp:282-283 and :397-405
// copy into Object::trackresult_.  ICP rows first, then photometric rows; a
// term that is switched off leaves 0.
__global__ void row_codes_kernel(GNArgs a, int slot, int8_t* __restrict__ out,
                                 float* __restrict__ out_err) {
  __shared__ GNState S;
  if (threadIdx.x == 0) {
    S = a.st[slot];
    S.Tf = S.evalTf;
    S.invTf = inverse(S.evalTf);
  }
  __syncthreads();
  const int w = a.pyr.w[0], h = a.pyr.h[0], n = w * h;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  Row r;
  int8_t ci = 0, cr = 0;
  float ei = 0.f, er = 0.f;  // TrackData::error of rows with result 1
  if (a.use_icp) {
    r.result = 0;
    if (S.kind == 0) icp_camera(a, S, 0, p, r);
    else icp_object(a, S, 0, p, r);
    ci = (int8_t)r.result;
    if (ci == 1) ei = r.e;
  }
  if (a.use_rgb) {
    r.result = 0;
    rgb_row(a, S, a.rV[slot], 0, p, w, h, r);
    cr = (int8_t)r.result;
    if (cr == 1) er = r.e;
  }
  out[p] = ci;
  out[n + p] = cr;
  if (out_err) {
    out_err[p] = ei;
    out_err[n + p] = er;
  }
}

int track_results(Context* ctx, int slot, int8_t* d_out, float* d_err, float* pose_eval) {
  if (!ctx->track || !ctx->track->have_ref) {
    ctx->last_error = "mf_track_results: no tracking has run";
    return MF_E_STATE;
  }
  const int n = ctx->W * ctx->H;
  GNArgs a = make_args(ctx, 0, 0);
  row_codes_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(a, slot, d_out, d_err);
  MF_CUDA(cudaGetLastError());
  if (pose_eval) {
    static_assert(sizeof(M4) == 64, "M4 is 16 row-major floats");
    MF_CUDA(cudaMemcpyAsync(pose_eval, &ctx->track->d_state[slot].evalTf, sizeof(M4),
                            cudaMemcpyDeviceToHost, ctx->stream));
    MF_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return MF_OK;
}

int refine_mask_use_motion(Context* ctx, int id, const int8_t* d_res, int use_icp, int use_rgb) {
  TrackState* T = ctx->track;
  if (!d_res) {
    if (!T || !T->d_mres) {
      ctx->last_error = "mf_refine_mask_use_motion: no motion residuals yet";
      return MF_E_STATE;
    }
    d_res = T->d_mres;
  }
  const int n = ctx->W * ctx->H;
  refine_mask_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(ctx->d_masks + (size_t)id * n,
                                                              d_res, n, use_icp, use_rgb);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}


// The planes of the last mf_motion_residuals (for renders), or MF_E_STATE.
int motion_planes(Context* ctx, const int8_t** res, const float** err) {
  if (!ctx->track || !ctx->track->d_mres) {
    ctx->last_error = "no motion residuals yet";
    return MF_E_STATE;
  }
  *res = ctx->track->d_mres;
  *err = ctx->track->d_merr;
  return MF_OK;
}

}  // namespace mf

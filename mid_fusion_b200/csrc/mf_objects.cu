// Object management next to the hot path: the placement of a new object's
// volume (Kfusion::spawnNewObjectKernel, apps/kfusion/src/cpp/kfusion.cpp:
// 1080-1150) and the per-object semantic class fusion
// (Object::fuseSemanticLabel, apps/kfusion/src/cpp/object/object.cpp:223-252).
#include <cmath>
#include <cstring>
#include <vector>
#include "mf_internal.h"

namespace mf {

constexpr int SPAWN_THREADS = 1024;

// The masked pixels' world vertices (depth2vertexKernel with the level-0
// inverse intrinsics, then T_w_c), reduced in the reference's row-major order:
// every chunk of 1024 pixels is compacted in order into shared memory and one
// thread folds it into the running minima, maxima and float sums, so the
// float sums round exactly as the reference's sequential loop does.
__global__ void __launch_bounds__(SPAWN_THREADS)
spawn_stats_kernel(const float* __restrict__ depth, const uint8_t* __restrict__ mask, int W,
                   int H, M4 invK, M4 T_w_c, float* __restrict__ out) {
  __shared__ F3 s_v[SPAWN_THREADS];
  __shared__ int s_warp[SPAWN_THREADS / 32 + 1];
  const int n = W * H, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  float sum[3] = {0.f, 0.f, 0.f};
  int count = 0;
  for (int base = 0; base < n; base += SPAWN_THREADS) {
    const int p = base + t;
    const bool m = p < n && mask[p] != 0;
    F3 w = mk3(0.f);
    if (m) {
      const int x = p % W, y = p / W;
      const float d = depth[p];
      const F3 v = d > 0 ? d * rotate(invK, mk3((float)x, (float)y, 1.f)) : mk3(0.f);
      w = xform(T_w_c, v);
    }
    const unsigned ball = __ballot_sync(0xffffffffu, m);
    if (lane == 0) s_warp[warp] = __popc(ball);
    __syncthreads();
    if (t == 0) {  // exclusive prefix over the warps
      int acc = 0;
      for (int i = 0; i < SPAWN_THREADS / 32; ++i) {
        const int c = s_warp[i];
        s_warp[i] = acc;
        acc += c;
      }
      s_warp[SPAWN_THREADS / 32] = acc;
    }
    __syncthreads();
    if (m) s_v[s_warp[warp] + __popc(ball & ((1u << lane) - 1u))] = w;
    __syncthreads();
    if (t == 0) {
      const int k = s_warp[SPAWN_THREADS / 32];
      for (int i = 0; i < k; ++i) {
        const F3 v = s_v[i];
        if (v.x > mx[0]) mx[0] = v.x;
        if (v.x < mn[0]) mn[0] = v.x;
        if (v.y > mx[1]) mx[1] = v.y;
        if (v.y < mn[1]) mn[1] = v.y;
        if (v.z > mx[2]) mx[2] = v.z;
        if (v.z < mn[2]) mn[2] = v.z;
        sum[0] += v.x;
        sum[1] += v.y;
        sum[2] += v.z;
      }
      count += k;
    }
    __syncthreads();
  }
  if (t == 0) {
    for (int i = 0; i < 3; ++i) {
      out[i] = mn[i];
      out[3 + i] = mx[i];
      out[6 + i] = sum[i];
    }
    out[9] = __int_as_float(count);
  }
}

int spawn_object(Context* ctx, const uint8_t* mask, float* T_w_o, float* volume_size,
                 int* volume_resol) {
  const size_t WH = (size_t)ctx->W * ctx->H;
  // the mask and the 10 result words share one staging allocation
  const size_t mask_bytes = (WH + 15) / 16 * 16;
  if (int rc = ensure_export(ctx, mask_bytes + 64)) return rc;
  uint8_t* d_mask = (uint8_t*)ctx->d_export;
  float* d_out = (float*)(d_mask + mask_bytes);
  MF_CUDA(cudaMemcpyAsync(d_mask, mask, WH, cudaMemcpyDefault, ctx->stream));
  float Tc[16];
  MF_CUDA(cudaMemcpyAsync(Tc, ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  const mf_config& c = ctx->cfg;
  spawn_stats_kernel<<<1, SPAWN_THREADS, 0, ctx->stream>>>(
      ctx->d_depth, d_mask, ctx->W, ctx->H,
      inverse_camera_matrix(F4{c.k[0], c.k[1], c.k[2], c.k[3]}), load_m4(Tc), d_out);
  MF_CUDA(cudaGetLastError());
  float s[10];
  MF_CUDA(cudaMemcpyAsync(s, d_out, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  int count;
  std::memcpy(&count, &s[9], sizeof(int));
  // kfusion.cpp:1119-1146 (float arithmetic, the reference's comparison-based
  // fminf / fmaxf)
  const float x_avg = s[6] / count, y_avg = s[7] / count, z_avg = s[8] / count;
  const float ex = s[3] - s[0], ey = s[4] - s[1], ez = (s[5] - s[2]) / 2;
  const float max_size = fmx(ex, fmx(ey, ez));
  const float size = fmn((float)(2.5 * max_size), 5.0f);
  int resol = 0;  // the reference leaves it unset outside its four ranges
  if (size < 0.64) resol = 256;
  if ((0.64 < size) && (size < 1.28)) resol = 512;
  if ((1.28 < size) && (size < 2.56)) resol = 1024;
  if ((2.56 < size) && (size < 5.12)) resol = 2048;
  for (int i = 0; i < 16; ++i) T_w_o[i] = (i % 5 == 0) ? 1.f : 0.f;
  T_w_o[3] = x_avg - size / 2;
  T_w_o[7] = y_avg - size / 2;
  T_w_o[11] = z_avg - size / 2;
  *volume_size = size;
  *volume_resol = resol;
  return count;
}

// Object::Object (object.cpp:11-34): the class probabilities and class id of
// the segmentation that created the object, fused once.
int set_semantics(Context* ctx, int id, int class_id, const float* probs, int n) {
  Instance& in = ctx->inst[id];
  in.sem.assign(probs, probs + n);
  in.class_id = class_id;
  in.fused_time = 1;
  return MF_OK;
}

// Object::fuse_semantic_kernel + fuseSemanticLabel (object.cpp:197-252): a
// running mean of the class probabilities weighted by recognition counts, in
// float; the class is 1 + the first index of the largest mean probability.
int fuse_semantics(Context* ctx, int id, int class_id, const float* probs, int n,
                   int recog_times) {
  Instance& in = ctx->inst[id];
  if (class_id == 0) return MF_OK;
  if ((int)in.sem.size() != n) {
    ctx->last_error = "mf_fuse_semantics: label number differs from the object's";
    return MF_E_ARG;
  }
  const float ft = static_cast<float>(in.fused_time);
  const float rt = static_cast<float>(recog_times);
  const float tot = static_cast<float>(in.fused_time + recog_times);
  int best = 0;
  for (int i = 0; i < n; ++i) {
    in.sem[i] = (in.sem[i] * ft + probs[i] * rt) / tot;
    if (in.sem[i] > in.sem[best]) best = i;
  }
  in.class_id = best + 1;
  in.fused_time += recog_times;
  return MF_OK;
}

}  // namespace mf

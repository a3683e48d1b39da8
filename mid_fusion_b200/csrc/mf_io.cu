// Input and output formats around the hot path:
//  - Kfusion::preprocessing's input stage (apps/kfusion/src/cpp/kfusion.cpp:
//    210-217): uint16 millimetre depth and uchar3 colour of a sensor frame,
//    subsampled by an integer ratio, to metres, float colour and grey;
//  - the SLAMBench .raw sequence reader (RawDepthReader,
//    apps/kfusion/include/interface.h:207-335);
//  - the TUM-format pose writer (Kfusion::save_poses, kfusion.cpp:1591-1626).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "mf_internal.h"

namespace mf {

// mm2metersKernel (preprocessing.cpp:132-159) and rgb2intensity
// (preprocessing.cpp:73-102, rgb2gs commons.h:150-154): output pixel (x, y)
// reads input pixel (x * ratio, y * ratio).
__global__ void raw_frame_kernel(const uint16_t* __restrict__ depth_mm,
                                 const uint8_t* __restrict__ rgb8, int in_w, int ratio, int W,
                                 int H, float* __restrict__ depth, F3* __restrict__ rgb,
                                 float* __restrict__ grey) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= W * H) return;
  const int x = p % W, y = p / W;
  const size_t q = (size_t)x * ratio + (size_t)in_w * y * ratio;
  if (depth_mm) depth[p] = depth_mm[q] / 1000.0f;
  if (rgb8) {
    const uint8_t r8 = rgb8[3 * q], g8 = rgb8[3 * q + 1], b8 = rgb8[3 * q + 2];
    rgb[p] = mk3(r8 / 255.0f, g8 / 255.0f, b8 / 255.0f);
    grey[p] = (0.299f * r8 + 0.587f * g8 + 0.114f * b8) / 255.f;
  }
}

int frame_upload_raw(Context* ctx, const uint16_t* depth_mm, const uint8_t* rgb, int in_w,
                     int in_h) {
  // the reference's ratio checks (preprocessing.cpp:135-146), an error here
  if (in_w < ctx->W || in_h < ctx->H || in_w % ctx->W || in_h % ctx->H ||
      in_w / ctx->W != in_h / ctx->H) {
    ctx->last_error = "mf_frame_upload_raw: invalid ratio";
    return MF_E_ARG;
  }
  const int ratio = in_w / ctx->W;
  const size_t in_n = (size_t)in_w * in_h;
  const size_t dbytes = (2 * in_n + 15) / 16 * 16;
  if (int rc = ensure_export(ctx, dbytes + 3 * in_n)) return rc;
  uint16_t* d_d = (uint16_t*)ctx->d_export;
  uint8_t* d_c = (uint8_t*)ctx->d_export + dbytes;
  if (depth_mm)
    MF_CUDA(cudaMemcpyAsync(d_d, depth_mm, 2 * in_n, cudaMemcpyDefault, ctx->stream));
  if (rgb) MF_CUDA(cudaMemcpyAsync(d_c, rgb, 3 * in_n, cudaMemcpyDefault, ctx->stream));
  const int n = ctx->W * ctx->H;
  raw_frame_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(
      depth_mm ? d_d : nullptr, rgb ? d_c : nullptr, in_w, ratio, ctx->W, ctx->H, ctx->d_depth,
      ctx->d_rgb, ctx->d_grey);
  MF_CUDA(cudaGetLastError());
  // the caller's buffers are borrowed only for the call
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

// Quaternion (x, y, z, w) of the rotation part of a 4x4 pose: the trace /
// largest-diagonal method (Shoemake, "Animating rotation with quaternion
// curves", 1985), in float, the form getQuaternion (preprocessing.cpp:
// 312-320) gets from Eigen::Quaternionf's rotation-matrix constructor.
void pose_quaternion(const float* T, float* q) {
  auto m = [&](int i, int j) { return T[4 * i + j]; };
  float t = m(0, 0) + m(1, 1) + m(2, 2);
  if (t > 0.f) {
    t = std::sqrt(t + 1.0f);
    q[3] = 0.5f * t;
    t = 0.5f / t;
    q[0] = (m(2, 1) - m(1, 2)) * t;
    q[1] = (m(0, 2) - m(2, 0)) * t;
    q[2] = (m(1, 0) - m(0, 1)) * t;
  } else {
    int i = 0;
    if (m(1, 1) > m(0, 0)) i = 1;
    if (m(2, 2) > m(i, i)) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    t = std::sqrt(m(i, i) - m(j, j) - m(k, k) + 1.0f);
    q[i] = 0.5f * t;
    t = 0.5f / t;
    q[3] = (m(k, j) - m(j, k)) * t;
    q[j] = (m(j, i) + m(i, j)) * t;
    q[k] = (m(k, i) + m(i, k)) * t;
  }
}

// One line of Kfusion::save_poses: frame, translation, quaternion, each
// followed by a tab, as std::ostream prints floats by default (%g).
int tum_line(int frame, const float* T_translation, const float* T_rotation, char* buf,
             int cap) {
  float q[4];
  pose_quaternion(T_rotation, q);
  return std::snprintf(buf, cap, "%d\t%g\t%g\t%g\t%g\t%g\t%g\t%g\t\n", frame,
                       (double)T_translation[3], (double)T_translation[7],
                       (double)T_translation[11], (double)q[0], (double)q[1], (double)q[2],
                       (double)q[3]);
}

}  // namespace mf

// ------------------------------------------------------------------ .raw reader
// A SLAMBench .raw sequence: per frame uint32 (w, h), uint16 depth[w*h] in
// millimetres, uint32 (w, h), uchar3 rgb[w*h]; every frame the size of the
// first (RawDepthReader seeks to frame * frame_size).
struct mf_raw {
  FILE* f = nullptr;
  unsigned w = 0, h = 0;
  long long frame_bytes = 0, n_frames = 0, next = 0;
};

extern "C" {

int mf_raw_open(const char* path, mf_raw** out, int* width, int* height, long long* n_frames) {
  if (!path || !out) return MF_E_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return MF_E_NOT_FOUND;
  unsigned size[2];
  if (std::fread(size, sizeof(size), 1, f) != 1 || size[0] == 0 || size[1] == 0) {
    std::fclose(f);
    return MF_E_ARG;
  }
  mf_raw* r = new mf_raw;
  r->f = f;
  r->w = size[0];
  r->h = size[1];
  const long long n = (long long)size[0] * size[1];
  r->frame_bytes = 4 * (long long)sizeof(unsigned) + n * 2 + n * 3;
  std::fseek(f, 0, SEEK_END);
  r->n_frames = std::ftell(f) / r->frame_bytes;
  std::fseek(f, 0, SEEK_SET);
  *out = r;
  if (width) *width = (int)r->w;
  if (height) *height = (int)r->h;
  if (n_frames) *n_frames = r->n_frames;
  return MF_OK;
}

int mf_raw_read(mf_raw* r, long long frame, uint16_t* depth_mm, uint8_t* rgb) {
  if (!r) return MF_E_ARG;
  if (frame < 0) frame = r->next;
  if (frame >= r->n_frames) return MF_E_NOT_FOUND;  // end of the sequence
  std::fseek(r->f, (long)(frame * r->frame_bytes), SEEK_SET);
  unsigned size[2];
  const size_t n = (size_t)r->w * r->h;
  if (std::fread(size, sizeof(size), 1, r->f) != 1 || size[0] != r->w || size[1] != r->h)
    return MF_E_ARG;
  if (depth_mm) {
    if (std::fread(depth_mm, 2, n, r->f) != n) return MF_E_ARG;
  } else {
    std::fseek(r->f, (long)(2 * n), SEEK_CUR);
  }
  if (std::fread(size, sizeof(size), 1, r->f) != 1 || size[0] != r->w || size[1] != r->h)
    return MF_E_ARG;
  if (rgb && std::fread(rgb, 3, n, r->f) != n) return MF_E_ARG;
  r->next = frame + 1;
  return MF_OK;
}

int mf_raw_close(mf_raw* r) {
  if (!r) return MF_E_ARG;
  if (r->f) std::fclose(r->f);
  delete r;
  return MF_OK;
}

int mf_pose_quaternion(const float T[16], float q[4]) {
  if (!T || !q) return MF_E_ARG;
  mf::pose_quaternion(T, q);
  return MF_OK;
}

int mf_tum_line(int frame, const float T_translation[16], const float T_rotation[16], char* buf,
                int cap) {
  if (!T_translation || !T_rotation || !buf || cap <= 0) return MF_E_ARG;
  const int n = mf::tum_line(frame, T_translation, T_rotation, buf, cap);
  return n < cap ? n : MF_E_ARG;
}

}  // extern "C"

// Headless renders: the reference's visualisation kernels
// (apps/kfusion/src/cpp/rendering/rendering.cpp) as CUDA kernels writing
// uchar4 (or uchar3) images into device memory, one thread per pixel.  The
// shaded volume render, which raycasts, lives with the raycast in
// mf_raycast.cu; the colour conversions (to_u8) are in mf_common.cuh.
#include <cstring>
#include <vector>
#include "mf_internal.h"

namespace mf {

static int div_up(long long a, int b) { return (int)((a + b - 1) / b); }

// gs2rgb (apps/kfusion/include/commons.h:87-147): a fixed-value, fixed-
// saturation hue ramp over six sextants, in double.
__device__ uchar4 gs2rgb(double h) {
  const double v = 0.75, m = 0.25, sv = 0.6667;
  h *= 6.0;
  const int sextant = (int)h;
  const double fract = h - sextant;
  const double vsf = v * sv * fract;
  const double mid1 = m + vsf, mid2 = v - vsf;
  double r, g, b;
  switch (sextant) {
    case 0: r = v; g = mid1; b = m; break;
    case 1: r = mid2; g = v; b = m; break;
    case 2: r = m; g = v; b = mid1; break;
    case 3: r = m; g = mid2; b = v; break;
    case 4: r = mid1; g = m; b = v; break;
    case 5: r = v; g = m; b = mid2; break;
    default: r = 0; g = 0; b = 0; break;
  }
  return make_uchar4(to_u8d(r * 255), to_u8d(g * 255), to_u8d(b * 255), 0);
}

// renderDepthKernel, rendering.cpp:366-393.
__global__ void render_depth_kernel(const float* __restrict__ depth, int n, float nearPlane,
                                    float farPlane, uchar4* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float rangeScale = 1 / (farPlane - nearPlane);
  const float d = depth[p];
  if (d < nearPlane) out[p] = make_uchar4(255, 255, 255, 0);
  else if (d > farPlane) out[p] = make_uchar4(0, 0, 0, 0);
  else out[p] = gs2rgb((d - nearPlane) * rangeScale);
}

// renderIntensityKernel, rendering.cpp:648-664.
__global__ void render_intensity_kernel(const float* __restrict__ grey, int n,
                                        uchar4* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float gs = 255.f * grey[p];
  out[p] = u4(gs, gs, gs, 255.f);
}

// renderNormalKernel, rendering.cpp:346-364 (uchar3 output).
__global__ void render_normal_kernel(const F3* __restrict__ normal, int n,
                                     unsigned char* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  F3 v = normal[p];
  unsigned char r = 0, g = 0, b = 0;
  if (v.x != -2) {
    v = normalize(v);
    r = to_u8(v.x * 128 + 128);
    g = to_u8(v.y * 128 + 128);
    b = to_u8(v.z * 128 + 128);
  }
  out[3 * p] = r; out[3 * p + 1] = g; out[3 * p + 2] = b;
}

// mode 0: renderTrackKernel (rendering.cpp:395-432) on the ICP rows;
// mode 1: renderRGBTrackKernel (:434-487) on the photometric rows;
// mode 2: render_RGBD_TrackKernel (:183-237) on both.
__global__ void render_track_kernel(const int8_t* __restrict__ res, const float* __restrict__ err,
                                    int n, int mode, uchar4* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  uchar4 c;
  if (mode == 0) {
    switch (res[p]) {
      case 1: c = make_uchar4(128, 128, 128, 0); break;
      case -1: c = make_uchar4(0, 0, 0, 0); break;
      case -2: c = make_uchar4(255, 0, 0, 0); break;
      case -3: c = make_uchar4(0, 255, 0, 0); break;
      case -4: c = make_uchar4(0, 0, 255, 0); break;
      case -5: c = make_uchar4(255, 255, 0, 0); break;
      case -6: c = make_uchar4(255, 175, 175, 0); break;
      default: c = make_uchar4(255, 200, 128, 0); break;
    }
  } else if (mode == 1) {
    const int r = res[n + p];
    switch (r) {
      case 1: {
        const float e = fabsf((float)((double)err[n + p] * 255.0));
        c = u4(e, e, e, 255.f);
        break;
      }
      case -1: c = make_uchar4(0, 255, 0, 0); break;
      case -2: c = make_uchar4(0, 0, 0, 0); break;
      case -3: c = make_uchar4(255, 0, 0, 0); break;
      case -4: c = make_uchar4(0, 0, 255, 0); break;
      case -5: c = make_uchar4(255, 255, 0, 0); break;
      default: c = make_uchar4(255, 128, 128, 0); break;
    }
  } else {
    const int ri = res[p], rr = res[n + p];
    if (ri == 1 && rr == 1) {
      const float e = (float)fabs((double)err[n + p] * 255.0);
      c = u4(e, e, e, 255.f);
    } else if ((ri < -3 && ri > -6) || (rr < -3 && rr > -6)) {
      c = make_uchar4(255, 0, 0, 0);
    } else if (ri == -2 || rr == -2 || ri == -3 || rr == -3) {
      c = make_uchar4(255, 255, 0, 0);
    } else if (ri == -1 || rr == -1) {
      c = make_uchar4(0, 255, 0, 0);
    } else if (ri == -6 || rr == -6) {
      c = make_uchar4(255, 175, 175, 0);
    } else {
      c = make_uchar4(128, 128, 128, 0);
    }
  }
  out[p] = c;
}

struct MaskArgs {
  const int* label;
  const F3* rgb;             // input colour in [0, 1]
  const uchar4* colors;
  int n_colors;
  const int8_t* const* rows;  // per label: result rows (ICP, photometric), may be null
  int n_rows;
  int n, mode;
  uchar4* out;
};

// mode 0: renderInstanceMaskKernel (rendering.cpp:797-820; renderClassMaskKernel
// :822-847 is the same with the colours indexed by class);
// mode 1: renderMaskWithImageKernel (:679-723);
// mode 2: renderMaskMotionWithImageKernel (:725-795).
__global__ void render_mask_kernel(MaskArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  const int id = a.label[p];
  const uchar4 lc = (id >= 0 && id < a.n_colors) ? a.colors[id] : make_uchar4(0, 0, 0, 0);
  if (a.mode == 0) {
    a.out[p] = lc;
    return;
  }
  const float alpha = 0.3f;
  const F3 c = a.rgb[p];
  const F3 rgb = mk3(c.x * 255.f, c.y * 255.f, c.z * 255.f);
  float r, g, b;
  if (a.mode == 1) {
    if (id == -2) {
      r = rgb.x * alpha + 128 * (1 - alpha);
      g = rgb.y * alpha + 128 * (1 - alpha);
      b = rgb.z * 0 + 255 * (1);
    } else if (id != 0) {
      r = rgb.x * alpha + lc.x * (1 - alpha);
      g = rgb.y * alpha + lc.y * (1 - alpha);
      b = rgb.z * alpha + lc.z * (1 - alpha);
    } else {
      r = rgb.x; g = rgb.y; b = rgb.z;
    }
  } else {
    const int8_t* rows = (id >= 0 && id < a.n_rows) ? a.rows[id] : nullptr;
    const bool outlier = rows && (rows[p] < -3 || rows[a.n + p] < -3);
    if (id == -2) {
      r = rgb.x * alpha + 255 * (1 - alpha);
      g = rgb.y * alpha + 175 * (1 - alpha);
      b = rgb.z * alpha + 175 * (1 - alpha);
    } else if (id == 0) {
      if (outlier) {
        r = rgb.x * alpha + 255 * (1 - alpha);
        g = rgb.y * alpha + 0 * (1 - alpha);
        b = rgb.z * alpha + 0 * (1 - alpha);
      } else {
        r = rgb.x; g = rgb.y; b = rgb.z;
      }
    } else if (outlier) {
      r = rgb.x; g = rgb.y; b = rgb.z;
    } else {
      r = rgb.x * alpha + lc.x * (1 - alpha);
      g = rgb.y * alpha + lc.y * (1 - alpha);
      b = rgb.z * alpha + lc.z * (1 - alpha);
    }
  }
  a.out[p] = u4(r, g, b, 0.f);
}

// ------------------------------------------------------------------ host side
// Renders go straight into device memory; a host destination is served from a
// context scratch image and a synchronous copy.
int render_target(Context* ctx, void* out, size_t bytes, void** target) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, out) == cudaSuccess &&
      (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged)) {
    *target = out;
    return MF_OK;
  }
  cudaGetLastError();  // an unregistered host pointer is not an error here
  if (!ctx->d_render) {
    MF_CUDA(cudaMalloc(&ctx->d_render, (size_t)ctx->W * ctx->H * 4));
  }
  if (bytes > (size_t)ctx->W * ctx->H * 4) {
    ctx->last_error = "render: image larger than the frame";
    return MF_E_ARG;
  }
  *target = ctx->d_render;
  return MF_OK;
}

int render_finish(Context* ctx, void* out, void* target, size_t bytes) {
  MF_CUDA(cudaGetLastError());
  if (target != out) {
    MF_CUDA(cudaMemcpyAsync(out, target, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    MF_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return MF_OK;
}

// A small colour table or pointer table staged to the device (render scratch
// tail), ordered on the context stream.
int render_stage_small(Context* ctx, const void* src, size_t bytes, void** dst) {
  if (ctx->render_small_bytes < bytes) {
    if (ctx->d_render_small) cudaFree(ctx->d_render_small);
    ctx->d_render_small = nullptr;
    ctx->render_small_bytes = 0;
    MF_CUDA(cudaMalloc(&ctx->d_render_small, bytes));
    ctx->render_small_bytes = bytes;
  }
  MF_CUDA(cudaMemcpyAsync(ctx->d_render_small, src, bytes, cudaMemcpyHostToDevice,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  *dst = ctx->d_render_small;
  return MF_OK;
}

int render_image(Context* ctx, int which, uint8_t* out) {
  const int n = ctx->W * ctx->H;
  const size_t bytes = (size_t)n * (which == 2 ? 3 : 4);
  void* target = nullptr;
  if (int rc = render_target(ctx, out, bytes, &target)) return rc;
  const mf_config& c = ctx->cfg;
  switch (which) {
    case 0:
      render_depth_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(
          ctx->d_depth, n, c.near_plane, c.far_plane, (uchar4*)target);
      break;
    case 1:
      render_intensity_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(ctx->d_grey, n,
                                                                         (uchar4*)target);
      break;
    default:
      render_normal_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(ctx->d_normal, n,
                                                                      (unsigned char*)target);
      break;
  }
  return render_finish(ctx, out, target, bytes);
}

int render_track(Context* ctx, int mode, const int8_t* d_res, const float* d_err, uint8_t* out) {
  const int n = ctx->W * ctx->H;
  const size_t bytes = (size_t)n * 4;
  void* target = nullptr;
  if (int rc = render_target(ctx, out, bytes, &target)) return rc;
  render_track_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(d_res, d_err, n, mode,
                                                                 (uchar4*)target);
  return render_finish(ctx, out, target, bytes);
}

int render_mask(Context* ctx, int mode, const int32_t* d_labels, const uint8_t* colors,
                int n_colors, const int8_t* const* d_rows, int n_rows, uint8_t* out) {
  const int n = ctx->W * ctx->H;
  const size_t bytes = (size_t)n * 4;
  void* target = nullptr;
  if (int rc = render_target(ctx, out, bytes, &target)) return rc;
  // one staging buffer: colours, then the row pointers (8-byte aligned)
  const size_t cbytes = (4 * (size_t)n_colors + 7) / 8 * 8;
  const size_t pbytes = sizeof(void*) * (size_t)n_rows;
  std::vector<unsigned char> host(cbytes + pbytes + 8);
  if (n_colors > 0) std::memcpy(host.data(), colors, 4 * (size_t)n_colors);
  if (n_rows > 0) std::memcpy(host.data() + cbytes, d_rows, pbytes);
  void* d = nullptr;
  if (int rc = render_stage_small(ctx, host.data(), host.size(), &d)) return rc;
  MaskArgs a;
  a.label = d_labels ? d_labels : ctx->d_label;
  a.rgb = ctx->d_rgb;
  a.colors = (const uchar4*)d;
  a.n_colors = n_colors;
  a.rows = n_rows > 0 ? (const int8_t* const*)((unsigned char*)d + cbytes) : nullptr;
  a.n_rows = n_rows;
  a.n = n;
  a.mode = mode;
  a.out = (uchar4*)target;
  render_mask_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(a);
  return render_finish(ctx, out, target, bytes);
}

}  // namespace mf

// C ABI of the MID-Fusion B200 library (declared in include/midfusion_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "mf_internal.h"

using namespace mf;

struct mf_context : public mf::Context {};

namespace mf {

// rgb2intensity, apps/kfusion/src/cpp/preprocessing/preprocessing.cpp:73-102
// (ratio 1): float RGB in [0, 1] and grey = rgb2gs (commons.h:150-154).
__global__ void rgb_convert_kernel(const uint8_t* __restrict__ rgb8, F3* __restrict__ rgb,
                                   float* __restrict__ grey, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float r = rgb8[3 * p], g = rgb8[3 * p + 1], b = rgb8[3 * p + 2];
  rgb[p] = mk3(r / 255.0f, g / 255.0f, b / 255.0f);
  grey[p] = (0.299f * r + 0.587f * g + 0.114f * b) / 255.f;
}

// instance_seg::generalize_label for ground-truth masks,
// apps/kfusion/src/cpp/segmentation/segmentation.cpp:10-48: 1 on the instance,
// 0 on the ring added by a 5x5 elliptic dilation, -1 elsewhere.
__global__ void generalize_kernel(const uint16_t* __restrict__ labels, int W, int H,
                                  const int* __restrict__ inst_labels, int n_inst,
                                  float* __restrict__ masks) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int i = blockIdx.z;
  if (x >= W || i >= n_inst) return;
  const int L = inst_labels[i];
  float v;
  if (labels[x + y * W] == L) {
    v = 1.f;
  } else {
    bool ring = false;
    for (int dy = -2; dy <= 2 && !ring; ++dy)
      for (int dx = -2; dx <= 2; ++dx) {
        if ((dy == -2 || dy == 2) && dx != 0) continue;  // cv::MORPH_ELLIPSE 5x5
        const int xx = x + dx, yy = y + dy;
        if (xx < 0 || yy < 0 || xx >= W || yy >= H) continue;
        if (labels[xx + yy * W] == L) { ring = true; break; }
      }
    v = ring ? 0.f : -1.f;
  }
  masks[(size_t)i * W * H + x + y * W] = v;
}

__global__ void fill_kernel(float* __restrict__ p, float v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

int launch_generalize(Context* ctx) {
  const int n = (int)ctx->inst.size();
  if (n == 0) return MF_OK;
  dim3 grid((ctx->W + 127) / 128, ctx->H, n);
  generalize_kernel<<<grid, 128, 0, ctx->stream>>>(ctx->d_labels, ctx->W, ctx->H,
                                                   ctx->d_inst_label, n, ctx->d_masks);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

}  // namespace mf

static int check(mf_context* ctx) { return ctx ? MF_OK : MF_E_ARG; }

static IdList all_ids(mf_context* ctx) {
  IdList l;
  l.n = (int)ctx->inst.size();
  for (int i = 0; i < l.n; ++i) l.v[i] = i;
  return l;
}

extern "C" {

int mf_config_default(mf_config* c, int width, int height) {
  if (!c || width <= 0 || height <= 0) return MF_E_ARG;
  std::memset(c, 0, sizeof(*c));
  c->width = width;
  c->height = height;
  c->k[0] = 525.f * width / 640.f;
  c->k[1] = 525.f * width / 640.f;
  c->k[2] = (width - 1) * 0.5f;
  c->k[3] = (height - 1) * 0.5f;
  c->mu = 0.1f;
  c->near_plane = 0.1f;
  c->far_plane = 4.0f;
  c->max_weight = 100;
  c->pyramid_levels = 3;
  c->gn_iterations[0] = 10; c->gn_iterations[1] = 5; c->gn_iterations[2] = 4;
  c->robust_kernel = MF_ROBUST_CAUCHY;
  c->use_icp = 1;
  c->use_rgb = 1;
  c->pool_blocks = 1 << 17;
  c->max_instances = 16;
  c->batched = 1;
  return MF_OK;
}

const char* mf_last_error(const mf_context* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

int mf_create(const mf_config* cfg, mf_context** out) {
  if (!cfg || !out || cfg->width <= 0 || cfg->height <= 0 || cfg->pool_blocks <= 0 ||
      cfg->max_instances <= 0 || cfg->max_instances > MAX_INSTANCES ||
      cfg->pool_blocks > (1LL << 30))
    return MF_E_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MF_E_CUDA;
  mf_context* ctx = new mf_context;
  ctx->cfg = *cfg;
  ctx->W = cfg->width;
  ctx->H = cfg->height;
  cudaGetDevice(&ctx->device);
  auto fail = [&](int rc) { mf_destroy(ctx); return rc; };
  // the main stream at the highest priority, the side stream of the overlapped
  // background integration at the lowest: pending CTAs of the frame's
  // critical path (tracking) are dispatched first
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_high) != cudaSuccess)
    return fail(MF_E_CUDA);
  ctx->own_stream = true;
  if (cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_start, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_pre, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_obj, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_gen, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return fail(MF_E_CUDA);
  const size_t WH = (size_t)ctx->W * ctx->H;
  const size_t cap = (size_t)cfg->pool_blocks;
  Pool& P = ctx->pool;
  P.cap = (int)cap;
  const size_t nv = cap * 512;
  bool ok = cudaMalloc(&P.tsdf, nv * 4) == cudaSuccess && cudaMalloc(&P.wt, nv * 4) == cudaSuccess &&
            cudaMalloc(&P.r, nv * 4) == cudaSuccess && cudaMalloc(&P.g, nv * 4) == cudaSuccess &&
            cudaMalloc(&P.b, nv * 4) == cudaSuccess && cudaMalloc(&P.c, nv * 4) == cudaSuccess &&
            cudaMalloc(&P.fg, nv * 8) == cudaSuccess && cudaMalloc(&P.w, nv * 4) == cudaSuccess &&
            cudaMalloc(&P.meta, cap * sizeof(int4)) == cudaSuccess &&
            cudaMalloc(&P.active, cap) == cudaSuccess && cudaMalloc(&P.count, sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&ctx->d_vols, sizeof(Volume) * MAX_INSTANCES) == cudaSuccess &&
       cudaMalloc(&ctx->d_Two, sizeof(float) * 16 * MAX_INSTANCES) == cudaSuccess &&
       cudaMalloc(&ctx->d_Twc, sizeof(float) * 16) == cudaSuccess &&
       cudaMalloc(&ctx->d_frames, sizeof(InstFrame) * MAX_INSTANCES) == cudaSuccess &&
       cudaMalloc(&ctx->d_status, sizeof(int)) == cudaSuccess &&
       cudaMalloc(&ctx->d_reserved, sizeof(unsigned long long) * MAX_INSTANCES) == cudaSuccess &&
       cudaMalloc(&ctx->d_inst_label, sizeof(int) * MAX_INSTANCES) == cudaSuccess &&
       cudaMalloc(&ctx->d_visit, sizeof(int) * cap) == cudaSuccess &&
       cudaMalloc(&ctx->d_visit_count, sizeof(int)) == cudaSuccess &&
       cudaMalloc(&ctx->d_visit_side, sizeof(int) * cap) == cudaSuccess &&
       cudaMalloc(&ctx->d_visit_count_side, sizeof(int)) == cudaSuccess &&
       cudaMalloc(&ctx->d_depth, 4 * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_rgb8, 3 * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_rgb, sizeof(F3) * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_grey, 4 * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_masks, 4 * WH * cfg->max_instances) == cudaSuccess &&
       cudaMalloc(&ctx->d_labels, 2 * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_vertex, sizeof(F3) * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_normal, sizeof(F3) * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_label, sizeof(int) * WH) == cudaSuccess &&
       cudaMalloc(&ctx->d_rayhit, sizeof(F4) * WH * cfg->max_instances) == cudaSuccess &&
       cudaMalloc(&ctx->d_raytf, sizeof(float2) * WH * cfg->max_instances) == cudaSuccess;
  if (!ok) {
    ctx->last_error = "device allocation failed";
    return fail(MF_E_CUDA);
  }
  // Fresh pool slots hold the reference's initial voxel {1, 0, 0, 0, 0, 0, 0, 0}
  // (voxel_traits<SDF>::initValue, continuous/volume_traits.hpp:40); blocks are
  // never released, so a newly acquired slot needs no further initialisation.
  fill_kernel<<<1184, 256, 0, ctx->stream>>>(P.tsdf, 1.f, nv);
  cudaMemsetAsync(P.wt, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.r, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.g, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.b, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.c, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.fg, 0, nv * 8, ctx->stream);
  cudaMemsetAsync(P.w, 0, nv * 4, ctx->stream);
  cudaMemsetAsync(P.active, 0, cap, ctx->stream);
  cudaMemsetAsync(P.count, 0, sizeof(int), ctx->stream);
  cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
  cudaMemsetAsync(ctx->d_vertex, 0, sizeof(F3) * WH, ctx->stream);
  cudaMemsetAsync(ctx->d_normal, 0, sizeof(F3) * WH, ctx->stream);
  cudaMemsetAsync(ctx->d_label, 0, sizeof(int) * WH, ctx->stream);
  cudaMemsetAsync(ctx->d_depth, 0, 4 * WH, ctx->stream);
  cudaMemsetAsync(ctx->d_masks, 0, 4 * WH * cfg->max_instances, ctx->stream);
  float I[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  cudaMemcpyAsync(ctx->d_Twc, I, sizeof(I), cudaMemcpyHostToDevice, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    ctx->last_error = "device initialisation failed";
    return fail(MF_E_CUDA);
  }
  *out = ctx;
  return MF_OK;
}

int mf_destroy(mf_context* ctx) {
  if (!ctx) return MF_E_ARG;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->upload) cudaStreamSynchronize(ctx->upload);
  for (int s = 0; s < 2; ++s) {
    if (ctx->stg_depth[s]) cudaFree(ctx->stg_depth[s]);
    if (ctx->stg_rgb8[s]) cudaFree(ctx->stg_rgb8[s]);
    if (ctx->stg_labels[s]) cudaFree(ctx->stg_labels[s]);
    if (ctx->ev_staged[s]) cudaEventDestroy(ctx->ev_staged[s]);
    if (ctx->ev_consumed[s]) cudaEventDestroy(ctx->ev_consumed[s]);
  }
  if (ctx->upload) cudaStreamDestroy(ctx->upload);
  pipeline_free(ctx);
  track_free(ctx);
  for (auto& in : ctx->inst) volume_free(in);
  Pool& P = ctx->pool;
  void* ps[] = {P.tsdf, P.wt, P.r, P.g, P.b, P.c, P.fg, P.w, P.meta, P.active, P.count,
                ctx->d_vols, ctx->d_Two, ctx->d_Twc, ctx->d_frames, ctx->d_status,
                ctx->d_reserved, ctx->d_inst_label, ctx->d_visit, ctx->d_visit_count,
                ctx->d_visit_side, ctx->d_visit_count_side, ctx->d_depth, ctx->d_rgb8, ctx->d_rgb, ctx->d_grey, ctx->d_masks,
                ctx->d_labels, ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->d_export,
                ctx->d_render, ctx->d_render_small, ctx->d_rayhit, ctx->d_raytf,
                ctx->d_mc_tris};
  for (void* p : ps) if (p) cudaFree(p);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_pre) cudaEventDestroy(ctx->ev_pre);
  if (ctx->ev_obj) cudaEventDestroy(ctx->ev_obj);
  if (ctx->ev_gen) cudaEventDestroy(ctx->ev_gen);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  delete ctx;
  return MF_OK;
}

int mf_status(mf_context* ctx, int* flags) {
  if (check(ctx) || !flags) return MF_E_ARG;
  int v = 0;
  MF_CUDA(cudaMemcpyAsync(&v, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  *flags = v;
  return MF_OK;
}

int mf_get_stream(mf_context* ctx, void** stream) {
  if (check(ctx) || !stream) return MF_E_ARG;
  *stream = (void*)ctx->stream;
  return MF_OK;
}

int mf_synchronize(mf_context* ctx) {
  if (check(ctx)) return MF_E_ARG;
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_instance_add(mf_context* ctx, int size, float dim, const float T_w_o[16], int label,
                    int* id) {
  if (check(ctx) || !T_w_o || !(dim > 0)) return MF_E_ARG;
  if ((int)ctx->inst.size() >= ctx->cfg.max_instances) return MF_E_ARG;
  if (size < 16 || size > 4096 || (size & (size - 1))) return MF_E_ARG;
  Instance in;
  in.size = size;
  in.dim = dim;
  in.label = label;
  // Object::integrate_volume_kernel, object.cpp:132-140: the allocation list holds
  // (dim / (8 * voxelsize)) * W * H keys.
  const float voxelsize = dim / (unsigned)size;
  const int num_vox_per_pix = (int)(dim / (8u * voxelsize));
  in.reserved = (size_t)num_vox_per_pix * ctx->W * ctx->H;
  if (int rc = volume_create(ctx, in)) return rc;
  const int i = (int)ctx->inst.size();
  ctx->inst.push_back(in);
  const unsigned long long res = in.reserved;
  MF_CUDA(cudaMemcpyAsync(ctx->d_vols + i, &ctx->inst[i].vol, sizeof(Volume),
                          cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(ctx->d_Two + 16 * i, T_w_o, 64, cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(ctx->d_reserved + i, &res, sizeof(res), cudaMemcpyHostToDevice,
                          ctx->stream));
  MF_CUDA(cudaMemcpyAsync(ctx->d_inst_label + i, &label, sizeof(int), cudaMemcpyHostToDevice,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->inst.size() == 1) {
    // lib/octree.hpp:934 keeps the ray direction epsilon in a function-local
    // static, initialised by the first ray iterator: the first volume's size.
    ctx->ray_epsilon = exp2f((float)(-std::log2((double)size)));
  }
  if (id) *id = i;
  return MF_OK;
}

int mf_instance_count(mf_context* ctx, int* n) {
  if (check(ctx) || !n) return MF_E_ARG;
  *n = (int)ctx->inst.size();
  return MF_OK;
}

int mf_instance_set_pose(mf_context* ctx, int id, const float T[16]) {
  if (check(ctx) || !T) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  MF_CUDA(cudaMemcpyAsync(ctx->d_Two + 16 * id, T, 64, cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_instance_get_pose(mf_context* ctx, int id, float T[16]) {
  if (check(ctx) || !T) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  MF_CUDA(cudaMemcpyAsync(T, ctx->d_Two + 16 * id, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_set_camera_pose(mf_context* ctx, const float T[16]) {
  if (check(ctx) || !T) return MF_E_ARG;
  if (int rc = track_init(ctx)) return rc;
  track_save_prev_camera(ctx);  // the replaced pose becomes T_w_c1 for object tracking
  MF_CUDA(cudaMemcpyAsync(ctx->d_Twc, T, 64, cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_get_camera_pose(mf_context* ctx, float T[16]) {
  if (check(ctx) || !T) return MF_E_ARG;
  MF_CUDA(cudaMemcpyAsync(T, ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_frame_upload(mf_context* ctx, const float* depth, const uint8_t* rgb,
                    const float* masks, int n_masks) {
  if (check(ctx)) return MF_E_ARG;
  if (n_masks < 0 || n_masks > ctx->cfg.max_instances || (masks && n_masks == 0)) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (depth)
    MF_CUDA(cudaMemcpyAsync(ctx->d_depth, depth, 4 * WH, cudaMemcpyHostToDevice, ctx->stream));
  if (rgb) {
    MF_CUDA(cudaMemcpyAsync(ctx->d_rgb8, rgb, 3 * WH, cudaMemcpyHostToDevice, ctx->stream));
    rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
        ctx->d_rgb8, ctx->d_rgb, ctx->d_grey, (int)WH);
    MF_CUDA(cudaGetLastError());
  }
  if (masks)
    MF_CUDA(cudaMemcpyAsync(ctx->d_masks, masks, 4 * WH * n_masks, cudaMemcpyHostToDevice,
                            ctx->stream));
  // the host buffers are borrowed only for the call
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_frame_set_device(mf_context* ctx, const float* d_depth, const uint8_t* d_rgb,
                        const float* d_masks, int n_masks) {
  if (check(ctx)) return MF_E_ARG;
  if (n_masks < 0 || n_masks > ctx->cfg.max_instances) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (d_depth)
    MF_CUDA(cudaMemcpyAsync(ctx->d_depth, d_depth, 4 * WH, cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_rgb) {
    rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
        d_rgb, ctx->d_rgb, ctx->d_grey, (int)WH);
    MF_CUDA(cudaGetLastError());
  }
  if (d_masks)
    MF_CUDA(cudaMemcpyAsync(ctx->d_masks, d_masks, 4 * WH * n_masks, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  return MF_OK;
}

int mf_frame_labels(mf_context* ctx, const uint16_t* labels) {
  if (check(ctx) || !labels) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaMemcpyAsync(ctx->d_labels, labels, 2 * WH, cudaMemcpyHostToDevice, ctx->stream));
  if (int rc = launch_generalize(ctx)) return rc;
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_integrate(mf_context* ctx, const int* ids, int n) {
  if (check(ctx) || n < 0 || (n > 0 && !ids)) return MF_E_ARG;
  for (int i = 0; i < n; ++i)
    if (ids[i] < 0 || ids[i] >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  if (ctx->cfg.batched) {
    IdList l;
    l.n = n;
    for (int i = 0; i < n; ++i) l.v[i] = ids[i];
    if (int rc = stage_prepare(ctx, l)) return rc;
    if (int rc = stage_alloc(ctx, l)) return rc;
    if (int rc = stage_integrate(ctx, l)) return rc;
  } else {
    for (int i = 0; i < n; ++i) {  // one instance per launch, like the reference's loop
      IdList l;
      l.n = 1;
      l.v[0] = ids[i];
      if (int rc = stage_prepare(ctx, l)) return rc;
      if (int rc = stage_alloc(ctx, l)) return rc;
      if (int rc = stage_integrate(ctx, l)) return rc;
    }
  }
  return MF_OK;
}

int mf_alloc_update(mf_context* ctx, int id, const uint64_t* keys, int n) {
  if (check(ctx) || n < 0 || (n > 0 && !keys)) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  uint64_t zero = 0;
  return alloc_keys(ctx, id, n > 0 ? keys : &zero, n);
}

int mf_raycast(mf_context* ctx) {
  if (check(ctx)) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  const IdList l = all_ids(ctx);
  if (int rc = stage_prepare(ctx, l)) return rc;
  return stage_raycast(ctx, l, ctx->ray_epsilon);
}

int mf_raycast_records(mf_context* ctx, const int* ids, int n, mf_ray_record* d_records,
                       mf_ray_origin* d_origins) {
  if (check(ctx) || !ids || n <= 0 || n > MAX_INSTANCES || !d_records || !d_origins)
    return MF_E_ARG;
  IdList l;
  l.n = n;
  for (int k = 0; k < n; ++k) {
    if (ids[k] < 0 || ids[k] >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
    l.v[k] = ids[k];
  }
  return raycast_records(ctx, l, d_records, d_origins);
}

int mf_raycast_fold(mf_context* ctx, const mf_ray_record* d_records,
                    const mf_ray_origin* d_origins) {
  if (check(ctx) || !d_records || !d_origins) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return raycast_fold(ctx, d_records, d_origins);
}

int mf_download_raycast(mf_context* ctx, float* vertex, float* normal, int32_t* label) {
  if (check(ctx)) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (vertex)
    MF_CUDA(cudaMemcpyAsync(vertex, ctx->d_vertex, 12 * WH, cudaMemcpyDeviceToHost, ctx->stream));
  if (normal)
    MF_CUDA(cudaMemcpyAsync(normal, ctx->d_normal, 12 * WH, cudaMemcpyDeviceToHost, ctx->stream));
  if (label)
    MF_CUDA(cudaMemcpyAsync(label, ctx->d_label, 4 * WH, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_block_count(mf_context* ctx, int id, int* n) {
  if (check(ctx) || !n) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return export_blocks(ctx, id, nullptr, nullptr, nullptr, nullptr, 0, n);
}

int mf_export_blocks(mf_context* ctx, int id, uint64_t* keys, int32_t* coords, uint8_t* active,
                     void* voxels, int cap, int* n) {
  if (check(ctx)) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return export_blocks(ctx, id, keys, coords, active, voxels, cap, n);
}

int mf_node_count(mf_context* ctx, int id, int* n) {
  if (check(ctx) || !n) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return export_nodes(ctx, id, nullptr, nullptr, nullptr, nullptr, 0, n);
}

int mf_export_nodes(mf_context* ctx, int id, uint64_t* keys, uint32_t* side,
                    uint8_t* children_mask, void* values, int cap, int* n) {
  if (check(ctx)) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return export_nodes(ctx, id, keys, side, children_mask, values, cap, n);
}

int mf_root_children(mf_context* ctx, int id, uint8_t* mask) {
  if (check(ctx) || !mask) return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return root_children(ctx, id, mask);
}

int mf_interp(mf_context* ctx, int id, const float* pos, int n, int field, float* out) {
  if (check(ctx) || n < 0 || (n > 0 && (!pos || !out)) || field < 0 || field > 4)
    return MF_E_ARG;
  if (id < 0 || id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return interp_points(ctx, id, pos, n, field, out);
}

int mf_process_frame(mf_context* ctx, const float* depth, const uint8_t* rgb,
                     const uint16_t* labels) {
  if (check(ctx) || !depth || !rgb) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaMemcpyAsync(ctx->d_depth, depth, 4 * WH, cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(ctx->d_rgb8, rgb, 3 * WH, cudaMemcpyHostToDevice, ctx->stream));
  rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->d_rgb8, ctx->d_rgb, ctx->d_grey, (int)WH);
  MF_CUDA(cudaGetLastError());
  if (labels)
    MF_CUDA(cudaMemcpyAsync(ctx->d_labels, labels, 2 * WH, cudaMemcpyHostToDevice, ctx->stream));
  return process_frame(ctx, labels != nullptr);
}

int mf_process_frame_motion(mf_context* ctx, const float* depth, const uint8_t* rgb,
                            const uint16_t* labels, float residual_threshold,
                            float moved_threshold, uint32_t* moving_labels) {
  if (check(ctx) || !depth || !rgb || !labels || !moving_labels || !(residual_threshold > 0))
    return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaMemcpyAsync(ctx->d_depth, depth, 4 * WH, cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(ctx->d_rgb8, rgb, 3 * WH, cudaMemcpyHostToDevice, ctx->stream));
  rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->d_rgb8, ctx->d_rgb, ctx->d_grey, (int)WH);
  MF_CUDA(cudaGetLastError());
  MF_CUDA(cudaMemcpyAsync(ctx->d_labels, labels, 2 * WH, cudaMemcpyHostToDevice, ctx->stream));
  return process_frame_motion(ctx, residual_threshold, moved_threshold, moving_labels);
}

int mf_process_frame_device(mf_context* ctx, const float* d_depth, const uint8_t* d_rgb,
                            const uint16_t* d_labels) {
  if (check(ctx) || !d_depth || !d_rgb) return MF_E_ARG;
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaMemcpyAsync(ctx->d_depth, d_depth, 4 * WH, cudaMemcpyDeviceToDevice, ctx->stream));
  rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
      d_rgb, ctx->d_rgb, ctx->d_grey, (int)WH);
  MF_CUDA(cudaGetLastError());
  if (d_labels)
    MF_CUDA(cudaMemcpyAsync(ctx->d_labels, d_labels, 2 * WH, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  return process_frame(ctx, d_labels != nullptr);
}

// The upload stream, the two input slots and their events, on first use.  A
// call that failed part way leaves what it made (mf_destroy frees it) and the
// next call makes the rest; ev_consumed[1], made last, marks the set whole.
static int staging_init(Context* ctx) {
  if (ctx->ev_consumed[1]) return MF_OK;
  const size_t WH = (size_t)ctx->W * ctx->H;
  if (!ctx->upload) MF_CUDA(cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking));
  for (int s = 0; s < 2; ++s) {
    if (!ctx->stg_depth[s]) MF_CUDA(cudaMalloc(&ctx->stg_depth[s], 4 * WH));
    if (!ctx->stg_rgb8[s]) MF_CUDA(cudaMalloc(&ctx->stg_rgb8[s], 3 * WH));
    if (!ctx->stg_labels[s]) MF_CUDA(cudaMalloc(&ctx->stg_labels[s], 2 * WH));
    if (!ctx->ev_staged[s])
      MF_CUDA(cudaEventCreateWithFlags(&ctx->ev_staged[s], cudaEventDisableTiming));
    if (!ctx->ev_consumed[s])
      MF_CUDA(cudaEventCreateWithFlags(&ctx->ev_consumed[s], cudaEventDisableTiming));
  }
  return MF_OK;
}

int mf_frame_stage(mf_context* ctx, int slot, const float* depth, const uint8_t* rgb,
                   const uint16_t* labels) {
  if (check(ctx) || slot < 0 || slot > 1 || !depth || !rgb) return MF_E_ARG;
  if (ctx->stg_pending[slot]) {
    ctx->last_error = "mf_frame_stage: slot " + std::to_string(slot) +
                      " holds a frame that mf_process_staged has not taken yet";
    return MF_E_STATE;
  }
  if (int rc = staging_init(ctx)) return rc;
  const size_t WH = (size_t)ctx->W * ctx->H;
  // the frame last processed from this slot has copied it out (an event never
  // recorded is complete)
  MF_CUDA(cudaStreamWaitEvent(ctx->upload, ctx->ev_consumed[slot], 0));
  MF_CUDA(cudaMemcpyAsync(ctx->stg_depth[slot], depth, 4 * WH, cudaMemcpyHostToDevice,
                          ctx->upload));
  MF_CUDA(cudaMemcpyAsync(ctx->stg_rgb8[slot], rgb, 3 * WH, cudaMemcpyHostToDevice, ctx->upload));
  if (labels)
    MF_CUDA(cudaMemcpyAsync(ctx->stg_labels[slot], labels, 2 * WH, cudaMemcpyHostToDevice,
                            ctx->upload));
  MF_CUDA(cudaEventRecord(ctx->ev_staged[slot], ctx->upload));
  ctx->stg_labels_set[slot] = labels != nullptr;
  ctx->stg_pending[slot] = true;
  return MF_OK;
}

int mf_process_staged(mf_context* ctx, int slot) {
  if (check(ctx) || slot < 0 || slot > 1) return MF_E_ARG;
  if (!ctx->stg_pending[slot]) {
    ctx->last_error = "mf_process_staged: nothing staged in slot " + std::to_string(slot);
    return MF_E_STATE;
  }
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_staged[slot], 0));
  MF_CUDA(cudaMemcpyAsync(ctx->d_depth, ctx->stg_depth[slot], 4 * WH, cudaMemcpyDeviceToDevice,
                          ctx->stream));
  rgb_convert_kernel<<<(unsigned)((WH + 255) / 256), 256, 0, ctx->stream>>>(
      ctx->stg_rgb8[slot], ctx->d_rgb, ctx->d_grey, (int)WH);
  MF_CUDA(cudaGetLastError());
  const bool labels = ctx->stg_labels_set[slot];
  if (labels)
    MF_CUDA(cudaMemcpyAsync(ctx->d_labels, ctx->stg_labels[slot], 2 * WH,
                            cudaMemcpyDeviceToDevice, ctx->stream));
  MF_CUDA(cudaEventRecord(ctx->ev_consumed[slot], ctx->stream));
  ctx->stg_pending[slot] = false;
  return process_frame(ctx, labels);
}

int mf_upload_stream(mf_context* ctx, void** stream) {
  if (check(ctx) || !stream) return MF_E_ARG;
  if (int rc = staging_init(ctx)) return rc;
  *stream = (void*)ctx->upload;
  return MF_OK;
}

int mf_get_poses(mf_context* ctx, float* T_w_c, float* T_w_o) {
  if (check(ctx)) return MF_E_ARG;
  if (T_w_c)
    MF_CUDA(cudaMemcpyAsync(T_w_c, ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
  if (T_w_o)
    MF_CUDA(cudaMemcpyAsync(T_w_o, ctx->d_Two, 64 * ctx->inst.size(), cudaMemcpyDeviceToHost,
                            ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_frame_stats(mf_context* ctx, long long* out, int n) {
  if (check(ctx) || !out || n < 2) return MF_E_ARG;
  int pc = 0, vc = 0, vs = 0;
  MF_CUDA(cudaMemcpyAsync(&pc, ctx->pool.count, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(&vc, ctx->d_visit_count, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  if (ctx->visit_side_used)
    MF_CUDA(cudaMemcpyAsync(&vs, ctx->d_visit_count_side, sizeof(int), cudaMemcpyDeviceToHost,
                            ctx->stream));
  std::vector<unsigned long long> em(ctx->inst.size(), 0);
  for (size_t i = 0; i < ctx->inst.size(); ++i)
    MF_CUDA(cudaMemcpyAsync(&em[i], ctx->inst[i].vol.emit_total, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  // the device counter keeps counting requests once the pool is full
  // (MF_STATUS_POOL_FULL reports that): the blocks held are at most cap
  out[0] = std::min(pc, ctx->pool.cap);
  out[1] = vc + vs;  // the last frame's visited blocks (both lists when overlapped)
  for (size_t i = 0; i < ctx->inst.size() && (int)i + 2 < n; ++i) out[2 + i] = (long long)em[i];
  if ((int)ctx->inst.size() + 2 < n) out[2 + ctx->inst.size()] = (long long)graph_kernel_nodes(ctx);
  return MF_OK;
}

int mf_profile(mf_context* ctx, int reps, double* out, int n) {
  if (check(ctx) || !out || n < 6 || reps < 1) return MF_E_ARG;
  if (int rc = profile_gn(ctx, reps, &out[0], &out[1])) return rc;
  if (int rc = profile_integrate(ctx, reps, &out[2], &out[3])) return rc;
  return profile_raycast(ctx, reps, &out[4], &out[5]);
}

int mf_set_graphs(mf_context* ctx, int enable) {
  if (check(ctx)) return MF_E_ARG;
  ctx->use_graphs = enable != 0;
  return MF_OK;
}

int mf_set_gn_persistent(mf_context* ctx, int enable) {
  if (check(ctx)) return MF_E_ARG;
  if (ctx->gn_persistent != (enable != 0)) {
    ctx->gn_persistent = enable != 0;
    ++ctx->tune.gen;  // captured frame graphs are rebuilt
  }
  return MF_OK;
}

int mf_set_overlap(mf_context* ctx, int ctas) {
  if (check(ctx) || ctas > 65535) return MF_E_ARG;
  if (ctas < 0) ctas = -1;
  if (ctx->overlap_ctas != ctas) {
    ctx->overlap_ctas = ctas;
    ++ctx->tune.gen;  // captured frame graphs are rebuilt
  }
  return MF_OK;
}

int mf_tune_candidates(int stage, int* n) {
  if (!n || (stage != MF_TUNE_RAYCAST && stage != MF_TUNE_INTEGRATE)) return MF_E_ARG;
  *n = tune_variant_count(stage);
  return MF_OK;
}

int mf_tune_describe(int stage, int variant, char* buf, int cap) {
  if (!buf || cap < 1 || variant < 0 || variant >= tune_variant_count(stage)) return MF_E_ARG;
  if (stage == MF_TUNE_RAYCAST) ray_variant_describe(variant, buf, cap);
  else int_variant_describe(variant, buf, cap);
  return MF_OK;
}

int mf_autotune(mf_context* ctx, int reps, float* raycast_us, float* integrate_us) {
  if (check(ctx) || reps < 1) return MF_E_ARG;
  float ray[MAX_TUNE_VARIANTS] = {0}, integ[MAX_TUNE_VARIANTS] = {0};
  if (int rc = autotune(ctx, reps, ray, integ)) return rc;
  if (raycast_us) std::memcpy(raycast_us, ray, sizeof(ray));
  if (integrate_us) std::memcpy(integrate_us, integ, sizeof(integ));
  return MF_OK;
}

int mf_tune_get(mf_context* ctx, int stage, int* variant) {
  if (check(ctx) || !variant) return MF_E_ARG;
  if (stage == MF_TUNE_RAYCAST) *variant = ctx->tune.ray;
  else if (stage == MF_TUNE_INTEGRATE) *variant = ctx->tune.integrate;
  else return MF_E_ARG;
  return MF_OK;
}

int mf_tune_set(mf_context* ctx, int stage, int variant) {
  if (check(ctx)) return MF_E_ARG;
  return tune_set(ctx, stage, variant);
}

int mf_preprocess(mf_context* ctx) {
  if (check(ctx)) return MF_E_ARG;
  return track_preprocess(ctx);
}

int mf_set_ref_from_current(mf_context* ctx) {
  if (check(ctx)) return MF_E_ARG;
  return track_set_ref(ctx);
}

int mf_track_camera(mf_context* ctx, uint32_t moving_labels) {
  if (check(ctx)) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return track_camera(ctx, moving_labels);
}

int mf_retrack_camera(mf_context* ctx, uint32_t moving_labels) {
  if (check(ctx)) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return track_camera(ctx, moving_labels, 1);
}

int mf_track_objects(mf_context* ctx, const int* ids, int n) {
  if (check(ctx) || n < 0 || n > 31 || (n > 0 && !ids)) return MF_E_ARG;
  IdList l;
  l.n = n;
  for (int i = 0; i < n; ++i) {
    if (ids[i] <= 0 || ids[i] >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
    l.v[i] = ids[i];
  }
  return track_objects(ctx, l);
}

int mf_track_info(mf_context* ctx, int slot, int* iterations, double* sums, double* pose) {
  if (check(ctx) || slot < 0 || slot >= ctx->cfg.max_instances) return MF_E_ARG;
  const int rc = track_info(ctx, slot, iterations, sums, pose);
  return rc < 0 ? rc : MF_OK;
}

int mf_track_eval(mf_context* ctx, int slot, int level, const float* pose, double* sums) {
  if (check(ctx) || !sums || slot < 0 || slot >= ctx->cfg.max_instances || level < 0 ||
      level >= ctx->cfg.pyramid_levels)
    return MF_E_ARG;
  return track_eval(ctx, slot, level, pose, sums);
}

int mf_track_eval_static(mf_context* ctx, int slot, int level, const float* pose,
                         double* sums) {
  if (check(ctx) || !sums || slot < 0 || slot >= ctx->cfg.max_instances || level < 0 ||
      level >= ctx->cfg.pyramid_levels)
    return MF_E_ARG;
  return track_eval_static(ctx, slot, level, pose, sums);
}

int mf_debug_gn_step(mf_context* ctx, int n, const double* state, const double* sums,
                     double* out_device, double* out_host) {
  if (check(ctx) || n < 0 || n > 65535 || (n > 0 && (!state || !sums || !out_device || !out_host)))
    return MF_E_ARG;
  if (n == 0) return MF_OK;
  return gn_step_check(ctx, n, state, sums, out_device, out_host);
}

int mf_camera_cost(mf_context* ctx, const float* T_live, double* out, float* d_grad_tsdf) {
  if (check(ctx) || !T_live || !out) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return camera_cost(ctx, T_live, d_grad_tsdf ? 1 : 0, out, d_grad_tsdf);
}

int mf_pool_slots(mf_context* ctx, int32_t* meta, long long cap, long long* n) {
  if (check(ctx) || !n || (cap > 0 && !meta)) return MF_E_ARG;
  int used = 0;
  MF_CUDA(cudaMemcpyAsync(&used, ctx->pool.count, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  used = std::min(used, ctx->pool.cap);
  *n = used;
  const long long m = std::min<long long>(used, cap);
  if (m > 0)
    MF_CUDA(cudaMemcpyAsync(meta, ctx->pool.meta, sizeof(int4) * m, cudaMemcpyDeviceToHost,
                            ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_pool_tsdf(mf_context* ctx, float** d_tsdf, long long* n) {
  if (check(ctx) || !d_tsdf || !n) return MF_E_ARG;
  *d_tsdf = ctx->pool.tsdf;
  *n = (long long)ctx->pool.cap * 512;
  return MF_OK;
}

int mf_download_pyramid(mf_context* ctx, int level, int which, float* out) {
  if (check(ctx) || !out || level < 0 || level >= ctx->cfg.pyramid_levels) return MF_E_ARG;
  return track_download_level(ctx, level, which, out);
}

int mf_motion_residuals(mf_context* ctx, float residual_threshold, float moved_threshold,
                        float* inlier_ratio, uint32_t* moving_labels) {
  if (check(ctx) || !(residual_threshold > 0)) return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return motion_residuals(ctx, residual_threshold, moved_threshold, inlier_ratio, moving_labels);
}

int mf_motion_download(mf_context* ctx, int8_t* results, float* errors, float* live_vertex,
                       int32_t* live_label) {
  if (check(ctx)) return MF_E_ARG;
  return motion_download(ctx, results, errors, live_vertex, live_label);
}

int mf_track_results(mf_context* ctx, int id, int8_t* d_results, float* d_errors,
                     float* pose_eval) {
  if (check(ctx) || !d_results || id < 0) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return track_results(ctx, id, d_results, d_errors, pose_eval);
}

int mf_object_residuals(mf_context* ctx, int id, float threshold, int8_t* d_results,
                        float* T_virtual) {
  if (check(ctx) || !d_results || id < 1 || !(threshold > 0)) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  const int rc = object_residuals(ctx, id, threshold, d_results, T_virtual);
  if (rc == MF_OK && T_virtual) MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return rc;
}

int mf_refine_mask_use_motion(mf_context* ctx, int id, const int8_t* d_results) {
  if (check(ctx) || id < 0) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return refine_mask_use_motion(ctx, id, d_results, ctx->cfg.use_icp, ctx->cfg.use_rgb);
}

int mf_download_mask(mf_context* ctx, int id, float* out) {
  if (check(ctx) || !out || id < 0) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  const size_t WH = (size_t)ctx->W * ctx->H;
  MF_CUDA(cudaMemcpyAsync(out, ctx->d_masks + id * WH, 4 * WH, cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mf_render_volume(mf_context* ctx, const float* T_w_c, int render_color, float largestep,
                     const float* ambient, const uint8_t* colors, int n_colors, uint8_t* out) {
  if (check(ctx) || !out || !(largestep > 0) || n_colors < 0 || (n_colors > 0 && !colors))
    return MF_E_ARG;
  if (ctx->inst.empty()) return MF_E_STATE;
  return render_volume(ctx, T_w_c, render_color, largestep, ambient, colors, n_colors, out);
}

int mf_render_depth(mf_context* ctx, uint8_t* out) {
  if (check(ctx) || !out) return MF_E_ARG;
  return render_image(ctx, 0, out);
}

int mf_render_intensity(mf_context* ctx, uint8_t* out) {
  if (check(ctx) || !out) return MF_E_ARG;
  return render_image(ctx, 1, out);
}

int mf_render_normal(mf_context* ctx, uint8_t* out) {
  if (check(ctx) || !out) return MF_E_ARG;
  return render_image(ctx, 2, out);
}

int mf_render_track(mf_context* ctx, int mode, const int8_t* d_results, const float* d_errors,
                    uint8_t* out) {
  if (check(ctx) || !out || mode < 0 || mode > 2) return MF_E_ARG;
  if (!d_results) {
    const int8_t* r = nullptr;
    const float* e = nullptr;
    if (int rc = motion_planes(ctx, &r, &e)) return rc;
    d_results = r;
    d_errors = e;
  }
  if (mode != 0 && !d_errors) return MF_E_ARG;
  return render_track(ctx, mode, d_results, d_errors, out);
}

int mf_render_mask(mf_context* ctx, int mode, const int32_t* d_labels, const uint8_t* colors,
                   int n_colors, const int8_t* const* d_rows, int n_rows, uint8_t* out) {
  if (check(ctx) || !out || mode < 0 || mode > 2 || n_colors < 0 || (n_colors > 0 && !colors) ||
      n_rows < 0 || (n_rows > 0 && !d_rows))
    return MF_E_ARG;
  return render_mask(ctx, mode, d_labels, colors, n_colors, d_rows, n_rows, out);
}

int mf_spawn_object(mf_context* ctx, const uint8_t* mask, float* T_w_o, float* volume_size,
                    int* volume_resol, int* n_pixels) {
  if (check(ctx) || !mask || !T_w_o || !volume_size || !volume_resol) return MF_E_ARG;
  const int n = spawn_object(ctx, mask, T_w_o, volume_size, volume_resol);
  if (n < 0) return n;
  if (n_pixels) *n_pixels = n;
  return MF_OK;
}

int mf_instance_set_semantics(mf_context* ctx, int id, int class_id, const float* probs,
                              int n_classes) {
  if (check(ctx) || id < 0 || n_classes < 0 || (n_classes > 0 && !probs)) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return set_semantics(ctx, id, class_id, probs, n_classes);
}

int mf_fuse_semantics(mf_context* ctx, int id, int class_id, const float* probs, int n_classes,
                      int recog_times) {
  if (check(ctx) || id < 0 || n_classes < 0 || (n_classes > 0 && !probs) || recog_times < 0)
    return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return fuse_semantics(ctx, id, class_id, probs, n_classes, recog_times);
}

int mf_instance_semantics(mf_context* ctx, int id, int* class_id, int* fused_time, float* probs,
                          int cap) {
  if (check(ctx) || id < 0 || cap < 0) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  const Instance& in = ctx->inst[id];
  if (class_id) *class_id = in.class_id;
  if (fused_time) *fused_time = in.fused_time;
  if (probs)
    for (int i = 0; i < cap && i < (int)in.sem.size(); ++i) probs[i] = in.sem[i];
  return MF_OK;
}

int mf_frame_upload_raw(mf_context* ctx, const uint16_t* depth_mm, const uint8_t* rgb,
                        int in_width, int in_height) {
  if (check(ctx) || in_width <= 0 || in_height <= 0) return MF_E_ARG;
  return frame_upload_raw(ctx, depth_mm, rgb, in_width, in_height);
}

int mf_save_poses(mf_context* ctx, const char* prefix, int frame) {
  if (check(ctx) || !prefix) return MF_E_ARG;
  const int n = (int)ctx->inst.size();
  std::vector<float> T(16 * (n + 1));
  MF_CUDA(cudaMemcpyAsync(T.data(), ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
  if (n > 0)
    MF_CUDA(cudaMemcpyAsync(T.data() + 16, ctx->d_Two, 64 * (size_t)n, cudaMemcpyDeviceToHost,
                            ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; ++i) {
    Instance& in = ctx->inst[i];
    const bool cam = in.label == 0;
    const std::string path = std::string(prefix) + (cam ? "_camera" : "_" + std::to_string(in.label));
    FILE* f = std::fopen(path.c_str(), in.pose_saved ? "a" : "w");
    if (!f) {
      ctx->last_error = "mf_save_poses: cannot open " + path;
      return MF_E_NOT_FOUND;
    }
    in.pose_saved = true;
    char line[256];
    // kfusion.cpp:1615-1617 writes the camera's translation on every line,
    // with the instance's own rotation
    const int len = tum_line(frame, T.data(), cam ? T.data() : T.data() + 16 * (i + 1), line,
                             sizeof(line));
    std::fwrite(line, 1, len, f);
    std::fclose(f);
  }
  return MF_OK;
}

int mf_mesh(mf_context* ctx, int id, int float_bounds, float* tris, long long cap,
            long long* n_tris) {
  if (check(ctx) || id < 0 || !n_tris || cap < 0) return MF_E_ARG;
  if (id >= (int)ctx->inst.size()) return MF_E_NOT_FOUND;
  return mesh_volume(ctx, id, float_bounds, tris, cap, n_tris);
}

int mf_mesh_set_triangle_table(mf_context* ctx, const int* table) {
  if (check(ctx)) return MF_E_ARG;
  return mesh_set_table(ctx, table);
}

int mf_write_vtk_mesh(const char* path, const float* tris, long long n) {
  if (!path || n < 0 || (n > 0 && !tris)) return MF_E_ARG;
  return write_vtk_mesh(path, tris, n);
}

int mf_dump_mesh(mf_context* ctx, const char* prefix) {
  if (check(ctx) || !prefix) return MF_E_ARG;
  for (int i = 0; i < (int)ctx->inst.size(); ++i) {
    long long n = 0;
    if (int rc = mesh_volume(ctx, i, 0, nullptr, 0, &n)) return rc;
    std::vector<float> tris(9 * (size_t)n + 9);
    if (int rc = mesh_volume(ctx, i, 0, tris.data(), n, &n)) return rc;
    const std::string path =
        std::string(prefix) + "_" + std::to_string(ctx->inst[i].label) + ".vtk";
    if (int rc = write_vtk_mesh(path.c_str(), tris.data(), n)) {
      ctx->last_error = "mf_dump_mesh: cannot write " + path;
      return rc;
    }
  }
  return MF_OK;
}

}  // extern "C"

// Launch-shape autotuner (no reference counterpart).
//
// Two kernels of the frame have launch shapes that change their speed but not
// their results, because each output element is computed by one thread from
// the same inputs whatever the shape:
//  - raycast_objects_kernel: the pixel tile of a 128-thread CTA and the
//    register bound (residency) it is compiled for (ray_variants);
//  - integrate_blocks_kernel: how many 512-thread CTAs are resident per SM,
//    which sets both the register bound and the persistent grid (int_variants).
// autotune() times every candidate on the context's current frame with CUDA
// events and keeps the fastest.  The map is never touched: the raycasts write
// scratch maps and the integrations update a scratch copy of the pool slots
// in use.  A new choice bumps Tune::gen, so the next batched frame re-captures
// its graph with the chosen shapes.
#include <algorithm>
#include <cstring>
#include "mf_internal.h"

namespace mf {

namespace {

// RAII holder of the tuner's scratch device memory and events.
struct Scratch {
  void* p = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Scratch() {
    if (p) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// Mean time per launch of `launch` over `reps` launches, best of `trials`
// (the first trial also warms the instruction cache and L2).
template <typename F>
int time_launches(Context* ctx, Scratch& s, int reps, int trials, F launch, float* us) {
  float best = 3.4e38f;
  for (int t = 0; t < trials; ++t) {
    MF_CUDA(cudaEventRecord(s.e0, ctx->stream));
    for (int r = 0; r < reps; ++r)
      if (int rc = launch()) return rc;
    MF_CUDA(cudaEventRecord(s.e1, ctx->stream));
    MF_CUDA(cudaEventSynchronize(s.e1));
    float ms = 0;
    MF_CUDA(cudaEventElapsedTime(&ms, s.e0, s.e1));
    best = std::min(best, 1e3f * ms / reps);
  }
  *us = best;
  return MF_OK;
}

// dst <- a scratch copy of n elements of src, carved from f.
template <typename T>
int carve(Context* ctx, char*& f, T*& dst, const T* src, size_t n) {
  dst = (T*)f;
  f += n * sizeof(T);
  MF_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
  return MF_OK;
}

// The fastest candidate; the current one is kept unless another is more than
// 1 % faster (timing noise must not flip the choice back and forth).
int pick(const float* us, int n, int current) {
  int best = 0;
  for (int v = 1; v < n; ++v)
    if (us[v] < us[best]) best = v;
  return us[current] <= 1.01f * us[best] ? current : best;
}

}  // namespace

int tune_variant_count(int stage) {
  if (stage == MF_TUNE_RAYCAST) return ray_variant_count();
  if (stage == MF_TUNE_INTEGRATE) return int_variant_count();
  return 0;
}

int autotune(Context* ctx, int reps, float* ray_us, float* int_us) {
  const int n = (int)ctx->inst.size();
  if (n == 0) return MF_E_STATE;
  IdList all;
  all.n = n;
  uint32_t mask = 0;
  for (int i = 0; i < n; ++i) all.v[i] = i, mask |= 1u << i;
  const size_t WH = (size_t)ctx->W * ctx->H;
  int used = 0;
  MF_CUDA(cudaMemcpyAsync(&used, ctx->pool.count, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  used = std::min(used, ctx->pool.cap);
  // scratch: raycast maps, then the pool fields of the slots in use
  const size_t voxels = (size_t)used * 512;
  const size_t map_bytes = (WH * (2 * sizeof(F3) + sizeof(int)) + 255) & ~(size_t)255;
  const size_t field_bytes = voxels * (5 * sizeof(float) + 2 * sizeof(int) + sizeof(double));
  Scratch s;
  MF_CUDA(cudaMalloc(&s.p, map_bytes + field_bytes + (size_t)used + 256));
  MF_CUDA(cudaEventCreate(&s.e0));
  MF_CUDA(cudaEventCreate(&s.e1));
  char* base = (char*)s.p;
  F3* vert = (F3*)base;
  F3* norm = vert + WH;
  int* lab = (int*)(norm + WH);
  // instance frames for the current poses (what the next stages would use)
  if (int rc = stage_prepare(ctx, all)) return rc;

  const Tune before = ctx->tune;
  // raycast candidates
  const int nr = ray_variant_count();
  for (int v = 0; v < nr; ++v) {
    ctx->tune.ray = v;
    const int rc = time_launches(ctx, s, reps, 3, [&] {
      return stage_raycast_to(ctx, all, ctx->ray_epsilon, vert, norm, lab);
    }, &ray_us[v]);
    if (rc) { ctx->tune = before; return rc; }
  }
  ctx->tune.ray = before.ray;
  // integration candidates on a scratch copy of the slots in use
  const int ni = int_variant_count();
  if (used > 0) {
    Pool sp = ctx->pool;
    char* f = base + map_bytes;
    int rc = 0;
    rc |= carve(ctx, f, sp.tsdf, ctx->pool.tsdf, voxels);
    rc |= carve(ctx, f, sp.wt, ctx->pool.wt, voxels);
    rc |= carve(ctx, f, sp.r, ctx->pool.r, voxels);
    rc |= carve(ctx, f, sp.g, ctx->pool.g, voxels);
    rc |= carve(ctx, f, sp.b, ctx->pool.b, voxels);
    rc |= carve(ctx, f, sp.fg, ctx->pool.fg, voxels);
    rc |= carve(ctx, f, sp.c, ctx->pool.c, voxels);
    rc |= carve(ctx, f, sp.w, ctx->pool.w, voxels);
    rc |= carve(ctx, f, sp.active, ctx->pool.active, (size_t)used);
    if (rc) return MF_E_CUDA;
    if (int e = build_visit_list(ctx, mask)) return e;
    for (int v = 0; v < ni; ++v) {
      const int e = time_launches(ctx, s, reps, 3, [&] {
        return launch_integrate_blocks(ctx, sp, v);
      }, &int_us[v]);
      if (e) return e;
    }
  } else {
    for (int v = 0; v < ni; ++v) int_us[v] = 0.f;
  }
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  const int best_r = pick(ray_us, nr, before.ray);
  const int best_i = used > 0 ? pick(int_us, ni, before.integrate) : before.integrate;
  if (best_r != before.ray || best_i != before.integrate) {
    ctx->tune.ray = best_r;
    ctx->tune.integrate = best_i;
    ++ctx->tune.gen;
  }
  return MF_OK;
}

int tune_set(Context* ctx, int stage, int variant) {
  if (variant < 0 || variant >= tune_variant_count(stage)) return MF_E_ARG;
  int& slot = stage == MF_TUNE_RAYCAST ? ctx->tune.ray : ctx->tune.integrate;
  if (slot != variant) {
    slot = variant;
    ++ctx->tune.gen;
  }
  return MF_OK;
}

}  // namespace mf

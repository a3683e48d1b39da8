// Multi-instance octree raycasting on the device.
//
// raycastObjectList (apps/kfusion/src/cpp/rendering/rendering.cpp:9-181): per
// pixel, every instance in list order is raycast in its own frame; the nearest
// hit wins (ties go to the higher foreground probability) and its vertex,
// normal and label form the composite model maps.  The per-object model maps
// of the reference (m_vertex / m_normal for every object and pixel) are not
// materialised: they equal the composite maps where label == object and
// (0, INVALID normal) elsewhere, and the tracking kernels derive them on the fly.
#include "mf_internal.h"
#include "mf_sample.cuh"

namespace mf {

// Ray iterator constructor + first next(), lib/octree.hpp:919-1130 (ESVO
// traversal in [1, 2]^3).  Returns the entry distance of the first allocated
// block along the ray in voxel units, or -1.  Nodes are (level, Morton index);
// the traversal stack holds one entry per level.  The loop carries an
// iteration guard (never reached by a valid traversal; it only protects the
// GPU from a corrupted table).
__device__ __noinline__ float ray_first_block(const Volume& V, F3 origin, F3 direction,
                                              float nearPlane,
                                 float farPlane, float epsilon, int* status) {
  int st_m[MAX_LEVELS];
  float st_t[MAX_LEVELS];
  int st_l[MAX_LEVELS];
#pragma unroll
  for (int i = 0; i < MAX_LEVELS; ++i) { st_m[i] = 0; st_t[i] = 0.f; st_l[i] = 0; }
  F3 pos = mk3(1.f, 1.f, 1.f);
  int idx = 0;
  int p_level = 0, p_m = 0;  // parent: the root
  float scale_exp2 = 0.5f;
  int scale = CAST_STACK_DEPTH - 1;
  const int min_scale = CAST_STACK_DEPTH - V.block_level;
  const float voxelSize = V.dim / V.size;
  F3 d;
  d.x = fabsf(direction.x) < epsilon ? copysignf(epsilon, direction.x) : direction.x;
  d.y = fabsf(direction.y) < epsilon ? copysignf(epsilon, direction.y) : direction.y;
  d.z = fabsf(direction.z) < epsilon ? copysignf(epsilon, direction.z) : direction.z;
  const F3 so = origin / V.dim + 1.f;
  const F3 t_coef = mk3(-1.f / fabsf(d.x), -1.f / fabsf(d.y), -1.f / fabsf(d.z));
  F3 t_bias = t_coef * so;
  int octant_mask = 7;
  if (d.x > 0.0f) octant_mask ^= 1, t_bias.x = 3.0f * t_coef.x - t_bias.x;
  if (d.y > 0.0f) octant_mask ^= 2, t_bias.y = 3.0f * t_coef.y - t_bias.y;
  if (d.z > 0.0f) octant_mask ^= 4, t_bias.z = 3.0f * t_coef.z - t_bias.z;
  float t_min = fmx(fmx(2.0f * t_coef.x - t_bias.x, 2.0f * t_coef.y - t_bias.y),
                    2.0f * t_coef.z - t_bias.z);
  float t_max = fmn(fmn(t_coef.x - t_bias.x, t_coef.y - t_bias.y), t_coef.z - t_bias.z);
  float h = t_max;
  t_min = fmx(t_min, nearPlane / V.dim);
  t_max = fmn(t_max, farPlane / V.dim);
  if (1.5f * t_coef.x - t_bias.x > t_min) idx ^= 1, pos.x = 1.5f;
  if (1.5f * t_coef.y - t_bias.y > t_min) idx ^= 2, pos.y = 1.5f;
  if (1.5f * t_coef.z - t_bias.z > t_min) idx ^= 4, pos.z = 1.5f;

  for (int guard = 0; guard < 65536; ++guard) {
    if (scale >= CAST_STACK_DEPTH) return -1.f;
    const F3 t_corner = pos * t_coef - t_bias;
    const float tc_max = fmn(fmn(t_corner.x, t_corner.y), t_corner.z);
    const int ci = idx ^ octant_mask ^ 7;
    const int c_m = p_m * 8 + ci;
    bool has_child;
    if (p_level + 1 == V.block_level) has_child = V.block_tab[c_m] >= 0;
    else has_child = V.node_tab[V.node_off[p_level + 1] + c_m] != 0;
    if (scale == min_scale && has_child) {
      return t_min * V.dim / voxelSize;
    } else if (has_child && t_min <= t_max) {  // descend
      const float tv_max = fmn(t_max, tc_max);
      const float half = scale_exp2 * 0.5f;
      const F3 t_center = half * t_coef + t_corner;
      if (tc_max < h) {
        const int si = CAST_STACK_DEPTH - 1 - scale;  // = parent level
        st_m[si] = p_m; st_l[si] = p_level; st_t[si] = t_max;
      }
      h = tc_max;
      p_level += 1;
      p_m = c_m;
      scale--;
      scale_exp2 = half;
      idx = (t_center.x > t_min) | ((t_center.y > t_min) << 1) | ((t_center.z > t_min) << 2);
      pos.x += scale_exp2 * (float)(bool)(idx & 1);
      pos.y += scale_exp2 * (float)(bool)(idx & 2);
      pos.z += scale_exp2 * (float)(bool)(idx & 4);
      t_max = tv_max;
      continue;
    }
    // advance_ray
    const int step_mask = (t_corner.x <= tc_max) | ((t_corner.y <= tc_max) << 1) |
                          ((t_corner.z <= tc_max) << 2);
    pos.x -= scale_exp2 * (float)(bool)(step_mask & 1);
    pos.y -= scale_exp2 * (float)(bool)(step_mask & 2);
    pos.z -= scale_exp2 * (float)(bool)(step_mask & 4);
    t_min = tc_max;
    idx ^= step_mask;
    if ((idx & step_mask) != 0) {
      unsigned differing = 0;
      if (step_mask & 1) differing |= (unsigned)(__float_as_int(pos.x) ^ __float_as_int(pos.x + scale_exp2));
      if (step_mask & 2) differing |= (unsigned)(__float_as_int(pos.y) ^ __float_as_int(pos.y + scale_exp2));
      if (step_mask & 4) differing |= (unsigned)(__float_as_int(pos.z) ^ __float_as_int(pos.z + scale_exp2));
      scale = (__float_as_int((float)differing) >> 23) - 127;
      scale_exp2 = __int_as_float((scale - CAST_STACK_DEPTH + 127) << 23);
      if (scale >= CAST_STACK_DEPTH) return -1.f;  // left the root: no block on the ray
      const int si = CAST_STACK_DEPTH - 1 - scale;
      if (si < 0 || si >= V.block_level) {
        atomicOr(status, ST_RAY_GUARD);
        return -1.f;
      }
      p_m = st_m[si]; p_level = st_l[si]; t_max = st_t[si];
      const int shx = __float_as_int(pos.x) >> scale;
      const int shy = __float_as_int(pos.y) >> scale;
      const int shz = __float_as_int(pos.z) >> scale;
      pos.x = __int_as_float(shx << scale);
      pos.y = __int_as_float(shy << scale);
      pos.z = __int_as_float(shz << scale);
      idx = (shx & 1) | ((shy & 1) << 1) | ((shz & 1) << 2);
      h = 0.0f;
    }
  }
  atomicOr(status, ST_RAY_GUARD);
  return -1.f;
}

// raycast(const Volume<SDF>&, origin, direction, ...),
// apps/kfusion/src/cpp/kfusion/rendering_impl.hpp:80-140.
__device__ __noinline__ F4 raycast_volume(const Pool& P, const Volume& V, F3 origin,
                                          F3 direction,
                             float nearPlane, float farPlane, float mu, float step,
                             float largestep) {
  const F3 invR = mk3(1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z);
  const F3 tbot = (-1.f * invR) * origin;
  const F3 ttop = invR * (V.dim - origin);
  const F3 tmin = mk3(fmn(ttop.x, tbot.x), fmn(ttop.y, tbot.y), fmn(ttop.z, tbot.z));
  const F3 tmax = mk3(fmx(ttop.x, tbot.x), fmx(ttop.y, tbot.y), fmx(ttop.z, tbot.z));
  const float largest_tmin = fmx(fmx(tmin.x, tmin.y), fmx(tmin.x, tmin.z));
  const float smallest_tmax = fmn(fmn(tmax.x, tmax.y), fmn(tmax.x, tmax.z));
  const float tnear = fmx(largest_tmin, nearPlane);
  const float tfar = fmn(smallest_tmax, farPlane);
  const float inv = V.size / V.dim;
  if (tnear < tfar) {
    BlockMemo memo;
    float t = tnear, stepsize = largestep;
    F3 position = origin + direction * t;
    float f_t = volume_interp_m<0>(P, V, position, memo), f_tt = 0;
    if (f_t > 0) {
      // (guarded: a valid march takes at most (far - near) / step steps)
      for (int guard = 0; t < tfar && guard < (1 << 20); t += stepsize, ++guard) {
        // Volume::get -> get_fine at the truncated voxel (volume_template.hpp:83-88);
        // the weight test data.y < 0 can never hold for SDF voxels.
        const I3 s = to_i3(mk3(position.x * inv, position.y * inv, position.z * inv));
        f_tt = tsdf_at_m(P, V, memo, s.x, s.y, s.z);
        // f_tt <= 0.1 compares in double; for a float that is f_tt < 0.1f.
        if (f_tt < 0.1f && f_tt >= -0.5f) f_tt = volume_interp_m<0>(P, V, position, memo);
        if (f_tt < 0) break;
        stepsize = fmx(f_tt * mu, step);
        position = position + stepsize * direction;
        f_t = f_tt;
      }
      if (f_tt < 0) {
        t = t + stepsize * f_tt / (f_t - f_tt);
        const F3 p = origin + direction * t;
        return F4{p.x, p.y, p.z, t};
      }
    }
  }
  return F4{0, 0, 0, 0};
}

struct RayArgs {
  F3* vertex; F3* normal; int* label;
  int W, H;
  float nearPlane, farPlane, mu, epsilon;
};

// One thread per pixel, instances in list order (the reference's object loop).
__global__ void __launch_bounds__(128)
raycast_objects_kernel(Pool pool, const Volume* __restrict__ vols,
                       const InstFrame* __restrict__ frames, IdList ids, RayArgs a,
                       int* __restrict__ status) {
  const int x = blockIdx.x * 16 + (threadIdx.x & 15);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
  __shared__ int s_slot[8 * 128];
  const float INVALID = -2;
  float nearest = 1.0e3f;
  double high_fg = 0.f;
  int miss = 0;
  const M4 view = frames[ids.v[0]].view;
  const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
  for (int o = 0; o < ids.n; ++o) {
    const int i = ids.v[o];
    const Volume& V = vols[i];
    const InstFrame& F = frames[i];
    const float step = V.dim / V.size;
    const float largestep = step * 8;
    const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
    const float nfar = fmn(nearest, a.farPlane);
    const float t_min = ray_first_block(V, F.o_origin, o_dir, a.nearPlane, nfar, a.epsilon, status);
    const F4 hit = t_min > 0.f
                       ? raycast_volume(pool, V, F.o_origin, o_dir,
                                        t_min * V.dim / (unsigned)V.size, nfar, a.mu, step,
                                        largestep)
                       : F4{0, 0, 0, 0};
    const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
    if (hd > nearest) { miss++; continue; }
    const double fg = volume_interp(pool, V, mk3(hit.x, hit.y, hit.z), 1);
    if (fg <= 0.5f) { miss++; continue; }
    if (hd == nearest) {
      if (!(fg > high_fg)) { miss++; continue; }
    } else if (hd < nearest) {
      nearest = hd;
    } else {
      miss++;
      continue;
    }
    high_fg = fg;
    a.label[p] = F.label;
    a.vertex[p] = xform(F.T_w_o, mk3(hit.x, hit.y, hit.z));
    const F3 gn = volume_grad(pool, V, mk3(hit.x, hit.y, hit.z), s_slot + threadIdx.x, 128);
    if (length(gn) == 0) a.normal[p].x = INVALID;
    else a.normal[p] = normalize(rotate(F.T_w_o, gn));
  }
  if (miss == ids.n) {
    a.vertex[p] = mk3(0.f);
    a.normal[p] = mk3(INVALID, 0, 0);
    a.label[p] = (int)INVALID;
  }
}

int profile_raycast(Context* ctx, int reps, double* us) {
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  if (int rc = stage_prepare(ctx, all)) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx->stream);
  for (int r = 0; r < reps; ++r)
    if (int rc = stage_raycast(ctx, all, ctx->ray_epsilon)) return rc;
  cudaEventRecord(e1, ctx->stream);
  MF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *us = 1e3 * ms / reps;
  return MF_OK;
}

int stage_raycast(Context* ctx, const IdList& ids, float epsilon) {
  if (ids.n == 0) return MF_OK;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H,
            c.near_plane, c.far_plane, c.mu, epsilon};
  dim3 grid((ctx->W + 15) / 16, (ctx->H + 7) / 8);
  raycast_objects_kernel<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames,
                                                        ids, a, ctx->d_status);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

}  // namespace mf

#include <cstdio>
#include <cstring>
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

// True when ray_first_block cannot return a block that the march could use:
// the ray, with the direction clamped exactly as ray_first_block clamps it,
// misses both the box of the allocated blocks other than block 0 (`box`,
// voxel corners) and block 0 itself between nearPlane and farPlane.  Boxes
// and the t range are widened by two voxels, far beyond the float rounding of
// either test, so a ray that could reach a block is never skipped.  (A block
// that ray_first_block finds beyond farPlane makes the march return a miss,
// which is what skipping the ray gives.)
__device__ __forceinline__ bool ray_misses_blocks(const Volume& V, const int* box, F3 origin,
                                                  F3 direction, float nearPlane,
                                                  float farPlane, float epsilon) {
  F3 d;
  d.x = fabsf(direction.x) < epsilon ? copysignf(epsilon, direction.x) : direction.x;
  d.y = fabsf(direction.y) < epsilon ? copysignf(epsilon, direction.y) : direction.y;
  d.z = fabsf(direction.z) < epsilon ? copysignf(epsilon, direction.z) : direction.z;
  // the volume cube is [0, 1]^3 and t runs along d in these units
  const float vn = 1.f / (float)V.size;
  const float mg = 2.f * vn;
  const F3 o = origin / V.dim;
  const F3 inv = mk3(1.f / d.x, 1.f / d.y, 1.f / d.z);
  const float t0 = nearPlane / V.dim - mg, t1 = farPlane / V.dim + mg;
  auto hits = [&](float lx, float ly, float lz, float hx, float hy, float hz) {
    const float ax = (lx - o.x) * inv.x, bx = (hx - o.x) * inv.x;
    const float ay = (ly - o.y) * inv.y, by = (hy - o.y) * inv.y;
    const float az = (lz - o.z) * inv.z, bz = (hz - o.z) * inv.z;
    const float te = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), t0));
    const float tx = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), t1));
    return te <= tx;
  };
  if (hits(-mg, -mg, -mg, 8 * vn + mg, 8 * vn + mg, 8 * vn + mg)) return false;
  if (box[0] > box[3]) return true;  // no other block
  return !hits(box[0] * vn - mg, box[1] * vn - mg, box[2] * vn - mg, (box[3] + 8) * vn + mg,
               (box[4] + 8) * vn + mg, (box[5] + 8) * vn + mg);
}

// raycast(const Volume<SDF>&, origin, direction, ...),
// apps/kfusion/src/cpp/kfusion/rendering_impl.hpp:80-140.  With TC, *tc gets
// the march parameter t of the sample at which the crossing was found
// (+infinity when the march finds none).
template <bool TC = false>
__device__ __noinline__ F4 raycast_volume(const Pool& P, const Volume& V, F3 origin,
                                          F3 direction,
                             float nearPlane, float farPlane, float mu, float step,
                             float largestep, float* tc = nullptr) {
  if (TC) *tc = INFINITY;
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
        if (TC) *tc = t;
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
// 128 threads cover a TW x (128 / TW) pixel tile; MINB is the residency the
// register allocation is bounded for (1: unbounded).  Every variant computes
// each pixel alike, so the autotuner may pick any of them (ray_variants).
template <int TW, int MINB>
__global__ void __launch_bounds__(128, MINB)
raycast_objects_kernel(Pool pool, const Volume* __restrict__ vols,
                       const InstFrame* __restrict__ frames, IdList ids, RayArgs a,
                       int* __restrict__ status) {
  const int x = blockIdx.x * TW + (threadIdx.x % TW);
  const int y = blockIdx.y * (128 / TW) + (threadIdx.x / TW);
  __shared__ int s_slot[8 * 128];
  // per instance: the box of its allocated blocks and the foreground value a
  // missed ray reads (the reference interpolates fg at the zero hit point)
  __shared__ int s_box[MAX_INSTANCES][6];
  __shared__ float s_fg0[MAX_INSTANCES];
  for (int o = threadIdx.x; o < ids.n; o += blockDim.x) {
    const Volume& V = vols[ids.v[o]];
    for (int j = 0; j < 6; ++j) s_box[o][j] = V.bbox[j];
    s_fg0[o] = volume_interp(pool, V, mk3(0.f, 0.f, 0.f), 1);
  }
  __syncthreads();
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
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
    const float t_min =
        ray_misses_blocks(V, s_box[o], F.o_origin, o_dir, a.nearPlane, nfar, a.epsilon)
            ? -1.f
            : ray_first_block(V, F.o_origin, o_dir, a.nearPlane, nfar, a.epsilon, status);
    const F4 hit = t_min > 0.f
                       ? raycast_volume(pool, V, F.o_origin, o_dir,
                                        t_min * V.dim / (unsigned)V.size, nfar, a.mu, step,
                                        largestep)
                       : F4{0, 0, 0, 0};
    const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
    if (hd > nearest) { miss++; continue; }
    const bool at0 = hit.x == 0.f && hit.y == 0.f && hit.z == 0.f;
    const double fg = at0 ? s_fg0[o] : volume_interp(pool, V, mk3(hit.x, hit.y, hit.z), 1);
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

// ------------------------------------------------------------------------
// Phased composite raycast: the same maps as raycast_objects_kernel, in two
// launches.
//  1. raycast_hits_kernel (grid.z = instance): every instance's ray of every
//     pixel, traversed and marched up to the far plane, not to the running
//     nearest hit: the hit (x, y, z, t), the march parameter tc of the sample
//     at which the crossing was found (+inf: none) and the foreground value at
//     the hit.  The warps of a CTA all work on one instance.
//  2. raycast_fold_kernel: per pixel, the reference's composite over the
//     instances in list order.  The reference bounds instance o's traversal
//     and march by nfar = min(nearest, far) (rendering.cpp:47-62): with the
//     same start and the same steps, the bounded march finds the unbounded
//     march's crossing exactly when that crossing's sample lies before nfar
//     (tc < nfar), and otherwise returns the zero hit, whose foreground is
//     read at the volume origin.  The fold applies that rule, then the
//     nearest-hit / foreground / tie tests, and computes the gradient of the
//     final winner only.
// The bounded traversal reaches the same first block as the unbounded one
// whenever the march's crossing lies before nfar (the block's entry and all
// its ancestors' lie before the crossing); the maps equal the one-kernel
// path's bit for bit (autotuner identity test).
struct RayRec {
  F4* hit;      // [o * W * H + p]
  float2* tf;   // (tc, foreground at the hit)
};

template <int TW>
__global__ void __launch_bounds__(128)
raycast_hits_kernel(Pool pool, const Volume* __restrict__ vols,
                    const InstFrame* __restrict__ frames, IdList ids, RayArgs a, RayRec rec,
                    int rec_base, int* __restrict__ status) {
  const int x = blockIdx.x * TW + (threadIdx.x % TW);
  const int y = blockIdx.y * (128 / TW) + (threadIdx.x / TW);
  if (x >= a.W || y >= a.H) return;
  const int o = blockIdx.z;
  const int i = ids.v[o];
  const Volume& V = vols[i];
  const InstFrame& F = frames[i];
  const int p = x + y * a.W;
  const M4 view = frames[ids.v[0]].view;
  const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
  const float step = V.dim / V.size;
  const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
  const float t_min =
      ray_misses_blocks(V, V.bbox, F.o_origin, o_dir, a.nearPlane, a.farPlane, a.epsilon)
          ? -1.f
          : ray_first_block(V, F.o_origin, o_dir, a.nearPlane, a.farPlane, a.epsilon, status);
  F4 hit = F4{0, 0, 0, 0};
  float tc = INFINITY, fg = 0.f;
  if (t_min > 0.f) {
    hit = raycast_volume<true>(pool, V, F.o_origin, o_dir, t_min * V.dim / (unsigned)V.size,
                               a.farPlane, a.mu, step, step * 8, &tc);
    if (tc < INFINITY) fg = volume_interp(pool, V, mk3(hit.x, hit.y, hit.z), 1);
  }
  const size_t q = (size_t)(rec_base + o) * a.W * a.H + p;
  rec.hit[q] = hit;
  rec.tf[q] = make_float2(tc, fg);
}

template <int TW>
__global__ void __launch_bounds__(128)
raycast_fold_kernel(Pool pool, const Volume* __restrict__ vols,
                    const InstFrame* __restrict__ frames, IdList ids, RayArgs a, RayRec rec) {
  const int x = blockIdx.x * TW + (threadIdx.x % TW);
  const int y = blockIdx.y * (128 / TW) + (threadIdx.x / TW);
  __shared__ int s_slot[8 * 128];
  __shared__ float s_fg0[MAX_INSTANCES];
  for (int o = threadIdx.x; o < ids.n; o += blockDim.x)
    s_fg0[o] = volume_interp(pool, vols[ids.v[o]], mk3(0.f, 0.f, 0.f), 1);
  __syncthreads();
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
  const size_t WH = (size_t)a.W * a.H;
  const float INVALID = -2;
  float nearest = 1.0e3f;
  double high_fg = 0.f;
  int miss = 0;
  unsigned winners = 0;   // every instance that became the running winner
  unsigned zeroh = 0;     // ... with the zero hit of a march bounded before its crossing
  int win = -1;
  F4 win_hit = F4{0, 0, 0, 0};
  for (int o = 0; o < ids.n; ++o) {
    const InstFrame& F = frames[ids.v[o]];
    const float nfar = fmn(nearest, a.farPlane);
    const float2 tf = rec.tf[o * WH + p];
    F4 hit = F4{0, 0, 0, 0};
    double fg = s_fg0[o];
    const bool crossed = tf.x < nfar;
    if (crossed) {
      hit = rec.hit[o * WH + p];
      fg = tf.y;
    }
    const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
    if (hd > nearest) { miss++; continue; }
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
    winners |= 1u << o;
    if (!crossed) zeroh |= 1u << o;
    win = o;
    win_hit = hit;
  }
  if (win < 0) {
    if (miss == ids.n) {
      a.vertex[p] = mk3(0.f);
      a.normal[p] = mk3(INVALID, 0, 0);
      a.label[p] = (int)INVALID;
    }
    return;
  }
  const InstFrame& F = frames[ids.v[win]];
  a.label[p] = F.label;
  a.vertex[p] = xform(F.T_w_o, mk3(win_hit.x, win_hit.y, win_hit.z));
  const F3 gn = volume_grad(pool, vols[ids.v[win]], mk3(win_hit.x, win_hit.y, win_hit.z),
                            s_slot + threadIdx.x, 128);
  if (length(gn) != 0) {
    a.normal[p] = normalize(rotate(F.T_w_o, gn));
    return;
  }
  // a zero gradient writes only the normal's x (rendering.cpp:105-107, 126-128):
  // y and z are those of the latest earlier winner with a nonzero gradient, as
  // the reference's successive writes leave them, or the map's previous values
  a.normal[p].x = INVALID;
  for (int o = win - 1; o >= 0; --o) {
    if (!(winners & (1u << o))) continue;
    const InstFrame& Fo = frames[ids.v[o]];
    const F4 hit = (zeroh & (1u << o)) ? F4{0, 0, 0, 0} : rec.hit[o * WH + p];
    const F3 g2 = volume_grad(pool, vols[ids.v[o]], mk3(hit.x, hit.y, hit.z),
                              s_slot + threadIdx.x, 128);
    if (length(g2) != 0) {
      const F3 n2 = normalize(rotate(Fo.T_w_o, g2));
      a.normal[p].y = n2.y;
      a.normal[p].z = n2.z;
      return;
    }
  }
}

// ------------------------------------------------------------------------
// Instance-sharded raycast (mf_raycast_records / mf_raycast_fold): the
// phased path's records, with the world normal of every crossing computed by
// the GPU that holds the volume, so that the fold needs no volume.
__global__ void __launch_bounds__(128)
raycast_records_kernel(Pool pool, const Volume* __restrict__ vols,
                       const InstFrame* __restrict__ frames, IdList ids, M4 view, RayArgs a,
                       mf_ray_record* __restrict__ rec, int* __restrict__ status) {
  __shared__ int s_slot[8 * 128];
  const int x = blockIdx.x * 16 + (threadIdx.x % 16);
  const int y = blockIdx.y * 8 + (threadIdx.x / 16);
  if (x >= a.W || y >= a.H) return;
  const int o = blockIdx.z;
  const int i = ids.v[o];
  const Volume& V = vols[i];
  const InstFrame& F = frames[i];
  const int p = x + y * a.W;
  const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
  const float step = V.dim / V.size;
  const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
  const float t_min =
      ray_misses_blocks(V, V.bbox, F.o_origin, o_dir, a.nearPlane, a.farPlane, a.epsilon)
          ? -1.f
          : ray_first_block(V, F.o_origin, o_dir, a.nearPlane, a.farPlane, a.epsilon, status);
  F4 hit = F4{0, 0, 0, 0};
  float tc = INFINITY;
  if (t_min > 0.f)
    hit = raycast_volume<true>(pool, V, F.o_origin, o_dir, t_min * V.dim / (unsigned)V.size,
                               a.farPlane, a.mu, step, step * 8, &tc);
  mf_ray_record r;
  r.hit[0] = hit.x; r.hit[1] = hit.y; r.hit[2] = hit.z; r.hit[3] = hit.w;
  r.tc = tc;
  r.fg = 0.f;
  r.normal[0] = r.normal[1] = r.normal[2] = 0.f;
  r.zero_grad = 1;
  r.pad[0] = r.pad[1] = 0;
  if (tc < INFINITY) {
    const F3 h = mk3(hit.x, hit.y, hit.z);
    r.fg = volume_interp(pool, V, h, 1);
    const F3 gn = volume_grad(pool, V, h, s_slot + threadIdx.x, 128);
    if (length(gn) != 0) {
      const F3 n = normalize(rotate(F.T_w_o, gn));
      r.normal[0] = n.x; r.normal[1] = n.y; r.normal[2] = n.z;
      r.zero_grad = 0;
    }
  }
  rec[(size_t)o * a.W * a.H + p] = r;
}

// foreground and world normal of each listed instance at the zero hit
__global__ void raycast_origins_kernel(Pool pool, const Volume* __restrict__ vols,
                                       const InstFrame* __restrict__ frames, IdList ids,
                                       mf_ray_origin* __restrict__ out) {
  __shared__ int s_slot[8 * 32];
  const int o = threadIdx.x;
  if (o >= ids.n) return;
  const Volume& V = vols[ids.v[o]];
  const InstFrame& F = frames[ids.v[o]];
  mf_ray_origin r;
  r.fg = volume_interp(pool, V, mk3(0.f, 0.f, 0.f), 1);
  const F3 gn = volume_grad(pool, V, mk3(0.f, 0.f, 0.f), s_slot + threadIdx.x, 32);
  r.zero_grad = length(gn) == 0 ? 1 : 0;
  const F3 n = r.zero_grad ? mk3(0.f) : normalize(rotate(F.T_w_o, gn));
  r.normal[0] = n.x; r.normal[1] = n.y; r.normal[2] = n.z;
  r.pad[0] = r.pad[1] = r.pad[2] = 0;
  out[o] = r;
}

// the composite of raycast_fold_kernel from records (all instances, in order)
__global__ void __launch_bounds__(128)
raycast_fold_records_kernel(const InstFrame* __restrict__ frames, IdList ids, RayArgs a,
                            const mf_ray_record* __restrict__ rec,
                            const mf_ray_origin* __restrict__ orig) {
  const int x = blockIdx.x * 16 + (threadIdx.x % 16);
  const int y = blockIdx.y * 8 + (threadIdx.x / 16);
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
  const size_t WH = (size_t)a.W * a.H;
  const float INVALID = -2;
  float nearest = 1.0e3f;
  double high_fg = 0.f;
  int miss = 0;
  int win = -1;
  F4 win_hit = F4{0, 0, 0, 0};
  F3 win_n = mk3(0.f), last_full = mk3(0.f);
  bool win_zero = true, have_full = false;
  for (int o = 0; o < ids.n; ++o) {
    const InstFrame& F = frames[ids.v[o]];
    const float nfar = fmn(nearest, a.farPlane);
    const mf_ray_record& r = rec[o * WH + p];
    F4 hit = F4{0, 0, 0, 0};
    double fg;
    F3 n;
    bool zero;
    if (r.tc < nfar) {
      hit = F4{r.hit[0], r.hit[1], r.hit[2], r.hit[3]};
      fg = r.fg;
      n = mk3(r.normal[0], r.normal[1], r.normal[2]);
      zero = r.zero_grad != 0;
    } else {
      fg = orig[o].fg;
      n = mk3(orig[o].normal[0], orig[o].normal[1], orig[o].normal[2]);
      zero = orig[o].zero_grad != 0;
    }
    const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
    if (hd > nearest) { miss++; continue; }
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
    // the reference writes each winner's normal as it wins (only x when its
    // gradient is zero): y and z end as the latest full write's
    if (win >= 0 && !win_zero) { last_full = win_n; have_full = true; }
    win = o;
    win_hit = hit;
    win_n = n;
    win_zero = zero;
  }
  if (win < 0) {
    if (miss == ids.n) {
      a.vertex[p] = mk3(0.f);
      a.normal[p] = mk3(INVALID, 0, 0);
      a.label[p] = (int)INVALID;
    }
    return;
  }
  const InstFrame& F = frames[ids.v[win]];
  a.label[p] = F.label;
  a.vertex[p] = xform(F.T_w_o, mk3(win_hit.x, win_hit.y, win_hit.z));
  if (!win_zero) {
    a.normal[p] = win_n;
  } else {
    a.normal[p].x = INVALID;
    if (have_full) {
      a.normal[p].y = last_full.y;
      a.normal[p].z = last_full.z;
    }
  }
}

int raycast_records(Context* ctx, const IdList& ids, mf_ray_record* d_records,
                    mf_ray_origin* d_origins) {
  if (ids.n == 0) return MF_OK;
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  if (int rc = stage_prepare(ctx, all)) return rc;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H, c.near_plane,
            c.far_plane, c.mu, ctx->ray_epsilon};
  // every instance's frame holds the same camera view (rendering.cpp:17)
  InstFrame f0;
  MF_CUDA(cudaMemcpyAsync(&f0, ctx->d_frames, sizeof(InstFrame), cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  dim3 grid((ctx->W + 15) / 16, (ctx->H + 7) / 8, ids.n);
  raycast_records_kernel<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames,
                                                         ids, f0.view, a, d_records,
                                                         ctx->d_status);
  raycast_origins_kernel<<<1, 32, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames, ids,
                                                    d_origins);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

int raycast_fold(Context* ctx, const mf_ray_record* d_records, const mf_ray_origin* d_origins) {
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  if (int rc = stage_prepare(ctx, all)) return rc;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H, c.near_plane,
            c.far_plane, c.mu, ctx->ray_epsilon};
  dim3 grid((ctx->W + 15) / 16, (ctx->H + 7) / 8);
  raycast_fold_records_kernel<<<grid, 128, 0, ctx->stream>>>(ctx->d_frames, all, a, d_records,
                                                             d_origins);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// Algorithmic bytes of one composite raycast (the per-unit figures of the
// raycast's roofline): the same march as raycast_objects_kernel, counting
// instead of writing.  Per ray and instance: 8 B for every voxel read of the
// march (tsdf + weight of Volume::get), 32 B for every trilinear TSDF
// interpolation (8 taps), 64 B for the foreground interpolation of a
// candidate hit (8 FP64 taps) and 192 B for its gradient (48 voxel reads);
// per pixel 28 B of output (vertex, normal, label).  Counted on the device
// after the timed launches (profile_raycast), never inside a frame.
__device__ __noinline__ void march_count(const Pool& P, const Volume& V, F3 origin, F3 direction,
                                         float nearPlane, float farPlane, float mu, float step,
                                         float largestep, unsigned long long* cnt, F4* out) {
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
  unsigned long long samples = 0, interps = 0;
  *out = F4{0, 0, 0, 0};
  if (tnear < tfar) {
    BlockMemo memo;
    float t = tnear, stepsize = largestep;
    F3 position = origin + direction * t;
    float f_t = volume_interp_m<0>(P, V, position, memo), f_tt = 0;
    ++interps;
    if (f_t > 0) {
      for (int guard = 0; t < tfar && guard < (1 << 20); t += stepsize, ++guard) {
        const I3 s = to_i3(mk3(position.x * inv, position.y * inv, position.z * inv));
        f_tt = tsdf_at_m(P, V, memo, s.x, s.y, s.z);
        ++samples;
        if (f_tt < 0.1f && f_tt >= -0.5f) {
          f_tt = volume_interp_m<0>(P, V, position, memo);
          ++interps;
        }
        if (f_tt < 0) break;
        stepsize = fmx(f_tt * mu, step);
        position = position + stepsize * direction;
        f_t = f_tt;
      }
      if (f_tt < 0) {
        t = t + stepsize * f_tt / (f_t - f_tt);
        const F3 p = origin + direction * t;
        *out = F4{p.x, p.y, p.z, t};
      }
    }
  }
  cnt[0] += samples;
  cnt[1] += interps;
}

__global__ void raycast_count_kernel(Pool pool, const Volume* __restrict__ vols,
                                     const InstFrame* __restrict__ frames, IdList ids, RayArgs a,
                                     int* __restrict__ status,
                                     unsigned long long* __restrict__ totals) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  unsigned long long c[4] = {0, 0, 0, 0};  // samples, interps, fg reads, gradients
  if (x < a.W) {
    float nearest = 1.0e3f;
    double high_fg = 0.f;
    const M4 view = frames[ids.v[0]].view;
    const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
    for (int o = 0; o < ids.n; ++o) {
      const int i = ids.v[o];
      const Volume& V = vols[i];
      const InstFrame& F = frames[i];
      const float step = V.dim / V.size;
      const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
      const float nfar = fmn(nearest, a.farPlane);
      const float t_min = ray_first_block(V, F.o_origin, o_dir, a.nearPlane, nfar, a.epsilon,
                                          status);
      F4 hit = F4{0, 0, 0, 0};
      if (t_min > 0.f)
        march_count(pool, V, F.o_origin, o_dir, t_min * V.dim / (unsigned)V.size, nfar, a.mu,
                    step, step * 8, c, &hit);
      const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
      if (hd > nearest) continue;
      const double fg = volume_interp(pool, V, mk3(hit.x, hit.y, hit.z), 1);
      ++c[2];
      if (fg <= 0.5f) continue;
      if (hd == nearest) {
        if (!(fg > high_fg)) continue;
      } else if (hd < nearest) {
        nearest = hd;
      } else {
        continue;
      }
      high_fg = fg;
      ++c[3];
    }
  }
  for (int k = 0; k < 4; ++k) {
    unsigned long long v = c[k];
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(totals + k, v);
  }
}

static int count_raycast_bytes(Context* ctx, const IdList& ids, double* bytes) {
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H, c.near_plane,
            c.far_plane, c.mu, ctx->ray_epsilon};
  unsigned long long* d = nullptr;
  MF_CUDA(cudaMalloc(&d, 4 * sizeof(unsigned long long)));
  cudaMemsetAsync(d, 0, 4 * sizeof(unsigned long long), ctx->stream);
  raycast_count_kernel<<<dim3((ctx->W + 127) / 128, ctx->H), 128, 0, ctx->stream>>>(
      ctx->pool, ctx->d_vols, ctx->d_frames, ids, a, ctx->d_status, d);
  unsigned long long h[4] = {0, 0, 0, 0};
  cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("raycast byte count: ") + cudaGetErrorString(e);
    return MF_E_CUDA;
  }
  *bytes = 8.0 * h[0] + 32.0 * h[1] + 64.0 * h[2] + 192.0 * h[3] + 28.0 * ctx->W * ctx->H;
  return MF_OK;
}

int profile_raycast(Context* ctx, int reps, double* us, double* bytes) {
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
  return bytes ? count_raycast_bytes(ctx, all, bytes) : MF_OK;
}

int stage_raycast(Context* ctx, const IdList& ids, float epsilon) {
  return stage_raycast_to(ctx, ids, epsilon, ctx->d_vertex, ctx->d_normal, ctx->d_label);
}

// Launch-shape candidates of the composite raycast: the one-kernel path
// (raycast_objects_kernel) by tile width x register bound, and the phased path
// (raycast_hits_kernel + raycast_fold_kernel) by tile width.  Entry 0 is the
// default.
using RayFn = void (*)(Pool, const Volume*, const InstFrame*, IdList, RayArgs, int*);
using HitsFn = void (*)(Pool, const Volume*, const InstFrame*, IdList, RayArgs, RayRec, int,
                        int*);
using FoldFn = void (*)(Pool, const Volume*, const InstFrame*, IdList, RayArgs, RayRec);
struct RayVariant {
  int tw, minb;
  RayFn fn;        // one kernel, or nullptr for the phased path
  HitsFn hits;
  FoldFn fold;
};
static const RayVariant ray_variants[] = {
    {16, 1, raycast_objects_kernel<16, 1>, nullptr, nullptr},
    {32, 1, raycast_objects_kernel<32, 1>, nullptr, nullptr},
    {8, 1, raycast_objects_kernel<8, 1>, nullptr, nullptr},
    {16, 6, raycast_objects_kernel<16, 6>, nullptr, nullptr},
    {32, 6, raycast_objects_kernel<32, 6>, nullptr, nullptr},
    {8, 6, raycast_objects_kernel<8, 6>, nullptr, nullptr},
    {16, 8, raycast_objects_kernel<16, 8>, nullptr, nullptr},
    {32, 8, raycast_objects_kernel<32, 8>, nullptr, nullptr},
    {8, 8, raycast_objects_kernel<8, 8>, nullptr, nullptr},
    {16, 0, nullptr, raycast_hits_kernel<16>, raycast_fold_kernel<16>},
    {32, 0, nullptr, raycast_hits_kernel<32>, raycast_fold_kernel<32>},
    {8, 0, nullptr, raycast_hits_kernel<8>, raycast_fold_kernel<8>},
};
constexpr int N_RAY_VARIANTS = (int)(sizeof(ray_variants) / sizeof(ray_variants[0]));
static_assert(N_RAY_VARIANTS <= MAX_TUNE_VARIANTS, "raycast candidate table too long");

int ray_variant_count() { return N_RAY_VARIANTS; }

void ray_variant_describe(int v, char* buf, int cap) {
  const RayVariant& r = ray_variants[v];
  if (!r.fn)
    snprintf(buf, cap, "raycast phased (per-instance hits, then the composite fold), tile %dx%d",
             r.tw, 128 / r.tw);
  else if (r.minb > 1)
    snprintf(buf, cap, "raycast tile %dx%d, registers bounded for %d CTAs/SM", r.tw, 128 / r.tw,
             r.minb);
  else
    snprintf(buf, cap, "raycast tile %dx%d, registers unbounded", r.tw, 128 / r.tw);
}

int stage_raycast_to(Context* ctx, const IdList& ids, float epsilon, F3* vertex, F3* normal,
                     int* label) {
  if (ids.n == 0) return MF_OK;
  const mf_config& c = ctx->cfg;
  RayArgs a{vertex, normal, label, ctx->W, ctx->H, c.near_plane, c.far_plane, c.mu, epsilon};
  const RayVariant& r = ray_variants[ctx->tune.ray];
  const int th = 128 / r.tw;
  dim3 grid((ctx->W + r.tw - 1) / r.tw, (ctx->H + th - 1) / th);
  if (r.fn) {
    r.fn<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames, ids, a,
                                        ctx->d_status);
  } else {
    if (ids.n > ctx->cfg.max_instances) return MF_E_ARG;
    const RayRec rec{ctx->d_rayhit, ctx->d_raytf};
    r.hits<<<dim3(grid.x, grid.y, ids.n), 128, 0, ctx->stream>>>(
        ctx->pool, ctx->d_vols, ctx->d_frames, ids, a, rec, 0, ctx->d_status);
    r.fold<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames, ids, a, rec);
  }
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

bool raycast_is_phased(const Context* ctx) { return ray_variants[ctx->tune.ray].fn == nullptr; }

// The phased composite in parts: the per-instance marches of `ids` into the
// records of list positions base .. base + ids.n - 1 (each instance's march
// is independent of the others'), and the fold over the whole list.  Only
// with a phased launch shape (raycast_is_phased).
int stage_raycast_hits(Context* ctx, const IdList& ids, int base, float epsilon) {
  if (ids.n == 0) return MF_OK;
  const RayVariant& r = ray_variants[ctx->tune.ray];
  if (r.fn || base < 0 || base + ids.n > ctx->cfg.max_instances) return MF_E_STATE;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H, c.near_plane,
            c.far_plane, c.mu, epsilon};
  const int th = 128 / r.tw;
  const dim3 grid((ctx->W + r.tw - 1) / r.tw, (ctx->H + th - 1) / th, ids.n);
  const RayRec rec{ctx->d_rayhit, ctx->d_raytf};
  r.hits<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames, ids, a, rec, base,
                                        ctx->d_status);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

int stage_raycast_fold(Context* ctx, const IdList& ids, float epsilon) {
  if (ids.n == 0) return MF_OK;
  const RayVariant& r = ray_variants[ctx->tune.ray];
  if (r.fn || ids.n > ctx->cfg.max_instances) return MF_E_STATE;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H, c.near_plane,
            c.far_plane, c.mu, epsilon};
  const int th = 128 / r.tw;
  const dim3 grid((ctx->W + r.tw - 1) / r.tw, (ctx->H + th - 1) / th);
  const RayRec rec{ctx->d_rayhit, ctx->d_raytf};
  r.fold<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames, ids, a, rec);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// ------------------------------------------------------------------------
// Adjoint of the composite raycast (no reference counterpart): carries
// dE/d(model vertex) and dE/d(model normal) of a pixel back to the TSDF values
// of the winning instance's voxels.  The vertex is T_w_o (o + d t*), where the
// march (raycast_volume) ends with the secant step
//   t* = t_k + s_{k-1} f_k / (f_{k-1} - f_k),
// every sample position depends on the earlier step lengths
// s_j = max(mu f_j, voxel), and every sample value f_j is a voxel read (get) or
// a trilinear interpolation.  The backward sweep needs the samples in reverse:
// the forward march is replayed once with a checkpoint of the sample position
// every ADJ_SEG samples, and each segment is replayed again, from its checkpoint,
// just before it is swept; no per-sample state is stored beyond one segment.
// The normal is normalize(R grad(tsdf, hit)); its adjoint reaches the 32 taps
// of the central differences and, through their trilinear weights, the hit.
constexpr int ADJ_SEG = 32;      // samples per checkpoint
constexpr int ADJ_MAX_CP = 64;   // checkpoints: rays of up to 2048 samples

// Scatters g * d f / d tsdf of the trilinear interpolation at `pos`
// (volume_interp_m) and returns d f / d t along `dir`.
__device__ float interp_adjoint(const Pool& P, const Volume& V, BlockMemo& m, F3 pos, F3 dir,
                                float g, float* __restrict__ grad) {
  const float inv = V.size / V.dim;
  const F3 pv = mk3(pos.x * inv, pos.y * inv, pos.z * inv);
  const F3 fl = floor3(pv);
  const I3 base = to_i3(fl);
  const F3 f = mk3(pv.x - fl.x, pv.y - fl.y, pv.z - fl.z);
  const int lx = imx(base.x, 0), ly = imx(base.y, 0), lz = imx(base.z, 0);
  float dfx = 0.f, dfy = 0.f, dfz = 0.f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int x = lx + (i & 1), y = ly + ((i >> 1) & 1), z = lz + (i >> 2);
    const int ts = memo_slot(V, m, x, y, z);
    const float val = ts < 0 ? 1.f : __ldg(P.tsdf + (size_t)ts * 512 + voxel_index(x, y, z));
    const float wx = (i & 1) ? f.x : 1.f - f.x, wy = (i & 2) ? f.y : 1.f - f.y,
                wz = (i & 4) ? f.z : 1.f - f.z;
    if (ts >= 0 && g != 0.f)
      atomicAdd(grad + (size_t)ts * 512 + voxel_index(x, y, z), g * wx * wy * wz);
    dfx += val * ((i & 1) ? 1.f : -1.f) * wy * wz;
    dfy += val * ((i & 2) ? 1.f : -1.f) * wx * wz;
    dfz += val * ((i & 4) ? 1.f : -1.f) * wx * wy;
  }
  return inv * (dfx * dir.x + dfy * dir.y + dfz * dir.z);
}

// The same for one sample of raycast_volume's loop: a voxel read, or the
// interpolation when the read lies in [-0.5, 0.1).
__device__ float sample_adjoint(const Pool& P, const Volume& V, BlockMemo& m, F3 pos, F3 dir,
                                float g, float* __restrict__ grad) {
  const float inv = V.size / V.dim;
  const I3 s = to_i3(mk3(pos.x * inv, pos.y * inv, pos.z * inv));
  const int sl = memo_slot(V, m, s.x, s.y, s.z);
  const float fv = sl < 0 ? 1.f : __ldg(P.tsdf + (size_t)sl * 512 + voxel_index(s.x, s.y, s.z));
  if (fv < 0.1f && fv >= -0.5f) return interp_adjoint(P, V, m, pos, dir, g, grad);
  if (sl >= 0 && g != 0.f) atomicAdd(grad + (size_t)sl * 512 + voxel_index(s.x, s.y, s.z), g);
  return 0.f;
}

// The sample value of raycast_volume's loop at `pos`.
__device__ __forceinline__ float march_value(const Pool& P, const Volume& V, BlockMemo& m,
                                             F3 pos) {
  const float inv = V.size / V.dim;
  const I3 s = to_i3(mk3(pos.x * inv, pos.y * inv, pos.z * inv));
  float f = tsdf_at_m(P, V, m, s.x, s.y, s.z);
  if (f < 0.1f && f >= -0.5f) f = volume_interp_m<0>(P, V, pos, m);
  return f;
}

// Replays raycast_volume and sweeps its march backwards with dE/dt* = g_t.
// Returns 1 when done, 0 when the replay found no hit (nothing to do), -1 when
// the march is longer than the checkpoints cover (the ray is skipped).
__device__ __noinline__ int march_adjoint(const Pool& P, const Volume& V, F3 origin,
                                          F3 direction, float nearPlane, float farPlane,
                                          float mu, float step, float largestep, float g_t,
                                          float* __restrict__ grad, F3* hit) {
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
  if (!(tnear < tfar)) return 0;
  BlockMemo memo;
  float t = tnear, stepsize = largestep;
  F3 position = origin + direction * t;
  float f_t = volume_interp_m<0>(P, V, position, memo), f_tt = 0;
  if (!(f_t > 0)) return 0;
  const F3 p0 = position;
  F3 cp_p[ADJ_MAX_CP];  // sample position at each checkpoint
  int k = 0;
  for (int guard = 0; t < tfar && guard < (1 << 20); t += stepsize, ++guard) {
    if (k % ADJ_SEG == 0) {
      const int c = k / ADJ_SEG;
      if (c >= ADJ_MAX_CP) return -1;
      cp_p[c] = position;
    }
    const I3 s = to_i3(mk3(position.x * inv, position.y * inv, position.z * inv));
    f_tt = tsdf_at_m(P, V, memo, s.x, s.y, s.z);
    if (f_tt < 0.1f && f_tt >= -0.5f) f_tt = volume_interp_m<0>(P, V, position, memo);
    if (f_tt < 0) break;
    stepsize = fmx(f_tt * mu, step);
    position = position + stepsize * direction;
    f_t = f_tt;
    ++k;
  }
  if (!(f_tt < 0)) return 0;
  {
    const float th = t + stepsize * f_tt / (f_t - f_tt);
    *hit = origin + direction * th;
  }
  // t* = t_k + s f_k / (a - f_k) with s = s_{k-1} and a = f_{k-1} (for k = 0 the
  // constant largestep and the interpolation that opened the march)
  const float den = f_t - f_tt;
  const float g_fk = g_t * stepsize * f_t / (den * den);
  const float g_s = g_t * f_tt / den;
  const float g_a = -g_t * stepsize * f_tt / (den * den);
  float GT = g_t;  // dE/dt_j, carried backwards
  float seg_f[ADJ_SEG];
  F3 seg_p[ADJ_SEG];
  for (int c = k / ADJ_SEG; c >= 0; --c) {
    // replay samples j0 .. j1 of this segment from its checkpoint
    const int j0 = c * ADJ_SEG, j1 = min(j0 + ADJ_SEG - 1, k);
    F3 pos = cp_p[c];
    for (int j = j0; j <= j1; ++j) {
      seg_p[j - j0] = pos;
      const float f = march_value(P, V, memo, pos);
      seg_f[j - j0] = f;
      if (j < j1) pos = pos + fmx(f * mu, step) * direction;
    }
    for (int j = j1; j >= j0; --j) {
      float gf;
      if (j == k) {
        gf = g_fk;
      } else {
        // t_{j+1} = t_j + s_j, s_j = max(mu f_j, voxel)
        const float gsj = GT + (j == k - 1 ? g_s : 0.f);
        gf = (seg_f[j - j0] * mu > step ? mu * gsj : 0.f) + (j == k - 1 ? g_a : 0.f);
      }
      GT += gf * sample_adjoint(P, V, memo, seg_p[j - j0], direction, gf, grad);
    }
  }
  if (k == 0)  // the opening interpolation was the secant's other end
    (void)interp_adjoint(P, V, memo, p0, direction, g_a, grad);
  return 1;
}

// Adjoint of volume_grad at pos: scatters the 32 taps' share of gG (dE/dG)
// and returns dE/d pos through the trilinear weights.
__device__ F3 grad_adjoint(const Pool& P, const Volume& V, F3 pos_m, F3 gG,
                           float* __restrict__ grad) {
  const float inv = V.size / V.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const F3 fl = floor3(pos);
  const I3 base = to_i3(fl);
  const F3 f = mk3(pos.x - fl.x, pos.y - fl.y, pos.z - fl.z);
  const int s1 = V.size - 1;
  const int cx[4] = {imx(base.x - 1, 0), imx(base.x, 0), imn(base.x + 1, s1), imn(base.x + 2, s1)};
  const int cy[4] = {imx(base.y - 1, 0), imx(base.y, 0), imn(base.y + 1, s1), imn(base.y + 2, s1)};
  const int cz[4] = {imx(base.z - 1, 0), imx(base.z, 0), imn(base.z + 1, s1), imn(base.z + 2, s1)};
  const float sc = V.dim / V.size * 0.5f;
  const F3 gr = gG * sc;  // dE / d(gr) before the scale
  auto slot = [&](int a, int b, int c) { return block_slot(V, cx[a], cy[b], cz[c]); };
  auto val = [&](int a, int b, int c) {
    const int sl = slot(a, b, c);
    return sl < 0 ? 1.f : __ldg(P.tsdf + (size_t)sl * 512 + voxel_index(cx[a], cy[b], cz[c]));
  };
  auto add = [&](int a, int b, int c, float g) {
    const int sl = slot(a, b, c);
    if (sl >= 0 && g != 0.f) atomicAdd(grad + (size_t)sl * 512 + voxel_index(cx[a], cy[b], cz[c]), g);
  };
  const float wx[2] = {1.f - f.x, f.x}, wy[2] = {1.f - f.y, f.y}, wz[2] = {1.f - f.z, f.z};
  F3 gf = mk3(0.f);  // dE/d(fractional position)
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        const float w = wx[a] * wy[b] * wz[c];
        const float sx = a ? 1.f : -1.f, sy = b ? 1.f : -1.f, sz = c ? 1.f : -1.f;
        const float dx = val(2 + a, 1 + b, 1 + c) - val(a, 1 + b, 1 + c);
        const float dy = val(1 + a, 2 + b, 1 + c) - val(1 + a, b, 1 + c);
        const float dz = val(1 + a, 1 + b, 2 + c) - val(1 + a, 1 + b, c);
        add(2 + a, 1 + b, 1 + c, gr.x * w); add(a, 1 + b, 1 + c, -gr.x * w);
        add(1 + a, 2 + b, 1 + c, gr.y * w); add(1 + a, b, 1 + c, -gr.y * w);
        add(1 + a, 1 + b, 2 + c, gr.z * w); add(1 + a, 1 + b, c, -gr.z * w);
        const float s = gr.x * dx + gr.y * dy + gr.z * dz;
        gf.x += s * sx * wy[b] * wz[c];
        gf.y += s * sy * wx[a] * wz[c];
        gf.z += s * sz * wx[a] * wy[b];
      }
  return gf * inv;
}

// One thread per model pixel; pixels whose map adjoints are zero return.
__global__ void __launch_bounds__(128)
raycast_adjoint_kernel(Pool pool, const Volume* __restrict__ vols,
                       const InstFrame* __restrict__ frames, IdList ids, RayArgs a,
                       const double* __restrict__ gV, const double* __restrict__ gN,
                       float* __restrict__ grad, int* __restrict__ status) {
  const int x = blockIdx.x * 16 + (threadIdx.x & 15);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
  const F3 gv = mk3((float)gV[3 * p], (float)gV[3 * p + 1], (float)gV[3 * p + 2]);
  const F3 gn = mk3((float)gN[3 * p], (float)gN[3 * p + 1], (float)gN[3 * p + 2]);
  if (gv.x == 0.f && gv.y == 0.f && gv.z == 0.f && gn.x == 0.f && gn.y == 0.f && gn.z == 0.f)
    return;
  __shared__ int s_slot[8 * 128];
  // replay the composite (raycast_objects_kernel) to find the winner
  float nearest = 1.0e3f;
  double high_fg = 0.f;
  int win = -1;
  F4 whit{0, 0, 0, 0};
  float wnfar = 0.f, wtmin = 0.f;
  F3 wdir = mk3(0.f);
  const M4 view = frames[ids.v[0]].view;
  const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
  for (int o = 0; o < ids.n; ++o) {
    const int i = ids.v[o];
    const Volume& V = vols[i];
    const InstFrame& F = frames[i];
    const float step = V.dim / V.size;
    const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
    const float nfar = fmn(nearest, a.farPlane);
    const float t_min = ray_first_block(V, F.o_origin, o_dir, a.nearPlane, nfar, a.epsilon, status);
    const F4 hit = t_min > 0.f
                       ? raycast_volume(pool, V, F.o_origin, o_dir,
                                        t_min * V.dim / (unsigned)V.size, nfar, a.mu, step,
                                        step * 8)
                       : F4{0, 0, 0, 0};
    const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
    if (hd > nearest) continue;
    const double fg = volume_interp(pool, V, mk3(hit.x, hit.y, hit.z), 1);
    if (fg <= 0.5f) continue;
    if (hd == nearest) {
      if (!(fg > high_fg)) continue;
    } else if (hd < nearest) {
      nearest = hd;
    } else {
      continue;
    }
    high_fg = fg;
    win = i; whit = hit; wnfar = nfar; wtmin = t_min; wdir = o_dir;
  }
  if (win < 0) return;
  const Volume& V = vols[win];
  const InstFrame& F = frames[win];
  const F3 X = mk3(whit.x, whit.y, whit.z);
  const F3 vm = xform(F.T_w_o, X);
  const F3 mv = a.vertex[p];
  if (vm.x != mv.x || vm.y != mv.y || vm.z != mv.z) {  // the replay must be exact
    atomicOr(status, ST_ADJOINT);
    return;
  }
  F3 gX = rotate_t(gv, F.T_w_o);  // dE/dX from the vertex
  if (gn.x != 0.f || gn.y != 0.f || gn.z != 0.f) {
    const F3 G = volume_grad(pool, V, X, s_slot + threadIdx.x, 128);
    const float gl = length(G);
    if (gl > 0.f) {
      const F3 n = normalize(rotate(F.T_w_o, G));
      const F3 gRG = (gn - dot(n, gn) * n) * (1.f / gl);
      gX = gX + grad_adjoint(pool, V, X, rotate_t(gRG, F.T_w_o), grad);
    }
  }
  if (whit.w == 0.f) return;  // a miss claimed by the corner's foreground: no march
  const float step = V.dim / V.size;
  F3 rep;
  const int r = march_adjoint(pool, V, F.o_origin, wdir, wtmin * V.dim / (unsigned)V.size,
                              wnfar, a.mu, step, step * 8, dot(wdir, gX), grad, &rep);
  if (r < 0 || (r == 1 && (rep.x != X.x || rep.y != X.y || rep.z != X.z)))
    atomicOr(status, ST_ADJOINT);
}

int stage_raycast_adjoint(Context* ctx, const IdList& ids, const double* gV, const double* gN,
                          float* d_grad) {
  if (ids.n == 0) return MF_OK;
  const mf_config& c = ctx->cfg;
  RayArgs a{ctx->d_vertex, ctx->d_normal, ctx->d_label, ctx->W, ctx->H,
            c.near_plane, c.far_plane, c.mu, ctx->ray_epsilon};
  dim3 grid((ctx->W + 15) / 16, (ctx->H + 7) / 8);
  raycast_adjoint_kernel<<<grid, 128, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames,
                                                        ids, a, gV, gN, d_grad, ctx->d_status);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// ------------------------------------------------------------------------
// The shaded volume render (headless).
struct RenderArgs {
  Pool pool;
  const Volume* vols;
  const InstFrame* frames;   // T_w_o, inverse(T_w_o), label of every instance
  IdList ids;                // instances in list order
  int W, H;
  M4 view;                   // T_w_c * inverse(K) of the render pose
  F3 w_origin;               // get_translation(T_w_c)
  float nearPlane, farPlane, mu, largestep, epsilon;
  F3 ambient;
  int render_color, do_raycast;
  const uchar4* colors;      // label colours
  int n_colors;
  const F3* vertex; const F3* normal; const int* label;  // maps for do_raycast == 0
  uchar4* out;
  int* status;
};

// renderVolume_many_Kernel, rendering.cpp:489-646.  With do_raycast the
// composite hit is found again with this function's own rules (the tie and
// the zero-gradient cases differ from raycastObjectList); otherwise the maps
// of the last raycast are shaded.
__global__ void __launch_bounds__(128) render_volume_kernel(RenderArgs a) {
  const int x = blockIdx.x * 16 + (threadIdx.x & 15);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
  if (x >= a.W || y >= a.H) return;
  const int p = x + y * a.W;
  __shared__ int s_slot[8 * 128];
  F3 w_hit = mk3(0.f), w_norm = mk3(0.f);
  int w_label = 0;
  if (a.do_raycast) {
    float nearest = 1.0e10f;
    double high_fg = 0.f;
    int miss = 0;
    const F3 w_dir = rotate(a.view, mk3((float)x, (float)y, 1.f));
    for (int o = 0; o < a.ids.n; ++o) {
      const int i = a.ids.v[o];
      const Volume& V = a.vols[i];
      const InstFrame& F = a.frames[i];
      const float step = V.dim / V.size;
      const F3 o_origin = xform(F.inv_T_w_o, a.w_origin);
      const F3 o_dir = normalize(rotate(F.inv_T_w_o, w_dir));
      const float nfar = fmn(nearest, a.farPlane);
      const float t_min = ray_first_block(V, o_origin, o_dir, a.nearPlane, nfar, a.epsilon,
                                          a.status);
      const F4 hit = t_min > 0.f
                         ? raycast_volume(a.pool, V, o_origin, o_dir,
                                          t_min * V.dim / (unsigned)V.size, nfar, a.mu, step,
                                          a.largestep)
                         : F4{0, 0, 0, 0};
      const float hd = F.label == 0 ? hit.w + 0.05f : hit.w;
      if (hd > nearest) { miss++; continue; }
      const double fg = volume_interp(a.pool, V, mk3(hit.x, hit.y, hit.z), 1);
      if (fg <= 0.5f) { miss++; continue; }
      if (hd == nearest) {
        if (fg > high_fg) high_fg = fg;
        else { miss++; continue; }
      }
      if (hit.w > 0) {
        nearest = hd;
        const F3 o_hit = mk3(hit.x, hit.y, hit.z);
        const F3 g = volume_grad(a.pool, V, o_hit, s_slot + threadIdx.x, 128);
        if (length(g) > 0) {
          w_norm = rotate(F.T_w_o, g);
          w_hit = xform(F.T_w_o, o_hit);
          w_label = F.label;
        }
      } else {
        miss++;
      }
    }
    if (miss == a.ids.n) {
      a.out[p] = make_uchar4(0, 0, 0, 0);
      return;
    }
  } else {
    w_hit = a.vertex[p];
    w_norm = a.normal[p];
    w_label = a.label[p];
  }
  F3 col = mk3(0.f);
  for (int o = 0; o < a.ids.n; ++o) {
    const int i = a.ids.v[o];
    const InstFrame& F = a.frames[i];
    if (w_label != F.label) continue;
    const F3 o_hit = xform(F.inv_T_w_o, w_hit);
    const F3 diff = normalize(a.w_origin - w_hit);
    const float dir = fmx(dot(normalize(w_norm), diff), 0.f);
    F3 rgb;
    if (a.render_color) {
      const Volume& V = a.vols[i];
      rgb = mk3(volume_interp(a.pool, V, o_hit, 2), volume_interp(a.pool, V, o_hit, 3),
                volume_interp(a.pool, V, o_hit, 4));
    } else if (w_label == 0) {
      rgb = mk3(1.f);
    } else {
      const uchar4 c = (w_label >= 0 && w_label < a.n_colors) ? a.colors[w_label]
                                                               : make_uchar4(0, 0, 0, 0);
      rgb = mk3((float)c.x, (float)c.y, (float)c.z);
      rgb = mk3(rgb.x / 255, rgb.y / 255, rgb.z / 255);
    }
    // clamp(make_float3(dir) * rgb + ambient, 0, 1) * 255; the background's
    // label colour path has no product (make_float3(dir) + ambient)
    const F3 lit = (a.render_color || w_label != 0)
                       ? mk3(dir * rgb.x, dir * rgb.y, dir * rgb.z)
                       : mk3(dir);
    col = mk3(fmx(0.f, fmn(lit.x + a.ambient.x, 1.f)), fmx(0.f, fmn(lit.y + a.ambient.y, 1.f)),
              fmx(0.f, fmn(lit.z + a.ambient.z, 1.f)));
    col = col * 255.f;
  }
  a.out[p] = u4(col.x, col.y, col.z, 0.f);
}

int render_volume(Context* ctx, const float* T_w_c, int render_color, float largestep,
                  const float* ambient, const uint8_t* colors, int n_colors, uint8_t* out) {
  const mf_config& c = ctx->cfg;
  const size_t bytes = (size_t)ctx->W * ctx->H * 4;
  void* target = nullptr;
  if (int rc = render_target(ctx, out, bytes, &target)) return rc;
  IdList all;
  all.n = (int)ctx->inst.size();
  for (int i = 0; i < all.n; ++i) all.v[i] = i;
  // the instances' T_w_o and inverse; the camera frame of the current pose
  if (int rc = stage_prepare(ctx, all)) return rc;
  float Tc[16];
  if (T_w_c) {
    std::memcpy(Tc, T_w_c, sizeof(Tc));
  } else {
    MF_CUDA(cudaMemcpyAsync(Tc, ctx->d_Twc, 64, cudaMemcpyDeviceToHost, ctx->stream));
    MF_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  void* d_colors = nullptr;
  if (n_colors > 0) {
    if (int rc = render_stage_small(ctx, colors, 4 * (size_t)n_colors, &d_colors)) return rc;
  }
  const M4 T = load_m4(Tc);
  RenderArgs a;
  a.pool = ctx->pool;
  a.vols = ctx->d_vols;
  a.frames = ctx->d_frames;
  a.ids = all;
  a.W = ctx->W;
  a.H = ctx->H;
  a.view = mul(T, inverse_camera_matrix(F4{c.k[0], c.k[1], c.k[2], c.k[3]}));
  a.w_origin = get_translation(T);
  // Kfusion::renderVolume passes farPlane * 2 (kfusion.cpp:1303-1304)
  a.nearPlane = c.near_plane;
  a.farPlane = c.far_plane * 2.0f;
  a.mu = c.mu;
  a.largestep = largestep;
  a.epsilon = ctx->ray_epsilon;
  a.ambient = ambient ? mk3(ambient[0], ambient[1], ambient[2]) : mk3(0.1f);
  a.render_color = render_color;
  a.do_raycast = T_w_c != nullptr;
  a.colors = (const uchar4*)d_colors;
  a.n_colors = n_colors;
  a.vertex = ctx->d_vertex;
  a.normal = ctx->d_normal;
  a.label = ctx->d_label;
  a.out = (uchar4*)target;
  a.status = ctx->d_status;
  dim3 grid((ctx->W + 15) / 16, (ctx->H + 7) / 8);
  render_volume_kernel<<<grid, 128, 0, ctx->stream>>>(a);
  return render_finish(ctx, out, target, bytes);
}

}  // namespace mf

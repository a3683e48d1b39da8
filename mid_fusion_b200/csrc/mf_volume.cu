// Voxel-block allocation and projective TSDF integration on the device.
//
// Allocation is sort-free: each octree level is a dense table indexed by the
// Morton code of its octants, so the reference's sort + unique_multiscale +
// level-by-level updateLevel (lib/octree.hpp:761-863) becomes (1) every ray
// sample of an unallocated block adds to that table entry's request count and
// (2) one pass over the block table creates the requested blocks and flags their
// ancestors.  The resulting key sets and topology equal the reference's; the
// request counts also reproduce the reference's allocation-list quirks (see
// alloc_commit_kernel).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include "mf_internal.h"
#include "mf_sample.cuh"

namespace mf {

// ------------------------------------------------------------------ prepare
// Per-instance matrices every stage needs, computed from the device-resident
// camera and volume poses with the reference's float operation order.
__global__ void prepare_kernel(const float* __restrict__ Twc_p, const float* __restrict__ Two_p,
                               const Volume* __restrict__ vols, InstFrame* __restrict__ out,
                               F4 k, float mu, IdList ids,
                               const unsigned long long* __restrict__ reserved,
                               const int* __restrict__ labels) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ids.n) return;
  const int i = ids.v[t];
  const M4 T_w_c = load_m4(Twc_p), T_w_o = load_m4(Two_p + 16 * i);
  const Volume V = vols[i];
  InstFrame f;
  f.T_w_o = T_w_o;
  f.inv_T_w_o = inverse(T_w_o);
  const M4 K = camera_matrix(k);
  f.kPose = mul(T_w_c, inverse(K));
  f.o_cam = xform(f.inv_T_w_o, get_translation(T_w_c));
  const float vs = V.dim / V.size;
  f.inv_voxel = 1 / vs;
  f.band = 2 * mu;
  f.num_steps = (int)ceilf(f.band * f.inv_voxel);
  f.reserved = reserved[i];
  f.Tcw = mul(inverse(T_w_c), T_w_o);
  f.KTcw = mul(K, f.Tcw);
  f.delta = rotate(f.Tcw, mk3(vs, 0, 0));
  f.cam_delta = rotate(K, f.delta);
  const M4 view = mul(T_w_c, inverse_camera_matrix(k));
  f.view = view;
  f.o_origin = xform(f.inv_T_w_o, get_translation(view));
  f.label = labels[i];
  out[i] = f;
}

// ------------------------------------------------------------------ allocation
// buildVolumeAllocationList, apps/kfusion/src/cpp/kfusion/alloc_impl.hpp:121-191.
// One thread per ray-casting (pixel, instance).  A sample in an allocated
// block marks it active; a sample in an unallocated block adds to that block's
// request count (runs of equal blocks along a ray are added at once).  The
// emission order of the single-threaded reference (row, column, step) of the
// thread's last emitted sample is folded into last_emit with atomicMax.
__global__ void __launch_bounds__(256)
alloc_mark_kernel(const float* __restrict__ depth, const float* __restrict__ masks, int W,
                  int H, const Volume* __restrict__ vols, const InstFrame* __restrict__ frames,
                  IdList ids, Pool pool) {
  const int inst = ids.v[blockIdx.y];
  const Volume& V = vols[inst];
  const InstFrame& F = frames[inst];
  unsigned count = 0, last_order = 0, last_idx = 0;
  // The CTA's pixels that cast a ray (depth != 0, mask >= 0) are packed, in
  // pixel order, onto its first threads: an object's pixels are sparse, and a
  // ray of 100 samples on one lane of a warp idled the other 31.  Every result
  // below is a sum, a maximum or an idempotent flag, so which thread handles
  // which pixel does not change it.
  __shared__ int s_pix[256];
  __shared__ float s_d[256];
  __shared__ int s_wn[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const float dq = q < W * H ? depth[q] : 0.f;
    const bool ray = dq != 0 && !(masks[(size_t)inst * W * H + (q < W * H ? q : 0)] < 0);
    const unsigned b = __ballot_sync(0xffffffffu, ray);
    if (lane == 0) s_wn[warp] = __popc(b);
    __syncthreads();
    int base = 0;
    for (int w = 0; w < warp; ++w) base += s_wn[w];
    if (ray) {
      const int slot = base + __popc(b & ((1u << lane) - 1u));
      s_pix[slot] = q;
      s_d[slot] = dq;
    }
    __syncthreads();
  }
  int n_rays = 0;
  for (int w = 0; w < 8; ++w) n_rays += s_wn[w];
  const bool has_ray = (int)threadIdx.x < n_rays;
  const int p = has_ray ? s_pix[threadIdx.x] : 0;
  const float d = has_ray ? s_d[threadIdx.x] : 0.f;
  // no early return: every lane reaches the warp reduction below
  if (has_ray) {
    const unsigned x = p % W, y = p / W;
    const float size_f = (float)(unsigned)V.size;
    const F3 w_vertex = xform(F.kPose, mk3((x + 0.5f) * d, (y + 0.5f) * d, d));
    const F3 o_vertex = xform(F.inv_T_w_o, w_vertex);
    const F3 direction = normalize(F.o_cam - o_vertex);
    const F3 origin = o_vertex - (F.band * 0.5f) * direction;
    const F3 step = (direction * F.band) / (float)F.num_steps;
    F3 pos = origin;
    int run_idx = -1, run_len = 0;
    int cur_key = -1, cur_slot = -1;
    uint32_t cur_bidx = 0;
    for (int i = 0; i < F.num_steps; i++) {
      // the reference floors pos / voxel and tests 0 <= floor < size; with an
      // integer size that holds exactly when 0 <= pos / voxel < size, and there
      // the truncating conversion is the floor (one conversion per axis
      // instead of a floor and a conversion; NaN fails the test either way)
      const float fx = pos.x * F.inv_voxel, fy = pos.y * F.inv_voxel, fz = pos.z * F.inv_voxel;
      if (fx < size_f && fy < size_f && fz < size_f && fx >= 0 && fy >= 0 && fz >= 0) {
        const I3 v{(int)fx, (int)fy, (int)fz};
        const int key = (v.x >> 3) | ((v.y >> 3) << 10) | ((v.z >> 3) << 20);
        if (key != cur_key) {  // a new block along the ray: look it up once
          cur_key = key;
          cur_bidx = (uint32_t)morton3(v.x >> 3, v.y >> 3, v.z >> 3);
          cur_slot = V.block_tab[cur_bidx];
          if (cur_slot >= 0) pool.active[cur_slot] = 1;
        }
        if (cur_slot < 0) {
          if ((int)cur_bidx == run_idx) {
            ++run_len;
          } else {
            if (run_len) atomicAdd(&V.req[run_idx], (uint32_t)run_len);
            run_idx = (int)cur_bidx;
            run_len = 1;
          }
          ++count;
          last_order = (unsigned)p * (unsigned)F.num_steps + (unsigned)i;
          last_idx = cur_bidx;
        }
      }
      pos = pos + step;
    }
    if (run_len) atomicAdd(&V.req[run_idx], (uint32_t)run_len);
  }
  // one emission-count and one last-emission atomic per warp
  unsigned long long last = count ? (((unsigned long long)last_order << 32) | last_idx) : 0ULL;
  unsigned long long tot = count;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    tot += __shfl_xor_sync(0xffffffffu, tot, o);
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, last, o);
    last = other > last ? other : last;
  }
  if ((threadIdx.x & 31) == 0 && tot) {
    atomicAdd(V.emit_total, tot);
    atomicMax(V.last_emit, last);
  }
}

// Grows the instance's box of allocated blocks (read by the raycast to skip
// rays that cannot meet a block); block 0 is left out, the raycast tests it on
// its own.
__device__ __forceinline__ void note_block(const Volume& V, long long bidx, int cx, int cy,
                                           int cz) {
  if (bidx == 0) return;
  atomicMin(&V.bbox[0], cx); atomicMin(&V.bbox[1], cy); atomicMin(&V.bbox[2], cz);
  atomicMax(&V.bbox[3], cx); atomicMax(&V.bbox[4], cy); atomicMax(&V.bbox[5], cz);
}

// Octree::alloc_update + updateLevel, lib/octree.hpp:761-786, :826-863.
// One thread per (block-table entry, instance).  Reference semantics kept:
//  - the list's slot 0 is never written (alloc_impl.hpp:175, pre-increment) and
//    stays 0, and unique_multiscale keeps keys[0] unconditionally
//    (lib/algorithms/unique.hpp:76-79), so the path to block (0,0,0) is
//    allocated by every call;
//  - [0, count) is passed on while the keys sit in slots 1..count, so the last
//    emitted key is not allocated unless another sample requested its block.
__global__ void __launch_bounds__(256)
alloc_commit_kernel(const Volume* __restrict__ vols, const InstFrame* __restrict__ frames,
                    IdList ids, Pool pool, int* __restrict__ status) {
  const int inst = ids.v[blockIdx.y];
  const Volume& V = vols[inst];
  const long long n_tab = 1LL << (3 * V.block_level);
  const long long bidx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (bidx >= n_tab) return;
  const uint32_t r = V.req[bidx];
  if (r == 0 && bidx != 0) return;
  const unsigned long long total = *V.emit_total;
  const unsigned long long last = *V.last_emit;
  bool need = (r > 0) || (bidx == 0);
  if (total >= frames[inst].reserved) {
    if (bidx == 0) atomicOr(status, ST_ALLOC_OVERFLOW);
  } else if (r == 1 && bidx != 0 && (long long)(last & 0xffffffffULL) == bidx) {
    need = false;  // the dropped last slot was this block's only request
  }
  if (need && V.block_tab[bidx] < 0) {
    const int slot = atomicAdd(pool.count, 1);
    if (slot >= pool.cap) {
      atomicOr(status, ST_POOL_FULL);
    } else {
      const int cx = (int)gather3((uint64_t)bidx) << 3;
      const int cy = (int)gather3((uint64_t)bidx >> 1) << 3;
      const int cz = (int)gather3((uint64_t)bidx >> 2) << 3;
      pool.meta[slot] = make_int4(cx, cy, cz, inst);
      pool.active[slot] = 1;
      V.block_tab[bidx] = slot;
      note_block(V, bidx, cx, cy, cz);
      for (int l = V.block_level - 1; l >= 1; --l)
        V.node_tab[V.node_off[l] + (bidx >> (3 * (V.block_level - l)))] = 1;
    }
  }
  if (r) V.req[bidx] = 0;
}

// Octree::alloc_update on caller-supplied keys: (code, level) pairs already
// reduced on the host to "create the octant at this level and its ancestors".
__global__ void alloc_keys_kernel(const Volume* __restrict__ vols, int inst,
                                  const unsigned long long* __restrict__ codes,
                                  const int* __restrict__ levels, int n, Pool pool,
                                  int* __restrict__ status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const Volume& V = vols[inst];
  const int L = levels[t];
  const unsigned long long code = codes[t];
  for (int l = 1; l <= L && l < V.block_level; ++l)
    V.node_tab[V.node_off[l] + (long long)(code >> (3 * (V.max_level - l)))] = 1;
  if (L == V.block_level) {
    const long long bidx = (long long)(code >> (3 * (V.max_level - V.block_level)));
    if (atomicCAS(&V.block_tab[bidx], -1, -2) == -1) {
      const int slot = atomicAdd(pool.count, 1);
      if (slot >= pool.cap) {
        atomicOr(status, ST_POOL_FULL);
        V.block_tab[bidx] = -1;
        return;
      }
      const int cx = (int)gather3(bidx) << 3, cy = (int)gather3(bidx >> 1) << 3,
                cz = (int)gather3(bidx >> 2) << 3;
      pool.meta[slot] = make_int4(cx, cy, cz, inst);
      pool.active[slot] = 1;
      V.block_tab[bidx] = slot;
      note_block(V, bidx, cx, cy, cz);
    }
  }
}

// ------------------------------------------------------------------ integration
// projective_functor::build_active_list, lib/functors/projective_functor.hpp:54-71
// with algorithms::filter (lib/algorithms/filter.hpp:42-61, predicates ORed):
// a block is visited when it is active or its corner projects into the frame.
__global__ void __launch_bounds__(256)
visit_list_kernel(Pool pool, const Volume* __restrict__ vols,
                  const InstFrame* __restrict__ frames, uint32_t inst_mask, int W, int H,
                  int* __restrict__ visit, int* __restrict__ visit_count) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  bool take = false;
  if (slot < *pool.count) {
    const int4 m = pool.meta[slot];
    if ((inst_mask >> m.w) & 1u) {
      if (pool.active[slot]) {
        take = true;
      } else {
        const Volume& V = vols[m.w];
        const float vs = V.dim / V.size;
        const F3 bc = mk3((float)m.x, (float)m.y, (float)m.z) * vs;
        const F3 vc = xform(frames[m.w].KTcw, bc);
        const int px = (int)(vc.x / vc.z), py = (int)(vc.y / vc.z);
        take = px >= 0 && px < W && py >= 0 && py < H;
      }
    }
  }
  // warp-aggregated append
  const unsigned ballot = __ballot_sync(0xffffffffu, take);
  if (!ballot) return;
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == __ffs(ballot) - 1) base = atomicAdd(visit_count, __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, __ffs(ballot) - 1);
  if (take) visit[base + __popc(ballot & ((1u << lane) - 1))] = slot;
}

struct SdfArgs {
  const float* depth; const F3* rgb; const float* masks;
  int W, H; float mu; float maxweight;
};

// sdf_update::operator(), apps/kfusion/src/cpp/kfusion/mapping_impl.hpp:17-49,
// on one voxel held as separate field references.
template <typename FT, typename FW, typename FC, typename FG, typename FWI>
__device__ __forceinline__ void sdf_update(const SdfArgs& a, const float* mask, F3 pos,
                                           float px_f, float py_f, FT& tsdf, FW& wt,
                                           float* r, float* g, float* b, FC& c, FG& fg,
                                           FWI& w) {
  const unsigned px = (unsigned)px_f, py = (unsigned)py_f;
  const float depthSample = a.depth[px + a.W * py];
  const float m = mask[px + a.W * py];
  if (depthSample <= 0 || m < 0) return;
  const float diff =
      (depthSample - pos.z) * sqrtf(1 + sq(pos.x / pos.z) + sq(pos.y / pos.z));
  if (diff > -a.mu) {
    const float sdf = fmn(1.f, diff / a.mu);
    float x = tsdf, y = wt;
    x = clampf((y * x + sdf) / (y + 1), -1.f, 1.f);
    y = fmn(y + 1, a.maxweight);
    tsdf = x; wt = y;
    const F3 rgb = a.rgb[px + a.W * py];
    const int cc = c;
    *r = (rgb.x + *r * cc) / (cc + 1);
    *g = (rgb.y + *g * cc) / (cc + 1);
    *b = (rgb.z + *b * cc) / (cc + 1);
    c = cc + 1;
    const int ww = w;
    fg = ((double)m + fg * ww) / (ww + 1);
    w = ww + 1;
  }
}

// Hint: bring the 144 128-byte lines holding the eight voxel fields of pool
// slot `slot` (7 x 2 KB of 4-byte fields, 4 KB of fg) into L2, one line per
// thread of the first 144.
__device__ __forceinline__ void prefetch_block_fields(const Pool& pool, int slot) {
  const int t = threadIdx.x;
  if (t >= 144) return;
  const size_t o = (size_t)slot * 512;
  const int fi = t >> 4;
  const void* base = fi == 0   ? (const void*)(pool.tsdf + o)
                     : fi == 1 ? (const void*)(pool.wt + o)
                     : fi == 2 ? (const void*)(pool.r + o)
                     : fi == 3 ? (const void*)(pool.g + o)
                     : fi == 4 ? (const void*)(pool.b + o)
                     : fi == 5 ? (const void*)(pool.c + o)
                     : fi == 6 ? (const void*)(pool.w + o)
                               : (const void*)(pool.fg + o);
  const char* p = (const char*)base + (fi < 7 ? (t & 15) : t - 112) * 128;
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// projective_functor::update_block, lib/functors/projective_functor.hpp:73-111.
// Persistent CTAs of 512 threads, one visited block at a time, one voxel per
// thread: every field plane is read and written coalesced, and only for voxels
// that pass the update test.  The next block's slot and corner are loaded
// during the current one, and the instances' constants come from shared
// memory, so a block's dependent chain is the pixel fetch and the voxel
// read-modify-write.
// MINB 512-thread CTAs are resident per SM (the register bound) and the grid
// is MINB CTAs per SM; with PF the CTA prefetches the next block's voxel
// fields into L2 while it works on the current one.  Every variant updates
// each voxel alike (int_variants).
template <int MINB, bool PF>
__global__ void __launch_bounds__(512, MINB)
integrate_blocks_kernel(Pool pool, const Volume* __restrict__ vols,
                        const InstFrame* __restrict__ frames, SdfArgs args, F4 k,
                        const int* __restrict__ visit, const int* __restrict__ visit_count) {
  const int n = *visit_count;
  const M4 K = camera_matrix(k);
  const float wlim = args.W - 1.5f, hlim = args.H - 1.5f;
  const int W = args.W;
  const float mu = args.mu, maxweight = args.maxweight;
  // the instances' constants, staged once per CTA (the tables hold
  // MAX_INSTANCES entries)
  __shared__ M4 s_Tcw[MAX_INSTANCES];
  __shared__ F3 s_delta[MAX_INSTANCES], s_cdelta[MAX_INSTANCES];
  __shared__ float s_vs[MAX_INSTANCES];
  for (int i = threadIdx.x; i < MAX_INSTANCES; i += blockDim.x) {
    s_Tcw[i] = frames[i].Tcw;
    s_delta[i] = frames[i].delta;
    s_cdelta[i] = frames[i].cam_delta;
    s_vs[i] = vols[i].dim / vols[i].size;
  }
  __syncthreads();
  // one voxel per thread; the next block's corner is fetched one block ahead
  // and (PF) the slot after it two blocks ahead
  const int v = threadIdx.x;
  const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
  int item = blockIdx.x;
  int next_slot = item < n ? visit[item] : 0;
  int4 next_m = item < n ? pool.meta[next_slot] : make_int4(0, 0, 0, 0);
  int after_slot = 0;
  if (PF && item + (int)gridDim.x < n) after_slot = visit[item + gridDim.x];
  for (; item < n; item += gridDim.x) {
    const int slot = next_slot;
    const int4 m = next_m;
    if (item + gridDim.x < n) {
      if (PF) {
        prefetch_block_fields(pool, after_slot);
        next_slot = after_slot;
        if (item + 2 * gridDim.x < n) after_slot = visit[item + 2 * gridDim.x];
      } else {
        next_slot = visit[item + gridDim.x];
      }
      next_m = pool.meta[next_slot];
    }
    const float vs = s_vs[m.w];
    const float* mask = args.masks + (size_t)m.w * args.W * args.H;
    // voxel -> pixel
    const F3 start = xform(s_Tcw[m.w], mk3(m.x * vs, (m.y + y) * vs, (m.z + z) * vs));
    const F3 camerastart = xform(K, start);
    const F3 cv = camerastart + ((float)x * s_cdelta[m.w]);
    const F3 pos = start + ((float)x * s_delta[m.w]);
    bool vis = false;
    int pix = 0;
    if (pos.z >= 0.0001f) {
      const float inv = 1.f / cv.z;
      const float pxf = cv.x * inv + 0.5f, pyf = cv.y * inv + 0.5f;
      if (!(pxf < 0.5f || pxf > wlim || pyf < 0.5f || pyf > hlim)) {
        vis = true;
        pix = (int)((unsigned)pxf + W * (unsigned)pyf);
      }
    }
    // depth / mask at the pixel, the update test of sdf_update
    const float depthS = vis ? __ldg(args.depth + pix) : 0.f;
    const float mval = vis ? __ldg(mask + pix) : -1.f;
    bool upd = false;
    float sdf = 0.f;
    if (vis && depthS > 0 && mval >= 0) {
      const float diff = (depthS - pos.z) * sqrtf(1 + sq(pos.x / pos.z) + sq(pos.y / pos.z));
      if (diff > -mu) {
        upd = true;
        sdf = fmn(1.f, diff / mu);
      }
    }
    // read-modify-write of the voxel
    if (upd) {
      const size_t o = (size_t)slot * 512 + v;
      const float t = pool.tsdf[o], wt = pool.wt[o], r = pool.r[o], g = pool.g[o],
                  b = pool.b[o];
      const int c = pool.c[o], w = pool.w[o];
      const double fg = pool.fg[o];
      const F3 rgb = args.rgb[pix];
      // sdf_update, apps/kfusion/src/cpp/kfusion/mapping_impl.hpp:26-46
      pool.tsdf[o] = clampf((wt * t + sdf) / (wt + 1), -1.f, 1.f);
      pool.wt[o] = fmn(wt + 1, maxweight);
      pool.r[o] = (rgb.x + r * c) / (c + 1);
      pool.g[o] = (rgb.y + g * c) / (c + 1);
      pool.b[o] = (rgb.z + b * c) / (c + 1);
      pool.c[o] = c + 1;
      pool.fg[o] = ((double)mval + fg * w) / (w + 1);
      pool.w[o] = w + 1;
    }
    const int any = __syncthreads_or(vis);
    if (threadIdx.x == 0) pool.active[slot] = any ? 1 : 0;
  }
}

// Work counts of update_block for the roofline: voxels whose pixel is read
// (visible: depth and mask fetched) and voxels updated (fields read + written).
__global__ void __launch_bounds__(256)
integrate_count_kernel(Pool pool, const Volume* __restrict__ vols,
                       const InstFrame* __restrict__ frames, SdfArgs args, F4 k,
                       const int* __restrict__ visit, const int* __restrict__ visit_count,
                       unsigned long long* __restrict__ counts) {
  const int n = *visit_count;
  const M4 K = camera_matrix(k);
  const float wlim = args.W - 1.5f, hlim = args.H - 1.5f;
  unsigned long long nvis = 0, nupd = 0;
  for (int item = blockIdx.x; item < n; item += gridDim.x) {
    const int slot = visit[item];
    const int4 m = pool.meta[slot];
    const Volume& V = vols[m.w];
    const InstFrame& F = frames[m.w];
    const float vs = V.dim / V.size;
    const float* mask = args.masks + (size_t)m.w * args.W * args.H;
    for (int h = 0; h < 2; ++h) {
      const int v = threadIdx.x + h * 256;
      const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
      const F3 start = xform(F.Tcw, mk3(m.x * vs, (m.y + y) * vs, (m.z + z) * vs));
      const F3 cv = xform(K, start) + ((float)x * F.cam_delta);
      const F3 p = start + ((float)x * F.delta);
      if (p.z < 0.0001f) continue;
      const float inv = 1.f / cv.z;
      const float pxf = cv.x * inv + 0.5f, pyf = cv.y * inv + 0.5f;
      if (pxf < 0.5f || pxf > wlim || pyf < 0.5f || pyf > hlim) continue;
      ++nvis;
      const int pix = (int)((unsigned)pxf + args.W * (unsigned)pyf);
      const float d = args.depth[pix];
      if (d <= 0 || mask[pix] < 0) continue;
      const float diff = (d - p.z) * sqrtf(1 + sq(p.x / p.z) + sq(p.y / p.z));
      if (diff > -args.mu) ++nupd;
    }
  }
  atomicAdd(&counts[0], nvis);
  atomicAdd(&counts[1], nupd);
}

// projective_functor::update_node, lib/functors/projective_functor.hpp:113-137,
// over every internal node of the selected instances.  The reference takes the
// node's voxel from unpack_morton(code) with the level bits still in the code,
// and offsets child i by dir * rotate(Tcw, (h, h, h)) element-wise; both kept.
// One thread per (node, child): the eight children update disjoint values, so
// the reference's loop over them runs as eight threads.
__global__ void __launch_bounds__(128)
integrate_nodes_kernel(const Volume* __restrict__ vols, const InstFrame* __restrict__ frames,
                       SdfArgs args, F4 k, IdList ids) {
  const int inst = ids.v[blockIdx.y];
  const Volume& V = vols[inst];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long e = t >> 3;
  const int i = (int)(t & 7);
  if (e >= V.n_nodes || !V.node_tab[e]) return;
  int l = 1;
  while (l + 1 < V.block_level && e >= V.node_off[l + 1]) ++l;
  const unsigned long long mcode = (unsigned long long)(e - V.node_off[l]);
  const unsigned long long code = (mcode << (3 * (V.max_level - l))) | (unsigned long long)l;
  const InstFrame& F = frames[inst];
  const M4 K = camera_matrix(k);
  const float vs = V.dim / V.size;
  const unsigned side = (unsigned)V.size >> l;
  const F3 voxel = mk3((float)(int)gather3(code), (float)(int)gather3(code >> 1),
                       (float)(int)gather3(code >> 2));
  const F3 delta = rotate(F.Tcw, mk3(0.5f * vs * side));
  const F3 delta_c = rotate(K, delta);
  const F3 base_cam = xform(F.Tcw, voxel * vs);
  const F3 basepix = xform(K, base_cam);
  const float* mask = args.masks + (size_t)inst * args.W * args.H;
  const float wlim = args.W - 1.5f, hlim = args.H - 1.5f;
  const F3 dir = mk3((float)((i & 1) > 0), (float)((i & 2) > 0), (float)((i & 4) > 0));
  const F3 vox_cam = base_cam + dir * delta;
  const F3 pix_hom = basepix + dir * delta_c;
  if (vox_cam.z < 0.0001f) return;
  const float inv = 1.f / pix_hom.z;
  const float pxf = pix_hom.x * inv + 0.5f, pyf = pix_hom.y * inv + 0.5f;
  if (pxf < 0.5f || pxf > wlim || pyf < 0.5f || pyf > hlim) return;
  const size_t o = (size_t)e * 8 + i;
  sdf_update(args, mask, vox_cam, pxf, pyf, V.n_tsdf[o], V.n_wt[o], &V.n_r[o], &V.n_g[o],
             &V.n_b[o], V.n_c[o], V.n_fg[o], V.n_w[o]);
}

__global__ void interp_points_kernel(Pool pool, const Volume* __restrict__ vols, int inst,
                                     const float* __restrict__ pos, int n, int field,
                                     float* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  out[t] = volume_interp(pool, vols[inst], mk3(pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]),
                         field);
}

// Gather selected blocks into the reference's 40-byte AoS voxel layout.
__global__ void export_blocks_kernel(Pool pool, const int* __restrict__ slots, int n,
                                     unsigned char* __restrict__ out) {
  const int b = blockIdx.x;
  if (b >= n) return;
  const int slot = slots[b];
  for (int v = threadIdx.x; v < 512; v += blockDim.x) {
    const size_t o = (size_t)slot * 512 + v;
    unsigned char* d = out + ((size_t)b * 512 + v) * 40;
    *(float*)(d + 0) = pool.tsdf[o];
    *(float*)(d + 4) = pool.wt[o];
    *(float*)(d + 8) = pool.r[o];
    *(float*)(d + 12) = pool.g[o];
    *(float*)(d + 16) = pool.b[o];
    *(int*)(d + 20) = pool.c[o];
    *(double*)(d + 24) = pool.fg[o];
    *(int*)(d + 32) = pool.w[o];
    *(int*)(d + 36) = 0;
  }
}

// ------------------------------------------------------------------ host side
static int div_up(long long a, int b) { return (int)((a + b - 1) / b); }

template <typename T>
static cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

__global__ void fill_node_values_kernel(Volume V) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V.n_nodes * 8) return;
  V.n_tsdf[i] = 1.f; V.n_wt[i] = 0.f; V.n_r[i] = 0.f; V.n_g[i] = 0.f; V.n_b[i] = 0.f;
  V.n_c[i] = 0; V.n_fg[i] = 0.0; V.n_w[i] = 0;
}

int volume_create(Context* ctx, Instance& in) {
  Volume& V = in.vol;
  std::memset(&V, 0, sizeof(V));
  V.size = in.size;
  V.dim = in.dim;
  int ml = 0;
  while ((1 << ml) < in.size) ++ml;
  V.max_level = ml;
  V.block_level = ml - 3;
  long long off = 0;
  for (int l = 1; l < V.block_level; ++l) { V.node_off[l] = off; off += 1LL << (3 * l); }
  V.node_off[V.block_level] = off;
  V.n_nodes = off;
  const long long n_tab = 1LL << (3 * V.block_level);
  MF_CUDA(dalloc(&V.block_tab, n_tab));
  MF_CUDA(cudaMemsetAsync(V.block_tab, 0xff, sizeof(int32_t) * n_tab, ctx->stream));
  MF_CUDA(dalloc(&V.req, n_tab));
  MF_CUDA(cudaMemsetAsync(V.req, 0, sizeof(uint32_t) * n_tab, ctx->stream));
  MF_CUDA(dalloc(&V.node_tab, V.n_nodes));
  MF_CUDA(cudaMemsetAsync(V.node_tab, 0, V.n_nodes ? V.n_nodes : 1, ctx->stream));
  const size_t nv = (size_t)V.n_nodes * 8;
  MF_CUDA(dalloc(&V.n_tsdf, nv)); MF_CUDA(dalloc(&V.n_wt, nv));
  MF_CUDA(dalloc(&V.n_r, nv)); MF_CUDA(dalloc(&V.n_g, nv)); MF_CUDA(dalloc(&V.n_b, nv));
  MF_CUDA(dalloc(&V.n_c, nv)); MF_CUDA(dalloc(&V.n_fg, nv)); MF_CUDA(dalloc(&V.n_w, nv));
  MF_CUDA(dalloc(&V.last_emit, 1)); MF_CUDA(dalloc(&V.emit_total, 1));
  MF_CUDA(dalloc(&V.bbox, 6));
  const int empty_box[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  MF_CUDA(cudaMemcpyAsync(V.bbox, empty_box, sizeof(empty_box), cudaMemcpyHostToDevice,
                          ctx->stream));
  if (nv) fill_node_values_kernel<<<div_up(nv, 256), 256, 0, ctx->stream>>>(V);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

void volume_free(Instance& in) {
  Volume& V = in.vol;
  void* ps[] = {V.block_tab, V.req, V.node_tab, V.n_tsdf, V.n_wt, V.n_r, V.n_g, V.n_b,
                V.n_c, V.n_fg, V.n_w, V.last_emit, V.emit_total, V.bbox};
  for (void* p : ps) if (p) cudaFree(p);
  std::memset(&V, 0, sizeof(V));
}


int stage_prepare(Context* ctx, const IdList& ids) {
  if (ids.n == 0) return MF_OK;
  const mf_config& c = ctx->cfg;
  prepare_kernel<<<1, 32, 0, ctx->stream>>>(ctx->d_Twc, ctx->d_Two, ctx->d_vols, ctx->d_frames,
                                             F4{c.k[0], c.k[1], c.k[2], c.k[3]}, c.mu, ids,
                                             ctx->d_reserved, ctx->d_inst_label);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

int stage_alloc(Context* ctx, const IdList& ids) {
  if (ids.n == 0) return MF_OK;
  const int WH = ctx->W * ctx->H;
  int max_tab = 0;
  for (int i = 0; i < ids.n; ++i) {
    const Volume& V = ctx->inst[ids.v[i]].vol;
    MF_CUDA(cudaMemsetAsync(V.last_emit, 0, sizeof(unsigned long long), ctx->stream));
    MF_CUDA(cudaMemsetAsync(V.emit_total, 0, sizeof(unsigned long long), ctx->stream));
    max_tab = std::max(max_tab, 1 << (3 * V.block_level));
  }
  alloc_mark_kernel<<<dim3(div_up(WH, 256), ids.n), 256, 0, ctx->stream>>>(
      ctx->d_depth, ctx->d_masks, ctx->W, ctx->H, ctx->d_vols, ctx->d_frames, ids, ctx->pool);
  MF_CUDA(cudaGetLastError());
  alloc_commit_kernel<<<dim3(div_up(max_tab, 256), ids.n), 256, 0, ctx->stream>>>(
      ctx->d_vols, ctx->d_frames, ids, ctx->pool, ctx->d_status);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// Timing and algorithmic bytes of integrate_blocks_kernel on the current
// frame (re-integrates the frame `reps` times; used after the timed region).
int profile_integrate(Context* ctx, int reps, double* us, double* bytes) {
  const int n = (int)ctx->inst.size();
  IdList all;
  all.n = n;
  for (int i = 0; i < n; ++i) all.v[i] = i;
  const mf_config& c = ctx->cfg;
  if (int rc = stage_prepare(ctx, all)) return rc;
  uint32_t mask = 0;
  for (int i = 0; i < n; ++i) mask |= 1u << i;
  MF_CUDA(cudaMemsetAsync(ctx->d_visit_count, 0, sizeof(int), ctx->stream));
  visit_list_kernel<<<div_up(ctx->pool.cap, 256), 256, 0, ctx->stream>>>(
      ctx->pool, ctx->d_vols, ctx->d_frames, mask, ctx->W, ctx->H, ctx->d_visit,
      ctx->d_visit_count);
  SdfArgs a{ctx->d_depth, ctx->d_rgb, ctx->d_masks, ctx->W, ctx->H, c.mu, (float)c.max_weight};
  const F4 k{c.k[0], c.k[1], c.k[2], c.k[3]};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  unsigned long long* d_cnt = nullptr;
  MF_CUDA(cudaMalloc(&d_cnt, 2 * sizeof(unsigned long long)));
  MF_CUDA(cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), ctx->stream));
  integrate_count_kernel<<<sms * 8, 256, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, ctx->d_frames,
                                                          a, k, ctx->d_visit, ctx->d_visit_count,
                                                          d_cnt);
  unsigned long long cnt[2] = {0, 0};
  int nv = 0;
  MF_CUDA(cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(&nv, ctx->d_visit_count, sizeof(int), cudaMemcpyDeviceToHost,
                          ctx->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx->stream);
  for (int r = 0; r < reps; ++r)
    if (int rc = launch_integrate_blocks(ctx, ctx->pool, ctx->tune.integrate)) return rc;
  cudaEventRecord(e1, ctx->stream);
  MF_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_cnt);
  MF_CUDA(cudaGetLastError());
  *us = 1e3 * ms / reps;
  // per visible voxel: depth + mask (8 B); per updated voxel: the 36-byte field
  // payload read and written and the pixel's rgb (12 B); per block: slot + meta.
  *bytes = 8.0 * cnt[0] + (36.0 + 36.0 + 12.0) * cnt[1] + 20.0 * nv;
  return MF_OK;
}

// Launch-shape candidates of integrate_blocks_kernel; entry 0 is the default.
struct IntVariant {
  int minb;
  bool prefetch;
  void (*fn)(Pool, const Volume*, const InstFrame*, SdfArgs, F4, const int*, const int*);
};
static const IntVariant int_variants[] = {
    {4, false, integrate_blocks_kernel<4, false>}, {3, false, integrate_blocks_kernel<3, false>},
    {2, false, integrate_blocks_kernel<2, false>}, {4, true, integrate_blocks_kernel<4, true>},
    {3, true, integrate_blocks_kernel<3, true>},   {2, true, integrate_blocks_kernel<2, true>},
};
constexpr int N_INT_VARIANTS = (int)(sizeof(int_variants) / sizeof(int_variants[0]));
static_assert(N_INT_VARIANTS <= MAX_TUNE_VARIANTS, "integration candidate table too long");

int int_variant_count() { return N_INT_VARIANTS; }

void int_variant_describe(int v, char* buf, int cap) {
  snprintf(buf, cap, "integrate %d x 512-thread CTAs per SM%s", int_variants[v].minb,
           int_variants[v].prefetch ? ", next block's fields prefetched to L2" : "");
}

// ctas > 0: that many CTAs instead of the variant's residency times the SM
// count (the grid-stride loop over the visit list gives the same voxels).
int launch_integrate_blocks(Context* ctx, const Pool& pool, int variant, int ctas) {
  const mf_config& c = ctx->cfg;
  SdfArgs a{ctx->d_depth, ctx->d_rgb, ctx->d_masks, ctx->W, ctx->H, c.mu, (float)c.max_weight};
  const F4 k{c.k[0], c.k[1], c.k[2], c.k[3]};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const IntVariant& v = int_variants[variant];
  const int grid = ctas > 0 ? ctas : sms * v.minb;
  v.fn<<<grid, 512, 0, ctx->stream>>>(pool, ctx->d_vols, ctx->d_frames, a, k, ctx->d_visit,
                                      ctx->d_visit_count);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

// projective_functor::build_active_list over the instances in `inst_mask`.
int build_visit_list(Context* ctx, uint32_t inst_mask) {
  MF_CUDA(cudaMemsetAsync(ctx->d_visit_count, 0, sizeof(int), ctx->stream));
  visit_list_kernel<<<div_up(ctx->pool.cap, 256), 256, 0, ctx->stream>>>(
      ctx->pool, ctx->d_vols, ctx->d_frames, inst_mask, ctx->W, ctx->H, ctx->d_visit,
      ctx->d_visit_count);
  MF_CUDA(cudaGetLastError());
  return MF_OK;
}

int stage_integrate(Context* ctx, const IdList& ids, int ctas) {
  if (ids.n == 0) return MF_OK;
  const mf_config& c = ctx->cfg;
  uint32_t mask = 0;
  long long max_nodes = 0;
  for (int i = 0; i < ids.n; ++i) {
    mask |= 1u << ids.v[i];
    max_nodes = std::max(max_nodes, ctx->inst[ids.v[i]].vol.n_nodes);
  }
  if (int rc = build_visit_list(ctx, mask)) return rc;
  if (int rc = launch_integrate_blocks(ctx, ctx->pool, ctx->tune.integrate, ctas)) return rc;
  SdfArgs a{ctx->d_depth, ctx->d_rgb, ctx->d_masks, ctx->W, ctx->H, c.mu, (float)c.max_weight};
  const F4 k{c.k[0], c.k[1], c.k[2], c.k[3]};
  if (max_nodes > 0) {
    integrate_nodes_kernel<<<dim3(div_up(max_nodes * 8, 128), ids.n), 128, 0, ctx->stream>>>(
        ctx->d_vols, ctx->d_frames, a, k, ids);
    MF_CUDA(cudaGetLastError());
  }
  return MF_OK;
}

// Octree::alloc_update(keys, n), lib/octree.hpp:761-786, on explicit keys.
// Set semantics of the reference: after sorting, every key of level L >= 1
// creates its prefix octant at level min(L, block level) and the ancestors;
// the smallest key is kept at every level (unique.hpp:76-79), which creates
// its whole path down to a block.
int alloc_keys(Context* ctx, int id, const uint64_t* keys, int n) {
  Instance& in = ctx->inst[id];
  const Volume& V = in.vol;
  std::vector<unsigned long long> codes;
  std::vector<int> levels;
  uint64_t kmin = ~0ULL;
  const int cnt = n < 1 ? 1 : n;  // unique_multiscale returns 1 for n < 2
  for (int i = 0; i < cnt; ++i) kmin = std::min<uint64_t>(kmin, keys[i]);
  for (int i = 0; i < cnt; ++i) {
    int L = (int)(keys[i] & SCALE_MASK);
    if (keys[i] == kmin) L = V.block_level;
    if (L < 1) continue;
    if (L > V.block_level) L = V.block_level;
    codes.push_back(keys[i] & ~SCALE_MASK);
    levels.push_back(L);
  }
  if (codes.empty()) return MF_OK;
  unsigned long long* d_codes = nullptr;
  int* d_levels = nullptr;
  MF_CUDA(cudaMalloc(&d_codes, sizeof(unsigned long long) * codes.size()));
  MF_CUDA(cudaMalloc(&d_levels, sizeof(int) * levels.size()));
  MF_CUDA(cudaMemcpyAsync(d_codes, codes.data(), sizeof(unsigned long long) * codes.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(d_levels, levels.data(), sizeof(int) * levels.size(),
                          cudaMemcpyHostToDevice, ctx->stream));
  alloc_keys_kernel<<<div_up((long long)codes.size(), 256), 256, 0, ctx->stream>>>(
      ctx->d_vols, id, d_codes, d_levels, (int)codes.size(), ctx->pool, ctx->d_status);
  MF_CUDA(cudaGetLastError());
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  cudaFree(d_codes);
  cudaFree(d_levels);
  return MF_OK;
}

int ensure_export(Context* ctx, size_t bytes) {
  if (ctx->export_bytes >= bytes) return MF_OK;
  if (ctx->d_export) cudaFree(ctx->d_export);
  ctx->d_export = nullptr;
  ctx->export_bytes = 0;
  MF_CUDA(cudaMalloc(&ctx->d_export, bytes));
  ctx->export_bytes = bytes;
  return MF_OK;
}

int export_blocks(Context* ctx, int id, uint64_t* keys, int32_t* coords, uint8_t* active,
                  void* voxels, int cap, int* n_out) {
  const Volume& V = ctx->inst[id].vol;
  const long long n_tab = 1LL << (3 * V.block_level);
  std::vector<int32_t> tab(n_tab);
  MF_CUDA(cudaMemcpyAsync(tab.data(), V.block_tab, sizeof(int32_t) * n_tab,
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  std::vector<int> slots;
  std::vector<long long> bidx;
  for (long long b = 0; b < n_tab; ++b)
    if (tab[b] >= 0) { slots.push_back(tab[b]); bidx.push_back(b); }
  const int n = (int)slots.size();
  if (n_out) *n_out = n;
  if (!keys && !coords && !active && !voxels) return MF_OK;
  if (n > cap) return MF_E_ARG;
  if (n == 0) return MF_OK;
  std::vector<uint8_t> act;
  if (active) {
    std::vector<uint8_t> all(ctx->pool.cap);
    MF_CUDA(cudaMemcpy(all.data(), ctx->pool.active, ctx->pool.cap, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) active[i] = all[slots[i]];
  }
  for (int i = 0; i < n; ++i) {
    const uint64_t b = (uint64_t)bidx[i];
    if (keys) keys[i] = (b << (3 * (V.max_level - V.block_level))) | (uint64_t)V.block_level;
    if (coords) {
      coords[3 * i] = (int)gather3(b) << 3;
      coords[3 * i + 1] = (int)gather3(b >> 1) << 3;
      coords[3 * i + 2] = (int)gather3(b >> 2) << 3;
    }
  }
  if (voxels) {
    const int chunk = 4096;
    if (int rc = ensure_export(ctx, (size_t)chunk * 512 * 40 + sizeof(int) * chunk)) return rc;
    int* d_slots = (int*)((char*)ctx->d_export + (size_t)chunk * 512 * 40);
    for (int s0 = 0; s0 < n; s0 += chunk) {
      const int m = std::min(chunk, n - s0);
      MF_CUDA(cudaMemcpyAsync(d_slots, slots.data() + s0, sizeof(int) * m,
                              cudaMemcpyHostToDevice, ctx->stream));
      export_blocks_kernel<<<m, 256, 0, ctx->stream>>>(ctx->pool, d_slots, m,
                                                       (unsigned char*)ctx->d_export);
      MF_CUDA(cudaGetLastError());
      MF_CUDA(cudaMemcpyAsync((char*)voxels + (size_t)s0 * 512 * 40, ctx->d_export,
                              (size_t)m * 512 * 40, cudaMemcpyDeviceToHost, ctx->stream));
      MF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
  }
  return MF_OK;
}

int export_nodes(Context* ctx, int id, uint64_t* keys, uint32_t* side, uint8_t* cmask,
                 void* values, int cap, int* n_out) {
  const Volume& V = ctx->inst[id].vol;
  const long long nn = V.n_nodes;
  std::vector<uint8_t> nt(nn > 0 ? nn : 1);
  const long long n_tab = 1LL << (3 * V.block_level);
  std::vector<int32_t> tab(n_tab);
  if (nn > 0)
    MF_CUDA(cudaMemcpyAsync(nt.data(), V.node_tab, nn, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaMemcpyAsync(tab.data(), V.block_tab, sizeof(int32_t) * n_tab,
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  std::vector<long long> ent;
  for (long long e = 0; e < nn; ++e) if (nt[e]) ent.push_back(e);
  const int n = (int)ent.size();
  if (n_out) *n_out = n;
  if (!keys && !side && !cmask && !values) return MF_OK;
  if (n > cap) return MF_E_ARG;
  std::vector<float> f[5];
  std::vector<int> ci, wi;
  std::vector<double> fg;
  if (values && nn > 0) {
    float* planes[5] = {V.n_tsdf, V.n_wt, V.n_r, V.n_g, V.n_b};
    for (int q = 0; q < 5; ++q) {
      f[q].resize(nn * 8);
      MF_CUDA(cudaMemcpy(f[q].data(), planes[q], sizeof(float) * nn * 8, cudaMemcpyDeviceToHost));
    }
    ci.resize(nn * 8); wi.resize(nn * 8); fg.resize(nn * 8);
    MF_CUDA(cudaMemcpy(ci.data(), V.n_c, sizeof(int) * nn * 8, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(wi.data(), V.n_w, sizeof(int) * nn * 8, cudaMemcpyDeviceToHost));
    MF_CUDA(cudaMemcpy(fg.data(), V.n_fg, sizeof(double) * nn * 8, cudaMemcpyDeviceToHost));
  }
  for (int i = 0; i < n; ++i) {
    const long long e = ent[i];
    int l = 1;
    while (l + 1 < V.block_level && e >= V.node_off[l + 1]) ++l;
    const uint64_t m = (uint64_t)(e - V.node_off[l]);
    if (keys) keys[i] = (m << (3 * (V.max_level - l))) | (uint64_t)l;
    if (side) side[i] = (uint32_t)(V.size >> l);
    if (cmask) {
      uint8_t cm = 0;
      for (int c = 0; c < 8; ++c) {
        const uint64_t child = m * 8 + c;
        const bool ex = (l + 1 == V.block_level) ? tab[child] >= 0 : nt[V.node_off[l + 1] + child] != 0;
        if (ex) cm |= (uint8_t)(1 << c);
      }
      cmask[i] = cm;
    }
    if (values) {
      for (int c = 0; c < 8; ++c) {
        unsigned char* d = (unsigned char*)values + ((size_t)i * 8 + c) * 40;
        const size_t o = (size_t)e * 8 + c;
        std::memcpy(d + 0, &f[0][o], 4); std::memcpy(d + 4, &f[1][o], 4);
        std::memcpy(d + 8, &f[2][o], 4); std::memcpy(d + 12, &f[3][o], 4);
        std::memcpy(d + 16, &f[4][o], 4); std::memcpy(d + 20, &ci[o], 4);
        std::memcpy(d + 24, &fg[o], 8); std::memcpy(d + 32, &wi[o], 4);
        std::memset(d + 36, 0, 4);
      }
    }
  }
  return MF_OK;
}

int root_children(Context* ctx, int id, uint8_t* mask) {
  const Volume& V = ctx->inst[id].vol;
  uint8_t cm = 0;
  if (V.block_level == 1) {
    int32_t tab[8];
    MF_CUDA(cudaMemcpy(tab, V.block_tab, sizeof(tab), cudaMemcpyDeviceToHost));
    for (int c = 0; c < 8; ++c) if (tab[c] >= 0) cm |= (uint8_t)(1 << c);
  } else {
    uint8_t nt[8];
    MF_CUDA(cudaMemcpy(nt, V.node_tab + V.node_off[1], 8, cudaMemcpyDeviceToHost));
    for (int c = 0; c < 8; ++c) if (nt[c]) cm |= (uint8_t)(1 << c);
  }
  *mask = cm;
  return MF_OK;
}

int interp_points(Context* ctx, int id, const float* pos, int n, int field, float* out) {
  if (n <= 0) return MF_OK;
  if (int rc = ensure_export(ctx, sizeof(float) * 4 * n)) return rc;
  float* d_pos = (float*)ctx->d_export;
  float* d_out = d_pos + 3 * n;
  MF_CUDA(cudaMemcpyAsync(d_pos, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
  interp_points_kernel<<<div_up(n, 256), 256, 0, ctx->stream>>>(ctx->pool, ctx->d_vols, id, d_pos,
                                                                n, field, d_out);
  MF_CUDA(cudaGetLastError());
  MF_CUDA(cudaMemcpyAsync(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

}  // namespace mf

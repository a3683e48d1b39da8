// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
// Restatement of the reference octree and SDF hot-path kernels; every
// function cites the reference file:line it follows.
#include "or_volume.hpp"
#include <algorithm>
#include <cstdlib>

namespace orc {

static inline int ilog2(int v) { int l = 0; while ((1 << l) < v) ++l; return l; }

void Volume::init(int size_, float dim_) {  // lib/octree.hpp:407-417
  size = size_; dim = dim_;
  max_level = ilog2(size);
  block_level = max_level - 3;
  blocks.clear(); block_of.clear(); nodes.clear(); node_of.clear();
  for (int i = 0; i < 8; ++i) root_values[i] = voxel_init();
  root_children = 0;
  alloc_list.clear(); reserved = 0;
}

int Volume::block_index(int x, int y, int z) const {
  // lib/octree.hpp:439-457 (fetch).  Coordinates outside [0, size) alias in
  // the reference's bit-descent; they are treated as unallocated here.
  if (x < 0 || y < 0 || z < 0 || x >= size || y >= size || z >= size) return -1;
  auto it = block_of.find(encode(x, y, z, block_level, max_level));
  return it == block_of.end() ? -1 : it->second;
}

const Voxel* Volume::voxel(int x, int y, int z) const {
  const int b = block_index(x, y, z);
  if (b < 0) return nullptr;
  const Block& B = blocks[b];
  return &B.v[(x - B.cx) + (y - B.cy) * 8 + (z - B.cz) * 64];  // lib/node.hpp:144-149
}

bool Volume::child_exists(int level, int cx, int cy, int cz, int child) const {
  const int half = size >> (level + 1);
  const int x = cx + (child & 1) * half, y = cy + ((child >> 1) & 1) * half,
            z = cz + ((child >> 2) & 1) * half;
  const key_t k = encode(x, y, z, level + 1, max_level);
  if (level + 1 == block_level) return block_of.count(k) != 0;
  return node_of.count(k) != 0;
}

// lib/algorithms/unique.hpp:49-71
int unique_multiscale(key_t* keys, int n, key_t level_mask) {
  int end = 1;
  const key_t key_mask = ~level_mask;
  if (n < 2) return end;
  key_t prev_key = keys[0] & key_mask, prev_level = keys[0] & level_mask;
  for (int i = 1; i < n; ++i) {
    const key_t key = keys[i] & key_mask, level = keys[i] & level_mask;
    if (key != prev_key) keys[end++] = keys[i];
    else if (level > prev_level) keys[end - 1] = keys[i];
    prev_key = key; prev_level = level;
  }
  return end;
}
// lib/algorithms/unique.hpp:73-98
int unique_multiscale_level(key_t* keys, int n, key_t level_mask, unsigned cur) {
  int end = 1;
  const key_t key_mask = ~level_mask;
  if (n < 2) return end;
  key_t prev_key = keys[0] & key_mask, prev_level = keys[0] & level_mask;
  for (int i = 1; i < n; ++i) {
    const key_t key = keys[i] & key_mask, level = keys[i] & level_mask;
    if (level >= cur) {
      if (key != prev_key) keys[end++] = keys[i];
      else if (level > prev_level) keys[end - 1] = keys[i];
      prev_key = key; prev_level = level;
    }
  }
  return end;
}

// lib/octree.hpp:761-786 (alloc_update) + :826-863 (updateLevel), serial.
void Volume::alloc_update(key_t* keys, int n) {
  std::sort(keys, keys + n);
  n = unique_multiscale(keys, n, SCALE_MASK);
  std::vector<key_t> at_level(n);
  const int shift = MAX_BITS - max_level - 1;
  for (int level = 1; level <= block_level; ++level) {
    const key_t mask = mask_bits(level + shift) | SCALE_MASK;
    for (int i = 0; i < n; ++i) at_level[i] = keys[i] & mask;
    const int last = unique_multiscale_level(at_level.data(), n, SCALE_MASK, level);
    for (int i = 0; i < last; ++i) {
      const key_t my = at_level[i] & ~SCALE_MASK;
      // walk levels 1..level from the root; create what is missing
      int parent_node = -1;  // -1: the root (index into `nodes` otherwise)
      unsigned edge = size / 2;
      for (int l = 1; l <= level; ++l) {
        const int shift_l = max_level - l;
        const int idx = (int)((my >> (3 * shift_l)) & 7);  // child_id, octant_ops.hpp:110-116
        const key_t ck = (my & mask_bits(l + shift)) | (key_t)l;  // the child on this path
        if (l == block_level) {
          if (!block_of.count(ck)) {
            Block B;
            unsigned x, y, z; unpack(my, x, y, z);
            B.cx = (int)x; B.cy = (int)y; B.cz = (int)z;
            B.code = my | (key_t)l; B.active = true;
            for (int v = 0; v < 512; ++v) B.v[v] = voxel_init();
            block_of[ck] = (int)blocks.size();
            blocks.push_back(B);
            (parent_node < 0 ? root_children : nodes[parent_node].children_mask) |=
                (unsigned char)(1 << idx);
          }
        } else {
          auto it = node_of.find(ck);
          if (it == node_of.end()) {
            // updateLevel stores myKey | level, myKey being the walking key.
            Node N; N.code = my | (key_t)l; N.side = edge; N.children_mask = 0;
            for (int v = 0; v < 8; ++v) N.v[v] = voxel_init();
            node_of[ck] = (int)nodes.size();
            nodes.push_back(N);
            (parent_node < 0 ? root_children : nodes[parent_node].children_mask) |=
                (unsigned char)(1 << idx);
            it = node_of.find(ck);
          }
          parent_node = it->second;
        }
        edge /= 2;
      }
    }
  }
}

// apps/kfusion/src/cpp/kfusion/alloc_impl.hpp:121-191, single-threaded.  The
// list lives in the volume; slot 0 is never written (pre-increment) and the
// returned count excludes the last written slot.
unsigned build_volume_allocation_list(Volume& vol, const float* depth, const float* mask,
                                      int W, int H, const M4& T_w_c, const M4& T_w_o,
                                      const M4& K, float band) {
  const float voxelSize = vol.dim / vol.size;
  const float inverseVoxelSize = 1 / voxelSize;
  const unsigned size = (unsigned)vol.size;
  const unsigned block_scale = (unsigned)(vol.max_level - 3);
  const M4 invK = inverse(K);
  const M4 kPose = mul(T_w_c, invK);
  const M4 invTwo = inverse(T_w_o);
  const F3 o_cam = invTwo * get_translation(T_w_c);
  const int numSteps = (int)std::ceil(band * inverseVoxelSize);
  unsigned voxelCount = 0;
  key_t* list = vol.alloc_list.data();
  const size_t reserved = vol.reserved;
  for (unsigned y = 0; y < (unsigned)H; y++)
    for (unsigned x = 0; x < (unsigned)W; x++) {
      if (depth[x + y * W] == 0 || mask[x + y * W] < 0) continue;
      const float d = depth[x + y * W];
      const F3 w_vertex = kPose * mk3((x + 0.5f) * d, (y + 0.5f) * d, d);
      const F3 o_vertex = invTwo * w_vertex;
      const F3 direction = normalize(o_cam - o_vertex);
      const F3 origin = o_vertex - (band * 0.5f) * direction;
      const F3 step = (direction * band) / (float)numSteps;
      F3 pos = origin;
      for (int i = 0; i < numSteps; i++) {
        const F3 s = floor3(pos * inverseVoxelSize);
        if (s.x < size && s.y < size && s.z < size && s.x >= 0 && s.y >= 0 && s.z >= 0) {
          const I3 v = to_i3(s);
          const int b = vol.block_index(v.x, v.y, v.z);
          if (b < 0) {
            const key_t k = encode(v.x, v.y, v.z, block_scale, vol.max_level);
            const unsigned idx = ++voxelCount;
            if (idx < reserved) list[idx] = k;
            else break;
          } else {
            vol.blocks[b].active = true;
          }
        }
        pos += step;
      }
    }
  return voxelCount >= reserved ? (unsigned)reserved : voxelCount;
}

// lib/algorithms/filter.hpp:42-51
static bool in_frustum(const Block& b, float vs, const M4& camera, int W, int H) {
  const F3 bc = mk3((float)b.cx, (float)b.cy, (float)b.cz) * vs;
  const F3 vc = camera * bc;
  const int px = (int)(vc.x / vc.z), py = (int)(vc.y / vc.z);
  return px >= 0 && px < W && py >= 0 && py < H;
}

struct SdfUpdate {  // apps/kfusion/src/cpp/kfusion/mapping_impl.hpp:15-49
  const float* depth; const F3* rgb; const float* mask; int W; float mu; int maxweight;
  void operator()(Voxel& data, F3 pos, F2 pixel) const {
    const unsigned px = (unsigned)pixel.x, py = (unsigned)pixel.y;
    const float depthSample = depth[px + W * py];
    if (depthSample <= 0 || mask[px + W * py] < 0) return;
    const float diff = (depthSample - pos.z) *
                       std::sqrt(1 + sq(pos.x / pos.z) + sq(pos.y / pos.z));
    if (diff > -mu) {
      const float sdf = fmn(1.f, diff / mu);
      data.x = clampf((data.y * data.x + sdf) / (data.y + 1), -1.f, 1.f);
      data.y = fmn(data.y + 1, (float)maxweight);
      const F3 m = rgb[px + W * py];
      data.r = (m.x + data.r * data.c) / (data.c + 1);
      data.g = (m.y + data.g * data.c) / (data.c + 1);
      data.b = (m.z + data.b * data.c) / (data.c + 1);
      data.c += 1;
      const float fg_measured = mask[px + W * py];
      data.fg = (fg_measured + data.fg * data.w) / (data.w + 1);
      data.w++;
    }
  }
};

// lib/functors/projective_functor.hpp:54-156 (build_active_list + update_block +
// update_node).  Active list = active OR corner in frustum (filter.hpp:56-61 ORs
// the predicates).
void integrate(Volume& vol, const float* depth, const F3* rgb, const float* mask, int W,
               int H, const M4& Tcw, const M4& K, float mu, int maxweight) {
  const float vs = vol.dim / vol.size;
  const M4 KT = mul(K, Tcw);
  SdfUpdate f{depth, rgb, mask, W, mu, maxweight};
  std::vector<int> active;
  for (int i = 0; i < (int)vol.blocks.size(); ++i)
    if (vol.blocks[i].active || in_frustum(vol.blocks[i], vs, KT, W, H)) active.push_back(i);
  const F3 delta = rotate(Tcw, mk3(vs, 0, 0));
  const F3 cameraDelta = rotate(K, delta);
  // blocks are independent (projective_functor.hpp:144 parallelises the same loop)
#pragma omp parallel for schedule(dynamic, 16)
  for (size_t ai = 0; ai < active.size(); ++ai) {
    Block& B = vol.blocks[active[ai]];
    bool visible = false;
    for (unsigned z = B.cz; z < (unsigned)B.cz + 8; ++z)
      for (unsigned y = B.cy; y < (unsigned)B.cy + 8; ++y) {
        const F3 start = Tcw * mk3(B.cx * vs, y * vs, z * vs);
        const F3 camerastart = K * start;
        for (unsigned x = 0; x < 8; ++x) {
          const F3 cv = camerastart + ((float)x * cameraDelta);
          const F3 pos = start + ((float)x * delta);
          if (pos.z < 0.0001f) continue;
          const float inv = 1.f / cv.z;
          const F2 pixel{cv.x * inv + 0.5f, cv.y * inv + 0.5f};
          if (pixel.x < 0.5f || pixel.x > W - 1.5f || pixel.y < 0.5f || pixel.y > H - 1.5f)
            continue;
          visible = true;
          f(B.v[x + (y - B.cy) * 8 + (z - B.cz) * 64], pos, pixel);
        }
      }
    B.active = visible;
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (size_t ni = 0; ni < vol.nodes.size(); ++ni) {
    Node& N = vol.nodes[ni];
    unsigned ux, uy, uz; unpack(N.code, ux, uy, uz);  // includes the level bits
    const F3 voxel = mk3((float)(int)ux, (float)(int)uy, (float)(int)uz);
    const F3 d = rotate(Tcw, mk3(0.5f * vs * N.side));
    const F3 dc = rotate(K, d);
    const F3 base_cam = Tcw * (voxel * vs);
    const F3 basepix = K * base_cam;
    for (int i = 0; i < 8; ++i) {
      const F3 dir = mk3((float)((i & 1) > 0), (float)((i & 2) > 0), (float)((i & 4) > 0));
      const F3 vox_cam = base_cam + dir * d;
      const F3 pix_hom = basepix + dir * dc;
      if (vox_cam.z < 0.0001f) continue;
      const float inv = 1.f / pix_hom.z;
      const F2 pixel{pix_hom.x * inv + 0.5f, pix_hom.y * inv + 0.5f};
      if (pixel.x < 0.5f || pixel.x > W - 1.5f || pixel.y < 0.5f || pixel.y > H - 1.5f)
        continue;
      f(N.v[i], vox_cam, pixel);
    }
  }
}

unsigned integrate_volume_kernel(Volume& vol, const float* depth, const F3* rgb,
                                 const float* mask, int W, int H, const M4& T_w_c,
                                 const M4& T_w_o, F4 k, float mu) {
  const float voxelsize = vol.dim / (unsigned)vol.size;
  if (!vol.reserved) {  // object.cpp:132-140
    const int num_vox_per_pix = (int)(vol.dim / (8 * voxelsize));
    vol.reserved = (size_t)num_vox_per_pix * W * H;
    vol.alloc_list.assign(vol.reserved, 0);
  }
  const unsigned n = build_volume_allocation_list(vol, depth, mask, W, H, T_w_c, T_w_o,
                                                  camera_matrix(k), 2 * mu);
  // alloc_update(list, n) sorts and dedupes [0, n); unique_multiscale returns
  // 1 for n < 2, so slot 0 (always key 0) is processed even when n == 0.
  std::vector<key_t> keys(vol.alloc_list.begin(),
                          vol.alloc_list.begin() + (n == 0 ? 1 : n));
  vol.alloc_update(keys.data(), (int)n);
  integrate(vol, depth, rgb, mask, W, H, mul(inverse(T_w_c), T_w_o), camera_matrix(k), mu,
            100);
  return n;
}

// ---------------------------------------------------------------------------
// Sampling (lib/octree.hpp:359-379 get_fine, :479-501 interp,
// lib/interpolation/interp_gather.hpp:105-236, :593-680 grad).  Every gather
// tap resolves to the block voxel if the block exists and to the init/empty
// value (tsdf 1, fg 0) otherwise, which is what all eight crossmask cases do.
float get_fine_tsdf(const Volume& v, int x, int y, int z) {
  const Voxel* p = v.voxel(x, y, z);
  return p ? p->x : 1.f;
}
static float sample_field(const Volume& v, int x, int y, int z, int field) {
  const Voxel* p = v.voxel(x, y, z);
  if (!p) return field == 0 ? 1.f : 0.f;
  switch (field) {
    case 0: return p->x;
    case 1: return (float)p->fg;
    case 2: return p->r;
    case 3: return p->g;
    default: return p->b;
  }
}
float interp(const Volume& v, F3 pos_m, int field) {
  const float inv = v.size / v.dim;  // volume_template.hpp:97-104
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const I3 base = to_i3(floor3(pos));
  const F3 f = frac3(pos);
  const I3 lo{imax(base.x, 0), imax(base.y, 0), imax(base.z, 0)};
  float p[8];
  for (int i = 0; i < 8; ++i)
    p[i] = sample_field(v, lo.x + (i & 1), lo.y + ((i >> 1) & 1), lo.z + ((i >> 2) & 1), field);
  return (((p[0] * (1 - f.x) + p[1] * f.x) * (1 - f.y) +
           (p[2] * (1 - f.x) + p[3] * f.x) * f.y) * (1 - f.z) +
          ((p[4] * (1 - f.x) + p[5] * f.x) * (1 - f.y) +
           (p[6] * (1 - f.x) + p[7] * f.x) * f.y) * f.z);
}

F3 grad_tsdf(const Volume& v, F3 pos_m) {  // lib/octree.hpp:593-680
  const float inv = v.size / v.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const I3 base = to_i3(floor3(pos));
  const F3 f = frac3(pos);
  const int s1 = v.size - 1;
  const I3 ll{imax(base.x - 1, 0), imax(base.y - 1, 0), imax(base.z - 1, 0)};
  const I3 lu{imax(base.x, 0), imax(base.y, 0), imax(base.z, 0)};
  const I3 ul{imin(base.x + 1, s1), imin(base.y + 1, s1), imin(base.z + 1, s1)};
  const I3 uu{imin(base.x + 2, s1), imin(base.y + 2, s1), imin(base.z + 2, s1)};
  const I3& lo = lu; const I3& up = ul;
  auto g = [&](int x, int y, int z) { return get_fine_tsdf(v, x, y, z); };
  F3 gr;
  gr.x = (((g(ul.x, lo.y, lo.z) - g(ll.x, lo.y, lo.z)) * (1 - f.x) +
           (g(uu.x, lo.y, lo.z) - g(lu.x, lo.y, lo.z)) * f.x) * (1 - f.y) +
          ((g(ul.x, up.y, lo.z) - g(ll.x, up.y, lo.z)) * (1 - f.x) +
           (g(uu.x, up.y, lo.z) - g(lu.x, up.y, lo.z)) * f.x) * f.y) * (1 - f.z) +
         (((g(ul.x, lo.y, up.z) - g(ll.x, lo.y, up.z)) * (1 - f.x) +
           (g(uu.x, lo.y, up.z) - g(lu.x, lo.y, up.z)) * f.x) * (1 - f.y) +
          ((g(ul.x, up.y, up.z) - g(ll.x, up.y, up.z)) * (1 - f.x) +
           (g(uu.x, up.y, up.z) - g(lu.x, up.y, up.z)) * f.x) * f.y) * f.z;
  gr.y = (((g(lo.x, ul.y, lo.z) - g(lo.x, ll.y, lo.z)) * (1 - f.x) +
           (g(up.x, ul.y, lo.z) - g(up.x, ll.y, lo.z)) * f.x) * (1 - f.y) +
          ((g(lo.x, uu.y, lo.z) - g(lo.x, lu.y, lo.z)) * (1 - f.x) +
           (g(up.x, uu.y, lo.z) - g(up.x, lu.y, lo.z)) * f.x) * f.y) * (1 - f.z) +
         (((g(lo.x, ul.y, up.z) - g(lo.x, ll.y, up.z)) * (1 - f.x) +
           (g(up.x, ul.y, up.z) - g(up.x, ll.y, up.z)) * f.x) * (1 - f.y) +
          ((g(lo.x, uu.y, up.z) - g(lo.x, lu.y, up.z)) * (1 - f.x) +
           (g(up.x, uu.y, up.z) - g(up.x, lu.y, up.z)) * f.x) * f.y) * f.z;
  gr.z = (((g(lo.x, lo.y, ul.z) - g(lo.x, lo.y, ll.z)) * (1 - f.x) +
           (g(up.x, lo.y, ul.z) - g(up.x, lo.y, ll.z)) * f.x) * (1 - f.y) +
          ((g(lo.x, up.y, ul.z) - g(lo.x, up.y, ll.z)) * (1 - f.x) +
           (g(up.x, up.y, ul.z) - g(up.x, up.y, ll.z)) * f.x) * f.y) * (1 - f.z) +
         (((g(lo.x, lo.y, uu.z) - g(lo.x, lo.y, lu.z)) * (1 - f.x) +
           (g(up.x, lo.y, uu.z) - g(up.x, lo.y, lu.z)) * f.x) * (1 - f.y) +
          ((g(lo.x, up.y, uu.z) - g(lo.x, up.y, lu.z)) * (1 - f.x) +
           (g(up.x, up.y, uu.z) - g(up.x, up.y, lu.z)) * f.x) * f.y) * f.z;
  const float s = v.dim / v.size;
  return gr * mk3(s, s, s) * 0.5f;
}

// ---------------------------------------------------------------------------
// lib/octree.hpp:919-1130, the ray iterator's constructor and first next().
static inline int f2i(float f) { int i; std::memcpy(&i, &f, 4); return i; }
static inline float i2f(int i) { float f; std::memcpy(&f, &i, 4); return f; }

float ray_first_block(const Volume& V, F3 origin, F3 direction, float nearPlane,
                      float farPlane, float epsilon) {
  const int CAST = 23;
  struct Handle { int level, cx, cy, cz; };
  struct Entry { Handle parent; float t_max; };
  Entry stack[CAST];
  for (int i = 0; i < CAST; ++i) stack[i] = Entry{Handle{0, 0, 0, 0}, 0.f};
  F3 pos = mk3(1.f, 1.f, 1.f);
  int idx = 0;
  Handle parent{0, 0, 0, 0};
  float scale_exp2 = 0.5f;
  int scale = CAST - 1;
  const int min_scale = CAST - (int)std::log2((double)(V.size / 8));
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

  F3 t_corner; float tc_max;
  for (int guard = 0; scale < CAST && guard < 1 << 20; ++guard) {
    t_corner = pos * t_coef - t_bias;
    tc_max = fmn(fmn(t_corner.x, t_corner.y), t_corner.z);
    const int ci = idx ^ octant_mask ^ 7;
    const bool has_child = V.child_exists(parent.level, parent.cx, parent.cy, parent.cz, ci);
    if (scale == min_scale && has_child) {
      return t_min * V.dim / voxelSize;
    } else if (has_child && t_min <= t_max) {  // descend
      const float tv_max = fmn(t_max, tc_max);
      const float half = scale_exp2 * 0.5f;
      const F3 t_center = half * t_coef + t_corner;
      if (tc_max < h) stack[scale] = Entry{parent, t_max};
      h = tc_max;
      const int hs = V.size >> (parent.level + 1);
      parent = Handle{parent.level + 1, parent.cx + (ci & 1) * hs,
                      parent.cy + ((ci >> 1) & 1) * hs, parent.cz + ((ci >> 2) & 1) * hs};
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
      if (step_mask & 1) differing |= (unsigned)(f2i(pos.x) ^ f2i(pos.x + scale_exp2));
      if (step_mask & 2) differing |= (unsigned)(f2i(pos.y) ^ f2i(pos.y + scale_exp2));
      if (step_mask & 4) differing |= (unsigned)(f2i(pos.z) ^ f2i(pos.z + scale_exp2));
      scale = (f2i((float)differing) >> 23) - 127;
      scale_exp2 = i2f((scale - CAST + 127) << 23);
      // scale >= 23: the ray left the root and next() returns -1 (the reference
      // first reads stack[23], one past the array; the value is never used).
      if (scale >= CAST) return -1.f;
      parent = stack[scale].parent;
      t_max = stack[scale].t_max;
      const int shx = f2i(pos.x) >> scale, shy = f2i(pos.y) >> scale, shz = f2i(pos.z) >> scale;
      pos.x = i2f(shx << scale); pos.y = i2f(shy << scale); pos.z = i2f(shz << scale);
      idx = (shx & 1) | ((shy & 1) << 1) | ((shz & 1) << 2);
      h = 0.0f;
    }
  }
  return -1.f;
}

static float get_tsdf_at(const Volume& v, F3 p) {  // volume_template.hpp:83-88
  const float inv = v.size / v.dim;
  const I3 s = to_i3(mk3(p.x * inv, p.y * inv, p.z * inv));
  return get_fine_tsdf(v, s.x, s.y, s.z);
}

// apps/kfusion/src/cpp/kfusion/rendering_impl.hpp:80-140
F4 raycast(const Volume& v, F3 origin, F3 direction, float nearPlane, float farPlane,
           float mu, float step, float largestep, float* tc) {
  if (tc) *tc = INFINITY;
  const F3 invR = mk3(1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z);
  const F3 tbot = (-1.f * invR) * origin;
  const F3 ttop = invR * (v.dim - origin);
  const F3 tmin = fmn3(ttop, tbot), tmax = fmx3(ttop, tbot);
  const float largest_tmin = fmx(fmx(tmin.x, tmin.y), fmx(tmin.x, tmin.z));
  const float smallest_tmax = fmn(fmn(tmax.x, tmax.y), fmn(tmax.x, tmax.z));
  const float tnear = fmx(largest_tmin, nearPlane);
  const float tfar = fmn(smallest_tmax, farPlane);
  if (tnear < tfar) {
    float t = tnear, stepsize = largestep;
    F3 position = origin + direction * t;
    float f_t = interp(v, position, 0), f_tt = 0;
    if (f_t > 0) {
      for (; t < tfar; t += stepsize) {
        f_tt = get_tsdf_at(v, position);  // weight (data.y) is never negative for SDF
        if ((double)f_tt <= 0.1 && f_tt >= -0.5f) f_tt = interp(v, position, 0);
        if (f_tt < 0) break;
        stepsize = fmx(f_tt * mu, step);
        position += stepsize * direction;
        f_t = f_tt;
      }
      if (f_tt < 0) {
        if (tc) *tc = t;
        t = t + stepsize * f_tt / (f_t - f_tt);
        const F3 p = origin + direction * t;
        return F4{p.x, p.y, p.z, t};
      }
    }
  }
  return F4{0, 0, 0, 0};
}

// apps/kfusion/src/cpp/rendering/rendering.cpp:9-181, every object in view.
void raycast_object_list(const RaycastInstance* inst, int n, F3* vertex, F3* normal,
                         int* label_img, const M4& T_w_c, F4 k, int W, int H,
                         float nearPlane, float farPlane, float mu, float epsilon) {
  const float INVALID = -2;
  const M4 view = mul(T_w_c, inverse_camera_matrix(k));
  std::vector<M4> inv(n);
  for (int i = 0; i < n; ++i) inv[i] = inverse(inst[i].T_w_o);
  // pixels are independent (rendering.cpp:18 parallelises the same loop)
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int p = x + y * W;
      float nearest = 1.0e3f;
      double high_fg = 0.f;
      int miss = 0;
      for (int o = 0; o < n; ++o) {
        const Volume& vol = *inst[o].vol;
        const int label = inst[o].label;
        const float step = vol.dim / vol.size;  // Object::volume_step, object.cpp:53
        const float largestep = step * 8;
        const F3 o_origin = inv[o] * get_translation(view);
        const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
        const F3 o_dir = normalize(rotate(inv[o], w_dir));
        const float nfar = fmn(nearest, farPlane);
        const float t_min = ray_first_block(vol, o_origin, o_dir, nearPlane, nfar, epsilon);
        const F4 hit = t_min > 0.f ? raycast(vol, o_origin, o_dir,
                                             t_min * vol.dim / (unsigned)vol.size, nfar, mu,
                                             step, largestep)
                                   : F4{0, 0, 0, 0};
        const float hd = label == 0 ? hit.w + 0.05f : hit.w;
        if (hd > nearest) { miss++; continue; }
        const double fg = interp(vol, mk3(hit.x, hit.y, hit.z), 1);
        if (fg <= 0.5f) { miss++; continue; }
        bool take = false;
        if (hd == nearest) {
          if (fg > high_fg) take = true; else { miss++; continue; }
        } else if (hd < nearest) {
          nearest = hd; take = true;
        } else { miss++; continue; }
        if (take) {
          high_fg = fg;
          label_img[p] = label;
          vertex[p] = inst[o].T_w_o * mk3(hit.x, hit.y, hit.z);
          const F3 gn = grad_tsdf(vol, mk3(hit.x, hit.y, hit.z));
          if (length(gn) == 0) normal[p].x = INVALID;
          else normal[p] = normalize(rotate(inst[o].T_w_o, gn));
        }
      }
      if (miss == n) {
        vertex[p] = mk3(0.f);
        normal[p] = mk3(INVALID, 0, 0);
        label_img[p] = (int)INVALID;
      }
    }
}

// Test support, no reference counterpart: one instance's records of the
// instance-sharded composite (the device's mf_raycast_records): per pixel 12
// floats -- the hit (x, y, z, t) of the march to the far plane, the march
// parameter of its crossing sample (+inf: none), the foreground at the hit,
// the world normal, a zero-gradient flag and 2 zeros -- and 8 floats of the
// zero hit: foreground and world normal at the volume origin, its flag, 3 zeros.
void raycast_records(const RaycastInstance& in, const M4& T_w_c, F4 k, int W, int H,
                     float nearPlane, float farPlane, float mu, float epsilon, float* rec,
                     float* origin) {
  const Volume& vol = *in.vol;
  const M4 view = mul(T_w_c, inverse_camera_matrix(k));
  const M4 inv = inverse(in.T_w_o);
  const float step = vol.dim / vol.size;
  auto normal_of = [&](F3 h, float* out) {
    const F3 gn = grad_tsdf(vol, h);
    if (length(gn) == 0) { out[0] = out[1] = out[2] = 0.f; out[3] = 1.f; return; }
    const F3 n = normalize(rotate(in.T_w_o, gn));
    out[0] = n.x; out[1] = n.y; out[2] = n.z; out[3] = 0.f;
  };
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      float* r = rec + 12 * (size_t)(x + y * W);
      const F3 o_origin = inv * get_translation(view);
      const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
      const F3 o_dir = normalize(rotate(inv, w_dir));
      const float t_min = ray_first_block(vol, o_origin, o_dir, nearPlane, farPlane, epsilon);
      float tc = INFINITY;
      const F4 hit = t_min > 0.f ? raycast(vol, o_origin, o_dir,
                                           t_min * vol.dim / (unsigned)vol.size, farPlane, mu,
                                           step, step * 8, &tc)
                                 : F4{0, 0, 0, 0};
      r[0] = hit.x; r[1] = hit.y; r[2] = hit.z; r[3] = hit.w;
      r[4] = tc;
      r[5] = 0.f;
      r[6] = r[7] = r[8] = 0.f; r[9] = 1.f;
      r[10] = r[11] = 0.f;
      if (tc < INFINITY) {
        const F3 h = mk3(hit.x, hit.y, hit.z);
        r[5] = interp(vol, h, 1);
        normal_of(h, r + 6);
      }
    }
  origin[0] = interp(vol, mk3(0.f, 0.f, 0.f), 1);
  normal_of(mk3(0.f, 0.f, 0.f), origin + 1);
  origin[5] = origin[6] = origin[7] = 0.f;
}

// Test support, no reference counterpart: marks the pixels where any
// instance's raycast (first-block search, march, foreground interpolation at
// the hit; every instance with the full far plane, so a superset of the rays
// the composite actually evaluates) reads a voxel outside [0, size) that the
// reference aliases into an allocated block.  The reference's bit descent
// (lib/octree.hpp:359-379) maps such coordinates into another block and
// indexes that block's voxel array out of its bounds (lib/node.hpp:144-149),
// so its result there depends on memory layout; the restatement reads them as
// unallocated.  Parity tests exclude these pixels.
// A read at (x, y, z) outside [0, size) whose aliased block (the reference
// descends by the coordinate bits below size) is allocated: there the
// reference returns some voxel of that block or memory past it, the
// restatement the unallocated value.  Aliasing into an unallocated block gives
// the unallocated value in both.
static bool aliased_read(const Volume& v, int x, int y, int z) {
  if (x >= 0 && y >= 0 && z >= 0 && x < v.size && y < v.size && z < v.size) return false;
  const int m = v.size - 1;
  return v.block_index(x & m, y & m, z & m) >= 0;
}
static bool oob_voxel(const Volume& v, F3 p) {
  const float inv = v.size / v.dim;
  const I3 s = to_i3(mk3(p.x * inv, p.y * inv, p.z * inv));
  return aliased_read(v, s.x, s.y, s.z);
}
static bool oob_cell(const Volume& v, F3 pm) {
  const float inv = v.size / v.dim;
  const I3 b = to_i3(floor3(mk3(pm.x * inv, pm.y * inv, pm.z * inv)));
  const I3 lo{imax(b.x, 0), imax(b.y, 0), imax(b.z, 0)};
  for (int i = 0; i < 8; ++i)
    if (aliased_read(v, lo.x + (i & 1), lo.y + ((i >> 1) & 1), lo.z + ((i >> 2) & 1)))
      return true;
  return false;
}
static bool raycast_touches_oob(const Volume& v, F3 origin, F3 direction, float nearPlane,
                                float farPlane, float mu, float step, float largestep) {
  const F3 invR = mk3(1.0f / direction.x, 1.0f / direction.y, 1.0f / direction.z);
  const F3 tbot = (-1.f * invR) * origin;
  const F3 ttop = invR * (v.dim - origin);
  const F3 tmin = fmn3(ttop, tbot), tmax = fmx3(ttop, tbot);
  const float tnear = fmx(fmx(fmx(tmin.x, tmin.y), fmx(tmin.x, tmin.z)), nearPlane);
  const float tfar = fmn(fmn(fmn(tmax.x, tmax.y), fmn(tmax.x, tmax.z)), farPlane);
  if (!(tnear < tfar)) return false;
  float t = tnear, stepsize = largestep;
  F3 position = origin + direction * t;
  if (oob_cell(v, position)) return true;
  float f_t = interp(v, position, 0), f_tt = 0;
  if (!(f_t > 0)) return false;
  for (; t < tfar; t += stepsize) {
    if (oob_voxel(v, position)) return true;
    f_tt = get_tsdf_at(v, position);
    if ((double)f_tt <= 0.1 && f_tt >= -0.5f) {
      if (oob_cell(v, position)) return true;
      f_tt = interp(v, position, 0);
    }
    if (f_tt < 0) break;
    stepsize = fmx(f_tt * mu, step);
    position += stepsize * direction;
    f_t = f_tt;
  }
  if (f_tt < 0) {
    t = t + stepsize * f_tt / (f_t - f_tt);
    if (oob_cell(v, origin + direction * t)) return true;
  }
  return false;
}

void raycast_oob_mask(const RaycastInstance* inst, int n, unsigned char* mask, const M4& T_w_c,
                      F4 k, int W, int H, float nearPlane, float farPlane, float mu,
                      float epsilon) {
  const M4 view = mul(T_w_c, inverse_camera_matrix(k));
  std::vector<M4> inv(n);
  for (int i = 0; i < n; ++i) inv[i] = inverse(inst[i].T_w_o);
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      unsigned char m = 0;
      for (int o = 0; o < n && !m; ++o) {
        const Volume& vol = *inst[o].vol;
        const float step = vol.dim / vol.size;
        const F3 o_origin = inv[o] * get_translation(view);
        const F3 o_dir = normalize(rotate(inv[o], rotate(view, mk3((float)x, (float)y, 1.f))));
        const float t_min = ray_first_block(vol, o_origin, o_dir, nearPlane, farPlane, epsilon);
        if (t_min > 0.f &&
            raycast_touches_oob(vol, o_origin, o_dir, t_min * vol.dim / (unsigned)vol.size,
                                farPlane, mu, step, 8 * step))
          m = 1;
      }
      mask[x + y * W] = m;
    }
}

}  // namespace orc

// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
//
// Restatement of the reference octree (lib/octree.hpp, lib/node.hpp,
// lib/octant_ops.hpp, lib/utils/morton_utils.hpp, lib/algorithms/unique.hpp)
// and of the SDF hot-path kernels built on it:
//   buildVolumeAllocationList  apps/kfusion/src/cpp/kfusion/alloc_impl.hpp:121-191
//   Octree::alloc_update       lib/octree.hpp:761-786, updateLevel :826-863
//   projective_functor         lib/functors/projective_functor.hpp:43-166
//   sdf_update                 apps/kfusion/src/cpp/kfusion/mapping_impl.hpp:15-72
//   ray_iterator               lib/octree.hpp:919-1130
//   raycast                    apps/kfusion/src/cpp/kfusion/rendering_impl.hpp:80-140
//   raycastObjectList          apps/kfusion/src/cpp/rendering/rendering.cpp:9-181
// The octree is kept in hash maps keyed by the reference's 64-bit keys, so the
// oracle shares no data structure with the device implementation.
#pragma once
#include <cstdint>
#include <unordered_map>
#include <vector>
#include "or_math.hpp"

namespace orc {

typedef uint64_t key_t;
constexpr int MAX_BITS = 21;
constexpr key_t SCALE_MASK = 0x1FF;

// voxel_traits<SDF>::ComputeType, apps/kfusion/src/cpp/continuous/volume_traits.hpp:24-33
struct Voxel {
  float x, y, r, g, b;
  int c;
  double fg;
  int w;
};
static_assert(sizeof(Voxel) == 40, "reference voxel layout is 40 bytes");
inline Voxel voxel_init() { Voxel v{1.f, 0.f, 0.f, 0.f, 0.f, 0, 0.0, 0}; return v; }

inline key_t mask_bits(int i) {  // lib/octree_defines.h:58-80, MASK[i]
  const key_t all = 0x7fffffffffffffffULL;
  return (all >> (60 - 3 * i)) << (60 - 3 * i) & all;
}
inline key_t expand_bits(uint64_t v) {
  v &= 0x1fffff; key_t r = 0;
  for (int i = 0; i < 21; ++i) r |= ((v >> i) & 1ULL) << (3 * i);
  return r;
}
inline uint64_t compact_bits(key_t v) {
  uint64_t r = 0;
  for (int i = 0; i < 21; ++i) r |= ((v >> (3 * i)) & 1ULL) << i;
  return r;
}
inline key_t morton(uint64_t x, uint64_t y, uint64_t z) {
  return expand_bits(x) | (expand_bits(y) << 1) | (expand_bits(z) << 2);
}
inline void unpack(key_t code, unsigned& x, unsigned& y, unsigned& z) {
  x = (unsigned)compact_bits(code); y = (unsigned)compact_bits(code >> 1);
  z = (unsigned)compact_bits(code >> 2);
}
inline key_t encode(int x, int y, int z, int level, int max_depth) {  // octant_ops.hpp:51-55
  const int offset = MAX_BITS - max_depth + level - 1;
  return (morton(x, y, z) & mask_bits(offset)) | (key_t)level;
}

struct Block {
  int cx, cy, cz;
  key_t code;
  bool active;
  Voxel v[512];
};
struct Node {
  key_t code;
  unsigned side;
  unsigned char children_mask;
  Voxel v[8];
};

struct Volume {
  int size = 0;      // voxels per side
  float dim = 0.f;   // metres per side
  int max_level = 0, block_level = 0;
  std::vector<Block> blocks;                 // allocation order
  std::unordered_map<key_t, int> block_of;   // block key (code|level) -> index
  std::vector<Node> nodes;                   // internal nodes (levels 1..block_level-1)
  std::unordered_map<key_t, int> node_of;    // node key (code|level) -> index
  Voxel root_values[8];
  unsigned char root_children = 0;
  std::vector<key_t> alloc_list;             // persistent, slot 0 never written
  size_t reserved = 0;

  void init(int size_, float dim_);
  float voxel_size() const { return dim / size; }
  int block_index(int x, int y, int z) const;          // -1 if unallocated/out of range
  const Voxel* voxel(int x, int y, int z) const;       // nullptr if unallocated
  bool child_exists(int level, int cx, int cy, int cz, int child) const;
  void alloc_update(key_t* keys, int n);
};

int unique_multiscale(key_t* keys, int n, key_t level_mask);
int unique_multiscale_level(key_t* keys, int n, key_t level_mask, unsigned cur);
unsigned build_volume_allocation_list(Volume& vol, const float* depth, const float* mask,
                                      int W, int H, const M4& T_w_c, const M4& T_w_o,
                                      const M4& K, float band);
void integrate(Volume& vol, const float* depth, const F3* rgb, const float* mask, int W,
               int H, const M4& Tcw, const M4& K, float mu, int maxweight);
// Object::integrate_volume_kernel, apps/kfusion/src/cpp/object/object.cpp:128-195
unsigned integrate_volume_kernel(Volume& vol, const float* depth, const F3* rgb,
                                 const float* mask, int W, int H, const M4& T_w_c,
                                 const M4& T_w_o, F4 k, float mu);

float get_fine_tsdf(const Volume& v, int x, int y, int z);
float interp(const Volume& v, F3 pos_m, int field);   // 0 tsdf, 1 fg, 2-4 r, g, b
F3 grad_tsdf(const Volume& v, F3 pos_m);
float ray_first_block(const Volume& v, F3 origin, F3 dir, float nearp, float farp,
                      float epsilon);
F4 raycast(const Volume& v, F3 origin, F3 dir, float nearp, float farp, float mu,
           float step, float largestep, float* tc = nullptr);

struct RaycastInstance {
  const Volume* vol;
  M4 T_w_o;
  int label;
};
void raycast_object_list(const RaycastInstance* inst, int n, F3* vertex, F3* normal,
                         int* label_img, const M4& T_w_c, F4 k, int W, int H,
                         float nearp, float farp, float mu, float epsilon);
// one instance's records of the instance-sharded composite (test support)
void raycast_records(const RaycastInstance& in, const M4& T_w_c, F4 k, int W, int H,
                     float nearp, float farp, float mu, float epsilon, float* rec,
                     float* origin);
// pixels whose raycast reads voxels outside [0, size) (test support)
void raycast_oob_mask(const RaycastInstance* inst, int n, unsigned char* mask, const M4& T_w_c,
                      F4 k, int W, int H, float nearp, float farp, float mu, float epsilon);

}  // namespace orc

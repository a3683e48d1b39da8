// TEST INFRASTRUCTURE ONLY.  Builds oracle/_ref/libmf_ref.so from the
// reference's own sources where they lie (lib/, utils/, and the header-only
// SDF kernels under apps/kfusion/src/cpp/), so the CPU oracle can be checked
// against the reference itself.  This file is glue written for this project:
// it supplies the TooN-backed helpers of apps/kfusion/include/commons.h that the
// reference headers call (commons.h itself needs TooN, which is not vendored)
// and exposes a C ABI for the tests.  Nothing here is shipped or measured as the
// product.
#include <queue>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <tuple>
#include "math_utils.h"
#include "or_math.hpp"

// --- commons.h:631-662 stand-ins (same arithmetic as the oracle's restatement)
static inline orc::M4 to_orc(const Matrix4& m) { orc::M4 r; std::memcpy(&r, &m, 64); return r; }
static inline Matrix4 from_orc(const orc::M4& m) { Matrix4 r; std::memcpy(&r, &m, 64); return r; }
inline Matrix4 inverse(const Matrix4& A) { return from_orc(orc::inverse(to_orc(A))); }
inline Matrix4 operator*(const Matrix4& A, const Matrix4& B) {
  return from_orc(orc::mul(to_orc(A), to_orc(B)));
}
inline Matrix4 getCameraMatrix(const float4& k) {
  return from_orc(orc::camera_matrix(orc::F4{k.x, k.y, k.z, k.w}));
}
inline Matrix4 getInverseCameraMatrix(const float4& k) {
  return from_orc(orc::inverse_camera_matrix(orc::F4{k.x, k.y, k.z, k.w}));
}

#include "octree.hpp"
#include "continuous/volume_instance.hpp"
#include "kfusion/alloc_impl.hpp"
#include "kfusion/mapping_impl.hpp"
#include "functors/projective_functor.hpp"
#include "kfusion/rendering_impl.hpp"

// the reference's marching cubes (lib/algorithms/meshing.hpp) names the app's
// FieldType and Triangle (commons.h:156-162) without declaring them
#include <mutex>
#include <sstream>
#include <vector>
typedef SDF FieldType;
struct Triangle { float3 vertexes[3]; };
#include "algorithms/meshing.hpp"

typedef octlib::key_t refkey_t;

struct RefVol {
  Volume<SDF> vol;
  refkey_t* list = nullptr;
  size_t reserved = 0;
};

static Matrix4 load_m4(const float* p) { Matrix4 m; std::memcpy(&m, p, 64); return m; }

extern "C" {

void* ref_vol_create(int size, float dim) {
  RefVol* r = new RefVol;
  r->vol.init(size, dim);
  return r;
}
void ref_vol_destroy(void* h) {
  RefVol* r = (RefVol*)h;
  free(r->list);
  delete r;
}

// Object::integrate_volume_kernel, apps/kfusion/src/cpp/object/object.cpp:128-195
// (SDF branch) around the reference's own calls.
unsigned ref_integrate(void* h, const float* depth, const float* rgb3, const float* mask,
                       int W, int H, const float* Twc, const float* Two, const float* k4,
                       float mu) {
  RefVol& r = *(RefVol*)h;
  const Matrix4 T_w_c = load_m4(Twc), T_w_o = load_m4(Two);
  const float4 k = make_float4(k4[0], k4[1], k4[2], k4[3]);
  const float voxelsize = r.vol._size / r.vol._resol;
  const int num_vox_per_pix = r.vol._size / ((VoxelBlock<SDF>::side) * voxelsize);
  const size_t total = (size_t)num_vox_per_pix * W * H;
  if (!r.reserved) {
    r.list = (refkey_t*)calloc(sizeof(refkey_t) * total, 1);
    r.reserved = total;
  }
  cv::Mat m(H, W, CV_32FC1, (void*)mask);
  const unsigned allocated = buildVolumeAllocationList(
      r.list, r.reserved, r.vol._map_index, T_w_c, T_w_o, getCameraMatrix(k), depth, m,
      make_uint2(W, H), r.vol._resol, voxelsize, 2 * mu);
  r.vol._map_index.alloc_update(r.list, allocated);
  struct sdf_update funct(depth, (const float3*)rgb3, m, make_uint2(W, H), mu, 100);
  iterators::projective_functor<SDF, Octree, struct sdf_update> it(
      r.vol._map_index, funct, inverse(T_w_c) * T_w_o, getCameraMatrix(k), make_int2(W, H));
  it.apply();
  return allocated;
}

void ref_alloc_update(void* h, refkey_t* keys, int n) {
  ((RefVol*)h)->vol._map_index.alloc_update(keys, n);
}

int ref_block_count(void* h) { return (int)((RefVol*)h)->vol._map_index.getBlockBuffer().size(); }
int ref_node_count(void* h) { return (int)((RefVol*)h)->vol._map_index.getNodesBuffer().size(); }
unsigned char ref_root_children(void* h) {
  return ((RefVol*)h)->vol._map_index.root()->children_mask_;
}

// Blocks in pool order: key, corner coordinates, active flag, 512 AoS voxels (40 B).
void ref_export_blocks(void* h, refkey_t* keys, int* coords, unsigned char* active,
                       void* voxels) {
  auto& pool = ((RefVol*)h)->vol._map_index.getBlockBuffer();
  for (size_t i = 0; i < pool.size(); ++i) {
    VoxelBlock<SDF>* b = pool[i];
    keys[i] = b->code;
    const int3 c = b->coordinates();
    coords[3 * i] = c.x; coords[3 * i + 1] = c.y; coords[3 * i + 2] = c.z;
    active[i] = b->active() ? 1 : 0;
    if (voxels) std::memcpy((char*)voxels + i * 512 * 40, b->getBlockRawPtr(), 512 * 40);
  }
}
void ref_export_nodes(void* h, refkey_t* keys, unsigned* side, unsigned char* cmask,
                      void* values) {
  auto& pool = ((RefVol*)h)->vol._map_index.getNodesBuffer();
  for (size_t i = 0; i < pool.size(); ++i) {
    Node<SDF>* n = pool[i];
    keys[i] = n->code; side[i] = n->side; cmask[i] = n->children_mask_;
    if (values) std::memcpy((char*)values + i * 8 * 40, n->value_, 8 * 40);
  }
}

float ref_interp(void* h, const float* p, int field) {
  const float3 pos = make_float3(p[0], p[1], p[2]);
  auto& vol = ((RefVol*)h)->vol;
  switch (field) {
    case 0: return vol.interp(pos, [](const auto& v) { return v.x; });
    case 1: return vol.interp(pos, [](const auto& v) { return v.fg; });
    case 2: return vol.interp(pos, [](const auto& v) { return v.r; });
    case 3: return vol.interp(pos, [](const auto& v) { return v.g; });
    default: return vol.interp(pos, [](const auto& v) { return v.b; });
  }
}
void ref_grad(void* h, const float* p, float* out) {
  const float3 g = ((RefVol*)h)->vol.grad(make_float3(p[0], p[1], p[2]),
                                          [](const auto& v) { return v.x; });
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
}

// The ray iterator keeps its direction epsilon in a function-local static set by
// the first iterator ever built (lib/octree.hpp:934); this pins it.
void ref_pin_epsilon(int size) {
  Octree<SDF> o;
  o.init(size, 1.f);
  ray_iterator<SDF> it(o, make_float3(0.5f), make_float3(0.f, 0.f, 1.f), 0.1f, 1.f);
  (void)it;
}

float ref_ray_first_block(void* h, const float* o, const float* d, float nearp, float farp) {
  ray_iterator<SDF> ray(((RefVol*)h)->vol._map_index, make_float3(o[0], o[1], o[2]),
                        make_float3(d[0], d[1], d[2]), nearp, farp);
  return std::get<0>(ray.next());
}

void ref_raycast(void* h, const float* o, const float* d, float nearp, float farp, float mu,
                 float step, float largestep, float* out) {
  const float4 r = raycast(((RefVol*)h)->vol, make_float3(o[0], o[1], o[2]),
                           make_float3(d[0], d[1], d[2]), nearp, farp, mu, step, largestep);
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

// raycastObjectList, apps/kfusion/src/cpp/rendering/rendering.cpp:9-181, with
// every object in view; the loop body calls the reference's ray_iterator,
// raycast, Volume::interp and Volume::grad.
void ref_raycast_objects(void** vols, const float* Two, const int* labels, int n,
                         const float* Twc, const float* k4, int W, int H, float nearPlane,
                         float farPlane, float mu, float* vertex_out, float* normal_out,
                         int* label_img) {
  const float INVALID = -2;
  float3* vertex = (float3*)vertex_out;
  float3* normal = (float3*)normal_out;
  const float4 k = make_float4(k4[0], k4[1], k4[2], k4[3]);
  const Matrix4 view = load_m4(Twc) * getInverseCameraMatrix(k);
  // the reference's pixel loop is an OpenMP loop over rows (rendering.cpp:18);
  // every pixel writes only its own outputs.  The serial parity build ignores
  // the pragma.
#pragma omp parallel for
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float nearest_hit_t = 1.0e3;
      double high_fg_prob = 0.f;
      int miss_count = 0;
      const int p = x + y * W;
      for (int o = 0; o < n; ++o) {
        const Volume<FieldType>& volume = ((RefVol*)vols[o])->vol;
        const int label = labels[o];
        const float step = volume._size / volume._resol;
        const float largestep = step * BLOCK_SIDE;
        const Matrix4 T_w_o = load_m4(Two + 16 * o);
        const float3 w_orgin = get_translation(view);
        const float3 o_origin = inverse(T_w_o) * w_orgin;
        const float3 w_direction = rotate(view, make_float3(x, y, 1.f));
        const float3 o_direction = normalize(rotate(inverse(T_w_o), w_direction));
        const float nearest_farPlane = fminf(nearest_hit_t, farPlane);
        ray_iterator<FieldType> ray(volume._map_index, o_origin, o_direction, nearPlane,
                                    nearest_farPlane);
        const float t_min = std::get<0>(ray.next());
        const float4 o_hit = t_min > 0.f
                                 ? raycast(volume, o_origin, o_direction,
                                           t_min * volume._size / volume._resol,
                                           nearest_farPlane, mu, step, largestep)
                                 : make_float4(0.f);
        const float hit_distance = label == 0 ? o_hit.w + 0.05f : o_hit.w;
        if (hit_distance > nearest_hit_t) { miss_count++; continue; }
        const double fg_prob =
            volume.interp(make_float3(o_hit), [](const auto& val) { return val.fg; });
        if (fg_prob <= 0.5f) { miss_count++; continue; }
        if (hit_distance == nearest_hit_t) {
          if (fg_prob > high_fg_prob) {
            high_fg_prob = fg_prob;
          } else { miss_count++; continue; }
        } else if (hit_distance < nearest_hit_t) {
          nearest_hit_t = hit_distance;
          high_fg_prob = fg_prob;
        } else { miss_count++; continue; }
        label_img[p] = label;
        vertex[p] = T_w_o * make_float3(o_hit);
        const float3 n3 = volume.grad(make_float3(o_hit), [](const auto& val) { return val.x; });
        if (length(n3) == 0) normal[p].x = INVALID;
        else normal[p] = normalize(rotate(T_w_o, n3));
      }
      if (miss_count == n) {
        vertex[p] = make_float3(0);
        normal[p] = make_float3(INVALID, 0, 0);
        label_img[p] = (int)INVALID;
      }
    }
}

// meshing::compute_index of cell (x, y, z) with the inside test of
// Kfusion::dump_mesh (tsdf < 0); 0 when the cell's block is not allocated
int ref_mc_index(void* h, int x, int y, int z) {
  auto& vol = ((RefVol*)h)->vol;
  const VoxelBlock<SDF>* b = vol._map_index.fetch(x, y, z);
  if (!b) return -1;
  auto inside = [](const Volume<SDF>::compute_type& v) { return v.x < 0.f; };
  return meshing::compute_index(vol._map_index, b, inside, x, y, z);
}
// meshing::interp_vertexes for edge 0..11 (the reference handles 0..2)
void ref_mc_vertex(void* h, int x, int y, int z, int edge, float* out) {
  auto& vol = ((RefVol*)h)->vol;
  auto select = [](const Volume<SDF>::compute_type& v) { return v.x; };
  const float3 p = meshing::interp_vertexes(vol._map_index, select, x, y, z, edge);
  out[0] = p.x; out[1] = p.y; out[2] = p.z;
}
// The reference's own triangulation table (lib/algorithms/edge_tables.h
// triTable, compiled in with meshing.hpp): 256 x 16 ints into out.
void ref_tri_table(int* out) { std::memcpy(out, triTable, sizeof(triTable)); }

// algorithms::marching_cube as Kfusion::dump_mesh calls it: the triangle count,
// and up to cap triangles (9 floats each) into out
long long ref_marching_cube(void* h, float* out, long long cap) {
  auto& vol = ((RefVol*)h)->vol;
  auto inside = [](const Volume<SDF>::compute_type& v) { return v.x < 0.f; };
  auto select = [](const Volume<SDF>::compute_type& v) { return v.x; };
  std::vector<Triangle> mesh;
  algorithms::marching_cube(vol._map_index, select, inside, mesh);
  for (long long i = 0; i < (long long)mesh.size() && i < cap; ++i)
    for (int k = 0; k < 3; ++k) {
      out[9 * i + 3 * k] = mesh[i].vertexes[k].x;
      out[9 * i + 3 * k + 1] = mesh[i].vertexes[k].y;
      out[9 * i + 3 * k + 2] = mesh[i].vertexes[k].z;
    }
  return (long long)mesh.size();
}

}  // extern "C"

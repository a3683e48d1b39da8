// TEST INFRASTRUCTURE ONLY — C ABI of the CPU oracle for the Python tests.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load it.
#include <cstring>
#include <vector>
#include "or_volume.hpp"

using namespace orc;

extern "C" {

void* or_vol_create(int size, float dim) {
  Volume* v = new Volume;
  v->init(size, dim);
  return v;
}
void or_vol_destroy(void* h) { delete (Volume*)h; }

unsigned or_integrate(void* h, const float* depth, const float* rgb3, const float* mask,
                      int W, int H, const float* Twc, const float* Two, const float* k4,
                      float mu) {
  return integrate_volume_kernel(*(Volume*)h, depth, (const F3*)rgb3, mask, W, H,
                                 load_m4(Twc), load_m4(Two), F4{k4[0], k4[1], k4[2], k4[3]},
                                 mu);
}

// Allocation list exactly as buildVolumeAllocationList leaves it: slots
// [0, count) are returned (slot 0 is the never-written zero slot).
unsigned or_build_alloc_list(void* h, const float* depth, const float* mask, int W, int H,
                             const float* Twc, const float* Two, const float* k4, float mu,
                             uint64_t* out, size_t cap) {
  Volume& v = *(Volume*)h;
  const float voxelsize = v.dim / (unsigned)v.size;
  if (!v.reserved) {
    const int num_vox_per_pix = (int)(v.dim / (8 * voxelsize));
    v.reserved = (size_t)num_vox_per_pix * W * H;
    v.alloc_list.assign(v.reserved, 0);
  }
  const unsigned n = build_volume_allocation_list(
      v, depth, mask, W, H, load_m4(Twc), load_m4(Two),
      camera_matrix(F4{k4[0], k4[1], k4[2], k4[3]}), 2 * mu);
  for (unsigned i = 0; i < n && i < cap; ++i) out[i] = v.alloc_list[i];
  return n;
}

void or_alloc_update(void* h, uint64_t* keys, int n) { ((Volume*)h)->alloc_update(keys, n); }

int or_block_count(void* h) { return (int)((Volume*)h)->blocks.size(); }
int or_node_count(void* h) { return (int)((Volume*)h)->nodes.size(); }
unsigned char or_root_children(void* h) { return ((Volume*)h)->root_children; }

void or_export_blocks(void* h, uint64_t* keys, int* coords, unsigned char* active,
                      void* voxels) {
  const Volume& v = *(Volume*)h;
  for (size_t i = 0; i < v.blocks.size(); ++i) {
    const Block& b = v.blocks[i];
    keys[i] = b.code;
    coords[3 * i] = b.cx; coords[3 * i + 1] = b.cy; coords[3 * i + 2] = b.cz;
    active[i] = b.active ? 1 : 0;
    if (voxels) std::memcpy((char*)voxels + i * 512 * 40, b.v, 512 * 40);
  }
}
void or_export_nodes(void* h, uint64_t* keys, unsigned* side, unsigned char* cmask,
                     void* values) {
  const Volume& v = *(Volume*)h;
  for (size_t i = 0; i < v.nodes.size(); ++i) {
    keys[i] = v.nodes[i].code; side[i] = v.nodes[i].side; cmask[i] = v.nodes[i].children_mask;
    if (values) std::memcpy((char*)values + i * 8 * 40, v.nodes[i].v, 8 * 40);
  }
}

float or_interp(void* h, const float* p, int field) {
  return interp(*(Volume*)h, mk3(p[0], p[1], p[2]), field);
}
void or_grad(void* h, const float* p, float* out) {
  const F3 g = grad_tsdf(*(Volume*)h, mk3(p[0], p[1], p[2]));
  out[0] = g.x; out[1] = g.y; out[2] = g.z;
}
float or_ray_first_block(void* h, const float* o, const float* d, float nearp, float farp,
                         float eps) {
  return ray_first_block(*(Volume*)h, mk3(o[0], o[1], o[2]), mk3(d[0], d[1], d[2]), nearp,
                         farp, eps);
}
void or_raycast(void* h, const float* o, const float* d, float nearp, float farp, float mu,
                float step, float largestep, float* out) {
  const F4 r = raycast(*(Volume*)h, mk3(o[0], o[1], o[2]), mk3(d[0], d[1], d[2]), nearp, farp,
                       mu, step, largestep);
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}
void or_raycast_objects(void** vols, const float* Two, const int* labels, int n,
                        const float* Twc, const float* k4, int W, int H, float nearp,
                        float farp, float mu, float eps, float* vertex, float* normal,
                        int* label_img) {
  std::vector<RaycastInstance> inst(n);
  for (int i = 0; i < n; ++i) {
    inst[i].vol = (const Volume*)vols[i];
    inst[i].T_w_o = load_m4(Two + 16 * i);
    inst[i].label = labels[i];
  }
  raycast_object_list(inst.data(), n, (F3*)vertex, (F3*)normal, label_img, load_m4(Twc),
                      F4{k4[0], k4[1], k4[2], k4[3]}, W, H, nearp, farp, mu, eps);
}

void or_raycast_records(void* vol, const float* Two, int label, const float* Twc,
                        const float* k4, int W, int H, float nearp, float farp, float mu,
                        float eps, float* rec, float* origin) {
  RaycastInstance in;
  in.vol = (const Volume*)vol;
  in.T_w_o = load_m4(Two);
  in.label = label;
  raycast_records(in, load_m4(Twc), F4{k4[0], k4[1], k4[2], k4[3]}, W, H, nearp, farp, mu, eps,
                  rec, origin);
}

void or_raycast_oob_mask(void** vols, const float* Two, int n, const float* Twc,
                         const float* k4, int W, int H, float nearp, float farp, float mu,
                         float eps, unsigned char* mask) {
  std::vector<RaycastInstance> inst(n);
  for (int i = 0; i < n; ++i) {
    inst[i].vol = (const Volume*)vols[i];
    inst[i].T_w_o = load_m4(Two + 16 * i);
    inst[i].label = 0;
  }
  raycast_oob_mask(inst.data(), n, mask, load_m4(Twc), F4{k4[0], k4[1], k4[2], k4[3]}, W, H,
                   nearp, farp, mu, eps);
}

// Unit-level entry points for the reference's own unit tests.
int or_unique_multiscale(uint64_t* keys, int n, uint64_t level_mask, int cur_level) {
  return cur_level < 0 ? unique_multiscale(keys, n, level_mask)
                       : unique_multiscale_level(keys, n, level_mask, (unsigned)cur_level);
}
uint64_t or_encode(int x, int y, int z, int level, int max_depth) {
  return encode(x, y, z, level, max_depth);
}
uint64_t or_morton(unsigned x, unsigned y, unsigned z) { return morton(x, y, z); }
void or_unpack(uint64_t code, unsigned* xyz) { unpack(code, xyz[0], xyz[1], xyz[2]); }
float or_bilinear(const float* img, int w, float x, float y) {
  return bilinear(img, w, F2{x, y});
}

}  // extern "C"

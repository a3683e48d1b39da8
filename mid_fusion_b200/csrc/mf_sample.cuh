// Octree sampling on the device: point reads, trilinear interpolation and the
// central-difference gradient, with the reference's arithmetic.
#pragma once
#include "mf_common.cuh"

namespace mf {

// Volume::interp, continuous/volume_template.hpp:97-104 -> Octree::interp,
// lib/octree.hpp:479-501 + gather_points (lib/interpolation/interp_gather.hpp):
// every tap reads the block voxel when the block exists and the init / empty
// value (tsdf 1, fg 0) otherwise.
__device__ __forceinline__ float tap(const Pool& P, const Volume& V, int x, int y, int z,
                                     int field) {
  const int s = block_slot(V, x, y, z);
  if (s < 0) return field == 0 ? 1.f : 0.f;
  const size_t o = (size_t)s * 512 + voxel_index(x, y, z);
  return field == 0 ? P.tsdf[o] : (float)P.fg[o];
}
__device__ __forceinline__ float volume_interp(const Pool& P, const Volume& V, F3 pos_m, int field) {
  const float inv = V.size / V.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const F3 fl = floor3(pos);
  const I3 base = to_i3(fl);
  const F3 f = mk3(pos.x - fl.x, pos.y - fl.y, pos.z - fl.z);
  const int lx = imx(base.x, 0), ly = imx(base.y, 0), lz = imx(base.z, 0);
  float p[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) p[i] = tap(P, V, lx + (i & 1), ly + ((i >> 1) & 1), lz + (i >> 2), field);
  return (((p[0] * (1 - f.x) + p[1] * f.x) * (1 - f.y) +
           (p[2] * (1 - f.x) + p[3] * f.x) * f.y) * (1 - f.z) +
          ((p[4] * (1 - f.x) + p[5] * f.x) * (1 - f.y) +
           (p[6] * (1 - f.x) + p[7] * f.x) * f.y) * f.z);
}


__device__ __forceinline__ float tsdf_at(const Pool& P, const Volume& V, int x, int y, int z) {
  const int s = block_slot(V, x, y, z);
  return s < 0 ? 1.f : P.tsdf[(size_t)s * 512 + voxel_index(x, y, z)];
}

// Octree::grad(pos, select), lib/octree.hpp:593-680: 48 reads through the
// cached get(x, y, z, block), which falls back to the init value (not to the
// node value) when a block is missing, i.e. get_fine semantics.
__device__ __forceinline__ F3 volume_grad(const Pool& P, const Volume& V, F3 pos_m) {
  const float inv = V.size / V.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const F3 fl = floor3(pos);
  const I3 base = to_i3(fl);
  const F3 f = mk3(pos.x - fl.x, pos.y - fl.y, pos.z - fl.z);
  const int s1 = V.size - 1;
  const I3 ll{imx(base.x - 1, 0), imx(base.y - 1, 0), imx(base.z - 1, 0)};
  const I3 lu{imx(base.x, 0), imx(base.y, 0), imx(base.z, 0)};
  const I3 ul{imn(base.x + 1, s1), imn(base.y + 1, s1), imn(base.z + 1, s1)};
  const I3 uu{imn(base.x + 2, s1), imn(base.y + 2, s1), imn(base.z + 2, s1)};
  const I3& lo = lu;
  const I3& up = ul;
#define G(X, Y, Z) tsdf_at(P, V, X, Y, Z)
  F3 gr;
  gr.x = (((G(ul.x, lo.y, lo.z) - G(ll.x, lo.y, lo.z)) * (1 - f.x) +
           (G(uu.x, lo.y, lo.z) - G(lu.x, lo.y, lo.z)) * f.x) * (1 - f.y) +
          ((G(ul.x, up.y, lo.z) - G(ll.x, up.y, lo.z)) * (1 - f.x) +
           (G(uu.x, up.y, lo.z) - G(lu.x, up.y, lo.z)) * f.x) * f.y) * (1 - f.z) +
         (((G(ul.x, lo.y, up.z) - G(ll.x, lo.y, up.z)) * (1 - f.x) +
           (G(uu.x, lo.y, up.z) - G(lu.x, lo.y, up.z)) * f.x) * (1 - f.y) +
          ((G(ul.x, up.y, up.z) - G(ll.x, up.y, up.z)) * (1 - f.x) +
           (G(uu.x, up.y, up.z) - G(lu.x, up.y, up.z)) * f.x) * f.y) * f.z;
  gr.y = (((G(lo.x, ul.y, lo.z) - G(lo.x, ll.y, lo.z)) * (1 - f.x) +
           (G(up.x, ul.y, lo.z) - G(up.x, ll.y, lo.z)) * f.x) * (1 - f.y) +
          ((G(lo.x, uu.y, lo.z) - G(lo.x, lu.y, lo.z)) * (1 - f.x) +
           (G(up.x, uu.y, lo.z) - G(up.x, lu.y, lo.z)) * f.x) * f.y) * (1 - f.z) +
         (((G(lo.x, ul.y, up.z) - G(lo.x, ll.y, up.z)) * (1 - f.x) +
           (G(up.x, ul.y, up.z) - G(up.x, ll.y, up.z)) * f.x) * (1 - f.y) +
          ((G(lo.x, uu.y, up.z) - G(lo.x, lu.y, up.z)) * (1 - f.x) +
           (G(up.x, uu.y, up.z) - G(up.x, lu.y, up.z)) * f.x) * f.y) * f.z;
  gr.z = (((G(lo.x, lo.y, ul.z) - G(lo.x, lo.y, ll.z)) * (1 - f.x) +
           (G(up.x, lo.y, ul.z) - G(up.x, lo.y, ll.z)) * f.x) * (1 - f.y) +
          ((G(lo.x, up.y, ul.z) - G(lo.x, up.y, ll.z)) * (1 - f.x) +
           (G(up.x, up.y, ul.z) - G(up.x, up.y, ll.z)) * f.x) * f.y) * (1 - f.z) +
         (((G(lo.x, lo.y, uu.z) - G(lo.x, lo.y, lu.z)) * (1 - f.x) +
           (G(up.x, lo.y, uu.z) - G(up.x, lo.y, lu.z)) * f.x) * (1 - f.y) +
          ((G(lo.x, up.y, uu.z) - G(lo.x, up.y, lu.z)) * (1 - f.x) +
           (G(up.x, up.y, uu.z) - G(up.x, up.y, lu.z)) * f.x) * f.y) * f.z;
#undef G
  const float s = V.dim / V.size;
  return gr * mk3(s, s, s) * 0.5f;
}

}  // namespace mf

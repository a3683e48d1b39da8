// Octree sampling on the device: point reads, trilinear interpolation and the
// central-difference gradient, with the reference's arithmetic.
#pragma once
#include "mf_common.cuh"

namespace mf {

// Per-thread memo of the last block looked up: consecutive samples along a ray
// mostly fall into the same 8^3 block, so the table lookup is skipped.
struct BlockMemo {
  int key = -1;
  int slot = -1;
};

// Pool slot of the block holding voxel (x, y, z), through the memo.
__device__ __forceinline__ int memo_slot(const Volume& V, BlockMemo& m, int x, int y, int z) {
  if ((unsigned)x >= (unsigned)V.size || (unsigned)y >= (unsigned)V.size ||
      (unsigned)z >= (unsigned)V.size)
    return -1;
  const int key = (x >> 3) | ((y >> 3) << 10) | ((z >> 3) << 20);
  if (key != m.key) {
    m.key = key;
    m.slot = V.block_tab[morton3(x >> 3, y >> 3, z >> 3)];
  }
  return m.slot;
}

// Volume::interp, continuous/volume_template.hpp:97-104 -> Octree::interp,
// lib/octree.hpp:479-501 + gather_points (lib/interpolation/interp_gather.hpp):
// every tap reads the block voxel when the block exists and the init / empty
// value (tsdf 1, fg 0) otherwise.  When the 2x2x2 cell lies inside one block
// (gather_points' "all local" case) a single block lookup serves all taps.
template <int FIELD>
__device__ __forceinline__ float tap_val(const Pool& P, int slot, int v) {
  if (slot < 0) return FIELD == 0 ? 1.f : 0.f;
  const size_t o = (size_t)slot * 512 + v;
  return FIELD == 0 ? __ldg(P.tsdf + o) : (float)__ldg(P.fg + o);
}

template <int FIELD>
__device__ __noinline__ float volume_interp_m(const Pool& P, const Volume& V, F3 pos_m,
                                              BlockMemo& m) {
  const float inv = V.size / V.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const F3 fl = floor3(pos);
  const I3 base = to_i3(fl);
  const F3 f = mk3(pos.x - fl.x, pos.y - fl.y, pos.z - fl.z);
  const int lx = imx(base.x, 0), ly = imx(base.y, 0), lz = imx(base.z, 0);
  float p[8];
  if ((lx & 7) != 7 && (ly & 7) != 7 && (lz & 7) != 7) {
    const int slot = memo_slot(V, m, lx, ly, lz);
    const int v0 = voxel_index(lx, ly, lz);
    p[0] = tap_val<FIELD>(P, slot, v0);       p[1] = tap_val<FIELD>(P, slot, v0 + 1);
    p[2] = tap_val<FIELD>(P, slot, v0 + 8);   p[3] = tap_val<FIELD>(P, slot, v0 + 9);
    p[4] = tap_val<FIELD>(P, slot, v0 + 64);  p[5] = tap_val<FIELD>(P, slot, v0 + 65);
    p[6] = tap_val<FIELD>(P, slot, v0 + 72);  p[7] = tap_val<FIELD>(P, slot, v0 + 73);
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int x = lx + (i & 1), y = ly + ((i >> 1) & 1), z = lz + (i >> 2);
      p[i] = tap_val<FIELD>(P, memo_slot(V, m, x, y, z), voxel_index(x, y, z));
    }
  }
  return (((p[0] * (1 - f.x) + p[1] * f.x) * (1 - f.y) +
           (p[2] * (1 - f.x) + p[3] * f.x) * f.y) * (1 - f.z) +
          ((p[4] * (1 - f.x) + p[5] * f.x) * (1 - f.y) +
           (p[6] * (1 - f.x) + p[7] * f.x) * f.y) * f.z);
}

__device__ __forceinline__ float volume_interp(const Pool& P, const Volume& V, F3 pos_m,
                                               int field) {
  BlockMemo m;
  return field == 0 ? volume_interp_m<0>(P, V, pos_m, m) : volume_interp_m<1>(P, V, pos_m, m);
}

__device__ __forceinline__ float tsdf_at(const Pool& P, const Volume& V, int x, int y, int z) {
  const int s = block_slot(V, x, y, z);
  return s < 0 ? 1.f : P.tsdf[(size_t)s * 512 + voxel_index(x, y, z)];
}

__device__ __forceinline__ float tsdf_at_m(const Pool& P, const Volume& V, BlockMemo& m, int x,
                                           int y, int z) {
  const int s = memo_slot(V, m, x, y, z);
  return s < 0 ? 1.f : __ldg(P.tsdf + (size_t)s * 512 + voxel_index(x, y, z));
}

// Octree::grad(pos, select), lib/octree.hpp:593-680: 48 reads through the
// cached get(x, y, z, block), which falls back to the init value (not to the
// node value) when a block is missing, i.e. get_fine semantics.  The taps span
// at most 2 blocks per axis; their slots are resolved once.
// Not inlined: called once per accepted hit; inlining its 48 taps into the
// raycast loop overflows the instruction cache.
static __device__ __noinline__ F3 volume_grad(const Pool& P, const Volume& V, F3 pos_m) {
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
  // block neighbourhood: first block (of ll) and second block (of the largest tap)
  const int bx0 = ll.x >> 3, by0 = ll.y >> 3, bz0 = ll.z >> 3;
  const int bx1 = imx(uu.x, lu.x) >> 3, by1 = imx(uu.y, lu.y) >> 3, bz1 = imx(uu.z, lu.z) >> 3;
  int slot8[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = (c & 1) ? bx1 : bx0, by = (c & 2) ? by1 : by0, bz = (c & 4) ? bz1 : bz0;
    slot8[c] = block_slot(V, bx << 3, by << 3, bz << 3);
  }
  auto g = [&](int x, int y, int z) -> float {
    if ((unsigned)x >= (unsigned)V.size || (unsigned)y >= (unsigned)V.size ||
        (unsigned)z >= (unsigned)V.size)
      return 1.f;
    const int tx = x >> 3, ty = y >> 3, tz = z >> 3;
    int sl;
    if ((tx == bx0 || tx == bx1) && (ty == by0 || ty == by1) && (tz == bz0 || tz == bz1))
      sl = slot8[(tx != bx0 ? 1 : 0) | (ty != by0 ? 2 : 0) | (tz != bz0 ? 4 : 0)];
    else  // only when the sample position itself lies outside the volume
      sl = V.block_tab[morton3(tx, ty, tz)];
    return sl < 0 ? 1.f : __ldg(P.tsdf + (size_t)sl * 512 + voxel_index(x, y, z));
  };
#define G(X, Y, Z) g(X, Y, Z)
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

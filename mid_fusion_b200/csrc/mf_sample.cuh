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
// FIELD: 0 tsdf, 1 foreground probability, 2-4 colour r, g, b; an
// unallocated voxel reads its initial value (tsdf 1, the rest 0).
template <int FIELD>
__device__ __forceinline__ float tap_val(const Pool& P, int slot, int v) {
  if (slot < 0) return FIELD == 0 ? 1.f : 0.f;
  const size_t o = (size_t)slot * 512 + v;
  switch (FIELD) {
    case 0: return __ldg(P.tsdf + o);
    case 1: return (float)__ldg(P.fg + o);
    case 2: return __ldg(P.r + o);
    case 3: return __ldg(P.g + o);
    default: return __ldg(P.b + o);
  }
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
  switch (field) {
    case 0: return volume_interp_m<0>(P, V, pos_m, m);
    case 1: return volume_interp_m<1>(P, V, pos_m, m);
    case 2: return volume_interp_m<2>(P, V, pos_m, m);
    case 3: return volume_interp_m<3>(P, V, pos_m, m);
    default: return volume_interp_m<4>(P, V, pos_m, m);
  }
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
// at most 2 blocks per axis; their slots are resolved once.  General form,
// used when the sample's voxel lies outside the volume (see volume_grad).
static __device__ __noinline__ F3 volume_grad_generic(const Pool& P, const Volume& V, F3 pos_m) {
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

// Octree::grad with every tap inside the volume (the sample's voxel in
// [0, size)): the 48 reads touch 32 distinct voxels, which are loaded once
// each; per axis the four tap coordinates lie in at most two blocks, whose
// eight combinations are resolved once and kept in shared memory (`st`, this
// thread's column of a [8][stride] table).  Same expression, same float order.
// Not inlined: called once per accepted hit, and the raycast loop around it
// is bound by instruction fetch.
static __device__ __noinline__ F3 volume_grad(const Pool& P, const Volume& V, F3 pos_m,
                                              int* __restrict__ st, int stride) {
  const float inv = V.size / V.dim;
  const F3 pos = mk3(pos_m.x * inv, pos_m.y * inv, pos_m.z * inv);
  const F3 fl = floor3(pos);
  const I3 base = to_i3(fl);
  const int s1 = V.size - 1;
  if ((unsigned)base.x > (unsigned)s1 || (unsigned)base.y > (unsigned)s1 ||
      (unsigned)base.z > (unsigned)s1)
    return volume_grad_generic(P, V, pos_m);
  const F3 f = mk3(pos.x - fl.x, pos.y - fl.y, pos.z - fl.z);
  // tap coordinates ll, lu, ul, uu per axis (lo = lu, up = ul)
  const int cx[4] = {imx(base.x - 1, 0), base.x, imn(base.x + 1, s1), imn(base.x + 2, s1)};
  const int cy[4] = {imx(base.y - 1, 0), base.y, imn(base.y + 1, s1), imn(base.y + 2, s1)};
  const int cz[4] = {imx(base.z - 1, 0), base.z, imn(base.z + 1, s1), imn(base.z + 2, s1)};
  const int bx0 = cx[0] >> 3, by0 = cy[0] >> 3, bz0 = cz[0] >> 3;
  const int bx1 = cx[3] >> 3, by1 = cy[3] >> 3, bz1 = cz[3] >> 3;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    st[c * stride] = V.block_tab[morton3((c & 1) ? bx1 : bx0, (c & 2) ? by1 : by0,
                                         (c & 4) ? bz1 : bz0)];
  int sx[4], sy[4], sz[4], ox[4], oy[4], oz[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    sx[i] = ((cx[i] >> 3) != bx0 ? 1 : 0) * stride;
    sy[i] = ((cy[i] >> 3) != by0 ? 2 : 0) * stride;
    sz[i] = ((cz[i] >> 3) != bz0 ? 4 : 0) * stride;
    ox[i] = cx[i] & 7;
    oy[i] = (cy[i] & 7) << 3;
    oz[i] = (cz[i] & 7) << 6;
  }
  auto tap = [&](int xi, int yi, int zi) -> float {
    const int sl = st[sx[xi] + sy[yi] + sz[zi]];
    return sl < 0 ? 1.f : __ldg(P.tsdf + (size_t)sl * 512 + (ox[xi] + oy[yi] + oz[zi]));
  };
  const float t011 = tap(0, 1, 1);
  const float t012 = tap(0, 1, 2);
  const float t021 = tap(0, 2, 1);
  const float t022 = tap(0, 2, 2);
  const float t101 = tap(1, 0, 1);
  const float t102 = tap(1, 0, 2);
  const float t110 = tap(1, 1, 0);
  const float t111 = tap(1, 1, 1);
  const float t112 = tap(1, 1, 2);
  const float t113 = tap(1, 1, 3);
  const float t120 = tap(1, 2, 0);
  const float t121 = tap(1, 2, 1);
  const float t122 = tap(1, 2, 2);
  const float t123 = tap(1, 2, 3);
  const float t131 = tap(1, 3, 1);
  const float t132 = tap(1, 3, 2);
  const float t201 = tap(2, 0, 1);
  const float t202 = tap(2, 0, 2);
  const float t210 = tap(2, 1, 0);
  const float t211 = tap(2, 1, 1);
  const float t212 = tap(2, 1, 2);
  const float t213 = tap(2, 1, 3);
  const float t220 = tap(2, 2, 0);
  const float t221 = tap(2, 2, 1);
  const float t222 = tap(2, 2, 2);
  const float t223 = tap(2, 2, 3);
  const float t231 = tap(2, 3, 1);
  const float t232 = tap(2, 3, 2);
  const float t311 = tap(3, 1, 1);
  const float t312 = tap(3, 1, 2);
  const float t321 = tap(3, 2, 1);
  const float t322 = tap(3, 2, 2);
  F3 gr;
  gr.x = (((t211 - t011) * (1 - f.x) +
           (t311 - t111) * f.x) * (1 - f.y) +
          ((t221 - t021) * (1 - f.x) +
           (t321 - t121) * f.x) * f.y) * (1 - f.z) +
         (((t212 - t012) * (1 - f.x) +
           (t312 - t112) * f.x) * (1 - f.y) +
          ((t222 - t022) * (1 - f.x) +
           (t322 - t122) * f.x) * f.y) * f.z;
  gr.y = (((t121 - t101) * (1 - f.x) +
           (t221 - t201) * f.x) * (1 - f.y) +
          ((t131 - t111) * (1 - f.x) +
           (t231 - t211) * f.x) * f.y) * (1 - f.z) +
         (((t122 - t102) * (1 - f.x) +
           (t222 - t202) * f.x) * (1 - f.y) +
          ((t132 - t112) * (1 - f.x) +
           (t232 - t212) * f.x) * f.y) * f.z;
  gr.z = (((t112 - t110) * (1 - f.x) +
           (t212 - t210) * f.x) * (1 - f.y) +
          ((t122 - t120) * (1 - f.x) +
           (t222 - t220) * f.x) * f.y) * (1 - f.z) +
         (((t113 - t111) * (1 - f.x) +
           (t213 - t211) * f.x) * (1 - f.y) +
          ((t123 - t121) * (1 - f.x) +
           (t223 - t221) * f.x) * f.y) * f.z;
  const float s = V.dim / V.size;
  return gr * mk3(s, s, s) * 0.5f;
}

}  // namespace mf

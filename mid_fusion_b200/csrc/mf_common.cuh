// Device/host arithmetic and data layout shared by the MID-Fusion B200 kernels.
//
// Arithmetic follows the evaluation order of the reference's host math
// (utils/cutil_math.h, utils/math_utils.h, apps/kfusion/include/commons.h) so
// that integer outcomes (allocation keys, pixel indices, inlier tests) match
// the reference bit for bit.  The library is compiled with -fmad=false: no
// multiply-add is fused, which is how the reference's IEEE single-precision
// expressions evaluate when compiled without contraction.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MF_HD __host__ __device__ __forceinline__

namespace mf {

// ----------------------------------------------------------------- scalars
// utils/cutil_math.h:43-49: the reference's host fminf/fmaxf are plain
// comparisons (fminf(NaN, b) == b, fminf(a, NaN) == NaN), not IEEE minNum.
MF_HD float fmn(float a, float b) { return a < b ? a : b; }
MF_HD float fmx(float a, float b) { return a > b ? a : b; }
MF_HD int imn(int a, int b) { return a < b ? a : b; }
MF_HD int imx(int a, int b) { return a > b ? a : b; }
MF_HD float clampf(float f, float a, float b) { return fmx(a, fmn(f, b)); }  // cutil_math.h:981
// The reference converts float (or double) colour values to unsigned char
// implicitly (make_uchar4(float, ...)).  Out of range that is undefined
// behaviour; built with gcc for x86-64 the value goes through a 32-bit integer
// and the low byte is kept.  to_u8 does the same, so renders agree with the
// reference as built there (a direct float-to-u8 conversion on the device
// would saturate instead).
MF_HD unsigned char to_u8(float v) { return (unsigned char)(int)v; }
MF_HD unsigned char to_u8d(double v) { return (unsigned char)(int)v; }
MF_HD uchar4 u4(float x, float y, float z, float w) {
  return make_uchar4(to_u8(x), to_u8(y), to_u8(z), to_u8(w));
}
MF_HD float sq(float r) { return r * r; }

struct F3 { float x, y, z; };
struct F4 { float x, y, z, w; };
struct I3 { int x, y, z; };
struct M4 { F4 r[4]; };  // Matrix4: r[i] is row i (utils/math_utils.h:47-49)

MF_HD F3 mk3(float x, float y, float z) { F3 v; v.x = x; v.y = y; v.z = z; return v; }
MF_HD F3 mk3(float s) { return mk3(s, s, s); }
MF_HD F3 operator+(F3 a, F3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
MF_HD F3 operator-(F3 a, F3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
MF_HD F3 operator*(F3 a, F3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
MF_HD F3 operator*(F3 a, float b) { return mk3(a.x * b, a.y * b, a.z * b); }
MF_HD F3 operator*(float b, F3 a) { return mk3(b * a.x, b * a.y, b * a.z); }
MF_HD F3 operator/(F3 a, float b) { return mk3(a.x / b, a.y / b, a.z / b); }
MF_HD F3 operator+(F3 a, float b) { return mk3(a.x + b, a.y + b, a.z + b); }
MF_HD F3 operator-(float b, F3 a) { return mk3(b - a.x, b - a.y, b - a.z); }
MF_HD float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MF_HD F3 cross(F3 a, F3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
MF_HD float length(F3 v) { return sqrtf(dot(v, v)); }
// cutil_math.h:1156-1160 with the host rsqrtf (1/sqrtf), correctly rounded here.
MF_HD F3 normalize(F3 v) { const float inv = 1.0f / sqrtf(dot(v, v)); return v * inv; }
MF_HD F3 floor3(F3 v) { return mk3(floorf(v.x), floorf(v.y), floorf(v.z)); }
MF_HD F3 xyz(F4 a) { return mk3(a.x, a.y, a.z); }
MF_HD I3 to_i3(F3 a) { I3 r; r.x = (int)a.x; r.y = (int)a.y; r.z = (int)a.z; return r; }

MF_HD F3 get_translation(const M4& m) { return mk3(m.r[0].w, m.r[1].w, m.r[2].w); }
MF_HD F3 xform(const M4& M, F3 v) {  // Matrix4 * float3, utils/math_utils.h:105-110
  return mk3(dot(xyz(M.r[0]), v) + M.r[0].w, dot(xyz(M.r[1]), v) + M.r[1].w,
             dot(xyz(M.r[2]), v) + M.r[2].w);
}
MF_HD F3 rotate(const M4& M, F3 v) {  // utils/math_utils.h:112-115
  return mk3(dot(xyz(M.r[0]), v), dot(xyz(M.r[1]), v), dot(xyz(M.r[2]), v));
}
MF_HD F3 rotate_t(F3 v, const M4& M) {  // v^T M, utils/math_utils.h:117-121
  return mk3(dot(mk3(M.r[0].x, M.r[1].x, M.r[2].x), v),
             dot(mk3(M.r[0].y, M.r[1].y, M.r[2].y), v),
             dot(mk3(M.r[0].z, M.r[1].z, M.r[2].z), v));
}
MF_HD float m_at(const M4& m, int i, int j) {
  const F4& r = m.r[i];
  return j == 0 ? r.x : j == 1 ? r.y : j == 2 ? r.z : r.w;
}
MF_HD void m_set(M4& m, int i, int j, float v) {
  F4& r = m.r[i];
  if (j == 0) r.x = v; else if (j == 1) r.y = v; else if (j == 2) r.z = v; else r.w = v;
}
// 4x4 float product accumulated k = 0..3 (commons.h:657-662 via TooN).
MF_HD M4 mul(const M4& A, const M4& B) {
  M4 R;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float s = m_at(A, i, 0) * m_at(B, 0, j);
#pragma unroll
      for (int k = 1; k < 4; ++k) s += m_at(A, i, k) * m_at(B, k, j);
      m_set(R, i, j, s);
    }
  return R;
}
// commons.h:649-655 (TooN gaussian_elimination, not vendored): Gaussian
// elimination with partial pivoting on [A | I], then back substitution, float.
MF_HD M4 inverse(const M4& A) {
  // Fully unrolled so every index is a compile-time constant (registers, no
  // local memory); the pivot swap is a predicated exchange of whole rows, so the
  // arithmetic is exactly that of the plain partial-pivoting elimination.
  float a[4][4], b[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) { a[i][j] = m_at(A, i, j); b[i][j] = (i == j) ? 1.f : 0.f; }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    int p = c;
    float best = fabsf(a[c][c]);
#pragma unroll
    for (int r = c + 1; r < 4; ++r)
      if (fabsf(a[r][c]) > best) { best = fabsf(a[r][c]); p = r; }
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      if (p == r) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          float t = a[c][j]; a[c][j] = a[r][j]; a[r][j] = t;
          t = b[c][j]; b[c][j] = b[r][j]; b[r][j] = t;
        }
      }
    }
#pragma unroll
    for (int r = c + 1; r < 4; ++r) {
      const float f = a[r][c] / a[c][c];
#pragma unroll
      for (int j = c; j < 4; ++j) a[r][j] -= f * a[c][j];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[r][j] -= f * b[c][j];
    }
  }
  float R[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int r = 3; r >= 0; --r) {
      float s = b[r][j];
#pragma unroll
      for (int k = r + 1; k < 4; ++k) s -= a[r][k] * R[k][j];
      R[r][j] = s / a[r][r];
    }
  M4 out;
#pragma unroll
  for (int i = 0; i < 4; ++i) out.r[i] = F4{R[i][0], R[i][1], R[i][2], R[i][3]};
  return out;
}
// 16 floats (row-major Matrix4) from / to memory, four 4-float loads/stores
// when the pointer is 16-byte aligned.
MF_HD M4 load_m4(const float* p) {
  M4 m;
#pragma unroll
  for (int i = 0; i < 4; ++i) m.r[i] = F4{p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]};
  return m;
}
MF_HD void store_m4(float* p, const M4& m) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    p[4 * i] = m.r[i].x; p[4 * i + 1] = m.r[i].y; p[4 * i + 2] = m.r[i].z; p[4 * i + 3] = m.r[i].w;
  }
}
MF_HD M4 camera_matrix(F4 k) {  // commons.h:631-638
  M4 K;
  K.r[0] = F4{k.x, 0, k.z, 0}; K.r[1] = F4{0, k.y, k.w, 0};
  K.r[2] = F4{0, 0, 1, 0}; K.r[3] = F4{0, 0, 0, 1};
  return K;
}
MF_HD M4 inverse_camera_matrix(F4 k) {  // commons.h:640-647
  M4 K;
  K.r[0] = F4{1.0f / k.x, 0, -k.z / k.x, 0}; K.r[1] = F4{0, 1.0f / k.y, -k.w / k.y, 0};
  K.r[2] = F4{0, 0, 1, 0}; K.r[3] = F4{0, 0, 0, 1};
  return K;
}

// ----------------------------------------------------------------- Morton keys
// 64-bit key = 3 x 21-bit interleave (x bit 0, y bit 1, z bit 2) masked to the
// level's prefix, OR the level in the low 9 bits (lib/octant_ops.hpp:43-60,
// lib/utils/morton_utils.hpp:38-73, lib/octree_defines.h:38-80).
MF_HD uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}
MF_HD uint32_t gather3(uint64_t v) {
  v &= 0x1249249249249249ULL;
  v = (v | v >> 2) & 0x10c30c30c30c30c3ULL;
  v = (v | v >> 4) & 0x100f00f00f00f00fULL;
  v = (v | v >> 8) & 0x1f0000ff0000ffULL;
  v = (v | v >> 16) & 0x1f00000000ffffULL;
  v = (v | v >> 32) & 0x1fffffULL;
  return (uint32_t)v;
}
MF_HD uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
constexpr uint64_t SCALE_MASK = 0x1FF;
constexpr int MAX_LEVELS = 12;  // volumes up to 2^(12+3) voxels per side
constexpr int CAST_STACK_DEPTH = 23;

// ----------------------------------------------------------------- status
enum Status : int {
  ST_POOL_FULL = 1,        // block pool exhausted during allocation
  ST_ALLOC_OVERFLOW = 2,   // more samples emitted than the reference list holds
  ST_RAY_GUARD = 4,        // ray iterator hit its iteration guard
  ST_GN_SINGULAR = 8,      // a normal-equation system fell back to the eigen solve
  ST_ADJOINT = 16,         // a raycast adjoint skipped a ray (too many samples) or its replay differed
};

// ----------------------------------------------------------------- layout
// One contiguous block pool per GPU, shared by every instance.  Each field of
// the reference voxel (voxel_traits<SDF>, continuous/volume_traits.hpp:24-33) is
// its own plane of cap x 512 values, voxel v = x + 8y + 64z inside a block.
struct Pool {
  float* tsdf;  float* wt;  float* r;  float* g;  float* b;
  int* c;  double* fg;  int* w;
  int4* meta;          // corner voxel (x, y, z), owning instance
  uint8_t* active;     // VoxelBlock::active_
  int* count;          // slots in use (device counter)
  int cap;
};

// One octree per instance, flattened to dense per-level tables indexed by the
// Morton code of the octant at that level (child c of node m is 8m + c).
// Internal levels 1..block_level-1 hold existence flags and the eight child
// values Node::value_[8] as SoA planes; the block level holds pool slots.
struct Volume {
  int size, max_level, block_level;
  float dim;
  int32_t* block_tab;          // 8^block_level entries, -1 = unallocated
  uint8_t* node_tab;           // internal levels concatenated
  long long node_off[MAX_LEVELS];  // offset of level l (l >= 1) in node_tab
  long long n_nodes;           // entries in node_tab
  float* n_tsdf; float* n_wt; float* n_r; float* n_g; float* n_b;
  int* n_c; double* n_fg; int* n_w;  // n_nodes x 8 each
  int* bbox;                   // corners (voxels) of the allocated blocks other than
                               // block 0: min x, y, z then max x, y, z (empty: min > max)
  uint32_t* req;               // allocation requests per block-table entry
  unsigned long long* last_emit;  // (emission order << 32) | table index
  unsigned long long* emit_total;
};

MF_HD float voxel_size(const Volume& v) { return v.dim / v.size; }

// Pool slot of the block holding voxel (x, y, z); -1 when unallocated or when
// the coordinate lies outside [0, size) (the reference's bit descent aliases
// such coordinates; they only arise on rays grazing the volume boundary).
__device__ __forceinline__ int block_slot(const Volume& V, int x, int y, int z) {
  if ((unsigned)x >= (unsigned)V.size || (unsigned)y >= (unsigned)V.size ||
      (unsigned)z >= (unsigned)V.size)
    return -1;
  return V.block_tab[morton3(x >> 3, y >> 3, z >> 3)];
}
__device__ __forceinline__ int voxel_index(int x, int y, int z) {
  return (x & 7) + ((y & 7) << 3) + ((z & 7) << 6);
}

}  // namespace mf

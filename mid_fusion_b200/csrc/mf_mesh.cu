// Mesh export: marching cubes over one instance's octree, the reference's
// algorithms::marching_cube (lib/algorithms/meshing.hpp:20-208) as
// Kfusion::dump_mesh calls it (kfusion.cpp:1560-1588, inside = tsdf < 0), and
// writeVtkMesh (apps/kfusion/include/commons.h:945-1011).
//
// One CTA per allocated block, one thread per cell, two passes: the first
// counts each block's kept triangles, the second writes them at the block's
// offset in cell order (x-major, then y, then z, as the reference loops).
// Blocks are taken in Morton order.  The triangulation table is this
// project's (gen_mc_tables.py) unless the caller supplies one
// (mf_mesh_set_triangle_table: the reference's triTable gives its triangles
// one for one); the cell test, the edge intersections and the vertex bounds
// are the reference's.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "mf_internal.h"
#include "mf_mc_tables.h"

namespace mf {

// corner offsets and edges (meshing.hpp:31-74); each edge is interpolated from
// its first corner to its second
__constant__ int8_t c_corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1},
                                      {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};
__constant__ int8_t c_edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                                     {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

struct MeshArgs {
  Pool pool;
  Volume V;
  const int8_t* tris;      // triangulation table, 256 x 3 * MF_MC_MAX_TRIS edge indices
  const int* slots;        // the instance's blocks, Morton order
  int n_blocks;
  const long long* offset; // first triangle of each block (pass 2)
  int* count;              // kept triangles of each block (pass 1)
  float* out;              // 9 floats per triangle
  float bound;             // vertex bound: (int)dim as the reference, or dim
};

// get_fine (lib/octree.hpp:360-379): the voxel, or the initial value (tsdf
// 1, weight 0, fg 0, count 0) where the block is not allocated
struct Corner { float x, y; double fg; int w; };
__device__ __forceinline__ Corner corner_at(const MeshArgs& a, int x, int y, int z) {
  const int s = block_slot(a.V, x, y, z);
  if (s < 0) return Corner{1.f, 0.f, 0.0, 0};
  const size_t o = (size_t)s * 512 + voxel_index(x, y, z);
  return Corner{a.pool.tsdf[o], a.pool.wt[o], a.pool.fg[o], a.pool.w[o]};
}

// meshing::compute_intersection (meshing.hpp:20-29)
__device__ __forceinline__ F3 edge_vertex(const MeshArgs& a, const float* tsdf8, int x, int y,
                                          int z, int e) {
  const float voxelSize = a.V.dim / a.V.size;
  const int c0 = c_edge[e][0], c1 = c_edge[e][1];
  const unsigned sx = x + c_corner[c0][0], sy = y + c_corner[c0][1], sz = z + c_corner[c0][2];
  const unsigned dx = x + c_corner[c1][0], dy = y + c_corner[c1][1], dz = z + c_corner[c1][2];
  const F3 s = mk3(sx * voxelSize, sy * voxelSize, sz * voxelSize);
  const F3 d = mk3(dx * voxelSize, dy * voxelSize, dz * voxelSize);
  const float v1 = tsdf8[c0], v2 = tsdf8[c1];
  const float t = (float)(0.0 - v1);
  const F3 dd = d - s;
  const float den = v2 - v1;
  return mk3(s.x + (t * dd.x) / den, s.y + (t * dd.y) / den, s.z + (t * dd.z) / den);
}

// meshing::checkVertex (meshing.hpp:148-150), whose int dim is the
// volume's extent truncated (meshing.hpp:169)
__device__ __forceinline__ bool outside_dim(F3 p, float dim) {
  return p.x <= 0 || p.y <= 0 || p.z <= 0 || p.x > dim || p.y > dim || p.z > dim;
}

template <bool EMIT>
__global__ void __launch_bounds__(512) mesh_kernel(MeshArgs a) {
  __shared__ int s_warp[16];
  const int b = blockIdx.x;
  const int slot = a.slots[b];
  const int4 m = a.pool.meta[slot];
  const int t = threadIdx.x;
  const int x = m.x + (t >> 6), y = m.y + ((t >> 3) & 7), z = m.z + (t & 7);
  const int size = a.V.size;
  const int bound = size - 1;  // clamp(corner + 8, 0, size - 1)
  const float dim = a.bound;
  int index = 0;
  float tsdf8[8];
  if (x < min(m.x + 8, bound) && y < min(m.y + 8, bound) && z < min(m.z + 8, bound)) {
    // meshing::compute_index (meshing.hpp:76-132)
    bool ok = true;
    Corner c[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      c[i] = corner_at(a, x + c_corner[i][0], y + c_corner[i][1], z + c_corner[i][2]);
      tsdf8[i] = c[i].x;
      if (c[i].y == 0.f) ok = false;
    }
    const double fg_threshold = 0.5f;
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (c[i].fg <= fg_threshold || c[i].w <= 3) ok = false;
    if (ok)
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (c[i].x < 0.f) index |= 1 << i;
  }
  // kept triangles of this cell, in table order
  const int8_t* tr = a.tris + index * (3 * MF_MC_MAX_TRIS);
  F3 v[3 * MF_MC_MAX_TRIS];
  int kept = 0;
  for (int e = 0; e < 3 * MF_MC_MAX_TRIS && tr[e] != -1; e += 3) {
    const F3 p0 = edge_vertex(a, tsdf8, x, y, z, tr[e]);
    const F3 p1 = edge_vertex(a, tsdf8, x, y, z, tr[e + 1]);
    const F3 p2 = edge_vertex(a, tsdf8, x, y, z, tr[e + 2]);
    if (outside_dim(p0, dim) || outside_dim(p1, dim) || outside_dim(p2, dim)) continue;
    v[3 * kept] = p0;
    v[3 * kept + 1] = p1;
    v[3 * kept + 2] = p2;
    ++kept;
  }
  // exclusive scan of the cells' counts in thread (cell) order
  const int lane = t & 31, warp = t >> 5;
  int inc = kept;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += n;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (t < 32) {
    int w = t < 16 ? s_warp[t] : 0;
#pragma unroll
    for (int d = 1; d < 16; d <<= 1) {
      const int n = __shfl_up_sync(0xffffffffu, w, d);
      if (t >= d) w += n;
    }
    if (t < 16) s_warp[t] = w;  // inclusive over warps
  }
  __syncthreads();
  const int before = inc - kept + (warp > 0 ? s_warp[warp - 1] : 0);
  if (!EMIT) {
    if (t == 511) a.count[b] = before + kept;
    return;
  }
  float* o = a.out + 9 * (a.offset[b] + before);
  for (int k = 0; k < 3 * kept; ++k) {
    o[3 * k] = v[k].x;
    o[3 * k + 1] = v[k].y;
    o[3 * k + 2] = v[k].z;
  }
}

// The context's triangulation table on the device: `table` (256 rows of 16
// ints, edge triples ended by -1, the layout of the reference's triTable,
// lib/algorithms/edge_tables.h), or the built-in one when table is NULL.
int mesh_set_table(Context* ctx, const int* table) {
  int8_t t[256][3 * MF_MC_MAX_TRIS];
  if (!table) {
    std::memcpy(t, MF_MC_TRIS, sizeof(t));
  } else {
    for (int r = 0; r < 256; ++r) {
      const int* row = table + 16 * r;
      int n = 0;
      while (n < 16 && row[n] != -1) ++n;
      if (n == 16 || n % 3 != 0 || n > 3 * MF_MC_MAX_TRIS) {
        ctx->last_error = "mf_mesh_set_triangle_table: row " + std::to_string(r) +
                          " is not at most 5 edge triples ended by -1";
        return MF_E_ARG;
      }
      for (int e = 0; e < 3 * MF_MC_MAX_TRIS; ++e) {
        if (e < n && (row[e] < 0 || row[e] > 11)) {
          ctx->last_error = "mf_mesh_set_triangle_table: edge index outside 0..11 in row " +
                            std::to_string(r);
          return MF_E_ARG;
        }
        t[r][e] = e < n ? (int8_t)row[e] : (int8_t)-1;
      }
    }
  }
  if (!ctx->d_mc_tris) MF_CUDA(cudaMalloc(&ctx->d_mc_tris, sizeof(t)));
  MF_CUDA(cudaMemcpyAsync(ctx->d_mc_tris, t, sizeof(t), cudaMemcpyHostToDevice, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  return MF_OK;
}

int mesh_volume(Context* ctx, int id, int float_bounds, float* tris, long long cap,
                long long* n_tris) {
  if (!ctx->d_mc_tris)
    if (int rc = mesh_set_table(ctx, nullptr)) return rc;
  const Volume& V = ctx->inst[id].vol;
  // the instance's blocks in Morton order (the block table's own order)
  const long long n_tab = 1LL << (3 * V.block_level);
  std::vector<int32_t> tab(n_tab);
  MF_CUDA(cudaMemcpyAsync(tab.data(), V.block_tab, sizeof(int32_t) * n_tab,
                          cudaMemcpyDeviceToHost, ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  std::vector<int> slots;
  for (long long i = 0; i < n_tab; ++i)
    if (tab[i] >= 0) slots.push_back(tab[i]);
  const int nb = (int)slots.size();
  *n_tris = 0;
  if (nb == 0) return MF_OK;
  // staging: slots, counts, offsets
  const size_t sb = (sizeof(int) * nb + 15) / 16 * 16;
  if (int rc = ensure_export(ctx, 2 * sb + sizeof(long long) * nb)) return rc;
  int* d_slots = (int*)ctx->d_export;
  int* d_count = (int*)((char*)ctx->d_export + sb);
  long long* d_off = (long long*)((char*)ctx->d_export + 2 * sb);
  MF_CUDA(cudaMemcpyAsync(d_slots, slots.data(), sizeof(int) * nb, cudaMemcpyHostToDevice,
                          ctx->stream));
  MeshArgs a;
  a.tris = ctx->d_mc_tris;
  a.pool = ctx->pool;
  a.V = V;
  a.slots = d_slots;
  a.n_blocks = nb;
  a.offset = d_off;
  a.count = d_count;
  a.out = nullptr;
  a.bound = float_bounds ? V.dim : (float)(int)V.dim;
  mesh_kernel<false><<<nb, 512, 0, ctx->stream>>>(a);
  MF_CUDA(cudaGetLastError());
  std::vector<int> cnt(nb);
  MF_CUDA(cudaMemcpyAsync(cnt.data(), d_count, sizeof(int) * nb, cudaMemcpyDeviceToHost,
                          ctx->stream));
  MF_CUDA(cudaStreamSynchronize(ctx->stream));
  std::vector<long long> off(nb);
  long long total = 0;
  for (int i = 0; i < nb; ++i) { off[i] = total; total += cnt[i]; }
  *n_tris = total;
  if (!tris || cap < total || total == 0) return MF_OK;
  // the triangles: straight into a device destination, else through scratch
  cudaPointerAttributes at{};
  const bool dev = cudaPointerGetAttributes(&at, tris) == cudaSuccess &&
                   (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  float* d_out = tris;
  if (!dev) MF_CUDA(cudaMalloc(&d_out, sizeof(float) * 9 * total));
  MF_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice,
                          ctx->stream));
  a.out = d_out;
  mesh_kernel<true><<<nb, 512, 0, ctx->stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !dev)
    e = cudaMemcpyAsync(tris, d_out, sizeof(float) * 9 * total, cudaMemcpyDeviceToHost,
                        ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (!dev) cudaFree(d_out);
  if (e != cudaSuccess) {
    ctx->last_error = std::string("mf_mesh: ") + cudaGetErrorString(e);
    return MF_E_CUDA;
  }
  return MF_OK;
}

// writeVtkMesh (commons.h:945-1011) without point or cell data: every
// triangle its own three points, floats as std::ostream prints them (%g).
int write_vtk_mesh(const char* path, const float* tris, long long n) {
  FILE* f = std::fopen(path, "w");
  if (!f) return MF_E_NOT_FOUND;
  std::fprintf(f, "# vtk DataFile Version 1.0\nvtk mesh generated from KFusion\nASCII\n"
                  "DATASET POLYDATA\nPOINTS %lld FLOAT\n", 3 * n);
  for (long long i = 0; i < 3 * n; ++i)
    std::fprintf(f, "%g %g %g\n", (double)tris[3 * i], (double)tris[3 * i + 1],
                 (double)tris[3 * i + 2]);
  std::fprintf(f, "POLYGONS %lld %lld\n", n, 4 * n);
  for (long long i = 0; i < n; ++i)
    std::fprintf(f, "3 %lld %lld %lld\n", 3 * i, 3 * i + 1, 3 * i + 2);
  std::fprintf(f, "\n");
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  return ok ? MF_OK : MF_E_ARG;
}

}  // namespace mf

// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
//
// Marching cubes over one octree, following the reference's mesher
// (lib/algorithms/meshing.hpp:20-208, as Kfusion::dump_mesh calls it,
// kfusion.cpp:1560-1588): its cell test, edge intersections and vertex bounds,
// with the triangulation table the library generates from the cube's geometry
// (mid_fusion_b200/csrc/gen_mc_tables.py).  Cells are
// visited block by block in Morton order of the blocks, x-major inside a
// block.
#include <algorithm>
#include <cstdint>
#include <vector>
#include "or_volume.hpp"
#include "../mid_fusion_b200/csrc/mf_mc_tables.h"

using namespace orc;

namespace {

const int CORNER[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1},
                          {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};
// meshing.hpp:31-62: each edge from its first corner to its second
const int EDGE[12][2] = {{0, 1}, {1, 2}, {2, 3}, {0, 3}, {4, 5}, {5, 6},
                         {6, 7}, {4, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

Voxel get_fine(const Volume& v, int x, int y, int z) {
  const Voxel* p = v.voxel(x, y, z);
  return p ? *p : voxel_init();
}

// meshing::compute_index (meshing.hpp:76-132) with inside = tsdf < 0
int mc_index(const Volume& v, int x, int y, int z) {
  Voxel p[8];
  for (int i = 0; i < 8; ++i) p[i] = get_fine(v, x + CORNER[i][0], y + CORNER[i][1], z + CORNER[i][2]);
  for (int i = 0; i < 8; ++i)
    if (p[i].y == 0.f) return 0;
  const double fg_threshold = 0.5f;
  const int w_threshold = 3;
  for (int i = 0; i < 8; ++i)
    if (p[i].fg <= fg_threshold || p[i].w <= w_threshold) return 0;
  int index = 0;
  for (int i = 0; i < 8; ++i)
    if (p[i].x < 0.f) index |= 1 << i;
  return index;
}

// meshing::compute_intersection (meshing.hpp:20-29) along edge e
F3 mc_vertex(const Volume& v, int x, int y, int z, int e) {
  const float voxelSize = v.dim / v.size;
  const int* a = CORNER[EDGE[e][0]];
  const int* b = CORNER[EDGE[e][1]];
  const unsigned sx = x + a[0], sy = y + a[1], sz = z + a[2];
  const unsigned dx = x + b[0], dy = y + b[1], dz = z + b[2];
  const F3 s = mk3(sx * voxelSize, sy * voxelSize, sz * voxelSize);
  const F3 d = mk3(dx * voxelSize, dy * voxelSize, dz * voxelSize);
  const float v1 = get_fine(v, sx, sy, sz).x;
  const float v2 = get_fine(v, dx, dy, dz).x;
  return s + ((float)(0.0 - v1) * (d - s)) / (v2 - v1);
}

bool outside(F3 p, float dim) {  // meshing::checkVertex, meshing.hpp:148-150
  return p.x <= 0 || p.y <= 0 || p.z <= 0 || p.x > dim || p.y > dim || p.z > dim;
}

}  // namespace

// The triangulation table or_mesh uses: the built-in one, or a caller's
// (or_mesh_set_table: 256 x 16 ints, edge triples ended by -1).
int8_t g_tris[256][3 * MF_MC_MAX_TRIS];
bool g_tris_set = false;

extern "C" {

void or_mesh_set_table(const int* table) {
  for (int r = 0; r < 256; ++r)
    for (int e = 0; e < 3 * MF_MC_MAX_TRIS; ++e) {
      if (!table) { g_tris[r][e] = MF_MC_TRIS[r][e]; continue; }
      int n = 0;
      while (n < 16 && table[16 * r + n] != -1) ++n;
      g_tris[r][e] = e < n ? (int8_t)table[16 * r + e] : (int8_t)-1;
    }
  g_tris_set = true;
}

int or_mc_index(void* h, int x, int y, int z) {
  const Volume& v = *(const Volume*)h;
  if (v.block_index(x, y, z) < 0) return -1;
  return mc_index(v, x, y, z);
}

void or_mc_vertex(void* h, int x, int y, int z, int e, float* out) {
  const F3 p = mc_vertex(*(const Volume*)h, x, y, z, e);
  out[0] = p.x; out[1] = p.y; out[2] = p.z;
}

// Triangles (9 floats each, volume frame, metres) into out (cap triangles);
// returns the total count.  float_bounds: bound the vertices by the float
// extent instead of the reference's int one.
long long or_mesh(void* h, float* out, long long cap, int float_bounds) {
  const Volume& v = *(const Volume*)h;
  const int size = v.size;
  // meshing.hpp:169 keeps the extent as an int
  const float dim = float_bounds ? v.dim : (float)(int)v.dim;
  std::vector<std::pair<orc::key_t, int>> order;
  for (int b = 0; b < (int)v.blocks.size(); ++b) order.push_back({v.blocks[b].code, b});
  std::sort(order.begin(), order.end());
  long long n = 0;
  for (const auto& kb : order) {
    const Block& B = v.blocks[kb.second];
    const int xb = std::min(std::max(B.cx + 8, 0), size - 1);
    const int yb = std::min(std::max(B.cy + 8, 0), size - 1);
    const int zb = std::min(std::max(B.cz + 8, 0), size - 1);
    for (int x = B.cx; x < xb; ++x)
      for (int y = B.cy; y < yb; ++y)
        for (int z = B.cz; z < zb; ++z) {
          const int idx = mc_index(v, x, y, z);
          const int8_t* t = g_tris_set ? g_tris[idx] : MF_MC_TRIS[idx];
          for (int e = 0; e < 3 * MF_MC_MAX_TRIS && t[e] != -1; e += 3) {
            const F3 p0 = mc_vertex(v, x, y, z, t[e]);
            const F3 p1 = mc_vertex(v, x, y, z, t[e + 1]);
            const F3 p2 = mc_vertex(v, x, y, z, t[e + 2]);
            if (outside(p0, dim) || outside(p1, dim) || outside(p2, dim)) continue;
            if (n < cap) {
              const F3 ps[3] = {p0, p1, p2};
              for (int k = 0; k < 3; ++k) {
                out[9 * n + 3 * k] = ps[k].x;
                out[9 * n + 3 * k + 1] = ps[k].y;
                out[9 * n + 3 * k + 2] = ps[k].z;
              }
            }
            ++n;
          }
        }
  }
  return n;
}

}  // extern "C"

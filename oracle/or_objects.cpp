// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
//
// Restatement of the object spawning statistics
// (Kfusion::spawnNewObjectKernel, apps/kfusion/src/cpp/kfusion.cpp:1080-1150)
// and the semantic class fusion (Object::fuseSemanticLabel,
// apps/kfusion/src/cpp/object/object.cpp:223-252), sequential as there.
#include <cmath>
#include <cstdint>
#include <vector>
#include "or_math.hpp"

using namespace orc;

extern "C" {

// T_w_o[16], size and resolution of the new volume; returns the masked pixel
// count.  resol 0 where the reference leaves it unset.
int or_spawn_object(const float* depth, const uint8_t* mask, int W, int H, const float* k,
                    const float* T_w_c, float* T_w_o, float* volume_size, int* volume_resol) {
  const M4 invK = inverse_camera_matrix(F4{k[0], k[1], k[2], k[3]});
  const M4 T = load_m4(T_w_c);
  float x_min = INFINITY, y_min = INFINITY, z_min = INFINITY;
  float x_max = -INFINITY, y_max = -INFINITY, z_max = -INFINITY;
  float x_avg = 0, y_avg = 0, z_avg = 0;
  int count = 0;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      if (mask[x + y * W] == 0) continue;
      const float d = depth[x + y * W];
      const F3 v = d > 0 ? d * rotate(invK, mk3((float)x, (float)y, 1.f)) : mk3(0.f);
      const F3 w = T * v;
      if (w.x > x_max) x_max = w.x;
      if (w.x < x_min) x_min = w.x;
      if (w.y > y_max) y_max = w.y;
      if (w.y < y_min) y_min = w.y;
      if (w.z > z_max) z_max = w.z;
      if (w.z < z_min) z_min = w.z;
      x_avg += w.x;
      y_avg += w.y;
      z_avg += w.z;
      count++;
    }
  x_avg = x_avg / count;
  y_avg = y_avg / count;
  z_avg = z_avg / count;
  const float max_size = fmx(x_max - x_min, fmx(y_max - y_min, (z_max - z_min) / 2));
  const float size = fmn(2.5 * max_size, 5.0);
  int resol = 0;
  if (size < 0.64) resol = 256;
  if ((0.64 < size) && (size < 1.28)) resol = 512;
  if ((1.28 < size) && (size < 2.56)) resol = 1024;
  if ((2.56 < size) && (size < 5.12)) resol = 2048;
  for (int i = 0; i < 16; ++i) T_w_o[i] = (i % 5 == 0) ? 1.f : 0.f;
  T_w_o[3] = x_avg - size / 2;
  T_w_o[7] = y_avg - size / 2;
  T_w_o[11] = z_avg - size / 2;
  *volume_size = size;
  *volume_resol = resol;
  return count;
}

// fuseSemanticLabel on a fused vector in place; returns the new class id.
int or_fuse_semantics(float* fused, int n, int* fused_time, const float* probs,
                      int recog_times) {
  std::vector<float> out(n);
  for (int i = 0; i < n; ++i)
    out[i] = (fused[i] * static_cast<float>(*fused_time) + probs[i] * recog_times) /
             static_cast<float>(*fused_time + recog_times);
  int max_id = 0;
  for (int i = 1; i < n; ++i)
    if (out[i] > out[max_id]) max_id = i;
  for (int i = 0; i < n; ++i) fused[i] = out[i];
  *fused_time += recog_times;
  return max_id + 1;
}

}  // extern "C"

// TEST INFRASTRUCTURE ONLY — CPU oracle (see or_math.hpp header note).
//
// Restatement of the reference's visualisation kernels,
// apps/kfusion/src/cpp/rendering/rendering.cpp, into uchar4 (uchar3) images.
// The reference converts float colour values to unsigned char implicitly;
// gcc on x86-64 does that through a 32-bit integer keeping the low byte,
// which u8() states explicitly (and so without undefined behaviour here).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include "or_volume.hpp"

using namespace orc;

namespace {

struct U4 { unsigned char x, y, z, w; };
inline unsigned char u8(float v) { return (unsigned char)(int)v; }
inline unsigned char u8d(double v) { return (unsigned char)(int)v; }
inline U4 u4(float x, float y, float z, float w) { return U4{u8(x), u8(y), u8(z), u8(w)}; }
inline U4 c4(int x, int y, int z, int w) {
  return U4{(unsigned char)x, (unsigned char)y, (unsigned char)z, (unsigned char)w};
}

// gs2rgb, apps/kfusion/include/commons.h:87-147
U4 gs2rgb(double h) {
  double v = 0.75, r, g, b;
  double m = 0.25, sv = 0.6667;
  h *= 6.0;
  int sextant = (int)h;
  double fract = h - sextant;
  double vsf = v * sv * fract;
  double mid1 = m + vsf, mid2 = v - vsf;
  switch (sextant) {
    case 0: r = v; g = mid1; b = m; break;
    case 1: r = mid2; g = v; b = m; break;
    case 2: r = m; g = v; b = mid1; break;
    case 3: r = m; g = mid2; b = v; break;
    case 4: r = mid1; g = m; b = v; break;
    case 5: r = v; g = m; b = mid2; break;
    default: r = 0; g = 0; b = 0; break;
  }
  return U4{u8d(r * 255), u8d(g * 255), u8d(b * 255), 0};
}

}  // namespace

extern "C" {

// renderVolume_many_Kernel, rendering.cpp:489-646.  T_w_c NULL: shade the
// given maps (doraycast == false); else raycast every volume from T_w_c.
void or_render_volume(void** vols, const float* Two, const int* labels, int n,
                      const float* T_w_c, const float* k, int W, int H, float nearPlane,
                      float farPlane, float mu, float largestep, float epsilon,
                      const float* ambient, int render_color, const unsigned char* colors,
                      int n_colors, const float* vertex, const float* normal,
                      const int* label_img, const float* T_shade, unsigned char* out) {
  std::vector<M4> Tw(n), inv(n);
  for (int i = 0; i < n; ++i) { Tw[i] = load_m4(Two + 16 * i); inv[i] = inverse(Tw[i]); }
  const M4 T = load_m4(T_w_c ? T_w_c : T_shade);
  const F3 w_orgin = get_translation(T);
  const M4 view = mul(T, inverse_camera_matrix(F4{k[0], k[1], k[2], k[3]}));
  const F3 amb = mk3(ambient[0], ambient[1], ambient[2]);
  U4* o4 = (U4*)out;
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int p = x + y * W;
      F3 w_hit = mk3(0.f), w_norm = mk3(0.f), col = mk3(0.f);
      int w_label = 0;
      if (T_w_c) {
        float nearest = 1.0e10f;
        double high_fg = 0.f;
        int miss = 0;
        for (int o = 0; o < n; ++o) {
          const Volume& vol = *(const Volume*)vols[o];
          const float step = vol.dim / vol.size;
          const F3 o_origin = inv[o] * w_orgin;
          const F3 w_dir = rotate(view, mk3((float)x, (float)y, 1.f));
          const F3 o_dir = normalize(rotate(inv[o], w_dir));
          const float nfar = fmn(nearest, farPlane);
          const float t_min = ray_first_block(vol, o_origin, o_dir, nearPlane, nfar, epsilon);
          const F4 hit = t_min > 0.f ? raycast(vol, o_origin, o_dir,
                                               t_min * vol.dim / (unsigned)vol.size, nfar, mu,
                                               step, largestep)
                                     : F4{0, 0, 0, 0};
          const float hd = labels[o] == 0 ? hit.w + 0.05f : hit.w;
          if (hd > nearest) { miss++; continue; }
          const double fg = interp(vol, mk3(hit.x, hit.y, hit.z), 1);
          if (fg <= 0.5f) { miss++; continue; }
          if (hd == nearest) {
            if (fg > high_fg) high_fg = fg;
            else { miss++; continue; }
          }
          if (hit.w > 0) {
            nearest = hd;
            const F3 o_hit = mk3(hit.x, hit.y, hit.z);
            const F3 g = grad_tsdf(vol, o_hit);
            if (length(g) > 0) {
              w_norm = rotate(Tw[o], g);
              w_hit = Tw[o] * o_hit;
              w_label = labels[o];
            }
          } else {
            miss++;
          }
        }
        if (miss == n) { o4[p] = c4(0, 0, 0, 0); continue; }
      } else {
        w_hit = mk3(vertex[3 * p], vertex[3 * p + 1], vertex[3 * p + 2]);
        w_norm = mk3(normal[3 * p], normal[3 * p + 1], normal[3 * p + 2]);
        w_label = label_img[p];
      }
      for (int o = 0; o < n; ++o) {
        if (w_label != labels[o]) continue;
        const Volume& vol = *(const Volume*)vols[o];
        const F3 o_hit = inv[o] * w_hit;
        const F3 diff = normalize(w_orgin - w_hit);
        const float dir = fmx(dot(normalize(w_norm), diff), 0.f);
        if (render_color) {
          const F3 rgb = mk3(interp(vol, o_hit, 2), interp(vol, o_hit, 3), interp(vol, o_hit, 4));
          const F3 v = mk3(dir) * rgb + amb;
          col = mk3(clampf(v.x, 0.f, 1.f), clampf(v.y, 0.f, 1.f), clampf(v.z, 0.f, 1.f)) * 255;
        } else if (w_label == 0) {
          const F3 v = mk3(dir) + amb;
          col = mk3(clampf(v.x, 0.f, 1.f), clampf(v.y, 0.f, 1.f), clampf(v.z, 0.f, 1.f)) * 255;
        } else {
          const unsigned char* c = (w_label >= 0 && w_label < n_colors) ? colors + 4 * w_label
                                                                         : nullptr;
          const F3 rgb = c ? mk3(c[0], c[1], c[2]) / 255 : mk3(0.f);
          const F3 v = mk3(dir) * rgb + amb;
          col = mk3(clampf(v.x, 0.f, 1.f), clampf(v.y, 0.f, 1.f), clampf(v.z, 0.f, 1.f)) * 255;
        }
      }
      o4[p] = u4(col.x, col.y, col.z, 0.f);
    }
}

// renderDepthKernel, rendering.cpp:366-393
void or_render_depth(const float* depth, int n, float nearPlane, float farPlane,
                     unsigned char* out) {
  U4* o4 = (U4*)out;
  const float rangeScale = 1 / (farPlane - nearPlane);
  for (int p = 0; p < n; ++p) {
    if (depth[p] < nearPlane) o4[p] = c4(255, 255, 255, 0);
    else if (depth[p] > farPlane) o4[p] = c4(0, 0, 0, 0);
    else o4[p] = gs2rgb((depth[p] - nearPlane) * rangeScale);
  }
}

// renderIntensityKernel, rendering.cpp:648-664
void or_render_intensity(const float* grey, int n, unsigned char* out) {
  U4* o4 = (U4*)out;
  for (int p = 0; p < n; ++p) {
    const float gs = 255.f * grey[p];
    o4[p] = u4(gs, gs, gs, 255.f);
  }
}

// renderNormalKernel, rendering.cpp:346-364 (uchar3)
void or_render_normal(const float* normal, int n, unsigned char* out) {
  for (int p = 0; p < n; ++p) {
    F3 v = mk3(normal[3 * p], normal[3 * p + 1], normal[3 * p + 2]);
    if (v.x == -2) {
      out[3 * p] = out[3 * p + 1] = out[3 * p + 2] = 0;
    } else {
      v = normalize(v);
      out[3 * p] = u8(v.x * 128 + 128);
      out[3 * p + 1] = u8(v.y * 128 + 128);
      out[3 * p + 2] = u8(v.z * 128 + 128);
    }
  }
}

// mode 0 renderTrackKernel (:395-432), 1 renderRGBTrackKernel (:434-487),
// 2 render_RGBD_TrackKernel (:183-237); rows ICP first, then photometric
void or_render_track(const signed char* res, const float* err, int n, int mode,
                     unsigned char* out) {
  U4* o4 = (U4*)out;
  for (int p = 0; p < n; ++p) {
    if (mode == 0) {
      switch (res[p]) {
        case 1: o4[p] = c4(128, 128, 128, 0); break;
        case -1: o4[p] = c4(0, 0, 0, 0); break;
        case -2: o4[p] = c4(255, 0, 0, 0); break;
        case -3: o4[p] = c4(0, 255, 0, 0); break;
        case -4: o4[p] = c4(0, 0, 255, 0); break;
        case -5: o4[p] = c4(255, 255, 0, 0); break;
        case -6: o4[p] = c4(255, 175, 175, 0); break;
        default: o4[p] = c4(255, 200, 128, 0); break;
      }
    } else if (mode == 1) {
      float e = err[n + p];
      switch (res[n + p]) {
        case 1: e = std::fabs(e * 255.0); o4[p] = u4(e, e, e, 255.f); break;
        case -1: o4[p] = c4(0, 255, 0, 0); break;
        case -2: o4[p] = c4(0, 0, 0, 0); break;
        case -3: o4[p] = c4(255, 0, 0, 0); break;
        case -4: o4[p] = c4(0, 0, 255, 0); break;
        case -5: o4[p] = c4(255, 255, 0, 0); break;
        default: o4[p] = c4(255, 128, 128, 0); break;
      }
    } else {
      const int ri = res[p], rr = res[n + p];
      if (ri == 1 && rr == 1) {
        const float e = std::fabs(err[n + p] * 255.0);
        o4[p] = u4(e, e, e, 255.f);
      } else if ((ri < -3 && ri > -6) || (rr < -3 && rr > -6)) {
        o4[p] = c4(255, 0, 0, 0);
      } else if (ri == -2 || rr == -2) {
        o4[p] = c4(255, 255, 0, 0);
      } else if (ri == -3 || rr == -3) {
        o4[p] = c4(255, 255, 0, 0);
      } else if (ri == -1 || rr == -1) {
        o4[p] = c4(0, 255, 0, 0);
      } else if (ri == -6 || rr == -6) {
        o4[p] = c4(255, 175, 175, 0);
      } else {
        o4[p] = c4(128, 128, 128, 0);
      }
    }
  }
}

// mode 0 renderInstanceMaskKernel (:797-820), 1 renderMaskWithImageKernel
// (:679-723), 2 renderMaskMotionWithImageKernel (:725-795).  rows[label]:
// that instance's result rows (2 n), or null.  Labels outside the colour
// table read black (the reference indexes out of range there).
void or_render_mask(const int* label, const float* rgb3, int n, int mode,
                    const unsigned char* colors, int n_colors, const signed char* const* rows,
                    int n_rows, unsigned char* out) {
  U4* o4 = (U4*)out;
  const float alpha = 0.3;
  for (int p = 0; p < n; ++p) {
    const int id = label[p];
    const U4 lc = (id >= 0 && id < n_colors)
                      ? c4(colors[4 * id], colors[4 * id + 1], colors[4 * id + 2],
                           colors[4 * id + 3])
                      : c4(0, 0, 0, 0);
    if (mode == 0) { o4[p] = lc; continue; }
    const F3 rgb = mk3(rgb3[3 * p], rgb3[3 * p + 1], rgb3[3 * p + 2]) * 255.0;
    unsigned char r, g, b;
    if (mode == 1) {
      if (id == -2) {
        r = u8(rgb.x * alpha + 128 * (1 - alpha));
        g = u8(rgb.y * alpha + 128 * (1 - alpha));
        b = u8(rgb.z * 0 + 255 * (1));
      } else if (id != 0) {
        r = u8(rgb.x * alpha + lc.x * (1 - alpha));
        g = u8(rgb.y * alpha + lc.y * (1 - alpha));
        b = u8(rgb.z * alpha + lc.z * (1 - alpha));
      } else {
        r = u8(rgb.x); g = u8(rgb.y); b = u8(rgb.z);
      }
    } else {
      const signed char* rw = (id >= 0 && id < n_rows) ? rows[id] : nullptr;
      const bool outlier = rw && (rw[p] < -3 || rw[n + p] < -3);
      if (id == -2) {
        r = u8(rgb.x * alpha + 255 * (1 - alpha));
        g = u8(rgb.y * alpha + 175 * (1 - alpha));
        b = u8(rgb.z * alpha + 175 * (1 - alpha));
      } else if (id == 0) {
        if (outlier) {
          r = u8(rgb.x * alpha + 255 * (1 - alpha));
          g = u8(rgb.y * alpha + 0 * (1 - alpha));
          b = u8(rgb.z * alpha + 0 * (1 - alpha));
        } else {
          r = u8(rgb.x); g = u8(rgb.y); b = u8(rgb.z);
        }
      } else if (outlier) {
        r = u8(rgb.x); g = u8(rgb.y); b = u8(rgb.z);
      } else {
        r = u8(rgb.x * alpha + lc.x * (1 - alpha));
        g = u8(rgb.y * alpha + lc.y * (1 - alpha));
        b = u8(rgb.z * alpha + lc.z * (1 - alpha));
      }
    }
    o4[p] = U4{r, g, b, 0};
  }
}

}  // extern "C"

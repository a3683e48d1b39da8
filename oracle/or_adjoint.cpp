// TEST INFRASTRUCTURE ONLY — part of the CPU oracle (see or_math.hpp).
//
// The camera-tracking cost at pyramid level 0 as a function of the TSDF voxel
// values and of the live pose, evaluated in double (or float) precision, so
// that central differences check the device's hand-written adjoint:
//
//   E = sum_p rho(e_icp(p)) + rho(e_rgb(p)),   rho = Huber (k = 1.345)
//
// with the model maps (vertex, normal) from the composite multi-instance
// raycast at the reference pose (apps/kfusion/src/cpp/rendering/rendering.cpp:
// 9-181, kfusion/rendering_impl.hpp:80-140), the photometric reference vertex
// rendered from them (tracking.cpp:218-238), and the camera ICP / photometric
// rows of tracking.cpp:923-1020 and :1023-1111 (nearest-pixel ICP model
// lookup, bilinear live-intensity lookup, reference whitening).  The traversal
// to the first allocated block (ray_first_block) depends only on which blocks
// exist, so it is shared with the float restatement; every voxel value read
// after it goes through one accessor that can add a perturbation.
#include <cmath>
#include <vector>
#include "or_volume.hpp"

using namespace orc;

namespace oad {

template <typename T> struct V3 { T x, y, z; };
template <typename T> V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <typename T> V3<T> operator+(V3<T> a, V3<T> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> V3<T> operator-(V3<T> a, V3<T> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> V3<T> operator*(T s, V3<T> a) { return v3(s * a.x, s * a.y, s * a.z); }
template <typename T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> T len(V3<T> a) { return std::sqrt(dot(a, a)); }
template <typename T> struct Mat { T m[3][4]; };  // rigid / projective rows 0..2
template <typename T> Mat<T> from_f(const float* p) {
  Mat<T> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) r.m[i][j] = (T)p[4 * i + j];
  return r;
}
template <typename T> Mat<T> from_d(const double* p) {
  Mat<T> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) r.m[i][j] = (T)p[4 * i + j];
  return r;
}
template <typename T> V3<T> xf(const Mat<T>& M, V3<T> v) {
  return v3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z + M.m[0][3],
            M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z + M.m[1][3],
            M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z + M.m[2][3]);
}
template <typename T> V3<T> rot(const Mat<T>& M, V3<T> v) {
  return v3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z,
            M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z,
            M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z);
}
// inverse of a rigid transform
template <typename T> Mat<T> rigid_inv(const Mat<T>& M) {
  Mat<T> r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.m[i][j] = M.m[j][i];
  for (int i = 0; i < 3; ++i)
    r.m[i][3] = -(r.m[i][0] * M.m[0][3] + r.m[i][1] * M.m[1][3] + r.m[i][2] * M.m[2][3]);
  return r;
}

struct Pert {
  int inst, x, y, z;
  double d;
};

template <typename T> struct Field {
  const Volume* v;
  int inst;
  const std::vector<Pert>* pert;
  T tsdf(int x, int y, int z) const {
    const Voxel* p = v->voxel(x, y, z);
    if (!p) return (T)1;
    T r = (T)p->x;
    for (const Pert& q : *pert)
      if (q.inst == inst && q.x == x && q.y == y && q.z == z) r += (T)q.d;
    return r;
  }
  T fg(int x, int y, int z) const {
    const Voxel* p = v->voxel(x, y, z);
    return p ? (T)p->fg : (T)0;
  }
  T inv() const { return (T)v->size / (T)v->dim; }
  template <int FG> T interp(V3<T> pm) const {
    const T iv = inv();
    const V3<T> pos = v3(pm.x * iv, pm.y * iv, pm.z * iv);
    const int bx = (int)std::floor(pos.x), by = (int)std::floor(pos.y), bz = (int)std::floor(pos.z);
    const T fx = pos.x - std::floor(pos.x), fy = pos.y - std::floor(pos.y),
            fz = pos.z - std::floor(pos.z);
    const int lx = bx < 0 ? 0 : bx, ly = by < 0 ? 0 : by, lz = bz < 0 ? 0 : bz;
    T p[8];
    for (int i = 0; i < 8; ++i) {
      const int x = lx + (i & 1), y = ly + ((i >> 1) & 1), z = lz + (i >> 2);
      p[i] = FG ? fg(x, y, z) : tsdf(x, y, z);
    }
    return (((p[0] * (1 - fx) + p[1] * fx) * (1 - fy) + (p[2] * (1 - fx) + p[3] * fx) * fy) *
                (1 - fz) +
            ((p[4] * (1 - fx) + p[5] * fx) * (1 - fy) + (p[6] * (1 - fx) + p[7] * fx) * fy) * fz);
  }
  T get(V3<T> p) const {
    const T iv = inv();
    return tsdf((int)(p.x * iv), (int)(p.y * iv), (int)(p.z * iv));
  }
  V3<T> grad(V3<T> pm) const {
    const T iv = inv();
    const V3<T> pos = v3(pm.x * iv, pm.y * iv, pm.z * iv);
    const int bx = (int)std::floor(pos.x), by = (int)std::floor(pos.y), bz = (int)std::floor(pos.z);
    const T fx = pos.x - std::floor(pos.x), fy = pos.y - std::floor(pos.y),
            fz = pos.z - std::floor(pos.z);
    const int s1 = v->size - 1;
    auto mx = [](int a, int b) { return a > b ? a : b; };
    auto mn = [](int a, int b) { return a < b ? a : b; };
    const int cx[4] = {mx(bx - 1, 0), mx(bx, 0), mn(bx + 1, s1), mn(bx + 2, s1)};
    const int cy[4] = {mx(by - 1, 0), mx(by, 0), mn(by + 1, s1), mn(by + 2, s1)};
    const int cz[4] = {mx(bz - 1, 0), mx(bz, 0), mn(bz + 1, s1), mn(bz + 2, s1)};
    auto t = [&](int a, int b, int c) { return tsdf(cx[a], cy[b], cz[c]); };
    const T wx[2] = {1 - fx, fx}, wy[2] = {1 - fy, fy}, wz[2] = {1 - fz, fz};
    V3<T> g = v3<T>(0, 0, 0);
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) {
          const T w = wx[a] * wy[b] * wz[c];
          g.x += w * (t(2 + a, 1 + b, 1 + c) - t(a, 1 + b, 1 + c));
          g.y += w * (t(1 + a, 2 + b, 1 + c) - t(1 + a, b, 1 + c));
          g.z += w * (t(1 + a, 1 + b, 2 + c) - t(1 + a, 1 + b, c));
        }
    const T s = (T)v->dim / (T)v->size * (T)0.5;
    return v3(g.x * s, g.y * s, g.z * s);
  }
};

// kfusion/rendering_impl.hpp:80-140 in T.  Returns t* (0 on a miss).
template <typename T>
T march(const Field<T>& F, V3<T> o, V3<T> d, T nearp, T farp, T mu, T step, T largestep,
        V3<T>* hit) {
  const T dim = (T)F.v->dim;
  const V3<T> invR = v3((T)1 / d.x, (T)1 / d.y, (T)1 / d.z);
  const V3<T> tbot = v3(-invR.x * o.x, -invR.y * o.y, -invR.z * o.z);
  const V3<T> ttop = v3(invR.x * (dim - o.x), invR.y * (dim - o.y), invR.z * (dim - o.z));
  auto mn = [](T a, T b) { return a < b ? a : b; };
  auto mx = [](T a, T b) { return a > b ? a : b; };
  const V3<T> tmin = v3(mn(ttop.x, tbot.x), mn(ttop.y, tbot.y), mn(ttop.z, tbot.z));
  const V3<T> tmax = v3(mx(ttop.x, tbot.x), mx(ttop.y, tbot.y), mx(ttop.z, tbot.z));
  const T tnear = mx(mx(mx(tmin.x, tmin.y), mx(tmin.x, tmin.z)), nearp);
  const T tfar = mn(mn(mn(tmax.x, tmax.y), mn(tmax.x, tmax.z)), farp);
  if (!(tnear < tfar)) return 0;
  T t = tnear, stepsize = largestep;
  V3<T> pos = o + t * d;
  T f_t = F.template interp<0>(pos), f_tt = 0;
  if (!(f_t > 0)) return 0;
  for (int guard = 0; t < tfar && guard < (1 << 20); t += stepsize, ++guard) {
    f_tt = F.get(pos);
    if (f_tt < (T)0.1f && f_tt >= (T)-0.5f) f_tt = F.template interp<0>(pos);
    if (f_tt < 0) break;
    stepsize = mx(f_tt * mu, step);
    pos = pos + stepsize * d;
    f_t = f_tt;
  }
  if (!(f_tt < 0)) return 0;
  t = t + stepsize * f_tt / (f_t - f_tt);
  *hit = o + t * d;
  return t;
}

template <typename T> T huber(T e) {
  const T k = (T)1.345, a = std::fabs(e);
  return a <= k ? (T)0.5 * e * e : k * (a - (T)0.5 * k);
}

template <typename T>
double camera_cost(void** vols, const float* Two, const int* labels, int n, const float* Twr,
                   const double* Tlive, const float* k4, int W, int H, float nearp, float farp,
                   float mu, float eps, const float* lV, const float* lN, const float* lC,
                   const float* lI, const float* rI, const float* rVtx, int use_icp, int use_rgb,
                   const std::vector<Pert>& pert, double* rows) {
  const T INV = (T)-2;
  // ---- composite model maps (rendering.cpp:9-181)
  const M4 Tr = load_m4(Twr);
  const M4 view = mul(Tr, inverse_camera_matrix(F4{k4[0], k4[1], k4[2], k4[3]}));
  std::vector<V3<T>> mv((size_t)W * H), mnrm((size_t)W * H);
  std::vector<Field<T>> Fs(n);
  std::vector<Mat<T>> Tw(n);
  std::vector<M4> inv(n);
  for (int i = 0; i < n; ++i) {
    Fs[i] = Field<T>{(const Volume*)vols[i], i, &pert};
    Tw[i] = from_f<T>(Two + 16 * i);
    inv[i] = inverse(load_m4(Two + 16 * i));
  }
#pragma omp parallel for schedule(dynamic, 4)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const size_t p = (size_t)x + (size_t)y * W;
      T nearest = (T)1.0e3f;
      T high_fg = 0;
      int miss = 0;
      V3<T> vert = v3<T>(0, 0, 0), nrm = v3<T>(INV, 0, 0);
      for (int o = 0; o < n; ++o) {
        const Volume& vol = *(const Volume*)vols[o];
        const float stepf = vol.dim / vol.size;
        const F3 oo = inv[o] * get_translation(view);
        const F3 od = normalize(rotate(inv[o], rotate(view, mk3((float)x, (float)y, 1.f))));
        const T nfar = nearest < (T)farp ? nearest : (T)farp;
        const float t_min = ray_first_block(vol, oo, od, nearp, (float)nfar, eps);
        V3<T> hit = v3<T>(0, 0, 0);
        T tw = 0;
        if (t_min > 0.f)
          tw = march(Fs[o], v3<T>(oo.x, oo.y, oo.z), v3<T>(od.x, od.y, od.z),
                     (T)(t_min * vol.dim / (unsigned)vol.size), nfar, (T)mu, (T)stepf,
                     (T)stepf * 8, &hit);
        const T hd = labels[o] == 0 ? tw + (T)0.05f : tw;
        if (hd > nearest) { miss++; continue; }
        const T fg = Fs[o].template interp<1>(hit);
        if (fg <= (T)0.5f) { miss++; continue; }
        if (hd == nearest) {
          if (!(fg > high_fg)) { miss++; continue; }
        } else if (hd < nearest) {
          nearest = hd;
        } else { miss++; continue; }
        high_fg = fg;
        vert = xf(Tw[o], hit);
        const V3<T> g = Fs[o].grad(hit);
        const T gl = len(g);
        if (gl == 0) nrm.x = INV;
        else nrm = ((T)1 / gl) * rot(Tw[o], g);
      }
      if (miss == n) { vert = v3<T>(0, 0, 0); nrm = v3<T>(INV, 0, 0); }
      mv[p] = vert;
      mnrm[p] = nrm;
    }
  // ---- rows at level 0
  const Mat<T> Tl = from_d<T>(Tlive), iTl = rigid_inv(Tl);
  const Mat<T> Twr_t = from_f<T>(Twr), iTwr = rigid_inv(Twr_t);
  const T fx = (T)k4[0], fy = (T)k4[1], cx = (T)k4[2], cy = (T)k4[3];
  const T sigma_bright = (T)(float)(std::sqrt(100.0f) / 255.0);
  const T ic_rgb = (T)1 / sigma_bright;
  double E = 0, nrows = 0;
#pragma omp parallel for reduction(+ : E, nrows) schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const size_t p = (size_t)x + (size_t)y * W;
      if (use_icp && lN[3 * p] != -2.f) {
        const V3<T> nl = v3<T>(lN[3 * p], lN[3 * p + 1], lN[3 * p + 2]);
        const V3<T> pv = xf(Tl, v3<T>(lV[3 * p], lV[3 * p + 1], lV[3 * p + 2]));
        const V3<T> pc = xf(iTwr, pv);
        const T px = fx * pc.x / pc.z + cx, py = fy * pc.y / pc.z + cy;
        if (px >= 1 && px <= (T)(W - 2) && py >= 1 && py <= (T)(H - 2)) {
          const size_t q = (size_t)(unsigned)px + (size_t)(unsigned)py * W;
          const V3<T> rn = mnrm[q];
          if (rn.x != INV) {
            const V3<T> diff = mv[q] - pv;
            const V3<T> pn = rot(Tl, nl);
            if (len(diff) <= (T)0.1f && dot(pn, rn) >= (T)0.8f) {
              const T sig = rn.x * rn.x * (T)lC[3 * p] + rn.y * rn.y * (T)lC[3 * p + 1] +
                            rn.z * rn.z * (T)lC[3 * p + 2];
              const T e = std::sqrt((T)1 / sig) * dot(rn, diff);
              E += (double)huber(e);
              nrows += 1;
            }
          }
        }
      }
      if (use_rgb) {
        const V3<T> mvp = mv[p];
        const T d = mvp.z > 0 ? xf(iTwr, mvp).z : (T)0;
        if (d > 0) {
          const V3<T> rv = v3<T>(d * ((T)x - cx) / fx, d * ((T)y - cy) / fy, d);
          const V3<T> rl = v3<T>(rVtx[3 * p], rVtx[3 * p + 1], rVtx[3 * p + 2]);
          if (!(len(rv - rl) > (T)0.1f && rl.z > 0)) {
            const V3<T> lv = xf(iTl, xf(Twr_t, rv));
            const T px = fx * lv.x / lv.z + cx, py = fy * lv.y / lv.z + cy;
            if (px >= 1 && px <= (T)(W - 2) && py >= 1 && py <= (T)(H - 2)) {
              const T fx0 = std::floor(px), fy0 = std::floor(py);
              const int bx = (int)fx0, by = (int)fy0;
              const T ax = px - fx0, ay = py - fy0;
              const T i00 = lI[bx + by * W], i10 = lI[bx + 1 + by * W],
                      i01 = lI[bx + (by + 1) * W], i11 = lI[bx + 1 + (by + 1) * W];
              const T bil = i00 * (1 - ax) * (1 - ay) + i10 * (1 - ay) * ax +
                            i01 * (1 - ax) * ay + i11 * ax * ay;
              const T e = ic_rgb * ((T)rI[p] - bil);
              E += (double)huber(e);
              nrows += 1;
            }
          }
        }
      }
    }
  if (rows) *rows = nrows;
  return E;
}

}  // namespace oad

extern "C" double oa_camera_cost(void** vols, const float* Two, const int* labels, int n,
                                 const float* Twr, const double* Tlive, const float* k4, int W,
                                 int H, float nearp, float farp, float mu, float eps,
                                 const float* lV, const float* lN, const float* lC,
                                 const float* lI, const float* rI, const float* rVtx,
                                 int use_icp, int use_rgb, int fp64, const int* pert_idx,
                                 const double* pert_val, int n_pert, double* rows) {
  std::vector<oad::Pert> pert(n_pert);
  for (int i = 0; i < n_pert; ++i)
    pert[i] = oad::Pert{pert_idx[4 * i], pert_idx[4 * i + 1], pert_idx[4 * i + 2],
                        pert_idx[4 * i + 3], pert_val[i]};
  if (fp64)
    return oad::camera_cost<double>(vols, Two, labels, n, Twr, Tlive, k4, W, H, nearp, farp,
                                    mu, eps, lV, lN, lC, lI, rI, rVtx, use_icp, use_rgb, pert,
                                    rows);
  return oad::camera_cost<float>(vols, Two, labels, n, Twr, Tlive, k4, W, H, nearp, farp, mu,
                                 eps, lV, lN, lC, lI, rI, rVtx, use_icp, use_rgb, pert, rows);
}

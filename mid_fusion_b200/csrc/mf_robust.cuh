// IRLS weight and robust loss of one residual: the device's GN rows use it,
// and host builds of the same code check it against the reference.
//
// Tracking::calc_robust_weight / calc_robust_residual (apps/kfusion/src/cpp/
// tracking/tracking.cpp:1474-1532), evaluated in double and returned as float.
// None and Huber equal the reference bit for bit.  Tukey and Cauchy square in
// double here, where the reference squares through `float sq(float)`
// (utils/math_utils.h:92), i.e. rounds r / b and 1 - r^2 / b^2 to float
// first: their weights and losses differ from the reference's by at most one
// float ulp of 1 and a few ulps of the loss (the Tukey weight most, relative
// to itself, near its cutoff where it vanishes).
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define MF_ROBUST_HD __host__ __device__ __forceinline__
#else
#define MF_ROBUST_HD inline
#endif

namespace mf {

// kind: 0 none, 1 Huber (k 1.345), 2 Tukey (b 4.6851), 3 Cauchy (k 2.3849)
// (tracking.h:19-24, :343-345).
MF_ROBUST_HD void robust(float e, int kind, float& w, float& loss) {
  const double r = e;
  double wd = 1.0, l;
  switch (kind) {
    case 1: {
      const double a = fabs(r);
      if (a <= 1.345) { wd = 1.0; l = 0.5 * r * r; }
      else { wd = 1.345 / a; l = 1.345 * (a - 0.5 * 1.345); }
      break;
    }
    case 2: {
      const double b = 4.6851, a = fabs(r);
      if (a <= b) {
        const double u = 1.0 - r * r / (b * b);
        wd = u * u;
        const double v = 1.0 - (r / b) * (r / b);
        l = b * b / 6.0 * (1.0 - v * v * v);
      } else { wd = 0; l = b * b / 6.0; }
      break;
    }
    case 3: {
      const double q = (r / 2.3849) * (r / 2.3849);
      wd = 1 / (1 + q);
      l = 0.5 * 2.3849 * 2.3849 * log(1.0 + q);
      break;
    }
    default: l = 0.5 * r * r;
  }
  w = (float)wd;
  loss = (float)l;
}

}  // namespace mf

#undef MF_ROBUST_HD

// libtorch autograd Function of the camera-tracking cost and its hand-written
// adjoint (mf_camera_cost, include/midfusion_b200.h; no reference
// counterpart):
//
//   E(twist, tsdf) = cost at T_live = exp(twist) T0 of the live frame against
//                    the model raycast from the context's TSDF at the current
//                    camera pose (the reference pose)
//
// forward evaluates E through the C ABI; backward re-runs the cost with the
// adjoint (the raycast samples are recomputed there, not stored by the forward
// pass), which adds dE/d(tsdf) into a fresh gradient tensor and returns
// dE/d(eps) for a left perturbation exp(eps) T of the evaluated pose.  The
// chain rule to the twist uses the left Jacobian of SE(3) at the twist:
// dE/d twist = J_l(twist)^T dE/d eps, J_l by central differences of the SE(3)
// logarithm in double (J_l = I at twist = 0).
#include <torch/extension.h>

#include <cmath>
#include <cstring>

#include "../../include/midfusion_b200.h"

namespace {

using Mat4 = std::array<double, 16>;

Mat4 mul4(const Mat4& a, const Mat4& b) {
  Mat4 r{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += a[4 * i + k] * b[4 * k + j];
      r[4 * i + j] = s;
    }
  return r;
}

// exp of a twist (v, w), translation first: R = I + A [w]x + B [w]x^2,
// t = (I + B [w]x + C [w]x^2) v
Mat4 se3_exp(const double* xi) {
  const double w[3] = {xi[3], xi[4], xi[5]};
  const double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2], th = std::sqrt(th2);
  double A, B, C;
  if (th < 1e-8) {
    A = 1 - th2 / 6;
    B = 0.5 - th2 / 24;
    C = 1.0 / 6 - th2 / 120;
  } else {
    A = std::sin(th) / th;
    B = (1 - std::cos(th)) / th2;
    C = (1 - A) / th2;
  }
  const double W[3][3] = {{0, -w[2], w[1]}, {w[2], 0, -w[0]}, {-w[1], w[0], 0}};
  double W2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) W2[i][j] = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
  Mat4 T{};
  for (int i = 0; i < 3; ++i) {
    double t = 0;
    for (int j = 0; j < 3; ++j) {
      const double I = i == j ? 1.0 : 0.0;
      T[4 * i + j] = I + A * W[i][j] + B * W2[i][j];
      t += (I + B * W[i][j] + C * W2[i][j]) * xi[j];
    }
    T[4 * i + 3] = t;
  }
  T[15] = 1;
  return T;
}

// log of a rigid transform: (v, w), translation first
void se3_log(const Mat4& T, double* xi) {
  const double tr = T[0] + T[5] + T[10];
  const double c = std::min(1.0, std::max(-1.0, (tr - 1) / 2));
  double th = std::acos(c);
  const double sk[3] = {0.5 * (T[9] - T[6]), 0.5 * (T[2] - T[8]), 0.5 * (T[4] - T[1])};
  double w[3];
  const double f = th < 1e-8 ? 1.0 : th / std::sin(th);
  for (int i = 0; i < 3; ++i) w[i] = sk[i] * f;
  th = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  const double W[3][3] = {{0, -w[2], w[1]}, {w[2], 0, -w[0]}, {-w[1], w[0], 0}};
  double V[3][3];
  const double B = th < 1e-8 ? 0.5 : (1 - std::cos(th)) / (th * th);
  const double C = th < 1e-8 ? 1.0 / 6 : (1 - std::sin(th) / th) / (th * th);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double w2 = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
      V[i][j] = (i == j ? 1.0 : 0.0) + B * W[i][j] + C * w2;
    }
  // v = V^-1 t (Cramer's rule on the 3x3)
  const double t[3] = {T[3], T[7], T[11]};
  const double det = V[0][0] * (V[1][1] * V[2][2] - V[1][2] * V[2][1]) -
                     V[0][1] * (V[1][0] * V[2][2] - V[1][2] * V[2][0]) +
                     V[0][2] * (V[1][0] * V[2][1] - V[1][1] * V[2][0]);
  for (int k = 0; k < 3; ++k) {
    double M[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] = j == k ? t[i] : V[i][j];
    xi[k] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
             M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
             M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) / det;
  }
  for (int i = 0; i < 3; ++i) xi[3 + i] = w[i];
}

Mat4 inverse_rigid(const Mat4& T) {
  Mat4 r{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[4 * i + j] = T[4 * j + i];
  for (int i = 0; i < 3; ++i)
    r[4 * i + 3] = -(r[4 * i] * T[3] + r[4 * i + 1] * T[7] + r[4 * i + 2] * T[11]);
  r[15] = 1;
  return r;
}

// J with exp(twist + d) ~ exp(J d) exp(twist), by central differences (h = 1e-7)
void left_jacobian(const double* tw, double J[6][6]) {
  const Mat4 Ti = inverse_rigid(se3_exp(tw));
  const double h = 1e-7;
  for (int i = 0; i < 6; ++i) {
    double p[6], m[6], lp[6], lm[6];
    for (int k = 0; k < 6; ++k) p[k] = m[k] = tw[k];
    p[i] += h;
    m[i] -= h;
    se3_log(mul4(se3_exp(p), Ti), lp);
    se3_log(mul4(se3_exp(m), Ti), lm);
    for (int k = 0; k < 6; ++k) J[k][i] = (lp[k] - lm[k]) / (2 * h);
  }
}

std::array<float, 16> live_pose(const torch::Tensor& twist, const torch::Tensor& T0) {
  const auto tw = twist.detach().to(torch::kCPU, torch::kFloat64).contiguous();
  const auto b = T0.detach().to(torch::kCPU, torch::kFloat64).contiguous();
  Mat4 base;
  std::memcpy(base.data(), b.data_ptr<double>(), sizeof(base));
  const Mat4 T = mul4(se3_exp(tw.data_ptr<double>()), base);
  std::array<float, 16> f;
  for (int i = 0; i < 16; ++i) f[i] = (float)T[i];
  return f;
}

void check_rc(mf_context* ctx, int rc) {
  TORCH_CHECK(rc == MF_OK, "mf_camera_cost failed (", rc, "): ", mf_last_error(ctx));
}

}  // namespace

struct CameraCostFunction : public torch::autograd::Function<CameraCostFunction> {
  // twist: (6,) float64 (v, w); tsdf: float32 CUDA tensor, one value per pool
  // voxel (the pool's own TSDF plane, or a tensor copied into it); context:
  // the mf_context* as an integer; T0: (4, 4) float64 base pose.
  static torch::Tensor forward(torch::autograd::AutogradContext* actx, torch::Tensor twist,
                               torch::Tensor tsdf, int64_t context, torch::Tensor T0) {
    mf_context* ctx = reinterpret_cast<mf_context*>(context);
    float* pool = nullptr;
    long long n = 0;
    check_rc(ctx, mf_pool_tsdf(ctx, &pool, &n));
    TORCH_CHECK(tsdf.is_cuda() && tsdf.scalar_type() == torch::kFloat32 && tsdf.numel() == n,
                "tsdf must be a float32 CUDA tensor with one value per pool voxel");
    if (tsdf.data_ptr<float>() != pool) {
      auto pool_t = torch::from_blob(pool, {n}, tsdf.options());
      pool_t.copy_(tsdf.reshape({n}));
    }
    const auto T = live_pose(twist, T0);
    double out[8];
    check_rc(ctx, mf_camera_cost(ctx, T.data(), out, nullptr));
    actx->save_for_backward({twist, tsdf, T0});
    actx->saved_data["context"] = context;
    return torch::tensor(out[0], torch::dtype(torch::kFloat64));
  }

  static torch::autograd::tensor_list backward(torch::autograd::AutogradContext* actx,
                                               torch::autograd::tensor_list grad_out) {
    const auto saved = actx->get_saved_variables();
    const auto& twist = saved[0];
    const auto& tsdf = saved[1];
    const auto& T0 = saved[2];
    mf_context* ctx = reinterpret_cast<mf_context*>(actx->saved_data["context"].toInt());
    auto grad = torch::zeros({tsdf.numel()}, tsdf.options());
    const auto T = live_pose(twist, T0);
    double out[8];
    check_rc(ctx, mf_camera_cost(ctx, T.data(), out, grad.data_ptr<float>()));
    const auto tw = twist.detach().to(torch::kCPU, torch::kFloat64).contiguous();
    double J[6][6];
    left_jacobian(tw.data_ptr<double>(), J);
    auto g_twist = torch::zeros({6}, torch::dtype(torch::kFloat64));
    auto* g = g_twist.data_ptr<double>();
    for (int i = 0; i < 6; ++i) {
      double s = 0;
      for (int k = 0; k < 6; ++k) s += J[k][i] * out[1 + k];
      g[i] = s;
    }
    const auto gE = grad_out[0].detach().to(torch::kCPU, torch::kFloat64);
    const double scale = gE.item<double>();
    return {(g_twist * scale).to(twist.options()), (grad * scale).view_as(tsdf),
            torch::Tensor(), torch::Tensor()};
  }
};

torch::Tensor camera_cost(torch::Tensor twist, torch::Tensor tsdf, int64_t context,
                          torch::Tensor T0) {
  return CameraCostFunction::apply(twist, tsdf, context, T0);
}

// the SE(3) helpers of the backward pass, for the CPU tests
torch::Tensor se3_exp_t(torch::Tensor twist) {
  const auto tw = twist.detach().to(torch::kCPU, torch::kFloat64).contiguous();
  const Mat4 T = se3_exp(tw.data_ptr<double>());
  return torch::from_blob((void*)T.data(), {4, 4}, torch::dtype(torch::kFloat64)).clone();
}
torch::Tensor left_jacobian_t(torch::Tensor twist) {
  const auto tw = twist.detach().to(torch::kCPU, torch::kFloat64).contiguous();
  double J[6][6];
  left_jacobian(tw.data_ptr<double>(), J);
  return torch::from_blob(J, {6, 6}, torch::dtype(torch::kFloat64)).clone();
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) {
  m.def("camera_cost", &camera_cost,
        "E = camera_cost(twist, tsdf, context_ptr, T0): the camera-tracking cost with "
        "its hand-written adjoint as a libtorch autograd Function");
  m.def("se3_exp", &se3_exp_t, "exp of a twist (v, w), translation first");
  m.def("left_jacobian", &left_jacobian_t, "left Jacobian of SE(3) at a twist");
}

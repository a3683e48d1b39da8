"""SE(3) helpers of the autograd wrapper and of its libtorch extension (CPU
only)."""
import numpy as np
import torch

from mid_fusion_b200.autograd import left_jacobian, se3_log
from mid_fusion_b200.scene import se3_exp


def test_log_inverts_exp():
    rng = np.random.default_rng(1)
    for _ in range(20):
        xi = np.concatenate([rng.normal(size=3) * 0.5, rng.normal(size=3) * 0.8])
        np.testing.assert_allclose(se3_log(se3_exp(xi)), xi, atol=1e-9)


def test_left_jacobian():
    np.testing.assert_allclose(left_jacobian(np.zeros(6)), np.eye(6), atol=1e-8)
    xi = np.array([0.1, -0.2, 0.05, 0.3, 0.1, -0.2])
    J = left_jacobian(xi)
    d = np.array([1e-6, -2e-6, 3e-6, -1e-6, 2e-6, 1e-6])
    # exp(xi + d) ~ exp(J d) exp(xi)
    lhs = se3_exp(xi + d)
    rhs = se3_exp(J @ d) @ se3_exp(xi)
    np.testing.assert_allclose(lhs, rhs, atol=1e-11)


def test_libtorch_extension_helpers_match():
    """The libtorch extension (csrc_torch/mf_autograd.cpp) loads without a GPU,
    exports the autograd Function's entry point, and its SE(3) exponential and
    left Jacobian equal the Python ones."""
    from mid_fusion_b200 import autograd as A
    ext = A._extension()
    assert callable(ext.camera_cost)
    rng = np.random.default_rng(3)
    for _ in range(5):
        xi = np.concatenate([rng.normal(size=3) * 0.3, rng.normal(size=3) * 0.4])
        np.testing.assert_allclose(ext.se3_exp(torch.from_numpy(xi)).numpy(), se3_exp(xi),
                                   atol=1e-12)
        np.testing.assert_allclose(ext.left_jacobian(torch.from_numpy(xi)).numpy(),
                                   left_jacobian(xi), atol=1e-7)
    np.testing.assert_allclose(ext.left_jacobian(torch.zeros(6, dtype=torch.float64)).numpy(),
                               np.eye(6), atol=1e-8)

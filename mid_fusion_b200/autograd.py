"""torch.autograd wrapper of the camera-tracking cost and its hand-written
adjoint (mf_camera_cost in include/midfusion_b200.h).

    E(twist, tsdf) = cost at T_live = exp(twist) T0 of the live frame against
                     the model raycast from the context's TSDF at the current
                     camera pose (the reference pose)

The TSDF parameter is the pool's own TSDF plane seen as a torch tensor
(``pool_tsdf_tensor``): optimising it edits the map in place.  The forward
pass evaluates the cost; the backward pass re-runs it with the adjoint (the
raycast samples are recomputed there, not stored by the forward pass).

The device returns dE/d(eps) for a left perturbation exp(eps) T at the
evaluated pose T.  For T = exp(twist) T0 the chain rule needs the left
Jacobian of SE(3) at the twist: d E / d twist = J_l(twist)^T d E / d eps, with
J_l evaluated by central differences of the SE(3) logarithm in FP64 (exact to
~1e-9 relative; J_l = I at twist = 0).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .scene import se3_exp


class _DeviceArray:
    """A raw device allocation presented through __cuda_array_interface__."""

    def __init__(self, ptr, n, typestr="<f4"):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3}


def pool_tsdf_tensor(context):
    """The context's pool TSDF values (pool capacity x 512 float32, voxel v of
    pool slot s at s * 512 + v) as a torch tensor sharing the device memory."""
    ptr, n = context.pool_tsdf()
    return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")


def se3_log(T):
    """Twist (v, w), translation first, of a rigid 4x4 transform."""
    R, t = T[:3, :3], T[:3, 3]
    c = min(1.0, max(-1.0, (np.trace(R) - 1.0) / 2.0))
    th = math.acos(c)
    W = 0.5 * (R - R.T)
    if th < 1e-8:
        w = np.array([W[2, 1], W[0, 2], W[1, 0]])
    else:
        w = np.array([W[2, 1], W[0, 2], W[1, 0]]) * th / math.sin(th)
    th = float(np.linalg.norm(w))
    Wx = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if th < 1e-8:
        V = np.eye(3) + 0.5 * Wx
    else:
        B = (1 - math.cos(th)) / th ** 2
        C = (1 - math.sin(th) / th) / th ** 2
        V = np.eye(3) + B * Wx + C * Wx @ Wx
    return np.concatenate([np.linalg.solve(V, t), w])


def left_jacobian(twist, h=1e-7):
    """J with exp(twist + d) ~ exp(J d) exp(twist), by central differences."""
    twist = np.asarray(twist, np.float64)
    Ti = np.linalg.inv(se3_exp(twist))
    J = np.zeros((6, 6))
    for i in range(6):
        e = np.zeros(6)
        e[i] = h
        J[:, i] = (se3_log(se3_exp(twist + e) @ Ti) - se3_log(se3_exp(twist - e) @ Ti)) / (2 * h)
    return J


_EXT = None


def _extension():
    """The libtorch autograd Function (csrc_torch/mf_autograd.cpp), loaded
    from its in-tree build; there is no Python fallback."""
    global _EXT
    if _EXT is None:
        import importlib.machinery
        import importlib.util
        import os
        from . import build as B
        path = B.torch_ext_path()
        if not os.path.exists(path):
            raise RuntimeError(f"libtorch extension not built: {path} "
                               "(run python -m mid_fusion_b200.build)")
        loader = importlib.machinery.ExtensionFileLoader(B.TORCH_EXT_NAME, path)
        spec = importlib.util.spec_from_file_location(B.TORCH_EXT_NAME, path, loader=loader)
        mod = importlib.util.module_from_spec(spec)
        loader.exec_module(mod)
        _EXT = mod
    return _EXT


class CameraCost:
    """E = CameraCost.apply(twist, tsdf, context, T0): the camera-tracking
    cost as a libtorch torch::autograd::Function (CameraCostFunction in
    csrc_torch/mf_autograd.cpp), whose backward runs the hand-written adjoint.

    twist: (6,) float64 tensor (v, w); tsdf: the tensor from pool_tsdf_tensor
    (or any float32 CUDA tensor of the same length, which is copied into the
    pool first); context: a capi.Context with a preprocessed live frame and a
    reference frame; T0: 4x4 base pose (numpy)."""

    @staticmethod
    def apply(twist, tsdf, context, T0):
        import ctypes
        T0t = torch.as_tensor(np.asarray(T0, np.float64))
        ptr = ctypes.cast(context.h, ctypes.c_void_p).value
        return _extension().camera_cost(twist, tsdf, int(ptr), T0t)

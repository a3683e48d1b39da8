"""TEST / BASELINE INFRASTRUCTURE ONLY: the CPU frame pipeline used as the
reported CPU baseline (bench.py's cpu_baseline leg and --impl reference arm).

One frame = the reference's per-frame order (apps/kfusion/src/benchmark.cpp:113-159):
camera tracking (Tracking::trackLiveFrame) and object tracking
(Tracking::trackEachObject) against the last raycast, then
Object::integrate_volume_kernel for every instance and raycastObjectList.

kind "reference": allocation, integration and raycast run the reference's own
code (lib/ + the header-only SDF kernels, compiled with OpenMP into
oracle/_ref/libmf_ref_omp.so); tracking runs this project's restatement,
because the reference's tracking needs TooN / OpenCV, which are not available.
kind "port": everything runs the restatement (oracle/liboracle.so).
Both use every host thread through OpenMP, as the reference does.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OMP = os.path.join(HERE, "_ref", "libmf_ref_omp.so")


def _tests_path():
    p = os.path.join(os.path.dirname(HERE), "tests")
    if p not in sys.path:
        sys.path.insert(0, p)


class CpuPipeline:
    def __init__(self, scene, use_reference=True, fp64=False):
        _tests_path()
        import _oracle as O
        self.O = O
        self.s = scene
        self.kind = "port"
        impl = O.oracle()
        if use_reference and os.path.exists(REF_OMP):
            impl = O.Impl(REF_OMP, "ref_")
            impl.lib.ref_pin_epsilon(scene.instances[0].size)
            self.kind = "reference"
        self.impl = impl
        s = scene
        self.vols = [impl.volume(i.size, i.dim) for i in s.instances]
        self.labels = [i.label for i in s.instances]
        self.trk = O.Tracker(s.width, s.height, s.k, robust=1, fp64=fp64)
        # labels of the object instances: their model pixels are ICP outliers
        # of the camera (trackLiveFrame's mask variant, tracking.cpp:1750-1879)
        self.moving = [i.label for i in s.instances[1:]]
        H, W = s.height, s.width
        self.vertex = np.zeros((H, W, 3), np.float32)
        self.normal = np.zeros((H, W, 3), np.float32)
        self.label_img = np.zeros((H, W), np.int32)
        self.T = s.cam_poses[0].astype(np.float32)
        self.poses = [P.astype(np.float32) for P in s.volume_poses(0)]
        self.frame = 0

    def step(self, depth, rgb, labels):
        from mid_fusion_b200.scene import generalize_masks
        s = self.s
        self.trk.set_frame(rgb, depth)
        if self.frame > 0:
            T_prev = self.T
            self.trk.set_mask((np.isin(self.label_img, self.moving) * 255).astype(np.uint8))
            self.T = self.trk.track_camera(T_prev, T_prev, self.vertex,
                                           self.normal).astype(np.float32)
            for i in range(1, len(self.vols)):
                self.poses[i] = self.trk.track_object(self.poses[i], self.T, T_prev, self.vertex,
                                                      self.normal, self.label_img,
                                                      self.labels[i]).astype(np.float32)
        masks = generalize_masks(labels, self.labels)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(self.vols):
            v.integrate(depth, rgb3, masks[i], self.T, self.poses[i], s.k, 0.1)
        self.impl.raycast_objects(self.vols, self.poses, self.labels, self.T, s.k, s.width,
                                  s.height, eps_size=s.instances[0].size, vertex=self.vertex,
                                  normal=self.normal, label_img=self.label_img)
        self.trk.set_ref()
        self.frame += 1


def threads():
    n = os.environ.get("OMP_NUM_THREADS")
    return int(n) if n else (os.cpu_count() or 1)


def time_frames(scene, frames, n_first, n_timed, use_reference=True):
    """Runs frames [0, n_first + n_timed); times the last n_timed.  Returns
    (seconds per frame, kind)."""
    p = CpuPipeline(scene, use_reference)
    t = []
    for f in range(n_first + n_timed):
        d, rgb, lab = frames[f]
        t0 = time.perf_counter()
        p.step(d, rgb, lab)
        if f >= n_first:
            t.append(time.perf_counter() - t0)
    return float(np.mean(t)), p.kind

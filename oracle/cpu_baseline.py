"""TEST / BASELINE INFRASTRUCTURE ONLY: the CPU frame pipeline used as the
reported CPU baseline (bench.py's cpu_baseline leg and --impl reference arm),
and the per-frame pose check of the bench's cpu_baseline leg.

One frame = the reference's per-frame order (apps/kfusion/src/benchmark.cpp:113-159,
Kfusion::tracking / integration / raycasting): preprocessing, camera tracking
(Tracking::trackLiveFrame, masked by the object pixels of the last raycast as in
kfusion.cpp:370-400) and object tracking (Tracking::trackEachObject) against the
last raycast, then Object::integrate_volume_kernel for every instance and
raycastObjectList.

kind "reference": every stage runs the reference's own code, compiled
unmodified with OpenMP from apps/kfusion/src/cpp/{tracking,preprocessing,object,
rendering} and lib/ into oracle/_ref/libmf_ref_track_omp.so (the reference's
Release flags, -g -O1) or libmf_ref_track_omp_o3.so (-O3).
kind "port": everything runs the project's restatement (oracle/liboracle.so).
Both use every host thread through OpenMP, as the reference does.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BUILDS = {"stock": os.path.join(HERE, "_ref", "libmf_ref_track_omp.so"),
              "o3": os.path.join(HERE, "_ref", "libmf_ref_track_omp_o3.so")}


def _tests_path():
    p = os.path.join(os.path.dirname(HERE), "tests")
    if p not in sys.path:
        sys.path.insert(0, p)


def reference_available(build="stock"):
    return os.path.exists(REF_BUILDS[build])


class CpuPipeline:
    def __init__(self, scene, use_reference=True, fp64=False, build="stock"):
        _tests_path()
        import _oracle as O
        self.O = O
        self.s = s = scene
        H, W = s.height, s.width
        self.labels = [i.label for i in s.instances]
        # object pixels of the last raycast are ICP outliers of the camera
        self.moving = [i.label for i in s.instances[1:]]
        self.vertex = np.zeros((H, W, 3), np.float32)
        self.normal = np.zeros((H, W, 3), np.float32)
        self.label_img = np.zeros((H, W), np.int32)
        self.T = s.cam_poses[0].astype(np.float32)
        self.poses = [P.astype(np.float32) for P in s.volume_poses(0)]
        self.frame = 0
        if use_reference and reference_available(build):
            self.kind = "reference"
            lib = O.reference_tracking(REF_BUILDS[build])
            # the direction epsilon of the reference's ray iterator comes from
            # the first octree it traverses: the background's
            lib.rt_pin_epsilon(s.instances[0].size)
            self.trk = O.RefTracker(W, H, s.k, robust=1, lib=lib)
            self.objs = [O.RefObject(self.trk, P, size=i.size, dim=i.dim, label=i.label)
                         for i, P in zip(s.instances, self.poses)]
            self.render = O.RefRender(W, H, lib=lib)
        else:
            self.kind = "port"
            self.impl = O.oracle()
            self.vols = [self.impl.volume(i.size, i.dim) for i in s.instances]
            self.trk = O.Tracker(W, H, s.k, robust=1, fp64=fp64)

    def step(self, depth, rgb, labels):
        from mid_fusion_b200.scene import generalize_masks
        s = self.s
        mask = (np.isin(self.label_img, self.moving) * 255).astype(np.uint8)
        masks = generalize_masks(labels, self.labels)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        if self.kind == "reference":
            self.trk.set_frame(rgb, depth)
            if self.frame > 0:
                T_prev = self.T
                self.T = self.trk.track_camera(T_prev, T_prev, self.vertex, self.normal,
                                               mask=mask)
                for o in self.objs[1:]:
                    self.trk.track_object(o, self.T, T_prev)
            for i, o in enumerate(self.objs):
                o.integrate(depth, rgb3, masks[i], self.T, s.k, 0.1, self.frame)
            self.vertex, self.normal, self.label_img = self.render.raycast(self.objs, self.T, s.k)
            self.poses = [o.pose()[0] for o in self.objs]
        else:
            self.trk.set_frame(rgb, depth)
            if self.frame > 0:
                T_prev = self.T
                self.trk.set_mask(mask)
                self.T = self.trk.track_camera(T_prev, T_prev, self.vertex,
                                               self.normal).astype(np.float32)
                for i in range(1, len(self.vols)):
                    self.poses[i] = self.trk.track_object(
                        self.poses[i], self.T, T_prev, self.vertex, self.normal, self.label_img,
                        self.labels[i]).astype(np.float32)
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


def cpu_model():
    """The host CPU's model name (the first `model name` of /proc/cpuinfo), or
    None where it cannot be read."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def time_frames(scene, frames, n_first, n_timed, use_reference=True, build="stock"):
    """Runs frames [0, n_first + n_timed); times the last n_timed.  Returns
    (seconds per frame, kind)."""
    p = CpuPipeline(scene, use_reference, build=build)
    t = []
    for f in range(n_first + n_timed):
        d, rgb, lab = frames[f]
        t0 = time.perf_counter()
        p.step(d, rgb, lab)
        if f >= n_first:
            t.append(time.perf_counter() - t0)
    return float(np.mean(t)), p.kind


def _pose_err(A, B):
    """(translation distance in m, rotation angle in rad) between two poses."""
    A = np.asarray(A, np.float64)
    B = np.asarray(B, np.float64)
    dt = float(np.linalg.norm(A[:3, 3] - B[:3, 3]))
    R = A[:3, :3].T @ B[:3, :3]
    # the angle from both the skew part (accurate for small angles) and the trace
    w = 0.5 * np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    return dt, float(np.arctan2(np.linalg.norm(w), 0.5 * (np.trace(R) - 1.0)))


def pose_check(scene, frames, gpu_cam, gpu_obj, gpu_maps, n, tol=1e-5):
    """Per-frame pose agreement from the same start: for frames 1..n, the
    reference's tracker (serial parity build of tracking.cpp) and the all-FP64
    oracle each track frame f from the device's frame f-1 pose, model maps and
    object poses; the result is compared with the device's frame f poses.
    gpu_cam[f] (4x4), gpu_obj[f] (K x 4 x 4), gpu_maps[f] = (vertex, normal,
    label) after frame f.  Returns the max errors over the frames (m / rad),
    camera and objects separately, of device vs reference, device vs FP64 and
    reference vs FP64; one record per (frame, problem) with the three errors;
    and the criterion: a pose passes when it lies within `tol` of the
    reference's and of the FP64 oracle's, widened by twice the reference's
    own distance r to the FP64 oracle (where the reference's single-precision
    rounding already moves it by r, another summation order lands elsewhere
    within about r of the exact answer)."""
    _tests_path()
    import _oracle as O
    s = scene
    W, H = s.width, s.height
    labels = [i.label for i in s.instances]
    out = {k: {"camera_m": 0.0, "camera_rad": 0.0, "objects_m": 0.0, "objects_rad": 0.0}
           for k in ("device_vs_reference", "device_vs_fp64_oracle",
                     "reference_vs_fp64_oracle")}
    records = []

    def upd(key, part, e):
        out[key][part + "_m"] = max(out[key][part + "_m"], e[0])
        out[key][part + "_rad"] = max(out[key][part + "_rad"], e[1])

    def record(f, what, T_dev, T_ref, T_64):
        e64 = _pose_err(T_dev, T_64)
        rec = {"frame": f, "problem": what, "device_vs_fp64": [round(v, 9) for v in e64]}
        if T_ref is not None:
            er, r64 = _pose_err(T_dev, T_ref), _pose_err(T_ref, T_64)
            rec["device_vs_reference"] = [round(v, 9) for v in er]
            rec["reference_vs_fp64"] = [round(v, 9) for v in r64]
            rec["within_tol_of_reference"] = bool(max(er) <= tol)
            rec["passes"] = bool(all(max(er[k], e64[k]) <= tol + 2 * r64[k] for k in (0, 1)))
        records.append(rec)

    have_ref = O.reference_tracking() is not None
    for f in range(1, n + 1):
        d0, rgb0, _ = frames[f - 1]
        d1, rgb1, _ = frames[f]
        vm, nm, lm = gpu_maps[f - 1]
        T_prev = np.asarray(gpu_cam[f - 1], np.float32)
        mask = (np.isin(lm, labels[1:]) * 255).astype(np.uint8)
        D = O.Tracker(W, H, s.k, robust=1, fp64=True)
        D.set_frame(rgb0, d0)
        D.set_ref()
        D.set_frame(rgb1, d1)
        D.set_mask(mask)
        Td = D.track_camera(T_prev, T_prev, vm, nm)
        upd("device_vs_fp64_oracle", "camera", _pose_err(gpu_cam[f], Td))
        Tr = None
        if have_ref:
            R = O.RefTracker(W, H, s.k)
            R.set_frame(rgb0, d0)
            R.set_ref()
            R.set_frame(rgb1, d1)
            Tr = R.track_camera(T_prev, T_prev, vm, nm, mask=mask)
            upd("device_vs_reference", "camera", _pose_err(gpu_cam[f], Tr))
            upd("reference_vs_fp64_oracle", "camera", _pose_err(Tr, Td))
        record(f, "camera", gpu_cam[f], Tr, Td)
        Tc = np.asarray(gpu_cam[f], np.float32)
        for i, label in enumerate(labels[1:], 1):
            if not np.any(lm == label):
                continue
            P_prev = np.asarray(gpu_obj[f - 1][i], np.float32)
            Pd = D.track_object(P_prev, Tc, T_prev, vm, nm, lm, label)
            upd("device_vs_fp64_oracle", "objects", _pose_err(gpu_obj[f][i], Pd))
            Pr = None
            if have_ref:
                sel = (lm == label)[..., None]
                mv = np.where(sel, vm, np.float32(0)).astype(np.float32)
                mn = np.where(sel, nm, np.array([-2.0, 0, 0], np.float32)).astype(np.float32)
                ob = R.object(P_prev, mv, mn)
                Pr, _ = R.track_object(ob, Tc, T_prev)
                upd("device_vs_reference", "objects", _pose_err(gpu_obj[f][i], Pr))
                upd("reference_vs_fp64_oracle", "objects", _pose_err(Pr, Pd))
            record(f, f"object {i}", gpu_obj[f][i], Pr, Pd)
    if not have_ref:
        del out["device_vs_reference"], out["reference_vs_fp64_oracle"]
    else:
        out["within_tol_of_reference"] = sum(r["within_tol_of_reference"] for r in records)
        out["passes_criterion"] = sum(r["passes"] for r in records)
    out["problems"] = len(records)
    out["tol"] = tol
    out["frames"] = n
    out["records"] = records
    return out

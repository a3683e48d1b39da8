"""TEST INFRASTRUCTURE ONLY: precision study of the mixed-precision pipeline
over a long sequence (300 frames of the 640x480 three-object workload against
an all-FP64 oracle run; a study script run on a GPU host, not a test).

The bench's scene (640x480, background 512^3 @ 1 cm + 3 objects 256^3 @ 2 mm,
each with its own twist) for many frames through the device pipeline
(mf_process_frame, batched: FP32 per-pixel rows, FP64 reductions, 6x6 solve
and SE(3) update, FP32 maps), compared with the oracles in one of two ways:

* --mode reseeded (per frame, from the same start): frame f is tracked again
  by the reference's tracking.cpp (oracle/_ref, when built) and by the
  all-FP64 oracle from the device's frame f-1 pose, model maps and object
  poses (oracle/cpu_baseline.py pose_check); reported per frame: device vs
  reference, device vs FP64 and reference vs FP64, camera and objects.  The
  device's volumes are also integrated by the oracle at the device's poses
  every `--tsdf-every` frames and compared (TSDF in units of mu; the mapping
  is bit-exact, so 0 is expected).
* --mode closed: the oracle pipeline with all-FP64 tracking
  (oracle/cpu_baseline.py with fp64=True; mapping in the reference's single
  precision) as an independent closed loop from the same frames; reported per
  frame: the pose differences, each loop's camera drift from ground truth,
  and every `--tsdf-every` frames the largest TSDF difference on blocks both
  hold and the number of blocks only one holds.  Differences compound.

    python oracle/precision_study.py --frames 300 --mode reseeded > study.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, HERE, os.path.join(ROOT, "tests")]


def _scene(n, W, H):
    from mid_fusion_b200.scene import make_scene
    return make_scene("multi", W, H, n_frames=n, seed=11, n_objects=3, bg_size=512, bg_dim=5.12,
                      obj_size=256, obj_dim=0.512)


def _render(a):
    f, n, W, H = a
    return (f,) + tuple(_scene(n, W, H).render(f))


def rot_err(A, B):
    R = np.linalg.solve(np.asarray(A, np.float64)[:3, :3], np.asarray(B, np.float64)[:3, :3])
    return float(np.linalg.norm(0.5 * np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0],
                                                R[1, 0] - R[0, 1]])))


def tsdf_diff(ctx, vols, i):
    kg, _, _, xg = ctx.blocks(i)
    ko, _, _, xo = vols[i].blocks()
    common, ig, io = np.intersect1d(kg, ko, return_indices=True)
    d = float(np.abs(xg["x"][ig] - xo["x"][io]).max()) if len(common) else 0.0
    return d, int(len(kg) + len(ko) - 2 * len(common))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=300)
    ap.add_argument("--width", type=int, default=640)
    ap.add_argument("--tsdf-every", type=int, default=25)
    ap.add_argument("--workers", type=int, default=min(32, os.cpu_count() or 4))
    ap.add_argument("--mode", default="reseeded", choices=["reseeded", "closed"])
    a = ap.parse_args()
    W, H = a.width, a.width * 3 // 4
    with mp.get_context("spawn").Pool(a.workers) as pool:
        frames = sorted(pool.map(_render, [(f, a.frames, W, H) for f in range(a.frames)]))
    import torch  # noqa: F401
    import cpu_baseline as CB
    from mid_fusion_b200.capi import Context
    s = _scene(a.frames, W, H)
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 18, batched=True, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    n = len(s.instances)
    if a.mode == "reseeded":
        return reseeded(a, s, ctx, frames, n, CB)
    cpu = CB.CpuPipeline(s, use_reference=False, fp64=True)
    rows = []
    for f, d, rgb, lab in frames:
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        assert ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                        np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                        lab16.ctypes.data_as(C.c_void_p)) == 0
        Tc = np.zeros(16, np.float32)
        To = np.zeros(16 * n, np.float32)
        ctx.lib.mf_get_poses(ctx.h, Tc.ctypes.data_as(C.c_void_p), To.ctypes.data_as(C.c_void_p))
        Tc, To = Tc.reshape(4, 4), To.reshape(n, 4, 4)
        cpu.step(d, rgb, lab)
        gt = s.cam_poses[f]
        row = {"frame": f,
               "cam_dt_m": float(np.linalg.norm(Tc[:3, 3] - cpu.T[:3, 3])),
               "cam_dr_rad": rot_err(Tc, cpu.T),
               "obj_dt_m": max([float(np.linalg.norm(To[i][:3, 3] - cpu.poses[i][:3, 3]))
                                for i in range(1, n)] or [0.0]),
               "drift_device_m": float(np.linalg.norm(Tc[:3, 3] - gt[:3, 3])),
               "drift_oracle_m": float(np.linalg.norm(cpu.T[:3, 3] - gt[:3, 3]))}
        if f % a.tsdf_every == 0 or f == a.frames - 1:
            diffs = [tsdf_diff(ctx, cpu.vols, i) for i in range(n)]
            row["tsdf_maxdiff_mu"] = max(x[0] for x in diffs)
            row["blocks_only_one"] = sum(x[1] for x in diffs)
        rows.append(row)
    def at(f):
        return rows[min(f, len(rows) - 1)]
    summary = {"frames": a.frames, "frame_size": [W, H], "status": ctx.status(),
               "at": {str(f): at(f) for f in (1, 10, 50, 100, 200, a.frames - 1)
                      if f < a.frames}}
    print(json.dumps({"summary": summary, "per_frame": rows}))


def reseeded(a, s, ctx, frames, n, CB):
    import _oracle as O
    from mid_fusion_b200.scene import generalize_masks
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vols = [orc.volume(i.size, i.dim) for i in s.instances]
    rows, prev = [], None
    for f, d, rgb, lab in frames:
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        assert ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                        np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                        lab16.ctypes.data_as(C.c_void_p)) == 0
        Tc = np.zeros(16, np.float32)
        To = np.zeros(16 * n, np.float32)
        ctx.lib.mf_get_poses(ctx.h, Tc.ctypes.data_as(C.c_void_p), To.ctypes.data_as(C.c_void_p))
        cur = (Tc.reshape(4, 4), To.reshape(n, 4, 4), ctx.download_raycast())
        # the oracle's integration at the device's poses (bit-exact mapping)
        masks = generalize_masks(lab, labels)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(d, rgb3, masks[i], cur[0], cur[1][i], s.k, 0.1)
        row = {"frame": f,
               "drift_device_m": float(np.linalg.norm(cur[0][:3, 3] - s.cam_poses[f][:3, 3]))}
        if prev is not None:
            chk = CB.pose_check(s, [frames[f - 1][1:], (d, rgb, lab)], [prev[0], cur[0]],
                                [prev[1], cur[1]], [prev[2], cur[2]], 1)
            row.update({k: v for k, v in chk.items() if k != "frames"})
        if f % a.tsdf_every == 0 or f == len(frames) - 1:
            diffs = [tsdf_diff(ctx, vols, i) for i in range(n)]
            row["tsdf_maxdiff_mu"] = max(x[0] for x in diffs)
            row["blocks_only_one"] = sum(x[1] for x in diffs)
        rows.append(row)
        prev = cur
    keys = ("device_vs_reference", "device_vs_fp64_oracle", "reference_vs_fp64_oracle")
    worst = {k: {m: max(r[k][m] for r in rows if k in r) for m in
                 ("camera_m", "camera_rad", "objects_m", "objects_rad")}
             for k in keys if any(k in r for r in rows)}
    summary = {"mode": "reseeded", "frames": len(frames), "frame_size": [s.width, s.height],
               "status": ctx.status(), "worst": worst,
               "tsdf_maxdiff_mu": max(r.get("tsdf_maxdiff_mu", 0.0) for r in rows)}
    print(json.dumps({"summary": summary, "per_frame": rows}))


if __name__ == "__main__":
    main()

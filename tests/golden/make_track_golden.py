"""Generates tests/golden/track_golden.npz from the reference's own tracking.

Runs the reference's tracking.cpp / preprocessing.cpp / object.cpp (compiled
unmodified into oracle/_ref/libmf_ref_track.so by `make -C oracle ref`, which
needs the reference tree) and its volume code (oracle/_ref/libmf_ref.so) on a
small seeded two-object scene, and stores the inputs and outputs: pyramid
plane digests, the camera pose and per-level sums of trackLiveFrame (plain and
masked), every object's pose and sums from trackEachObject, and the motion
residual rows of compute_residuals.  tests/test_oracle_golden.py checks the
single-precision tracking oracle against them, so the oracle stays pinned to
the reference on machines where the reference tree is absent.

    make -C oracle ref && python tests/golden/make_track_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import _oracle as O  # noqa: E402
from mid_fusion_b200.scene import generalize_masks, make_scene  # noqa: E402

W, H = 128, 96
INVALID = np.float32(-2.0)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ref = O.reference()
    if ref is None or O.reference_tracking() is None:
        raise SystemExit("oracle/_ref missing: run `make -C oracle ref` first")
    s = make_scene("multi", W, H, n_frames=2, seed=11, bg_size=256, bg_dim=5.12, obj_size=128,
                   obj_dim=0.512, n_objects=2)
    ref.lib.ref_pin_epsilon(s.instances[0].size)
    labels = [i.label for i in s.instances]
    d0, rgb0, gt0 = s.render(0)
    d1, rgb1, gt1 = s.render(1)
    T0 = s.cam_poses[0].astype(np.float32)
    P0 = np.stack([p.astype(np.float32) for p in s.volume_poses(0)])
    vols = [ref.volume(i.size, i.dim) for i in s.instances]
    masks = generalize_masks(gt0, labels)
    for i, v in enumerate(vols):
        v.integrate(d0, rgb0.astype(np.float32) / np.float32(255), masks[i], T0, P0[i], s.k, 0.1)
    vm = np.zeros((H, W, 3), np.float32)
    nm = np.zeros((H, W, 3), np.float32)
    lm = np.zeros((H, W), np.int32)
    ref.raycast_objects(vols, list(P0), labels, T0, s.k, W, H, vertex=vm, normal=nm, label_img=lm)
    out = {"k": np.asarray(s.k, np.float32), "labels": np.asarray(labels, np.int32),
           "depth0": d0, "rgb0": rgb0, "depth1": d1, "rgb1": rgb1, "T0": T0, "P0": P0,
           "vertex": vm, "normal": nm, "label": lm}

    def tracker():
        t = O.RefTracker(W, H, s.k)
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
        return t

    R = tracker()
    for level in range(3):
        for which in range(7):
            out[f"pyr_l{level}_w{which}"] = np.array(digest(R.level(level, which)))
    Tc = R.track_camera(T0, T0, vm, nm)
    out["camera_pose"] = Tc
    out["camera_sums"] = np.stack([R.reduction(level) for level in range(3)])
    for i, label in enumerate(labels[1:], 1):
        sel = (lm == label)[..., None]
        mv = np.where(sel, vm, np.float32(0)).astype(np.float32)
        mn = np.where(sel, nm, np.array([INVALID, 0, 0], np.float32)).astype(np.float32)
        ob = R.object(P0[i], mv, mn)
        out[f"object{label}_pose"] = R.track_object(ob, Tc, T0)[0]
        out[f"object{label}_sums"] = np.stack([R.reduction(level) for level in range(3)])
    mask = (np.isin(lm, labels[1:]) * 255).astype(np.uint8)
    out["camera_pose_masked"] = tracker().track_camera(T0, T0, vm, nm, mask=mask)
    lv = np.zeros((H, W, 3), np.float32)
    ref.raycast_objects(vols, list(P0), labels, Tc, s.k, W, H, vertex=lv,
                        normal=np.zeros((H, W, 3), np.float32),
                        label_img=np.zeros((H, W), np.int32))
    out["live_vertex"] = lv
    res, err, _ = R.compute_residuals(Tc, T0, vm, nm, lv)
    out["residual_codes"] = res.astype(np.int8)
    out["residual_errors_valid"] = err[res == 1]
    path = os.path.join(HERE, "track_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes;",
          "object pixels", [int((lm == label).sum()) for label in labels[1:]])


if __name__ == "__main__":
    main()

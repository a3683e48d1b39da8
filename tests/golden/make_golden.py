"""Generates tests/golden/volume_golden.npz from the reference's own code.

Runs the reference's allocation, integration and multi-instance raycast
(lib/ + apps/kfusion/src/cpp/kfusion/*.hpp compiled unmodified into
oracle/_ref/libmf_ref.so by `make -C oracle ref`, which needs the reference
tree) on a small seeded scene and stores the inputs and outputs.  The CPU
tests check the oracle against these fixtures, so the oracle stays pinned to
the reference on machines where the reference tree is absent.

    make -C oracle ref && python tests/golden/make_golden.py
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

W, H, FRAMES = 96, 72, 3


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ref = O.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libmf_ref.so missing: run `make -C oracle ref` first")
    s = make_scene("multi", W, H, n_frames=FRAMES, seed=21, bg_size=128, bg_dim=5.12,
                   obj_size=64, obj_dim=0.512, n_objects=2)
    ref.lib.ref_pin_epsilon(s.instances[0].size)
    labels = [i.label for i in s.instances]
    vols = [ref.volume(i.size, i.dim) for i in s.instances]
    out = {"k": np.asarray(s.k, np.float32), "labels": np.asarray(labels, np.int32),
           "sizes": np.asarray([i.size for i in s.instances], np.int32),
           "dims": np.asarray([i.dim for i in s.instances], np.float32)}
    vtx = np.zeros((H, W, 3), np.float32)
    nrm = np.zeros((H, W, 3), np.float32)
    lab = np.zeros((H, W), np.int32)
    for f in range(FRAMES):
        d, rgb, gt = s.render(f)
        masks = generalize_masks(gt, labels)
        poses = np.stack([P.astype(np.float32) for P in s.volume_poses(f)])
        T = s.cam_poses[f].astype(np.float32)
        out[f"depth{f}"], out[f"rgb{f}"], out[f"masks{f}"] = d, rgb, masks
        out[f"poses{f}"], out[f"T{f}"] = poses, T
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
            keys, coords, active, vox = v.blocks()
            nk, side, cm, nv = v.nodes()
            out[f"f{f}_i{i}_block_keys"] = keys
            out[f"f{f}_i{i}_active"] = active
            out[f"f{f}_i{i}_node_keys"] = nk
            out[f"f{f}_i{i}_children"] = cm
            out[f"f{f}_i{i}_voxel_sha"] = np.array(digest(vox))
            out[f"f{f}_i{i}_node_sha"] = np.array(digest(nv))
        ref.raycast_objects(vols, list(poses), labels, T, s.k, W, H, vertex=vtx, normal=nrm,
                            label_img=lab)
        out[f"f{f}_vertex"], out[f"f{f}_normal"], out[f"f{f}_label"] = vtx.copy(), nrm.copy(), lab.copy()
    np.savez_compressed(os.path.join(HERE, "volume_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "volume_golden.npz"))


if __name__ == "__main__":
    main()

"""The headline workload at full size, exactly as bench.py runs it: 640x480
frames (fx = fy = 525), background octree 512^3 @ 1 cm plus a sphere, a box and
a cylinder with 256^3 @ 2 mm octrees, each object moving with its own seeded
twist, the batched frame (mf_process_frame, one CUDA graph per frame).

Frame by frame, in lockstep with the oracle:

* camera and object poses against the reference and the all-FP64 oracle,
  each tracked from the device's previous-frame poses and model maps
  (tests/_pose.py: within 1e-5 m / rad of the reference and of the FP64 run,
  widened by twice the reference's own distance to the FP64 run; or, after a
  decision flip of the GN's cost test, a pose one step away whose level-0
  cost is as low as the reference's to 2e-4);
* integration of all four volumes at the device's poses: block keys, corner
  coordinates, active flags and every voxel field, bit-exact;
* the composite raycast at the device's poses: vertex, normal and label
  maps, bit-exact.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import _oracle as O
from _pose import camera_cost, check_pose, object_cost
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402  (the bench's own workload definition)

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]
FRAMES = 4


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def test_headline_workload_in_lockstep_with_oracle():
    s = bench.scene_for(0, FRAMES)
    W, H = s.width, s.height
    assert (W, H) == (640, 480) and abs(s.k[0] - 525.0) < 1e-9
    assert [i.size for i in s.instances] == [512, 256, 256, 256]
    labels = [i.label for i in s.instances]
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 16, batched=True, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    orc = O.oracle()
    vols = [orc.volume(i.size, i.dim) for i in s.instances]
    trk32 = O.Tracker(W, H, s.k, robust=1, fp64=False)   # == the reference's tracking.cpp
    trk64 = O.Tracker(W, H, s.k, robust=1, fp64=True)
    vo = np.zeros((H, W, 3), np.float32)
    no = np.zeros((H, W, 3), np.float32)
    lo = np.zeros((H, W), np.int32)
    model = None
    strict = total = 0
    for f in range(FRAMES):
        d, rgb, lab = s.render(f)
        T_prev = ctx.camera_pose().copy()
        P_prev = [ctx.instance_pose(i).copy() for i in range(len(labels))]
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                      np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                      lab16.ctypes.data_as(C.c_void_p))
        assert rc == 0, ctx.lib.mf_last_error(ctx.h)
        T = ctx.camera_pose()
        P = [ctx.instance_pose(i) for i in range(len(labels))]
        for t in (trk32, trk64):
            t.set_frame(rgb, d)
        if f > 0:
            # the camera, with the last raycast's object pixels masked out
            mask = (np.isin(model[2], labels[1:]) * 255).astype(np.uint8)
            cams = []
            for t in (trk32, trk64):
                t.set_mask(mask)
                cams.append(t.track_camera(T_prev, T_prev, model[0], model[1]))
            total += 1
            strict += check_pose(T, cams[0], cams[1], f"frame {f} camera",
                                 cost=camera_cost(trk64, T_prev, model[0], model[1]))
            # every object, from its last pose, under the device's new camera pose
            for i in range(1, len(labels)):
                if not np.any(model[2] == labels[i]):
                    continue
                objs = [t.track_object(P_prev[i], T, T_prev, model[0], model[1], model[2],
                                       labels[i]) for t in (trk32, trk64)]
                total += 1
                strict += check_pose(P[i], objs[0], objs[1], f"frame {f} object {labels[i]}",
                                     cost=object_cost(trk64, P_prev[i], T, T_prev, model[0],
                                                      model[1], model[2], labels[i]))
        # integration at the device's poses, bit-exact
        masks = generalize_masks(lab, labels)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(d, rgb3, masks[i], T, P[i], s.k, 0.1)
            kg, cg, ag, xg = ctx.blocks(i)
            ko, co, ao, xo = v.blocks()
            assert np.array_equal(kg, ko) and np.array_equal(cg, co), (f, i)
            assert np.array_equal(ag, ao), (f, i)
            for fld in FIELDS:
                assert np.array_equal(xg[fld], xo[fld]), (f, i, fld)
        # the composite raycast at the device's poses, bit-exact
        orc.raycast_objects(vols, P, labels, T, s.k, W, H, eps_size=s.instances[0].size,
                            vertex=vo, normal=no, label_img=lo)
        model = ctx.download_raycast()
        assert np.array_equal(model[2], lo), f
        assert np.array_equal(model[0], vo) and np.array_equal(model[1], no), f
        for t in (trk32, trk64):
            t.set_ref()
    # most problems of this workload are well conditioned: within 1e-5 of the
    # reference itself
    assert total >= 3 * (FRAMES - 1) and strict >= total // 2, (strict, total)
    assert ctx.status() == 0
    ctx.close()

"""The plain single-octree method: a static room (4 spheres, 3 boxes, seeded
value-noise albedo), 320x240 frames at fx = fy = 262.5, one 256^3 octree over
2.56 m, mu = 0.1, pyramid {10, 5, 4}.

Frame by frame, through the whole pipeline (mf_process_frame), against the
oracle in lockstep: camera tracking from the same model maps against the
reference (the single-precision oracle, equal to the reference's
tracking.cpp bit for bit) and the all-FP64 oracle (tests/_pose.py: within
1e-5 m / rad of the reference and of the FP64 run, widened by twice the
reference's own distance r to the FP64 run, which its single-precision
arithmetic makes up to ~1e-4 on this room's poorly conditioned poses;
iteration counts equal where the
reference and the FP64 run agree on them), then integration at the device's
pose and the raycast, both bit-exact.
"""
import ctypes as C

import numpy as np
import pytest

import _oracle as O
from _pose import camera_cost, check_pose
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240
FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _rot_err(A, B):
    R = np.linalg.solve(A[:3, :3], B[:3, :3])
    return float(np.linalg.norm(0.5 * np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0],
                                                R[1, 0] - R[0, 1]])))


@pytest.mark.parametrize("batched", [True, False])
def test_room_sequence_in_lockstep_with_oracle(batched):
    s = make_scene("room", W, H, n_frames=4, seed=2, bg_size=256, bg_dim=2.56)
    assert len(s.instances) == 1 and abs(s.k[0] - 262.5) < 1e-6
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, batched=batched, robust="huber")
    ctx.add_instance(256, 2.56, np.eye(4), 0)
    ctx.set_camera_pose(s.cam_poses[0])
    orc = O.oracle()
    vol = orc.volume(256, 2.56)
    trk = O.Tracker(W, H, s.k, robust=1, fp64=True)
    trk32 = O.Tracker(W, H, s.k, robust=1, fp64=False)
    vo = np.zeros((H, W, 3), np.float32)
    no = np.zeros((H, W, 3), np.float32)
    lo = np.zeros((H, W), np.int32)
    model = None
    for f in range(s.n_frames):
        d, rgb, lab = s.render(f)
        T_prev = ctx.camera_pose().copy()
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                      np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                      lab16.ctypes.data_as(C.c_void_p))
        assert rc == 0, ctx.lib.mf_last_error(ctx.h)
        trk.set_frame(rgb, d)
        trk32.set_frame(rgb, d)
        T = ctx.camera_pose()
        if f > 0:
            T_or = trk.track_camera(T_prev, T_prev, model[0], model[1])
            it64 = trk.iterations()
            T32 = trk32.track_camera(T_prev, T_prev, model[0], model[1])
            it32 = trk32.iterations()
            it, _, _ = ctx.track_info(0)
            ok = check_pose(T, T32, T_or, f"frame {f}",
                            cost=camera_cost(trk, T_prev, model[0], model[1]))
            if ok and it32 == it64:
                assert list(it[:3]) == it64, (f, list(it[:3]), it64)
        # integration and raycast at the device's pose, bit-exact
        mask = generalize_masks(lab, [0])[0]
        vol.integrate(d, rgb.astype(np.float32) / np.float32(255.0), mask, T, np.eye(4), s.k,
                      0.1)
        kg, cg, ag, xg = ctx.blocks(0)
        ko, co, ao, xo = vol.blocks()
        assert np.array_equal(kg, ko) and np.array_equal(cg, co) and np.array_equal(ag, ao)
        for fld in FIELDS:
            assert np.array_equal(xg[fld], xo[fld]), (f, fld)
        orc.raycast_objects([vol], [np.eye(4)], [0], T, s.k, W, H, eps_size=256, vertex=vo,
                            normal=no, label_img=lo)
        model = ctx.download_raycast()
        assert np.array_equal(model[0], vo) and np.array_equal(model[1], no), f
        assert np.array_equal(model[2], lo), f
        trk.set_ref()
        trk32.set_ref()
    assert ctx.status() == 0
    ctx.close()

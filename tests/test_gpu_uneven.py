"""Twelve objects of uneven octree sizes (32^3 ... 256^3 at 2-5 mm) beside the
512^3 background: every block level from 2 to 6 in one batched launch.

* allocation, integration and the composite raycast against the oracle,
  bit-exact, batched and plain;
* the whole-frame pipeline (mf_process_frame: tracking, integration, raycast)
  batched against plain: identical poses and volumes;
* object tracking of every object against the reference (the
  single-precision oracle, equal to the reference's tracking.cpp bit for bit)
  and the all-FP64 oracle (tests/_pose.py: within 1e-5 m / rad of both,
  widened by twice the reference's own distance to the FP64 run).
"""
import ctypes as C

import numpy as np
import pytest

import _oracle as O
from _pose import check_pose, object_cost
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]
POSE_TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _scene(W, H, frames, seed=23):
    return make_scene("uneven", W, H, n_frames=frames, seed=seed, n_objects=12)


def _context(s, batched, pool=1 << 15):
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=pool, batched=batched, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    return ctx


@pytest.mark.parametrize("batched", [True, False])
def test_uneven_volumes_and_raycast_match_oracle(batched):
    s = _scene(160, 120, 2)
    assert sorted({i.size for i in s.instances[1:]}) == [32, 64, 128, 256]
    orc = O.oracle()
    ctx = _context(s, batched)
    vols = [orc.volume(i.size, i.dim) for i in s.instances]
    labels = [i.label for i in s.instances]
    vo = np.zeros((s.height, s.width, 3), np.float32)
    no = np.zeros((s.height, s.width, 3), np.float32)
    lo = np.zeros((s.height, s.width), np.int32)
    for f in range(s.n_frames):
        depth, rgb, lab = s.render(f)
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        for i, P in enumerate(poses):
            ctx.set_instance_pose(i, P)
        ctx.set_camera_pose(T)
        ctx.upload(depth, rgb, masks)
        ctx.integrate(list(range(len(vols))))
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(depth, rgb3, masks[i], T, poses[i], s.k, 0.1)
            kg, cg, ag, xg = ctx.blocks(i)
            ko, co, ao, xo = v.blocks()
            assert np.array_equal(kg, ko), f"instance {i} ({s.instances[i].size}^3): block keys"
            assert np.array_equal(cg, co) and np.array_equal(ag, ao)
            for fld in FIELDS:
                assert np.array_equal(xg[fld], xo[fld]), f"instance {i}: voxel field {fld}"
            nkg, _, cmg, nvg = ctx.nodes(i)
            nko, _, cmo, nvo = v.nodes()
            assert np.array_equal(nkg, nko) and np.array_equal(cmg, cmo)
            for fld in FIELDS:
                assert np.array_equal(nvg[fld], nvo[fld]), f"instance {i}: node field {fld}"
        ctx.raycast()
        vg, ng, lg = ctx.download_raycast()
        orc.raycast_objects(vols, poses, labels, T, s.k, s.width, s.height,
                            eps_size=s.instances[0].size, vertex=vo, normal=no, label_img=lo)
        assert np.array_equal(lg, lo), f"labels differ at {np.count_nonzero(lg != lo)} px"
        assert np.array_equal(vg, vo) and np.array_equal(ng, no)
    assert ctx.status() == 0
    ctx.close()


def _run_frames(s, batched):
    ctx = _context(s, batched)
    ctx.set_camera_pose(s.cam_poses[0])
    poses = []
    for f in range(s.n_frames):
        d, rgb, lab = s.render(f)
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                      np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                      lab16.ctypes.data_as(C.c_void_p))
        assert rc == 0, ctx.lib.mf_last_error(ctx.h)
        Tc = np.zeros(16, np.float32)
        To = np.zeros(16 * len(s.instances), np.float32)
        ctx.lib.mf_get_poses(ctx.h, Tc.ctypes.data_as(C.c_void_p), To.ctypes.data_as(C.c_void_p))
        poses.append((Tc.copy(), To.copy()))
    return ctx, poses


def test_uneven_pipeline_batched_equals_plain():
    s = _scene(160, 120, 4)
    cb, pb = _run_frames(s, True)
    cp, pp = _run_frames(s, False)
    for (tb, ob), (tp, op) in zip(pb, pp):
        np.testing.assert_array_equal(tb, tp)
        np.testing.assert_array_equal(ob, op)
    for i in range(len(s.instances)):
        kb, _, _, xb = cb.blocks(i)
        kp, _, _, xp = cp.blocks(i)
        assert np.array_equal(kb, kp)
        for fld in FIELDS:
            assert np.array_equal(xb[fld], xp[fld])
    assert cb.status() == 0 and cp.status() == 0
    cb.close()
    cp.close()


def _rot_err(A, B):
    R = np.linalg.solve(A[:3, :3], B[:3, :3])
    return float(np.linalg.norm(0.5 * np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0],
                                                R[1, 0] - R[0, 1]])))


@pytest.mark.parametrize("batched", [True, False])
def test_uneven_objects_track_like_fp64_oracle(batched):
    """Every object tracked from its frame-0 pose with the camera at frame 1.

    The per-pixel rows are FP32 (as in the reference); for small objects with
    few valid pixels the normal equations are ill-conditioned and the FP32
    oracle itself lands up to ~1e-4 away from the FP64 oracle.  Where the two
    oracles agree (same iterations, poses within 2e-6) the device must be
    the pose by tests/_pose.py; where the device is within 1e-5 of the
    reference and the reference and the FP64 run take the same iterations, the
    device takes them too."""
    W, H = 320, 240
    s = _scene(W, H, 2)
    labels = [i.label for i in s.instances]
    ctx = _context(s, batched)
    d, rgb, lab = s.render(0)
    T0 = s.cam_poses[0].astype(np.float32)
    T1 = s.cam_poses[1].astype(np.float32)
    ctx.set_camera_pose(T0)
    ctx.upload(d, rgb, generalize_masks(lab, labels))
    ctx.integrate(list(range(len(labels))))
    ctx.raycast()
    ctx.preprocess()
    ctx.set_ref_from_current()
    v, n, lbl = ctx.download_raycast()
    d1, rgb1, lab1 = s.render(1)
    trk = {}
    for fp64 in (True, False):
        t = O.Tracker(W, H, s.k, robust=1, fp64=fp64)
        t.set_frame(rgb, d)
        t.set_ref()
        t.set_frame(rgb1, d1)
        trk[fp64] = t
    ctx.upload(d1, rgb1, generalize_masks(lab1, labels))
    ctx.preprocess()
    ctx.set_camera_pose(T1)
    ids = list(range(1, len(labels)))
    ctx.track_objects(ids)
    strict = 0
    for i in ids:
        T_wo = s.volume_poses(0)[i].astype(np.float32)
        T64 = trk[True].track_object(T_wo, T1, T0, v, n, lbl, labels[i])
        it64 = trk[True].iterations()
        T32 = trk[False].track_object(T_wo, T1, T0, v, n, lbl, labels[i])
        it32 = trk[False].iterations()
        it, _, T_c2o2 = ctx.track_info(i)
        T_gpu = T1.astype(np.float64) @ T_c2o2
        ok = check_pose(T_gpu, T32, T64, f"object {i} ({s.instances[i].size}^3)",
                        cost=object_cost(trk[True], T_wo, T1, T0, v, n, lbl, labels[i]))
        if ok and it32 == it64:
            assert list(it[:3]) == it64, (i, list(it[:3]), it64)
        strict += ok
    # not vacuous: on this scene 5 of the 12 problems are well conditioned
    assert strict >= 4, strict
    ctx.close()

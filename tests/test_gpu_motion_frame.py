"""mf_process_frame_motion: the reference's per-frame flow with motion
segmentation (kfusion.cpp:265-466, 606-630) in one call, against the same
flow driven step by step through the separate entry points (each of them
checked against the oracle in tests/test_gpu_motion.py and
tests/test_gpu_volume.py): camera track, motion residuals and moving labels,
masked camera re-track, tracking of the moving objects only, residuals again,
each moving object's rows recomputed at its virtual camera pose, mask
refinement from the third frame on, integration, raycast, new reference.
Moving bits, camera and volume poses, the refined masks, every voxel of
every volume and the model maps agree bit for bit; the scene's objects move,
so the moving branch runs (checked), and frames 2-5 refine the masks.
"""
import ctypes as C

import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240
FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]
FRAMES = 6


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _context(s):
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    return ctx


def _poses(ctx, n):
    Tc = np.zeros(16, np.float32)
    To = np.zeros(16 * n, np.float32)
    rc = ctx.lib.mf_get_poses(ctx.h, Tc.ctypes.data_as(C.c_void_p),
                              To.ctypes.data_as(C.c_void_p))
    assert rc == 0
    return Tc, To


def _step_by_step(ctx, s, f, frame, buf0, buf1):
    """One frame of the flow through the separate entry points."""
    n = len(s.instances)
    labels = [i.label for i in s.instances]
    d, rgb, lab = s.render(f)
    ctx.upload(d, rgb, None)
    ctx.upload_labels(lab.astype(np.uint16))
    ctx.preprocess()
    bits = 0
    if frame > 0:
        ctx.track_camera()
        _, bits = ctx.motion_residuals(1.5, 0.9)
        moving = [i for i in range(1, n) if (bits >> labels[i]) & 1]
        if moving:
            ctx.retrack_camera(bits)
            ctx.track_objects(moving)
            ctx.motion_residuals(1.5, 0.9)
        if frame > 1:
            rows0 = None
            if not moving:
                ctx.track_results(0, buf0.data_ptr())
                rows0 = buf0.data_ptr()
            for i in range(n):
                rows = rows0
                if i in moving:
                    ctx.object_residuals(i, buf1.data_ptr(), 1.5)
                    rows = buf1.data_ptr()
                ctx.refine_mask_use_motion(i, rows)
    ctx.integrate(list(range(n)))
    ctx.raycast()
    ctx.set_ref_from_current()
    return bits


def test_process_frame_motion_equals_the_step_by_step_flow():
    import torch
    s = make_scene("multi", W, H, n_frames=FRAMES, seed=5, bg_size=256, obj_size=128,
                   n_objects=3)
    n = len(s.instances)
    one, steps = _context(s), _context(s)
    buf0 = torch.zeros(2 * W * H, dtype=torch.int8, device="cuda")
    buf1 = torch.zeros(2 * W * H, dtype=torch.int8, device="cuda")
    moved = 0
    for f in range(FRAMES):
        d, rgb, lab = s.render(f)
        bits_one = one.process_frame_motion(d, rgb, lab, 1.5, 0.9)
        bits_steps = _step_by_step(steps, s, f, f, buf0, buf1)
        assert bits_one == bits_steps, (f, bits_one, bits_steps)
        if bits_one:
            moved += 1
        for a, b in zip(_poses(one, n), _poses(steps, n)):
            assert np.array_equal(a, b), f
        for i in range(n):
            assert np.array_equal(one.mask(i), steps.mask(i)), (f, i)
    assert moved > 0, "no frame moved an object: the moving branch did not run"
    for i in range(n):
        ka, ca, aa, xa = one.blocks(i)
        kb, cb, ab, xb = steps.blocks(i)
        oa, ob = np.argsort(ka), np.argsort(kb)
        assert np.array_equal(ka[oa], kb[ob]) and np.array_equal(aa[oa], ab[ob])
        for fld in FIELDS:
            assert np.array_equal(xa[oa][fld], xb[ob][fld]), (i, fld)
    for a, b in zip(one.download_raycast(), steps.download_raycast()):
        assert np.array_equal(a, b)
    assert one.status() == 0 and steps.status() == 0
    one.close()
    steps.close()


def test_process_frame_motion_rejects_bad_arguments():
    s = make_scene("multi", W, H, n_frames=1, seed=5, bg_size=256, obj_size=128, n_objects=1)
    ctx = _context(s)
    d, rgb, lab = s.render(0)
    bits = C.c_uint32()
    lab16 = np.ascontiguousarray(lab.astype(np.uint16))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rgb = np.ascontiguousarray(rgb)
    assert ctx.lib.mf_process_frame_motion(ctx.h, P(d), P(rgb), None, C.c_float(1.5),
                                           C.c_float(0.9), C.byref(bits)) == -1
    assert ctx.lib.mf_process_frame_motion(ctx.h, P(d), P(rgb), P(lab16), C.c_float(0.0),
                                           C.c_float(0.9), C.byref(bits)) == -1
    assert ctx.lib.mf_process_frame_motion(ctx.h, P(d), P(rgb), P(lab16), C.c_float(1.5),
                                           C.c_float(0.9), None) == -1
    ctx.close()

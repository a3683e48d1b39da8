"""Staged frames (mf_frame_stage + mf_process_staged: the next frame's upload
on the context's upload stream while the current frame is processed) against
mf_process_frame on the same frames: the same camera and object poses and the
same model maps, bit for bit, frame after frame; and the slot state errors."""
import ctypes as C

import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context, MfError
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _context(s):
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 15, batched=True, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    return ctx


def _state(ctx, n):
    return (ctx.camera_pose().copy(), [ctx.instance_pose(i).copy() for i in range(n)],
            [a.copy() for a in ctx.download_raycast()])


def test_staged_frames_equal_process_frame():
    s = make_scene("multi", 320, 240, n_frames=5, seed=17, n_objects=3, bg_size=256,
                   obj_size=128)
    n = len(s.instances)
    frames = []
    for f in range(s.n_frames):
        d, rgb, lab = s.render(f)
        frames.append((np.ascontiguousarray(d, dtype=np.float32), np.ascontiguousarray(rgb),
                       np.ascontiguousarray(lab.astype(np.uint16))))

    a = _context(s)
    ref = []
    for d, rgb, lab in frames:
        rc = a.lib.mf_process_frame(a.h, d.ctypes.data_as(C.c_void_p),
                                    rgb.ctypes.data_as(C.c_void_p), lab.ctypes.data_as(C.c_void_p))
        assert rc == 0, a.lib.mf_last_error(a.h)
        ref.append(_state(a, n))
    assert a.status() == 0
    a.close()

    b = _context(s)
    out = []
    b.frame_stage(0, *frames[0])
    for f in range(len(frames)):
        if f + 1 < len(frames):
            b.frame_stage((f + 1) & 1, *frames[f + 1])  # uploads while frame f runs
        b.process_staged(f & 1)
        out.append(_state(b, n))
    assert b.status() == 0
    b.close()

    for f, ((ca, oa, ma), (cb, ob, mb)) in enumerate(zip(ref, out)):
        assert np.array_equal(ca, cb), f
        for i, (x, y) in enumerate(zip(oa, ob)):
            assert np.array_equal(x, y), (f, i)
        for x, y in zip(ma, mb):
            assert np.array_equal(x, y), f


def test_staged_slot_errors():
    s = make_scene("multi", 160, 120, n_frames=1, seed=3, n_objects=1, bg_size=256,
                   obj_size=64)
    ctx = _context(s)
    d, rgb, lab = s.render(0)
    d = np.ascontiguousarray(d, dtype=np.float32)
    rgb = np.ascontiguousarray(rgb)
    lab = np.ascontiguousarray(lab.astype(np.uint16))
    with pytest.raises(MfError, match="nothing staged"):
        ctx.process_staged(1)
    ctx.frame_stage(1, d, rgb, lab)
    with pytest.raises(MfError, match="not taken yet"):
        ctx.frame_stage(1, d, rgb, lab)
    ctx.process_staged(1)
    ctx.frame_stage(1, d, rgb, None)          # the slot is free again; labels optional
    ctx.process_staged(1)
    assert ctx.lib.mf_frame_stage(ctx.h, 2, d.ctypes.data_as(C.c_void_p),
                                  rgb.ctypes.data_as(C.c_void_p), None) == -1  # MF_E_ARG
    ctx.synchronize()
    assert ctx.status() == 0
    ctx.close()

"""Batched GN in one cooperative launch per pyramid level (mf_set_gn_persistent
1) against one launch per iteration (0, the default) and against the plain
host-driven loop: the same poses bit for bit, frame after frame, for the
3-object and the 12-object workloads; no barrier timed out."""
import ctypes as C

import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu

MF_STATUS_GN_TIMEOUT = 32


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _run(s, frames, batched, persistent):
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 15, batched=batched,
                  robust="huber")
    ctx.set_gn_persistent(persistent)
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    poses = []
    for d, rgb, lab in frames:
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                      np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                      lab16.ctypes.data_as(C.c_void_p))
        assert rc == 0, ctx.lib.mf_last_error(ctx.h)
        poses.append((ctx.camera_pose().copy(),
                      [ctx.instance_pose(i).copy() for i in range(len(s.instances))]))
    st = ctx.status()
    it = [ctx.track_info(i)[0] for i in range(len(s.instances))]
    ctx.close()
    return poses, st, it


@pytest.mark.parametrize("preset", ["multi", "uneven"])
def test_persistent_gn_equals_per_iteration_launches(preset):
    W, H = 320, 240
    if preset == "multi":
        s = make_scene("multi", W, H, n_frames=5, seed=11, n_objects=3, bg_size=256,
                       obj_size=128)
    else:
        s = make_scene("uneven", W, H, n_frames=4, seed=23, n_objects=12)
    frames = [s.render(f) for f in range(s.n_frames)]
    pa, sa, ia = _run(s, frames, True, True)
    pb, sb, ib = _run(s, frames, True, False)
    pc, sc, ic = _run(s, frames, False, True)
    assert sa & MF_STATUS_GN_TIMEOUT == 0
    assert sa == sb == sc == 0, (sa, sb, sc)
    for f, ((ca, oa), (cb, ob), (cc, oc)) in enumerate(zip(pa, pb, pc)):
        assert np.array_equal(ca, cb) and np.array_equal(ca, cc), f
        for i, (a, b, c) in enumerate(zip(oa, ob, oc)):
            assert np.array_equal(a, b) and np.array_equal(a, c), (f, i)
    # the iteration counts of the last frame's problems agree too
    for a, b in zip(ia, ib):
        assert list(a) == list(b)

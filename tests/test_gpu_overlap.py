"""The batched frame with the background's allocation, integration and (with
the phased raycast) its raycast marches overlapped with object tracking
(mf_set_overlap: a low-priority side stream joined into the frame graph)
against the in-order frame: the same camera and object poses, the same voxels
of every volume and the same model maps, bit for bit, frame after frame, for
the 3-object and the 12-object workloads, with the one-kernel and the phased
raycast and with the integration's own grid or few CTAs."""
import ctypes as C

import numpy as np
import pytest

from mid_fusion_b200 import build, capi
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _run(s, frames, overlap, ray=None):
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 15, batched=True, robust="huber")
    ctx.set_overlap(overlap)
    if ray is not None:
        ctx.tune_set(capi.TUNE_RAYCAST, ray)
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    out = []
    for d, rgb, lab in frames:
        lab16 = np.ascontiguousarray(lab.astype(np.uint16))
        rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                      np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                      lab16.ctypes.data_as(C.c_void_p))
        assert rc == 0, ctx.lib.mf_last_error(ctx.h)
        out.append((ctx.camera_pose().copy(),
                    [ctx.instance_pose(i).copy() for i in range(len(s.instances))],
                    [a.copy() for a in ctx.download_raycast()]))
    vols = [ctx.blocks(i) for i in range(len(s.instances))]
    st = ctx.status()
    ctx.close()
    return out, vols, st


def capi_ray_count():
    return capi.tune_candidates(capi.TUNE_RAYCAST)


def capi_ray_describe(v):
    return capi.tune_describe(capi.TUNE_RAYCAST, v)


@pytest.mark.parametrize("preset", ["multi", "uneven"])
def test_overlapped_background_integration_equals_in_order(preset):
    W, H = 320, 240
    if preset == "multi":
        s = make_scene("multi", W, H, n_frames=4, seed=11, n_objects=3, bg_size=256,
                       obj_size=128)
    else:
        s = make_scene("uneven", W, H, n_frames=3, seed=23, n_objects=12)
    frames = [s.render(f) for f in range(s.n_frames)]
    a, va, sa = _run(s, frames, 0)
    b, vb, sb = _run(s, frames, -1)    # the default: the launch shape's own grid
    c, vc, sc = _run(s, frames, 37)    # few CTAs: the background integration outlasts tracking
    # the phased raycast: the background's marches on the side stream too
    phased = [v for v in range(capi_ray_count()) if "phased" in capi_ray_describe(v)]
    d, vd, sd = _run(s, frames, -1, ray=phased[-1])
    e, ve, se = _run(s, frames, 37, ray=phased[0])
    assert sa == sb == sc == sd == se == 0
    for other, vother in ((b, vb), (c, vc), (d, vd), (e, ve)):
        for f, ((ca, oa, ma), (cb, ob, mb)) in enumerate(zip(a, other)):
            assert np.array_equal(ca, cb), f
            for i, (x, y) in enumerate(zip(oa, ob)):
                assert np.array_equal(x, y), (f, i)
            for x, y in zip(ma, mb):
                assert np.array_equal(x, y), f
        for i, ((ka, ca, aa, xa), (kb, cb, ab, xb)) in enumerate(zip(va, vother)):
            assert np.array_equal(ka, kb) and np.array_equal(ca, cb), i
            assert np.array_equal(aa, ab), i
            for fld in FIELDS:
                assert np.array_equal(xa[fld], xb[fld]), (i, fld)

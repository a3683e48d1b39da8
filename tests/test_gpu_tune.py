"""The launch-shape autotuner on the GPU.

Every candidate shape of the composite raycast and of the block integration
computes each pixel / voxel alike, so the maps, the volumes and the tracked
poses are bit-identical whichever shape runs.  mf_autotune times the
candidates on scratch copies and leaves the map and the model maps unchanged;
a tuned context then tracks and integrates exactly like an untuned one.
"""
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


def _scene(frames=3):
    # 160x120: the 8x16 raycast tile leaves a partial tile row at the bottom
    return make_scene("multi", 160, 120, n_frames=frames, seed=11, bg_size=256, obj_size=64,
                      n_objects=3)


def _context(s):
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 14, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    ctx.set_camera_pose(s.cam_poses[0])
    return ctx


def _frame(ctx, s, f):
    d, rgb, lab = s.render(f)
    lab16 = np.ascontiguousarray(lab.astype(np.uint16))
    rc = ctx.lib.mf_process_frame(ctx.h, d.ctypes.data_as(C.c_void_p),
                                  np.ascontiguousarray(rgb).ctypes.data_as(C.c_void_p),
                                  lab16.ctypes.data_as(C.c_void_p))
    assert rc == 0, ctx.lib.mf_last_error(ctx.h)
    Tc = np.zeros(16, np.float32)
    To = np.zeros(16 * len(s.instances), np.float32)
    ctx.lib.mf_get_poses(ctx.h, Tc.ctypes.data_as(C.c_void_p), To.ctypes.data_as(C.c_void_p))
    return Tc, To


def _volumes(ctx, n):
    out = []
    for i in range(n):
        k, c, a, x = ctx.blocks(i)
        order = np.argsort(k)
        out.append((k[order], c[order], a[order], x[order]))
    return out


def _assert_same_volumes(va, vb):
    for (ka, ca, aa, xa), (kb, cb, ab, xb) in zip(va, vb):
        assert np.array_equal(ka, kb) and np.array_equal(ca, cb) and np.array_equal(aa, ab)
        for f in FIELDS:
            assert np.array_equal(xa[f], xb[f]), f"voxel field {f} differs"


def test_every_raycast_shape_gives_identical_maps():
    s = _scene(2)
    ctx = _context(s)
    for f in range(2):
        _frame(ctx, s, f)
    ref = None
    for v in range(capi.tune_candidates(capi.TUNE_RAYCAST)):
        ctx.tune_set(capi.TUNE_RAYCAST, v)
        assert ctx.tune_get(capi.TUNE_RAYCAST) == v
        ctx.raycast()
        maps = ctx.download_raycast()
        if ref is None:
            ref = maps
            assert np.count_nonzero(ref[2] >= 0) > 1000  # the scene is in view
            continue
        for a, b in zip(ref, maps):
            assert np.array_equal(a, b), capi.tune_describe(capi.TUNE_RAYCAST, v)
    assert ctx.status() == 0
    ctx.close()


def test_every_integration_shape_gives_identical_volumes_and_poses():
    s = _scene(3)
    runs = []
    for v in range(capi.tune_candidates(capi.TUNE_INTEGRATE)):
        ctx = _context(s)
        ctx.tune_set(capi.TUNE_INTEGRATE, v)
        poses = [_frame(ctx, s, f) for f in range(s.n_frames)]
        runs.append((poses, _volumes(ctx, len(s.instances)), ctx.download_raycast()))
        assert ctx.status() == 0
        ctx.close()
    p0, v0, m0 = runs[0]
    for poses, vols, maps in runs[1:]:
        for (ta, oa), (tb, ob) in zip(p0, poses):
            assert np.array_equal(ta, tb) and np.array_equal(oa, ob)
        _assert_same_volumes(v0, vols)
        for a, b in zip(m0, maps):
            assert np.array_equal(a, b)


def test_autotune_keeps_the_map_and_tracks_like_an_untuned_context():
    s = _scene(5)
    tuned, plain = _context(s), _context(s)
    for f in range(2):
        assert all(np.array_equal(a, b) for a, b in zip(_frame(tuned, s, f), _frame(plain, s, f)))
    vols = _volumes(tuned, len(s.instances))
    maps = tuned.download_raycast()
    rep = tuned.autotune(reps=3)
    n_ray = capi.tune_candidates(capi.TUNE_RAYCAST)
    n_int = capi.tune_candidates(capi.TUNE_INTEGRATE)
    assert len(rep["raycast"]["us"]) == n_ray and len(rep["integrate"]["us"]) == n_int
    assert all(t > 0 for t in rep["raycast"]["us"] + rep["integrate"]["us"])
    for name in ("raycast", "integrate"):
        us, v = rep[name]["us"], rep[name]["chosen"]
        assert us[v] <= 1.01 * min(us) + 1e-6, (name, us, v)
    # the tuner wrote scratch copies only
    _assert_same_volumes(vols, _volumes(tuned, len(s.instances)))
    for a, b in zip(maps, tuned.download_raycast()):
        assert np.array_equal(a, b)
    # later frames (a re-captured graph with the chosen shapes) match bit for bit
    for f in range(2, s.n_frames):
        ta, oa = _frame(tuned, s, f)
        tb, ob = _frame(plain, s, f)
        assert np.array_equal(ta, tb) and np.array_equal(oa, ob)
    _assert_same_volumes(_volumes(tuned, len(s.instances)), _volumes(plain, len(s.instances)))
    assert tuned.status() == 0 and plain.status() == 0
    tuned.close()
    plain.close()

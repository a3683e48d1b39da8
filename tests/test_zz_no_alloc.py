"""mf_track_eval_static (normal equations with static device scratch, no
allocation) against mf_track_eval on the same context.

Collected last on purpose: it must also pass after every other GPU test has
run in the same process (other contexts, other devices' state).
"""
import ctypes as C

import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _tracked_context():
    s = make_scene("multi", W, H, n_frames=2, seed=5, bg_size=256, obj_size=64, n_objects=2)
    labels = [i.label for i in s.instances]
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, robust="huber")
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    d, rgb, lab = s.render(0)
    ctx.set_camera_pose(s.cam_poses[0])
    ctx.upload(d, rgb, generalize_masks(lab, labels))
    ctx.integrate(list(range(len(labels))))
    ctx.raycast()
    ctx.preprocess()
    ctx.set_ref_from_current()
    d, rgb, lab = s.render(1)
    ctx.upload(d, rgb, generalize_masks(lab, labels))
    ctx.preprocess()
    ctx.track_camera()                                  # sets up slot 0
    ctx.track_objects(list(range(1, len(labels))))      # sets up slots 1..
    return s, ctx


def _close(a, b):
    # identical per-pixel code and reduction order: the same sums, bit for bit
    assert np.array_equal(a, b), np.abs(a - b).max()


def test_static_scratch_matches_allocating_entry_point():
    s, ctx = _tracked_context()
    rng = np.random.default_rng(0)
    for slot in (0, 1):
        base = ctx.track_info(slot)[2]  # the problem's tracked FP64 pose
        for level in range(3):
            pose = base.astype(np.float64).copy()
            pose[:3, 3] += rng.normal(scale=0.002, size=3)
            pose = pose.astype(np.float32)
            first = ctx.track_eval_static(slot, level, pose)
            ref = ctx.track_eval(slot, level, pose)
            second = ctx.track_eval_static(slot, level, pose)
            assert ref[28] > 0, (slot, level, ref[28])
            _close(first, ref)
            _close(second, ref)
            # no pose: the problem's current float pose (track_eval just set it)
            _close(ctx.track_eval_static(slot, level, None), ref)
    assert ctx.status() == 0
    ctx.close()


def test_static_scratch_rejects_slots_without_a_problem():
    s, ctx = _tracked_context()
    sums = np.zeros(32, np.float64)
    for fn in (ctx.lib.mf_track_eval_static, ctx.lib.mf_track_eval):
        rc = fn(ctx.h, 5, 0, None, sums.ctypes.data_as(C.c_void_p))  # slots 0..2 are set up
        assert rc == -5  # MF_E_STATE
        assert b"no tracking problem" in ctx.lib.mf_last_error(ctx.h)
    assert ctx.status() == 0
    ctx.close()


def test_static_scratch_rejects_levels_beyond_its_size():
    # level 0 of 2560 x 1920 needs 6400 CTA partials; the scratch holds 4096
    ctx = Context(2560, 1920, pool_blocks=1 << 10)
    sums = np.zeros(32, np.float64)
    rc = ctx.lib.mf_track_eval_static(ctx.h, 0, 0, None, sums.ctypes.data_as(C.c_void_p))
    assert rc == -1  # MF_E_ARG
    assert b"4096" in ctx.lib.mf_last_error(ctx.h)
    ctx.close()

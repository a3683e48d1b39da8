"""The oracle's integration-through-objects, composite raycast, render and
static-state restatements against the reference's own code (CPU only;
skipped where oracle/_ref was not built, e.g. without the reference tree).

The reference side is object.cpp's Object::integrate_volume_kernel
(object.cpp:128-195), rendering.cpp's raycastObjectList (:9-181),
renderVolume_many_Kernel (:489-646), the depth / intensity / normal / track
renders (:183-237, 346-487, 648-664) and check_static_state (:907-947),
compiled unmodified into oracle/_ref/libmf_ref_track.so.
"""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.skipif(O.reference_tracking() is None,
                                reason="oracle/_ref not built (no reference tree)")

W, H = 160, 120
NEAR, FAR, MU = 0.1, 4.0, 0.1
EPS_SIZE = 256
if O.reference_tracking() is not None:
    # ray_iterator's direction epsilon is a static set by the first iterator
    # this library builds (lib/octree.hpp:931): pin it before any raycast.
    O.reference_tracking().rt_pin_epsilon(EPS_SIZE)


@pytest.fixture(scope="module")
def env():
    s = make_scene("multi", W, H, n_frames=2, seed=5, bg_size=EPS_SIZE, obj_size=128,
                   n_objects=3)
    assert s.instances[0].size == EPS_SIZE
    labels = [i.label for i in s.instances]
    orc = O.oracle()
    trk = O.RefTracker(W, H, s.k)
    poses = [p.astype(np.float32) for p in s.volume_poses(0)]
    vols = [orc.volume(i.size, i.dim) for i in s.instances]
    objs = [O.RefObject(trk, P, size=i.size, dim=i.dim, label=i.label)
            for i, P in zip(s.instances, poses)]
    T0 = s.cam_poses[0].astype(np.float32)
    d, rgb, lab = s.render(0)
    masks = generalize_masks(lab, labels)
    rgb3 = rgb.astype(np.float32) / np.float32(255.0)
    for i in range(len(labels)):
        vols[i].integrate(d, rgb3, masks[i], T0, poses[i], s.k, MU)
        objs[i].integrate(d, rgb3, masks[i], T0, s.k, MU)
    colors = np.random.default_rng(3).integers(0, 256, size=(91, 4)).astype(np.uint8)
    colors[:, 3] = 0
    return dict(s=s, labels=labels, poses=poses, vols=vols, objs=objs, trk=trk, T0=T0, d=d,
                rgb=rgb, rgb3=rgb3, colors=colors, RR=O.RefRender(W, H), R=O.Render(W, H),
                oob=orc.raycast_oob_mask(vols, poses, T0, s.k, W, H, eps_size=EPS_SIZE))


def test_object_integration_and_composite_raycast_match_reference(env):
    e = env
    orc = O.oracle()
    vo = np.zeros((H, W, 3), np.float32)
    no = np.zeros((H, W, 3), np.float32)
    lo = np.zeros((H, W), np.int32)
    orc.raycast_objects(e["vols"], e["poses"], e["labels"], e["T0"], e["s"].k, W, H,
                        eps_size=EPS_SIZE, vertex=vo, normal=no, label_img=lo)
    vr, nr, lr = e["RR"].raycast(e["objs"], e["T0"], e["s"].k, NEAR, FAR, MU)
    bad = np.any(vo != vr, axis=-1) | np.any(no != nr, axis=-1) | (lo != lr)
    # rays that read coordinates outside [0, size) hit undefined behaviour in
    # the reference (an aliased block): the oracle marks them
    assert not np.any(bad & ~e["oob"]), np.argwhere(bad & ~e["oob"])[:10]
    assert (lr >= 0).mean() > 0.5 and len(np.unique(lr)) >= 3


@pytest.mark.parametrize("color", [True, False])
def test_volume_render_matches_reference(env, color):
    e = env
    k = e["s"].k
    # with its own composite raycast, from the camera pose
    want = e["RR"].volume(e["objs"], e["T0"], k, NEAR, 2 * FAR, MU, 0.75 * MU, color, e["colors"])
    got = e["R"].volume(e["vols"], e["poses"], e["labels"], e["T0"], k, NEAR, 2 * FAR, MU,
                        0.75 * MU, float(np.float32(2.0 ** -np.log2(EPS_SIZE))), color, e["colors"])
    bad = (got != want).any(-1)
    assert not np.any(bad & ~e["oob"]), np.count_nonzero(bad & ~e["oob"])
    # shading the last raycast's maps
    maps = e["RR"].raycast(e["objs"], e["T0"], k, NEAR, FAR, MU)
    want = e["RR"].volume(e["objs"], e["T0"], k, NEAR, 2 * FAR, MU, 0.075, color, e["colors"],
                          maps=maps)
    got = e["R"].volume(e["vols"], e["poses"], e["labels"], None, k, NEAR, 2 * FAR, MU, 0.075,
                        float(np.float32(2.0 ** -np.log2(EPS_SIZE))), color, e["colors"],
                        maps=maps, T_shade=e["T0"])
    assert np.array_equal(got, want), np.count_nonzero((got != want).any(-1))


def test_image_renders_match_reference(env):
    e = env
    RR, R = e["RR"], e["R"]
    assert np.array_equal(RR.depth(e["d"], NEAR, FAR), R.depth(e["d"], NEAR, FAR))
    grey = e["trk"].grey(e["rgb"])
    assert np.array_equal(RR.intensity(grey), R.intensity(grey))
    _, n, _ = RR.raycast(e["objs"], e["T0"], e["s"].k, NEAR, FAR, MU)
    assert np.array_equal(RR.normal(n), R.normal(n))


def test_track_renders_and_static_state_match_reference(env):
    e = env
    s, k, T0 = e["s"], e["s"].k, e["T0"]
    vm, nm, lm = e["RR"].raycast(e["objs"], T0, k, NEAR, FAR, MU)
    d1, rgb1, _ = s.render(1)
    trk = O.RefTracker(W, H, k)
    trk.set_frame(e["rgb"], e["d"])
    trk.set_ref()
    trk.set_frame(rgb1, d1)
    Tc = trk.track_camera(T0, T0, vm, nm)
    lv, _, _ = e["RR"].raycast(e["objs"], Tc, k, NEAR, FAR, MU)
    res, err, _ = trk.compute_residuals(Tc, T0, vm, nm, lv)
    ok = res == 1
    err = np.where(ok, err, np.float32(0))   # rejected rows keep stale errors in the reference
    for mode in (0, 1, 2):
        want = e["RR"].track(res, err, mode)
        got = e["R"].track(res.astype(np.int8), err, mode)
        assert np.array_equal(got, want), mode
    # check_static_state's inlier mask and the inlier ratio Kfusion::tracking
    # computes from it (kfusion.cpp:309-315)
    for label in e["labels"][1:]:
        om = ((lm == label) * 255).astype(np.uint8)
        if not om.any():
            continue
        for icp, rgb in ((True, True), (True, False), (False, True)):
            inl = e["RR"].static_inliers(om, res, icp, rgb)
            ratio = np.float32(np.count_nonzero(inl)) / np.float32(np.count_nonzero(om))
            assert ratio == np.float32(O.inlier_ratio(res.astype(np.int8), lm, label, icp, rgb))


def test_mask_renders_match_reference(env):
    """renderInstanceMaskKernel, renderMaskWithImageKernel and
    renderMaskMotionWithImageKernel (rendering.cpp:679-820) against the
    oracle, on the composite label image and every instance's residual rows.
    Labels index the colour table; the reference reads colors[-2] (before the
    vector) for an invalid label in the instance mask, undefined, so the
    instance-mask comparison leaves those pixels out."""
    e = env
    s, k, T0 = e["s"], e["s"].k, e["T0"]
    vm, nm, lm = e["RR"].raycast(e["objs"], T0, k, NEAR, FAR, MU)
    assert (lm == -2).any() and (lm >= 0).all(where=lm != -2)
    d1, rgb1, _ = s.render(1)
    trk = O.RefTracker(W, H, k)
    trk.set_frame(e["rgb"], e["d"])
    trk.set_ref()
    trk.set_frame(rgb1, d1)
    Tc = trk.track_camera(T0, T0, vm, nm)
    lv, _, _ = e["RR"].raycast(e["objs"], Tc, k, NEAR, FAR, MU)
    res, _, _ = trk.compute_residuals(Tc, T0, vm, nm, lv)
    for o in e["objs"]:
        o.set_results(res)
    rows = [res.astype(np.int8)] * len(e["objs"])
    rgb3 = e["rgb3"]
    ok = lm != -2
    want = e["RR"].mask(lm, rgb3, 0, e["colors"])
    got = e["R"].mask(lm, rgb3, 0, e["colors"])
    assert np.array_equal(got[ok], want[ok])
    for mode in (1, 2):
        want = e["RR"].mask(lm, rgb3, mode, e["colors"], e["objs"] if mode == 2 else ())
        got = e["R"].mask(lm, rgb3, mode, e["colors"], rows if mode == 2 else ())
        assert np.array_equal(got, want), mode

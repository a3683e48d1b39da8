"""Motion segmentation (Tracking::compute_residuals, check_static_state,
Object::refine_mask_use_motion and the moving-object decision of
kfusion.cpp:287-338) against the oracle, bit-exact:

* the live raycast at the tracked camera pose (objects at their last poses);
* per-pixel ICP and photometric result codes and errors of the motion
  residuals, for ICP + photometric, ICP only and photometric only;
* per-object inlier ratios and the moving-label bits;
* the level-0 row codes of the camera and object GN problems
  (Object::trackresult_) at the pose they were evaluated at, the masked
  second camera track included, and the mask refinement from both.
"""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _setup(use_icp=True, use_rgb=True, seed=5):
    """Frame 0 integrated and raycast on the device and in the oracle; frame 1
    preprocessed and the camera tracked on the device."""
    s = make_scene("multi", W, H, n_frames=2, seed=seed, bg_size=256, obj_size=128,
                   n_objects=3)
    labels = [i.label for i in s.instances]
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, robust="huber", use_icp=use_icp,
                  use_rgb=use_rgb)
    orc = O.oracle()
    vols = []
    poses = s.volume_poses(0)
    for inst, T in zip(s.instances, poses):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
        vols.append(orc.volume(inst.size, inst.dim))
    T0 = s.cam_poses[0].astype(np.float32)
    d, rgb, lab = s.render(0)
    masks = generalize_masks(lab, labels)
    ctx.set_camera_pose(T0)
    ctx.upload(d, rgb, masks)
    ctx.integrate(list(range(len(labels))))
    rgb3 = rgb.astype(np.float32) / np.float32(255.0)
    for i, v in enumerate(vols):
        v.integrate(d, rgb3, masks[i], T0, poses[i], s.k, 0.1)
    ctx.raycast()
    ctx.preprocess()
    ref = {8: ctx.pyramid(0, 1).copy(), 9: ctx.pyramid(0, 2).copy()}
    ctx.set_ref_from_current()
    model = ctx.download_raycast()
    d1, rgb1, lab1 = s.render(1)
    masks1 = generalize_masks(lab1, labels)
    ctx.upload(d1, rgb1, masks1)
    ctx.preprocess()
    ctx.track_camera()
    trk = O.Tracker(W, H, s.k, robust=1, use_icp=use_icp, use_rgb=use_rgb, fp64=False)
    trk.set_frame(rgb, d)
    trk.set_ref()
    trk.set_frame(rgb1, d1)
    # the oracle's level-0 planes from the device's preprocessing (which
    # matches the oracle's to a few ulp: expf in the bilateral weights), so
    # that the per-pixel codes compare bit for bit
    for which in (1, 2, 3, 4, 5, 6):
        trk.set_level(0, which, ctx.pyramid(0, which))
    for which, plane in ref.items():
        trk.set_level(0, which, plane)
    return dict(s=s, ctx=ctx, orc=orc, vols=vols, poses=poses, labels=labels, T0=T0,
                model=model, masks1=masks1, trk=trk)


@pytest.mark.parametrize("terms", ["icp+rgb", "icp", "rgb"])
def test_motion_residuals_match_oracle(terms):
    use_icp, use_rgb = "icp" in terms, "rgb" in terms
    e = _setup(use_icp, use_rgb)
    ctx, s, labels = e["ctx"], e["s"], e["labels"]
    ratio, bits = ctx.motion_residuals(1.5, 0.9)
    res, err, lvert, llab = ctx.motion_download()
    T_w_l = ctx.camera_pose()
    # the live raycast (objects at their frame-0 poses), bit-exact
    vo = np.zeros((H, W, 3), np.float32)
    no = np.zeros((H, W, 3), np.float32)
    lo = np.zeros((H, W), np.int32)
    e["orc"].raycast_objects(e["vols"], e["poses"], labels, T_w_l, s.k, W, H,
                             eps_size=s.instances[0].size, vertex=vo, normal=no, label_img=lo)
    assert np.array_equal(llab, lo)
    assert np.array_equal(lvert, vo)
    v, n, _ = e["model"]
    ores, oerr = e["trk"].motion_residuals(T_w_l, e["T0"], v, n, lvert, 1.5)
    for plane, on in ((0, use_icp), (1, use_rgb)):
        r = res[plane]
        assert np.array_equal(r, ores[plane]), \
            (plane, np.count_nonzero(r != ores[plane]))
        assert np.array_equal(err[plane], oerr[plane]), plane
        if on:  # not vacuous: inliers and threshold outliers present
            assert np.count_nonzero(r == 1) > 5000, (plane, np.unique(r, return_counts=True))
            assert np.count_nonzero(r == -4) > 0, plane
        else:
            assert not r.any()
    expect = 0
    for i, l in enumerate(labels):
        o = O.inlier_ratio(res.reshape(-1), llab, l, use_icp, use_rgb) if i else -1.0
        assert ratio[i] == np.float32(o), (i, ratio[i], o)
        if i and 0.05 < o < 0.9:
            expect |= 1 << l
    assert bits == expect
    assert (ratio[1:] > 0).all(), ratio  # every object is in view
    assert ctx.status() == 0
    ctx.close()


def test_track_results_and_mask_refinement_match_oracle():
    import torch
    e = _setup()
    ctx, s, labels, trk = e["ctx"], e["s"], e["labels"], e["trk"]
    v, n, lbl = e["model"]
    T0 = e["T0"]
    buf = torch.zeros(2 * W * H, dtype=torch.int8, device="cuda")

    def codes(i):
        pose = ctx.track_results(i, buf.data_ptr())
        return pose, buf.cpu().numpy().reshape(2, H, W).copy()

    # the camera's rows at its last level-0 evaluation
    pose, c0 = codes(0)
    trk.camera_sums(0, pose, T0, v, n)
    assert np.array_equal(c0, trk.last_results())
    assert np.count_nonzero(c0[0] == 1) > 5000 and np.count_nonzero(c0[1] == 1) > 5000
    ratio, bits = ctx.motion_residuals(1.5, 0.9)
    res, _, _, _ = ctx.motion_download()
    # the masked second camera track with the moving objects (at least one)
    moving = bits or (1 << labels[1])
    ctx.retrack_camera(moving)
    pose2, c1 = codes(0)
    mask = (np.isin(lbl, [l for l in labels if moving >> l & 1]) * 255).astype(np.uint8)
    trk.set_mask(mask)
    trk.camera_sums(0, pose2, T0, v, n)
    assert np.array_equal(c1, trk.last_results())
    assert np.count_nonzero(c1[0] == -6) == np.count_nonzero(mask)
    trk.set_mask(np.zeros_like(mask))
    # objects tracked from the retracked camera pose
    ids = list(range(1, len(labels)))
    ctx.track_objects(ids)
    obj_codes = {}
    for i in ids:
        pose_i, ci = codes(i)
        trk.object_sums(0, pose_i, e["poses"][i], T0, v, n, lbl, labels[i])
        assert np.array_equal(ci, trk.last_results()), i
        assert np.count_nonzero(ci[0] == 1) > 100, i
        obj_codes[i] = (ci, buf.clone())
    # refine_mask_use_motion: the background with the motion residual planes,
    # each object with its own rows
    m0 = ctx.mask(0)
    assert np.array_equal(m0, e["masks1"][0])
    ctx.refine_mask_use_motion(0)
    got = ctx.mask(0)
    want = O.refine_mask_use_motion(m0, res.reshape(-1))
    assert np.array_equal(got, want)
    assert np.count_nonzero(got != m0) > 0
    for i in ids:
        ci, dev = obj_codes[i]
        mi = ctx.mask(i)
        ctx.refine_mask_use_motion(i, dev.data_ptr())
        assert np.array_equal(ctx.mask(i), O.refine_mask_use_motion(mi, ci.reshape(-1))), i
    assert ctx.status() == 0
    ctx.close()


def test_object_residuals_at_the_virtual_pose_match_oracle():
    """mf_object_residuals (kfusion.cpp:446-466): after the objects are
    tracked and the live raycast is redone at their new poses, each object's
    rows recomputed by compute_residuals at its virtual camera pose against
    its own pixels of the model maps and of the live raycast, against the
    oracle's compute_residuals on the same inputs, bit-exact; and the
    never-moving classes (Object::static_object) never move."""
    import torch
    e = _setup()
    ctx, labels = e["ctx"], e["labels"]
    ids = list(range(1, len(labels)))
    ctx.track_objects(ids)
    ctx.motion_residuals(1.5, 0.9)   # the live raycast at the objects' new poses
    _, _, lvert, llab = ctx.motion_download()
    v, n, lab = e["model"]
    T_w_r = e["T0"]
    buf = torch.zeros(2 * W * H, dtype=torch.int8, device="cuda")
    checked = 0
    for i in ids:
        T_virt = ctx.object_residuals(i, buf.data_ptr(), 1.5)
        got = buf.cpu().numpy().reshape(2, H, W)
        l = labels[i]
        own = (lab == l)[..., None]
        mv = np.where(own, v, np.float32(0)).astype(np.float32)
        mn = np.where(own, n, np.array([-2.0, 0, 0], np.float32)).astype(np.float32)
        lv = np.where((llab == l)[..., None], lvert, np.float32(0)).astype(np.float32)
        want, _ = e["trk"].motion_residuals(T_virt, T_w_r, mv, mn, lv, 1.5)
        assert np.array_equal(got, want), (i, np.count_nonzero(got != want))
        # the virtual pose maps the object's last pose to the new relative view
        T_wo1 = e["poses"][i].astype(np.float64)
        T_wo2 = ctx.instance_pose(i).astype(np.float64)
        T_c = ctx.camera_pose().astype(np.float64)
        np.testing.assert_allclose(np.linalg.inv(T_virt) @ T_wo1, np.linalg.inv(T_c) @ T_wo2,
                                   atol=1e-4)
        checked += int(np.count_nonzero(got[0] == 1) > 0)
    assert checked >= 2
    # a never-moving class: the same frame reports no motion for that object
    for i in ids:
        ctx.lib.mf_instance_set_semantics(ctx.h, i, 63, None, 0)
    _, bits = ctx.motion_residuals(1.5, 1.01)   # every object with inliers "moves"...
    assert bits == 0                             # ...unless its class never moves
    assert ctx.status() == 0
    ctx.close()

"""Known-answer checks of the oracle's motion segmentation restatement
(Tracking::compute_residuals, tracking.cpp:1535-1747; check_static_state,
rendering.cpp:907-947; Object::refine_mask_use_motion, object.cpp:255-315)
on cases whose result codes follow from the reference's rules by hand."""
import numpy as np

import _oracle as O

W, H = 32, 24
K = [30.0, 30.0, 15.5, 11.5]


def _tracker(use_icp=True, use_rgb=True):
    """A fronto-parallel plane at 1 m with constant intensity, live = reference."""
    d = np.ones((H, W), np.float32)
    rgb = np.full((H, W, 3), 128, np.uint8)
    t = O.Tracker(W, H, K, use_icp=use_icp, use_rgb=use_rgb, fp64=False)
    t.set_frame(rgb, d)
    t.set_ref()
    t.set_frame(rgb, d)
    return t


def _interior():
    m = np.zeros((H, W), bool)
    m[1:H - 1, 1:W - 1] = True
    return m


def test_identical_frames_are_inliers_with_zero_error():
    t = _tracker()
    v, n = t.level(0, 2), t.level(0, 3)
    I4 = np.eye(4, dtype=np.float32)
    res, err = t.motion_residuals(I4, I4, v, n, v, 1.5)
    valid = n[..., 0] != -2
    # ICP: no normal -> -1; a pixel projects onto itself, so the border
    # (outside [1, W-2] x [1, H-2]) is -2; inside, zero distance -> 1
    assert (res[0][~valid] == -1).all()
    inner = valid & _interior()
    assert inner.sum() > 400
    assert (res[0][inner] == 1).all() and (err[0][inner] == 0).all()
    assert (res[0][valid & ~_interior()] == -2).all()
    # photometric: constant intensity -> residual 0 inside, -2 on the border
    assert (res[1][_interior()] == 1).all() and (err[1] == 0).all()
    assert (res[1][~_interior()] == -2).all()


def test_distance_normal_and_missing_model_codes():
    t = _tracker(use_rgb=False)
    v, n = t.level(0, 2), t.level(0, 3)
    I4 = np.eye(4, dtype=np.float32)
    inner = (n[..., 0] != -2) & _interior()
    far = v.copy()
    far[..., 2] += 0.2  # model 0.2 m behind: length(diff) > 0.1 -> -4
    res, _ = t.motion_residuals(I4, I4, far, n, v, 1.5)
    assert (res[0][inner] == -4).all()
    flip = -n  # opposite normals: dot < 0.8 -> -5
    res, _ = t.motion_residuals(I4, I4, v, flip, v, 1.5)
    assert (res[0][inner] == -5).all()
    none = n.copy()
    none[..., 0] = -2  # no model normal -> -3
    res, _ = t.motion_residuals(I4, I4, v, none, v, 1.5)
    assert (res[0][inner] == -3).all()
    assert not res[1].any()  # photometric rows off


def test_photometric_occlusion_and_missing_render_codes():
    t = _tracker(use_icp=False)
    v, n = t.level(0, 2), t.level(0, 3)
    I4 = np.eye(4, dtype=np.float32)
    res, _ = t.motion_residuals(I4, I4, v, n, np.zeros_like(v), 1.5)
    assert (res[1] == -1).all()  # nothing rendered
    behind = v * np.float32(1.5)  # rendered surface 0.5 m behind the live one -> -5
    res, _ = t.motion_residuals(I4, I4, v, n, behind, 1.5)
    assert (res[1] == -5).all()
    assert not res[0].any()


def test_inlier_ratio_and_refinement_rules():
    n = 8
    icp = np.array([1, -1, -2, -3, -4, -5, -6, 1], np.int8)
    rgb = np.array([1, 1, 1, 1, 1, -4, -5, -3], np.int8)
    res = np.concatenate([icp, rgb])
    labels = np.array([2, 2, 2, 2, 2, 2, 3, 3], np.int32)
    # inlier: every row that is on is > -3
    assert O.inlier_ratio(res, labels, 2) == np.float32(3 / 6)
    assert O.inlier_ratio(res, labels, 3) == 0.0
    assert O.inlier_ratio(res, labels, 2, use_rgb=False) == np.float32(3 / 6)
    assert O.inlier_ratio(res, labels, 2, use_icp=False) == np.float32(5 / 6)
    assert O.inlier_ratio(res, labels, 7) == -1.0  # not in view
    mask = np.array([1, 0.5, 0, 0.1, 1, 1, 1, -1], np.float32)
    # inside the band: ICP -4 / -6 or photometric < -3 leave the mask
    want = np.array([1, 0.5, 0, 0.1, -1, -1, -1, -1], np.float32)
    assert np.array_equal(O.refine_mask_use_motion(mask, res), want)
    want_rgb = np.array([1, 0.5, 0, 0.1, 1, -1, -1, -1], np.float32)
    assert np.array_equal(O.refine_mask_use_motion(mask, res, use_icp=False), want_rgb)
    assert n == len(icp)

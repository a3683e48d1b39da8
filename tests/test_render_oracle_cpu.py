"""Known-answer checks of the oracle's render restatement
(rendering.cpp's visualisation kernels, gs2rgb of commons.h:87-147), values
worked out by hand from the reference's formulas."""
import numpy as np

import _oracle as O

W, H = 4, 2


def test_depth_render_ramp_and_planes():
    R = O.Render(W, H)
    near, far = 0.5, 2.5
    d = np.array([[0.4, 0.5, 1.5, 3.0], [2.5, 1.0, 0.0, 2.0]], np.float32)
    out = R.depth(d, near, far)
    assert tuple(out[0, 0]) == (255, 255, 255, 0)      # nearer than the near plane
    assert tuple(out[0, 3]) == (0, 0, 0, 0)            # beyond the far plane
    assert tuple(out[1, 2]) == (255, 255, 255, 0)      # no depth
    assert tuple(out[0, 1]) == (191, 63, 63, 0)        # h = 0: sextant 0
    assert tuple(out[0, 2]) == (63, 191, 191, 0)       # h = 0.5: sextant 3
    # h = 1 at the far plane: sextant 6, the default branch -> black
    assert tuple(out[1, 0]) == (0, 0, 0, 0)


def test_track_renders_colour_tables():
    R = O.Render(W, H)
    n = W * H
    icp = np.array([1, -1, -2, -3, -4, -5, -6, 7], np.int8)
    rgb = np.array([1, -1, -2, -3, -4, -5, 1, 3], np.int8)
    res = np.concatenate([icp, rgb])
    err = np.zeros(2 * n, np.float32)
    err[n] = 0.5     # |0.5 * 255| = 127.5 -> 127
    err[n + 6] = -1.2  # 306 -> low byte 50 (the x86-64 conversion)
    t0 = R.track(res, err, 0).reshape(n, 4)
    assert [tuple(c) for c in t0] == [(128, 128, 128, 0), (0, 0, 0, 0), (255, 0, 0, 0),
                                      (0, 255, 0, 0), (0, 0, 255, 0), (255, 255, 0, 0),
                                      (255, 175, 175, 0), (255, 200, 128, 0)]
    t1 = R.track(res, err, 1).reshape(n, 4)
    assert tuple(t1[0]) == (127, 127, 127, 255) and tuple(t1[6]) == (50, 50, 50, 255)
    assert [tuple(c) for c in t1[1:6]] == [(0, 255, 0, 0), (0, 0, 0, 0), (255, 0, 0, 0),
                                           (0, 0, 255, 0), (255, 255, 0, 0)]
    assert tuple(t1[7]) == (255, 128, 128, 0)
    t2 = R.track(res, err, 2).reshape(n, 4)
    assert tuple(t2[0]) == (127, 127, 127, 255)        # both rows inliers
    assert tuple(t2[4]) == (255, 0, 0, 0)              # -4: high residual
    assert tuple(t2[2]) == (255, 255, 0, 0)            # -2
    assert tuple(t2[1]) == (0, 255, 0, 0)              # -1
    assert tuple(t2[6]) == (255, 175, 175, 0)          # -6 with an inlier photometric row


def test_normal_intensity_and_mask_renders():
    R = O.Render(W, H)
    nr = np.zeros((H, W, 3), np.float32)
    nr[0, 0] = (0, 0, -1)
    nr[0, 1] = (1, 0, 0)     # 1 * 128 + 128 = 256 -> low byte 0
    nr[0, 2] = (-2, 5, 5)    # invalid
    nr[0, 3] = (0, 0, 2)     # normalised first
    out = R.normal(nr)
    assert tuple(out[0, 0]) == (128, 128, 0) and tuple(out[0, 1]) == (0, 128, 128)
    assert tuple(out[0, 2]) == (0, 0, 0) and tuple(out[0, 3]) == (128, 128, 0)
    g = np.array([[1.0, 0.5, 0.0, 0.25], [0.1, 0.2, 0.3, 0.4]], np.float32)
    assert [int(v) for v in R.intensity(g)[0, :, 0]] == [255, 127, 0, 63]
    assert (R.intensity(g)[..., 3] == 255).all()
    colors = np.array([[10, 20, 30, 0], [200, 100, 50, 0]], np.uint8)
    lab = np.array([[0, 1, -2, 5], [1, 1, 0, 0]], np.int32)
    m0 = R.mask(lab, np.zeros((H, W, 3), np.float32), 0, colors)
    assert tuple(m0[0, 0]) == (10, 20, 30, 0) and tuple(m0[0, 1]) == (200, 100, 50, 0)
    assert tuple(m0[0, 3]) == (0, 0, 0, 0)            # outside the table
    rgb = np.full((H, W, 3), 1.0, np.float32)
    m1 = R.mask(lab, rgb, 1, colors)
    # 255 * 0.3 + 200 * 0.7 = 216.5 -> 216; invalid: 255 * 0.3 + 128 * 0.7 -> 166, b 255
    assert tuple(m1[0, 1][:3]) == (216, 146, 111)
    assert tuple(m1[0, 2][:3]) == (166, 166, 255)
    assert tuple(m1[0, 0][:3]) == (255, 255, 255)     # background: the image

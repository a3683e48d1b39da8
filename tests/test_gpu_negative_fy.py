"""The tracking pyramid with a negative fy (the ICL-NUIM convention) on the
GPU against the FP32 oracle, which equals the reference's there
(tests/test_track_reference_cpu.py): the reference takes the rows above and
below in the other order for the normals (vertex2normalKernel with NegY,
tracking.cpp:805-810).  Frames rendered with fy > 0 and flipped upside down
are the same scene seen through (fx, -fy, cx, H - 1 - cy)."""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def test_pyramid_negative_fy_matches_oracle():
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    k = np.asarray(s.k, np.float32)
    kneg = np.array([k[0], -k[1], k[2], H - 1 - k[3]], np.float32)
    d, rgb, _ = s.render(1)
    d = np.ascontiguousarray(d[::-1], np.float32)
    rgb = np.ascontiguousarray(rgb[::-1])
    ctx = Context(W, H, k=kneg, pool_blocks=1 << 12, robust="huber")
    ctx.add_instance(s.instances[0].size, s.instances[0].dim, s.volume_poses(0)[0],
                     s.instances[0].label)
    ctx.upload(d, rgb, None)
    ctx.preprocess()
    trk = O.Tracker(W, H, kneg, robust=1, fp64=False)
    trk.set_frame(rgb, d)
    for l in range(3):
        gv, ov = ctx.pyramid(l, 2), trk.level(l, 2)
        np.testing.assert_allclose(gv, ov, rtol=2e-5, atol=1e-6, err_msg=f"vertex L{l}")
        gn, on = ctx.pyramid(l, 3), trk.level(l, 3)
        inv_g, inv_o = gn[..., 0] == -2, on[..., 0] == -2
        assert np.array_equal(inv_g, inv_o), f"invalid normals differ at L{l}"
        assert (~inv_g).sum() > 0.5 * inv_g.size, l
        # as in the fy > 0 pyramid test: the normals difference neighbouring
        # vertices, which amplifies ulp-level depth differences
        np.testing.assert_allclose(gn[~inv_g], on[~inv_o], rtol=0, atol=3e-4)
        # the swap matters: the normals face the camera (negative z in the
        # camera frame), as they do for fy > 0
        assert np.mean(gn[~inv_g][:, 2] < 0) > 0.9, l
    assert ctx.status() == 0
    ctx.close()

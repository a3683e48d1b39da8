"""Object spawning (mf_spawn_object) and semantic fusion (mf_fuse_semantics)
against the oracle's sequential restatement, exactly: the new volume's pose,
size and resolution from a mask of one object, of every pixel, of no pixel
and of a scattered random set; the fused class probabilities, class id and
fused count over a sequence of recognitions."""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.gpu

W, H = 640, 480


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def test_spawn_object_matches_oracle():
    s = make_scene("multi", W, H, n_frames=1, seed=7, bg_size=256, obj_size=128, n_objects=3)
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 12)
    ctx.add_instance(s.instances[0].size, s.instances[0].dim, s.volume_poses(0)[0], 0)
    d, rgb, lab = s.render(0)
    T = s.cam_poses[0].astype(np.float32)
    ctx.set_camera_pose(T)
    ctx.upload(d, rgb, None)
    rng = np.random.default_rng(1)
    masks = [(lab == s.instances[i].label) for i in range(1, len(s.instances))]
    masks += [np.ones((H, W), bool), np.zeros((H, W), bool), rng.random((H, W)) < 0.3]
    for j, m in enumerate(masks):
        m8 = m.astype(np.uint8) * 255
        Tg, sg, rg, ng = ctx.spawn_object(m8)
        To, so, ro, no = O.spawn_object(d, m8, s.k, T)
        assert ng == no == int(m.sum()), j
        assert rg == ro, (j, rg, ro)
        assert np.array_equal(np.float32(sg), np.float32(so), equal_nan=True), (j, sg, so)
        assert np.array_equal(Tg, To, equal_nan=True), (j, Tg, To)
    ctx.close()


def test_semantic_fusion_matches_oracle():
    ctx = Context(64, 48, pool_blocks=1 << 10)
    for i in range(3):
        ctx.add_instance(64, 0.5, np.eye(4), i)
    rng = np.random.default_rng(2)
    alpha = np.full(80, 0.3)
    for i in (1, 2):
        p0 = rng.dirichlet(alpha).astype(np.float32)
        ctx.set_semantics(i, int(np.argmax(p0)) + 1, p0)
        fused, ft = p0.copy(), 1
        for step in range(12):
            p = rng.dirichlet(alpha).astype(np.float32)
            cls = 0 if step == 5 else int(rng.integers(1, 81))
            rt = int(rng.integers(1, 4))
            ctx.fuse_semantics(i, cls, p, rt)
            if cls != 0:
                fused, ft, cid = O.fuse_semantics(fused, ft, p, rt)
            gcid, gft, gp = ctx.semantics(i)
            assert gft == ft and np.array_equal(gp, fused), (i, step)
            if cls != 0:
                assert gcid == cid
    ctx.close()

"""The instance-sharded composite raycast on one GPU: the instances split
between two emulated ranks, each rank's records (mf_raycast_records) gathered
in instance order as an all-gather would, and folded (mf_raycast_fold); the
maps equal the one-GPU composite (mf_raycast) bit for bit, on the 3-object
and the 12-object scenes over several frames."""
import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

REC, ORIG = 48, 32   # bytes of mf_ray_record, mf_ray_origin


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


@pytest.mark.parametrize("preset", ["multi", "uneven"])
def test_sharded_fold_equals_the_composite(preset):
    import torch
    W, H = 320, 240
    if preset == "multi":
        s = make_scene("multi", W, H, n_frames=3, seed=5, bg_size=256, obj_size=128,
                       n_objects=3)
    else:
        s = make_scene("uneven", W, H, n_frames=3, seed=23, n_objects=12)
    n = len(s.instances)
    labels = [i.label for i in s.instances]
    # one context composites with mf_raycast; the other, with the same
    # volumes, only through records and the fold (so that the maps' earlier
    # contents, which a zero-gradient normal keeps, evolve alike)
    ctx, shard = (Context(W, H, k=s.k, pool_blocks=1 << 15, robust="huber") for _ in range(2))
    for c in (ctx, shard):
        for inst, T in zip(s.instances, s.volume_poses(0)):
            c.add_instance(inst.size, inst.dim, T, inst.label)
    ranks = [list(range(0, n, 2)), list(range(1, n, 2))]   # two emulated GPUs
    recs = [torch.zeros((len(r), H, W, REC), dtype=torch.uint8, device="cuda") for r in ranks]
    origs = [torch.zeros((len(r), ORIG), dtype=torch.uint8, device="cuda") for r in ranks]
    gathered = torch.zeros((n, H, W, REC), dtype=torch.uint8, device="cuda")
    gorig = torch.zeros((n, ORIG), dtype=torch.uint8, device="cuda")
    for f in range(s.n_frames):
        d, rgb, lab = s.render(f)
        for c in (ctx, shard):
            for i, P in enumerate(s.volume_poses(f)):
                c.set_instance_pose(i, P)
            c.set_camera_pose(s.cam_poses[f])
            c.upload(d, rgb, generalize_masks(lab, labels))
            c.integrate(list(range(n)))
        ctx.raycast()
        want = [a.copy() for a in ctx.download_raycast()]
        for r, ids in enumerate(ranks):
            shard.raycast_records(ids, recs[r].data_ptr(), origs[r].data_ptr())
        torch.cuda.synchronize()
        for r, ids in enumerate(ranks):   # the all-gather, reassembled in instance order
            for k, i in enumerate(ids):
                gathered[i] = recs[r][k]
                gorig[i] = origs[r][k]
        torch.cuda.synchronize()
        shard.raycast_fold(gathered.data_ptr(), gorig.data_ptr())
        got = shard.download_raycast()
        for a, b, what in zip(got, want, ("vertex", "normal", "label")):
            assert np.array_equal(a, b), (f, what, np.argwhere(a != b)[:5])
        assert (want[2] >= 0).mean() > 0.5 and len(np.unique(want[2])) >= 3
    assert ctx.status() == 0 and shard.status() == 0
    ctx.close()
    shard.close()

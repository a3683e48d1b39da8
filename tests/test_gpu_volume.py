"""Allocation, integration and raycast on the GPU against the CPU oracle.

Bit-exact: block and node key sets, corner coordinates, children masks, active
flags, every voxel field (tsdf, weight, rgb, colour count, foreground
probability, foreground count) of every block and internal node, and the
composite raycast maps (vertex, normal, label).  The oracle itself is pinned to
the reference compiled from its own sources (tests/test_oracle_reference.py).
"""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "r", "g", "b", "c", "fg", "w"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _scene(seed=3, W=160, H=120, bg=256, obj=64, frames=3, n_objects=3):
    return make_scene("multi", W, H, n_frames=frames, seed=seed, bg_size=bg, obj_size=obj,
                      n_objects=n_objects)


def _assert_volume_equal(ctx, i, vol):
    kg, cg, ag, xg = ctx.blocks(i)
    ko, co, ao, xo = vol.blocks()
    assert np.array_equal(kg, ko), f"block keys differ: {len(kg)} vs {len(ko)}"
    assert np.array_equal(cg, co)
    assert np.array_equal(ag, ao), "active flags differ"
    for f in FIELDS:
        assert np.array_equal(xg[f], xo[f]), f"voxel field {f} differs"
    nkg, sg, cmg, nvg = ctx.nodes(i)
    nko, so, cmo, nvo = vol.nodes()
    assert np.array_equal(nkg, nko), "node keys differ"
    assert np.array_equal(sg, so)
    assert np.array_equal(cmg, cmo), "children masks differ"
    for f in FIELDS:
        assert np.array_equal(nvg[f], nvo[f]), f"node value field {f} differs"
    assert ctx.root_children(i) == vol.root_children()


@pytest.mark.parametrize("batched", [True, False])
def test_integrate_and_raycast_match_oracle(batched):
    s = _scene()
    orc = O.oracle()
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 13, batched=batched)
    vols = []
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
        vols.append(orc.volume(inst.size, inst.dim))
    labels = [i.label for i in s.instances]
    # the reference keeps its model maps across frames (a normal whose gradient is
    # zero only gets .x = INVALID), so the oracle keeps its buffers too
    vo = np.zeros((s.height, s.width, 3), np.float32)
    no = np.zeros((s.height, s.width, 3), np.float32)
    lo = np.zeros((s.height, s.width), np.int32)
    for f in range(s.n_frames):
        depth, rgb, lab = s.render(f)
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        for i, P in enumerate(poses):
            ctx.set_instance_pose(i, P)
        ctx.set_camera_pose(T)
        ctx.upload(depth, rgb, masks)
        ctx.integrate(list(range(len(vols))))
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(depth, rgb3, masks[i], T, poses[i], s.k, 0.1)
        for i, v in enumerate(vols):
            _assert_volume_equal(ctx, i, v)
        ctx.raycast()
        vg, ng, lg = ctx.download_raycast()
        orc.raycast_objects(vols, poses, labels, T, s.k, s.width, s.height,
                            eps_size=s.instances[0].size, vertex=vo, normal=no, label_img=lo)
        assert np.array_equal(lg, lo), f"labels differ at {np.count_nonzero(lg != lo)} px"
        assert np.array_equal(vg, vo), "vertex map differs"
        assert np.array_equal(ng, no), "normal map differs"
    assert ctx.status() == 0
    ctx.close()


def test_generalized_masks_on_device_match_host():
    s = _scene(frames=1)
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 12)
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
    depth, rgb, lab = s.render(0)
    masks = generalize_masks(lab, [i.label for i in s.instances])
    # integrate with device-generated masks and with host masks: same volume
    ctx2 = Context(s.width, s.height, k=s.k, pool_blocks=1 << 12)
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx2.add_instance(inst.size, inst.dim, T, inst.label)
    for c in (ctx, ctx2):
        c.set_camera_pose(s.cam_poses[0])
    ctx.upload(depth, rgb, None)
    ctx.upload_labels(lab)
    ctx2.upload(depth, rgb, masks)
    ids = list(range(len(s.instances)))
    ctx.integrate(ids)
    ctx2.integrate(ids)
    for i in ids:
        a, b = ctx.blocks(i), ctx2.blocks(i)
        assert np.array_equal(a[0], b[0])
        for f in FIELDS:
            assert np.array_equal(a[3][f], b[3][f])


def test_interp_matches_oracle():
    s = _scene(frames=1)
    orc = O.oracle()
    inst = s.instances[0]
    ctx = Context(s.width, s.height, k=s.k, pool_blocks=1 << 12)
    ctx.add_instance(inst.size, inst.dim, s.volume_poses(0)[0], 0)
    vol = orc.volume(inst.size, inst.dim)
    depth, rgb, lab = s.render(0)
    masks = generalize_masks(lab, [0])
    ctx.set_camera_pose(s.cam_poses[0])
    ctx.upload(depth, rgb, masks)
    ctx.integrate([0])
    vol.integrate(depth, rgb.astype(np.float32) / np.float32(255), masks[0], s.cam_poses[0],
                  s.volume_poses(0)[0], s.k, 0.1)
    rng = np.random.default_rng(0)
    pts = rng.uniform(0, inst.dim, size=(2000, 3)).astype(np.float32)
    for field in range(5):  # tsdf, fg, r, g, b
        g = ctx.interp(0, pts, field)
        o = np.array([vol.interp(p, field) for p in pts], np.float32)
        assert np.array_equal(g, o)


def test_alloc_update_matches_oracle_on_multiscale_keys():
    # the fixed coordinates of lib/test/algorithms/unique_unittest.cpp:76-101
    blocks = [(56, 12, 12), (56, 12, 15), (128, 128, 128), (128, 128, 125), (128, 128, 127),
              (128, 136, 129), (128, 136, 127), (136, 128, 136), (128, 240, 136),
              (128, 241, 136)]
    levels = [5, 5, 3, 5, 4, 5, 5, 5, 5, 5]
    orc = O.oracle()
    from mid_fusion_b200.capi import Context as Ctx
    keys = np.array([O.encode(x, y, z, l, 8) for (x, y, z), l in zip(blocks, levels)], np.uint64)
    ctx = Ctx(64, 48, pool_blocks=1 << 10)
    ctx.add_instance(256, 2.56, np.eye(4), 0)
    ctx.alloc_update(0, keys)
    vol = orc.volume(256, 2.56)
    vol.alloc_update(keys)
    kg, cg, ag, _ = ctx.blocks(0, with_voxels=False)
    ko, co, ao, _ = vol.blocks(with_voxels=False)
    assert np.array_equal(kg, ko) and np.array_equal(cg, co)
    nkg, sg, cmg, _ = ctx.nodes(0, with_values=False)
    nko, so, cmo, _ = vol.nodes(with_values=False)
    assert np.array_equal(nkg, nko) and np.array_equal(cmg, cmo) and np.array_equal(sg, so)

"""The oracle against the reference compiled from its own sources (CPU only;
skipped where oracle/_ref was not built, e.g. without the reference tree)."""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200.scene import generalize_masks, make_scene

ref = O.reference()
pytestmark = pytest.mark.skipif(ref is None, reason="oracle/_ref not built (no reference tree)")

# ray_iterator's direction epsilon is a function-local static set by the first
# ray_iterator of the process, from that octree's size (lib/octree.hpp:931):
# pin it once, before any test, and give the oracle the same size.
EPS_SIZE = 512
if ref is not None:
    ref.lib.ref_pin_epsilon(EPS_SIZE)


@pytest.mark.parametrize("preset,seed", [("multi", 3), ("multi", 8), ("uneven", 23)])
def test_oracle_matches_reference_sequence(preset, seed):
    W, H = 128, 96
    if preset == "multi":
        s = make_scene("multi", W, H, n_frames=3, seed=seed, bg_size=128, obj_size=64,
                       n_objects=2)
    else:  # 12 objects, octrees of 32^3 ... 256^3 at 2-5 mm, background 512^3
        s = make_scene("uneven", W, H, n_frames=3, seed=seed, n_objects=12)
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vo = [orc.volume(i.size, i.dim) for i in s.instances]
    vr = [ref.volume(i.size, i.dim) for i in s.instances]
    bo = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
    br = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
    for f in range(3):
        d, rgb, lab = s.render(f)
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i in range(len(labels)):
            a = vo[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
            b = vr[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
            assert a == b
            ko, co, ao, xo = vo[i].blocks()
            kr, cr, ar, xr = vr[i].blocks()
            assert np.array_equal(ko, kr) and np.array_equal(co, cr) and np.array_equal(ao, ar)
            assert xo.tobytes() == xr.tobytes()
            no, so, cmo, nvo = vo[i].nodes()
            nr, sr, cmr, nvr = vr[i].nodes()
            assert np.array_equal(no, nr) and np.array_equal(cmo, cmr) and np.array_equal(so, sr)
            assert nvo.tobytes() == nvr.tobytes()
            assert vo[i].root_children() == vr[i].root_children()
        orc.raycast_objects(vo, poses, labels, T, s.k, W, H, eps_size=EPS_SIZE,
                            vertex=bo[0], normal=bo[1], label_img=bo[2])
        ref.raycast_objects(vr, poses, labels, T, s.k, W, H, vertex=br[0], normal=br[1],
                            label_img=br[2])
        # Rays that sample coordinates outside [0, size) (e.g. entering a volume
        # through one of its upper faces) hit undefined behaviour in the
        # reference: its bit descent aliases them into another block and reads
        # past that block's voxel array (lib/octree.hpp:359-379,
        # lib/node.hpp:144-149).  The oracle and the device read them as
        # unallocated.  Every other pixel must agree exactly.
        oob = orc.raycast_oob_mask(vo, poses, T, s.k, W, H, eps_size=EPS_SIZE)
        bad = np.any(bo[0] != br[0], axis=-1) | np.any(bo[1] != br[1], axis=-1) | (bo[2] != br[2])
        assert not np.any(bad & ~oob), np.argwhere(bad & ~oob)[:10]
        assert oob.mean() < 0.05, oob.mean()
        for a, b in zip(bo, br):
            b[...] = a  # continue from the same maps


def test_alloc_update_multiscale_keys_match_reference():
    blocks = [(56, 12, 12), (56, 12, 15), (128, 128, 128), (128, 128, 125), (128, 128, 127),
              (128, 136, 129), (128, 136, 127), (136, 128, 136), (128, 240, 136), (128, 241, 136)]
    levels = [5, 5, 3, 5, 4, 5, 5, 5, 5, 5]
    keys = np.array([O.encode(x, y, z, l, 8) for (x, y, z), l in zip(blocks, levels)], np.uint64)
    orc = O.oracle()
    a, b = orc.volume(256, 2.56), ref.volume(256, 2.56)
    a.alloc_update(keys)
    b.alloc_update(keys)
    assert np.array_equal(a.blocks(False)[0], b.blocks(False)[0])
    na, nb = a.nodes(False), b.nodes(False)
    assert np.array_equal(na[0], nb[0]) and np.array_equal(na[2], nb[2])


def test_interp_and_grad_match_reference():
    s = make_scene("room", 96, 72, n_frames=1, seed=4, bg_size=128)
    orc = O.oracle()
    a, b = orc.volume(128, 5.12), ref.volume(128, 5.12)
    d, rgb, lab = s.render(0)
    m = generalize_masks(lab, [0])[0]
    rgb3 = rgb.astype(np.float32) / np.float32(255)
    for v in (a, b):
        v.integrate(d, rgb3, m, s.cam_poses[0], np.eye(4), s.k, 0.1)
    rng = np.random.default_rng(1)
    for p in rng.uniform(0.5, 4.6, size=(400, 3)).astype(np.float32):
        for field in range(5):  # tsdf, fg, r, g, b
            assert a.interp(p, field) == b.interp(p, field), field
        assert np.array_equal(a.grad(p), b.grad(p))


@pytest.mark.parametrize("mu", [0.02, 0.05, 0.2])
def test_oracle_matches_reference_other_truncation(mu):
    """Integration (every block and node field) and the composite raycast with
    truncation distances other than the default 0.1: oracle == reference."""
    W, H = 128, 96
    s = make_scene("multi", W, H, n_frames=3, seed=3, bg_size=128, obj_size=64, n_objects=2)
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vo = [orc.volume(i.size, i.dim) for i in s.instances]
    vr = [ref.volume(i.size, i.dim) for i in s.instances]
    for f in range(3):
        d, rgb, lab = s.render(f)
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i in range(len(labels)):
            assert (vo[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, mu) ==
                    vr[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, mu))
            ko, _, ao, xo = vo[i].blocks()
            kr, _, ar, xr = vr[i].blocks()
            assert np.array_equal(ko, kr) and np.array_equal(ao, ar)
            assert xo.tobytes() == xr.tobytes()
            assert vo[i].nodes()[3].tobytes() == vr[i].nodes()[3].tobytes()
        bo = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
        br = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
        orc.raycast_objects(vo, poses, labels, T, s.k, W, H, eps_size=EPS_SIZE, mu=mu,
                            vertex=bo[0], normal=bo[1], label_img=bo[2])
        ref.raycast_objects(vr, poses, labels, T, s.k, W, H, mu=mu, vertex=br[0], normal=br[1],
                            label_img=br[2])
        oob = orc.raycast_oob_mask(vo, poses, T, s.k, W, H, eps_size=EPS_SIZE)
        bad = np.any(bo[0] != br[0], axis=-1) | np.any(bo[1] != br[1], axis=-1) | (bo[2] != br[2])
        assert not np.any(bad & ~oob), np.argwhere(bad & ~oob)[:10]


@pytest.mark.parametrize("near,far", [(0.4, 4.0), (0.1, 1.2), (0.5, 1.5), (1.0, 8.0)])
def test_raycast_other_near_far_match_reference(near, far):
    """The composite raycast with near / far planes other than 0.1 / 4.0 (the
    ray iterator's range and the march's bound): oracle == reference."""
    W, H = 128, 96
    s = make_scene("multi", W, H, n_frames=1, seed=8, bg_size=128, obj_size=64, n_objects=2)
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vo = [orc.volume(i.size, i.dim) for i in s.instances]
    vr = [ref.volume(i.size, i.dim) for i in s.instances]
    d, rgb, lab = s.render(0)
    masks = generalize_masks(lab, labels)
    poses = s.volume_poses(0)
    T = s.cam_poses[0].astype(np.float32)
    rgb3 = rgb.astype(np.float32) / np.float32(255.0)
    for i in range(len(labels)):
        vo[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
        vr[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
    bo = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
    br = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
    orc.raycast_objects(vo, poses, labels, T, s.k, W, H, near=near, far=far, eps_size=EPS_SIZE,
                        vertex=bo[0], normal=bo[1], label_img=bo[2])
    ref.raycast_objects(vr, poses, labels, T, s.k, W, H, near=near, far=far, vertex=br[0],
                        normal=br[1], label_img=br[2])
    oob = orc.raycast_oob_mask(vo, poses, T, s.k, W, H, near=near, far=far, eps_size=EPS_SIZE)
    bad = np.any(bo[0] != br[0], axis=-1) | np.any(bo[1] != br[1], axis=-1) | (bo[2] != br[2])
    assert not np.any(bad & ~oob), np.argwhere(bad & ~oob)[:10]
    assert (bo[2] >= 0).sum() > 500


def test_integration_with_nan_negative_and_infinite_depths_matches_reference():
    """Allocation and integration from depth frames with NaN, negative and
    infinite values: every block, voxel and node value equal the reference's."""
    W, H = 128, 96
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=128, obj_size=64, n_objects=2)
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vo = [orc.volume(i.size, i.dim) for i in s.instances]
    vr = [ref.volume(i.size, i.dim) for i in s.instances]
    rng = np.random.default_rng(2)
    for f in range(2):
        d, rgb, lab = s.render(f)
        d = d.copy()
        d[rng.random(d.shape) < 0.01] = np.nan
        d[rng.random(d.shape) < 0.005] = -0.5
        d[rng.random(d.shape) < 0.002] = np.inf
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i in range(len(labels)):
            assert (vo[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1) ==
                    vr[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1))
            ko, _, ao, xo = vo[i].blocks()
            kr, _, ar, xr = vr[i].blocks()
            assert np.array_equal(ko, kr) and np.array_equal(ao, ar) and len(ko) > 0
            assert xo.tobytes() == xr.tobytes()
            assert vo[i].nodes()[3].tobytes() == vr[i].nodes()[3].tobytes()


@pytest.mark.parametrize("W,H", [(128, 96), (129, 97)])
def test_volume_path_negative_fy_matches_reference(W, H):
    """Allocation, integration and the composite raycast with a negative fy
    (the ICL-NUIM convention) on flipped frames, at an even and an odd frame
    size: oracle == reference."""
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=128, obj_size=64, n_objects=2)
    k = np.asarray(s.k, np.float32)
    kneg = np.array([k[0], -k[1], k[2], H - 1 - k[3]], np.float32)

    def flip(a):
        return np.ascontiguousarray(a[::-1])

    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vo = [orc.volume(i.size, i.dim) for i in s.instances]
    vr = [ref.volume(i.size, i.dim) for i in s.instances]
    for f in range(2):
        d, rgb, lab = (flip(a) for a in s.render(f))
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i in range(len(labels)):
            assert (vo[i].integrate(d, rgb3, masks[i], T, poses[i], kneg, 0.1) ==
                    vr[i].integrate(d, rgb3, masks[i], T, poses[i], kneg, 0.1))
            ko, _, _, xo = vo[i].blocks()
            kr, _, _, xr = vr[i].blocks()
            assert np.array_equal(ko, kr) and xo.tobytes() == xr.tobytes()
            assert vo[i].nodes()[3].tobytes() == vr[i].nodes()[3].tobytes()
        bo = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
        br = [np.zeros((H, W, 3), np.float32) for _ in range(2)] + [np.zeros((H, W), np.int32)]
        orc.raycast_objects(vo, poses, labels, T, kneg, W, H, eps_size=EPS_SIZE, vertex=bo[0],
                            normal=bo[1], label_img=bo[2])
        ref.raycast_objects(vr, poses, labels, T, kneg, W, H, vertex=br[0], normal=br[1],
                            label_img=br[2])
        oob = orc.raycast_oob_mask(vo, poses, T, kneg, W, H, eps_size=EPS_SIZE)
        bad = np.any(bo[0] != br[0], axis=-1) | np.any(bo[1] != br[1], axis=-1) | (bo[2] != br[2])
        assert not np.any(bad & ~oob) and (bo[2] >= 0).sum() > 5000

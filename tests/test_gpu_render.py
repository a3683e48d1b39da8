"""Headless renders (rendering.cpp's visualisation kernels) against the
oracle's restatement, byte for byte: the shaded volume render with its own
composite raycast (label colours and voxel colours, at the camera pose and at
a shifted view pose) and shading the last raycast's maps; depth, intensity and
normal renders; the three track renders on GN and motion result rows; the
three label renders."""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240
NEAR, FAR, MU = 0.1, 4.0, 0.1


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


@pytest.fixture(scope="module")
def env():
    import torch  # noqa: F401  (CUDA context for the device buffers)
    s = make_scene("multi", W, H, n_frames=2, seed=5, bg_size=256, obj_size=128, n_objects=3)
    labels = [i.label for i in s.instances]
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, robust="huber", near=NEAR, far=FAR)
    orc = O.oracle()
    vols, poses = [], s.volume_poses(0)
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
    colors = np.random.default_rng(3).integers(0, 256, size=(91, 4)).astype(np.uint8)
    colors[:, 3] = 0
    eps = float(np.float32(2.0 ** -np.log2(s.instances[0].size)))
    yield dict(s=s, ctx=ctx, vols=vols, poses=poses, labels=labels, T0=T0, d=d, rgb3=rgb3,
               cur_rgb3=rgb3, colors=colors, eps=eps, R=O.Render(W, H))
    ctx.close()


@pytest.mark.parametrize("color", [True, False])
@pytest.mark.parametrize("view", ["camera", "shifted"])
def test_volume_render_with_raycast(env, color, view):
    e = env
    T = e["T0"].copy()
    if view == "shifted":  # the reference's commented view offset (kfusion.cpp:1296-1300)
        T[:3, 3] -= 0.1
    largestep = 0.75 * MU
    got = e["ctx"].render_volume(T, render_color=color, largestep=largestep, colors=e["colors"])
    want = e["R"].volume(e["vols"], e["poses"], e["labels"], T, e["s"].k, NEAR, 2 * FAR, MU,
                         largestep, e["eps"], color, e["colors"])
    assert np.array_equal(got, want), np.count_nonzero((got != want).any(-1))
    assert np.count_nonzero(got[..., :3].any(-1)) > W * H // 2  # most pixels hit something
    assert e["ctx"].status() == 0


@pytest.mark.parametrize("color", [True, False])
def test_volume_render_of_last_raycast(env, color):
    e = env
    maps = e["ctx"].download_raycast()
    got = e["ctx"].render_volume(None, render_color=color, colors=e["colors"])
    want = e["R"].volume(e["vols"], e["poses"], e["labels"], None, e["s"].k, NEAR, 2 * FAR, MU,
                         0.075, e["eps"], color, e["colors"], maps=maps, T_shade=e["T0"])
    assert np.array_equal(got, want), np.count_nonzero((got != want).any(-1))


def test_depth_intensity_normal_renders(env):
    e = env
    ctx, R = e["ctx"], e["R"]
    assert np.array_equal(ctx.render_image("depth"), R.depth(e["d"], NEAR, FAR))
    r, g, b = (e["rgb3"][..., i] * np.float32(255.0) for i in range(3))
    grey = (np.float32(0.299) * r + np.float32(0.587) * g + np.float32(0.114) * b) / np.float32(
        255.0)
    assert np.array_equal(ctx.render_image("intensity"), R.intensity(grey))
    _, n, _ = ctx.download_raycast()
    assert np.array_equal(ctx.render_image("normal"), R.normal(n))


def test_track_renders(env):
    import torch
    e = env
    ctx, R = e["ctx"], e["R"]
    s = e["s"]
    # a second frame, the camera tracked, motion residuals: two sets of rows
    ctx.set_ref_from_current()
    d1, rgb1, lab1 = s.render(1)
    ctx.upload(d1, rgb1, generalize_masks(lab1, e["labels"]))
    ctx.preprocess()
    ctx.track_camera()
    res = torch.zeros(2 * W * H, dtype=torch.int8, device="cuda")
    err = torch.zeros(2 * W * H, dtype=torch.float32, device="cuda")
    ctx.track_results(0, res.data_ptr(), err.data_ptr())
    rh, eh = res.cpu().numpy(), err.cpu().numpy()
    assert (rh == 1).sum() > 10000 and np.abs(eh).max() > 0
    for mode in range(3):
        got = ctx.render_track(mode, res.data_ptr(), err.data_ptr())
        assert np.array_equal(got, R.track(rh, eh, mode)), mode
    ctx.motion_residuals(1.5, 0.9)
    mres, merr, _, _ = ctx.motion_download()
    for mode in range(3):
        assert np.array_equal(ctx.render_track(mode), R.track(mres, merr, mode)), mode
    # the context now holds frame 1; its rows feed the motion mask render
    e["cur_rgb3"] = rgb1.astype(np.float32) / np.float32(255.0)
    e["rows"] = res


def test_mask_renders(env):
    import torch
    e = env
    ctx, R = e["ctx"], e["R"]
    _, _, lab = ctx.download_raycast()
    assert (lab > 0).any()
    rgb3 = e["cur_rgb3"]
    for mode in (0, 1):
        got = ctx.render_mask(mode, e["colors"])
        assert np.array_equal(got, R.mask(lab, rgb3, mode, e["colors"])), mode
    # motion mode from a caller-given label image: the background and one
    # object with a row plane, the other labels without
    rows = e.get("rows")
    if rows is None:
        rows = torch.randint(-6, 2, (2 * W * H,), dtype=torch.int8, device="cuda")
    rows_host = rows.cpu().numpy()
    lab_dev = torch.from_numpy(lab.copy()).cuda()
    l1 = e["labels"][1]
    ptrs = [rows.data_ptr()] + [rows.data_ptr() if l == l1 else 0 for l in range(1, l1 + 1)]
    host_rows = [rows_host] + [rows_host if l == l1 else None for l in range(1, l1 + 1)]
    got = ctx.render_mask(2, e["colors"], d_labels=lab_dev.data_ptr(), d_rows=ptrs)
    assert np.array_equal(got, R.mask(lab, rgb3, 2, e["colors"], host_rows))

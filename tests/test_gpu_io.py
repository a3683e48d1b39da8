"""Kfusion::preprocessing's input stage on the device (mf_frame_upload_raw:
mm2metersKernel and rgb2intensity with an integer subsampling ratio) and the
TUM pose files (mf_save_poses), against numpy restatements."""
import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context, MfError, pose_quaternion

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


@pytest.mark.parametrize("ratio", [1, 2])
def test_raw_frame_upload(ratio):
    W, H = 160, 120
    rng = np.random.default_rng(ratio)
    d_mm = rng.integers(0, 8000, (H * ratio, W * ratio), dtype=np.uint16)
    rgb = rng.integers(0, 256, (H * ratio, W * ratio, 3), dtype=np.uint8)
    ctx = Context(W, H, pool_blocks=1 << 10)
    ctx.add_instance(64, 1.0, np.eye(4), 0)
    ctx.upload_raw(d_mm, rgb)
    sub_d = d_mm[::ratio, ::ratio].astype(np.float32)
    sub_c = rgb[::ratio, ::ratio].astype(np.float32)
    want_d = sub_d / np.float32(1000.0)
    r, g, b = sub_c[..., 0], sub_c[..., 1], sub_c[..., 2]
    want_grey = (np.float32(0.299) * r + np.float32(0.587) * g + np.float32(0.114) * b) / \
        np.float32(255.0)
    # the grey frame through the intensity render is 255 * grey truncated; the
    # depth through the pyramid's level-0 raw depth
    got_int = ctx.render_image("intensity")[..., 0]
    assert np.array_equal(got_int, (np.float32(255.0) * want_grey).astype(np.int32).astype(np.uint8))
    dep = ctx.render_image("depth")
    from _oracle import Render
    assert np.array_equal(dep, Render(W, H).depth(want_d, 0.1, 4.0))
    with pytest.raises(MfError):
        ctx.upload_raw(d_mm[:, :-1], None)   # not an integer ratio
    ctx.close()


def test_save_poses_files(tmp_path):
    ctx = Context(64, 48, pool_blocks=1 << 10)
    Tc = np.eye(4, dtype=np.float32)
    Tc[:3, 3] = [0.1, 0.2, 0.3]
    To = np.eye(4, dtype=np.float32)
    To[:3, :3] = [[0, -1, 0], [1, 0, 0], [0, 0, 1]]
    To[:3, 3] = [5, 6, 7]
    ctx.add_instance(64, 1.0, np.eye(4), 0)
    ctx.add_instance(64, 0.5, To, 3)
    ctx.set_camera_pose(Tc)
    prefix = tmp_path / "poses"
    ctx.save_poses(prefix, 1)
    ctx.save_poses(prefix, 2)
    cam = (tmp_path / "poses_camera").read_text().splitlines()
    obj = (tmp_path / "poses_3").read_text().splitlines()
    assert len(cam) == 2 and len(obj) == 2
    assert cam[0] == "1\t0.1\t0.2\t0.3\t0\t0\t0\t1\t"
    q = pose_quaternion(To)
    # the camera's translation with the object's rotation (kfusion.cpp:1615-1617)
    assert obj[1] == "2\t0.1\t0.2\t0.3\t%g\t%g\t%g\t%g\t" % tuple(float(v) for v in q)
    ctx.save_poses(prefix, 3)      # appends
    assert len((tmp_path / "poses_camera").read_text().splitlines()) == 3
    ctx.close()

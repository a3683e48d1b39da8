"""The bench's workloads on CPU: each scene the bench times has the shape its
JSON line names (frame size, intrinsics, instances and their octrees), and
the launch-shape options parse.  No device is touched."""
import subprocess
import sys
import os

import numpy as np

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_main_workload_is_the_3_object_scene():
    s = bench.scene_for(0, 2, "multi")
    assert (s.width, s.height) == (640, 480)
    assert np.allclose(s.k, (525.0, 525.0, 319.5, 239.5))
    sizes = [(i.size, round(i.dim, 3)) for i in s.instances]
    assert sizes == [(512, 5.12), (256, 0.512), (256, 0.512), (256, 0.512)]


def test_room_workload_is_the_single_octree_320x240_scene():
    s = bench.scene_for(0, bench.ROOM_FRAMES, "room")
    assert (s.width, s.height) == (320, 240)
    assert np.allclose(s.k, (262.5, 262.5, 159.5, 119.5))
    assert len(s.instances) == 1
    assert (s.instances[0].size, round(s.instances[0].dim, 3)) == (256, 2.56)
    assert np.allclose(s.volume_poses(0)[0], np.eye(4))
    assert bench.ROOM_FRAMES == 30 and "30 frames" in bench.ROOM
    d, rgb, lab = s.render(0)
    assert d.shape == (240, 320) and rgb.shape == (240, 320, 3)
    assert 0.9 < float((d > 0).mean()) <= 1.0  # 1 % dropouts


def test_uneven_workload_has_12_objects():
    s = bench.scene_for(0, 2, "uneven")
    assert (s.width, s.height) == (640, 480)
    assert len(s.instances) == 13
    assert {i.size for i in s.instances[1:]} <= {32, 64, 128, 256}


def test_uneven_sequence_keeps_its_objects_in_view():
    """The 200-frame uneven sequence: objects swing along their twists and the
    camera loops, so most objects stay in view to the end."""
    assert bench.UNEVEN_FRAMES == 200 and "200 frames" in bench.UNEVEN
    s = bench.scene_for(0, bench.UNEVEN_FRAMES, "uneven")
    for f in (0, 100, 199):
        _, _, lab = s.render(f)
        areas = [float((lab == i.label).mean()) for i in s.instances[1:]]
        assert sum(a > 0.001 for a in areas) >= 9, (f, areas)
        assert max(areas) > 0.15


def test_launch_shape_options_parse():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"],
                         capture_output=True, text=True, cwd=ROOT, timeout=120)
    assert out.returncode == 0
    assert "--shapes" in out.stdout and "--no-tune" in out.stdout

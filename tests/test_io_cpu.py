"""The formats around the hot path that run on the host: the SLAMBench .raw
reader (RawDepthReader, interface.h:207-335), the pose quaternion
(getQuaternion, preprocessing.cpp:312-320) and the TUM pose line
(Kfusion::save_poses, kfusion.cpp:1591-1626).  The library is loaded but no
device is used."""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from mid_fusion_b200 import build
from mid_fusion_b200.capi import RawReader, pose_quaternion, tum_line


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _write_raw(path, frames):
    with open(path, "wb") as f:
        for d, c in frames:
            h, w = d.shape
            f.write(np.array([w, h], np.uint32).tobytes())
            f.write(np.ascontiguousarray(d, np.uint16).tobytes())
            f.write(np.array([w, h], np.uint32).tobytes())
            f.write(np.ascontiguousarray(c, np.uint8).tobytes())


def test_raw_reader_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    frames = [(rng.integers(0, 65535, (6, 8), dtype=np.uint16),
               rng.integers(0, 255, (6, 8, 3), dtype=np.uint8)) for _ in range(3)]
    p = tmp_path / "seq.raw"
    _write_raw(p, frames)
    r = RawReader(p)
    assert (r.width, r.height, r.n_frames) == (8, 6, 3)
    for d, c in frames:                       # sequential reads
        gd, gc = r.read()
        assert np.array_equal(gd, d) and np.array_equal(gc, c)
    assert r.read() is None                   # end of the sequence
    gd, gc = r.read(1)                        # random access
    assert np.array_equal(gd, frames[1][0]) and np.array_equal(gc, frames[1][1])
    r.close()
    # a truncated last frame is not counted
    with open(p, "ab") as f:
        f.write(b"\x08\x00\x00\x00\x06\x00\x00\x00garbage")
    assert RawReader(p).n_frames == 3


def _quat_by_method(R):
    """The trace / largest-diagonal method in float32, restated in numpy."""
    m = np.asarray(R, np.float32)
    q = np.zeros(4, np.float32)
    t = np.float32(m[0, 0] + m[1, 1]) + m[2, 2]
    if t > 0:
        t = np.sqrt(t + np.float32(1))
        q[3] = np.float32(0.5) * t
        t = np.float32(0.5) / t
        q[0] = (m[2, 1] - m[1, 2]) * t
        q[1] = (m[0, 2] - m[2, 0]) * t
        q[2] = (m[1, 0] - m[0, 1]) * t
    else:
        i = 0
        if m[1, 1] > m[0, 0]:
            i = 1
        if m[2, 2] > m[i, i]:
            i = 2
        j, k = (i + 1) % 3, (i + 2) % 3
        t = np.sqrt(np.float32(m[i, i] - m[j, j]) - m[k, k] + np.float32(1))
        q[i] = np.float32(0.5) * t
        t = np.float32(0.5) / t
        q[3] = (m[k, j] - m[j, k]) * t
        q[j] = (m[j, i] + m[i, j]) * t
        q[k] = (m[k, i] + m[i, k]) * t
    return q


def test_pose_quaternion_both_branches():
    rng = np.random.default_rng(1)
    rots = list(Rotation.random(40, random_state=3).as_matrix())
    rots += [np.diag([1.0, -1.0, -1.0]), np.diag([-1.0, 1.0, -1.0]), np.diag([-1.0, -1.0, 1.0])]
    for R in rots:
        T = np.eye(4, dtype=np.float32)
        T[:3, :3] = R
        T[:3, 3] = rng.normal(size=3)
        q = pose_quaternion(T)
        assert np.array_equal(q, _quat_by_method(T[:3, :3]))
        ref = Rotation.from_matrix(R.astype(np.float64)).as_quat()   # (x, y, z, w)
        assert min(np.abs(q - ref).max(), np.abs(q + ref).max()) < 2e-6


def test_tum_line_format():
    T = np.eye(4, dtype=np.float32)
    T[:3, 3] = [0.5, -1.25, 3.0]
    R = np.eye(4, dtype=np.float32)
    R[:3, :3] = Rotation.from_euler("z", 90, degrees=True).as_matrix()
    line = tum_line(7, T, R)
    q = pose_quaternion(R)
    assert line == "7\t0.5\t-1.25\t3\t%g\t%g\t%g\t%g\t\n" % tuple(float(v) for v in q)
    assert line.split("\t")[6] == "0.707107"


def test_vtk_mesh_writer(tmp_path):
    from mid_fusion_b200.capi import write_vtk_mesh
    tris = np.array([[[0, 0, 0], [1, 0, 0], [0, 1.5, 0]],
                     [[0.25, 1e-7, 2], [3, 4, 5], [6, 7, 123456789]]], np.float32)
    p = tmp_path / "m.vtk"
    write_vtk_mesh(p, tris)
    want = ("# vtk DataFile Version 1.0\nvtk mesh generated from KFusion\nASCII\n"
            "DATASET POLYDATA\nPOINTS 6 FLOAT\n"
            "0 0 0\n1 0 0\n0 1.5 0\n0.25 1e-07 2\n3 4 5\n6 7 1.23457e+08\n"
            "POLYGONS 2 8\n3 0 1 2\n3 3 4 5\n\n")
    assert p.read_text() == want

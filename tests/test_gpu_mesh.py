"""Mesh export on the device (mf_mesh) against the oracle's marching cubes
(oracle/or_mesh.cpp, itself checked against the reference's
algorithms::marching_cube), triangle for triangle, on the background and an
object of a multi-object scene; mf_dump_mesh writes one VTK file per
instance."""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def test_mesh_matches_oracle(tmp_path):
    import torch
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=5, seed=5, bg_size=256, obj_size=128, n_objects=2)
    labels = [i.label for i in s.instances]
    ctx = Context(W, H, k=s.k, pool_blocks=1 << 15)
    orc = O.oracle()
    vols = []
    for inst, T in zip(s.instances, s.volume_poses(0)):
        ctx.add_instance(inst.size, inst.dim, T, inst.label)
        vols.append(orc.volume(inst.size, inst.dim))
    for f in range(5):
        d, rgb, lab = s.render(f)
        masks = generalize_masks(lab, labels)
        poses = s.volume_poses(f)
        T = s.cam_poses[f].astype(np.float32)
        for i, P in enumerate(poses):
            ctx.set_instance_pose(i, P)
        ctx.set_camera_pose(T)
        ctx.upload(d, rgb, masks)
        ctx.integrate(list(range(len(labels))))
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
    for i, v in enumerate(vols):
        for fb in (False, True):
            got = ctx.mesh(i, float_bounds=fb)
            want = O.mesh(orc, v, float_bounds=fb)
            assert len(got) == len(want), (i, fb, len(got), len(want))
            assert np.array_equal(got, want), (i, fb)
            # the reference's int bound empties the 0.512 m object volumes
            assert len(got) > 200 if (i == 0 or fb) else len(got) == 0, (i, fb, len(got))
    # into device memory as well
    n = len(ctx.mesh(0))
    dev = torch.zeros((n, 3, 3), dtype=torch.float32, device="cuda")
    import ctypes as C
    cnt = C.c_longlong()
    assert ctx.lib.mf_mesh(ctx.h, 0, 0, C.c_void_p(dev.data_ptr()), n, C.byref(cnt)) == 0
    assert cnt.value == n and np.array_equal(dev.cpu().numpy(), ctx.mesh(0))
    ctx.dump_mesh(tmp_path / "mesh")
    for l in labels:
        text = (tmp_path / f"mesh_{l}.vtk").read_text().splitlines()
        assert text[0] == "# vtk DataFile Version 1.0" and text[4].startswith("POINTS ")
    assert ctx.status() == 0
    ctx.close()


def test_mesh_with_the_reference_table_is_the_reference_mesh():
    """mf_mesh_set_triangle_table with the reference's own triTable (read from
    its compiled mesher, oracle/_ref): the device's triangles equal the
    oracle's with the same table triangle for triangle, and the reference's
    algorithms::marching_cube as a set (its order follows its block list)."""
    import ctypes as C
    ref = O.reference()
    if ref is None:
        pytest.skip("oracle/_ref not built")
    t = np.zeros((256, 16), np.int32)
    ref.lib.ref_tri_table.argtypes = [C.c_void_p]
    ref.lib.ref_tri_table(t.ctypes.data_as(C.c_void_p))
    s = make_scene("room", 160, 120, n_frames=4, seed=4, bg_size=128)
    inst = s.instances[0]
    ctx = Context(160, 120, k=s.k, pool_blocks=1 << 13)
    ctx.add_instance(inst.size, inst.dim, np.eye(4), inst.label)
    orc = O.oracle()
    a, b = orc.volume(inst.size, inst.dim), ref.volume(inst.size, inst.dim)
    for f in range(4):
        d, rgb, lab = s.render(f)
        m = generalize_masks(lab, [inst.label])
        T = s.cam_poses[f].astype(np.float32)
        ctx.set_camera_pose(T)
        ctx.upload(d, rgb, m)
        ctx.integrate([0])
        rgb3 = rgb.astype(np.float32) / np.float32(255)
        for v in (a, b):
            v.integrate(d, rgb3, m[0], T, np.eye(4), s.k, 0.1)
    ctx.set_triangle_table(t)
    got = ctx.mesh(0)
    lib = orc.lib
    lib.or_mesh_set_table.argtypes = [C.c_void_p]
    lib.or_mesh_set_table(t.ctypes.data_as(C.c_void_p))
    try:
        want = O.mesh(orc, a)
    finally:
        lib.or_mesh_set_table(None)
    assert len(got) == len(want) > 1000 and np.array_equal(got, want)
    mb = O.mesh(ref, b)

    def canon(x):
        flat = x.reshape(len(x), 9)
        return flat[np.lexsort(flat.T[::-1])]
    assert np.array_equal(canon(got), canon(mb))
    # NULL restores the built-in table; a malformed row is rejected
    ctx.set_triangle_table(None)
    assert np.array_equal(ctx.mesh(0), O.mesh(orc, a))
    bad = t.copy()
    bad[7, :] = 3
    with pytest.raises(Exception):
        ctx.set_triangle_table(bad)
    assert ctx.status() == 0
    ctx.close()

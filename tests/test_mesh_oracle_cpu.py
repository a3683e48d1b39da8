"""Marching cubes: the oracle's mesher (oracle/or_mesh.cpp) against the
reference's own algorithms::marching_cube (lib/algorithms/meshing.hpp,
compiled into oracle/_ref), and the generated triangulation tables
(mid_fusion_b200/csrc/gen_mc_tables.py) on their own.

The cell test (compute_index) and the twelve edge intersections
(interp_vertexes) are compared bit for bit on every cell of the volume.  The
triangulation tables are this project's, derived from the cube's geometry:
for each of the 256 corner patterns they cut the same polygons as the
reference's table (same triangle count per pattern, same edges), but a
polygon of four or more vertices may be split along another diagonal.  So the
meshes are compared as surfaces: the same number of triangles, the same set of
vertices, and areas and enclosed volumes within 1e-3 relative."""
import os
import sys

import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200.scene import generalize_masks, make_scene

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "mid_fusion_b200", "csrc"))
import gen_mc_tables as G  # noqa: E402

ref = O.reference()


def _volumes():
    s = make_scene("room", 160, 120, n_frames=6, seed=4, bg_size=128)
    inst = s.instances[0]
    orc = O.oracle()
    a = orc.volume(inst.size, inst.dim)
    b = ref.volume(inst.size, inst.dim) if ref is not None else None
    for f in range(6):
        d, rgb, lab = s.render(f)
        m = generalize_masks(lab, [0])[0]
        rgb3 = rgb.astype(np.float32) / np.float32(255)
        for v in (a, b):
            if v is not None:
                v.integrate(d, rgb3, m, s.cam_poses[f], s.volume_poses(f)[0], s.k, 0.1)
    return inst, a, b


def _area_volume(tris):
    t = tris.astype(np.float64)
    cr = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    area = 0.5 * np.linalg.norm(cr, axis=1).sum()
    vol = np.einsum("ij,ij->i", t[:, 0], np.cross(t[:, 1], t[:, 2])).sum() / 6.0
    return area, vol


def test_tables_are_closed_and_oriented():
    G.check_orientation()
    for seed in range(3):
        G.check_closed(n_cells=5, seed=seed)
    assert max(len(G.triangulate(p)) for p in range(256)) == G.MAX_TRIS


@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (no reference tree)")
def test_cells_and_mesh_match_reference():
    inst, a, b = _volumes()
    keys, coords, _, _ = a.blocks(False)
    n_surface = 0
    for cx, cy, cz in coords:
        for i in range(0, 512, 3):
            x, y, z = int(cx + (i >> 6)), int(cy + ((i >> 3) & 7)), int(cz + (i & 7))
            if max(x, y, z) >= inst.size - 1:
                continue
            ia, va = O.mc_cell(O.oracle(), a, x, y, z)
            ib, vb = O.mc_cell(ref, b, x, y, z)
            assert ia == ib, (x, y, z)
            if ia not in (-1, 0, 255):
                n_surface += 1
                assert np.array_equal(va, vb, equal_nan=True), (x, y, z)
    assert n_surface > 500
    ma, mb = O.mesh(O.oracle(), a), O.mesh(ref, b)
    assert len(ma) == len(mb) > 5000
    va = np.unique(ma.reshape(-1, 3), axis=0)
    vb = np.unique(mb.reshape(-1, 3), axis=0)
    assert np.array_equal(va, vb)
    (aa, xa), (ab, xb) = _area_volume(ma), _area_volume(mb)
    assert abs(aa - ab) <= 1e-3 * ab, (aa, ab)
    assert abs(xa - xb) <= 1e-3 * abs(xb), (xa, xb)


def ref_triangle_table():
    """The reference's own triTable (lib/algorithms/edge_tables.h), read from
    the reference's compiled mesher (oracle/_ref/libmf_ref.so)."""
    import ctypes as C
    t = np.zeros((256, 16), np.int32)
    ref.lib.ref_tri_table.argtypes = [C.c_void_p]
    ref.lib.ref_tri_table(t.ctypes.data_as(C.c_void_p))
    return t


def sorted_triangles(tris):
    """Triangles (n, 3, 3) in a canonical order (the reference's order depends
    on its block list and OpenMP): rows sorted lexicographically."""
    flat = tris.reshape(len(tris), 9)
    return flat[np.lexsort(flat.T[::-1])]


@pytest.mark.skipif(ref is None, reason="oracle/_ref not built (no reference tree)")
def test_mesh_with_the_reference_table_matches_reference_triangle_for_triangle():
    """With the reference's own triangulation table the oracle's mesher emits
    the reference's triangles: the same triangle (same vertices, same vertex
    order) for every triangle, bit for bit."""
    import ctypes as C
    inst, a, b = _volumes()
    lib = O.oracle().lib
    lib.or_mesh_set_table.argtypes = [C.c_void_p]
    t = ref_triangle_table()
    assert (t[:, 15] == -1).all() and (t >= -1).all() and (t <= 11).all()
    lib.or_mesh_set_table(t.ctypes.data_as(C.c_void_p))
    try:
        ma, mb = O.mesh(O.oracle(), a), O.mesh(ref, b)
    finally:
        lib.or_mesh_set_table(None)
    assert len(ma) == len(mb) > 5000
    assert np.array_equal(sorted_triangles(ma), sorted_triangles(mb))

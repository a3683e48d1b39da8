"""Generates mf_mc_tables.h: the marching-cubes triangulation of every one of
the 256 inside/outside corner patterns, derived here from the cube's geometry
(not taken from a published table).

Corner and edge numbering follow the reference's mesher
(lib/algorithms/meshing.hpp: interp_vertexes :31-62, gather_points :64-74),
so the tables index its edges; each edge is interpolated from its first
corner to its second:

    corners 0 (0,0,0) 1 (1,0,0) 2 (1,0,1) 3 (0,0,1)
            4 (0,1,0) 5 (1,1,0) 6 (1,1,1) 7 (0,1,1)        (x, y, z) offsets
    edges   0: 0-1  1: 1-2  2: 2-3  3: 0-3   (the y = 0 face)
            4: 4-5  5: 5-6  6: 6-7  7: 4-7   (the y = 1 face)
            8: 0-4  9: 1-5 10: 2-6 11: 3-7   (along y)

Bit i of a pattern is set when corner i is inside (tsdf < 0).  Method:

1. On every cube face the cut edges (ends on different sides) are joined in
   pairs by segments.  A face with two cut edges has one segment; a face
   with four (inside corners diagonal) has two, each cutting off one inside
   corner, so inside corners are never joined across a face.  The rule
   depends only on the face's own corners, so two cells sharing a face make
   the same choice and the surface has no cracks.
2. Each segment is directed with the face's inside corners on its left as
   seen from outside the cube.  The segments then chain into closed loops:
   the oriented boundary of the inside region on the cube's surface.
3. Each loop is fanned into triangles, wound so that the right-handed normal
   points to the outside (increasing tsdf), from the first point whose
   diagonals all cross the cell's interior (none lies in a cube face, where
   the neighbouring cell could cut the same chord).

    python gen_mc_tables.py > mf_mc_tables.h
"""
import itertools

import numpy as np

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)]
EDGES = [(0, 1), (1, 2), (2, 3), (0, 3), (4, 5), (5, 6), (6, 7), (4, 7),
         (0, 4), (1, 5), (2, 6), (3, 7)]
FACES = [  # corner cycle, outward normal
    ((0, 1, 2, 3), (0, -1, 0)),
    ((4, 5, 6, 7), (0, 1, 0)),
    ((0, 3, 7, 4), (-1, 0, 0)),
    ((1, 2, 6, 5), (1, 0, 0)),
    ((0, 1, 5, 4), (0, 0, -1)),
    ((3, 2, 6, 7), (0, 0, 1)),
]
MAX_TRIS = 5
# the two faces each edge lies on
FACES_OF = [frozenset(f for f, (cyc, _) in enumerate(FACES)
                      if a in cyc and b in cyc) for a, b in EDGES]


def edge_of(a, b):
    for i, (p, q) in enumerate(EDGES):
        if {p, q} == {a, b}:
            return i
    raise KeyError((a, b))


def mid(e):
    a, b = EDGES[e]
    return (np.array(CORNERS[a], float) + np.array(CORNERS[b], float)) / 2


def triangulate(pattern):
    inside = [(pattern >> i) & 1 == 1 for i in range(8)]
    nxt = {}
    for cyc, normal in FACES:
        n = np.array(normal, float)
        segs = []  # (edge, edge, inside corner on the cut-off side)
        cut = [(cyc[i], cyc[(i + 1) % 4]) for i in range(4)
               if inside[cyc[i]] != inside[cyc[(i + 1) % 4]]]
        if len(cut) == 2:
            ins = [c for c in cyc if inside[c]]
            segs.append((edge_of(*cut[0]), edge_of(*cut[1]), ins[0]))
        elif len(cut) == 4:
            for k in range(4):
                c = cyc[k]
                if inside[c]:
                    prev, succ = cyc[(k - 1) % 4], cyc[(k + 1) % 4]
                    segs.append((edge_of(prev, c), edge_of(c, succ), c))
        for e1, e2, c in segs:
            p, q = mid(e1), mid(e2)
            side = np.dot(np.cross(q - p, n), np.array(CORNERS[c], float) - p)
            if side < 0:
                e1, e2 = e2, e1
            assert e1 not in nxt, (pattern, e1)
            nxt[e1] = e2
    loops, seen = [], set()
    for start in sorted(nxt):
        if start in seen:
            continue
        loop, e = [], start
        while e not in seen:
            seen.add(e)
            loop.append(e)
            e = nxt[e]
        assert e == start, (pattern, loop)
        loops.append(loop)
    tris = []
    for loop in loops:
        # fan from the first point whose diagonals all cross the cell's
        # interior: a diagonal between two points of one face would lie in
        # that face, and the cell on its other side may cut the same chord
        k = len(loop)
        for r in range(k):
            fan = loop[r:] + loop[:r]
            if all(not (FACES_OF[fan[0]] & FACES_OF[fan[i]]) for i in range(2, k - 1)):
                break
        else:
            raise AssertionError((pattern, loop))
        for i in range(1, k - 1):
            tris.append((fan[0], fan[i], fan[i + 1]))
    return tris


def check_orientation():
    """Pattern 1 (corner 0 inside): the normal points away from corner 0."""
    (a, b, c), = triangulate(1)
    nrm = np.cross(mid(b) - mid(a), mid(c) - mid(a))
    assert np.dot(nrm, np.array([1.0, 1.0, 1.0])) > 0, nrm


def check_closed(n_cells=6, seed=0):
    """On a random field the triangles of all cells form a closed surface
    away from the grid boundary: every interior mesh edge is shared by
    exactly two triangles, with opposite directions."""
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(n_cells + 1,) * 3)
    use = {}
    for x, y, z in itertools.product(range(n_cells), repeat=3):
        pat = 0
        for i, (dx, dy, dz) in enumerate(CORNERS):
            if f[x + dx, y + dy, z + dz] < 0:
                pat |= 1 << i
        for tri in triangulate(pat):
            keys = []
            for e in tri:
                a, b = EDGES[e]
                pa = (x + CORNERS[a][0], y + CORNERS[a][1], z + CORNERS[a][2])
                pb = (x + CORNERS[b][0], y + CORNERS[b][1], z + CORNERS[b][2])
                keys.append(tuple(sorted([pa, pb])))
            for i in range(3):
                k = (keys[i], keys[(i + 1) % 3])
                use[k] = use.get(k, 0) + 1
    for (u, v), cnt in use.items():
        on_boundary = any(c in (0, n_cells) for p in (u, v) for pt in p for c in pt)
        if on_boundary:
            continue
        assert cnt == 1 and use.get((v, u), 0) == 1, (u, v, cnt)


def main():
    check_orientation()
    check_closed()
    rows, counts = [], []
    for pat in range(256):
        tris = triangulate(pat)
        assert len(tris) <= MAX_TRIS, (pat, len(tris))
        flat = [e for t in tris for e in t]
        counts.append(len(tris))
        rows.append(flat + [-1] * (3 * MAX_TRIS - len(flat)))
    print("// Generated by gen_mc_tables.py (see there for the method); do not edit.")
    print("#pragma once")
    print("#include <cstdint>")
    print(f"#define MF_MC_MAX_TRIS {MAX_TRIS}")
    print("// triangles of each corner pattern as edge triples, -1 padded")
    print(f"static const int8_t MF_MC_TRIS[256][{3 * MAX_TRIS}] = {{")
    for pat, r in enumerate(rows):
        print("  {" + ", ".join(str(v) for v in r) + "},")
    print("};")
    print("static const uint8_t MF_MC_COUNT[256] = {")
    for i in range(0, 256, 16):
        print("  " + ", ".join(str(c) for c in counts[i:i + 16]) + ",")
    print("};")


if __name__ == "__main__":
    main()

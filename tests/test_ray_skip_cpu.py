"""The raycast skips an instance's octree traversal for rays that cannot meet
its box of allocated blocks (ray_misses_blocks in mid_fusion_b200/csrc/
mf_raycast.cu).  The GPU parity tests show the maps stay bit-exact on the test
scenes; this checks the skip rule itself on many more rays, including grazing
and axis-aligned ones whose direction the traversal clamps: the rule is
restated here in float32 and compared with the oracle's ray_first_block (the
reference's ESVO traversal, lib/octree.hpp:919-1130).  Whenever the rule skips
a ray, the traversal finds no block, or one whose entry lies at or beyond
far, where the march returns a miss as well."""
import ctypes as C

import numpy as np
import pytest

import _oracle as O

F = np.float32


def ray_misses_blocks(size, dim, box, origin, direction, near, far, eps):
    d = direction.astype(F).copy()
    for a in range(3):
        if abs(d[a]) < eps:
            d[a] = np.copysign(F(eps), d[a])
    vn = F(1) / F(size)
    mg = F(2) * vn
    o = origin.astype(F) / F(dim)
    inv = F(1) / d
    t0 = F(near) / F(dim) - mg
    t1 = F(far) / F(dim) + mg

    def hits(lo, hi):
        a = (lo - o) * inv
        b = (hi - o) * inv
        te = max(F(np.max(np.minimum(a, b))), t0)
        tx = min(F(np.min(np.maximum(a, b))), t1)
        return te <= tx

    if hits(np.full(3, -mg, F), np.full(3, F(8) * vn + mg, F)):
        return False
    if box[0] > box[3]:
        return True
    lo = box[:3].astype(F) * vn - mg
    hi = (box[3:].astype(F) + F(8)) * vn + mg
    return not hits(lo, hi)


def _volume(size, dim, corners):
    orc = O.oracle()
    vol = orc.volume(size, dim)
    max_level = int(np.log2(size))
    keys = np.array([O.encode(x, y, z, max_level - 3, max_level) for x, y, z in corners],
                    np.uint64)
    vol.alloc_update(keys)
    _, coords, _, _ = vol.blocks(with_voxels=False)
    others = coords[np.any(coords != 0, axis=1)]
    box = (np.concatenate([others.min(0), others.max(0)]).astype(np.int32) if len(others)
           else np.array([1, 1, 1, 0, 0, 0], np.int32))
    return orc, vol, box


def _rays(rng, n, dim, size, eps, corners):
    """Random rays, half of them aimed at a point inside or on the edge of an
    allocated block, some with components the traversal clamps."""
    vs = dim / size
    origins = rng.uniform(-1.5 * dim, 2.5 * dim, (n, 3))
    dirs = rng.normal(size=(n, 3))
    aim = rng.random(n) < 0.5
    c = np.asarray(corners, np.float64)[rng.integers(0, len(corners), n)]
    # inside the block, or on one of its faces (grazing rays)
    frac = rng.uniform(0.0, 8.0, (n, 3))
    face = rng.random(n) < 0.3
    frac[face, rng.integers(0, 3, n)[face]] = rng.choice([0.0, 8.0], face.sum())
    target = (c + frac) * vs
    dirs[aim] = target[aim] - origins[aim]
    # grazing and axis-aligned directions: components the traversal clamps
    kind = rng.integers(0, 4, n)
    for i in np.nonzero(kind == 1)[0]:
        dirs[i, rng.integers(0, 3)] = rng.uniform(-0.5, 0.5) * eps
    for i in np.nonzero((kind == 2) & ~aim)[0]:
        a = rng.integers(0, 3)
        dirs[i] = 0.0
        dirs[i, a] = rng.choice([-1.0, 1.0])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    near = rng.uniform(0.0, 0.1, n).astype(F)
    far = rng.uniform(0.02, 4.0, n).astype(F)
    return origins.astype(F), dirs.astype(F), near, far


@pytest.mark.parametrize("size,dim,corners,seed", [
    # a 3x3x3 cluster of 8-voxel blocks in a 64^3 object volume at 2 mm
    (64, 0.128, [(x, y, z) for x in (24, 32, 40) for y in (24, 32, 40) for z in (16, 24, 32)], 1),
    # scattered blocks in a 256^3 room volume at 1 cm, block 0 among them
    (256, 2.56, [(0, 0, 0), (200, 8, 96), (64, 240, 8), (128, 128, 128), (16, 16, 232)], 2),
])
def test_skipped_rays_find_no_block_before_far(size, dim, corners, seed):
    orc, vol, box = _volume(size, dim, corners)
    first_block = orc.lib.or_ray_first_block
    eps = float(np.exp2(-np.log2(size)))
    rng = np.random.default_rng(seed)
    origins, dirs, near, far = _rays(rng, 20000, dim, size, eps, corners)
    skipped = hits_found = 0
    for o, d, nr, fr in zip(origins, dirs, near, far):
        t = first_block(vol.h, np.ascontiguousarray(o), np.ascontiguousarray(d), float(nr),
                        float(fr), eps)
        t_m = F(t) * F(dim) / F(size)
        if t > 0 and t_m < fr:
            hits_found += 1
        if ray_misses_blocks(size, dim, box, o, d, nr, fr, eps):
            skipped += 1
            assert not (t > 0 and t_m < fr), (o, d, nr, fr, t)
    # the rule is not vacuous: it skips many rays and the traversal finds many
    assert skipped > 4000 and hits_found > 200, (skipped, hits_found)

"""The CPU oracle against golden vectors of the reference (CPU only).

* tests/golden/volume_golden.npz: allocation, integration and multi-instance
  raycast outputs of the reference's own code (oracle/_ref, generated by
  tests/golden/make_golden.py), compared bit for bit.
* tests/golden/track_golden.npz: the reference's own tracking
  (tracking.cpp / preprocessing.cpp / object.cpp, generated by
  tests/golden/make_track_golden.py): pyramid digests, camera poses and
  per-level sums (plain and masked trackLiveFrame), object poses and sums
  (trackEachObject) and motion residual rows, which the single-precision
  tracking oracle reproduces bit for bit.
* Fixed cases of the reference's unit tests: unique_multiscale counts
  (lib/test/algorithms/unique_unittest.cpp:113-143), bilinear interpolation on
  a checkerboard (apps/kfusion/test/preprocessing/interp_unittest.cpp:24-51),
  Morton round trips (lib/test/utils/morton_unittest.cpp:38-67) and the key
  probe hash(8, 0, 0) = 0x205 of a 256^3 octree.
"""
import ctypes as C
import hashlib
import os

import numpy as np
import pytest

import _oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "volume_golden.npz")
TRACK_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "track_golden.npz")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def lib():
    lib = O.oracle().lib
    lib.or_unique_multiscale.restype = C.c_int
    lib.or_unique_multiscale.argtypes = [np.ctypeslib.ndpointer(np.uint64), C.c_int, C.c_uint64,
                                         C.c_int]
    lib.or_encode.restype = C.c_uint64
    lib.or_encode.argtypes = [C.c_int] * 5
    lib.or_morton.restype = C.c_uint64
    lib.or_morton.argtypes = [C.c_uint] * 3
    lib.or_unpack.argtypes = [C.c_uint64, np.ctypeslib.ndpointer(np.uint32)]
    lib.or_bilinear.restype = C.c_float
    lib.or_bilinear.argtypes = [np.ctypeslib.ndpointer(np.float32), C.c_int, C.c_float, C.c_float]
    return lib


def test_volume_golden_vectors():
    g = np.load(GOLDEN)
    orc = O.oracle()
    sizes, dims, labels = g["sizes"], g["dims"], list(g["labels"])
    H, W = g["depth0"].shape
    vols = [orc.volume(int(s), float(d)) for s, d in zip(sizes, dims)]
    vtx = np.zeros((H, W, 3), np.float32)
    nrm = np.zeros((H, W, 3), np.float32)
    lab = np.zeros((H, W), np.int32)
    f = 0
    while f"depth{f}" in g:
        d, rgb, masks = g[f"depth{f}"], g[f"rgb{f}"], g[f"masks{f}"]
        poses, T = g[f"poses{f}"], g[f"T{f}"]
        rgb3 = rgb.astype(np.float32) / np.float32(255.0)
        for i, v in enumerate(vols):
            v.integrate(d, rgb3, masks[i], T, poses[i], g["k"], 0.1)
            keys, coords, active, vox = v.blocks()
            nk, side, cm, nv = v.nodes()
            assert np.array_equal(keys, g[f"f{f}_i{i}_block_keys"]), (f, i)
            assert np.array_equal(active, g[f"f{f}_i{i}_active"]), (f, i)
            assert np.array_equal(nk, g[f"f{f}_i{i}_node_keys"]), (f, i)
            assert np.array_equal(cm, g[f"f{f}_i{i}_children"]), (f, i)
            assert digest(vox) == str(g[f"f{f}_i{i}_voxel_sha"]), (f, i)
            assert digest(nv) == str(g[f"f{f}_i{i}_node_sha"]), (f, i)
        orc.raycast_objects(vols, list(poses), labels, T, g["k"], W, H,
                            eps_size=int(sizes[0]), vertex=vtx, normal=nrm, label_img=lab)
        assert np.array_equal(lab, g[f"f{f}_label"])
        assert np.array_equal(vtx, g[f"f{f}_vertex"])
        assert np.array_equal(nrm, g[f"f{f}_normal"])
        f += 1
    assert f >= 2


def test_track_golden_vectors():
    g = np.load(TRACK_GOLDEN)
    H, W = g["depth0"].shape
    k, labels = g["k"], [int(x) for x in g["labels"]]
    T0, P0, vm, nm, lm = g["T0"], g["P0"], g["vertex"], g["normal"], g["label"]

    def tracker():
        t = O.Tracker(W, H, k, robust=1, fp64=False)
        t.set_frame(g["rgb0"], g["depth0"])
        t.set_ref()
        t.set_frame(g["rgb1"], g["depth1"])
        return t

    def sums(t, level):
        out = np.zeros(32, np.float64)
        t.lib.ot_last_sums(t.h, level, out)
        return out.astype(np.float32)

    F = tracker()
    for level in range(3):
        for which in range(7):
            assert digest(F.level(level, which)) == str(g[f"pyr_l{level}_w{which}"]), (level, which)
    Tc = F.track_camera(T0, T0, vm, nm).astype(np.float32)
    assert np.array_equal(Tc, g["camera_pose"])
    for level in range(3):
        assert np.array_equal(sums(F, level), g["camera_sums"][level]), level
    for i, label in enumerate(labels[1:], 1):
        To = F.track_object(P0[i], Tc, T0, vm, nm, lm, label).astype(np.float32)
        assert np.array_equal(To, g[f"object{label}_pose"]), label
        for level in range(3):
            assert np.array_equal(sums(F, level), g[f"object{label}_sums"][level]), (label, level)
    Fm = tracker()
    Fm.set_mask((np.isin(lm, labels[1:]) * 255).astype(np.uint8))
    assert np.array_equal(Fm.track_camera(T0, T0, vm, nm).astype(np.float32),
                          g["camera_pose_masked"])
    res, err = F.motion_residuals(Tc, T0, vm, nm, g["live_vertex"])
    assert np.array_equal(res, g["residual_codes"])
    assert np.array_equal(err[res == 1], g["residual_errors_valid"])


def test_unique_multiscale_counts(lib):
    # UniqueMultiscaleTest fixture, lib/test/algorithms/unique_unittest.cpp:76-100
    blocks = [(56, 12, 12), (56, 12, 15), (128, 128, 128), (128, 128, 125), (128, 128, 127),
              (128, 136, 129), (128, 136, 127), (136, 128, 136), (128, 240, 136), (128, 241, 136)]
    levels = [7, 7, 3, 5, 6, 7, 7, 7, 7, 7]
    keys = np.array([lib.or_encode(x, y, z, l, 8) & 0xFFFFFFFF for (x, y, z), l in
                     zip(blocks, levels)], np.uint64)
    k1 = np.sort(keys)
    assert lib.or_unique_multiscale(k1, 10, 0x1FF, -1) == 7
    k2 = np.sort(keys)
    assert lib.or_unique_multiscale(k2, 10, 0x1FF, 6) == 6


def test_bilinear_checkerboard(lib):
    img = np.zeros((64, 64), np.float32)
    for y in range(63):
        for x in range(63):
            img[y, x] = (x & 1) ^ (y & 1)
    cases = [((31.0, 32.0), 1.0), ((24.0, 52.0), 0.0), ((24.5, 52.5), 0.5),
             ((24.25, 52.25), 0.375), ((0.82, 0.74), 0.3464)]
    for (x, y), want in cases:
        got = lib.or_bilinear(img.reshape(-1), 64, x, y)
        assert abs(got - want) <= 4 * np.spacing(np.float32(max(abs(want), 1e-30))) + 1e-7, (x, y, got)


def test_morton_round_trip(lib):
    rng = np.random.default_rng(0)
    out = np.zeros(3, np.uint32)
    for _ in range(2000):
        v = rng.integers(0, 4097, 3)
        code = lib.or_morton(int(v[0]), int(v[1]), int(v[2]))
        lib.or_unpack(code, out)
        assert tuple(out) == tuple(v)
    for z in (2048, 3001, 4095):
        for y in (2048, 2049):
            for x in range(0, 4096, 37):
                lib.or_unpack(lib.or_morton(x, y, z), out)
                assert tuple(out) == (x, y, z)


def test_block_key_probe(lib):
    # 256^3 octree, block level 5: hash(8, 0, 0) = 0x205
    assert lib.or_encode(8, 0, 0, 5, 8) == 0x205
    assert O.encode(8, 0, 0, 5, 8) == 0x205

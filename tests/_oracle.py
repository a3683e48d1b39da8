"""ctypes bindings of the CPU oracle (oracle/liboracle.so) and, when it was
built here, of the reference's own hot path (oracle/_ref/libmf_ref.so).

Test infrastructure only: the oracle is the checker, never the thing measured.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libmf_ref.so")
REF_TRACK_SO = os.path.join(ROOT, "oracle", "_ref", "libmf_ref_track.so")

P = C.c_void_p
FP = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
U64P = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
U32P = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
U8P = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")

VOXEL_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("r", "<f4"), ("g", "<f4"), ("b", "<f4"),
                        ("c", "<i4"), ("fg", "<f8"), ("w", "<i4"), ("_pad", "<i4")])
assert VOXEL_DTYPE.itemsize == 40


def encode(x, y, z, level, max_depth):
    """keyops::encode, lib/octant_ops.hpp:51-55 (pure Python, for fixtures)."""
    def spread(v):
        r = 0
        for i in range(21):
            r |= ((v >> i) & 1) << (3 * i)
        return r
    offset = 21 - max_depth + level - 1
    full = 0x7FFFFFFFFFFFFFFF
    mask = (full >> (60 - 3 * offset)) << (60 - 3 * offset) & full
    return ((spread(x) | spread(y) << 1 | spread(z) << 2) & mask) | level


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _bind(lib, prefix):
    def fn(name, res, *args):
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = list(args)
        return f
    b = {}
    b["vol_create"] = fn("vol_create", P, C.c_int, C.c_float)
    b["vol_destroy"] = fn("vol_destroy", None, P)
    b["integrate"] = fn("integrate", C.c_uint, P, FP, FP, FP, C.c_int, C.c_int, FP, FP, FP,
                        C.c_float)
    b["alloc_update"] = fn("alloc_update", None, P, U64P, C.c_int)
    b["block_count"] = fn("block_count", C.c_int, P)
    b["node_count"] = fn("node_count", C.c_int, P)
    b["root_children"] = fn("root_children", C.c_ubyte, P)
    b["export_blocks"] = fn("export_blocks", None, P, U64P, I32P, U8P, C.c_void_p)
    b["export_nodes"] = fn("export_nodes", None, P, U64P, U32P, U8P, C.c_void_p)
    b["interp"] = fn("interp", C.c_float, P, FP, C.c_int)
    b["grad"] = fn("grad", None, P, FP, FP)
    b["raycast"] = fn("raycast", None, P, FP, FP, C.c_float, C.c_float, C.c_float, C.c_float,
                      C.c_float, FP)
    return b


class VolumeHandle:
    """One octree volume held by the oracle or by the compiled reference."""

    def __init__(self, impl, size, dim):
        self.impl, self.size, self.dim = impl, size, dim
        self.h = impl.b["vol_create"](size, float(dim))

    def __del__(self):
        try:
            self.impl.b["vol_destroy"](self.h)
        except Exception:
            pass

    def integrate(self, depth, rgb3, mask, T_w_c, T_w_o, k, mu):
        H, W = depth.shape
        return self.impl.b["integrate"](self.h, _f32(depth), _f32(rgb3), _f32(mask), W, H,
                                        _f32(T_w_c), _f32(T_w_o), _f32(k), float(mu))

    def alloc_update(self, keys):
        keys = np.ascontiguousarray(keys, np.uint64).copy()
        if keys.size == 0:
            keys = np.zeros(1, np.uint64)
            self.impl.b["alloc_update"](self.h, keys, 0)
        else:
            self.impl.b["alloc_update"](self.h, keys, len(keys))

    def blocks(self, with_voxels=True):
        n = self.impl.b["block_count"](self.h)
        keys = np.zeros(n, np.uint64)
        coords = np.zeros((n, 3), np.int32)
        active = np.zeros(n, np.uint8)
        vox = np.zeros((n, 512), VOXEL_DTYPE) if with_voxels else None
        self.impl.b["export_blocks"](self.h, keys, coords, active,
                                     vox.ctypes.data if with_voxels else None)
        order = np.argsort(keys, kind="stable")
        return (keys[order], coords[order], active[order],
                vox[order] if with_voxels else None)

    def nodes(self, with_values=True):
        n = self.impl.b["node_count"](self.h)
        keys = np.zeros(n, np.uint64)
        side = np.zeros(n, np.uint32)
        cmask = np.zeros(n, np.uint8)
        vals = np.zeros((n, 8), VOXEL_DTYPE) if with_values else None
        self.impl.b["export_nodes"](self.h, keys, side, cmask,
                                    vals.ctypes.data if with_values else None)
        order = np.argsort(keys, kind="stable")
        return (keys[order], side[order], cmask[order],
                vals[order] if with_values else None)

    def root_children(self):
        return int(self.impl.b["root_children"](self.h))

    def interp(self, pos, field=0):
        return self.impl.b["interp"](self.h, _f32(pos), field)

    def grad(self, pos):
        out = np.zeros(3, np.float32)
        self.impl.b["grad"](self.h, _f32(pos), out)
        return out


class Impl:
    def __init__(self, path, prefix):
        self.lib = C.CDLL(path)
        self.prefix = prefix
        self.b = _bind(self.lib, prefix)
        if prefix == "or_":
            f = self.lib.or_raycast_objects
            f.restype = None
            f.argtypes = [C.POINTER(P), FP, I32P, C.c_int, FP, FP, C.c_int, C.c_int, C.c_float,
                          C.c_float, C.c_float, C.c_float, FP, FP, I32P]
            g = self.lib.or_ray_first_block
            g.restype = C.c_float
            g.argtypes = [P, FP, FP, C.c_float, C.c_float, C.c_float]
        else:
            f = self.lib.ref_raycast_objects
            f.restype = None
            f.argtypes = [C.POINTER(P), FP, I32P, C.c_int, FP, FP, C.c_int, C.c_int, C.c_float,
                          C.c_float, C.c_float, FP, FP, I32P]
            g = self.lib.ref_ray_first_block
            g.restype = C.c_float
            g.argtypes = [P, FP, FP, C.c_float, C.c_float]
            e = self.lib.ref_pin_epsilon
            e.restype = None
            e.argtypes = [C.c_int]

    def volume(self, size, dim):
        return VolumeHandle(self, size, dim)

    def raycast_objects(self, vols, poses, labels, T_w_c, k, W, H, near=0.1, far=4.0, mu=0.1,
                        eps_size=None, vertex=None, normal=None, label_img=None):
        n = len(vols)
        arr = (P * n)(*[v.h for v in vols])
        vertex = np.zeros((H, W, 3), np.float32) if vertex is None else vertex
        normal = np.zeros((H, W, 3), np.float32) if normal is None else normal
        label_img = np.zeros((H, W), np.int32) if label_img is None else label_img
        Two = _f32(np.stack(poses).reshape(n, 16))
        labels = np.ascontiguousarray(labels, np.int32)
        if self.prefix == "or_":
            eps = float(np.float32(2.0 ** -np.log2(eps_size or vols[0].size)))
            self.lib.or_raycast_objects(arr, Two, labels, n, _f32(T_w_c), _f32(k), W, H, near,
                                        far, mu, eps, vertex, normal, label_img)
        else:
            self.lib.ref_raycast_objects(arr, Two, labels, n, _f32(T_w_c), _f32(k), W, H, near,
                                         far, mu, vertex, normal, label_img)
        return vertex, normal, label_img

    def raycast_oob_mask(self, vols, poses, T_w_c, k, W, H, near=0.1, far=4.0, mu=0.1,
                         eps_size=None):
        """Pixels whose raycast reads voxels outside [0, size) (oracle only)."""
        n = len(vols)
        arr = (P * n)(*[v.h for v in vols])
        mask = np.zeros((H, W), np.uint8)
        eps = float(np.float32(2.0 ** -np.log2(eps_size or vols[0].size)))
        f = self.lib.or_raycast_oob_mask
        f.restype = None
        f.argtypes = [C.POINTER(P), FP, C.c_int, FP, FP, C.c_int, C.c_int, C.c_float, C.c_float,
                      C.c_float, C.c_float, U8P]
        f(arr, _f32(np.stack(poses).reshape(n, 16)), n, _f32(T_w_c), _f32(k), W, H, near, far,
          mu, eps, mask)
        return mask.astype(bool)


def camera_cost(vols, poses, labels, T_w_r, T_live, k, W, H, live, use_icp=True, use_rgb=True,
                fp64=True, pert=(), near=0.1, far=4.0, mu=0.1, eps_size=None):
    """The camera cost at level 0 (oracle/or_adjoint.cpp) for central
    differences: vols are oracle volumes, live = dict of level-0 float arrays
    vertex, normal, cov, intensity, ref_intensity, ref_vertex; pert = iterable
    of (instance, x, y, z, delta) added to voxel TSDF values.  Returns (E, rows)."""
    lib = oracle().lib
    F64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    f = lib.oa_camera_cost
    f.restype = C.c_double
    f.argtypes = [C.POINTER(P), FP, I32P, C.c_int, FP, F64, FP, C.c_int, C.c_int, C.c_float,
                  C.c_float, C.c_float, C.c_float, FP, FP, FP, FP, FP, FP, C.c_int, C.c_int,
                  C.c_int, I32P, F64, C.c_int, F64]
    n = len(vols)
    arr = (P * n)(*[v.h for v in vols])
    pert = list(pert)
    pidx = np.array([[p[0], p[1], p[2], p[3]] for p in pert], np.int32).reshape(-1, 4)
    pval = np.array([p[4] for p in pert], np.float64)
    if len(pert) == 0:
        pidx = np.zeros((1, 4), np.int32)
        pval = np.zeros(1, np.float64)
    rows = np.zeros(1, np.float64)
    eps = float(np.float32(2.0 ** -np.log2(eps_size or vols[0].size)))
    E = f(arr, _f32(np.stack(poses).reshape(n, 16)), np.ascontiguousarray(labels, np.int32), n,
          _f32(T_w_r), np.ascontiguousarray(np.asarray(T_live, np.float64).reshape(16)),
          _f32(k), W, H, near, far, mu, eps, _f32(live["vertex"]), _f32(live["normal"]),
          _f32(live["cov"]), _f32(live["intensity"]), _f32(live["ref_intensity"]),
          _f32(live["ref_vertex"]), int(use_icp), int(use_rgb), int(fp64),
          np.ascontiguousarray(pidx), np.ascontiguousarray(pval), len(pert), rows)
    return float(E), int(rows[0])


_cache = {}


def inlier_ratio(results, labels, label, use_icp=True, use_rgb=True):
    """check_static_state + the inlier ratio of kfusion.cpp:312-320 (-1 when
    the label has no pixel)."""
    lib = oracle().lib
    lib.ot_inlier_ratio.restype = C.c_float
    res = np.ascontiguousarray(results, np.int8)
    lab = np.ascontiguousarray(labels, np.int32)
    return float(lib.ot_inlier_ratio(res.ctypes.data_as(C.c_void_p),
                                     lab.ctypes.data_as(C.c_void_p), int(label), lab.size,
                                     int(use_icp), int(use_rgb)))


def refine_mask_use_motion(mask, results, use_icp=True, use_rgb=True):
    """Object::refine_mask_use_motion on a copy of mask."""
    lib = oracle().lib
    out = np.array(mask, np.float32, copy=True, order="C")
    res = np.ascontiguousarray(results, np.int8)
    lib.ot_refine_mask_use_motion(out.ctypes.data_as(C.c_void_p), res.ctypes.data_as(C.c_void_p),
                                  out.size, int(use_icp), int(use_rgb))
    return out


class Render:
    """The oracle's restatement of the reference's render kernels
    (oracle/or_render.cpp); images as numpy uint8 arrays."""

    def __init__(self, W, H):
        self.lib = oracle().lib
        self.W, self.H = W, H

    def _out(self, c=4):
        return np.zeros((self.H, self.W, c), np.uint8)

    def volume(self, vols, poses, labels, T_w_c, k, near, far, mu, largestep, epsilon,
               render_color, colors, maps=None, T_shade=None, ambient=(0.1, 0.1, 0.1)):
        """renderVolume_many_Kernel; T_w_c None shades `maps` = (vertex,
        normal, label) from T_shade."""
        n = len(vols)
        arr = (P * n)(*[v.h for v in vols])
        out = self._out()
        col = np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        if maps is None:
            v = nr = np.zeros((self.H, self.W, 3), np.float32)
            lab = np.zeros((self.H, self.W), np.int32)
        else:
            v, nr, lab = (_f32(maps[0]), _f32(maps[1]), np.ascontiguousarray(maps[2], np.int32))
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        self.lib.or_render_volume(
            arr, vp(_f32(np.stack(poses).reshape(n, 16))),
            vp(np.ascontiguousarray(labels, np.int32)), n,
            None if T_w_c is None else vp(_f32(T_w_c).reshape(16)), vp(_f32(k)), self.W, self.H,
            C.c_float(near), C.c_float(far), C.c_float(mu), C.c_float(largestep),
            C.c_float(epsilon), vp(_f32(ambient)), int(render_color), vp(col), len(col), vp(v),
            vp(nr), vp(lab), None if T_shade is None else vp(_f32(T_shade).reshape(16)), vp(out))
        return out

    def depth(self, depth, near, far):
        out = self._out()
        d = _f32(depth)
        self.lib.or_render_depth(d.ctypes.data_as(C.c_void_p), d.size, C.c_float(near),
                                 C.c_float(far), out.ctypes.data_as(C.c_void_p))
        return out

    def intensity(self, grey):
        out = self._out()
        g = _f32(grey)
        self.lib.or_render_intensity(g.ctypes.data_as(C.c_void_p), g.size,
                                     out.ctypes.data_as(C.c_void_p))
        return out

    def normal(self, normal):
        out = self._out(3)
        nr = _f32(normal)
        self.lib.or_render_normal(nr.ctypes.data_as(C.c_void_p), nr.size // 3,
                                  out.ctypes.data_as(C.c_void_p))
        return out

    def track(self, res, err, mode):
        out = self._out()
        r = np.ascontiguousarray(res, np.int8)
        e = _f32(err)
        self.lib.or_render_track(r.ctypes.data_as(C.c_void_p), e.ctypes.data_as(C.c_void_p),
                                 self.W * self.H, int(mode), out.ctypes.data_as(C.c_void_p))
        return out

    def mask(self, label, rgb3, mode, colors, rows=()):
        out = self._out()
        lab = np.ascontiguousarray(label, np.int32)
        rgb = _f32(rgb3)
        col = np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        keep = [None if r is None else np.ascontiguousarray(r, np.int8) for r in rows]
        ptrs = (C.c_void_p * max(len(keep), 1))(
            *[None if r is None else r.ctypes.data_as(C.c_void_p).value for r in keep])
        self.lib.or_render_mask(lab.ctypes.data_as(C.c_void_p), rgb.ctypes.data_as(C.c_void_p),
                                lab.size, int(mode), col.ctypes.data_as(C.c_void_p), len(col),
                                ptrs, len(keep), out.ctypes.data_as(C.c_void_p))
        return out


def spawn_object(depth, mask, k, T_w_c):
    """Kfusion::spawnNewObjectKernel: (T_w_o, volume_size, volume_resol, n)."""
    lib = oracle().lib
    lib.or_spawn_object.restype = C.c_int
    d = _f32(depth)
    m = np.ascontiguousarray(mask, np.uint8)
    T = np.zeros(16, np.float32)
    size, resol = C.c_float(), C.c_int()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    n = lib.or_spawn_object(vp(d), vp(m), d.shape[1], d.shape[0], vp(_f32(k)),
                            vp(_f32(T_w_c).reshape(16)), vp(T), C.byref(size), C.byref(resol))
    return T.reshape(4, 4), size.value, resol.value, n


def fuse_semantics(fused, fused_time, probs, recog_times=1):
    """Object::fuseSemanticLabel: (new fused vector, new count, class id)."""
    lib = oracle().lib
    lib.or_fuse_semantics.restype = C.c_int
    f = np.array(fused, np.float32, copy=True)
    ft = C.c_int(fused_time)
    p = _f32(probs)
    cid = lib.or_fuse_semantics(f.ctypes.data_as(C.c_void_p), f.size, C.byref(ft),
                                p.ctypes.data_as(C.c_void_p), int(recog_times))
    return f, ft.value, cid


def mesh(impl, vol, float_bounds=False):
    """Marching-cubes triangles (n, 3, 3) of one volume: the oracle's (or_mesh)
    or the reference's own algorithms::marching_cube (ref_marching_cube, the
    int bound only)."""
    if impl.prefix == "or_":
        f = impl.lib.or_mesh
        f.argtypes = [P, C.c_void_p, C.c_longlong, C.c_int]
        extra = (int(float_bounds),)
    else:
        assert not float_bounds
        f = impl.lib.ref_marching_cube
        f.argtypes = [P, C.c_void_p, C.c_longlong]
        extra = ()
    f.restype = C.c_longlong
    n = f(vol.h, None, 0, *extra)
    out = np.zeros((max(n, 1), 3, 3), np.float32)
    f(vol.h, out.ctypes.data_as(C.c_void_p), n, *extra)
    return out[:n]


def mc_cell(impl, vol, x, y, z):
    """compute_index of a cell (-1 when its block is unallocated) and the
    twelve edge intersections (12, 3)."""
    p = impl.prefix
    fi = getattr(impl.lib, p + "mc_index")
    fi.restype = C.c_int
    fi.argtypes = [P, C.c_int, C.c_int, C.c_int]
    fv = getattr(impl.lib, p + "mc_vertex")
    fv.restype = None
    fv.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, FP]
    verts = np.zeros((12, 3), np.float32)
    for e in range(12):
        fv(vol.h, x, y, z, e, verts[e])
    return fi(vol.h, x, y, z), verts


def oracle():
    if "or" not in _cache:
        _cache["or"] = Impl(ORACLE_SO, "or_")
    return _cache["or"]


def reference():
    """The reference's own hot path, or None when oracle/_ref was not built."""
    if not os.path.exists(REF_SO):
        return None
    if "ref" not in _cache:
        _cache["ref"] = Impl(REF_SO, "ref_")
    return _cache["ref"]


def reference_tracking(path=REF_TRACK_SO):
    """The reference's own tracking / preprocessing / object / rendering code
    (oracle/_ref/libmf_ref_track.so, or another build of it at `path`), or
    None when it was not built."""
    if not os.path.exists(path):
        return None
    key = "reftrk:" + path
    if key not in _cache:
        lib = C.CDLL(path)
        I32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        V = C.c_void_p

        def fn(name, res, *args):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = list(args)
        fn("rt_create", P, C.c_int, C.c_int, C.c_int, I32, C.c_int, C.c_int, C.c_int)
        fn("rt_destroy", None, P)
        fn("rt_rgb2intensity", None, U8P, C.c_int, C.c_int, FP, FP)
        fn("rt_set_frame", None, P, FP, FP, FP, V)
        fn("rt_set_ref_from_current", None, P)
        fn("rt_track_live", C.c_int, P, FP, FP, FP, FP, FP, V)
        fn("rt_reduction", None, P, C.c_int, FP)
        fn("rt_robust", None, P, C.c_int, FP, C.c_int, FP, FP)
        fn("rt_get_level", C.c_int, P, C.c_int, C.c_int, FP)
        fn("rt_track_data", None, P, C.c_int, I32, FP, FP)
        fn("rt_compute_residuals", None, P, FP, FP, FP, FP, FP, C.c_int, C.c_int, C.c_float)
        fn("rt_object_create", P, C.c_int, C.c_int, FP, C.c_int, C.c_float, C.c_int)
        fn("rt_object_destroy", None, P)
        fn("rt_object_set_maps", None, P, C.c_int, C.c_int, V, V, V)
        fn("rt_object_set_pose", None, P, V, V)
        fn("rt_object_pose", None, P, FP, FP)
        fn("rt_track_object", None, P, P, FP, FP, FP, FP, FP)
        fn("rt_object_take_results", None, P, P)
        fn("rt_refine_mask_use_motion", None, P, FP, C.c_int, C.c_int, C.c_int, C.c_int)
        fn("rt_object_set_static_state", C.c_int, P, C.c_int)
        fn("rt_object_fuse_semantics", C.c_int, P, FP, C.c_int, FP)
        fn("rt_pin_epsilon", None, C.c_int)
        fn("rt_object_set_label", None, P, C.c_int)
        fn("rt_object_integrate", None, P, FP, FP, FP, C.c_int, C.c_int, FP, FP, C.c_float,
           C.c_int)
        fn("rt_raycast_objects", None, V, C.c_int, FP, FP, C.c_int, C.c_int, C.c_float,
           C.c_float, C.c_float, FP, FP, I32)
        fn("rt_render_volume", None, V, C.c_int, U8P, C.c_int, C.c_int, FP, FP, C.c_float,
           C.c_float, C.c_float, C.c_float, FP, C.c_int, C.c_int, FP, FP, I32, U8P, C.c_int)
        fn("rt_render_depth", None, U8P, FP, C.c_int, C.c_int, C.c_float, C.c_float)
        fn("rt_render_intensity", None, U8P, FP, C.c_int, C.c_int)
        fn("rt_render_normal", None, U8P, FP, C.c_int, C.c_int)
        fn("rt_render_track", None, U8P, I32, FP, C.c_int, C.c_int, C.c_int)
        fn("rt_check_static_state", None, U8P, U8P, I32, C.c_int, C.c_int, C.c_int, C.c_int)
        fn("rt_render_mask", None, U8P, FP, I32, C.c_int, C.c_int, C.c_int, U8P, C.c_int, V,
           C.c_int)
        fn("rt_object_set_results", None, P, I32, C.c_int, C.c_int)
        _cache[key] = lib
    return _cache[key]


def _vp(a):
    return None if a is None else a.ctypes.data


class RefTracker:
    """The reference's Tracking class (tracking.cpp) compiled from its own
    sources: ICP + photometric rows, robust kernel Huber by default."""

    def __init__(self, W, H, k, iters=(10, 5, 4), robust=1, use_icp=True, use_rgb=True,
                 lib=None):
        self.lib = lib or reference_tracking()
        assert self.lib is not None, "oracle/_ref/libmf_ref_track.so not built"
        self.W, self.H, self.k = W, H, _f32(k)
        self.levels = len(iters)
        self.h = self.lib.rt_create(W, H, len(iters), np.asarray(iters, np.int32), robust,
                                    int(use_icp), int(use_rgb))

    def __del__(self):
        try:
            self.lib.rt_destroy(self.h)
        except Exception:
            pass

    def grey(self, rgb):
        g = np.zeros((self.H, self.W), np.float32)
        c = np.zeros((self.H, self.W, 3), np.float32)
        self.lib.rt_rgb2intensity(np.ascontiguousarray(rgb, np.uint8), self.W, self.H, g, c)
        return g

    def set_frame(self, rgb, depth, human_mask=None):
        self._grey = self.grey(rgb)
        self._depth = _f32(depth)
        m = None if human_mask is None else np.ascontiguousarray(human_mask, np.uint8)
        self.lib.rt_set_frame(self.h, self.k, self._grey, self._depth, _vp(m))

    def set_ref(self):
        self.lib.rt_set_ref_from_current(self.h)

    def track_camera(self, T_in, T_w_r, vertex, normal, mask=None):
        T = _f32(T_in).reshape(16).copy()
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.lib.rt_track_live(self.h, T, _f32(T_w_r).reshape(16), self.k, _f32(vertex),
                               _f32(normal), _vp(m))
        return T.reshape(4, 4)

    def object(self, T_w_o, vertex=None, normal=None, vertex_bef=None, class_id=1):
        o = RefObject(self, T_w_o, class_id)
        o.set_maps(vertex, normal, vertex_bef)
        return o

    def track_object(self, obj, T_w_c2, T_w_c1):
        self.lib.rt_track_object(self.h, obj.h, self.k, _f32(T_w_c2).reshape(16),
                                 _f32(T_w_c1).reshape(16), self._grey, self._depth)
        return obj.pose()

    def reduction(self, level):
        out = np.zeros(32, np.float32)
        self.lib.rt_reduction(self.h, level, out)
        return out

    def robust(self, kind, e):
        """calc_robust_weight / calc_robust_residual of float32 residuals e:
        (weights, losses)."""
        e = np.ascontiguousarray(e, np.float32)
        w = np.zeros_like(e)
        loss = np.zeros_like(e)
        self.lib.rt_robust(self.h, int(kind), e, e.size, w, loss)
        return w, loss

    def level(self, l, which):
        w, h = self.W >> l, self.H >> l
        out = np.zeros(w * h * 3, np.float32)
        self.lib.rt_get_level(self.h, l, which, out)
        if which in (2, 3, 6, 7, 9):
            return out.reshape(h, w, 3)
        return out[:w * h].reshape(h, w)

    def track_data(self, level=0):
        n = 2 * self.W * self.H
        res = np.zeros(n, np.int32)
        err = np.zeros(n, np.float32)
        J = np.zeros(6 * n, np.float32)
        self.lib.rt_track_data(self.h, level, res, err, J)
        return (res.reshape(2, self.H, self.W), err.reshape(2, self.H, self.W),
                J.reshape(2, self.H, self.W, 6))

    def compute_residuals(self, T_w_l, T_w_r, vertex, normal, vertex_l, use_icp=True,
                          use_rgb=True, threshold=1.5):
        self.lib.rt_compute_residuals(self.h, _f32(T_w_l).reshape(16), _f32(T_w_r).reshape(16),
                                      _f32(vertex), _f32(normal), _f32(vertex_l), int(use_icp),
                                      int(use_rgb), float(threshold))
        return self.track_data(0)


class RefObject:
    """The reference's Object (object.cpp): pose, volume, model maps, result
    rows and semantic state (a small 64^3 volume unless size / dim are given)."""

    def __init__(self, trk, T_w_o, class_id=1, size=64, dim=1.0, label=None):
        self.lib, self.W, self.H = trk.lib, trk.W, trk.H
        self.h = self.lib.rt_object_create(trk.W, trk.H, _f32(T_w_o).reshape(16), int(size),
                                           float(dim), class_id)
        if label is not None:
            self.lib.rt_object_set_label(self.h, int(label))

    def integrate(self, depth, rgb3, mask, T_w_c, k, mu=0.1, frame=0):
        self.lib.rt_object_integrate(self.h, _f32(depth), _f32(rgb3), _f32(mask), self.W, self.H,
                                     _f32(T_w_c).reshape(16), _f32(k), float(mu), int(frame))

    def __del__(self):
        try:
            self.lib.rt_object_destroy(self.h)
        except Exception:
            pass

    def set_maps(self, vertex=None, normal=None, vertex_bef=None):
        keep = [None if a is None else _f32(a) for a in (vertex, normal, vertex_bef)]
        self.lib.rt_object_set_maps(self.h, self.W, self.H, *[_vp(a) for a in keep])

    def set_pose(self, T_w_o=None, T_virtual=None):
        keep = [None if a is None else _f32(a).reshape(16) for a in (T_w_o, T_virtual)]
        self.lib.rt_object_set_pose(self.h, *[_vp(a) for a in keep])

    def pose(self):
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        self.lib.rt_object_pose(self.h, a, b)
        return a.reshape(4, 4), b.reshape(4, 4)

    def set_results(self, res):
        self.lib.rt_object_set_results(self.h, np.ascontiguousarray(res, np.int32).reshape(-1),
                                       self.W, self.H)

    def take_results(self, trk):
        self.lib.rt_object_take_results(self.h, trk.h)

    def refine_mask(self, mask, use_icp=True, use_rgb=True):
        m = _f32(mask).copy()
        self.lib.rt_refine_mask_use_motion(self.h, m, self.W, self.H, int(use_icp), int(use_rgb))
        return m

    def set_static_state(self, state):
        return bool(self.lib.rt_object_set_static_state(self.h, int(state)))

    def fuse_semantics(self, prob, recog_time=1):
        out = np.zeros(80, np.float32)
        cid = self.lib.rt_object_fuse_semantics(self.h, _f32(prob), int(recog_time), out)
        return cid, out


class RefRender:
    """The reference's raycastObjectList and render kernels (rendering.cpp),
    compiled from its own sources, over RefObject lists."""

    def __init__(self, W, H, lib=None):
        self.lib = lib or reference_tracking()
        assert self.lib is not None, "oracle/_ref/libmf_ref_track.so not built"
        self.W, self.H = W, H

    @staticmethod
    def _objs(objs):
        return (C.c_void_p * len(objs))(*[o.h for o in objs])

    def raycast(self, objs, T_w_c, k, near=0.1, far=4.0, mu=0.1):
        v = np.zeros((self.H, self.W, 3), np.float32)
        n = np.zeros((self.H, self.W, 3), np.float32)
        lab = np.zeros((self.H, self.W), np.int32)
        self.lib.rt_raycast_objects(self._objs(objs), len(objs), _f32(T_w_c).reshape(16), _f32(k),
                                    self.W, self.H, near, far, mu, v, n, lab)
        return v, n, lab

    def volume(self, objs, T_w_c, k, near, far, mu, largestep, render_color, colors, maps=None,
               ambient=(0.1, 0.1, 0.1)):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        if maps is None:
            v = nr = np.zeros((self.H, self.W, 3), np.float32)
            lab = np.zeros((self.H, self.W), np.int32)
        else:
            v, nr, lab = _f32(maps[0]), _f32(maps[1]), np.ascontiguousarray(maps[2], np.int32)
        col = np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        self.lib.rt_render_volume(self._objs(objs), len(objs), out, self.W, self.H,
                                  _f32(T_w_c).reshape(16), _f32(k), near, far, mu, largestep,
                                  _f32(ambient), int(maps is None), int(render_color), v, nr, lab,
                                  col, len(col))
        return out

    def depth(self, depth, near, far):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        self.lib.rt_render_depth(out, _f32(depth), self.W, self.H, near, far)
        return out

    def intensity(self, grey):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        self.lib.rt_render_intensity(out, _f32(grey), self.W, self.H)
        return out

    def normal(self, normal):
        out = np.zeros((self.H, self.W, 3), np.uint8)
        self.lib.rt_render_normal(out, _f32(normal), self.W, self.H)
        return out

    def track(self, res, err, mode):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        self.lib.rt_render_track(out, np.ascontiguousarray(res, np.int32), _f32(err), self.W,
                                 self.H, int(mode))
        return out

    def mask(self, label, rgb3, mode, colors, objs=()):
        """renderInstanceMaskKernel (0), renderMaskWithImageKernel (1),
        renderMaskMotionWithImageKernel (2, objs[label]'s result rows)."""
        out = np.zeros((self.H, self.W, 4), np.uint8)
        col = np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        arr = self._objs(objs) if objs else None
        self.lib.rt_render_mask(out, _f32(rgb3), np.ascontiguousarray(label, np.int32), self.W,
                                self.H, int(mode), col, len(col), arr, len(objs))
        return out

    def static_inliers(self, object_mask, res, use_icp=True, use_rgb=True):
        out = np.zeros((self.H, self.W), np.uint8)
        self.lib.rt_check_static_state(out, np.ascontiguousarray(object_mask, np.uint8),
                                       np.ascontiguousarray(res, np.int32), self.W, self.H,
                                       int(use_icp), int(use_rgb))
        return out


class Tracker:
    """The tracking oracle (fp64=True: all-FP64; False: the reference's FP32 order)."""

    def __init__(self, W, H, k, iters=(10, 5, 4), robust=1, use_icp=True, use_rgb=True,
                 fp64=True):
        lib = oracle().lib
        self.lib = lib
        self.W, self.H = W, H
        I32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        U8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        F64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        lib.ot_create.restype = P
        lib.ot_create.argtypes = [C.c_int, C.c_int, FP, C.c_int, I32, C.c_int, C.c_int, C.c_int,
                                  C.c_int]
        lib.ot_destroy.argtypes = [P]
        lib.ot_set_frame.argtypes = [P, U8, FP]
        lib.ot_set_ref_from_current.argtypes = [P]
        lib.ot_set_outlier_mask.argtypes = [P, U8]
        lib.ot_track_camera.argtypes = [P, FP, FP, FP, FP, FP, C.c_void_p]
        lib.ot_track_object.argtypes = [P, FP, FP, FP, FP, FP, I32, C.c_int, FP, C.c_void_p]
        lib.ot_camera_sums.argtypes = [P, C.c_int, FP, FP, FP, FP, F64]
        lib.ot_object_sums.argtypes = [P, C.c_int, FP, FP, FP, FP, FP, I32, C.c_int, F64]
        lib.ot_last_sums.argtypes = [P, C.c_int, F64]
        lib.ot_last_iterations.restype = C.c_int
        lib.ot_last_iterations.argtypes = [P, C.c_int]
        lib.ot_get_level.restype = C.c_int
        lib.ot_get_level.argtypes = [P, C.c_int, C.c_int, FP]
        I8 = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
        lib.ot_motion_residuals.restype = C.c_int
        lib.ot_motion_residuals.argtypes = [P, FP, FP, FP, FP, FP, C.c_float, I8, FP]
        lib.ot_last_results.restype = C.c_int
        lib.ot_last_results.argtypes = [P, I8]
        lib.ot_set_level.restype = C.c_int
        lib.ot_set_level.argtypes = [P, C.c_int, C.c_int, FP]
        it = np.zeros(4, np.int32)
        it[:len(iters)] = iters
        self.levels = len(iters)
        self.h = lib.ot_create(W, H, _f32(k), len(iters), it, robust, int(use_icp), int(use_rgb),
                               int(fp64))

    def __del__(self):
        try:
            self.lib.ot_destroy(self.h)
        except Exception:
            pass

    def set_frame(self, rgb, depth):
        self.lib.ot_set_frame(self.h, np.ascontiguousarray(rgb, np.uint8), _f32(depth))

    def set_ref(self):
        self.lib.ot_set_ref_from_current(self.h)

    def set_mask(self, mask):
        self.lib.ot_set_outlier_mask(self.h, np.ascontiguousarray(mask, np.uint8))

    def track_camera(self, T_in, T_w_r, vertex, normal):
        out = np.zeros(16, np.float32)
        out64 = np.zeros(16, np.float64)
        self.lib.ot_track_camera(self.h, _f32(T_in).reshape(16), _f32(T_w_r).reshape(16),
                                 _f32(vertex), _f32(normal), out, out64.ctypes.data)
        return out64.reshape(4, 4)

    def track_object(self, T_wo1, T_w_c2, T_w_c1, vertex, normal, labels, label):
        out = np.zeros(16, np.float32)
        out64 = np.zeros(16, np.float64)
        self.lib.ot_track_object(self.h, _f32(T_wo1).reshape(16), _f32(T_w_c2).reshape(16),
                                 _f32(T_w_c1).reshape(16), _f32(vertex), _f32(normal),
                                 np.ascontiguousarray(labels, np.int32), int(label), out,
                                 out64.ctypes.data)
        return out64.reshape(4, 4)

    def camera_sums(self, level, T_w_l, T_w_r, vertex, normal):
        out = np.zeros(32, np.float64)
        self.lib.ot_camera_sums(self.h, level, _f32(T_w_l).reshape(16), _f32(T_w_r).reshape(16),
                                _f32(vertex), _f32(normal), out)
        return out

    def object_sums(self, level, T_c2_o2, T_wo1, T_w_c1, vertex, normal, labels, label):
        out = np.zeros(32, np.float64)
        self.lib.ot_object_sums(self.h, level, _f32(T_c2_o2).reshape(16), _f32(T_wo1).reshape(16),
                                _f32(T_w_c1).reshape(16), _f32(vertex), _f32(normal),
                                np.ascontiguousarray(labels, np.int32), int(label), out)
        return out

    def motion_residuals(self, T_w_l, T_w_r, vertex, normal, live_vertex, threshold=1.5):
        """Tracking::compute_residuals at level 0: (results int8 (2, H, W),
        errors (2, H, W)); single-precision tracker only."""
        res = np.zeros((2, self.H, self.W), np.int8)
        err = np.zeros((2, self.H, self.W), np.float32)
        rc = self.lib.ot_motion_residuals(self.h, _f32(T_w_l).reshape(16),
                                          _f32(T_w_r).reshape(16), _f32(vertex), _f32(normal),
                                          _f32(live_vertex), threshold, res, err)
        assert rc == 0, "motion residuals need the single-precision tracker"
        return res, err

    def set_level(self, level, which, data):
        """Overwrite a pyramid plane (which as in level(); 8 = reference
        intensity, 9 = reference vertex)."""
        assert self.lib.ot_set_level(self.h, level, which, _f32(data).reshape(-1)) > 0

    def last_results(self):
        """Level-0 row codes (2, H, W) of the last camera / object evaluation."""
        out = np.zeros(2 * self.W * self.H, np.int8)
        n = self.lib.ot_last_results(self.h, out)
        assert n == out.size
        return out.reshape(2, self.H, self.W)

    def iterations(self):
        return [self.lib.ot_last_iterations(self.h, l) for l in range(self.levels)]

    def level(self, l, which):
        n = (self.W >> l) * (self.H >> l)
        out = np.zeros(n * 3, np.float32)
        if self.lib.ot_get_level(self.h, l, which, out) < 0:
            raise ValueError(f"pyramid plane {which} of level {l} is not computed yet")
        if which in (2, 3, 6, 7):
            return out.reshape(self.H >> l, self.W >> l, 3)
        return out[:n].reshape(self.H >> l, self.W >> l)

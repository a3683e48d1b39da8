"""ctypes binding of the C ABI in include/midfusion_b200.h.

The CUDA library is the product; this module only loads it and converts
numpy arrays to pointers.  Loading fails loudly when the library is missing:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmidfusion_b200.so")

MF_OK = 0
ERRORS = {-1: "MF_E_ARG", -2: "MF_E_CUDA", -3: "MF_E_POOL_FULL", -4: "MF_E_NOT_FOUND",
          -5: "MF_E_STATE", -6: "MF_E_TIMEOUT"}
STATUS_POOL_FULL, STATUS_ALLOC_OVERFLOW, STATUS_RAY_GUARD, STATUS_GN_FALLBACK = 1, 2, 4, 8
ROBUST = {"none": 0, "huber": 1, "tukey": 2, "cauchy": 3}

VOXEL_DTYPE = np.dtype([("x", "<f4"), ("y", "<f4"), ("r", "<f4"), ("g", "<f4"), ("b", "<f4"),
                        ("c", "<i4"), ("fg", "<f8"), ("w", "<i4"), ("_pad", "<i4")])

# Every symbol include/midfusion_b200.h declares (checked by the CPU tests).
EXPORTS = [
    "mf_config_default", "mf_create", "mf_destroy", "mf_last_error", "mf_status",
    "mf_get_stream", "mf_synchronize", "mf_instance_add", "mf_instance_count",
    "mf_instance_set_pose", "mf_instance_get_pose", "mf_set_camera_pose", "mf_get_camera_pose",
    "mf_frame_upload", "mf_frame_set_device", "mf_frame_labels", "mf_integrate",
    "mf_alloc_update", "mf_raycast", "mf_download_raycast", "mf_block_count",
    "mf_export_blocks", "mf_node_count", "mf_export_nodes", "mf_root_children", "mf_interp",
    "mf_preprocess", "mf_set_ref_from_current", "mf_track_camera", "mf_track_objects",
    "mf_track_info", "mf_track_eval", "mf_download_pyramid", "mf_process_frame",
    "mf_process_frame_device", "mf_get_poses", "mf_frame_stats", "mf_set_graphs",
    "mf_profile", "mf_track_eval_static", "mf_camera_cost", "mf_pool_tsdf", "mf_pool_slots",
    "mf_debug_gn_step", "mf_set_overlap",
    "mf_motion_residuals", "mf_motion_download", "mf_track_results",
    "mf_refine_mask_use_motion", "mf_download_mask", "mf_retrack_camera",
    "mf_render_volume", "mf_render_depth", "mf_render_intensity", "mf_render_normal",
    "mf_render_track", "mf_render_mask", "mf_spawn_object", "mf_instance_set_semantics",
    "mf_fuse_semantics", "mf_instance_semantics", "mf_frame_upload_raw", "mf_raw_open",
    "mf_raw_read", "mf_raw_close", "mf_save_poses", "mf_pose_quaternion", "mf_tum_line",
    "mf_mesh", "mf_write_vtk_mesh", "mf_dump_mesh", "mf_tune_candidates", "mf_tune_describe",
    "mf_autotune", "mf_tune_get", "mf_tune_set", "mf_process_frame_motion",
    "mf_set_gn_persistent", "mf_object_residuals", "mf_mesh_set_triangle_table",
    "mf_raycast_records", "mf_raycast_fold", "mf_frame_stage", "mf_process_staged",
    "mf_upload_stream",
]

TUNE_RAYCAST, TUNE_INTEGRATE, TUNE_MAX_VARIANTS = 0, 1, 16


class MfConfig(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("k", C.c_float * 4),
                ("mu", C.c_float), ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("max_weight", C.c_int), ("pyramid_levels", C.c_int),
                ("gn_iterations", C.c_int * 4), ("robust_kernel", C.c_int),
                ("use_icp", C.c_int), ("use_rgb", C.c_int), ("pool_blocks", C.c_longlong),
                ("max_instances", C.c_int), ("batched", C.c_int)]


class MfError(RuntimeError):
    pass


_lib = None


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MfError(f"CUDA library not built: {LIB_PATH} (run python -m mid_fusion_b200.build)")
        _lib = C.CDLL(LIB_PATH)
        _lib.mf_last_error.restype = C.c_char_p
        _lib.mf_last_error.argtypes = [C.c_void_p]
    return _lib


def _ptr(a, dtype):
    if a is None:
        return None
    assert a.dtype == dtype and a.flags.c_contiguous, (a.dtype, dtype)
    return a.ctypes.data_as(C.c_void_p)


def tune_candidates(stage):
    """Number of launch-shape candidates of a tuned stage (TUNE_RAYCAST, TUNE_INTEGRATE)."""
    n = C.c_int()
    rc = load().mf_tune_candidates(int(stage), C.byref(n))
    if rc != MF_OK:
        raise MfError(f"{ERRORS.get(rc, rc)} stage {stage}")
    return n.value


def tune_describe(stage, variant):
    buf = C.create_string_buffer(128)
    rc = load().mf_tune_describe(int(stage), int(variant), buf, len(buf))
    if rc != MF_OK:
        raise MfError(f"{ERRORS.get(rc, rc)} stage {stage} variant {variant}")
    return buf.value.decode()


def _m4(T):
    return np.ascontiguousarray(np.asarray(T, np.float32).reshape(16))


class Context:
    """One mf_context: the device-side state of the whole per-frame hot path."""

    def __init__(self, width, height, k=None, mu=0.1, pool_blocks=1 << 17, max_instances=16,
                 batched=True, robust="cauchy", use_icp=True, use_rgb=True,
                 gn_iterations=(10, 5, 4), near=0.1, far=4.0):
        self.lib = load()
        cfg = MfConfig()
        self._check(self.lib.mf_config_default(C.byref(cfg), width, height))
        if k is not None:
            for i in range(4):
                cfg.k[i] = float(k[i])
        cfg.mu = mu
        cfg.pool_blocks = int(pool_blocks)
        cfg.max_instances = max_instances
        cfg.batched = 1 if batched else 0
        cfg.robust_kernel = ROBUST[robust]
        cfg.use_icp, cfg.use_rgb = int(use_icp), int(use_rgb)
        cfg.pyramid_levels = len(gn_iterations)
        for i, it in enumerate(gn_iterations):
            cfg.gn_iterations[i] = it
        cfg.near_plane, cfg.far_plane = near, far
        self.cfg = cfg
        self.W, self.H = width, height
        h = C.c_void_p()
        self._check(self.lib.mf_create(C.byref(cfg), C.byref(h)), ctx=False)
        self.h = h
        self.n_instances = 0

    def _check(self, rc, ctx=True):
        if rc != MF_OK:
            msg = ""
            if ctx and getattr(self, "h", None):
                msg = self.lib.mf_last_error(self.h).decode()
            raise MfError(f"{ERRORS.get(rc, rc)} {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- setup
    def add_instance(self, size, dim, T_w_o, label):
        i = C.c_int()
        self._check(self.lib.mf_instance_add(self.h, int(size), C.c_float(dim),
                                             _ptr(_m4(T_w_o), np.float32), int(label),
                                             C.byref(i)))
        self.n_instances += 1
        return i.value

    def set_instance_pose(self, i, T):
        self._check(self.lib.mf_instance_set_pose(self.h, i, _ptr(_m4(T), np.float32)))

    def instance_pose(self, i):
        T = np.zeros(16, np.float32)
        self._check(self.lib.mf_instance_get_pose(self.h, i, _ptr(T, np.float32)))
        return T.reshape(4, 4)

    def set_camera_pose(self, T):
        self._check(self.lib.mf_set_camera_pose(self.h, _ptr(_m4(T), np.float32)))

    def camera_pose(self):
        T = np.zeros(16, np.float32)
        self._check(self.lib.mf_get_camera_pose(self.h, _ptr(T, np.float32)))
        return T.reshape(4, 4)

    # ---------------------------------------------------------------- frames
    def upload(self, depth=None, rgb=None, masks=None):
        d = None if depth is None else np.ascontiguousarray(depth, np.float32)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        m = None if masks is None else np.ascontiguousarray(masks, np.float32)
        n = 0 if m is None else m.shape[0]
        self._check(self.lib.mf_frame_upload(self.h, _ptr(d, np.float32), _ptr(r, np.uint8),
                                             _ptr(m, np.float32), n))

    def upload_labels(self, labels):
        lab = np.ascontiguousarray(labels, np.uint16)
        self._check(self.lib.mf_frame_labels(self.h, _ptr(lab, np.uint16)))

    # ---------------------------------------------------------------- stages
    def integrate(self, ids):
        ids = np.ascontiguousarray(ids, np.int32)
        self._check(self.lib.mf_integrate(self.h, _ptr(ids, np.int32), len(ids)))

    def alloc_update(self, i, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        self._check(self.lib.mf_alloc_update(self.h, i, _ptr(keys, np.uint64), len(keys)))

    def raycast(self):
        self._check(self.lib.mf_raycast(self.h))

    def raycast_records(self, ids, d_records, d_origins):
        """Records of instances `ids` into device memory (mf_ray_record: 48 B
        per instance and pixel; mf_ray_origin: 32 B per instance)."""
        arr = np.ascontiguousarray(ids, np.int32)
        self._check(self.lib.mf_raycast_records(self.h, _ptr(arr, np.int32), len(arr),
                                                C.c_void_p(d_records), C.c_void_p(d_origins)))

    def raycast_fold(self, d_records, d_origins):
        """The composite maps from every instance's records (device memory)."""
        self._check(self.lib.mf_raycast_fold(self.h, C.c_void_p(d_records),
                                             C.c_void_p(d_origins)))

    def download_raycast(self):
        v = np.zeros((self.H, self.W, 3), np.float32)
        n = np.zeros((self.H, self.W, 3), np.float32)
        lab = np.zeros((self.H, self.W), np.int32)
        self._check(self.lib.mf_download_raycast(self.h, _ptr(v, np.float32),
                                                 _ptr(n, np.float32), _ptr(lab, np.int32)))
        return v, n, lab

    def frame_stats(self):
        out = np.zeros(3 + self.n_instances, np.int64)
        self._check(self.lib.mf_frame_stats(self.h, _ptr(out, np.int64), len(out)))
        return {"pool_blocks": int(out[0]), "visited_blocks": int(out[1]),
                "emitted": [int(v) for v in out[2:2 + self.n_instances]],
                "graph_kernels": int(out[2 + self.n_instances])}

    def profile(self, reps=20):
        out = np.zeros(6, np.float64)
        self._check(self.lib.mf_profile(self.h, int(reps), _ptr(out, np.float64), len(out)))
        return {"gn_l0_us": out[0], "gn_l0_bytes": out[1], "integrate_us": out[2],
                "integrate_bytes": out[3], "raycast_us": out[4], "raycast_bytes": out[5]}

    def process_frame_motion(self, depth, rgb, labels, residual_threshold=1.5,
                             moved_threshold=0.9):
        """One frame through mf_process_frame_motion; returns the moving-label bits."""
        d = np.ascontiguousarray(depth, np.float32)
        r = np.ascontiguousarray(rgb, np.uint8)
        lab = np.ascontiguousarray(labels, np.uint16)
        bits = C.c_uint32()
        self._check(self.lib.mf_process_frame_motion(
            self.h, _ptr(d, np.float32), _ptr(r, np.uint8), _ptr(lab, np.uint16),
            C.c_float(residual_threshold), C.c_float(moved_threshold), C.byref(bits)))
        return bits.value

    def autotune(self, reps=5):
        """Time every launch-shape candidate on the current frame and keep the
        fastest (mf_autotune); returns the per-candidate times and the choice."""
        ray = np.zeros(TUNE_MAX_VARIANTS, np.float32)
        integ = np.zeros(TUNE_MAX_VARIANTS, np.float32)
        self._check(self.lib.mf_autotune(self.h, int(reps), _ptr(ray, np.float32),
                                         _ptr(integ, np.float32)))
        out = {}
        for name, stage, t in (("raycast", TUNE_RAYCAST, ray), ("integrate", TUNE_INTEGRATE, integ)):
            n = tune_candidates(stage)
            v = self.tune_get(stage)
            out[name] = {"us": [round(float(x), 2) for x in t[:n]], "chosen": v,
                         "shape": tune_describe(stage, v)}
        return out

    def tune_get(self, stage):
        v = C.c_int()
        self._check(self.lib.mf_tune_get(self.h, int(stage), C.byref(v)))
        return v.value

    def tune_set(self, stage, variant):
        self._check(self.lib.mf_tune_set(self.h, int(stage), int(variant)))

    def set_overlap(self, ctas):
        """mf_set_overlap: background integration overlapped with object
        tracking on a low-priority stream with `ctas` CTAs (0: off)."""
        self._check(self.lib.mf_set_overlap(self.h, int(ctas)))

    def set_gn_persistent(self, enable):
        self._check(self.lib.mf_set_gn_persistent(self.h, int(enable)))

    def status(self):
        f = C.c_int()
        self._check(self.lib.mf_status(self.h, C.byref(f)))
        return f.value

    def synchronize(self):
        self._check(self.lib.mf_synchronize(self.h))

    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.mf_get_stream(self.h, C.byref(s)))
        return s.value

    def upload_stream(self):
        s = C.c_void_p()
        self._check(self.lib.mf_upload_stream(self.h, C.byref(s)))
        return s.value

    def frame_stage(self, slot, depth, rgb, labels=None):
        """Upload a frame into input slot 0 or 1 (mf_frame_stage).  The arrays
        are borrowed: keep them alive and unchanged until the frame has been
        processed and mf_get_poses has returned."""
        lab = None if labels is None else labels.ctypes.data_as(C.c_void_p)
        self._check(self.lib.mf_frame_stage(self.h, int(slot), depth.ctypes.data_as(C.c_void_p),
                                            rgb.ctypes.data_as(C.c_void_p), lab))

    def process_staged(self, slot):
        self._check(self.lib.mf_process_staged(self.h, int(slot)))

    # ---------------------------------------------------------------- tracking
    def preprocess(self):
        self._check(self.lib.mf_preprocess(self.h))

    def set_ref_from_current(self):
        self._check(self.lib.mf_set_ref_from_current(self.h))

    def track_camera(self, moving_labels=()):
        bits = 0
        for l in moving_labels:
            bits |= 1 << int(l)
        self._check(self.lib.mf_track_camera(self.h, C.c_uint32(bits)))

    def retrack_camera(self, moving_bits):
        """mf_retrack_camera with label bits (as motion_residuals returns)."""
        self._check(self.lib.mf_retrack_camera(self.h, C.c_uint32(int(moving_bits))))

    def track_objects(self, ids):
        ids = np.ascontiguousarray(ids, np.int32)
        self._check(self.lib.mf_track_objects(self.h, _ptr(ids, np.int32), len(ids)))

    def track_info(self, slot):
        it = np.zeros(4, np.int32)
        sums = np.zeros((4, 32), np.float64)
        T = np.zeros(16, np.float64)
        self._check(self.lib.mf_track_info(self.h, slot, _ptr(it, np.int32),
                                           _ptr(sums, np.float64), _ptr(T, np.float64)))
        return it, sums, T.reshape(4, 4)

    def track_eval(self, slot, level, pose=None):
        sums = np.zeros(32, np.float64)
        p = None if pose is None else _m4(pose)
        self._check(self.lib.mf_track_eval(self.h, slot, level, _ptr(p, np.float32),
                                           _ptr(sums, np.float64)))
        return sums

    def debug_gn_step(self, state, sums):
        """mf_debug_gn_step: state (n, 36), sums (n, 32) -> (device, host)
        outputs, each (n, 68)."""
        state = np.ascontiguousarray(state, np.float64)
        sums = np.ascontiguousarray(sums, np.float64)
        n = state.shape[0]
        dev = np.zeros((n, 68), np.float64)
        host = np.zeros((n, 68), np.float64)
        self._check(self.lib.mf_debug_gn_step(self.h, n, _ptr(state, np.float64),
                                              _ptr(sums, np.float64), _ptr(dev, np.float64),
                                              _ptr(host, np.float64)))
        return dev, host

    def camera_cost(self, T_live, grad_tsdf_ptr=None):
        """E, dE/d twist (6) and the number of rows (mf_camera_cost); when
        grad_tsdf_ptr (a device address of pool_size() floats) is given,
        dE/d tsdf is added there."""
        out = np.zeros(8, np.float64)
        self._check(self.lib.mf_camera_cost(self.h, _ptr(_m4(T_live), np.float32),
                                            _ptr(out, np.float64),
                                            C.c_void_p(grad_tsdf_ptr) if grad_tsdf_ptr else None))
        return out[0], out[1:7].copy(), int(out[7])

    def pool_slots(self):
        """(n, 4) int32: corner voxel x, y, z and instance of each used pool slot."""
        n = C.c_longlong()
        self._check(self.lib.mf_pool_slots(self.h, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 4), np.int32)
        self._check(self.lib.mf_pool_slots(self.h, _ptr(out, np.int32), n.value, C.byref(n)))
        return out[:n.value]

    def pool_tsdf(self):
        """(device address, length) of the pool's TSDF values."""
        p = C.c_void_p()
        n = C.c_longlong()
        self._check(self.lib.mf_pool_tsdf(self.h, C.byref(p), C.byref(n)))
        return p.value, n.value

    def motion_residuals(self, threshold=1.5, moved=0.9):
        """Per-instance inlier ratios and the moving-label bits
        (mf_motion_residuals)."""
        ratio = np.zeros(max(self.n_instances, 1), np.float32)
        bits = C.c_uint32()
        self._check(self.lib.mf_motion_residuals(self.h, C.c_float(threshold), C.c_float(moved),
                                                 _ptr(ratio, np.float32), C.byref(bits)))
        return ratio[:self.n_instances], bits.value

    def motion_download(self):
        """(results int8 (2, H, W), errors (2, H, W), live vertex (H, W, 3),
        live label (H, W)) of the last motion_residuals."""
        res = np.zeros((2, self.H, self.W), np.int8)
        err = np.zeros((2, self.H, self.W), np.float32)
        vert = np.zeros((self.H, self.W, 3), np.float32)
        lab = np.zeros((self.H, self.W), np.int32)
        self._check(self.lib.mf_motion_download(self.h, _ptr(res, np.int8), _ptr(err, np.float32),
                                                _ptr(vert, np.float32), _ptr(lab, np.int32)))
        return res, err, vert, lab

    def track_results(self, i, d_ptr, d_err=None):
        """Result codes of instance i's last level-0 GN rows into device
        memory at d_ptr (2 * H * W int8), errors at d_err (2 * H * W float,
        optional); returns the pose they were evaluated at."""
        pose = np.zeros(16, np.float32)
        self._check(self.lib.mf_track_results(self.h, int(i), C.c_void_p(d_ptr),
                                              C.c_void_p(d_err) if d_err else None,
                                              _ptr(pose, np.float32)))
        return pose.reshape(4, 4)

    def object_residuals(self, i, d_ptr, threshold=1.5):
        """Object i's result rows recomputed at its virtual camera pose
        (kfusion.cpp:446-466) into device memory at d_ptr (2 * H * W int8);
        returns the virtual pose."""
        pose = np.zeros(16, np.float32)
        self._check(self.lib.mf_object_residuals(self.h, int(i), C.c_float(threshold),
                                                 C.c_void_p(d_ptr), _ptr(pose, np.float32)))
        return pose.reshape(4, 4)

    def upload_raw(self, depth_mm=None, rgb=None):
        """A sensor frame (uint16 mm depth, uint8 rgb) of an integer multiple of
        the frame size (mf_frame_upload_raw)."""
        d = None if depth_mm is None else np.ascontiguousarray(depth_mm, np.uint16)
        r = None if rgb is None else np.ascontiguousarray(rgb, np.uint8)
        h, w = (d if d is not None else r).shape[:2]
        self._check(self.lib.mf_frame_upload_raw(self.h, _ptr(d, np.uint16), _ptr(r, np.uint8),
                                                 int(w), int(h)))

    def mesh(self, i, float_bounds=False):
        """(n, 3, 3) float32 marching-cubes triangles of instance i (mf_mesh)."""
        n = C.c_longlong()
        fb = int(float_bounds)
        self._check(self.lib.mf_mesh(self.h, int(i), fb, None, 0, C.byref(n)))
        out = np.zeros((max(n.value, 1), 3, 3), np.float32)
        self._check(self.lib.mf_mesh(self.h, int(i), fb, _ptr(out, np.float32), n.value,
                                     C.byref(n)))
        return out[:n.value]

    def set_triangle_table(self, table=None):
        """The marching-cubes triangle table for mf_mesh (256 x 16 ints, -1
        ended), or None for the built-in one."""
        if table is None:
            self._check(self.lib.mf_mesh_set_triangle_table(self.h, None))
            return
        t = np.ascontiguousarray(table, np.int32).reshape(256, 16)
        self._check(self.lib.mf_mesh_set_triangle_table(self.h, _ptr(t, np.int32)))

    def dump_mesh(self, prefix):
        self._check(self.lib.mf_dump_mesh(self.h, str(prefix).encode()))

    def save_poses(self, prefix, frame):
        self._check(self.lib.mf_save_poses(self.h, str(prefix).encode(), int(frame)))

    # ---------------------------------------------------------------- objects
    def spawn_object(self, mask):
        """(T_w_o, volume_size, volume_resol, n_pixels) of mf_spawn_object."""
        m = np.ascontiguousarray(mask, np.uint8)
        T = np.zeros(16, np.float32)
        size, resol, n = C.c_float(), C.c_int(), C.c_int()
        self._check(self.lib.mf_spawn_object(self.h, _ptr(m, np.uint8), _ptr(T, np.float32),
                                             C.byref(size), C.byref(resol), C.byref(n)))
        return T.reshape(4, 4), size.value, resol.value, n.value

    def set_semantics(self, i, class_id, probs):
        p = np.ascontiguousarray(probs, np.float32)
        self._check(self.lib.mf_instance_set_semantics(self.h, int(i), int(class_id),
                                                       _ptr(p, np.float32), p.size))

    def fuse_semantics(self, i, class_id, probs, recog_times=1):
        p = np.ascontiguousarray(probs, np.float32)
        self._check(self.lib.mf_fuse_semantics(self.h, int(i), int(class_id), _ptr(p, np.float32),
                                               p.size, int(recog_times)))

    def semantics(self, i, n=80):
        """(class id, fused count, fused probabilities)."""
        cid, ft = C.c_int(), C.c_int()
        p = np.zeros(n, np.float32)
        self._check(self.lib.mf_instance_semantics(self.h, int(i), C.byref(cid), C.byref(ft),
                                                   _ptr(p, np.float32), n))
        return cid.value, ft.value, p

    # ---------------------------------------------------------------- renders
    def render_volume(self, T_w_c=None, render_color=True, largestep=0.075, ambient=None,
                      colors=None):
        """(H, W, 4) uint8 shaded render (mf_render_volume); T_w_c None shades
        the last raycast's maps."""
        out = np.zeros((self.H, self.W, 4), np.uint8)
        col = None if colors is None else np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        amb = None if ambient is None else np.ascontiguousarray(ambient, np.float32)
        self._check(self.lib.mf_render_volume(
            self.h, None if T_w_c is None else _ptr(_m4(T_w_c), np.float32),
            int(render_color), C.c_float(largestep), _ptr(amb, np.float32),
            _ptr(col, np.uint8), 0 if col is None else len(col), _ptr(out, np.uint8)))
        return out

    def render_image(self, which):
        """which: "depth", "intensity" (H, W, 4) or "normal" (H, W, 3)."""
        out = np.zeros((self.H, self.W, 3 if which == "normal" else 4), np.uint8)
        fn = {"depth": self.lib.mf_render_depth, "intensity": self.lib.mf_render_intensity,
              "normal": self.lib.mf_render_normal}[which]
        self._check(fn(self.h, _ptr(out, np.uint8)))
        return out

    def render_track(self, mode, d_res=None, d_err=None):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        self._check(self.lib.mf_render_track(self.h, int(mode),
                                             C.c_void_p(d_res) if d_res else None,
                                             C.c_void_p(d_err) if d_err else None,
                                             _ptr(out, np.uint8)))
        return out

    def render_mask(self, mode, colors, d_labels=None, d_rows=()):
        out = np.zeros((self.H, self.W, 4), np.uint8)
        col = np.ascontiguousarray(colors, np.uint8).reshape(-1, 4)
        rows = (C.c_void_p * max(len(d_rows), 1))(*[C.c_void_p(p) if p else None
                                                    for p in d_rows])
        self._check(self.lib.mf_render_mask(self.h, int(mode),
                                            C.c_void_p(d_labels) if d_labels else None,
                                            _ptr(col, np.uint8), len(col),
                                            rows if len(d_rows) else None, len(d_rows),
                                            _ptr(out, np.uint8)))
        return out

    def refine_mask_use_motion(self, i, d_ptr=None):
        """Refine instance i's mask with result planes at d_ptr (device), or
        with the last motion_residuals planes."""
        self._check(self.lib.mf_refine_mask_use_motion(self.h, int(i),
                                                       C.c_void_p(d_ptr) if d_ptr else None))

    def mask(self, i):
        out = np.zeros((self.H, self.W), np.float32)
        self._check(self.lib.mf_download_mask(self.h, int(i), _ptr(out, np.float32)))
        return out

    def track_eval_static(self, slot, level, pose=None):
        """mf_track_eval with static device scratch (allocates nothing)."""
        sums = np.zeros(32, np.float64)
        p = None if pose is None else _m4(pose)
        self._check(self.lib.mf_track_eval_static(self.h, slot, level, _ptr(p, np.float32),
                                                  _ptr(sums, np.float64)))
        return sums

    def pyramid(self, level, which):
        w, h = self.W >> level, self.H >> level
        out = np.zeros(w * h * 3, np.float32)
        self._check(self.lib.mf_download_pyramid(self.h, level, which, _ptr(out, np.float32)))
        if which in (2, 3, 6, 7):
            return out.reshape(h, w, 3)
        return out[:w * h].reshape(h, w)

    # ---------------------------------------------------------------- inspection
    def blocks(self, i, with_voxels=True):
        n = C.c_int()
        self._check(self.lib.mf_block_count(self.h, i, C.byref(n)))
        n = n.value
        keys = np.zeros(n, np.uint64)
        coords = np.zeros((n, 3), np.int32)
        active = np.zeros(n, np.uint8)
        vox = np.zeros((n, 512), VOXEL_DTYPE) if with_voxels else None
        m = C.c_int()
        self._check(self.lib.mf_export_blocks(
            self.h, i, _ptr(keys, np.uint64), _ptr(coords, np.int32), _ptr(active, np.uint8),
            None if vox is None else vox.ctypes.data_as(C.c_void_p), n, C.byref(m)))
        order = np.argsort(keys, kind="stable")
        return keys[order], coords[order], active[order], (None if vox is None else vox[order])

    def nodes(self, i, with_values=True):
        n = C.c_int()
        self._check(self.lib.mf_node_count(self.h, i, C.byref(n)))
        n = n.value
        keys = np.zeros(n, np.uint64)
        side = np.zeros(n, np.uint32)
        cm = np.zeros(n, np.uint8)
        vals = np.zeros((n, 8), VOXEL_DTYPE) if with_values else None
        m = C.c_int()
        self._check(self.lib.mf_export_nodes(
            self.h, i, _ptr(keys, np.uint64), _ptr(side, np.uint32), _ptr(cm, np.uint8),
            None if vals is None else vals.ctypes.data_as(C.c_void_p), n, C.byref(m)))
        order = np.argsort(keys, kind="stable")
        return keys[order], side[order], cm[order], (None if vals is None else vals[order])

    def root_children(self, i):
        m = C.c_uint8()
        self._check(self.lib.mf_root_children(self.h, i, C.byref(m)))
        return m.value

    def interp(self, i, pos, field=0):
        pos = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(-1, 3))
        out = np.zeros(len(pos), np.float32)
        self._check(self.lib.mf_interp(self.h, i, _ptr(pos, np.float32), len(pos), field,
                                       _ptr(out, np.float32)))
        return out


class RawReader:
    """The SLAMBench .raw sequence reader of the library (mf_raw_*): host code
    only, usable without a GPU."""

    def __init__(self, path):
        self.lib = load()
        h = C.c_void_p()
        w, hh, n = C.c_int(), C.c_int(), C.c_longlong()
        rc = self.lib.mf_raw_open(str(path).encode(), C.byref(h), C.byref(w), C.byref(hh),
                                  C.byref(n))
        if rc != MF_OK:
            raise MfError(f"{ERRORS.get(rc, rc)} cannot open {path}")
        self.h, self.width, self.height, self.n_frames = h, w.value, hh.value, n.value

    def read(self, frame=-1):
        """(depth uint16 (H, W), rgb uint8 (H, W, 3)), or None past the end."""
        d = np.zeros((self.height, self.width), np.uint16)
        c = np.zeros((self.height, self.width, 3), np.uint8)
        rc = self.lib.mf_raw_read(self.h, C.c_longlong(frame), _ptr(d, np.uint16),
                                  _ptr(c, np.uint8))
        if rc == -4:  # MF_E_NOT_FOUND: past the end
            return None
        if rc != MF_OK:
            raise MfError(f"{ERRORS.get(rc, rc)} reading frame {frame}")
        return d, c

    def close(self):
        if getattr(self, "h", None):
            self.lib.mf_raw_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pose_quaternion(T):
    """(x, y, z, w) of mf_pose_quaternion."""
    q = np.zeros(4, np.float32)
    load().mf_pose_quaternion(_ptr(_m4(T), np.float32), _ptr(q, np.float32))
    return q


def tum_line(frame, T_translation, T_rotation):
    buf = C.create_string_buffer(256)
    n = load().mf_tum_line(int(frame), _ptr(_m4(T_translation), np.float32),
                           _ptr(_m4(T_rotation), np.float32), buf, 256)
    if n < 0:
        raise MfError("mf_tum_line failed")
    return buf.value.decode()


def write_vtk_mesh(path, tris):
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    rc = load().mf_write_vtk_mesh(str(path).encode(), _ptr(t, np.float32), C.c_longlong(len(t)))
    if rc != MF_OK:
        raise MfError(f"{ERRORS.get(rc, rc)} writing {path}")

"""Seeded synthetic RGB-D sequences that stand in for the reference's datasets.

The reference is evaluated on TUM RGB-D / ICL-NUIM / MID-Fusion recordings, none
of which exist on this machine.  These scenes take their frame shapes,
intrinsics and value ranges from the reference's demo configuration
(``-k 525,525,319.5,239.5``; depth in metres after ``mm2metersKernel``,
apps/kfusion/src/cpp/preprocessing/preprocessing.cpp:132-159; RGB uint8) and
render analytic geometry by ray casting in numpy:

* a room (inside of an axis-aligned cube: walls, floor, ceiling),
* static spheres / boxes (part of the background instance 0),
* rigid moving objects (sphere, oriented box, capped cylinder), instance ids 1..K,
  each with its own octree volume centred on it (``spawnNewObjectKernel``,
  apps/kfusion/src/cpp/kfusion.cpp:1155-1159).

Depth noise follows sigma = 0.0012 + 0.0019 (z - 0.4)^2 with 1 % dropouts set to 0.
Albedo is a seeded two-octave value noise.  Everything is deterministic in the
seed.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


# --------------------------------------------------------------------------- math
def skew(w):
    return np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]], dtype=np.float64)


def se3_exp(xi):
    """SE(3) exponential of a twist (v, w), translation first."""
    v = np.asarray(xi[:3], np.float64)
    w = np.asarray(xi[3:], np.float64)
    th = float(np.linalg.norm(w))
    W = skew(w)
    if th < 1e-12:
        R = np.eye(3) + W
        V = np.eye(3) + 0.5 * W
    else:
        A = math.sin(th) / th
        B = (1 - math.cos(th)) / th ** 2
        C = (1 - A) / th ** 2
        R = np.eye(3) + A * W + B * W @ W
        V = np.eye(3) + B * W + C * W @ W
    T = np.eye(4)
    T[:3, :3] = R
    T[:3, 3] = V @ v
    return T


def rot_axis(axis, ang):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    return se3_exp(np.concatenate([np.zeros(3), a * ang]))[:3, :3]


def look_at(eye, target, up=(0.0, -1.0, 0.0)):
    """Camera-to-world pose: camera z forward, x right, y down."""
    eye = np.asarray(eye, np.float64)
    z = np.asarray(target, np.float64) - eye
    z /= np.linalg.norm(z)
    x = np.cross(np.asarray(up, np.float64) * -1.0, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    T = np.eye(4)
    T[:3, 0], T[:3, 1], T[:3, 2], T[:3, 3] = x, y, z, eye
    return T


# --------------------------------------------------------------------------- noise
class ValueNoise:
    """Seeded 3-D value noise, two octaves, per-channel lattices."""

    def __init__(self, rng, n=64):
        self.n = n
        self.lat = rng.random((3, n, n, n)).astype(np.float32)

    def __call__(self, p, freq=6.0):
        out = np.zeros(p.shape[:-1] + (3,), np.float32)
        for octave, amp in ((1.0, 0.65), (2.0, 0.35)):
            q = p * (freq * octave)
            i0 = np.floor(q).astype(np.int64)
            f = (q - i0).astype(np.float32)
            f = f * f * (3 - 2 * f)
            acc = 0
            for dz in (0, 1):
                for dy in (0, 1):
                    for dx in (0, 1):
                        ix = (i0[..., 0] + dx) % self.n
                        iy = (i0[..., 1] + dy) % self.n
                        iz = (i0[..., 2] + dz) % self.n
                        w = ((f[..., 0] if dx else 1 - f[..., 0]) *
                             (f[..., 1] if dy else 1 - f[..., 1]) *
                             (f[..., 2] if dz else 1 - f[..., 2]))
                        acc = acc + w[..., None] * self.lat[:, ix, iy, iz].transpose(
                            *range(1, ix.ndim + 1), 0)
            out += amp * acc
        return out


# --------------------------------------------------------------------------- shapes
@dataclasses.dataclass
class Shape:
    kind: str            # 'sphere' | 'box' | 'cylinder'
    size: tuple          # sphere (r,), box (sx, sy, sz) full sides, cylinder (r, h)
    pose: np.ndarray     # shape-to-world 4x4 at frame 0
    tint: np.ndarray     # rgb tint in [0,1]
    label: int = 0       # 0: part of the background instance
    twist: np.ndarray = None  # per-frame body twist (moving objects)
    sway: float = 0.0    # > 0: the motion swings back and forth with this period (frames)

    def pose_at(self, f):
        if self.twist is None:
            return self.pose
        if self.sway > 0:  # peak speed `twist` per frame, bounded excursion
            t = self.sway / (2 * math.pi) * math.sin(2 * math.pi * f / self.sway)
            return self.pose @ se3_exp(self.twist * t)
        return self.pose @ se3_exp(self.twist * f)

    def half_extent(self):
        if self.kind == "sphere":
            return self.size[0]
        if self.kind == "box":
            return 0.5 * float(np.linalg.norm(self.size))
        r, h = self.size
        return float(math.hypot(r, 0.5 * h))


def _intersect_local(kind, size, o, d):
    """Ray/primitive intersection in the shape frame.  Returns (t, n_local)."""
    n_rays = o.shape[0]
    t = np.full(n_rays, np.inf)
    nrm = np.zeros((n_rays, 3))
    if kind == "sphere":
        r = size[0]
        a = np.einsum("ij,ij->i", d, d)
        b = np.einsum("ij,ij->i", o, d)
        c = np.einsum("ij,ij->i", o, o) - r * r
        disc = b * b - a * c
        ok = disc >= 0
        s = np.sqrt(np.where(ok, disc, 0))
        t0 = (-b - s) / a
        hit = ok & (t0 > 1e-6)
        t[hit] = t0[hit]
        p = o + t[:, None] * d
        nrm[hit] = p[hit] / r
    elif kind == "box":
        h = 0.5 * np.asarray(size, np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / d
            t1 = (-h - o) * inv
            t2 = (h - o) * inv
        tmin = np.minimum(t1, t2)
        tmax = np.maximum(t1, t2)
        tn = tmin.max(axis=1)
        tf = tmax.min(axis=1)
        hit = (tn <= tf) & (tn > 1e-6)
        t[hit] = tn[hit]
        ax = tmin.argmax(axis=1)
        sgn = -np.sign(d[np.arange(n_rays), ax])
        nrm[np.arange(n_rays), ax] = sgn
        nrm[~hit] = 0
    else:  # capped cylinder, axis = local y
        r, hh = size[0], 0.5 * size[1]
        a = d[:, 0] ** 2 + d[:, 2] ** 2
        b = o[:, 0] * d[:, 0] + o[:, 2] * d[:, 2]
        c = o[:, 0] ** 2 + o[:, 2] ** 2 - r * r
        disc = b * b - a * c
        ok = (disc >= 0) & (a > 1e-12)
        s = np.sqrt(np.where(ok, disc, 0))
        with np.errstate(divide="ignore", invalid="ignore"):
            ts = np.where(ok, (-b - s) / np.where(a > 1e-12, a, 1), np.inf)
        ys = o[:, 1] + ts * d[:, 1]
        side = ok & (ts > 1e-6) & (np.abs(ys) <= hh)
        t = np.where(side, ts, np.inf)
        with np.errstate(divide="ignore", invalid="ignore"):
            for cap in (-hh, hh):
                tc = (cap - o[:, 1]) / d[:, 1]
                pc = o + tc[:, None] * d
                okc = (tc > 1e-6) & (pc[:, 0] ** 2 + pc[:, 2] ** 2 <= r * r) & (tc < t)
                t = np.where(okc, tc, t)
                nrm[okc] = np.array([0, np.sign(cap), 0])
        p = o + np.where(np.isfinite(t), t, 0)[:, None] * d
        nrm[side & (t == ts)] = np.stack([p[:, 0], np.zeros(n_rays), p[:, 2]], 1)[side & (t == ts)] / r
    return t, nrm


# --------------------------------------------------------------------------- scene
@dataclasses.dataclass
class Instance:
    """One octree volume: background (label 0) or a moving object."""
    label: int
    size: int           # voxels per side
    dim: float          # metres per side
    shape: Shape = None  # None for the background

    def volume_pose(self, f, bg_pose):
        if self.shape is None:
            return bg_pose.copy()
        T = self.shape.pose_at(f).copy()
        corner = np.eye(4)
        corner[:3, 3] = -0.5 * self.dim
        return T @ corner


class Scene:
    def __init__(self, width, height, k, room_lo, room_hi, statics, movers, instances,
                 cam_poses, seed, noise=True):
        self.width, self.height = width, height
        self.k = np.asarray(k, np.float32)
        self.room_lo = np.asarray(room_lo, np.float64)
        self.room_hi = np.asarray(room_hi, np.float64)
        self.statics, self.movers = statics, movers
        self.instances = instances
        self.cam_poses = cam_poses
        self.seed = seed
        self.noise = noise
        rng = np.random.default_rng(seed + 1)
        self.albedo = ValueNoise(rng)
        self.bg_pose = np.eye(4)

    @property
    def n_frames(self):
        return len(self.cam_poses)

    def volume_poses(self, f):
        return [inst.volume_pose(f, self.bg_pose) for inst in self.instances]

    def render(self, f):
        """Returns depth f32 [H,W] (m), rgb u8 [H,W,3], labels u16 [H,W]."""
        W, H = self.width, self.height
        fx, fy, cx, cy = [float(v) for v in self.k]
        T = self.cam_poses[f]
        xs, ys = np.meshgrid(np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
        dc = np.stack([(xs - cx) / fx, (ys - cy) / fy, np.ones_like(xs)], -1).reshape(-1, 3)
        o = np.broadcast_to(T[:3, 3], dc.shape).copy()
        dw = dc @ T[:3, :3].T
        # room: exit distance of the inner box
        with np.errstate(divide="ignore", invalid="ignore"):
            bound = np.where(dw > 0, self.room_hi, self.room_lo)
            tt = (bound - o) / dw
        tt = np.where(np.isfinite(tt) & (tt > 0), tt, np.inf)
        t_best = tt.min(axis=1)
        ax = tt.argmin(axis=1)
        n_best = np.zeros_like(dw)
        n_best[np.arange(len(ax)), ax] = -np.sign(dw[np.arange(len(ax)), ax])
        label = np.zeros(len(t_best), np.uint16)
        tint = np.tile(np.array([0.8, 0.78, 0.72]), (len(t_best), 1))
        for sh in list(self.statics) + list(self.movers):
            P = sh.pose_at(f)
            R, tv = P[:3, :3], P[:3, 3]
            ol = (o - tv) @ R
            dl = dw @ R
            t, nl = _intersect_local(sh.kind, sh.size, ol, dl)
            closer = t < t_best
            t_best = np.where(closer, t, t_best)
            n_best[closer] = (nl @ R.T)[closer]
            label[closer] = sh.label
            tint[closer] = sh.tint
        p = o + np.where(np.isfinite(t_best), t_best, 0)[:, None] * dw
        depth = np.where(np.isfinite(t_best), t_best, 0.0)  # dc has z = 1: t is the z-depth
        alb = self.albedo(p.astype(np.float32))
        light = np.array([0.3, -0.8, -0.5])
        light /= np.linalg.norm(light)
        shade = 0.55 + 0.45 * np.abs(n_best @ light)
        rgb = np.clip(alb * tint * shade[:, None] * 1.15, 0, 1)
        rgb = (rgb * 255 + 0.5).astype(np.uint8).reshape(H, W, 3)
        depth = depth.reshape(H, W)
        if self.noise:
            rng = np.random.default_rng(self.seed * 1000 + f)
            sigma = 0.0012 + 0.0019 * (depth - 0.4) ** 2
            depth = depth + rng.standard_normal(depth.shape) * sigma
            drop = rng.random(depth.shape) < 0.01
            depth[drop] = 0.0
        depth[depth < 0] = 0
        return depth.astype(np.float32), rgb, label.reshape(H, W)


def generalize_masks(labels, instance_labels):
    """Per-instance float masks as instance_seg::generalize_label builds them for
    ground-truth (not rendered) masks, apps/kfusion/src/cpp/segmentation/
    segmentation.cpp:10-48: 1 inside the instance, 0 on the ring added by a 5x5
    elliptic dilation (cv::MORPH_ELLIPSE), -1 elsewhere."""
    H, W = labels.shape
    ell = np.array([[0, 0, 1, 0, 0], [1, 1, 1, 1, 1], [1, 1, 1, 1, 1], [1, 1, 1, 1, 1],
                    [0, 0, 1, 0, 0]], bool)
    out = np.empty((len(instance_labels), H, W), np.float32)
    for i, lab in enumerate(instance_labels):
        m = labels == lab
        pad = np.zeros((H + 4, W + 4), bool)
        pad[2:-2, 2:-2] = m
        dil = np.zeros_like(m)
        for dy in range(5):
            for dx in range(5):
                if ell[dy, dx]:
                    dil |= pad[dy:dy + H, dx:dx + W]
        g = np.full((H, W), -1.0, np.float32)
        g[dil] = 0.0
        g[m] = 1.0
        out[i] = g
    return out


# --------------------------------------------------------------------------- presets
def _smooth_path(rng, n, base, target, max_step=0.009, max_rot_deg=0.9, period=0.0):
    """One closed loop over the n frames (or, with period > 0, a loop every
    `period` frames) of at most max_step per frame."""
    per = period if period > 0 else n
    amp = rng.uniform(0.5, 1.0, 3) * max_step * per / (2 * math.pi) * 0.9
    ph = rng.uniform(0, 2 * math.pi, 3)
    poses = []
    for f in range(n):
        s = f / max(per, 1) * 2 * math.pi
        eye = np.asarray(base) + amp * (np.sin(s + ph) - np.sin(ph))
        T = look_at(eye, target)
        ang = math.radians(max_rot_deg) * 0.3 * math.sin(0.7 * f + ph[0]) * min(f, 5) / 5
        R = rot_axis([0, 0, 1], ang)
        T[:3, :3] = T[:3, :3] @ R
        poses.append(T)
    return poses


def make_scene(preset="multi", width=640, height=480, n_frames=100, seed=1, n_objects=3,
               bg_size=512, bg_dim=5.12, obj_size=256, obj_dim=0.512, noise=True, sway=0.0):
    """``preset='room'``: one static room (plain method, one octree).
    ``preset='multi'``: background room + moving rigid objects, one octree each.
    ``preset='uneven'``: background room + ``n_objects`` (default use: 12) rigid
    primitives of seeded kinds and sizes (0.05-0.4 m), each with its own octree
    of 32^3, 64^3, 128^3 or 256^3 voxels at 2-5 mm; the largest object sits in
    the centre, the others on an ellipse around it, at depths chosen so that
    their mask areas span about 0.5 %-25 % of the frame.  ``sway`` > 0 (frames,
    'uneven' only): each object swings along its twist with that period
    instead of moving at a constant twist, and the camera loops with that
    period, so that long sequences keep the objects in view."""
    rng = np.random.default_rng(seed)
    scale = width / 640.0
    k = (525.0 * scale, 525.0 * scale, (width - 1) / 2.0, (height - 1) / 2.0)
    # room of 3.2 m centred in the background volume
    c = 0.5 * bg_dim
    lo = np.array([c - 1.6, c - 1.6, c - 1.6])
    hi = lo + 3.2
    statics = []
    for i in range(4):
        p = np.eye(4)
        p[:3, 3] = [rng.uniform(lo[0] + 0.5, hi[0] - 0.5), hi[1] - rng.uniform(0.1, 0.4),
                    rng.uniform(c + 0.3, hi[2] - 0.4)]
        r = rng.uniform(0.1, 0.4)
        p[1, 3] = hi[1] - r
        statics.append(Shape("sphere", (r,), p, rng.uniform(0.4, 1.0, 3)))
    for i in range(3):
        p = np.eye(4)
        side = rng.uniform(0.2, 0.6)
        p[:3, :3] = rot_axis([0, 1, 0], rng.uniform(0, math.pi))
        p[:3, 3] = [rng.uniform(lo[0] + 0.5, hi[0] - 0.5), hi[1] - 0.5 * side,
                    rng.uniform(c + 0.3, hi[2] - 0.4)]
        statics.append(Shape("box", (side, side, side), p, rng.uniform(0.4, 1.0, 3)))
    eye = np.array([c, c + 0.3, lo[2] + 0.7])
    target = np.array([c, c + 0.5, hi[2]])
    cams = _smooth_path(rng, n_frames, eye, target, period=sway if preset == "uneven" else 0.0)
    instances = [Instance(0, bg_size, bg_dim)]
    movers = []
    if preset == "multi":
        kinds = [("sphere", (0.12,)), ("box", (0.2, 0.1, 0.3)), ("cylinder", (0.06, 0.25))]
        for i in range(n_objects):
            kind, size = kinds[i % 3]
            p = np.eye(4)
            p[:3, :3] = rot_axis(rng.normal(size=3), rng.uniform(0, math.pi))
            ang = 2 * math.pi * (i + 0.5) / max(n_objects, 1)
            p[:3, 3] = eye + np.array([0.35 * math.cos(ang), 0.25 * math.sin(ang) + 0.2,
                                       1.1 + 0.15 * (i % 3)])
            tw = np.concatenate([rng.uniform(-1, 1, 3) * 0.004, rng.uniform(-1, 1, 3) *
                                 math.radians(0.6)])
            sh = Shape(kind, size, p, rng.uniform(0.3, 1.0, 3), label=i + 1, twist=tw)
            movers.append(sh)
            instances.append(Instance(i + 1, obj_size, obj_dim, sh))
    elif preset == "uneven":
        cam0 = cams[0]
        fpx = k[0]
        # object extents log-uniform over 0.05-0.4 m (largest first) and target
        # mask areas log-uniform over 0.5-15 %, the largest object 25 % in the
        # centre; the depth follows from extent and area
        extents = np.sort(np.exp(rng.uniform(np.log(0.05), np.log(0.4), n_objects)))[::-1]
        extents[0], extents[-1] = 0.4, 0.05
        areas = np.exp(rng.uniform(np.log(0.005), np.log(0.15), n_objects))
        areas[0] = 0.4  # of the bounding square: about 25 % for a box or sphere
        for i in range(n_objects):
            kind = ("sphere", "box", "cylinder")[int(rng.integers(3))]
            extent = float(extents[i])
            z = float(np.clip(extent * fpx / math.sqrt(areas[i] * width * height), 0.5, 3.0))
            if i == 0:
                x = y = 0.0
            else:  # on an ellipse around the central object
                ang = 2 * math.pi * (i - 1) / max(n_objects - 1, 1) + 0.3
                x = 0.45 * math.cos(ang) * z
                y = 0.33 * math.sin(ang) * z
            if kind == "sphere":
                size = (0.5 * extent,)
            elif kind == "box":
                size = tuple(extent * rng.uniform(0.6, 1.0, 3))
            else:
                size = (0.3 * extent, extent)
            # The volume is centred on the object with a margin (as
            # spawnNewObjectKernel sizes it): the smallest octree of 32^3 ...
            # 256^3 whose 5 mm voxels span twice the object's extent plus 6 cm,
            # sometimes the next finer one, at a voxel of 2-5 mm.  Without the
            # margin the volume corner lies in front of the object and takes
            # its foreground probability, and a raycast miss (which the
            # reference samples at the volume corner) would claim the pixel.
            need = 2.0 * extent + 0.06
            octree = next((o for o in (32, 64, 128, 256) if o * 0.005 >= need), 256)
            if octree < 256 and rng.random() < 0.3:
                octree *= 2
            voxel = float(np.clip(need / octree, 0.002, 0.005))
            dim = octree * voxel
            p = np.eye(4)
            p[:3, :3] = rot_axis(rng.normal(size=3), rng.uniform(0, math.pi))
            p[:3, 3] = (cam0 @ np.array([x, y, z, 1.0]))[:3]
            tw = np.concatenate([rng.uniform(-1, 1, 3) * 0.004, rng.uniform(-1, 1, 3) *
                                 math.radians(0.6)])
            sh = Shape(kind, size, p, rng.uniform(0.3, 1.0, 3), label=i + 1, twist=tw,
                       sway=sway)
            movers.append(sh)
            instances.append(Instance(i + 1, octree, dim, sh))
    return Scene(width, height, k, lo, hi, statics, movers, instances, cams, seed, noise)

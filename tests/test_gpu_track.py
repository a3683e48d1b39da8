"""Tracking on the GPU against the CPU oracle.

* Pyramid (bilateral filter, robust half-sampling, vertex / normal / gradient /
  ICP-covariance maps) against the FP32 oracle: the bilateral weights call the
  host's expf, which the device restates as the double exp rounded to float;
  the two differ where the host's expf misses the nearest float, so depth,
  intensity and vertex are bit-equal at >= 99.5 % of the pixels, all values
  within a few float ulps and the validity masks exactly.
* Normal equations (the 32 reduceKernel sums) at fixed poses against the
  all-FP64 oracle: the GPU evaluates residuals in FP32, sums at most four rows
  per thread in FP32 and reduces in FP64 from the warp level up, so sums agree
  to ~1e-5 relative and the inlier count exactly up to
  a handful of threshold flips.
* Full coarse-to-fine Gauss-Newton (camera and objects, batched device GN and
  the host-driven plain path) against the reference (the FP32 oracle) and the
  all-FP64 oracle from the same starting pose (tests/_pose.py: within 1e-5 m /
  rad of both, widened by twice the reference's own distance to FP64, or a
  decision flip of the cost test whose result is as good a minimizer).
"""
import numpy as np
import pytest

import _oracle as O
from _pose import camera_cost, check_pose, object_cost
from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.gpu

W, H = 320, 240


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


class Pipeline:
    """GPU context and FP64 oracle tracker fed the same frames."""

    def __init__(self, seed=5, batched=True, robust="huber", n_objects=2):
        self.s = make_scene("multi", W, H, n_frames=4, seed=seed, bg_size=256, obj_size=64,
                            n_objects=n_objects)
        s = self.s
        self.ctx = Context(W, H, k=s.k, pool_blocks=1 << 14, batched=batched, robust=robust)
        for inst, T in zip(s.instances, s.volume_poses(0)):
            self.ctx.add_instance(inst.size, inst.dim, T, inst.label)
        self.labels = [i.label for i in s.instances]
        self.trk = O.Tracker(W, H, s.k, robust=O_ROBUST[robust], fp64=True)
        self.trk32 = O.Tracker(W, H, s.k, robust=O_ROBUST[robust], fp64=False)

    def frame0(self):
        s, ctx = self.s, self.ctx
        d, rgb, lab = s.render(0)
        ctx.set_camera_pose(s.cam_poses[0])
        ctx.upload(d, rgb, generalize_masks(lab, self.labels))
        ctx.integrate(list(range(len(self.labels))))
        ctx.raycast()
        ctx.preprocess()
        ctx.set_ref_from_current()
        for t in (self.trk, self.trk32):
            t.set_frame(rgb, d)
            t.set_ref()
        self.model = ctx.download_raycast()

    def frame1(self):
        s, ctx = self.s, self.ctx
        d, rgb, lab = s.render(1)
        ctx.upload(d, rgb, generalize_masks(lab, self.labels))
        ctx.preprocess()
        for t in (self.trk, self.trk32):
            t.set_frame(rgb, d)
        return d, rgb


O_ROBUST = {"none": 0, "huber": 1, "tukey": 2, "cauchy": 3}


def test_pyramid_matches_oracle():
    p = Pipeline()
    p.frame0()
    p.frame1()
    for l in range(3):
        for which, name in ((0, "depth"), (1, "intensity"), (2, "vertex"), (4, "gradx"),
                            (5, "grady"), (6, "cov")):
            g = p.ctx.pyramid(l, which)
            o = p.trk32.level(l, which)
            assert np.array_equal(g == 0, o == 0), f"{name} L{l}: zero pattern differs"
            np.testing.assert_allclose(g, o, rtol=2e-5, atol=1e-6, err_msg=f"{name} L{l}")
            # the reference's arithmetic bit for bit except where the host's expf
            # (bilateral range weights) misses the nearest float
            if which in (0, 1, 2):
                same = float(np.mean(g.view(np.int32) == o.view(np.int32)))
                assert same >= 0.995, f"{name} L{l}: {same:.5f} of the values bit-equal"
        gn = p.ctx.pyramid(l, 3)
        on = p.trk32.level(l, 3)
        inv_g, inv_o = gn[..., 0] == -2, on[..., 0] == -2
        assert np.array_equal(inv_g, inv_o), f"invalid normals differ at L{l}"
        # normals difference neighbouring vertices, which amplifies ulp-level depth
        # differences of the bilateral filter by ~1e3
        np.testing.assert_allclose(gn[~inv_g], on[~inv_o], rtol=0, atol=3e-4)


def _perturb(T, rng, t=0.003, r=0.003):
    from mid_fusion_b200.scene import se3_exp
    xi = np.concatenate([rng.normal(size=3) * t, rng.normal(size=3) * r])
    return (se3_exp(xi) @ T.astype(np.float64)).astype(np.float32)


@pytest.mark.parametrize("level", [0, 1, 2])
def test_normal_equations_match_fp64_oracle(level):
    p = Pipeline()
    p.frame0()
    p.frame1()
    v, n, lab = p.model
    T_w_r = p.s.cam_poses[0].astype(np.float32)
    rng = np.random.default_rng(level)
    p.ctx.set_camera_pose(T_w_r)
    p.ctx.track_camera()  # sets up the camera problem (T_w_r, rendered reference)
    poses = [p.s.cam_poses[1].astype(np.float32)] + [_perturb(p.s.cam_poses[1], rng)
                                                     for _ in range(2)]
    for pose in poses:
        g = p.ctx.track_eval(0, level, pose)
        o = p.trk.camera_sums(level, pose, T_w_r, v, n)
        assert abs(g[28] - o[28]) <= max(3, 2e-4 * o[28]), (g[28], o[28])
        assert np.all(np.abs(g[29:32] - o[29:32]) <= np.maximum(3, 1e-3 * o[29:32]))
        scale = np.abs(o[:28]).max()
        np.testing.assert_allclose(g[:28], o[:28], rtol=2e-3, atol=2e-4 * scale)


def test_normal_equations_at_reference_pose_match_fp32_oracle():
    """At T_w_l == T_w_r every live pixel projects onto an integer model pixel,
    so the nearest-pixel correspondence (uint truncation, tracking.cpp:982)
    depends on the last bit of the projection: the GPU follows the reference's
    single-precision arithmetic (the FP32 oracle), not the FP64 oracle."""
    p = Pipeline()
    p.frame0()
    p.frame1()
    v, n, lab = p.model
    T_w_r = p.s.cam_poses[0].astype(np.float32)
    p.ctx.set_camera_pose(T_w_r)
    p.ctx.track_camera()
    for level in range(3):
        g = p.ctx.track_eval(0, level, T_w_r)
        o = p.trk32.camera_sums(level, T_w_r, T_w_r, v, n)
        assert abs(g[28] - o[28]) <= max(3, 2e-4 * o[28]), (level, g[28], o[28])


@pytest.mark.parametrize("batched", [True, False])
def test_track_camera_matches_fp64_oracle(batched):
    p = Pipeline(batched=batched)
    p.frame0()
    p.frame1()
    v, n, lab = p.model
    T0 = p.s.cam_poses[0].astype(np.float32)
    p.ctx.track_camera()
    it, sums, T_gpu = p.ctx.track_info(0)
    T_or = p.trk.track_camera(T0, T0, v, n)
    it_or = p.trk.iterations()
    T_32 = p.trk32.track_camera(T0, T0, v, n)
    it_32 = p.trk32.iterations()
    ok = check_pose(T_gpu, T_32, T_or, "camera", cost=camera_cost(p.trk, T0, v, n))
    if ok and it_32 == it_or:
        assert list(it[:3]) == it_or, (list(it[:3]), it_or)
    # the float pose handed back to the pipeline is the FP64 result rounded
    np.testing.assert_allclose(p.ctx.camera_pose(), T_gpu.astype(np.float32), atol=1e-6)


@pytest.mark.parametrize("batched", [True, False])
def test_track_objects_matches_fp64_oracle(batched):
    p = Pipeline(batched=batched)
    p.frame0()
    p.frame1()
    v, n, lab = p.model
    s = p.s
    T0, T1 = s.cam_poses[0].astype(np.float32), s.cam_poses[1].astype(np.float32)
    # camera at ground truth for frame 1; objects tracked from their frame-0 poses
    p.ctx.set_camera_pose(T1)
    ids = list(range(1, len(s.instances)))
    p.ctx.track_objects(ids)
    for i in ids:
        T_wo1 = s.volume_poses(0)[i].astype(np.float32)
        label = s.instances[i].label
        T_or = p.trk.track_object(T_wo1, T1, T0, v, n, lab, label)
        it_or = p.trk.iterations()
        T_32 = p.trk32.track_object(T_wo1, T1, T0, v, n, lab, label)
        it_32 = p.trk32.iterations()
        it, sums, T_c2o2 = p.ctx.track_info(i)
        T_gpu = T1.astype(np.float64) @ T_c2o2
        ok = check_pose(T_gpu, T_32, T_or, f"object {i}",
                        cost=object_cost(p.trk, T_wo1, T1, T0, v, n, lab, label))
        if ok and it_32 == it_or:
            assert list(it[:3]) == it_or, (i, list(it[:3]), it_or)

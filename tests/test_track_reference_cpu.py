"""The tracking oracle against the reference's own tracking code (CPU only;
skipped where oracle/_ref was not built, e.g. without the reference tree).

oracle/_ref/libmf_ref_track.so is the reference's tracking.cpp,
preprocessing.cpp and object.cpp compiled unmodified (serial, no fused
multiply-add) against the project's TooN / Eigen / OpenCV stand-ins
(oracle/shim/).  The single-precision restatement (oracle/or_track.cpp, the
oracle the GPU tests use) must equal it bit for bit:

* the pyramid: bilateral-filtered depth and intensity, robust half-samples,
  vertex / normal / gradient / ICP-covariance maps at every level
  (Tracking::set_params_frame, tracking.cpp:142-171, 776-871;
  preprocessing.cpp:11-309);
* camera tracking, Tracking::trackLiveFrame (tracking.cpp:208-357) and its
  masked overload (:1750-1879): the final pose and every level's last sums;
* object tracking, Tracking::trackEachObject (tracking.cpp:580-708), with the
  reference's per-object model maps built from the composite maps as
  raycastObjectList writes them (rendering.cpp:152-176);
* motion residuals, Tracking::compute_residuals (tracking.cpp:1535-1747):
  every row code, and the error of every valid row (a rejected row keeps
  whatever the buffer held before, in the reference);
* Object::refine_mask_use_motion, set_static_state with the never-moving
  class list, fuseSemanticLabel (object.cpp:222-325).

The FP64 oracle's distance to the reference is printed for the record: it is
the reference's own single-precision rounding, not a discrepancy of the
restatement.
"""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200.scene import generalize_masks, make_scene

pytestmark = pytest.mark.skipif(O.reference_tracking() is None,
                                reason="oracle/_ref not built (no reference tree)")

INVALID = -2.0


def _model(s, W, H, f=0):
    """Volumes integrated from frame f at the ground-truth poses and the
    composite raycast (the oracle's volume code, pinned to the reference's)."""
    orc = O.oracle()
    labels = [i.label for i in s.instances]
    vols = [orc.volume(i.size, i.dim) for i in s.instances]
    d, rgb, lab = s.render(f)
    masks = generalize_masks(lab, labels)
    T = s.cam_poses[f].astype(np.float32)
    P = [p.astype(np.float32) for p in s.volume_poses(f)]
    for i, v in enumerate(vols):
        v.integrate(d, rgb.astype(np.float32) / np.float32(255), masks[i], T, P[i], s.k, 0.1)
    vm = np.zeros((H, W, 3), np.float32)
    nm = np.zeros((H, W, 3), np.float32)
    lm = np.zeros((H, W), np.int32)
    orc.raycast_objects(vols, P, labels, T, s.k, W, H, eps_size=s.instances[0].size, vertex=vm,
                        normal=nm, label_img=lm)
    return vols, labels, T, P, vm, nm, lm


def _pair(s, W, H, f0=0, f1=1):
    d0, rgb0, _ = s.render(f0)
    d1, rgb1, _ = s.render(f1)
    R = O.RefTracker(W, H, s.k)
    F = O.Tracker(W, H, s.k, robust=1, fp64=False)
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    return R, F


def _object_maps(vm, nm, lm, label):
    sel = (lm == label)[..., None]
    mv = np.where(sel, vm, np.float32(0)).astype(np.float32)
    mn = np.where(sel, nm, np.array([INVALID, 0, 0], np.float32)).astype(np.float32)
    return mv, mn


def _sums(F, level):
    out = np.zeros(32, np.float64)
    F.lib.ot_last_sums(F.h, level, out)
    return out.astype(np.float32)


def test_pyramid_matches_reference():
    W, H = 320, 240
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    R, F = _pair(s, W, H)
    for level in range(3):
        for which in range(7):  # depth, intensity, vertex, normal, gx, gy, ICP covariance
            a, b = R.level(level, which), F.level(level, which)
            assert np.array_equal(a, b), (level, which)


@pytest.mark.parametrize("W,H,seed", [(320, 240, 5), (320, 240, 9), (160, 120, 2), (640, 480, 4)])
def test_camera_tracking_matches_reference(W, H, seed):
    s = make_scene("room", W, H, n_frames=2, seed=seed, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    R, F = _pair(s, W, H)
    D = O.Tracker(W, H, s.k, robust=1, fp64=True)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    D.set_frame(rgb0, d0)
    D.set_ref()
    D.set_frame(rgb1, d1)
    Tr = R.track_camera(T0, T0, vm, nm)
    Tf = F.track_camera(T0, T0, vm, nm).astype(np.float32)
    assert np.array_equal(Tr, Tf)
    for level in range(3):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level
    # the rendered reference depth / vertex pyramid of trackLiveFrame
    for level in range(3):
        assert np.array_equal(R.level(level, 7), F.level(level, 7)), level
    Td = D.track_camera(T0, T0, vm, nm)
    print(f"reference vs all-FP64 oracle: {np.abs(Td - Tr).max():.3g}")


def test_masked_camera_tracking_matches_reference():
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    _, labels, T0, _, vm, nm, lm = _model(s, W, H)
    R, F = _pair(s, W, H)
    mask = (np.isin(lm, labels[1:]) * 255).astype(np.uint8)
    Tr = R.track_camera(T0, T0, vm, nm, mask=mask)
    F.set_mask(mask)
    Tf = F.track_camera(T0, T0, vm, nm).astype(np.float32)
    assert np.array_equal(Tr, Tf)
    for level in range(3):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level


@pytest.mark.parametrize("preset", ["multi", "uneven", "headline"])
def test_object_tracking_matches_reference(preset):
    W, H = 320, 240
    if preset == "multi":
        s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    elif preset == "uneven":  # 12 objects, octrees 32^3 .. 256^3 at 2-5 mm
        s = make_scene("uneven", W, H, n_frames=2, seed=23, n_objects=12)
    else:  # the bench workload: 640x480, background 512^3 @ 1 cm + 3 objects 256^3 @ 2 mm
        W, H = 640, 480
        s = make_scene("multi", W, H, n_frames=2, seed=11, n_objects=3, bg_size=512,
                       bg_dim=5.12, obj_size=256, obj_dim=0.512)
    _, labels, T0, P0, vm, nm, lm = _model(s, W, H)
    R, F = _pair(s, W, H)
    Tc = R.track_camera(T0, T0, vm, nm)
    assert np.array_equal(Tc, F.track_camera(T0, T0, vm, nm).astype(np.float32))
    tracked = 0
    for i, label in enumerate(labels[1:], 1):
        mv, mn = _object_maps(vm, nm, lm, label)
        ob = R.object(P0[i], mv, mn)
        To_r, Tv_r = R.track_object(ob, Tc, T0)
        To_f = F.track_object(P0[i], Tc, T0, vm, nm, lm, label).astype(np.float32)
        assert np.array_equal(To_r, To_f), label
        for level in range(3):
            assert np.array_equal(R.reduction(level), _sums(F, level)), (label, level)
        tracked += int((lm == label).sum() > 0)
    assert tracked >= 3


def test_motion_residuals_match_reference():
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    vols, labels, T0, P0, vm, nm, lm = _model(s, W, H)
    R, F = _pair(s, W, H)
    Tc = R.track_camera(T0, T0, vm, nm)
    F.track_camera(T0, T0, vm, nm)
    # the live raycast: current camera pose, last object poses
    orc = O.oracle()
    lv = np.zeros((H, W, 3), np.float32)
    ln = np.zeros((H, W, 3), np.float32)
    ll = np.zeros((H, W), np.int32)
    orc.raycast_objects(vols, P0, labels, Tc, s.k, W, H, eps_size=s.instances[0].size, vertex=lv,
                        normal=ln, label_img=ll)
    res_r, err_r, _ = R.compute_residuals(Tc, T0, vm, nm, lv)
    res_f, err_f = F.motion_residuals(Tc, T0, vm, nm, lv)
    assert np.array_equal(res_r.astype(np.int8), res_f)
    ok = res_r == 1
    assert ok.sum() > 1000 and np.array_equal(err_r[ok], err_f[ok])
    assert len(np.unique(res_r)) >= 5  # valid, and several rejection codes
    # mask refinement of each object from those rows (object.cpp:255-315)
    masks = generalize_masks(s.render(1)[2], labels)
    for i, label in enumerate(labels[1:], 1):
        ob = R.object(P0[i])
        ob.take_results(R)
        for icp, rgb in ((True, True), (True, False), (False, True)):
            a = ob.refine_mask(masks[i], icp, rgb)
            b = O.refine_mask_use_motion(masks[i], res_f, icp, rgb)
            assert np.array_equal(a, b), (label, icp, rgb)


def test_static_state_and_semantic_fusion_match_reference():
    W, H = 32, 24
    R = O.RefTracker(W, H, (26.25, 26.25, 15.5, 11.5))
    # Object::set_static_state ignores a moving verdict for the classes in
    # Object::static_object (object.cpp:317-326): 63, 69, 70.
    for cls in (1, 5, 62, 63, 64, 69, 70, 71):
        ob = R.object(np.eye(4), class_id=cls)
        assert ob.set_static_state(True) is True
        assert ob.set_static_state(False) is (cls in (63, 69, 70)), cls
    rng = np.random.default_rng(4)
    ob = R.object(np.eye(4), class_id=0)
    fused, count = np.zeros(80, np.float32), 1
    for t in range(6):
        p = rng.dirichlet(np.full(80, 0.3)).astype(np.float32)
        p[rng.integers(80)] = 0.7
        rec = int(rng.integers(1, 3))
        cid_r, fused_r = ob.fuse_semantics(p, rec)
        fused, count, cid = O.fuse_semantics(fused, count, p, rec)
        assert cid_r == cid and np.array_equal(fused_r, fused), t


def test_frame_pipeline_matches_reference():
    """Whole frames in a closed loop: the reference's own per-frame code
    (trackLiveFrame masked by the last raycast's object pixels,
    trackEachObject, Object::integrate_volume_kernel, raycastObjectList; the
    serial parity build) against the same flow through the oracle, bit for bit
    over 4 frames."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    import cpu_baseline as CB
    W, H = 160, 120
    s = make_scene("multi", W, H, n_frames=4, seed=1, bg_size=256, obj_size=128)
    frames = [s.render(f) for f in range(4)]
    CB.REF_BUILDS["parity"] = O.REF_TRACK_SO
    a = CB.CpuPipeline(s, use_reference=True, build="parity")
    b = CB.CpuPipeline(s, use_reference=False)
    assert a.kind == "reference" and b.kind == "port"
    for f in range(4):
        a.step(*frames[f])
        b.step(*frames[f])
        assert np.array_equal(a.T, b.T), f
        for pa, pb in zip(a.poses, b.poses):
            assert np.array_equal(pa, pb), f
        assert np.array_equal(a.vertex, b.vertex) and np.array_equal(a.normal, b.normal), f
        assert np.array_equal(a.label_img, b.label_img), f


def test_bench_pose_check_is_zero_on_the_reference_itself():
    """bench.py's per-frame pose check (oracle/cpu_baseline.py pose_check),
    fed the reference pipeline's own poses and model maps as the "device"
    values: re-tracking each frame from the same start reproduces them
    exactly, so every device-vs-reference error is 0."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle"))
    import cpu_baseline as CB
    W, H = 160, 120
    s = make_scene("multi", W, H, n_frames=4, seed=1, bg_size=256, obj_size=128)
    frames = [s.render(f) for f in range(4)]
    CB.REF_BUILDS["parity"] = O.REF_TRACK_SO
    p = CB.CpuPipeline(s, use_reference=True, build="parity")
    cams, objs, maps = [], [], []
    for f in range(4):
        p.step(*frames[f])
        cams.append(p.T.copy())
        objs.append(np.stack(p.poses))
        maps.append((p.vertex.copy(), p.normal.copy(), p.label_img.copy()))
    chk = CB.pose_check(s, frames, cams, objs, maps, 3)
    assert chk["frames"] == 3
    assert all(v == 0.0 for v in chk["device_vs_reference"].values()), chk
    # the reference's own single-precision distance to the FP64 oracle, and the
    # "device" (here the reference) against FP64 are the same numbers
    assert chk["device_vs_fp64_oracle"] == chk["reference_vs_fp64_oracle"]
    assert 0.0 < chk["reference_vs_fp64_oracle"]["camera_m"] < 1e-3


def _product_robust(tmp_path_factory):
    """The device's robust() (mid_fusion_b200/csrc/mf_robust.cuh) compiled for
    the host, as the GN kernels compile it for the device: plain IEEE float and
    double operations, no contraction into fused multiply-adds."""
    import ctypes as C
    import os
    import subprocess
    d = tmp_path_factory.mktemp("robust")
    src = d / "robust_host.cpp"
    src.write_text('#include "mf_robust.cuh"\n'
                   'extern "C" void robust_host(int kind, const float* e, int n, float* w, '
                   'float* l) { for (int i = 0; i < n; ++i) mf::robust(e[i], kind, w[i], l[i]); }\n')
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "mid_fusion_b200", "csrc")
    so = d / "librobust_host.so"
    subprocess.run(["g++", "-O2", "-std=c++14", "-ffp-contract=off", "-fPIC", "-shared",
                    "-I", csrc, "-o", str(so), str(src)], check=True)
    lib = C.CDLL(str(so))
    FP = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    lib.robust_host.argtypes = [C.c_int, FP, C.c_int, FP, FP]
    lib.robust_host.restype = None

    def run(kind, e):
        w = np.zeros_like(e)
        loss = np.zeros_like(e)
        lib.robust_host(kind, e, e.size, w, loss)
        return w, loss
    return run


def test_robust_weights_match_reference(tmp_path_factory):
    """Tracking::calc_robust_weight / calc_robust_residual (tracking.cpp:
    1474-1532) against the device's robust() on residuals across each
    kernel's range (thresholds, signs, zeros, tiny and large values): none and
    Huber (the parity mode) bit for bit; Tukey and Cauchy, which the device
    squares in double where the reference squares in float, within one float
    ulp of 1 for the weight and 4 ulps for the loss."""
    rng = np.random.default_rng(3)
    e = np.concatenate([
        rng.normal(scale=0.5, size=50000), rng.normal(scale=3.0, size=50000),
        rng.normal(scale=20.0, size=20000), rng.uniform(-6, 6, size=50000),
        np.array([0.0, -0.0, 1e-30, -1e-30, 1e-8, 1.345, -1.345, 4.6851, -4.6851, 2.3849,
                  -2.3849, 1e6, -1e6]),
        np.nextafter(np.float32(1.345), np.float32(0)).reshape(1),
        np.nextafter(np.float32(4.6851), np.float32(10)).reshape(1)]).astype(np.float32)
    R = O.RefTracker(32, 24, np.array([20, 20, 16, 12], np.float32))
    dev = _product_robust(tmp_path_factory)
    for kind in range(4):
        wr, lr = R.robust(kind, e)
        wd, ld = dev(kind, e)
        if kind < 2:
            assert np.array_equal(wr, wd), (kind, np.flatnonzero(wr != wd)[:5])
            assert np.array_equal(lr, ld), (kind, np.flatnonzero(lr != ld)[:5])
        else:
            assert np.abs(wd - wr).max() <= np.float32(2.0 ** -23), kind
            ulps = np.abs(ld.view(np.int32).astype(np.int64) - lr.view(np.int32).astype(np.int64))
            assert ulps.max() <= 4, kind


@pytest.mark.parametrize("robust", [0, 1, 2, 3])
@pytest.mark.parametrize("use_icp,use_rgb", [(1, 1), (1, 0), (0, 1)])
def test_camera_tracking_every_robust_kernel_matches_reference(robust, use_icp, use_rgb):
    """trackLiveFrame with each robust kernel (none, Huber, Tukey, Cauchy: the
    reference's default) and with ICP rows only, photometric rows only, or
    both (Tracking(using_ICP, using_RGB)): the FP32 oracle's pose and every
    level's sums equal the reference's."""
    W, H = 320, 240
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, s.k, robust=robust, use_icp=bool(use_icp), use_rgb=bool(use_rgb))
    F = O.Tracker(W, H, s.k, robust=robust, fp64=False, use_icp=bool(use_icp),
                  use_rgb=bool(use_rgb))
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    Tr = R.track_camera(T0, T0, vm, nm)
    Tf = F.track_camera(T0, T0, vm, nm).astype(np.float32)
    assert np.array_equal(Tr, Tf)
    for level in range(3):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level


@pytest.mark.parametrize("iters", [(10,), (10, 5), (2, 2, 2), (4, 3, 1)])
def test_camera_tracking_pyramid_depths_match_reference(iters):
    """trackLiveFrame with one, two and three pyramid levels and other
    iteration counts: the FP32 oracle's pose and sums equal the reference's.
    (Four levels have no reference behaviour to match: its per-level
    photometric thresholds hold three entries, tracking.h:347-351, and a
    fourth level reads past them.)"""
    W, H = 320, 240
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, s.k, iters=iters)
    F = O.Tracker(W, H, s.k, iters=iters, robust=1, fp64=False)
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    assert np.array_equal(R.track_camera(T0, T0, vm, nm),
                          F.track_camera(T0, T0, vm, nm).astype(np.float32))
    for level in range(len(iters)):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level


@pytest.mark.parametrize("robust", [0, 2, 3])
@pytest.mark.parametrize("use_icp,use_rgb", [(1, 1), (1, 0), (0, 1)])
def test_object_tracking_every_robust_kernel_matches_reference(robust, use_icp, use_rgb):
    """trackEachObject (tracking.cpp:580-708) with the other robust kernels
    (Huber: test_object_tracking_matches_reference) and each row set: every
    object's pose and sums equal the reference's."""
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    _, labels, T0, P0, vm, nm, lm = _model(s, W, H)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, s.k, robust=robust, use_icp=bool(use_icp), use_rgb=bool(use_rgb))
    F = O.Tracker(W, H, s.k, robust=robust, fp64=False, use_icp=bool(use_icp),
                  use_rgb=bool(use_rgb))
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    Tc = R.track_camera(T0, T0, vm, nm)
    assert np.array_equal(Tc, F.track_camera(T0, T0, vm, nm).astype(np.float32))
    for i, label in enumerate(labels[1:], 1):
        mv, mn = _object_maps(vm, nm, lm, label)
        To_r, _ = R.track_object(R.object(P0[i], mv, mn), Tc, T0)
        To_f = F.track_object(P0[i], Tc, T0, vm, nm, lm, label).astype(np.float32)
        assert np.array_equal(To_r, To_f), label
        for level in range(3):
            assert np.array_equal(R.reduction(level), _sums(F, level)), (label, level)


@pytest.mark.parametrize("threshold", [0.5, 3.0])
@pytest.mark.parametrize("use_icp,use_rgb", [(1, 1), (1, 0), (0, 1)])
def test_motion_residuals_other_thresholds_and_rows_match_reference(threshold, use_icp, use_rgb):
    """compute_residuals (tracking.cpp:1535-1747) with other residual
    thresholds than the reference's 1.5 and with each row set: every row code
    and every valid row's error equal the reference's."""
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    vols, labels, T0, P0, vm, nm, _ = _model(s, W, H)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, s.k, use_icp=bool(use_icp), use_rgb=bool(use_rgb))
    F = O.Tracker(W, H, s.k, robust=1, fp64=False, use_icp=bool(use_icp), use_rgb=bool(use_rgb))
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    Tc = R.track_camera(T0, T0, vm, nm)
    assert np.array_equal(Tc, F.track_camera(T0, T0, vm, nm).astype(np.float32))
    lv = np.zeros((H, W, 3), np.float32)
    O.oracle().raycast_objects(vols, P0, labels, Tc, s.k, W, H, eps_size=s.instances[0].size,
                               vertex=lv, normal=np.zeros((H, W, 3), np.float32),
                               label_img=np.zeros((H, W), np.int32))
    res_r, err_r, _ = R.compute_residuals(Tc, T0, vm, nm, lv, use_icp=bool(use_icp),
                                          use_rgb=bool(use_rgb), threshold=threshold)
    res_f, err_f = F.motion_residuals(Tc, T0, vm, nm, lv, threshold=threshold)
    assert np.array_equal(res_r.astype(np.int8), res_f)
    ok = res_r == 1
    assert ok.sum() > 1000 and np.array_equal(err_r[ok], err_f[ok])


def test_camera_tracking_negative_fy_matches_reference():
    """A negative fy (the ICL-NUIM convention): the reference takes the rows
    above and below in the other order for the normals (vertex2normalKernel
    with NegY, tracking.cpp:805-810).  Frames rendered with fy > 0 and flipped
    upside down are the same scene seen through (fx, -fy, cx, H - 1 - cy);
    the FP32 oracle's pyramid, sums and pose equal the reference's."""
    W, H = 320, 240
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    k = np.asarray(s.k, np.float32)
    kneg = np.array([k[0], -k[1], k[2], H - 1 - k[3]], np.float32)

    def flip(a):
        return np.ascontiguousarray(a[::-1])

    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, kneg)
    F = O.Tracker(W, H, kneg, robust=1, fp64=False)
    for t in (R, F):
        t.set_frame(flip(rgb0), flip(d0))
        t.set_ref()
        t.set_frame(flip(rgb1), flip(d1))
    for level in range(3):
        for which in range(7):  # depth, intensity, vertex, normal, gradients, ICP covariance
            assert np.array_equal(R.level(level, which), F.level(level, which)), (level, which)
    Tr = R.track_camera(T0, T0, flip(vm), flip(nm))
    assert np.array_equal(Tr, F.track_camera(T0, T0, flip(vm), flip(nm)).astype(np.float32))
    for level in range(3):
        assert np.array_equal(R.level(level, 7), F.level(level, 7)), level  # rendered reference
        sums = R.reduction(level)
        assert np.array_equal(sums, _sums(F, level)), level
        assert sums[28] > 100, level


def test_camera_tracking_with_nan_and_negative_depths_matches_reference():
    """Depth frames with NaN and negative values (sensor erasures other than
    the zero dropouts the scenes have): the FP32 oracle's pyramid, sums and
    pose equal the reference's, NaNs in the same places."""
    W, H = 320, 240
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    rng = np.random.default_rng(1)
    d1 = d1.copy()
    d1[rng.random(d1.shape) < 0.005] = np.nan
    d1[rng.random(d1.shape) < 0.002] = -1.0
    R = O.RefTracker(W, H, s.k)
    F = O.Tracker(W, H, s.k, robust=1, fp64=False)
    for t in (R, F):
        t.set_frame(rgb0, d0)
        t.set_ref()
        t.set_frame(rgb1, d1)
    for level in range(3):
        for which in range(7):
            assert np.array_equal(R.level(level, which), F.level(level, which), equal_nan=True), \
                (level, which)
    assert np.array_equal(R.track_camera(T0, T0, vm, nm),
                          F.track_camera(T0, T0, vm, nm).astype(np.float32))
    for level in range(3):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level


def test_object_tracking_negative_fy_matches_reference():
    """trackEachObject with a negative fy on flipped frames and flipped model
    maps: every object's pose and sums equal the reference's."""
    W, H = 320, 240
    s = make_scene("multi", W, H, n_frames=2, seed=3, bg_size=256, obj_size=128, n_objects=3)
    _, labels, T0, P0, vm, nm, lm = _model(s, W, H)
    k = np.asarray(s.k, np.float32)
    kneg = np.array([k[0], -k[1], k[2], H - 1 - k[3]], np.float32)

    def flip(a):
        return np.ascontiguousarray(a[::-1])

    d0, rgb0, _ = s.render(0)
    d1, rgb1, _ = s.render(1)
    R = O.RefTracker(W, H, kneg)
    F = O.Tracker(W, H, kneg, robust=1, fp64=False)
    for t in (R, F):
        t.set_frame(flip(rgb0), flip(d0))
        t.set_ref()
        t.set_frame(flip(rgb1), flip(d1))
    vm, nm, lm = flip(vm), flip(nm), flip(lm)
    Tc = R.track_camera(T0, T0, vm, nm)
    assert np.array_equal(Tc, F.track_camera(T0, T0, vm, nm).astype(np.float32))
    for i, label in enumerate(labels[1:], 1):
        mv, mn = _object_maps(vm, nm, lm, label)
        To_r, _ = R.track_object(R.object(P0[i], mv, mn), Tc, T0)
        To_f = F.track_object(P0[i], Tc, T0, vm, nm, lm, label).astype(np.float32)
        assert np.array_equal(To_r, To_f), label
        for level in range(3):
            assert np.array_equal(R.reduction(level), _sums(F, level)), (label, level)


@pytest.mark.parametrize("W,H", [(322, 242), (321, 241)])
def test_camera_tracking_ragged_frame_sizes_match_reference(W, H):
    """Frame sizes that 4 does not divide, and odd ones: the pyramid's
    truncated level sizes (localImgSize_ = size >> level), the half-samples
    that drop the last row / column, the pose and the sums equal the
    reference's."""
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    R, F = _pair(s, W, H)
    for level in range(3):
        for which in range(7):
            assert np.array_equal(R.level(level, which), F.level(level, which)), (level, which)
    assert np.array_equal(R.track_camera(T0, T0, vm, nm),
                          F.track_camera(T0, T0, vm, nm).astype(np.float32))
    for level in range(3):
        assert np.array_equal(R.reduction(level), _sums(F, level)), level

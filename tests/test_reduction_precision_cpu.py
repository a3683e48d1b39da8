"""Precision of the GN reduction schemes on the reference's own rows (CPU only;
skipped where oracle/_ref was not built).

The reference's tracker (tracking.cpp, compiled unmodified into
oracle/_ref/libmf_ref_track.so) tracks a 640x480 room frame; its level-0
rows of the last evaluation (TrackData: result, error, J; tracking.cpp:923-1186)
are summed into the 29 normal-equation terms (sum rho(e), sum w e J,
sum w J J^T upper triangle, count; reduce, tracking.cpp:1191-1352) by:

* the reference itself: FP32 row-block sums (its own output, rt_reduction);
* the scheme the device implements (gn_tile_sums / warp_sum_fp64 /
  accumulate in mf_track.cu): each thread adds its at most 6 rows (3 level-0
  pixels x ICP and photometric) in FP32, and everything from the warp up is
  FP64;
* the scheme first specified for the device: the same FP32 thread partials,
  combined per CTA of 256 threads by compensated (Kahan) FP32 summation, and
  the CTA partials in FP64;
* FP64 throughout (weights, products and sums), the yardstick.

Each scheme is restated here in numpy with the device's tile layout (256
threads x 3 pixels per CTA at level 0, pixel p = tile * 768 + k * 256 + thread)
and its float products (w e, then times J_i; w J_i, then times J_j).  The
device's scheme must be at least as accurate as the Kahan scheme, and both far
more accurate than the reference's FP32 sums: the reason the device keeps its
FP64 sums instead of the Kahan partials.
"""
import numpy as np
import pytest

import _oracle as O
from mid_fusion_b200.scene import make_scene

pytestmark = pytest.mark.skipif(O.reference_tracking() is None,
                                reason="oracle/_ref not built (no reference tree)")

THREADS, PIX0 = 256, 3        # the device's CTA size and level-0 pixels per thread
IJ = [(i, j) for i in range(6) for j in range(i, 6)]


def _huber(e):
    """calc_robust_weight / calc_robust_residual, Huber k = 1.345, in double
    (tracking.cpp:1481-1488, 1511-1518)."""
    a = np.abs(e.astype(np.float64))
    w = np.where(a <= 1.345, 1.0, 1.345 / np.maximum(a, 1e-300))
    loss = np.where(a <= 1.345, 0.5 * a * a, 1.345 * (a - 0.5 * 1.345))
    return w, loss


def _terms(res, err, J, fp32):
    """Per-row terms (n x 29; rows that are not valid give 0).  fp32: the
    device's float arithmetic; else exact double products."""
    valid = res >= 1
    w, loss = _huber(err)
    n = res.shape[0]
    if fp32:
        T = np.zeros((n, 29), np.float32)
        wf = w.astype(np.float32)
        we = (wf * err).astype(np.float32)
        T[:, 0] = loss.astype(np.float32)
        for i in range(6):
            T[:, 1 + i] = we * J[:, i]
        for k, (i, j) in enumerate(IJ):
            T[:, 7 + k] = (wf * J[:, i]).astype(np.float32) * J[:, j]
    else:
        T = np.zeros((n, 29), np.float64)
        e, Jd = err.astype(np.float64), J.astype(np.float64)
        T[:, 0] = loss
        for i in range(6):
            T[:, 1 + i] = w * e * Jd[:, i]
        for k, (i, j) in enumerate(IJ):
            T[:, 7 + k] = w * Jd[:, i] * Jd[:, j]
    T[:, 28] = 1
    T[~valid] = 0
    return T


def _thread_partials(t_icp, t_rgb):
    """FP32 sums of each device thread's rows, in its order (pixel k's ICP
    row, then its photometric row, for k = 0, 1, 2): (tiles, threads, 29)."""
    n = t_icp.shape[0]
    per_tile = THREADS * PIX0
    tiles = -(-n // per_tile)
    pad = tiles * per_tile - n

    def lay(t):
        return np.concatenate([t, np.zeros((pad, 29), np.float32)]).reshape(
            tiles, PIX0, THREADS, 29)

    a, b = lay(t_icp), lay(t_rgb)
    acc = np.zeros((tiles, THREADS, 29), np.float32)
    for k in range(PIX0):
        acc = (acc + a[:, k]).astype(np.float32)
        acc = (acc + b[:, k]).astype(np.float32)
    return acc


def _kahan_cta(acc):
    """Compensated FP32 sum over each CTA's thread partials, in thread order."""
    s = np.zeros(acc.shape[::2], np.float32)
    c = np.zeros_like(s)
    for t in range(acc.shape[1]):
        y = (acc[:, t] - c).astype(np.float32)
        u = (s + y).astype(np.float32)
        c = ((u - s).astype(np.float32) - y).astype(np.float32)
        s = u
    return s


@pytest.fixture(scope="module")
def rows():
    W, H = 640, 480
    s = make_scene("room", W, H, n_frames=2, seed=5, bg_size=256, bg_dim=2.56)
    from test_track_reference_cpu import _model, _pair
    _, _, T0, _, vm, nm, _ = _model(s, W, H)
    R, _ = _pair(s, W, H)
    R.track_camera(T0, T0, vm, nm)
    res, err, J = R.track_data(0)
    return (res.reshape(2, -1), err.reshape(2, -1), J.reshape(2, -1, 6),
            R.reduction(0).astype(np.float64))


def test_device_reduction_at_least_as_accurate_as_kahan_partials(rows):
    res, err, J, ref = rows
    exact = sum(_terms(res[s], err[s], J[s], fp32=False) for s in range(2))
    truth = exact.sum(0)
    scale = np.abs(exact).sum(0)[:28]           # sum |term| per normal-equation entry
    # the rows and the reference's sums come from the same evaluation
    assert ref[28] == truth[28] == (res >= 1).sum()
    acc = _thread_partials(*(_terms(res[s], err[s], J[s], fp32=True) for s in range(2)))
    device = acc.astype(np.float64).sum(axis=(0, 1))
    kahan = _kahan_cta(acc).astype(np.float64).sum(0)

    def rel(v):
        return np.abs(v[:28] - truth[:28]) / scale

    r_ref, r_kahan, r_dev = rel(ref), rel(kahan), rel(device)
    print(f"max / median error relative to sum|term|: reference FP32 {r_ref.max():.2e} / "
          f"{np.median(r_ref):.2e}, Kahan CTA partials {r_kahan.max():.2e} / "
          f"{np.median(r_kahan):.2e}, device FP64 from the warp {r_dev.max():.2e} / "
          f"{np.median(r_dev):.2e}")
    assert r_ref.max() < 1e-5                     # the yardstick sums the reference's terms
    assert r_dev.max() <= r_kahan.max()
    assert np.median(r_dev) <= np.median(r_kahan)
    assert r_kahan.max() < r_ref.max() / 10
    assert r_dev.max() < 1e-8
    # the GN update x = (J^T W J)^-1 J^T W e from each set of sums
    def update(v):
        A = np.zeros((6, 6))
        for k, (i, j) in enumerate(IJ):
            A[i, j] = A[j, i] = v[7 + k]
        return np.linalg.solve(A, v[1:7])

    x = update(truth)
    dx = {name: np.abs(update(v) - x).max() / np.abs(x).max()
          for name, v in (("reference", ref), ("kahan", kahan), ("device", device))}
    print("GN update, max error relative to max |x|:",
          ", ".join(f"{k} {v:.2e}" for k, v in dx.items()))
    assert dx["device"] < dx["reference"]

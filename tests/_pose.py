"""Pose comparison of the GPU tests (test infrastructure).

The device's pose is compared with the reference's and with the all-FP64
oracle's, all tracked from the same start.  The reference here is the
single-precision tracking oracle (oracle/or_track.cpp), which equals the
reference's own tracking.cpp bit for bit (tests/test_track_reference_cpu.py,
tests/golden/track_golden.npz).
"""
import numpy as np

POSE_TOL = 1e-5  # m and rad


def pose_err(A, B):
    """(translation distance in m, rotation angle in rad) between two poses."""
    A = np.asarray(A, np.float64)
    B = np.asarray(B, np.float64)
    dt = float(np.linalg.norm(A[:3, 3] - B[:3, 3]))
    R = A[:3, :3].T @ B[:3, :3]
    w = 0.5 * np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    return dt, float(np.arctan2(np.linalg.norm(w), 0.5 * (np.trace(R) - 1.0)))


# A decision flip: near convergence the GN's cost test (tracking.cpp:313-321)
# compares costs that differ by less than the evaluation noise between two
# implementations (the reference's FP32 sums against FP64 sums, and rows that
# flip between validity codes when a pose moves by an ulp); the two then stop
# one GN step apart.  Such a result is accepted when it is as good a minimizer
# of the reference's own objective as the reference's result: its level-0 cost
# (evaluated by the FP64 oracle) exceeds the reference's by at most
# FLIP_COST_TOL relative, and it lies within FLIP_DIST of it.
FLIP_COST_TOL = 2e-4
FLIP_DIST = 5e-4   # m and rad


def check_pose(T_dev, T_ref, T_64, what, tol=POSE_TOL, cost=None):
    """The device's pose must lie within tol (m / rad) of the reference's and
    of the all-FP64 oracle's, both widened by twice the reference's own
    distance r to the FP64 run: the device evaluates the same
    single-precision rows but sums them in FP64, so it cannot follow the
    reference's rounding to the last bit; where that rounding moves the
    reference by r away from the exact (FP64) solution, another rounding of
    the same ill-conditioned problem lands elsewhere within about r of the
    exact answer, hence within about 2 r of the reference.  Where the
    reference agrees with FP64 (r ~ 0) this is the plain 1e-5.  Otherwise,
    with `cost` (world pose -> FP64 level-0 cost), a decision flip is accepted
    as described above.  Returns True when the device is within tol of the
    reference itself."""
    e_ref = pose_err(T_dev, T_ref)
    e_64 = pose_err(T_dev, T_64)
    r_64 = pose_err(T_ref, T_64)
    msg = (f"{what}: device vs reference {e_ref[0]:.3g} m {e_ref[1]:.3g} rad, device vs FP64 "
           f"{e_64[0]:.3g} m {e_64[1]:.3g} rad, reference vs FP64 {r_64[0]:.3g} m "
           f"{r_64[1]:.3g} rad")
    if not all(max(e_ref[k], e_64[k]) <= tol + 2 * r_64[k] for k in (0, 1)):
        assert cost is not None, msg
        assert all(e_ref[k] <= FLIP_DIST + 2 * r_64[k] for k in (0, 1)), msg
        c_dev, c_ref = cost(T_dev), cost(T_ref)
        assert c_dev <= c_ref * (1 + FLIP_COST_TOL), (
            f"{msg}; level-0 cost at the device's pose {c_dev:.9g}, at the reference's "
            f"{c_ref:.9g}")
    return e_ref[0] <= tol and e_ref[1] <= tol


def camera_cost(trk64, T_w_r, vertex, normal):
    """World camera pose -> the FP64 oracle's level-0 cost (sum of the robust
    losses over the valid rows) of its current frame against the model maps."""
    def f(T):
        s = trk64.camera_sums(0, np.asarray(T, np.float32), T_w_r, vertex, normal)
        return float(s[0] / max(s[28], 1.0))
    return f


def object_cost(trk64, T_wo1, T_w_c2, T_w_c1, vertex, normal, labels, label):
    """World object pose -> the FP64 oracle's level-0 object cost."""
    def f(T):
        T_c2_o2 = np.linalg.inv(np.asarray(T_w_c2, np.float64)) @ np.asarray(T, np.float64)
        s = trk64.object_sums(0, T_c2_o2.astype(np.float32), T_wo1, T_w_c1, vertex, normal,
                              labels, label)
        return float(s[0] / max(s[28], 1.0))
    return f

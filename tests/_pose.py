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


def check_pose(T_dev, T_ref, T_64, what, tol=POSE_TOL):
    """The device's pose must lie within tol (m / rad) of the reference's and
    of the all-FP64 oracle's, both widened by twice the reference's own
    distance r to the FP64 run: the device evaluates the same
    single-precision rows but sums them in FP64, so it cannot follow the
    reference's rounding to the last bit; where that rounding moves the
    reference by r away from the exact (FP64) solution, another rounding of
    the same ill-conditioned problem lands elsewhere within about r of the
    exact answer, hence within about 2 r of the reference.  Where the
    reference agrees with FP64 (r ~ 0) this is the plain 1e-5.  Returns True
    when the device is within tol of the reference itself."""
    e_ref = pose_err(T_dev, T_ref)
    e_64 = pose_err(T_dev, T_64)
    r_64 = pose_err(T_ref, T_64)
    for k, name in ((0, "m"), (1, "rad")):
        assert max(e_ref[k], e_64[k]) <= tol + 2 * r_64[k], (
            f"{what}: device vs reference {e_ref[k]:.3g} {name}, device vs FP64 "
            f"{e_64[k]:.3g}, reference vs FP64 {r_64[k]:.3g}")
    return e_ref[0] <= tol and e_ref[1] <= tol

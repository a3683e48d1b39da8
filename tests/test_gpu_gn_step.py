"""The batched GN's device step (one warp per problem, the factor's rows and
the pose elements spread over the lanes) against the plain path's host step
(tracking.cpp:287-335 / :657-686 restated serially), on the same inputs: the
same poses, flags and iteration counts bit for bit, through every branch of
the step -- update, convergence, step back on a cost increase, the truncated
solve of a rank-deficient system, the small-angle exponential, the object
problem without rows, and the level's first iteration (mf_debug_gn_step)."""
import numpy as np
import pytest

from mid_fusion_b200 import build
from mid_fusion_b200.capi import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _se3(rng, rot=0.3, trans=0.5):
    w = rng.normal(size=3)
    w *= rng.uniform(0, rot) / np.linalg.norm(w)
    th = np.linalg.norm(w)
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    R = np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K
    T = np.eye(4)
    T[:3, :3] = R
    T[:3, 3] = rng.uniform(-trans, trans, 3)
    return T


def _sums(J, r):
    """reduceKernel layout: error, J^T r (6), the 21 upper-triangle terms of
    J^T J (row-major), rows, three counts."""
    s = np.zeros(32)
    s[0] = float(r @ r)
    s[1:7] = J.T @ r
    A = J.T @ J
    s[7:28] = [A[i, j] for i in range(6) for j in range(i, 6)]
    s[28] = len(r)
    s[29:32] = [len(r), 0, 0]
    return s


def _cases(seed=7):
    rng = np.random.default_rng(seed)
    states, sums, what = [], [], []

    def add(name, J, r, prev_err=np.inf, kind=0, first=0, level=0):
        st = np.zeros(36)
        st[0:16] = _se3(rng).reshape(16)
        st[16:32] = _se3(rng).reshape(16)
        st[32] = prev_err
        st[33] = kind
        st[34] = first
        st[35] = level
        states.append(st)
        sums.append(_sums(J, r))
        what.append(name)

    for i in range(24):  # ordinary updates, both kinds, every level
        m = int(rng.integers(50, 3000))
        J = rng.normal(size=(m, 6)) * rng.uniform(0.1, 10, 6)
        r = rng.normal(size=m) * rng.uniform(1e-3, 1.0)
        add("update", J, r, prev_err=np.inf if i % 3 == 0 else 1e9, kind=i % 2,
            first=int(i % 4 == 1), level=i % 3)
    for i in range(8):  # converged: tiny step and cost
        m = 500
        J = rng.normal(size=(m, 6))
        r = rng.normal(size=m) * 1e-9
        add("converged", J, r, kind=i % 2, level=i % 3)
    for i in range(8):  # cost increase: step back
        m = 400
        J = rng.normal(size=(m, 6))
        r = rng.normal(size=m)
        add("step back", J, r, prev_err=float(r @ r) / m * 0.5, kind=i % 2, level=i % 3)
    for i in range(8):  # rank deficient: the truncated eigen solve
        m = 300
        J = rng.normal(size=(m, 6))
        J[:, 5] = J[:, 4] * (1 + 1e-9 * (i % 2))
        r = rng.normal(size=m) * 0.1
        add("rank deficient", J, r, kind=i % 2, level=i % 3)
    for i in range(8):  # small-angle exponential with a translation step
        m = 300
        J = rng.normal(size=(m, 6))
        x = np.concatenate([rng.uniform(-1, 1, 3) * 1e-3, rng.uniform(-1, 1, 3) * 1e-6])
        r = J @ x + rng.normal(size=m) * 1e-9
        add("small angle", J, r, kind=i % 2, level=i % 3)
    for i in range(4):  # object problem without rows
        add("no rows", np.zeros((0, 6)), np.zeros(0), prev_err=1.0, kind=1, first=i % 2,
            level=i % 3)
    for i in range(4):  # level's first iteration after a finite cost
        m = 200
        J = rng.normal(size=(m, 6))
        r = rng.normal(size=m)
        add("first", J, r, prev_err=1e-12, kind=i % 2, first=1, level=i % 3)
    return np.array(states), np.array(sums), what


def test_device_step_equals_host_step_bit_for_bit():
    ctx = Context(64, 48, robust="huber")
    states, sums, what = _cases()
    dev, host = ctx.debug_gn_step(states, sums)
    ctx.close()
    for i, name in enumerate(what):
        assert np.array_equal(dev[i], host[i], equal_nan=True), (
            name, i, np.flatnonzero(dev[i] != host[i]))
    # every branch was taken
    done, fallback = host[:, 33], host[:, 34]
    moved = np.any(host[:, 0:16] != states[:, 0:16], axis=1)
    kinds = {n: i for i, n in enumerate(what)}
    assert all(moved[i] and not done[i] for i, n in enumerate(what) if n == "update")
    assert all(done[i] and not moved[i] for i, n in enumerate(what) if n == "converged")
    assert all(done[i] and np.array_equal(host[i, 0:16], states[i, 16:32])
               for i, n in enumerate(what) if n == "step back")
    assert all(fallback[i] for i, n in enumerate(what) if n == "rank deficient")
    assert all(done[i] and host[i, 35] == 1 for i, n in enumerate(what) if n == "no rows")
    assert all(moved[i] for i, n in enumerate(what) if n in ("small angle", "first"))
    assert kinds

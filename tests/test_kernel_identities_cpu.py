"""Arithmetic identities the CUDA kernels rely on to match the reference,
checked on the CPU in float32.

Allocation marking (alloc_mark_kernel, mid_fusion_b200/csrc/mf_volume.cu):
the reference floors p = pos / voxel and tests 0 <= floor(p) < size before
converting to int (alloc_impl.hpp:121-191).  The kernel tests 0 <= p < size
and truncates.  For an integer size both tests accept the same p, NaN and
infinities included, and on the accepted p truncation equals the floor."""
import numpy as np
import pytest


def _reference(p, size):
    s = np.floor(p)
    ok = (s < np.float32(size)) & (s >= 0)
    return ok, np.where(ok, s, 0).astype(np.int64)


def _kernel(p, size):
    ok = (p < np.float32(size)) & (p >= 0)
    return ok, np.where(ok, np.trunc(np.where(ok, p, 0)), 0).astype(np.int64)


@pytest.mark.parametrize("size", [32, 64, 256, 512, 1024, 4096])
def test_floor_test_equals_range_test_and_truncation(size):
    f = np.float32
    ints = np.arange(-3, size + 4, dtype=np.float64)
    vals = [ints.astype(f)]
    # the float32 neighbours of every integer boundary
    for k in (1, 2, 3):
        up, dn = ints.astype(f), ints.astype(f)
        for _ in range(k):
            up = np.nextafter(up, f(np.inf))
            dn = np.nextafter(dn, f(-np.inf))
        vals += [up, dn]
    rng = np.random.default_rng(size)
    vals.append(rng.uniform(-2.0, size + 2.0, 200000).astype(f))
    vals.append(np.array([0.0, -0.0, np.nan, -np.nan, np.inf, -np.inf, 1e-45, -1e-45,
                          np.finfo(f).max, -np.finfo(f).max, 1e30, -1e30], f))
    p = np.concatenate(vals).astype(f)
    ok_r, v_r = _reference(p, size)
    ok_k, v_k = _kernel(p, size)
    assert np.array_equal(ok_r, ok_k)
    assert np.array_equal(v_r[ok_r], v_k[ok_k])
    assert np.all((v_k[ok_k] >= 0) & (v_k[ok_k] < size))


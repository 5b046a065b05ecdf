"""The allocation-free near-to-far entry point (fdtd_near2far_noalloc).

Callers whose device memory belongs to a pool or arena they must not
bypass, or that may not allocate while a job runs, use this entry point: it
stages everything in the library's static device scratch instead of calling
cudaMalloc. These tests call it through the C-ABI and hold it to the
allocating entry point's results, on two calls in a row (the scratch keeps
the previous call's contents, so the second call must not see stale data).
This file is collected last on purpose.
"""
import numpy as np
import pytest

from fdtdsarsim_b200 import _native

pytestmark = pytest.mark.gpu


def _planes(rng, ny, nx, dtype):
    return [(rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))).astype(dtype)
            for _ in range(4)]


@pytest.mark.parametrize('dtype', [np.complex64, np.complex128])
def test_noalloc_matches_allocating_entry_point_twice(dtype):
    rng = np.random.default_rng(21)
    calls = [
        (_planes(rng, 181, 221, dtype), np.linspace(-80.0, 80.0, 41), np.asarray([0.0, 35.0]), 61),
        (_planes(rng, 95, 63, dtype), np.linspace(-60.0, 70.0, 17), np.asarray([10.0]), 33),
    ]
    for planes, thetas, phis, nz in calls:
        ny, nx = planes[0].shape
        ref = _native.near2far(*planes, nx, ny, nz, 0.00116, 2.0e3, thetas, phis, 5.4e9)
        got = _native.near2far(*planes, nx, ny, nz, 0.00116, 2.0e3, thetas, phis, 5.4e9,
                               allocate=False)
        for k in ('E_theta', 'E_phi', 'H_theta', 'H_phi'):
            err = np.max(np.abs(got[k] - ref[k])) / np.max(np.abs(ref[k]))
            assert err < 1e-10, (k, err)


def test_noalloc_rejects_sizes_beyond_the_scratch():
    z = np.zeros((801, 801), np.complex128)   # 641601 cells > 600000
    with pytest.raises(_native.FdtdError) as ei:
        _native.near2far(z, z, z, z, 801, 801, 5, 0.001, 2.0e3, [0.0], [0.0], 5.4e9,
                         allocate=False)
    assert ei.value.code == _native.FDTD_ERR_INVALID
    assert 'scratch' in str(ei.value)
    small = np.zeros((5, 5), np.complex64)
    with pytest.raises(_native.FdtdError) as ei:
        _native.near2far(small, small, small, small, 5, 5, 5, 0.001, 2.0e3,
                         np.zeros(5000), [0.0], 5.4e9, allocate=False)
    assert ei.value.code == _native.FDTD_ERR_INVALID

"""Allocation-free tridiagonal eigenvalue entry point (GPU).

qd_tridiag_eigvals_noalloc must return exactly what the allocating entry
point qd_tridiag_bisect returns on the same band, on two calls in a row (the
second call reuses the file-scope scratch the first one left behind), and
both must agree with LAPACK on the tridiagonal matrix.  Collected last so it
also runs after every other GPU test has used the device.
"""

import numpy as np
import pytest
import scipy.linalg as sla

import qudos_b200 as q
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu


def _band(n, seed):
    """Random Hermitian tridiagonal matrix in band storage (ldb = 2)."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=n) * 3.0
    e = rng.normal(size=n - 1) + 1j * rng.normal(size=n - 1)
    AB = np.zeros((n, 2), dtype=np.complex128)  # row j = column j of the band: [diag, sub-diag]
    AB[:, 0] = d
    AB[:-1, 1] = e
    return AB, d, np.abs(e)


def _alloc_path(dAB, n, lo, hi):
    m = hi - lo + 1
    d, e2, bnd, w = L.DeviceBuffer(8 * n), L.DeviceBuffer(8 * n), L.DeviceBuffer(64), L.DeviceBuffer(8 * m)
    L.check(L.lib.qd_tridiag_bisect(dAB.ptr, 2, n, lo, hi, d.ptr, e2.ptr, bnd.ptr, w.ptr, None))
    L.check(L.lib.qd_device_synchronize())
    return w.download(np.empty(m))


def _noalloc_path(dAB, n, lo, hi):
    m = hi - lo + 1
    w = L.DeviceBuffer(8 * m)
    L.check(L.lib.qd_tridiag_eigvals_noalloc(dAB.ptr, 2, n, lo, hi, w.ptr, None))
    L.check(L.lib.qd_device_synchronize())
    return w.download(np.empty(m))


@pytest.mark.parametrize("n,lo,hi", [(1000, 480, 511), (4096, 0, 63), (20000, 11990, 12021)])
def test_noalloc_matches_allocating_entry(n, lo, hi):
    assert q.device_count() > 0, "no CUDA device visible"
    AB, d, e = _band(n, seed=n)
    dAB = L.DeviceBuffer(AB.nbytes)
    dAB.upload(AB)
    ref = _alloc_path(dAB, n, lo, hi)
    first = _noalloc_path(dAB, n, lo, hi)
    second = _noalloc_path(dAB, n, lo, hi)
    np.testing.assert_array_equal(first, ref)
    np.testing.assert_array_equal(second, ref)
    lapack = sla.eigvalsh_tridiagonal(d, e, select="i", select_range=(lo, hi))
    assert np.abs(first - lapack).max() <= 1e-12 * max(1.0, np.abs(lapack).max())


def test_noalloc_rejects_oversize():
    assert q.device_count() > 0, "no CUDA device visible"
    n = L.QD_STATIC_TRI_MAX + 1
    w = L.DeviceBuffer(8)
    dAB = L.DeviceBuffer(32)
    rc = L.lib.qd_tridiag_eigvals_noalloc(dAB.ptr, 2, n, 0, 0, w.ptr, None)
    assert rc == L.QD_ERR_ARG

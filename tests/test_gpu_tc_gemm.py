"""Tensor-core (tcgen05 kind::tf32, 3xTF32) complex64 GEMMs of the mixed
reduction against numpy complex128 products (GPU).

The 3xTF32 split carries about 22 significant bits per operand and FP32
accumulation, so errors are bounded relative to the magnitudes summed:
max |dX| <= 2e-6 * max(|A| |V|) * sqrt(K)-scaled norms; the tests use the
product of absolute values as the scale.
"""

import ctypes as C

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu

TOL = 4e-6


def _c64(rng, shape):
    return (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)


def _hermitian(rng, n):
    a = _c64(rng, (n, n)).astype(np.complex128)
    return np.asfortranarray(((a + a.conj().T) / 2).astype(np.complex64))


class _Work:
    def __init__(self, n, kmax):
        self.p = C.c_void_p()
        L.check(L.lib.qd_tc_work_alloc(n, kmax, C.byref(self.p)))

    def __del__(self):
        L.lib.qd_tc_work_free(self.p)


def _dev(arr):
    b = L.DeviceBuffer(arr.nbytes)
    b.upload(np.asfortranarray(arr).ravel(order="F"))
    return b


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


@pytest.mark.parametrize("n,off,nb", [(512, 0, 32), (1000, 64, 32), (1000, 64, 17), (2048, 990, 32), (336, 328, 8),
                                      (6144, 32, 32)])
def test_xprod(n, off, nb):
    rng = np.random.default_rng(n + off + nb)
    A = _hermitian(rng, n)
    m = n - off
    VT = np.asfortranarray(_c64(rng, (m, nb)))
    w = _Work(n, 256)
    dA, dV = _dev(A), _dev(VT)
    dX = L.DeviceBuffer(m * 32 * 8)
    for _ in range(2):  # second call reuses the work buffers
        L.check(L.lib.qd_tc_xprod(dA.ptr, n, n, off, m, dV.ptr, m, nb, dX.ptr, m, w.p, None))
        L.check(L.lib.qd_device_synchronize())
        L.check(L.lib.qd_tc_work_check(w.p))
    X = dX.download(np.empty((m, 32), dtype=np.complex64, order="F"))[:, :nb]
    A22 = A[off:, off:].astype(np.complex128)
    ref = A22 @ VT.astype(np.complex128)
    scale = (np.abs(A22) @ np.abs(VT.astype(np.complex128))).max()
    err = np.abs(X - ref).max() / scale
    assert err < TOL, err


@pytest.mark.parametrize("n,off,K", [(512, 0, 64), (1000, 32, 256), (1000, 488, 96), (300, 170, 40)])
def test_flush(n, off, K):
    rng = np.random.default_rng(n + off + K)
    A = _hermitian(rng, n)
    mt = n - off
    V = np.asfortranarray(_c64(rng, (n, 256)))
    W = np.asfortranarray(_c64(rng, (n, 256)))
    w = _Work(n, 256)
    dA, dV, dW = _dev(A), _dev(V), _dev(W)
    L.check(L.lib.qd_tc_flush(dA.ptr, n, off, mt, dV.ptr, dW.ptr, n, off, K, w.p, None))
    L.check(L.lib.qd_device_synchronize())
    L.check(L.lib.qd_tc_work_check(w.p))
    out = dA.download(np.empty((n, n), dtype=np.complex64, order="F"))
    v, ww = V[off:, :K].astype(np.complex128), W[off:, :K].astype(np.complex128)
    upd = v @ ww.conj().T + ww @ v.conj().T
    ref = A.astype(np.complex128)
    ref[off:, off:] -= upd
    scale = (np.abs(v) @ np.abs(ww).T).max() * 2 + np.abs(A).max()
    err = np.abs(out - ref).max() / scale
    assert err < TOL, err
    # rows/columns outside the trailing block are untouched
    assert np.array_equal(out[:off, :], A[:off, :]) and np.array_equal(out[:, :off], A[:, :off])

"""The eigensolver's own tall-and-skinny and FP64 block kernels against numpy
(GPU): qd_tsmm_nn, qd_tsmm_cn, qd_small_cn in complex64 and complex128, and
qd_hemm_lower_dev, qd_gram_dev, qd_zgemm_small_dev in complex128.  Errors are
measured relative to the sum of |terms| of each output: below 1e-4 for
complex64 and 1e-12 for complex128."""

import ctypes as C

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _dev(a):
    b = L.DeviceBuffer(max(a.nbytes, 16))
    b.upload(np.asfortranarray(a).ravel(order="F"))
    return b


def _get(buf, shape, dtype):
    out = np.empty(int(np.prod(shape)), dtype=dtype)
    buf.download(out)
    return out.reshape(shape, order="F")


def _rnd(rng, shape, dtype):
    return (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(dtype)


def _tol(dtype):
    return 1e-4 if dtype == np.complex64 else 1e-12


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("m,nc,K0,K1,bt", [(1000, 32, 64, 64, 1), (27000, 32, 224, 224, 1), (333, 7, 5, 0, 0),
                                           (5000, 32, 32, 0, 0), (129, 32, 256, 256, 0), (27000, 48, 32, 0, 0),
                                           (2000, 64, 40, 40, 1)])
def test_tsmm_nn(dtype, m, nc, K0, K1, bt):
    rng = np.random.default_rng(m + nc + K0)
    A0, A1 = _rnd(rng, (m, K0), dtype), _rnd(rng, (m, max(K1, 1)), dtype)
    B0 = _rnd(rng, (nc, K0) if bt else (K0, nc), dtype)
    B1 = _rnd(rng, (nc, max(K1, 1)) if bt else (max(K1, 1), nc), dtype)
    C0 = _rnd(rng, (m, nc), dtype)
    op = (lambda b: b.conj().T) if bt else (lambda b: b)
    c128 = lambda x: x.astype(np.complex128)  # noqa: E731
    ref = 0.5 * c128(C0) - c128(A0) @ c128(op(B0))
    scale = 0.5 * np.abs(c128(C0)) + np.abs(c128(A0)) @ np.abs(c128(op(B0)))
    nterms = 2 if K1 else 1
    if K1:
        ref = ref + 0.25 * c128(A1) @ c128(op(B1))
        scale = scale + 0.25 * np.abs(c128(A1)) @ np.abs(c128(op(B1)))
    dA0, dA1, dB0, dB1, dC = _dev(A0), _dev(A1), _dev(B0), _dev(B1), _dev(C0)
    vp = C.c_void_p
    A = (vp * 2)(dA0.ptr, dA1.ptr)
    B = (vp * 2)(dB0.ptr, dB1.ptr)
    lda = (C.c_int64 * 2)(m, m)
    ldb = (C.c_int64 * 2)(*([nc, nc] if bt else [K0, max(K1, 1)]))
    K = (C.c_int * 2)(K0, K1)
    btr = (C.c_int * 2)(bt, bt)
    al = (C.c_double * 2)(-1.0, 0.25)
    L.check(L.lib.qd_tsmm_nn(int(dtype == np.complex64), m, nc, nterms, A, lda, B, ldb, K, btr, al, dC.ptr, m, 0.5,
                             None))
    got = _get(dC, (m, nc), dtype)
    assert (np.abs(got - ref) / scale).max() < _tol(dtype)


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
@pytest.mark.parametrize("m,k1,nc", [(27000, 32, 32), (27000, 224, 32), (100, 256, 5), (64, 17, 32), (7000, 96, 20),
                                     (27000, 32, 48), (9472, 64, 64), (3000, 40, 33)])
def test_tsmm_cn(dtype, m, k1, nc):
    rng = np.random.default_rng(m + k1 + nc)
    A, B = _rnd(rng, (m, k1), dtype), _rnd(rng, (m, nc), dtype)
    A2, B2 = A.astype(np.complex128), B.astype(np.complex128)
    ref = A2.conj().T @ B2
    scale = np.abs(A2).T @ np.abs(B2)
    dA, dB, dC = _dev(A), _dev(B), L.DeviceBuffer(16 * k1 * nc)
    es = 8 if dtype == np.complex64 else 16
    nbytes = L.lib.qd_tsmm_cn_scratch_bytes(m, k1, nc, es)
    scr = L.DeviceBuffer(nbytes)
    L.check(L.lib.qd_tsmm_cn(int(dtype == np.complex64), m, dA.ptr, m, k1, dB.ptr, m, nc, dC.ptr, k1, scr.ptr, nbytes,
                             None))
    got = _get(dC, (k1, nc), dtype)
    assert (np.abs(got - ref) / scale).max() < _tol(dtype)


@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_small_cn(dtype):
    rng = np.random.default_rng(3)
    A, B = _rnd(rng, (32, 30), dtype), _rnd(rng, (32, 31), dtype)
    dA, dB, dC = _dev(A), _dev(B), L.DeviceBuffer(16 * 30 * 31)
    L.check(L.lib.qd_small_cn(int(dtype == np.complex64), 32, 30, 31, dA.ptr, 32, dB.ptr, 32, 0.5, dC.ptr, 30, None))
    got = _get(dC, (30, 31), dtype)
    A2, B2 = A.astype(np.complex128), B.astype(np.complex128)
    ref = 0.5 * A2.conj().T @ B2
    scale = 0.5 * np.abs(A2).T @ np.abs(B2)
    assert (np.abs(got - ref) / scale).max() < _tol(dtype)


@pytest.mark.parametrize("n,k", [(1000, 48), (2600, 80), (517, 7), (3000, 64)])
def test_hemm_gram_zgemm(n, k):
    rng = np.random.default_rng(n + k)
    Hf = _rnd(rng, (n, n), np.complex128)
    Hf = 0.5 * (Hf + Hf.conj().T)
    Lo = np.tril(Hf)
    Lo[np.diag_indices(n)] += 1j * 0.37  # imaginary parts on the diagonal are ignored
    X = _rnd(rng, (n, k), np.complex128)
    Y0 = _rnd(rng, (n, k), np.complex128)
    dH, dX, dY = _dev(Lo), _dev(X), _dev(Y0)
    L.check(L.lib.qd_hemm_lower_dev(n, dH.ptr, n, dX.ptr, n, k, dY.ptr, n, 0.5, None))
    got = _get(dY, (n, k), np.complex128)
    ref = Hf @ X + 0.5 * Y0
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
    dG = L.DeviceBuffer(16 * k * k)
    L.check(L.lib.qd_gram_dev(n, dX.ptr, n, k, dY.ptr, n, k, dG.ptr, k, None))
    G = _get(dG, (k, k), np.complex128)
    assert np.abs(G - X.conj().T @ ref).max() < 1e-12 * np.abs(G).max()
    Cm = _rnd(rng, (k, k), np.complex128)
    dCm, dZ = _dev(Cm), _dev(Y0)
    L.check(L.lib.qd_zgemm_small_dev(n, dX.ptr, n, k, dCm.ptr, k, k, dZ.ptr, n, -1.0, None))
    Z = _get(dZ, (n, k), np.complex128)
    assert np.abs(Z - (X @ Cm - Y0)).max() < 1e-12 * np.abs(X @ Cm).max()


def test_tsmm_cn_rejects_small_scratch():
    m, k1, nc = 9472, 32, 32
    dA, dB, dC = L.DeviceBuffer(8 * m * k1), L.DeviceBuffer(8 * m * nc), L.DeviceBuffer(8 * k1 * nc)
    scr = L.DeviceBuffer(1024)
    rc = L.lib.qd_tsmm_cn(1, m, dA.ptr, m, k1, dB.ptr, m, nc, dC.ptr, k1, scr.ptr, 1024, None)
    assert rc == L.QD_ERR_ARG

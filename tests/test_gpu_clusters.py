"""Degenerate clusters larger than the inverse-iteration block's eight warps
(GPU): a Hermitian matrix with a 12-fold degenerate eigenvalue inside the
window (random unitary eigenbasis).  The FP64 (mixed) solve must return the
window's eigenvalues within 1e-10 (1e-8) of the exact ones, vectors
orthonormal to 1e-10, and the 12 cluster vectors spanning the degenerate
subspace (largest principal angle below 1e-8, mixed 1e-4)."""

import numpy as np
import pytest
import scipy.linalg as sla

import qudos_b200 as q
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


@pytest.mark.parametrize("prec", [q.QD_PREC_FP64, q.QD_PREC_MIXED])
def test_twelve_fold_degenerate_cluster(prec):
    n = 768
    rng = np.random.default_rng(4)
    Q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    lam = np.sort(rng.uniform(-5.0, 5.0, size=n))
    lo = 400
    c = lam[lo + 8]
    lam[lo + 4:lo + 16] = c  # 12 equal eigenvalues inside the window; lam stays sorted
    A = (Q * lam) @ Q.conj().T
    A = 0.5 * (A + A.conj().T)
    hi = lo + 23
    m = hi - lo + 1
    H = L.DeviceBuffer(16 * n * n)
    H.upload(np.asfortranarray(np.tril(A)).ravel(order="F"))
    w, Z = L.DeviceBuffer(8 * m), L.DeviceBuffer(16 * n * m)
    L.check(L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, prec, w.ptr, Z.ptr, n, None))
    wg = w.download(np.empty(m))
    v = Z.download(np.empty((n, m), dtype=np.complex128, order="F"))
    ref = lam[lo:hi + 1]
    assert np.abs(wg - ref).max() < (1e-10 if prec == q.QD_PREC_FP64 else 1e-8)
    assert np.abs(v.conj().T @ v - np.eye(m)).max() < 1e-10
    ang = sla.subspace_angles(v[:, 4:16], Q[:, lo + 4:lo + 16])
    assert ang.max() < (1e-8 if prec == q.QD_PREC_FP64 else 1e-4)

"""Bounded device waits run out cleanly (GPU).

The limits of the panel factorisation's grid barrier and of the bulge
chasing's wait on the previous sweep are set to zero polls with
qd_set_wait_limits, so the first wait that does not succeed at once gives up.
The solve must return QD_ERR_TIMEOUT (not hang, not fault), the device must
stay usable, and with the default limits restored the same solve must succeed
and agree with LAPACK.  No wait is left unbounded and nothing is made to
fault: the kernels only see a poll limit of zero.
"""

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu

QD_ERR_TIMEOUT = 6


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _matrix(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    return np.asfortranarray(0.5 * (A + A.conj().T))


def _solve(A, lo, hi):
    n = A.shape[0]
    m = hi - lo + 1
    H = L.DeviceBuffer(A.nbytes)
    H.upload(np.asfortranarray(np.tril(A)).ravel(order="F"))
    w, Z = L.DeviceBuffer(8 * m), L.DeviceBuffer(16 * n * m)
    rc = L.lib.qd_eigh_window_dev(n, H.ptr, n, lo, hi, q.QD_PREC_FP64, w.ptr, Z.ptr, n, None)
    out = w.download(np.empty(m)) if rc == 0 else None
    return rc, out


@pytest.mark.parametrize("limits", [(0, -1, -1), (-1, 0, -1)], ids=["panel_barrier", "sweep_wait"])
def test_wait_runs_out_and_device_recovers(limits):
    n, lo, hi = 2048, 1000, 1031
    A = _matrix(n, 7)
    try:
        L.check(L.lib.qd_set_wait_limits(*limits))
        rc, _ = _solve(A, lo, hi)
    finally:
        L.check(L.lib.qd_set_wait_limits(-1, -1, -1))
    assert rc == QD_ERR_TIMEOUT, (rc, L.lib.qd_last_error_message())
    assert L.lib.qd_device_synchronize() == 0
    rc, w = _solve(A, lo, hi)
    assert rc == 0, L.lib.qd_last_error_message()
    ref = np.linalg.eigvalsh(A)[lo:hi + 1]
    assert np.abs(w - ref).max() < 1e-10 * np.abs(ref).max()

"""The CUDA path end to end on the reference's own example (GPU): Prism_111
energies and Bloch characters against PWEM_test_ref/energies_*.dat."""

import os

import numpy as np
import pytest

import qudos_b200 as q

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prism_111")


def _kramers(rows):
    return rows[0::2, 1:] + rows[1::2, 1:]


@pytest.mark.parametrize("prec", [q.QD_PREC_FP64, q.QD_PREC_MIXED])
def test_prism_111_golden(prec):
    pr = q.Problem(GOLDEN)
    w, v = pr.solve(prec)
    vb, cb = pr.energies(w, v)
    gvb = np.loadtxt(os.path.join(GOLDEN, "energies_vb.dat"))
    gcb = np.loadtxt(os.path.join(GOLDEN, "energies_cb.dat"))
    assert np.abs(vb[:, 0] - gvb[:, 0]).max() < 5e-9
    assert np.abs(cb[:, 0] - gcb[:, 0]).max() < 5e-9
    # Bloch characters in percent; the mixed path's vectors carry FP32-level
    # subspace errors before refinement, so its tolerance is looser
    tol = 1e-6 if prec == q.QD_PREC_FP64 else 1e-3
    assert np.abs(_kramers(vb) - _kramers(gvb)).max() < tol
    assert np.abs(_kramers(cb) - _kramers(gcb)).max() < tol

"""The drop-in boundary (GPU): the reference-named routines called through the
C ABI the way the reference's main program calls them, with the globals and
structs filled from the CPU oracle's own tables.

* hamiltonian_8_band (hamiltonian_8_band.c:23): lower triangle within 1e-12 of
  the oracle's assembly, strict upper triangle left untouched.
* diagonalise_hamiltonian (diagonalise_hamiltonian.c:24) on that host H, and
  eigenstates (eigenstates.c:23) from the globals: eigenvalues within 1e-9 eV
  of LAPACK zheevr, every Kramers pair's subspace within 1e-7 rad; with
  QD_PRECISION=mixed within 1 micro-eV.
* coulomb_matrix_elements (coulomb_matrix_elements.c:24) for the states that
  eigenstates returned: every element of the four arrays within 1e-10 of the
  oracle's (same states, so no gauge freedom), CME 1 and 4.
* the same routines fed from the library's own GPU table build agree with the
  status-returning qd_* API.
"""

import os

import numpy as np
import pytest
import scipy.linalg as sla

import qudos_b200 as q
from oracle import coulomb as ocoulomb, eigen, inputs, pipeline
from qudos_b200 import configs
from qudos_b200.refabi import ReferenceCall

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _oracle_call(pr, include_cme=0):
    t = pr.tables
    ns = pr.p["N_shape"]
    keys = ("xx", "yy", "zz", "yz", "xz", "xy")
    eps = [t.strain[k] for k in keys] if t.strain is not None else None
    conv = ([None] + [[t.conv[s][k] for k in keys + ("hydrostatic", "biaxial")] for s in range(1, ns)]
            if t.conv is not None else None)
    return ReferenceCall(pr.basis["N"], pr.geo, pr.params, t.chi, eps, conv, t.phi, F=pr.F, K=pr.basis["K"],
                         include_cme=include_cme)


@pytest.fixture(scope="module")
def deck(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("boundary"))
    configs.write_deck(d, *configs.pyramid_11(mg=2, n_states=2, cme=4))
    p, geo = inputs.load(d)
    pr = pipeline.prepare(p, geo)
    H = pipeline.assemble(pr)
    lo, hi = eigen.index_window(pr.n_pw, p["N_VB"], p["N_CB"])
    wr, vr = eigen.diagonalise(H, lo, hi)
    return d, p, pr, H, lo, hi, wr, vr


def _angles(v, vr):
    return max(sla.subspace_angles(v[:, k:k + 2], vr[:, k:k + 2]).max() for k in range(0, v.shape[1], 2))


def test_hamiltonian_8_band(deck):
    d, p, pr, H, lo, hi, wr, vr = deck
    Hg = _oracle_call(pr).hamiltonian()
    assert np.abs(np.triu(Hg, 1)).max() == 0.0
    assert np.abs(Hg - H).max() <= 1e-12 * np.abs(H).max()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_diagonalise_hamiltonian(deck, prec, monkeypatch):
    d, p, pr, H, lo, hi, wr, vr = deck
    monkeypatch.setenv("QD_PRECISION", prec)
    w, v = _oracle_call(pr).diagonalise(H, lo, hi)
    tol, atol = (1e-9, 1e-7) if prec == "fp64" else (1e-6, 1e-4)
    assert np.abs(w - wr).max() < tol
    assert _angles(v, vr) < atol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_eigenstates(deck, prec, monkeypatch):
    d, p, pr, H, lo, hi, wr, vr = deck
    monkeypatch.setenv("QD_PRECISION", prec)
    E, v = _oracle_call(pr).eigenstates(p["N_VB"], p["N_CB"])
    tol, atol = (1e-9, 1e-7) if prec == "fp64" else (1e-6, 1e-4)
    assert np.abs(E - wr).max() < tol
    assert _angles(v, vr) < atol


@pytest.mark.parametrize("cme", [1, 4])
def test_coulomb_matrix_elements(deck, cme, monkeypatch):
    d, p, pr, H, lo, hi, wr, vr = deck
    monkeypatch.setenv("QD_PRECISION", "fp64")
    call = _oracle_call(pr, include_cme=cme)
    E, v = call.eigenstates(p["N_VB"], p["N_CB"])
    NC = (p["N_C_Gx"], p["N_C_Gy"], p["N_C_Gz"])
    got = call.coulomb(NC, v, p["N_VB"], p["N_CB"])
    ref = ocoulomb.coulomb_matrix_elements(pr.basis, pr.geo, pr.params, v, 2 * p["N_VB"], 2 * p["N_CB"], NC,
                                           cme=cme, ranks=1)
    for k in ("hh", "ee", "eh_direct", "eh_exchange"):
        r = np.asarray(ref[k]).reshape(-1)
        assert np.abs(got[k] - r).max() <= 1e-10 * max(np.abs(r).max(), 1e-300), k


def test_reference_routines_fed_from_gpu_tables(deck, monkeypatch):
    d, p, pr, H, lo, hi, wr, vr = deck
    monkeypatch.setenv("QD_PRECISION", "fp64")
    gp = q.Problem(d)
    call = ReferenceCall.from_problem(gp)
    Hg = call.hamiltonian()
    assert np.abs(Hg - gp.assemble(mode=0)).max() <= 1e-13 * np.abs(Hg).max()
    E, v = call.eigenstates(p["N_VB"], p["N_CB"])
    w, vq = gp.solve(q.QD_PREC_FP64)
    assert np.abs(E - w).max() < 1e-10
    assert _angles(v, vq) < 1e-8
    assert os.environ.get("QD_PRECISION") == "fp64"

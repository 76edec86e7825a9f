"""CUDA path vs the CPU oracle on the same inputs (GPU).

Tables: shape transforms, strain, piezo potential and convolutions to 1e-11 of
their largest entry.  Assembly: max |dH| <= 1e-12 max |H|.  Eigenpairs: the
FP64 path within 1e-9 eV of LAPACK zheevr and every Kramers-pair subspace
within 1e-7 rad; the mixed path within 1 micro-eV.
"""

import numpy as np
import pytest
import scipy.linalg as sla

import qudos_b200 as q
from qudos_b200 import lib as L
from oracle import eigen, inputs, pipeline, strain as ostrain
import cases

pytestmark = pytest.mark.gpu

TABLE_TOL = 1e-11
ASSEMBLY_TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _rel(a, b):
    s = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / s


def _pair(name, mg, tmp_path):
    d = cases.CASES[name](mg, tmp_path)
    p, geo = inputs.load(d)
    return d, p, pipeline.prepare(p, geo), q.Problem(d)


@pytest.mark.parametrize("name", sorted(cases.CASES))
@pytest.mark.parametrize("mg", [1, 2])
def test_tables(name, mg, tmp_path):
    d, p, pr, gp = _pair(name, mg, tmp_path)
    gp.build_tables()
    shp = tuple(pr.basis["N_T"])
    ns = p["N_Shape"] if "N_Shape" in p else p["N_shape"]
    for s in range(1, ns):
        chi = gp.table(0, s, 0, shp)
        assert _rel(chi, pr.tables.chi[s]) < TABLE_TOL, ("chi", s)
    if p["Strain"]:
        for c, comp in enumerate(ostrain.COMPONENTS):
            assert _rel(gp.table(1, c, 0, shp), pr.tables.strain[comp]) < TABLE_TOL, ("strain", comp)
        if p["Piezo"]:
            assert _rel(gp.table(2, 0, 0, shp), pr.tables.phi) < TABLE_TOL, "phi"
        keys = list(ostrain.COMPONENTS) + ["hydrostatic", "biaxial"]
        for s in range(1, ns):
            for c, k in enumerate(keys):
                assert _rel(gp.table(3, s, c, shp), pr.tables.conv[s][k]) < TABLE_TOL, ("conv", s, k)


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_assembly_full_and_lower(name, tmp_path):
    d, p, pr, gp = _pair(name, 2, tmp_path)
    Ho = pipeline.assemble(pr, full=False)
    Hg = gp.assemble(mode=0)
    assert np.abs(np.triu(Hg, 1)).max() == 0.0  # upper triangle untouched (lower-only layout)
    assert np.abs(Hg - Ho).max() <= ASSEMBLY_TOL * np.abs(Ho).max()
    Hf = gp.assemble(mode=1)
    Hof = Ho + np.tril(Ho, -1).conj().T
    assert np.abs(Hf - Hof).max() <= ASSEMBLY_TOL * np.abs(Ho).max()


def _check_eigs(pr, H, w, v, e_tol, ang_tol):
    lo, hi = eigen.index_window(pr.n_pw, pr.p["N_VB"], pr.p["N_CB"])
    wr, vr = eigen.diagonalise(H, lo, hi)
    assert np.abs(w - wr).max() < e_tol
    Hf = np.tril(H) + np.tril(H, -1).conj().T
    res = np.linalg.norm(Hf @ v - v * w, axis=0).max()
    assert res < 1e3 * e_tol
    for k in range(0, len(w), 2):
        ang = sla.subspace_angles(v[:, k:k + 2], vr[:, k:k + 2]).max()
        assert ang < ang_tol, (k, ang)


@pytest.mark.parametrize("name", sorted(cases.CASES))
@pytest.mark.parametrize("mg", [1, 2, 3])
def test_eigensolve_fp64(name, mg, tmp_path):
    d, p, pr, gp = _pair(name, mg, tmp_path)
    w, v = gp.solve(q.QD_PREC_FP64)
    H = pipeline.assemble(pr)
    _check_eigs(pr, H, w, v, 1e-9, 1e-7)


@pytest.mark.parametrize("name", ["prism", "lens", "molecule"])
@pytest.mark.parametrize("mg", [2, 3])
def test_eigensolve_mixed(name, mg, tmp_path):
    d, p, pr, gp = _pair(name, mg, tmp_path)
    w, v = gp.solve(q.QD_PREC_MIXED)
    H = pipeline.assemble(pr)
    _check_eigs(pr, H, w, v, 1e-6, 1e-4)

"""Momentum matrix elements on the GPU (GPU).

* dH/dk from the assembly kernel's derivative mode against the oracle's
  (central difference of its assembly in K, exact for the degree-two
  polynomials in K): lower triangle within 1e-10 of max |dH/dk|, for the three
  polarisations, with strain, piezo, a field and a non-zero K.
* qd_momentum_matrix_elements for the states of an FP64 solve against the
  oracle's <vb| dH/dk |cb> with the same states: 1e-10 of the largest element.
* The reference-named routines (hamiltonian_derivative_8_band.c:23 and the
  reference's loop over momentum_matrix_element.c:24) fed from the library's
  tables agree with the qd_ entry point, and momentum_matrix_elements.dat is
  written in the reference's column layout.
"""

import os

import numpy as np
import pytest

import qudos_b200 as q
from oracle import inputs, momentum, pipeline
from qudos_b200.pwem import write_momentum_matrix_elements
from qudos_b200.refabi import ReferenceCall
import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


@pytest.mark.parametrize("name", ["pyramid", "nostrain_k", "isotropic"])
def test_dH_dk_matches_oracle(name, tmp_path):
    d = cases.CASES[name](2, tmp_path)
    p, geo = inputs.load(d)
    pr = pipeline.prepare(p, geo)
    gp = q.Problem(d)
    for a in range(3):
        ref = momentum.dH_dk(pr, a)
        got = gp.assemble_dk(a, mode=0)
        assert np.abs(np.triu(got, 1)).max() == 0.0
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max(), a
        gotf = gp.assemble_dk(a, mode=1)
        assert np.abs(gotf - momentum.full(ref)).max() <= 1e-10 * np.abs(ref).max(), a


@pytest.mark.parametrize("name", ["pyramid", "lens"])
def test_momentum_matrix_elements(name, tmp_path):
    d = cases.CASES[name](2, tmp_path)
    p, geo = inputs.load(d)
    pr = pipeline.prepare(p, geo)
    gp = q.Problem(d)
    w, v = gp.solve(q.QD_PREC_FP64)
    nv, nc = 2 * gp.n_vb, 2 * gp.n_cb
    got = gp.momentum(v, nv, nc)
    ref = momentum.momentum_matrix_elements(pr, v, nv, nc)
    assert np.abs(ref).max() > 0
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    # the reference-named routines, fed from the library's own tables
    call = ReferenceCall.from_problem(gp)
    Dz = call.hamiltonian_derivative(2)
    assert np.abs(Dz - gp.assemble_dk(2, mode=0)).max() <= 1e-13 * np.abs(Dz).max()
    mref = call.momentum_matrix_elements(v, gp.n_vb, gp.n_cb)
    assert np.abs(mref - got).max() <= 1e-12 * np.abs(got).max()
    write_momentum_matrix_elements(str(tmp_path), got)
    rows = np.loadtxt(os.path.join(str(tmp_path), "momentum_matrix_elements.dat"))
    assert rows.shape == (nc * nv, 2 + 15)  # [100], [010], [001], [110], [-110]
    hb = np.sqrt(7.61996 / 2.0)
    assert np.allclose(rows[:, 4], np.abs(got[0]).reshape(-1) / hb, rtol=1e-9, atol=0)

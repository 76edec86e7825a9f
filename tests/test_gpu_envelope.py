"""Real-space envelope functions on the GPU (GPU).

qd_envelope_functions and the reference-named envelope_functions
(envelope_functions.c:23) against the oracle's direct sums
F_b(r) = sum_G a_(b,G) exp(i (G + K).r) / sqrt(L1 L2 L3) on line scans of the
reference's grids and on random points, with a non-zero K: max |dF| <= 1e-12
of max |F|.  probability_density_*.dat files from the writer reproduce the
oracle's columns.
"""

import os

import numpy as np
import pytest

import qudos_b200 as q
from oracle import envelope, inputs, pipeline
from qudos_b200.pwem import write_probability_density
from qudos_b200.refabi import ReferenceCall
import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


@pytest.mark.parametrize("name", ["lens", "nostrain_k"])
def test_envelopes_match_oracle(name, tmp_path):
    d = cases.CASES[name](2, tmp_path)
    p, geo = inputs.load(d)
    pr = pipeline.prepare(p, geo)
    gp = q.Problem(d)
    w, v = gp.solve(q.QD_PREC_FP64)
    g0 = pr.geo[0]
    L = (g0["L1"], g0["L2"], g0["L3"])
    rng = np.random.default_rng(5)
    pts = [envelope.linescan_grid(dd, 57, L) for dd in (0, 3, 6)]
    pts.append(tuple(rng.uniform(-0.5, 0.5, size=(3, 101)) * np.array(L)[:, None]))
    for x, y, z in pts:
        F, P = gp.envelopes(v, x, y, z)
        Fo, Po = envelope.envelopes(pr.basis, L, v, x, y, z)
        assert np.abs(F - Fo).max() <= 1e-12 * np.abs(Fo).max()
        assert np.abs(P - Po).max() <= 1e-12 * np.abs(Po).max()
    # the reference-named routine, valence states (type 0)
    x, y, z = pts[0]
    call = ReferenceCall.from_problem(gp)
    nvs = 2 * gp.n_vb
    Fr, Pr = call.envelope_functions(v[:, :nvs], (gp.n_vb, gp.n_cb), 0, x, y, z)
    Fo, Po = envelope.envelopes(pr.basis, L, v[:, :nvs], x, y, z)
    assert np.abs(Fr - Fo).max() <= 1e-12 * np.abs(Fo).max()
    # writer columns
    Pg = gp.envelopes(v, x, y, z)[1]
    write_probability_density(str(tmp_path), 0, x, y, z, w[:nvs], Pg[:nvs], w[nvs:], Pg[nvs:])
    got = np.loadtxt(os.path.join(str(tmp_path), "probability_density_vb_1_100.dat"))
    ref = envelope.probability_rows(x, y, z, w[nvs - 1], Po[nvs - 1])
    assert np.allclose(got, ref, rtol=1e-6, atol=1e-6 * np.abs(ref[:, 4]).max())

"""Hellmann-Feynman gradients from the adjoint contraction (GPU).

The truncated-pyramid deck (qudos_b200.configs.pyramid_11) at 7^3 plane waves
and at its own size, 11^3 (N_H = 10648, the gradient workload).
Parameters: dot height, base half-width, composition x (the In fraction is
1 - x), the [001] field, and relative scales of the binary-table Ep and
gamma_1.
* Against central finite differences of the eigenvalues (each side a full
  FP64 solve of a perturbed deck, relative step 1e-5), for every Kramers pair
  of the window: relative error <= 1e-4 of the largest derivative.
* Against the oracle: the same expectation values with dH materialised from
  two oracle assemblies (central difference of H itself) and the same states;
  agreement to 1e-7 relative.
"""

import ctypes as C
import os

import numpy as np
import pytest

import qudos_b200 as q
from oracle import inputs, pipeline
from qudos_b200 import configs
from qudos_b200 import lib as L

pytestmark = pytest.mark.gpu

BASE = dict(height=5.0, half_base=9.0, x=0.4, fz=10.0)
PARAMS = [("height", (L.QD_GRAD_LENGTH, 1, 4)), ("half_base", (L.QD_GRAD_BASE, 1, 0)),
          ("x", (L.QD_GRAD_COMPOSITION, 1, 0)), ("fz", (L.QD_GRAD_FIELD, 0, 2)),
          ("Ep", (L.QD_GRAD_EP, 0, 0)), ("gamma1", (L.QD_GRAD_GAMMA1, 0, 0))]


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    assert q.device_count() > 0, "no CUDA device visible"


def _deck(tmp, name, mg, **kw):
    args = dict(BASE)
    args.update(kw)
    return configs.write_deck(os.path.join(str(tmp), name), *configs.pyramid_11(mg=mg, n_states=2, cme=0, **args))


def _scale(name, value):
    C.c_double.in_dll(L.lib, "qd_scale_" + name).value = value


def _solve(d):
    pr = q.Problem(d)
    w, v = pr.solve(q.QD_PREC_FP64)
    return pr, w, v


def _pairs(x):
    return 0.5 * (x[..., 0::2] + x[..., 1::2])


@pytest.fixture(scope="module", params=[3, 5], ids=["7cubed", "11cubed"])
def base_solution(tmp_path_factory, request):
    mg = request.param
    d = _deck(tmp_path_factory.mktemp("grad"), "base", mg)
    pr, w, v = _solve(d)
    g = pr.gradients(v, [p for _, p in PARAMS])
    return d, pr, w, v, g, mg


@pytest.mark.parametrize("k", range(len(PARAMS)))
def test_gradients_match_finite_differences(tmp_path, base_solution, k):
    d, pr, w, v, g, mg = base_solution
    name, _ = PARAMS[k]
    rel = 1e-5
    if name in ("Ep", "gamma1"):
        h = rel
        key = "Ep" if name == "Ep" else "gL1"
        try:
            _scale(key, 1.0 + h)
            wp = _solve(d)[1]
            _scale(key, 1.0 - h)
            wm = _solve(d)[1]
        finally:
            _scale(key, 1.0)
    else:
        h = rel * max(abs(BASE[name]), 1.0)
        wp = _solve(_deck(tmp_path, "p", mg, **{name: BASE[name] + h}))[1]
        wm = _solve(_deck(tmp_path, "m", mg, **{name: BASE[name] - h}))[1]
    fd = _pairs((wp - wm) / (2 * h))
    ad = _pairs(g[k])
    scale = np.abs(fd).max()
    assert scale > 0
    assert np.abs(ad - fd).max() <= 1e-4 * scale, (name, ad, fd)


def test_gradients_match_oracle_materialised_dH(tmp_path, base_solution):
    d, pr, w, v, g, mg = base_solution
    for k, name in ((0, "height"), (3, "fz"), (2, "x")):
        h = 1e-4 * max(abs(BASE[name]), 1.0)
        H = []
        for sgn in (1, -1):
            dd = _deck(tmp_path, "o%d%s" % (sgn, name), mg, **{name: BASE[name] + sgn * h})
            p, geo = inputs.load(dd)
            H.append(pipeline.assemble(pipeline.prepare(p, geo)))
        dH = (H[0] - H[1]) / (2 * h)
        # the oracle assembles the lower triangle: <v|dH|v> = 2 Re(v^H L v) - v^H diag(L) v
        ref = 2.0 * np.real(np.einsum("is,is->s", v.conj(), dH @ v)) - np.real(
            np.einsum("is,i,is->s", v.conj(), np.diag(dH), v))
        del H, dH
        assert np.abs(g[k] - ref).max() <= 1e-7 * np.abs(ref).max(), (name, g[k], ref)


def test_fft_correlation_matches_direct_contraction(base_solution):
    """The product path (reciprocal-space correlations by FFT) against the
    direct sum over the lower triangle of dH, same derivative tables."""
    d, pr, w, v, g, mg = base_solution
    method = C.c_int.in_dll(L.lib, "qd_grad_method")
    try:
        method.value = 1
        gd = pr.gradients(v, [p for _, p in PARAMS])
    finally:
        method.value = 0
    scale = np.abs(gd).max(axis=1, keepdims=True)
    assert np.all(np.abs(g - gd) <= 1e-10 * scale), np.abs(g - gd).max(axis=1) / scale[:, 0]


@pytest.mark.parametrize("name", ["height", "half_base", "x"])
def test_gradients_with_second_order_piezo(tmp_path, name):
    """Second-order piezoelectricity makes the coefficient table a polynomial
    of degree above two in the shape functions and in the material
    parameters; the length and composition derivatives then take the
    four-point stencil along dchi/dL and dmat/dx.  Against central
    differences of full FP64 solves (relative step 1e-5), 7^3 plane waves."""
    ov = ("-Piezo=2",)
    d = _deck(tmp_path, "base", 3)
    pr = q.Problem(d, ov)
    w, v = pr.solve(q.QD_PREC_FP64)
    k = [p for p, _ in PARAMS].index(name)
    g = pr.gradients(v, [PARAMS[k][1]])[0]
    h = 1e-5 * max(abs(BASE[name]), 1.0)
    wp = q.Problem(_deck(tmp_path, "p", 3, **{name: BASE[name] + h}), ov).solve(q.QD_PREC_FP64)[0]
    wm = q.Problem(_deck(tmp_path, "m", 3, **{name: BASE[name] - h}), ov).solve(q.QD_PREC_FP64)[0]
    fd = _pairs((wp - wm) / (2 * h))
    ad = _pairs(g)
    assert np.abs(ad - fd).max() <= 1e-4 * np.abs(fd).max(), (name, ad, fd)

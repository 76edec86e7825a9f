"""The CUDA path end to end on the reference's own examples (GPU), against
their PWEM_test_ref outputs:
* Prism_111 (N_H = 10648; free strain and Coulomb cells equal to the
  electronic cell; rotated hexagonal prism, piezo to second order);
* Truncated_pyramid (N_H = 7128; 101 shapes, a commensurate strain cell of
  3 x 3 x 4 electronic cells with M_S = 12, 12, 20, piezo to second order);
checking
* energies and Bloch characters (energies_*.dat);
* momentum matrix elements: sums of |p|^2 over CB pair x VB pair blocks for
  the five polarisations of momentum_matrix_elements.dat;
* probability densities of the example's line scans, summed over each Kramers
  pair (probability_density_*.dat).
The fixtures are extracted by tests/golden/make_golden.py."""

import os

import json

import numpy as np
import pytest

import qudos_b200 as q
from oracle import envelope
from test_oracle_golden import momentum_pair_sums, probability_pairs

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# fixture directory -> (line-scan direction index, tag) pairs of its golden densities
EXAMPLES = {"prism_111": ((0, "100"), (2, "001"), (6, "111")),
            "truncated_pyramid": ((0, "100"), (1, "010"), (2, "001"))}


def _kramers(rows):
    return rows[0::2, 1:] + rows[1::2, 1:]


@pytest.mark.parametrize("example", sorted(EXAMPLES))
@pytest.mark.parametrize("prec", [q.QD_PREC_FP64, q.QD_PREC_MIXED])
def test_golden_energies(example, prec):
    GOLDEN = os.path.join(HERE, example)
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


@pytest.mark.parametrize("example", sorted(EXAMPLES))
@pytest.mark.parametrize("prec", [q.QD_PREC_FP64, q.QD_PREC_MIXED])
def test_golden_momentum_and_densities(example, prec):
    GOLDEN = os.path.join(HERE, example)
    pr = q.Problem(GOLDEN)
    w, v = pr.solve(prec)
    nv, nc = 2 * pr.n_vb, 2 * pr.n_cb
    tol = 1e-8 if prec == q.QD_PREC_FP64 else 1e-4
    gold = json.load(open(os.path.join(GOLDEN, "momentum_pairs.json")))
    ours = momentum_pair_sums(pr.momentum(v, nv, nc))
    ref = np.array(gold["pair_sums"])
    assert np.abs(ours - ref).max() <= tol * np.abs(ref).max()
    dens = np.load(os.path.join(GOLDEN, "probability_pairs.npz"))
    geo = pr.geometry(pr.n_shape)[0]
    L = (geo["L1"], geo["L2"], geo["L3"])
    ptol = 1e-5 if prec == q.QD_PREC_FP64 else 1e-4
    for d, tag in EXAMPLES[example]:
        x, y, z = envelope.linescan_grid(d, 300, L)
        P = pr.envelopes(v, x, y, z)[1]
        vb = probability_pairs(P, [nv - 1 - k for k in range(nv)])
        cb = probability_pairs(P, [nv + k for k in range(nc)])
        for o, r in ((vb, dens["vb_" + tag]), (cb, dens["cb_" + tag])):
            assert np.all(np.abs(o - r) <= ptol * np.abs(r).max() + 2e-6 * np.abs(r)), tag

"""The oracle against the reference's own golden outputs (CPU).

code/example/Prism_111/Electronic_structure/PWEM_test_ref (copied into
tests/golden/prism_111 by tests/golden/make_golden.py):
* energies_{vb,cb}.dat: energies printed to 10 significant digits and the
  Bloch characters of each Kramers pair;
* coulomb_matrix_elements_{hh,ee,eh_direct}.dat (CME = 4: monopole, dipole and
  quadrupole corrections; 4 MPI ranks): the direct terms between Kramers pairs,
  J_PQ = sum_{i in P, k in Q} V(i, i, k, k), which do not depend on the phase
  or the rotation of the states within each pair;
* momentum_matrix_elements.dat: for each of the five polarisations the sums of
  |p|^2 over the (CB state, VB state) combinations of a CB pair and a VB pair;
* probability_density_{vb,cb}_<k>_{100,001,111}.dat: the line-scan probability
  densities (total and per band group) summed over each Kramers pair.
"""

import json
import os

import numpy as np
import pytest

from oracle import coulomb, eigen, envelope, inputs, momentum, pipeline

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prism_111")


@pytest.fixture(scope="module")
def prism_solution():
    p, geo = inputs.load(GOLDEN)
    pr = pipeline.prepare(p, geo)
    assert pr.n_h == 10648
    w, v = pipeline.solve(pr)
    return p, pr, w, v


@pytest.mark.slow
def test_prism_111_energies_match_golden(prism_solution):
    p, pr, w, v = prism_solution
    vb, cb = pipeline.energies(pr, w, v)
    gvb = eigen.read_energies(os.path.join(GOLDEN, "energies_vb.dat"))
    gcb = eigen.read_energies(os.path.join(GOLDEN, "energies_cb.dat"))
    # energies: 10 significant digits in the file
    assert np.abs(vb[:, 0] - gvb[:, 0]).max() < 5e-10
    assert np.abs(cb[:, 0] - gcb[:, 0]).max() < 5e-9
    # Bloch characters (percent), summed over each Kramers pair
    assert np.abs(pipeline.kramers_sum(vb) - pipeline.kramers_sum(gvb)).max() < 1e-7
    assert np.abs(pipeline.kramers_sum(cb) - pipeline.kramers_sum(gcb)).max() < 1e-7


@pytest.mark.slow
def test_prism_111_coulomb_direct_terms_match_golden(prism_solution):
    p, pr, w, v = prism_solution
    gold = json.load(open(os.path.join(GOLDEN, "coulomb_direct.json")))
    nv, nc = gold["n_vb_states"], gold["n_cb_states"]
    assert (nv, nc) == (2 * p["N_VB"], 2 * p["N_CB"]) and gold["CME"] == p["CME"] == 4
    NC = (p["N_C_Gx"], p["N_C_Gy"], p["N_C_Gz"])
    cme = coulomb.coulomb_matrix_elements(pr.basis, pr.geo, pr.params, v, nv, nc, NC, cme=p["CME"],
                                          ranks=gold["ranks"])
    ours = coulomb.direct_pair_terms(cme, nv, nc)
    for k in ("hh", "ee", "eh"):
        # 10 significant digits in the files
        assert np.abs(ours[k] - np.array(gold[k])).max() < 2e-10, k


def momentum_pair_sums(mme):
    """Sums of |p|^2 / (HBSQM / 2) over CB pair x VB pair blocks for the five
    polarisations of write_momentum_matrix_elements.c ([100], [010], [001],
    [110], [-110]); mme is (3, n_cb_states, n_vb_states) in eV Angstrom."""
    p = mme / np.sqrt(7.61996 / 2.0)
    pols = [p[0], p[1], p[2], (p[0] + p[1]) / np.sqrt(2.0), (-p[0] + p[1]) / np.sqrt(2.0)]
    nc, nv = p.shape[1], p.shape[2]
    return np.array([(np.abs(q) ** 2).reshape(nc // 2, 2, nv // 2, 2).sum(axis=(1, 3)) for q in pols])


def probability_pairs(F2, E_order):
    """Kramers-pair sums of the write_probability_density.c columns 5-9 for
    states in file order; F2 is (M, 8, n_grid)."""
    cols = []
    for k in E_order:
        p = 1000.0 * F2[k]
        cols.append(np.stack([p.sum(axis=0), p[3] + p[7], p[2] + p[6], p[1] + p[5], p[0] + p[4]], axis=1))
    return np.stack([cols[2 * q] + cols[2 * q + 1] for q in range(len(cols) // 2)])


@pytest.mark.slow
def test_prism_111_momentum_pairs_match_golden(prism_solution):
    p, pr, w, v = prism_solution
    gold = json.load(open(os.path.join(GOLDEN, "momentum_pairs.json")))
    nv, nc = 2 * p["N_VB"], 2 * p["N_CB"]
    ours = momentum_pair_sums(momentum.momentum_matrix_elements(pr, v, nv, nc))
    ref = np.array(gold["pair_sums"])
    # |p| printed to 11 significant digits
    assert np.abs(ours - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.slow
def test_prism_111_probability_densities_match_golden(prism_solution):
    p, pr, w, v = prism_solution
    gold = np.load(os.path.join(GOLDEN, "probability_pairs.npz"))
    g0 = pr.geo[0]
    L = (g0["L1"], g0["L2"], g0["L3"])
    nv, nc = 2 * p["N_VB"], 2 * p["N_CB"]
    for d, tag in ((0, "100"), (2, "001"), (6, "111")):
        x, y, z = envelope.linescan_grid(d, p["N_line"], L)
        assert np.abs(0.1 * np.stack([x, y, z], axis=1) - gold["xyz_" + tag]).max() < 1e-6
        F, F2 = envelope.envelopes(pr.basis, L, v, x, y, z)
        vb = probability_pairs(F2, [nv - 1 - k for k in range(nv)])  # files vb_1.. start at the highest state
        cb = probability_pairs(F2, [nv + k for k in range(nc)])
        for ours, ref in ((vb, gold["vb_" + tag]), (cb, gold["cb_" + tag])):
            # 7 significant digits in the files
            assert np.all(np.abs(ours - ref) <= 1e-5 * np.abs(ref).max() + 2e-6 * np.abs(ref)), tag


def test_lens_integral_qag_restatement_matches_gauss_legendre():
    """The lens integral I_J0 by the restated GSL QAG (61-point Kronrod rule,
    the reference's method) and by the 96-point Gauss-Legendre rule of the CUDA
    table kernel, over the (alpha, beta) range of the lens decks' grids and
    beyond (|alpha| <= 40, |beta| <= 60): agreement to 1e-13."""
    from oracle import shapes
    rng = np.random.default_rng(11)
    for alpha, beta in rng.uniform([-40.0, 0.0], [40.0, 60.0], size=(400, 2)):
        a = shapes.i_j0(alpha, beta)
        b = shapes.i_j0_gauss_legendre(alpha, beta)
        assert abs(a - b) <= 1e-13, (alpha, beta, a, b)

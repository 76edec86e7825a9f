"""The oracle against the reference's own golden outputs (CPU).

code/example/Prism_111/Electronic_structure/PWEM_test_ref (copied into
tests/golden/prism_111 by tests/golden/make_golden.py):
* energies_{vb,cb}.dat: energies printed to 10 significant digits and the
  Bloch characters of each Kramers pair;
* coulomb_matrix_elements_{hh,ee,eh_direct}.dat (CME = 4: monopole, dipole and
  quadrupole corrections; 4 MPI ranks): the direct terms between Kramers pairs,
  J_PQ = sum_{i in P, k in Q} V(i, i, k, k), which do not depend on the phase
  or the rotation of the states within each pair.
"""

import json
import os

import numpy as np
import pytest

from oracle import coulomb, eigen, inputs, pipeline

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

"""The oracle against the reference's own golden outputs (CPU).

code/example/Prism_111/Electronic_structure/PWEM_test_ref/energies_{vb,cb}.dat
(copied into tests/golden/prism_111 by tests/golden/make_golden.py): energies
printed to 10 significant digits and the Bloch characters of each Kramers pair.
"""

import os

import numpy as np
import pytest

from oracle import eigen, inputs, pipeline

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prism_111")


@pytest.mark.slow
def test_prism_111_energies_match_golden():
    p, geo = inputs.load(GOLDEN)
    pr = pipeline.prepare(p, geo)
    assert pr.n_h == 10648
    w, v = pipeline.solve(pr)
    vb, cb = pipeline.energies(pr, w, v)
    gvb = eigen.read_energies(os.path.join(GOLDEN, "energies_vb.dat"))
    gcb = eigen.read_energies(os.path.join(GOLDEN, "energies_cb.dat"))
    # energies: 10 significant digits in the file
    assert np.abs(vb[:, 0] - gvb[:, 0]).max() < 5e-10
    assert np.abs(cb[:, 0] - gcb[:, 0]).max() < 5e-9
    # Bloch characters (percent), summed over each Kramers pair
    assert np.abs(pipeline.kramers_sum(vb) - pipeline.kramers_sum(gvb)).max() < 1e-7
    assert np.abs(pipeline.kramers_sum(cb) - pipeline.kramers_sum(gcb)).max() < 1e-7

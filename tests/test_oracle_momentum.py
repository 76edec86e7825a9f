"""The oracle's momentum operator on the CPU: the central difference of the
assembly in K (exact for the degree-two polynomials in K) against the
reference's closed form of the conduction-band block
(hamiltonian_derivative_8_band_matrix_elements.c:27-90), and the Hermitian
symmetry of the momentum matrix elements' operator."""

import numpy as np
import pytest

from oracle import inputs, momentum, pipeline
import cases


@pytest.mark.parametrize("name", ["pyramid", "nostrain_k", "lens"])
def test_dH_dk_cb_block_matches_closed_form(name, tmp_path):
    d = cases.CASES[name](1, tmp_path)
    p, geo = inputs.load(d)
    pr = pipeline.prepare(p, geo)
    npw = pr.n_pw
    for a in range(3):
        D = momentum.dH_dk(pr, a)
        ref = momentum.de_cb_dk(pr, a)
        blk = D[:npw, :npw]
        assert np.abs(blk - np.tril(ref)).max() <= 1e-10 * np.abs(ref).max()
        # the same block for the spin-down conduction band
        assert np.abs(D[4 * npw:5 * npw, 4 * npw:5 * npw] - np.tril(ref)).max() <= 1e-10 * np.abs(ref).max()

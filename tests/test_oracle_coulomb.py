"""Internal consistency of the oracle's Coulomb restatement (CPU, small sizes).

* The FFT-based B functions equal the direct correlation
  B_ij(D) = sum_b sum_G conj(a_ib(G)) a_jb(G + D).
* For l >= k the integrals equal sum_D w(D) B_ij(D) B_kl(-D), the Coulomb
  integral of the pair densities.
* A Coulomb cell equal to the electronic cell reproduces B up to rounding;
  a larger cell maps B onto its larger grid.
"""

import numpy as np

from oracle import coulomb, shapes


def _states(N, M, seed):
    rng = np.random.default_rng(seed)
    n_h = 8 * N[0] * N[1] * N[2]
    v = rng.normal(size=(n_h, M)) + 1j * rng.normal(size=(n_h, M))
    return v / np.linalg.norm(v, axis=0)


def test_b_functions_are_correlations():
    N = (3, 2, 3)
    v = _states(N, 3, 1)
    B = coulomb.b_functions(v, N)
    a = v.T.reshape(3, 8, *N)
    sz = tuple(2 * n - 1 for n in N)
    for i, j in ((0, 0), (0, 2), (1, 2)):
        ref = np.zeros(sz, dtype=np.complex128)
        for dx in range(-N[0] + 1, N[0]):
            for dy in range(-N[1] + 1, N[1]):
                for dz in range(-N[2] + 1, N[2]):
                    s = 0.0
                    for gx in range(N[0]):
                        for gy in range(N[1]):
                            for gz in range(N[2]):
                                hx, hy, hz = gx + dx, gy + dy, gz + dz
                                if 0 <= hx < N[0] and 0 <= hy < N[1] and 0 <= hz < N[2]:
                                    s += np.sum(np.conj(a[i, :, gx, gy, gz]) * a[j, :, hx, hy, hz])
                    ref[dx + N[0] - 1, dy + N[1] - 1, dz + N[2] - 1] = s
        np.testing.assert_allclose(B[coulomb.pair_index(i, j)].reshape(sz), ref, atol=1e-13)


def test_integrals_l_ge_k_are_pair_density_integrals():
    N = (3, 3, 3)
    nv, nc = 2, 2
    v = _states(N, nv + nc, 2)
    L = (100.0, 100.0, 100.0)
    geo = [{"L1": L[0], "L2": L[1], "L3": L[2], "CL1": L[0], "CL2": L[1], "CL3": L[2]}]
    params = [{"nr": 3.5}]
    basis = shapes.make_basis(N, L)
    out = coulomb.coulomb_matrix_elements(basis, geo, params, v, nv, nc, N, cme=1)
    B = coulomb.b_functions(v, N)
    w = coulomb.wavevector_prefactor(basis, L, 3.5)
    n = nv
    for (i, j, k, l) in ((0, 0, 0, 0), (0, 1, 0, 1), (0, 0, 1, 1), (0, 1, 1, 1)):
        direct = np.sum(w * B[coulomb.pair_index(i, j)] * B[coulomb.pair_index(k, l)][::-1])
        assert abs(out["hh"][i * n ** 3 + j * n * n + k * n + l] - direct) < 1e-12 * max(1.0, abs(direct))


def test_coulomb_cell_copy_and_weights_agree():
    N = (3, 3, 3)
    v = _states(N, 2, 3)
    L = (80.0, 90.0, 70.0)
    basis = shapes.make_basis(N, L)
    B = coulomb.b_functions(v, N)
    same = coulomb.coulomb_supercell(B, basis, basis, L, L)
    np.testing.assert_allclose(same, B, rtol=1e-14, atol=1e-15)
    # a bigger cell along x: separable sinc weights onto the larger grid
    CL = (120.0, 90.0, 70.0)
    cb = shapes.make_basis((4, 3, 3), CL)
    big = coulomb.coulomb_supercell(B, basis, cb, L, CL)
    assert big.shape == (B.shape[0], 7 * 5 * 5)
    assert np.all(np.isfinite(big))

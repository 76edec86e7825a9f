"""Oracle restatement of the interband momentum matrix elements (test infrastructure).

Follows ``code/source/8_band/momentum_matrix_element.c:24-112`` (p = <psi_2|
dH/dk |psi_1> as zhemv + zdotc), the loop of ``8_band_main.c:1632-1655``
(conduction state psi_1, valence state psi_2 counted from the highest) and
``hamiltonian_derivative_8_band.c:23-500`` with the derivative band functions of
``hamiltonian_derivative_8_band_matrix_elements.c:27-969``.

Every element of H is a polynomial of degree two in the Bloch wave vector K
(the band functions of hamiltonian_8_band_matrix_elements.c carry K only in
(G + K)_a (G' + K)_b and linear terms), so dH/dk_a is restated here as the
central difference of the oracle's own assembly at K +- h e_a, which is exact
for such polynomials up to rounding; ``de_cb_dk`` restates the reference's
closed form for one band function (hamiltonian_derivative_8_band_matrix_elements.c:27-90)
so that the two forms can be checked against each other.
"""

import numpy as np

from . import hamiltonian

H_STEP = 1.0e-2  # 1/Angstrom


def _with_k(basis, K):
    b = dict(basis)
    b["K"] = tuple(K)
    return b


def dH_dk(pr, axis, h=H_STEP):
    """dH/dk_axis (lower triangle, N_H x N_H complex128) for a prepared oracle problem."""
    K = list(pr.basis["K"])
    Hs = []
    for sgn in (1.0, -1.0):
        Kp = list(K)
        Kp[axis] += sgn * h
        Hs.append(hamiltonian.assemble(_with_k(pr.basis, Kp), pr.geo, pr.params, pr.tables, pr.F, pr.p["Strain"],
                                       pr.p["Piezo"]))
    return (Hs[0] - Hs[1]) / (2.0 * h)


def full(Lower):
    """Hermitian matrix from its lower triangle (the diagonal's imaginary part dropped)."""
    d = np.real(np.diag(Lower))
    F = np.tril(Lower, -1)
    return F + F.conj().T + np.diag(d)


def momentum_matrix_elements(pr, v, n_vb_states, n_cb_states):
    """p[pol, c, iv] = <vb_(n_vb_states-1-iv)| dH/dk_pol |cb_c> (eV Angstrom) for the
    states v (N_H x (n_vb_states + n_cb_states), valence states first)."""
    out = np.zeros((3, n_cb_states, n_vb_states), dtype=np.complex128)
    vb = v[:, :n_vb_states][:, ::-1]
    cb = v[:, n_vb_states:n_vb_states + n_cb_states]
    for a in range(3):
        D = full(dH_dk(pr, a))
        out[a] = (vb.conj().T @ (D @ cb)).T
    return out


def de_cb_dk(pr, axis):
    """The E_CB block of dH/dk in closed form (hamiltonian_derivative_8_band_matrix_elements.c:27-90):
    1/2 HBSQM sc(G1 - G2) (G1_a + G2_a + 2 K_a), N_PW x N_PW."""
    npw = pr.n_pw
    idx = np.arange(npw)
    ctx = hamiltonian.BlockContext(pr.basis, pr.geo, pr.params, pr.tables, pr.F, pr.p["Strain"], pr.p["Piezo"],
                                   idx, idx)
    return 0.5 * hamiltonian.HBSQM * ctx.pme("sc") * ctx.ksum(axis)

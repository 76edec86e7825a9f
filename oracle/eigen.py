"""Oracle restatement of the index-window eigensolve and its outputs (test infrastructure).

Follows ``code/source/8_band/eigenstates.c:23-117`` (index window),
``diagonalise_hamiltonian.c:24-80`` (LAPACK ``zheevr``, RANGE='I', UPLO='L'),
``collect_eigenstates.c:23-75``, ``bloch_character.c:23-105`` and
``write_energies.c:23-93``.  The eigensolver is LAPACK ``zheevr`` from scipy's
bundled OpenBLAS, the same LAPACK routine the reference calls through MKL.
"""

import numpy as np
import scipy.linalg as sla

N_BAND = 8


def index_window(n_pw, n_vb, n_cb):
    """0-based inclusive [lo, hi] (eigenstates.c:29-36)."""
    idx_cb_min = (N_BAND - 2) * n_pw
    return idx_cb_min - 2 * n_vb, idx_cb_min + 2 * n_cb - 1


def diagonalise(H, lo, hi):
    """zheevr('V', 'I', 'L') on the lower triangle.  Returns (eigval[M], eigvec N_H x M)."""
    w, v = sla.eigh(H, lower=True, subset_by_index=[lo, hi], driver="evr",
                    overwrite_a=False, check_finite=False)
    return w, v


def collect(eigval, eigvec, n_vb):
    """Split into VB (first 2 N_vb, ascending) and CB states (collect_eigenstates.c:23-75)."""
    m_vb = 2 * n_vb
    return (eigval[:m_vb], eigvec[:, :m_vb]), (eigval[m_vb:], eigvec[:, m_vb:])


def bloch_character(vecs, n_pw):
    """Sum_G |a_b(G)|^2 per band b for each state (bloch_character.c:23-105).
    Returns (M, 8)."""
    a = np.abs(vecs.reshape(N_BAND, n_pw, -1)) ** 2
    return a.sum(axis=1).T


def energies_rows(E, bloch):
    """Columns of energies_*.dat: E, SO%, LH%, HH%, CB% (write_energies.c:50-84)."""
    return np.stack([E, 100.0 * (bloch[:, 3] + bloch[:, 7]), 100.0 * (bloch[:, 2] + bloch[:, 6]),
                     100.0 * (bloch[:, 1] + bloch[:, 5]), 100.0 * (bloch[:, 0] + bloch[:, 4])], axis=1)


def format_energies(rows):
    return "".join("%17.10e\t%17.10e\t%17.10e\t%17.10e\t%17.10e\n" % tuple(r) for r in rows)


def write_energies(directory, E_vb, bloch_vb, E_cb, bloch_cb):
    """energies_vb.dat is written highest state first, energies_cb.dat lowest first."""
    import os
    vb = energies_rows(E_vb, bloch_vb)[::-1]
    cb = energies_rows(E_cb, bloch_cb)
    with open(os.path.join(directory, "energies_vb.dat"), "w") as f:
        f.write(format_energies(vb))
    with open(os.path.join(directory, "energies_cb.dat"), "w") as f:
        f.write(format_energies(cb))


def read_energies(path):
    return np.loadtxt(path, ndmin=2)

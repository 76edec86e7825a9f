"""Oracle restatement of the real-space outputs (test infrastructure).

* ``envelopes``: ``code/source/8_band/envelope_functions.c:50-161``, the band
  envelopes F_b(r) = sum_G a_(b,G) exp(i (G + K).r) / sqrt(L1 L2 L3) at
  arbitrary points, and probability_b = |F_b|^2 (:174-189).
* ``linescan_grid``: the points of ``real_space_grid_linescan.c:23-160`` (lines
  through the cell centre along [100], [010], [001], [110], [101], [011], [111]).
* ``probability_rows``: the columns of ``write_probability_density.c:90-108``
  (positions in nm, energy, total / SO / LH / HH / CB densities in nm^-3).
"""

import math

import numpy as np

N_BAND = 8


def linescan_grid(direction, n_grid, L):
    """x, y, z (Angstrom) of the reference's line scan; L = (L1, L2, L3)."""
    lo = [-0.5 * L[0], -0.5 * L[1], -0.5 * L[2]]
    hi = [0.5 * L[0], 0.5 * L[1], 0.5 * L[2]]
    d = [(hi[a] - lo[a]) / (n_grid - 1.0) for a in range(3)]
    axes = {0: (0,), 1: (1,), 2: (2,), 3: (0, 1), 4: (0, 2), 5: (1, 2), 6: (0, 1, 2)}[direction]
    if len(axes) > 1:  # the shortest of the cell's lengths along the used axes limits the diagonal
        a0 = min(axes, key=lambda a: d[a])
        for a in axes:
            d[a], lo[a], hi[a] = d[a0], lo[a0], hi[a0]
    xyz = [np.zeros(n_grid) for _ in range(3)]
    for a in axes:
        v = np.empty(n_grid)
        v[0], v[-1] = lo[a], hi[a]
        for i in range(1, n_grid - 1):  # the reference accumulates the steps
            v[i] = v[i - 1] + d[a]
        xyz[a] = v
    return xyz


def envelopes(basis, L, vecs, x, y, z):
    """F (M, 8, n_grid) complex and |F|^2 for states vecs (N_H x M)."""
    Nx, Ny, Nz = basis["N"]
    NT = basis["N_T"]
    G = basis["G"]
    K = basis["K"]
    off = [NT[a] // 2 - basis["N"][a] // 2 for a in range(3)]
    ix, iy, iz = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    gx = (G[0][off[0] + ix.ravel()] + K[0])
    gy = (G[1][off[1] + iy.ravel()] + K[1])
    gz = (G[2][off[2] + iz.ravel()] + K[2])
    phase = np.exp(1j * (np.outer(x, gx) + np.outer(y, gy) + np.outer(z, gz))) / math.sqrt(L[0] * L[1] * L[2])
    npw = Nx * Ny * Nz
    a = vecs.reshape(N_BAND, npw, -1)          # (band, pw, state)
    F = np.einsum("gp,bps->sbg", phase, a)
    return F, np.abs(F) ** 2


def probability_rows(x, y, z, E, prob):
    """write_probability_density.c columns for one state: prob (8, n_grid)."""
    p = 1000.0 * prob
    return np.stack([0.1 * np.asarray(x), 0.1 * np.asarray(y), 0.1 * np.asarray(z), np.full(len(x), E),
                     p.sum(axis=0), p[3] + p[7], p[2] + p[6], p[1] + p[5], p[0] + p[4]], axis=1)

"""Oracle restatement of the Coulomb matrix elements (test infrastructure).

Follows the reference's ``coulomb_matrix_elements`` path
(code/source/8_band/coulomb_matrix_elements.c:24-627) on one process:

* ``pad_states``          zero-padded envelopes and their conjugate-reversed
                          copies per band (state_redistribution.c:23-169);
* ``b_functions``         B_ij(D) = sum_b IFFT(FFT(conjrev a_ib) FFT(a_jb)) on
                          the (2N-1)^3 grid for i <= j (B_convolutions.c:332-390);
* ``coulomb_supercell``   B on the Coulomb-cell grid, free cell lengths
                          (B_coulomb_supercell.c:23-139; identity when the
                          cells and plane-wave counts agree);
* ``coulomb_supercell_commensurate``  the same for Coulomb cells of RCL times
                          the electronic cell (B_coulomb_supercell_fft.c:23-100,
                          characteristic_function_coulomb_supercell.c:24-72);
* ``wavevector_prefactor``w(G) = e^2/eps0 / (V_C G^2 n_r^2), w(0) = 0
                          (coulomb_matrix_elements.c:370-401);
* ``corrections``         CME >= 2: Madelung constant, dipole and quadrupole
                          moments (coulomb_matrix_elements.c:252-556);
* ``integrals``           V_ijkl for the four blocks with the reference's
                          symmetry-reduced index loops (coulomb_integrals.c:23-356).

Two properties of the reference are restated as they are:
* For l < k the integrals use conj(w B^rev_lk) . B_ij (a zdotc over the
  reversed array), which is sum_D w(D) B_kl(D) B_ij(D) rather than the
  sum_D w(D) B_kl(-D) B_ij(D) used for l >= k.
* The real-space part of the Madelung sum (coulomb_matrix_elements.c:303-331)
  runs over the index block of rank ``myid - 1``; with one rank it adds
  nothing, with R ranks it covers all blocks but the last one.  ``ranks``
  selects the behaviour (the reference's example outputs were made with 4).

The four outputs are flat complex arrays in the layout the reference's main
program allocates (8_band_main.c:1752-1775): hh[i, j, k, l] over 2N_vb
states, ee over 2N_cb, eh_direct[i, j, k, l] (i, j hole, k, l electron) and
eh_exchange[i, j, k, l] (i, l hole, j, k electron); elements outside the
computed set stay zero.
"""

import math

import numpy as np
from scipy.special import erfc

from . import shapes

ESQEPS = 180.9513  # 8_band.h:52
EPS = 1.0e-08      # 8_band.h:59
N_BAND = 8


def pair_index(i, j):
    """Storage index of the pair (i <= j) (B_convolutions.c:395)."""
    return j * (j + 1) // 2 + i


def pad_states(vecs, N):
    """(M, 8, S) padded envelopes and conjugate-reversed copies on the
    (2Nx-1)(2Ny-1)(2Nz-1) grid (state_redistribution.c:45-66)."""
    Nx, Ny, Nz = N
    sz = (2 * Nx - 1, 2 * Ny - 1, 2 * Nz - 1)
    M = vecs.shape[1]
    a = vecs.T.reshape(M, N_BAND, Nx, Ny, Nz)
    pad = np.zeros((M, N_BAND) + sz, dtype=np.complex128)
    cpad = np.zeros_like(pad)
    pad[:, :, :Nx, :Ny, :Nz] = a
    cpad[:, :, :Nx, :Ny, :Nz] = np.conj(a[:, :, ::-1, ::-1, ::-1])
    return pad, cpad


def b_functions(vecs, N):
    """B_p for every pair p = (i <= j), each flattened on the padded grid
    (B_convolutions.c:332-390).  Returns (P, S)."""
    pad, cpad = pad_states(vecs, N)
    axes = (-3, -2, -1)
    F = np.fft.fftn(pad, axes=axes)
    Fc = np.fft.fftn(cpad, axes=axes)
    M = vecs.shape[1]
    S = F[0, 0].size
    B = np.zeros((M * (M + 1) // 2, S), dtype=np.complex128)
    for j in range(M):
        for i in range(j + 1):
            prod = Fc[i] * F[j]  # per band
            B[pair_index(i, j)] = np.fft.ifftn(prod, axes=axes).sum(axis=0).reshape(-1)
    return B


def coulomb_supercell(B, basis, cbasis, L, CL):
    """B on the Coulomb-cell grid (B_coulomb_supercell.c:23-139).  Separable
    weights I0(GC - G) per axis; an axis whose plane-wave count and length
    match the electronic cell is a copy (weight L at the matching index)."""
    NT = basis["N_T"]
    NCT = cbasis["N_T"]
    inv_vol = 1.0 / (L[0] * L[1] * L[2])
    W = []
    for a in range(3):
        same = cbasis["N"][a] == basis["N"][a] and L[a] == CL[a]
        w = np.zeros((NCT[a], NT[a]))
        gmax = cbasis["G"][a][NCT[a] - 1]
        for c in range(NCT[a]):
            for g in (range(c, c + 1) if same else range(NT[a])):
                d = cbasis["G"][a][c] - basis["G"][a][g]
                if abs(d) < EPS:
                    w[c, g] = L[a]
                elif abs(d) > gmax + EPS:
                    w[c, g] = 0.0
                else:
                    w[c, g] = 2.0 * math.sin(d * L[a] / 2.0) / d
        W.append(w)
    P = B.shape[0]
    Bt = B.reshape((P,) + NT)
    if all(cbasis["N"][a] == basis["N"][a] and L[a] == CL[a] for a in range(3)):
        # evaluated as the reference does: ((inv_vol * B) * I0x) * I0y) * I0z
        out = (((inv_vol * Bt) * L[0]) * L[1]) * L[2]
        return out.reshape(P, -1)
    out = np.einsum("xa,yb,zc,pabc->pxyz", W[0], W[1], W[2], Bt) * inv_vol
    return out.reshape(P, -1)


def coulomb_supercell_commensurate(B, basis, cbasis, geo, softening=0, sigma=0.0):
    """B on the Coulomb-cell grid for Coulomb_supercell_type 1, CL = RCL L
    (B_convolutions.c:170-300 and B_coulomb_supercell_fft.c:23-100): B is
    placed on every RCL-th point of a grid of NC_T + 2 RCL (N_T / 2) points per
    axis, convolved (forward FFTs, product, backward FFT with scale 1/size)
    with the electronic cell's cuboid (shape record 0) tabulated on the Coulomb
    grid with the Coulomb-cell normalisation, and the central NC_T block is
    scaled by CL1 CL2 CL3 / (L1 L2 L3).  ``B`` holds the pair functions on the
    (2N-1)^3 grid as returned by ``b_functions``."""
    g0 = geo[0]
    RC = (g0["RCL1"], g0["RCL2"], g0["RCL3"])
    NT = basis["N_T"]
    NCT = cbasis["N_T"]
    S = tuple(NCT[a] + 2 * RC[a] * (NT[a] // 2) for a in range(3))
    chi = shapes.chi_table(cbasis, geo, 0, 3, softening, sigma)
    X = np.zeros(S, dtype=np.complex128)
    X[:NCT[0], :NCT[1], :NCT[2]] = chi
    X = np.fft.fftn(X)
    P = B.shape[0]
    up = np.zeros((P,) + S, dtype=np.complex128)
    up[:, : RC[0] * NT[0]: RC[0], : RC[1] * NT[1]: RC[1], : RC[2] * NT[2]: RC[2]] = B.reshape((P,) + NT)
    axes = (-3, -2, -1)
    conv = np.fft.ifftn(np.fft.fftn(up, axes=axes) * X[None], axes=axes)
    o = [S[a] // 2 - NCT[a] // 2 for a in range(3)]
    scale = (g0["CL1"] * g0["CL2"] * g0["CL3"]) / (g0["L1"] * g0["L2"] * g0["L3"])
    out = scale * conv[:, o[0]: o[0] + NCT[0], o[1]: o[1] + NCT[1], o[2]: o[2] + NCT[2]]
    return out.reshape(P, -1)


def coulomb_grid_vectors(cbasis):
    NCT = cbasis["N_T"]
    gx, gy, gz = np.meshgrid(*cbasis["G"], indexing="ij")
    centre = np.zeros(NCT, dtype=bool)
    centre[NCT[0] // 2, NCT[1] // 2, NCT[2] // 2] = True
    return gx.reshape(-1), gy.reshape(-1), gz.reshape(-1), centre.reshape(-1)


def wavevector_prefactor(cbasis, CL, nr):
    """w(G) (coulomb_matrix_elements.c:370-401)."""
    gx, gy, gz, centre = coulomb_grid_vectors(cbasis)
    G = np.sqrt(gx * gx + gy * gy + gz * gz)
    w = np.zeros(gx.size, dtype=np.complex128)
    m = ~centre
    w[m] = ESQEPS / ((CL[0] * CL[1] * CL[2]) * G[m] * G[m] * nr ** 2.0)
    return w


def madelung(cbasis, CL, ranks=4):
    """Madelung constant a_mad summed over the reference's ranks
    (coulomb_matrix_elements.c:252-331)."""
    V = CL[0] * CL[1] * CL[2]
    ewald = math.sqrt(math.pi / (CL[0] * CL[1]))
    a = -2 * ewald / math.sqrt(math.pi) - math.pi / (ewald * ewald * V)
    gx, gy, gz, centre = coulomb_grid_vectors(cbasis)
    G2 = gx * gx + gy * gy + gz * gz
    m = ~centre
    a += np.sum((4 * math.pi / V) * np.exp(-G2[m] / (4 * ewald * ewald)) / G2[m])
    # real-space part: rank r sums the index block of rank r - 1
    NCT = cbasis["N_T"]
    n_conv = NCT[0] * NCT[1] * NCT[2]
    hy, hz = NCT[1] // 2, NCT[2] // 2
    disp, size = 0, 0
    total = 0.0
    for r in range(ranks):
        disp_r, size_r = 0, 0
        for q in range(r):
            disp_r += size_r
            size_r = n_conv // ranks + (1 if q < n_conv % ranks else 0)
        idx = np.arange(disp_r, disp_r + size_r)
        mx = idx // (hy * hz)
        my = (idx % (hy * hz)) // hz
        mz = (idx % (hy * hz)) % hz
        keep = (mx != 0) | (my != 0) | (mz != 0)
        R = np.sqrt((mx[keep] * CL[0]) ** 2 + (my[keep] * CL[1]) ** 2 + (mz[keep] * CL[2]) ** 2)
        total += np.sum(erfc(R * ewald) / R)
    return a + total


def dipole_vectors(cbasis, CL):
    """I_x, I_y, I_z on the Coulomb grid (coulomb_matrix_elements.c:403-430)."""
    gx, gy, gz, centre = coulomb_grid_vectors(cbasis)
    NCT = cbasis["N_T"]
    ix, iy, iz = np.meshgrid(*[np.arange(n) for n in NCT], indexing="ij")
    ix, iy, iz = ix.reshape(-1), iy.reshape(-1), iz.reshape(-1)
    cx, cy, cz = NCT[0] // 2, NCT[1] // 2, NCT[2] // 2
    out = []
    for a, (g, on_axis) in enumerate(((gx, (ix != cx) & (iy == cy) & (iz == cz)),
                                      (gy, (ix == cx) & (iy != cy) & (iz == cz)),
                                      (gz, (ix == cx) & (iy == cy) & (iz != cz)))):
        o = [(1, 2), (0, 2), (0, 1)][a]
        v = np.zeros(g.size, dtype=np.complex128)
        gg = g[on_axis]
        v[on_axis] = CL[o[0]] * CL[o[1]] * ((CL[a] / (1j * gg)) * np.cos(0.5 * gg * CL[a]) +
                                            (2.0j / (gg * gg)) * np.sin(0.5 * gg * CL[a]))
        out.append(v)
    return out


def quadrupole_vector(cbasis, CL):
    """J on the Coulomb grid (coulomb_matrix_elements.c:432-478)."""
    gx, gy, gz, centre = coulomb_grid_vectors(cbasis)
    NCT = cbasis["N_T"]
    ix, iy, iz = np.meshgrid(*[np.arange(n) for n in NCT], indexing="ij")
    ix, iy, iz = ix.reshape(-1), iy.reshape(-1), iz.reshape(-1)
    cx, cy, cz = NCT[0] // 2, NCT[1] // 2, NCT[2] // 2
    J = np.zeros(gx.size, dtype=np.complex128)
    for a, (g, on_axis) in enumerate(((gx, (ix != cx) & (iy == cy) & (iz == cz)),
                                      (gy, (ix == cx) & (iy != cy) & (iz == cz)),
                                      (gz, (ix == cx) & (iy == cy) & (iz != cz)))):
        o = [(1, 2), (0, 2), (0, 1)][a]
        gg = g[on_axis]
        L = CL[a]
        J[on_axis] += CL[o[0]] * CL[o[1]] * ((0.5 * L * L / gg) * np.sin(0.5 * L * gg) + (2j / gg) * (
            (L / (1j * gg)) * np.cos(0.5 * gg * L) + (2.0j / (gg * gg)) * np.sin(0.5 * gg * L)))
        J[centre] += (1 / 12.0) * L ** 3 * CL[o[0]] * CL[o[1]]
    return J


def corrections(B, cbasis, CL, M, cme, ranks=4):
    """a_mad, dipole moments d[l*M + k] (x, y, z) and quadrupole Q[pair]
    (coulomb_matrix_elements.c:252-556)."""
    out = {"a_mad": 0.0, "d": None, "Q": None}
    if cme >= 2:
        out["a_mad"] = madelung(cbasis, CL, ranks)
    if cme >= 3:
        I3 = dipole_vectors(cbasis, CL)
        d = np.zeros((3, M * M), dtype=np.complex128)
        for k in range(M):
            for l in range(M):
                for a in range(3):
                    if l >= k:
                        d[a, l * M + k] = np.dot(B[pair_index(k, l)], I3[a])
                    else:
                        d[a, l * M + k] = np.dot(np.conj(B[pair_index(l, k)]), I3[a])
        out["d"] = d
    if cme >= 4:
        J = quadrupole_vector(cbasis, CL)
        out["Q"] = B @ J
    return out


def _l_start_same(i, j, k):
    return k if j == i else (j if k == i else (i + 1 if k < j else i))


def integrals(B, Brw, nv, nc, nr, CL, corr, cme):
    """The four CME arrays (coulomb_integrals.c:23-356).  B: (P, S) pair
    functions; Brw: w * reversed B."""
    M = nv + nc
    V = CL[0] * CL[1] * CL[2]
    c_mono = -ESQEPS / (4 * math.pi * nr ** 2.0)
    c_dip = (ESQEPS / (4 * math.pi * nr ** 2.0)) * (4 * math.pi / (3 * V ** 3))
    c_quad = (-ESQEPS / (4 * math.pi * nr ** 2.0)) * (2 * math.pi / (3 * V ** 2))
    d = corr["d"]
    Q = corr["Q"]
    # all pair-pair contractions once: U[q, p] = sum Brw_q B_p, C[q, p] = sum conj(Brw_q) B_p
    U = Brw @ B.T
    Cc = np.conj(Brw) @ B.T

    def pair_term(i, j, k, l):
        p = pair_index(i, j)
        if l >= k:
            return U[pair_index(k, l), p]
        return Cc[pair_index(l, k), p]

    def dip(a_, b_):
        return c_dip * (d[0, a_] * d[0, b_] + d[1, a_] * d[1, b_] + d[2, a_] * d[2, b_])

    hh = np.zeros(nv ** 4, dtype=np.complex128)
    ee = np.zeros(nc ** 4, dtype=np.complex128)
    ehd = np.zeros(nv * nv * nc * nc, dtype=np.complex128)
    ehx = np.zeros(nv * nv * nc * nc, dtype=np.complex128)
    for blk, n, off, out in ((0, nv, 0, hh), (1, nc, nv, ee)):
        for i in range(n):
            for j in range(i, n):
                for k in range(i, n):
                    for l in range(_l_start_same(i, j, k), n):
                        I_, J_, K_, L_ = i + off, j + off, k + off, l + off
                        v = pair_term(I_, J_, K_, L_)
                        if cme >= 2 and i == j and k == l:
                            v += c_mono * corr["a_mad"]
                        if cme >= 3:
                            v += dip(J_ * M + I_, L_ * M + K_)
                        if cme >= 4:
                            if i == j and l >= k:
                                v += c_quad * Q[pair_index(K_, L_)]
                            elif i == j and l < k:
                                v += c_quad * np.conj(Q[pair_index(L_, K_)])
                            if k == l:
                                v += c_quad * Q[pair_index(I_, J_)]
                        out[i * n ** 3 + j * n * n + k * n + l] = v
    for i in range(nv):
        for j in range(i, nv):
            for k in range(nc):
                for l in range(k if j == i else 0, nc):
                    K_, L_ = nv + k, nv + l
                    v = pair_term(i, j, K_, L_)
                    if cme >= 2 and i == j and k == l:
                        v += c_mono * corr["a_mad"]
                    if cme >= 3:
                        v += dip(j * M + i, L_ * M + K_)
                    if cme >= 4:
                        if i == j and l >= k:
                            v += c_quad * Q[pair_index(K_, L_)]
                        elif i == j and l < k:
                            v += c_quad * np.conj(Q[pair_index(L_, K_)])
                        if k == l:
                            v += c_quad * Q[pair_index(i, j)]
                    ehd[i * nv * nc * nc + j * nc * nc + k * nc + l] = v
    for i in range(nv):
        for j in range(nc):
            for k in range(j, nc):
                for l in range(i if k == j else 0, nv):
                    v = Cc[pair_index(l, nv + k), pair_index(i, nv + j)]
                    if cme >= 3:
                        v += dip((nv + j) * M + i, l * M + nv + k)
                    ehx[i * nc * nc * nv + j * nc * nv + k * nv + l] = v
    return {"hh": hh, "ee": ee, "eh_direct": ehd, "eh_exchange": ehx}


def coulomb_matrix_elements(basis, geo, params, vecs, nv, nc, NC, cme=1, ranks=4, cell_type=0, softening=0,
                            sigma=0.0):
    """All four arrays for states vecs (N_H x (nv + nc), VB states first).
    ``cell_type`` is Coulomb_supercell_type (0 free lengths, 1 RCL multiples)."""
    g0 = geo[0]
    L = (g0["L1"], g0["L2"], g0["L3"])
    CL = (g0["CL1"], g0["CL2"], g0["CL3"])
    cbasis = shapes.make_basis(NC, CL)
    nr = params[0]["nr"]
    B = b_functions(vecs, basis["N"])
    if cell_type == 1:
        Bc = coulomb_supercell_commensurate(B, basis, cbasis, geo, softening, sigma)
    else:
        Bc = coulomb_supercell(B, basis, cbasis, L, CL)
    w = wavevector_prefactor(cbasis, CL, nr)
    Brw = Bc[:, ::-1] * w[None, :]
    corr = corrections(Bc, cbasis, CL, nv + nc, cme, ranks)
    return integrals(Bc, Brw, nv, nc, nr, CL, corr, cme)


def direct_pair_terms(cme_arrays, nv, nc):
    """Gauge-invariant direct terms between Kramers pairs:
    J_PQ = sum_{i in P, k in Q} V(i, i, k, k) for the hh, ee and eh blocks,
    from the computed (symmetry-reduced) elements."""
    hh, ee, ehd = cme_arrays["hh"], cme_arrays["ee"], cme_arrays["eh_direct"]

    def v4(arr, n, i, j, k, l):
        return arr[i * n ** 3 + j * n * n + k * n + l]

    out = {}
    for name, arr, n in (("hh", hh, nv), ("ee", ee, nc)):
        J = np.zeros((n // 2, n // 2))
        for P in range(n // 2):
            for Qp in range(n // 2):
                s = 0.0
                for i in (2 * P, 2 * P + 1):
                    for k in (2 * Qp, 2 * Qp + 1):
                        a, b = min(i, k), max(i, k)
                        s += v4(arr, n, a, a, b, b).real
                J[P, Qp] = s
        out[name] = J
    J = np.zeros((nv // 2, nc // 2))
    for P in range(nv // 2):
        for Qp in range(nc // 2):
            s = 0.0
            for i in (2 * P, 2 * P + 1):
                for k in (2 * Qp, 2 * Qp + 1):
                    s += ehd[i * nv * nc * nc + i * nc * nc + k * nc + k].real
            J[P, Qp] = s
    out["eh"] = J
    return out


def read_golden_direct(directory, nv, nc):
    """J_PQ from the reference's coulomb_matrix_elements_{hh,ee,eh_direct}.dat
    (written by write_coulomb_matrix_elements.c: hh columns are
    (nv - i, nv - k, nv - l, nv - j), ee (i+1, k+1, l+1, j+1), eh_direct
    (k+1, nv - i, nv - j, l+1), values V(i, j, k, l))."""
    import os

    def rows(name):
        out = {}
        with open(os.path.join(directory, name)) as f:
            for line in f:
                t = line.split()
                if len(t) < 7:
                    continue
                out[tuple(int(x) for x in t[:4])] = complex(float(t[4]), float(t[5]))
        return out

    hh = rows("coulomb_matrix_elements_hh.dat")
    ee = rows("coulomb_matrix_elements_ee.dat")
    eh = rows("coulomb_matrix_elements_eh_direct.dat")
    out = {}
    J = np.zeros((nv // 2, nv // 2))
    for P in range(nv // 2):
        for Qp in range(nv // 2):
            J[P, Qp] = sum(hh[(nv - i, nv - k, nv - k, nv - i)].real
                           for i in (2 * P, 2 * P + 1) for k in (2 * Qp, 2 * Qp + 1))
    out["hh"] = J
    J = np.zeros((nc // 2, nc // 2))
    for P in range(nc // 2):
        for Qp in range(nc // 2):
            J[P, Qp] = sum(ee[(i + 1, k + 1, k + 1, i + 1)].real
                           for i in (2 * P, 2 * P + 1) for k in (2 * Qp, 2 * Qp + 1))
    out["ee"] = J
    J = np.zeros((nv // 2, nc // 2))
    for P in range(nv // 2):
        for Qp in range(nc // 2):
            J[P, Qp] = sum(eh[(k + 1, nv - i, nv - i, k + 1)].real
                           for i in (2 * P, 2 * P + 1) for k in (2 * Qp, 2 * Qp + 1))
    out["eh"] = J
    return out

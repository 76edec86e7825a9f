"""Oracle restatement of the strain, piezoelectric and convolution tables.

Follows (test infrastructure):
  * ``strain_region_reciprocal_space.c:24-418`` + ``strain_fourier_coefficient.c:23-470``
    (position-independent elastic constants, and the perturbative position-dependent
    ones with ``convolutions_strain_correction.c:23-358``),
  * ``piezo_region_reciprocal_space.c:23-787`` + ``piezo_fourier_coefficient.c:24-132``,
  * ``strain_reciprocal_space.c:23-230`` / ``piezo_reciprocal_space.c:23-186``
    (free-length downsampling; the identity copy when the cells coincide),
  * ``strain_reciprocal_space_fft.c:23-362`` / ``piezo_reciprocal_space_fft.c``
    (commensurate strain cells SL = RL L: FFT convolution with the electronic
    cell's box, sampled at every RL-th strain-cell wave vector),
  * ``convolutions.c:24-411``.

Tables are numpy arrays of shape (N_xT, N_yT, N_zT) (flat index
iz + N_zT (iy + N_yT ix), as in the reference).  A "convolution" is the
reference's zero-padded FFT linear convolution on the (2 N_T - 1)^3 grid
cropped back to the central N_T^3 block.
"""

import numpy as np

COMPONENTS = ("xx", "yy", "zz", "yz", "xz", "xy")
_IJ = {"xx": (0, 0), "yy": (1, 1), "zz": (2, 2), "yz": (1, 2), "xz": (0, 2), "xy": (0, 1)}
EPS = 1.0e-08
# Second-order products (piezo_region_reciprocal_space.c:296-307) and their use in
# P = (Px, Py, Pz) (piezo_fourier_coefficient.c:79-91).
PRODUCTS = (("xx", "yz"), ("yy", "yz"), ("zz", "yz"), ("xy", "xz"), ("yy", "xz"), ("xx", "xz"),
            ("zz", "xz"), ("xy", "yz"), ("zz", "xy"), ("xx", "xy"), ("yy", "xy"), ("xz", "yz"))


def _grids(basis):
    Gx, Gy, Gz = basis["G"]
    return np.meshgrid(Gx, Gy, Gz, indexing="ij")


def strain_factor(comp, Gx, Gy, Gz, p0, isotropic):
    """Green-tensor factor multiplying eps0 * chi (strain_fourier_coefficient.c:108-173)."""
    i, j = _IJ[comp]
    G3 = (Gx, Gy, Gz)
    Gi, Gj = G3[i], G3[j]
    G = np.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    dij = 1.0 if i == j else 0.0
    C11, C12, C44 = p0["C11"], p0["C12"], p0["C44"]
    zero = np.abs(G) < EPS
    Gs = np.where(zero, 1.0, G)
    with np.errstate(divide="ignore", invalid="ignore"):
        if isotropic == 1:
            f0 = dij * (1.0 - (3.0 * C12 + 2.0 * C44) / (3.0 * C12 + 6.0 * C44))
            f = dij - (((3.0 * C12 + 2.0 * C44) * Gi * Gj) / ((C12 + 2.0 * C44) * Gs * Gs))
        else:
            D = C11 - C12 - 2.0 * C44
            s0 = 1.0 / (C44 + D / 3.0)
            f0 = dij * (1.0 - (0.5 * (C11 + 2.0 * C12) / 3.0) * (2.0 / (C44 + D / 3.0)) / (1.0 + (C12 + C44) * s0))
            s = ((Gx * Gx) / (C44 * Gs * Gs + D * Gx * Gx) + (Gy * Gy) / (C44 * Gs * Gs + D * Gy * Gy)
                 + (Gz * Gz) / (C44 * Gs * Gs + D * Gz * Gz))
            f = dij - (0.5 * (C11 + 2.0 * C12) * (2.0 * C44 * Gs * Gs + D * (Gi * Gi + Gj * Gj)) * Gi * Gj) / (
                (1.0 + (C12 + C44) * s) * (C44 * Gs * Gs + D * Gi * Gi) * (C44 * Gs * Gs + D * Gj * Gj))
    return np.where(zero, f0, f)


def green_tensor(comp, Gx, Gy, Gz, G, ssum, p0):
    """greens_function_tensor (strain_fourier_coefficient.c:394-470): the
    matrix material's elastic Green tensor component ij at G (G != 0)."""
    i, j = _IJ[comp]
    G3 = (Gx, Gy, Gz)
    Gi, Gj = G3[i], G3[j]
    C11, C12, C44 = p0["C11"], p0["C12"], p0["C44"]
    D = C11 - C12 - 2.0 * C44
    dij = 1.0 if i == j else 0.0
    return (dij / (C44 * G * G + D * Gi * Gi)) - ((C12 + C44) * Gi * Gj / (
        (1.0 + (C12 + C44) * ssum) * (C44 * G * G + D * Gi * Gi) * (C44 * G * G + D * Gj * Gj)))


def _order0_factor(comp, Gx, Gy, Gz, p0, ps, isotropic):
    """Zeroth-order factor of the position-dependent elastic constants
    (strain_fourier_coefficient.c:177-224): the shape's own C11, C12, C44 in the
    numerators, the matrix's in the Green tensor."""
    i, j = _IJ[comp]
    G3 = (Gx, Gy, Gz)
    Gi, Gj = G3[i], G3[j]
    G = np.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    dij = 1.0 if i == j else 0.0
    C11, C12, C44 = p0["C11"], p0["C12"], p0["C44"]
    zero = np.abs(G) < EPS
    Gs = np.where(zero, 1.0, G)
    with np.errstate(divide="ignore", invalid="ignore"):
        if isotropic == 1:
            f0 = dij * (-1 * (3.0 * ps["C12"] + 2.0 * ps["C44"]) / (3.0 * C12 + 6.0 * C44))
            f = -((3.0 * ps["C12"] + 2.0 * ps["C44"]) * Gi * Gj) / ((C12 + 2.0 * C44) * Gs * Gs)
        else:
            D = C11 - C12 - 2.0 * C44
            s0 = 1.0 / (C44 + D / 3.0)
            f0 = dij * ((-0.5 * (ps["C11"] + 2.0 * ps["C12"]) / 3.0) * (2.0 / (C44 + D / 3.0))
                        / (1.0 + (C12 + C44) * s0))
            ssum = ((Gx * Gx) / (C44 * Gs * Gs + D * Gx * Gx) + (Gy * Gy) / (C44 * Gs * Gs + D * Gy * Gy)
                    + (Gz * Gz) / (C44 * Gs * Gs + D * Gz * Gz))
            f = -(0.5 * (ps["C11"] + 2.0 * ps["C12"]) * (2.0 * C44 * Gs * Gs + D * (Gi * Gi + Gj * Gj)) * Gi * Gj) / (
                (1.0 + (C12 + C44) * ssum) * (C44 * Gs * Gs + D * Gi * Gi) * (C44 * Gs * Gs + D * Gj * Gj))
    return np.where(zero, f0, f)


def _correction_factor(comp, Gx, Gy, Gz, p0, ps, isotropic):
    """Factor multiplying chi_s (*) (previous correction) for correction orders
    >= 1 (strain_fourier_coefficient.c:226-386)."""
    G = np.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    zero = np.abs(G) < EPS
    Gs = np.where(zero, 1.0, G)
    C11, C12, C44 = p0["C11"], p0["C12"], p0["C44"]
    D = C11 - C12 - 2.0 * C44
    dC11, dC12, dC44 = ps["C11"] - C11, ps["C12"] - C12, ps["C44"] - C44
    i, j = _IJ[comp]
    if isotropic == 1:
        f0 = -(1.0 / (3.0 * C44)) * (ps["C11"] - C11 + 2.0 * ps["C12"] - 2.0 * C12) if i == j else 0.0
    else:
        s0 = 1.0 / (C44 + D / 3.0)
        f0 = -(s0 / 3.0) * (ps["C11"] - C11 + 2.0 * ps["C12"] - 2.0 * C12) if i == j else 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        ssum = ((Gx * Gx) / (C44 * Gs * Gs + D * Gx * Gx) + (Gy * Gy) / (C44 * Gs * Gs + D * Gy * Gy)
                + (Gz * Gz) / (C44 * Gs * Gs + D * Gz * Gz))

        def g(c):
            return green_tensor(c, Gx, Gy, Gz, Gs, ssum, p0)
        G3 = (Gx, Gy, Gz)
        Gi, Gj = G3[i], G3[j]
        if comp == "xx":
            f = -1.0 * (Gi * ((dC11 * Gx * g("xx")) + (dC12 * Gy * g("xy")) + (dC12 * Gz * g("xz"))))
        elif comp == "yy":
            f = -1.0 * (Gi * ((dC12 * Gx * g("xy")) + (dC11 * Gy * g("yy")) + (dC12 * Gz * g("yz"))))
        elif comp == "zz":
            f = -1.0 * (Gi * ((dC12 * Gx * g("xz")) + (dC12 * Gy * g("yz")) + (dC11 * Gz * g("zz"))))
        elif comp == "yz":
            f = -0.5 * dC44 * (Gi * ((Gz * g("yz")) + (Gy * g("zz"))) + Gj * ((Gz * g("yy")) + (Gy * g("yz"))))
        elif comp == "xz":
            f = -0.5 * dC44 * (Gi * ((Gz * g("xz")) + (Gx * g("zz"))) + Gj * ((Gz * g("xx")) + (Gx * g("xz"))))
        else:
            f = -0.5 * dC44 * (Gi * ((Gy * g("xy")) + (Gx * g("yy"))) + Gj * ((Gy * g("xx")) + (Gx * g("xy"))))
    return np.where(zero, f0, f)


def strain_region(basis, geo, params, chi_strain, isotropic, elastic_const=0, order=0):
    """epsilon_ij(G) on the strain grid (strain_region_reciprocal_space.c:24-418).

    elastic_const 0: position-independent elastic constants (the matrix's).
    elastic_const 1: the perturbative treatment of each shape's own constants,
    per shape: the initial term eps0 chi delta_ij, the zeroth-order term with
    the shape's constants, then ``order`` corrections, each the convolution of
    chi_s with the previous correction (zero-padded FFT, central block) times
    the Green-tensor factor of the constant differences."""
    if isotropic != 0:
        for p in params:
            p["C44"] = 0.5 * (p["C11"] - p["C12"])
    Gx, Gy, Gz = _grids(basis)
    eps = {c: np.zeros(Gx.shape, dtype=np.complex128) for c in COMPONENTS}
    if elastic_const == 0:
        fac = {c: strain_factor(c, Gx, Gy, Gz, params[0], isotropic) for c in COMPONENTS}
        for s in range(1, len(geo)):
            eps0 = (params[geo[s]["embedded"]]["a"] - params[s]["a"]) / params[0]["a"]
            for c in COMPONENTS:
                eps[c] += eps0 * chi_strain[s] * fac[c]
        return eps
    n = Gx.shape
    for s in range(1, len(geo)):
        ps = params[s]
        eps0 = (params[geo[s]["embedded"]]["a"] - ps["a"]) / params[0]["a"]
        for c in COMPONENTS:
            if _IJ[c][0] == _IJ[c][1]:
                eps[c] += eps0 * chi_strain[s]
        corr = {c: eps0 * chi_strain[s] * _order0_factor(c, Gx, Gy, Gz, params[0], ps, isotropic)
                for c in COMPONENTS}
        for c in COMPONENTS:
            eps[c] += corr[c]
        X = np.fft.fftn(pad(chi_strain[s]))
        for _ in range(order):
            conv = {c: conv_hat(X, np.fft.fftn(pad(corr[c])), n) for c in COMPONENTS}
            corr = {c: conv[c] * _correction_factor(c, Gx, Gy, Gz, params[0], ps, isotropic) for c in COMPONENTS}
            for c in COMPONENTS:
                eps[c] += corr[c]
    return eps


def pad(a):
    n = a.shape
    out = np.zeros(tuple(2 * k - 1 for k in n), dtype=np.complex128)
    out[: n[0], : n[1], : n[2]] = a
    return out


def crop(a, n):
    return a[n[0] // 2: n[0] // 2 + n[0], n[1] // 2: n[1] // 2 + n[1], n[2] // 2: n[2] // 2 + n[2]]


def conv_hat(A_hat, B_hat, n):
    """Central block of IFFT(A_hat * B_hat) (backward scale 1/size)."""
    return crop(np.fft.ifftn(A_hat * B_hat), n)


def piezo_coefficient(order, shape_idx, basis, geo, params, tab):
    """Contribution to phi(G) (piezo_fourier_coefficient.c:24-132).  ``tab`` holds
    the arrays the reference reads for this (order, shape)."""
    Gx, Gy, Gz = _grids(basis)
    G = np.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    p0 = params[0]
    if order == 1:
        if shape_idx == 0:
            e = p0["e14"]
            Px, Py, Pz = 2.0 * e * tab["yz"], 2.0 * e * tab["xz"], 2.0 * e * tab["xy"]
        else:
            e = params[shape_idx]["e14"] - params[geo[shape_idx]["embedded"]]["e14"]
            Px, Py, Pz = 2.0 * e * tab["char_yz"], 2.0 * e * tab["char_xz"], 2.0 * e * tab["char_xy"]
    else:
        if shape_idx == 0:
            B114, B124, B156 = p0["B114"], p0["B124"], p0["B156"]
            pre = ""
        else:
            pe = params[geo[shape_idx]["embedded"]]
            ps = params[shape_idx]
            B114, B124, B156 = ps["B114"] - pe["B114"], ps["B124"] - pe["B124"], ps["B156"] - pe["B156"]
            pre = "char_"
        t = lambda a, b: tab[pre + a + "_" + b]
        Px = 2.0 * B114 * t("xx", "yz") + 2.0 * B124 * t("yy", "yz") + 2.0 * B124 * t("zz", "yz") + 4.0 * B156 * t("xy", "xz")
        Py = 2.0 * B114 * t("yy", "xz") + 2.0 * B124 * t("xx", "xz") + 2.0 * B124 * t("zz", "xz") + 4.0 * B156 * t("xy", "yz")
        Pz = 2.0 * B114 * t("zz", "xy") + 2.0 * B124 * t("xx", "xy") + 2.0 * B124 * t("yy", "xy") + 4.0 * B156 * t("xz", "yz")
    with np.errstate(divide="ignore", invalid="ignore"):
        r = (-100.0j * (Gx * Px + Gy * Py + Gz * Pz)) / (8.854188 * p0["nr"] ** 2.0 * G ** 2.0)
    return np.where(G > EPS, r, 0.0)


def piezo_region(basis, geo, params, chi_strain, eps, include_piezo):
    """phi_pz(G) on the strain grid (piezo_region_reciprocal_space.c:23-787).
    First order is always added (the reference adds it unconditionally inside the
    routine); second order for Piezo = 2 or 3."""
    n = eps["xx"].shape
    E = {c: np.fft.fftn(pad(eps[c])) for c in COMPONENTS}
    phi = np.zeros(n, dtype=np.complex128)
    phi += piezo_coefficient(1, 0, basis, geo, params, eps)
    second = include_piezo in (2, 3)
    F = {}
    if second:
        prod = {a + "_" + b: conv_hat(E[a], E[b], n) for a, b in PRODUCTS}
        phi += piezo_coefficient(2, 0, basis, geo, params, prod)
        F = {k: np.fft.fftn(pad(v)) for k, v in prod.items()}
    for s in range(1, len(geo)):
        X = np.fft.fftn(pad(chi_strain[s]))
        tab = {"char_" + c: conv_hat(X, E[c], n) for c in COMPONENTS}
        phi += piezo_coefficient(1, s, basis, geo, params, tab)
        if second:
            tab2 = {"char_" + k: conv_hat(X, F[k], n) for k in F}
            phi += piezo_coefficient(2, s, basis, geo, params, tab2)
    return phi


def _axis_factor(Gs, Ge, L, same):
    """1-D factor of the free-length downsampling kernel (strain_reciprocal_space.c:113-137)."""
    if same:
        return np.diag(np.full(len(Ge), L))
    d = Gs[:, None] - Ge[None, :]
    with np.errstate(divide="ignore", invalid="ignore"):
        f = 2 * np.sin(d * L / 2) / d
    return np.where(np.abs(d) < EPS, L, f)


def downsample(table_s, basis, strain_basis, geo):
    """Strain-cell table -> electronic-structure cell for free lengths
    (strain_reciprocal_space.c:23-230, piezo_reciprocal_space.c:23-186):
    T_es(G) = (1/V_es) sum_GS T_s(GS) prod_a I0(GS_a - G_a), which is the identity
    (times V_es/V_es) when the two cells coincide."""
    g0 = geo[0]
    L = (g0["L1"], g0["L2"], g0["L3"])
    SL = (g0["SL1"], g0["SL2"], g0["SL3"])
    inv_v = 1.0 / (L[0] * L[1] * L[2])
    same = [basis["N"][a] == strain_basis["N"][a] and L[a] == SL[a] for a in range(3)]
    if all(same):
        return ((inv_v * table_s) * L[0]) * L[1] * L[2]
    Mx = _axis_factor(strain_basis["G"][0], basis["G"][0], L[0], same[0])
    My = _axis_factor(strain_basis["G"][1], basis["G"][1], L[1], same[1])
    Mz = _axis_factor(strain_basis["G"][2], basis["G"][2], L[2], same[2])
    return inv_v * np.einsum("abc,ai,bj,ck->ijk", table_s, Mx, My, Mz)


def downsample_commensurate(table_s, basis, strain_basis, geo, softening=0, sigma=0.0):
    """Strain-cell table -> electronic-structure cell for commensurate lengths
    (Strain_supercell_type 1, strain_reciprocal_space_fft.c:23-362 and
    piezo_reciprocal_space_fft.c, the same steps for phi): chi_0, the
    electronic cell's cuboid (shape record 0, normalised by the electronic cell
    volume, softened like every shape) on the strain grid, and the table are
    zero-padded to (2 N_ST - 1)^3, multiplied after a forward FFT and
    transformed back (backward scale 1/size); the electronic-cell coefficient of
    index i is the element RL i + N_ST - 1 - RL (N_T / 2) of the result along
    each axis."""
    from . import shapes
    chi0 = shapes.chi_table(strain_basis, geo, 0, 2, softening, sigma)
    conv = np.fft.ifftn(np.fft.fftn(pad(chi0)) * np.fft.fftn(pad(table_s)))
    g0 = geo[0]
    RL = (g0["RL1"], g0["RL2"], g0["RL3"])
    nS = table_s.shape
    nE = basis["N_T"]
    idx = [RL[a] * np.arange(nE[a]) + nS[a] - 1 - RL[a] * (nE[a] // 2) for a in range(3)]
    return conv[np.ix_(*idx)]


def strain_grid_too_small(p, geo):
    """8_band_main.c:159-192: with commensurate strain cells, M_S must reach
    about M RL / 2 along every axis.  Returns the axes that fail."""
    g0 = geo[0]
    bad = []
    for a, ax in enumerate("xyz"):
        n, ns, rl = p["N_G" + ax], p["N_S_G" + ax], g0["RL%d" % (a + 1)]
        if ns // 2 < (n // 2) * rl // 2 + ((n // 2) % 2) * (rl % 2):
            bad.append(ax)
    return bad


def convolutions(chi_es, strain_es, n_shape):
    """chi_s (*) epsilon_ij, hydrostatic and biaxial combinations (convolutions.c:24-411)."""
    n = strain_es["xx"].shape
    E = {c: np.fft.fftn(pad(strain_es[c])) for c in COMPONENTS}
    out = [None]
    for s in range(1, n_shape):
        X = np.fft.fftn(pad(chi_es[s]))
        t = {c: conv_hat(X, E[c], n) for c in COMPONENTS}
        t["hydrostatic"] = t["xx"] + t["yy"] + t["zz"]
        t["biaxial"] = t["xx"] + t["yy"] - 2.0 * t["zz"]
        out.append(t)
    return out

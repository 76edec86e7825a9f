"""Oracle restatement of the 8-band supercell Hamiltonian assembly (test infrastructure).

Follows ``code/source/8_band/hamiltonian_8_band.c:23-500`` (lower triangle,
column-major, band block map), ``hamiltonian_8_band_matrix_elements.c:27-969``
(the twelve band functions), ``parameter_matrix_element.c:23-48`` and
``field_fourier_coefficient.c:23-55``.  Each band function is evaluated for a
whole (row plane wave) x (column plane wave) block with numpy broadcasting.
"""

import math

import numpy as np

HBSQM = 7.61996

# (row band, column band) -> (factor, band function) for row >= col, 1-based bands
# CB, HH, LH, SO, CB, HH, LH, SO (hamiltonian_8_band.c:78-492).  Unlisted pairs are 0.
S2, S3 = math.sqrt(2.0), math.sqrt(3.0)
BLOCK_MAP = {
    (1, 1): (1.0, "E_CB"), (2, 1): (-S3, "T_minus"), (3, 1): (S2, "U"), (4, 1): (-1.0, "U"),
    (7, 1): (-1.0, "T_plus"), (8, 1): (-S2, "T_plus"),
    (2, 2): (1.0, "E_HH"), (3, 2): (S2, "S_conj"), (4, 2): (-1.0, "S_conj"),
    (7, 2): (-1.0, "R_conj"), (8, 2): (-S2, "R_conj"),
    (3, 3): (1.0, "E_LH"), (4, 3): (1.0, "Q"), (5, 3): (1.0, "T_plus"), (6, 3): (1.0, "R_conj"),
    (8, 3): (S3, "S_conj"),
    (4, 4): (1.0, "E_SO"), (5, 4): (S2, "T_plus"), (6, 4): (S2, "R_conj"), (7, 4): (-S3, "S_conj"),
    (5, 5): (1.0, "E_CB"), (6, 5): (-S3, "T_plus"), (7, 5): (S2, "U"), (8, 5): (-1.0, "U"),
    (6, 6): (1.0, "E_HH"), (7, 6): (S2, "S"), (8, 6): (-1.0, "S"),
    (7, 7): (1.0, "E_LH"), (8, 7): (1.0, "Q"),
    (8, 8): (1.0, "E_SO"),
}


class Tables:
    """Inputs of the assembly: the global arrays of the reference
    (8_band.h:218-225) for the electronic-structure cell."""

    def __init__(self, chi, strain=None, conv=None, phi=None):
        self.chi = chi          # list, index 0 unused; arrays (N_xT, N_yT, N_zT)
        self.strain = strain    # dict of the 6 components or None
        self.conv = conv        # list per shape of dicts (xx..xy, hydrostatic, biaxial)
        self.phi = phi          # piezo potential or None


class BlockContext:
    def __init__(self, basis, geo, params, tables, F, include_strain, include_piezo, rows, cols,
                 paired=False):
        Nx, Ny, Nz = basis["N"]
        NTx, NTy, NTz = basis["N_T"]
        self.b, self.geo, self.p, self.t = basis, geo, params, tables
        self.F = F
        self.strain_on = include_strain != 0 and tables.strain is not None
        self.piezo_on = self.strain_on and include_piezo != 0 and tables.phi is not None

        def dec(idx):
            return idx // (Ny * Nz), (idx % (Ny * Nz)) // Nz, (idx % (Ny * Nz)) % Nz

        if paired:
            r = dec(np.asarray(rows))
            c = dec(np.asarray(cols))
        else:
            r = dec(np.asarray(rows)[:, None])
            c = dec(np.asarray(cols)[None, :])
        self.r, self.c = r, c
        self.d = [r[a] - c[a] for a in range(3)]
        self.didx = (self.d[0] + NTx // 2, self.d[1] + NTy // 2, self.d[2] + NTz // 2)
        offs = [NTx // 2 - Nx // 2, NTy // 2 - Ny // 2, NTz // 2 - Nz // 2]
        G = basis["G"]
        self.g1 = [G[a][offs[a] + r[a]] for a in range(3)]
        self.g2 = [G[a][offs[a] + c[a]] for a in range(3)]
        self.K = basis["K"]
        self.delta0 = (self.d[0] == 0) & (self.d[1] == 0) & (self.d[2] == 0)

    def tab(self, a):
        return a[self.didx]

    def pme(self, name, fn=None):
        """parameter_matrix_element.c:23-48."""
        val = (lambda q: fn(q)) if fn else (lambda q: q[name])
        out = val(self.p[0]) * self.delta0.astype(np.float64)
        out = out.astype(np.complex128)
        for s in range(1, len(self.geo)):
            out = out + (val(self.p[s]) - val(self.p[self.geo[s]["embedded"]])) * self.tab(self.t.chi[s])
        return out

    def kin(self, a):
        """G1_a G2_a + K_a (G1_a + G2_a) (+ K_a^2 added by the caller)."""
        return self.g1[a] * self.g2[a] + self.K[a] * (self.g1[a] + self.g2[a])

    def ksum(self, a):
        return self.g1[a] + self.g2[a] + 2 * self.K[a]

    def field(self):
        """field_fourier_coefficient.c:23-55."""
        out = np.zeros(self.delta0.shape, dtype=np.complex128)
        F = (self.F[0], self.F[1], self.F[2])
        G = self.b["G"]
        NT = self.b["N_T"]
        N = self.b["N"]
        for a in range(3):
            o = [b for b in range(3) if b != a]
            m = (self.d[a] != 0) & (self.d[o[0]] == 0) & (self.d[o[1]] == 0)
            if F[a] == 0.0 or not np.any(m):
                continue
            off = NT[a] // 2 - N[a] // 2
            g1 = G[a][off + self.r[a]] + 0 * self.c[a]
            g2 = G[a][off + self.c[a]] + 0 * self.r[a]
            sign = np.where((self.d[a] + 1) % 2 == 0, 1.0, -1.0)
            with np.errstate(divide="ignore", invalid="ignore"):
                val = (1j * F[a] * sign) / (g2 - g1)
            out = out + np.where(m, val, 0.0)
        return out


def band_function(ctx, name):
    p0, geo, t = ctx.p[0], ctx.geo, ctx.t
    pd = lambda s, k: ctx.p[s][k] - ctx.p[geo[s]["embedded"]][k]
    st = (lambda c: ctx.tab(t.strain[c])) if ctx.strain_on else None
    cv = (lambda s, c: ctx.tab(t.conv[s][c])) if ctx.strain_on else None
    ns = len(geo)
    Kx, Ky, Kz = ctx.K
    I = 1j
    if name in ("E_CB", "E_HH", "E_LH", "E_SO"):
        if name == "E_CB":
            r = ctx.pme("E_cb")
            r = r + 0.5 * HBSQM * ctx.pme("sc") * (ctx.kin(0) + ctx.kin(1) + ctx.kin(2) + Kx * Kx + Ky * Ky + Kz * Kz)
        elif name == "E_SO":
            r = ctx.pme("E_so")
            r = r + -0.5 * HBSQM * ctx.pme("g1") * (ctx.kin(0) + ctx.kin(1) + ctx.kin(2) + Kx * Kx + Ky * Ky + Kz * Kz)
        else:
            if name == "E_HH":
                e, fa, fb = "E_hh", (lambda q: q["g1"] + q["g2"]), (lambda q: q["g1"] - 2.0 * q["g2"])
            else:
                e, fa, fb = "E_lh", (lambda q: q["g1"] - q["g2"]), (lambda q: q["g1"] + 2.0 * q["g2"])
            r = ctx.pme(e)
            r = (r + -0.5 * HBSQM * ctx.pme(None, fa) * (ctx.kin(0) + ctx.kin(1) + Kx * Kx + Ky * Ky)
                 - 0.5 * HBSQM * ctx.pme(None, fb) * (ctx.kin(2) + Kz * Kz))
        if ctx.strain_on:
            tr = st("xx") + st("yy") + st("zz")
            bi = st("xx") + st("yy") - 2.0 * st("zz")
            if name == "E_CB":
                r = r + p0["ac"] * tr
                for s in range(1, ns):
                    r = r + pd(s, "ac") * cv(s, "hydrostatic")
            elif name == "E_SO":
                r = r + p0["av"] * tr
                for s in range(1, ns):
                    r = r + pd(s, "av") * cv(s, "hydrostatic")
            else:
                sg = 1.0 if name == "E_HH" else -1.0
                r = r + (p0["av"] * tr + sg * 0.5 * p0["b"] * bi)
                for s in range(1, ns):
                    r = r + pd(s, "av") * cv(s, "hydrostatic") + sg * 0.5 * pd(s, "b") * cv(s, "biaxial")
            if ctx.piezo_on:
                r = r + ctx.tab(t.phi)
        r = r + ctx.field()
        return r
    if name == "Q":
        g2 = ctx.pme("g2")
        r = (-1.0 * math.sqrt(0.5) * HBSQM * g2 * (ctx.kin(0) + ctx.kin(1) + Kx * Kx + Ky * Ky)
             + math.sqrt(2.0) * HBSQM * g2 * (ctx.kin(2) + Kz * Kz))
        if ctx.strain_on:
            r = r + math.sqrt(0.5) * p0["b"] * (st("xx") + st("yy") - 2.0 * st("zz"))
            for s in range(1, ns):
                r = r + math.sqrt(0.5) * pd(s, "b") * cv(s, "biaxial")
        return r
    if name in ("R", "R_conj"):
        sg = -1.0 if name == "R" else 1.0
        g1x, g1y = ctx.g1[0] + Kx, ctx.g1[1] + Ky
        g2x, g2y = ctx.g2[0] + Kx, ctx.g2[1] + Ky
        r = (0.5 * math.sqrt(3.0) * HBSQM * ctx.pme("g2") * (ctx.kin(0) - ctx.kin(1) + Kx * Kx - Ky * Ky)
             + sg * I * 0.5 * math.sqrt(3.0) * HBSQM * ctx.pme("g3") * (g1x * g2y + g1y * g2x))
        if ctx.strain_on:
            r = r + (-0.5 * math.sqrt(3.0) * p0["b"] * (st("xx") - st("yy")) - sg * I * p0["d"] * st("xy"))
            for s in range(1, ns):
                r = r + (-0.5 * math.sqrt(3.0) * pd(s, "b") * (cv(s, "xx") - cv(s, "yy"))
                         - sg * I * pd(s, "d") * cv(s, "xy"))
        return r
    if name in ("S", "S_conj"):
        sg = -1.0 if name == "S" else 1.0
        g1x, g1y, g1z = ctx.g1[0] + Kx, ctx.g1[1] + Ky, ctx.g1[2] + Kz
        g2x, g2y, g2z = ctx.g2[0] + Kx, ctx.g2[1] + Ky, ctx.g2[2] + Kz
        g3 = ctx.pme("g3")
        r = (0.5 * math.sqrt(1.5) * HBSQM * g3 * (g1x * g2z + g1z * g2x)
             + sg * I * 0.5 * math.sqrt(1.5) * HBSQM * g3 * (g1y * g2z + g1z * g2y))
        if ctx.strain_on:
            r = r + -1.0 * math.sqrt(0.5) * p0["d"] * (st("xz") + sg * I * st("yz"))
            for s in range(1, ns):
                r = r + -1.0 * math.sqrt(0.5) * pd(s, "d") * (cv(s, "xz") + sg * I * cv(s, "yz"))
        return r
    if name in ("T_plus", "T_minus"):
        sg = 1.0 if name == "T_plus" else -1.0
        P = ctx.pme("P")
        kx, ky, kz = ctx.ksum(0), ctx.ksum(1), ctx.ksum(2)
        r = (P * kx) / (2.0 * math.sqrt(6.0)) + sg * (I * P * ky) / (2.0 * math.sqrt(6.0))
        if ctx.strain_on:
            c = -0.5 / math.sqrt(6)
            r = r + c * p0["P"] * ((st("xx") + sg * I * st("xy")) * kx + (st("xy") + sg * I * st("yy")) * ky
                                   + (st("xz") + sg * I * st("yz")) * kz)
            for s in range(1, ns):
                r = r + c * pd(s, "P") * (kx * (cv(s, "xx") + sg * I * cv(s, "xy"))
                                          + ky * (cv(s, "xy") + sg * I * cv(s, "yy"))
                                          + kz * (cv(s, "xz") + sg * I * cv(s, "yz")))
        return r
    if name == "U":
        P = ctx.pme("P")
        kx, ky, kz = ctx.ksum(0), ctx.ksum(1), ctx.ksum(2)
        r = (P * kz) / (2.0 * math.sqrt(3.0))
        if ctx.strain_on:
            c = -0.5 / math.sqrt(3)
            r = r + c * p0["P"] * (st("xz") * kx + st("yz") * ky + st("zz") * kz)
            for s in range(1, ns):
                r = r + c * pd(s, "P") * (kx * cv(s, "xz") + ky * cv(s, "yz") + kz * cv(s, "zz"))
        return r
    raise KeyError(name)


def assemble(basis, geo, params, tables, F, include_strain, include_piezo, full=False):
    """H (N_H x N_H complex128).  Lower triangle as the reference writes it
    (upper left zero); with ``full`` the upper triangle is the Hermitian mirror."""
    Nx, Ny, Nz = basis["N"]
    npw = Nx * Ny * Nz
    nh = 8 * npw
    H = np.zeros((nh, nh), dtype=np.complex128)
    idx = np.arange(npw)
    ctx = BlockContext(basis, geo, params, tables, F, include_strain, include_piezo, idx, idx)
    cache = {}
    for (rb, cb), (fac, name) in BLOCK_MAP.items():
        if name not in cache:
            cache[name] = band_function(ctx, name)
        blk = fac * cache[name]
        r0, c0 = (rb - 1) * npw, (cb - 1) * npw
        if rb == cb:
            blk = np.tril(blk)
        H[r0:r0 + npw, c0:c0 + npw] = blk
    if full:
        H = H + np.tril(H, -1).conj().T
    return H


def assemble_entries(basis, geo, params, tables, F, include_strain, include_piezo, rows, cols):
    """H[rows[k], cols[k]] for arbitrary (row >= col) index pairs, without
    building the matrix (used for spot checks at large N_H)."""
    Nx, Ny, Nz = basis["N"]
    npw = Nx * Ny * Nz
    rows = np.asarray(rows)
    cols = np.asarray(cols)
    out = np.zeros(rows.shape, dtype=np.complex128)
    rb = rows // npw + 1
    cb = cols // npw + 1
    for (b_r, b_c), (fac, name) in BLOCK_MAP.items():
        m = (rb == b_r) & (cb == b_c)
        if not np.any(m):
            continue
        ctx = BlockContext(basis, geo, params, tables, F, include_strain, include_piezo,
                           rows[m] % npw, cols[m] % npw, paired=True)
        out[m] = fac * band_function(ctx, name)
    return out

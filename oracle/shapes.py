"""Oracle restatement of the plane-wave grids and the shape Fourier transforms.

Follows ``code/source/8_band/basis_set.c:23-90``,
``code/source/8_band/characteristic_function_fourier.c:58-1411`` and
``code/source/8_band/characteristic_function_fourier_integrals.c:28-153``
(test infrastructure).

All 19 shapes of the reference: 0 cuboid, 1 sphere, 2 ellipsoid, 3
hemisphere, 4 lens (hemi-ellipsoid), 5 rectangular pyramid, 6 truncated
rectangular pyramid, 7 N-sided pyramid, 8 truncated N-sided pyramid, 9
cylinder, 10 cylindrical ring, 11 cone, 12 truncated cone, 13 truncated conic
ring, 14 elliptical cone, 15 truncated elliptical cone, 16 N-sided prism, 17
quantum well, 18 quantum wire.  The one-dimensional integrals of the curved
shapes (I_J0, I_2 and its variants, characteristic_function_fourier_integrals.c)
use the restated GSL QAG of ``quadrature``.  Every function is scalar and is
looped over by ``chi_table``; the oracle is meant for small grids.
"""

import cmath
import math

import numpy as np
from scipy.special import j0, j1

EPS = 1.0e-08


def basis_grid(n_T, L):
    """G_i = (2 pi / L)(0.5 (1 - n_T) + i), i < n_T (basis_set.c:62-85)."""
    i = np.arange(n_T, dtype=np.float64)
    return ((2.0 * math.pi) / L) * (0.5 * (1.0 - float(n_T)) + i)


def make_basis(N, L, K=(0.0, 0.0, 0.0)):
    """Basis with N plane waves per axis and grids of length 2N-1 (8_band_main.c:206-227)."""
    b = {"N": tuple(int(n) for n in N), "N_T": tuple(2 * int(n) - 1 for n in N), "K": tuple(K)}
    b["G"] = tuple(basis_grid(2 * int(n) - 1, l) for n, l in zip(N, L))
    return b


def _lround(x):
    """C lround: nearest integer, halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def sinc_pi(x):
    """gsl_sf_sinc: sin(pi x)/(pi x)."""
    return float(np.sinc(x))


# Gauss-Legendre rule for the cross-check of I_J0 (i_j0_gauss_legendre)
_GL_X, _GL_W = np.polynomial.legendre.leggauss(96)
_GL_X = 0.5 * (_GL_X + 1.0)
_GL_W = 0.5 * _GL_W


def _i_j0_integrand(alpha, beta):
    return lambda x: x * np.cos(alpha * np.sqrt(np.maximum(1.0 - x * x, 0.0))) * j0(beta * x)


def i_j0(alpha, beta):
    """I_J0(alpha, beta) = int_0^1 x cos(alpha sqrt(1-x^2)) J0(beta x) dx by the
    reference's method: gsl_integration_qag with the 61-point Gauss-Kronrod
    rule and EPS_ABS = EPS_REL = 1e-4, LIMIT = 1000
    (characteristic_function_fourier_integrals.c:107-153, 8_band.h:61-63),
    restated in ``quadrature.qag61``."""
    from .quadrature import qag61
    return qag61(_i_j0_integrand(alpha, beta), 0.0, 1.0, 1.0e-4, 1.0e-4, 1000)[0]


def i_j0_gauss_legendre(alpha, beta):
    """The same integral by a 96-point Gauss-Legendre rule (the rule the CUDA
    table kernel uses); cos(alpha sqrt(1-x^2)) is a power series in (1 - x^2),
    so the integrand is entire and both rules converge to rounding."""
    x = _GL_X
    return float(np.sum(_GL_W * _i_j0_integrand(alpha, beta)(x)))


def _qag(f, lo, hi):
    from .quadrature import qag61
    return qag61(f, lo, hi, 1.0e-4, 1.0e-4, 1000)[0]


def i_2(alpha, beta):
    """I_2 = int_0^1 x J0(alpha x) exp(i beta x) dx, real and imaginary parts by
    separate QAG calls (characteristic_function_fourier_integrals.c:217-285)."""
    re = _qag(lambda x: x * j0(alpha * x) * np.cos(beta * x), 0.0, 1.0)
    im = _qag(lambda x: x * j0(alpha * x) * np.sin(beta * x), 0.0, 1.0)
    return complex(re, im)


def i_2_gz(alpha):
    """int_0^1 x^2 J0(alpha x) dx (characteristic_function_fourier_integrals.c:342-390)."""
    return complex(_qag(lambda x: x * x * j0(alpha * x), 0.0, 1.0), 0.0)


def i_2_tc(alpha, R1, R2, beta):
    """int_{R1/(R2-R1)}^{R2/(R2-R1)} x J0((R2-R1) alpha x) exp(i beta x) dx
    (characteristic_function_fourier_integrals.c:451-521)."""
    lo, hi = R1 / (R2 - R1), R2 / (R2 - R1)
    a = (R2 - R1) * alpha
    re = _qag(lambda x: x * j0(a * x) * np.cos(beta * x), lo, hi)
    im = _qag(lambda x: x * j0(a * x) * np.sin(beta * x), lo, hi)
    return complex(re, im)


def i_2_tc_gz(alpha, R1, R2):
    """int_{R1/(R2-R1)}^{R2/(R2-R1)} x^2 J0((R2-R1) alpha x) dx
    (characteristic_function_fourier_integrals.c:577-627)."""
    lo, hi = R1 / (R2 - R1), R2 / (R2 - R1)
    a = (R2 - R1) * alpha
    return complex(_qag(lambda x: x * x * j0(a * x), lo, hi), 0.0)


def i_2_etc(alpha, beta, f):
    """int_f^1 x J0(alpha x) exp(i beta x / (1 - f)) dx
    (characteristic_function_fourier_integrals.c:688-757)."""
    b = beta / (1.0 - f)
    re = _qag(lambda x: x * j0(alpha * x) * np.cos(b * x), f, 1.0)
    im = _qag(lambda x: x * j0(alpha * x) * np.sin(b * x), f, 1.0)
    return complex(re, im)


def i_2_etc_gz(alpha, f):
    """int_f^1 x^2 J0(alpha x) dx (characteristic_function_fourier_integrals.c:813-861)."""
    return complex(_qag(lambda x: x * x * j0(alpha * x), f, 1.0), 0.0)


def i_e0(a, G):
    """characteristic_function_fourier_integrals.c:28-47."""
    if abs(G) < EPS:
        return complex(a)
    return (cmath.exp(1j * G * a) - 1.0) / (1j * G)


def pyramid_segment(Gx0, Gy0, Gz0, idx_side, N_side, g):
    """characteristic_function_fourier.c:1112-1296."""
    L1, L2, L3 = g["L1"], g["L2"], g["L3"]
    if N_side == 0:
        if idx_side in (0, 2):
            alpha = math.atan(L2 / L1)
        else:
            alpha = math.atan(L1 / L2)
    else:
        alpha = math.pi / float(N_side)
    if N_side == 0 and idx_side in (0, 2):
        x0, y0 = L1, L2
    elif N_side == 0 and idx_side in (1, 3):
        x0, y0 = L2, L1
    else:
        x0, y0 = L1, math.tan(alpha) * L1
    h = L3 if N_side == 0 else L2
    ang = 2.0 * alpha * float(idx_side)
    Gx = math.cos(ang) * Gx0 + math.sin(ang) * Gy0
    Gy = -1.0 * math.sin(ang) * Gx0 + math.cos(ang) * Gy0
    Gz = Gz0
    G_mag = math.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    I = 1j
    ex = cmath.exp
    if abs(G_mag) < EPS:
        return (x0 * y0 * h) / 3.0
    if abs(Gx) < EPS and abs(Gy) < EPS:
        return ((I * 2.0 * y0 * x0) / Gz) * ((1.0 - I * Gz * h - ex(-1.0 * I * Gz * h)) / (Gz * Gz * h * h) - 0.5)
    if abs(Gx) < EPS and abs(Gz) < EPS:
        return ((2.0 * h * x0) / (Gy * Gy * y0)) * (1.0 - math.sin(Gy * y0) / (Gy * y0))
    if abs(Gy) < EPS and abs(Gz) < EPS:
        return ((2.0 * h * y0) / (Gx * Gx * x0)) * (-1.0 - ex(-1.0 * I * Gx * x0) - (2.0 * I) / (Gx * x0)
                                                   + 2.0 * I * ex(-1.0 * I * Gx * x0) / (Gx * x0))
    if abs(Gx) < EPS:
        c = 2.0 * (math.cos(Gy * y0) - 1.0) / (Gy * y0)
        pre = (-1.0 * I * x0) / (Gz * Gy)
        if abs(Gy * y0 - Gz * h) < EPS:
            return pre * (ex(-1.0 * I * Gz * h) * (-1.0 * I + (ex(I * (Gy * y0 + Gz * h)) - 1.0) / (Gy * y0 + Gz * h)) - c)
        if abs(Gy * y0 + Gz * h) < EPS:
            return pre * (ex(-1.0 * I * Gz * h) * ((ex(-1.0 * I * (Gy * y0 - Gz * h)) - 1.0) / (Gy * y0 - Gz * h) + I) - c)
        return pre * (ex(-1.0 * I * Gz * h) * ((ex(-1.0 * I * (Gy * y0 - Gz * h)) - 1.0) / (Gy * y0 - Gz * h)
                                               + (ex(I * (Gy * y0 + Gz * h)) - 1.0) / (Gy * y0 + Gz * h)) - c)
    if abs(Gy) < EPS:
        pre = (2.0 * I * y0) / (Gz * x0)
        t2 = (ex(-1.0 * I * Gx * x0) * (1.0 + I * Gx * x0) - 1.0) / (Gx * Gx)
        if abs(Gx - (Gz * h) / x0) < EPS:
            return pre * (0.5 * ex(-1.0 * I * Gz * h) * x0 * x0 - t2)
        return pre * (ex(-1.0 * I * Gz * h) * (ex(-1.0 * I * (Gx * x0 - Gz * h)) * (1.0 + I * (Gx * x0 - Gz * h)) - 1.0)
                      / (Gx - (Gz * h) / x0) ** 2 - t2)
    if abs(Gz) < EPS:
        ap = Gx + (Gy * y0) / x0
        am = Gx - (Gy * y0) / x0
        if abs(Gx - (Gy * y0) / x0) < EPS:
            return (h / Gy) * (1.0 / ap - (I / (x0 * ap ** 2)) * (ex(-1.0 * I * x0 * ap) - 1.0) - 0.5 * I * x0)
        if abs(Gx + (Gy * y0) / x0) < EPS:
            return (h / Gy) * (-1.0 / am + (I / (x0 * am ** 2)) * (ex(-1.0 * I * x0 * am) - 1.0) + 0.5 * I * x0)
        return (h / Gy) * (1.0 / ap - 1.0 / am - (I / (x0 * ap ** 2)) * (ex(-1.0 * I * x0 * ap) - 1.0)
                           + (I / (x0 * am ** 2)) * (ex(-1.0 * I * x0 * am) - 1.0))
    e = ex(-1.0 * I * Gz * h)
    return (-1.0 / (Gy * Gz)) * (i_e0(x0, -1.0 * Gx - (Gy * y0) / x0 + (Gz * h) / x0) * e
                                 - i_e0(x0, -1.0 * Gx + (Gy * y0) / x0 + (Gz * h) / x0) * e
                                 - i_e0(x0, -1.0 * Gx - (Gy * y0) / x0)
                                 + i_e0(x0, -1.0 * Gx + (Gy * y0) / x0))


def prism_segment(Gx0, Gy0, Gz0, idx_side, N_side, g):
    """characteristic_function_fourier.c:1298-1411."""
    alpha = math.pi / float(N_side)
    x0, h = g["L1"], g["L2"]
    ang = (2.0 * math.pi * float(idx_side)) / N_side
    Gx = math.cos(ang) * Gx0 + math.sin(ang) * Gy0
    Gy = -1.0 * math.sin(ang) * Gx0 + math.cos(ang) * Gy0
    Gz = Gz0
    G_mag = math.sqrt(Gx ** 2 + Gy ** 2 + Gz ** 2)
    I = 1j
    ex = cmath.exp
    ta = math.tan(alpha)
    if abs(G_mag) < EPS:
        return x0 * x0 * h * ta
    if abs(Gx) < EPS and abs(Gy) < EPS:
        return 2.0 * x0 * x0 * ta * math.sin(0.5 * Gz * h) / Gz
    if abs(Gx) < EPS and abs(Gz) < EPS:
        return (2.0 * h / (Gy * Gy * ta)) * (1.0 - math.cos(Gy * x0 * ta))
    if abs(Gy) < EPS and abs(Gz) < EPS:
        return (2.0 * h * ta / Gx) * (1.0 * I * x0 * ex(-1.0 * I * Gx * x0) + (1.0 / Gx) * (ex(-1.0 * I * Gx * x0) - 1.0))
    if abs(Gx) < EPS:
        return (4.0 * math.sin(0.5 * Gz * h) / (Gy * Gy * Gz * ta)) * (1.0 - math.cos(Gy * x0 * ta))
    if abs(Gy) < EPS:
        return (4.0 * math.sin(0.5 * Gz * h) * ta / (Gz * Gx)) * (1.0 * I * x0 * ex(-1.0 * I * Gx * x0)
                                                                  + (1.0 / Gx) * (ex(-1.0 * I * Gx * x0) - 1.0))
    if abs(Gz) < EPS:
        pre = h / Gy
    else:
        pre = (2.0 / (Gy * Gz)) * math.sin(0.5 * Gz * h)
    if abs(Gy * ta + Gx) < EPS:
        return pre * (1.0 * I * x0 - (1.0 / (-Gy * ta + Gx)) * (1.0 - ex(1.0 * I * Gy * x0 * ta - 1.0 * I * Gx * x0)))
    if abs(-Gy * ta + Gx) < EPS:
        return pre * ((1.0 / (Gy * ta + Gx)) * (1.0 - ex(-1.0 * I * Gy * x0 * ta - 1.0 * I * Gx * x0)) - 1.0 * I * x0)
    return pre * ((1.0 / (Gy * ta + Gx)) * (1.0 - ex(-1.0 * I * Gy * x0 * ta - 1.0 * I * Gx * x0))
                  - (1.0 / (-Gy * ta + Gx)) * (1.0 - ex(1.0 * I * Gy * x0 * ta - 1.0 * I * Gx * x0)))


def chi(Gx0, Gy0, Gz0, geo, idx, cell, softening=0, sigma=0.0):
    """characteristic_function_fourier.c:58-1110 for one wave vector.

    ``cell`` is the supercell_type argument: 0 electronic-structure cell,
    1/2 strain cell, 3 Coulomb cell (selects the volume normalisation)."""
    g = geo[idx]
    g0 = geo[0]
    phase = cmath.exp(-1.0j * (Gx0 * g["Ox"] + Gy0 * g["Oy"] + Gz0 * g["Oz"]))
    if cell == 3:
        r = phase / (g0["CL1"] * g0["CL2"] * g0["CL3"])
    elif cell == 0 or idx == 0:
        r = phase / (g0["L1"] * g0["L2"] * g0["L3"])
    else:
        r = phase / (g0["SL1"] * g0["SL2"] * g0["SL3"])
    sa, ca = math.sin(math.pi * g["alpha"] / 180), math.cos(math.pi * g["alpha"] / 180)
    sb, cb = math.sin(math.pi * g["beta"] / 180), math.cos(math.pi * g["beta"] / 180)
    sg, cg = math.sin(math.pi * g["gamma"] / 180), math.cos(math.pi * g["gamma"] / 180)
    Gx = ((cb * ca * cg) - (sa * sg)) * Gx0 + ((cg * cb * sa) + (sg * ca)) * Gy0 + (-sb * cg) * Gz0
    Gy = ((cb * -ca * sg) - (sa * cg)) * Gx0 + ((-sg * cb * sa) + (cg * ca)) * Gy0 + (sb * sg) * Gz0
    Gz = (sb * ca) * Gx0 + (sa * sb) * Gy0 + (cb) * Gz0
    if softening != 0:
        r *= math.exp(-0.5 * sigma ** 2 * (Gx ** 2 + Gy ** 2 + Gz ** 2))
    shape = g["shape"]
    L1, L2, L3, L4 = g["L1"], g["L2"], g["L3"], g["L4"]
    G_mag = math.sqrt(Gx * Gx + Gy * Gy + Gz * Gz)
    G_par = math.sqrt(Gx * Gx + Gy * Gy)
    I = 1j
    J1 = lambda x: float(j1(x))  # noqa: E731
    if shape in (10, 13):
        # characteristic_function_fourier.c:580-620, 725-767: differences of two
        # shapes evaluated from the unrotated G (each with its own prefactor)
        g2 = dict(g)
        geo2 = list(geo)
        geo2[idx] = g2
        if shape == 10:
            g2["shape"] = 9
            g2["L2"] = L3
            r = chi(Gx0, Gy0, Gz0, geo2, idx, cell, softening, sigma)
            g2["L1"] = L2
            return r - chi(Gx0, Gy0, Gz0, geo2, idx, cell, softening, sigma)
        g2["shape"] = 12
        g2["L3"] = L4
        r = chi(Gx0, Gy0, Gz0, geo2, idx, cell, softening, sigma)
        g2["shape"] = 9
        g2["L1"] = L3
        g2["L2"] = L4
        return r - cmath.exp(-0.5 * I * Gz * L4) * chi(Gx0, Gy0, Gz0, geo2, idx, cell, softening, sigma)
    if shape == 0:
        r *= (L1 * sinc_pi((0.5 * Gx * L1) / math.pi) * L2 * sinc_pi((0.5 * Gy * L2) / math.pi)
              * L3 * sinc_pi((0.5 * Gz * L3) / math.pi))
    elif shape == 4:
        G_mag = math.sqrt((Gx * L1) ** 2 + (Gy * L2) ** 2 + (Gz * L3) ** 2)
        G_par = math.sqrt((Gx * L1) ** 2 + (Gy * L2) ** 2)
        if abs(G_mag) < EPS:
            r *= (2.0 * math.pi * L1 * L2 * L3) / 3.0
        else:
            sphere = (2.0 * math.pi * L1 * L2 * L3 * (math.sin(G_mag) - G_mag * math.cos(G_mag))) / G_mag ** 3
            if abs(G_par) < EPS:
                r *= sphere - (2.0 * math.pi * 1j * L1 * L2 / Gz) * (
                    0.5 - (math.cos(Gz * L3) + Gz * L3 * math.sin(L3 * Gz) - 1.0) / (Gz * L3) ** 2)
            elif abs(Gz) < EPS:
                r *= sphere
            else:
                r *= sphere - (2.0 * math.pi * 1j * L1 * L2 / Gz) * (float(j1(G_par)) / G_par - i_j0(Gz * L3, G_par))
    elif shape == 5:
        r *= sum(pyramid_segment(Gx, Gy, Gz, s, 0, geo[idx]) for s in range(4))
    elif shape == 6:
        g2 = dict(g)
        g2["L3"] = (L4 * L1) / (L1 - L3)
        seg = sum(pyramid_segment(Gx, Gy, Gz, s, 0, g2) for s in range(4))
        g2["L1"] = L3
        g2["L2"] = (L2 * L3) / L1
        g2["L3"] = (L4 * L3) / (L1 - L3)
        for s in range(4):
            seg -= cmath.exp(-1.0j * Gz * L4) * pyramid_segment(Gx, Gy, Gz, s, 0, g2)
        r *= seg
    elif shape == 1:  # sphere, radius L1
        if abs(G_mag) < EPS:
            r *= (4.0 * math.pi * L1 ** 3) / 3.0
        else:
            r *= (4.0 * math.pi * (math.sin(G_mag * L1) - G_mag * L1 * math.cos(G_mag * L1))) / G_mag ** 3
    elif shape == 2:  # ellipsoid, semi-axes L1, L2, L3
        Gs = math.sqrt((Gx * L1) ** 2 + (Gy * L2) ** 2 + (Gz * L3) ** 2)
        if abs(Gs) < EPS:
            r *= (4.0 * math.pi * L1 * L2 * L3) / 3.0
        else:
            r *= (4.0 * math.pi * L1 * L2 * L3 * (math.sin(Gs) - Gs * math.cos(Gs))) / Gs ** 3
    elif shape == 3:  # hemisphere, radius L1, base at the centre
        sph = 2.0 * math.pi * (math.sin(G_mag * L1) - G_mag * L1 * math.cos(G_mag * L1)) / (G_mag ** 3) \
            if abs(G_mag) >= EPS else 0.0
        if abs(G_mag) < EPS:
            r *= (2.0 * math.pi * L1 ** 3) / 3.0
        elif abs(G_par) < EPS and abs(Gz) > EPS:
            r *= sph - ((2.0 * math.pi * I * L1 ** 2) / Gz) * (
                0.5 - (L1 * Gz * math.sin(L1 * Gz) + math.cos(L1 * Gz) - 1.0) / (Gz * L1) ** 2)
        elif abs(Gz) < EPS and abs(G_par) > EPS:
            r *= sph
        else:
            r *= (sph - (2.0 * math.pi * I * L1 * J1(G_par * L1)) / (G_par * Gz)
                  + (2.0 * math.pi * I * L1 ** 2 * i_j0(Gz * L1, G_par * L1)) / Gz)
    elif shape == 7:  # N-sided pyramid: N = lround(L3 / 10), circumradius-type length L1, height L2
        n = _lround(0.1 * L3)
        r *= sum(pyramid_segment(Gx, Gy, Gz, k, n, g) for k in range(n))
    elif shape == 8:  # truncated N-sided pyramid: N = lround(L4 / 10)
        n = _lround(0.1 * L4)
        g2 = dict(g)
        g2["L2"] = (L1 * L3) / (L1 - L2)
        seg = sum(pyramid_segment(Gx, Gy, Gz, k, n, g2) for k in range(n))
        g2["L1"] = L2
        g2["L2"] = (L3 * L2) / (L1 - L2)
        for k in range(n):
            seg -= cmath.exp(-1.0 * I * Gz * L3) * pyramid_segment(Gx, Gy, Gz, k, n, g2)
        r *= seg
    elif shape == 9:  # cylinder, radius L1, height L2 (centred)
        if abs(G_mag) < EPS:
            r *= math.pi * L1 ** 2 * L2
        elif abs(G_par) < EPS and abs(Gz) > EPS:
            r *= 2.0 * math.pi * L1 ** 2 * math.sin(0.5 * Gz * L2) / Gz
        elif abs(Gz) < EPS and abs(G_par) > EPS:
            r *= (2.0 * math.pi * L1 * L2 * J1(G_par * L1)) / G_par
        else:
            r *= (4.0 * math.pi * L1 * math.sin(0.5 * Gz * L2) * J1(G_par * L1)) / (G_par * Gz)
    elif shape == 11:  # cone, base radius L1, height L2
        if abs(G_mag) < EPS:
            r *= (math.pi * L1 ** 2 * L2) / 3.0
        elif abs(G_par) < EPS:
            r *= (2.0 * I * math.pi * L1 ** 2 * ((1.0 - I * Gz * L2 - cmath.exp(-1.0 * I * Gz * L2)) / (Gz * L2) ** 2
                                                 - 0.5)) / Gz
        elif abs(Gz) < EPS:
            r *= (2.0 * math.pi * L1 ** 2 * L2) * (J1(G_par * L1) / (G_par * L1) - i_2_gz(G_par * L1))
        else:
            r *= ((2.0 * math.pi * L1 * L1 * I * cmath.exp(-1.0 * I * Gz * L2) * i_2(G_par * L1, Gz * L2)) / Gz
                  - (2.0 * math.pi * I * L1 * J1(G_par * L1)) / (G_par * Gz))
    elif shape == 12:  # truncated cone, base radius L1, top radius L2, height L3
        if abs(G_mag) < EPS:
            r *= (math.pi * L3 * (L1 * L1 + L1 * L2 + L2 * L2)) / 3.0
        elif abs(G_par) < EPS:
            e = cmath.exp(-1.0 * I * Gz * L3)
            r *= ((2.0 * I * math.pi) / Gz) * (
                (0.5 * L2 ** 2 * (e - 1.0))
                + ((L1 - L2) ** 2 / (Gz * L3) ** 2 * (e * ((I * Gz * L2 * L3) / (L1 - L2) - 1.0)
                                                       + (1.0 - (I * L1 * Gz * L3) / (L1 - L2))))
                - (0.5 * (L1 ** 2 - L2 ** 2)))
        elif abs(Gz) < EPS:
            r *= (2.0 * math.pi * L3) * ((L2 * J1(G_par * L2) / G_par)
                                         - ((L1 - L2) ** 2 * i_2_tc_gz(G_par, L2, L1))
                                         + ((L1 / (L1 - L2)) * (L1 * J1(G_par * L1) - L2 * J1(G_par * L2)) / G_par))
        else:
            r *= (2.0 * I * math.pi / Gz) * (
                (L2 * (cmath.exp(-1.0 * I * Gz * L3) - 1.0) * J1(G_par * L2) / G_par)
                + ((L1 - L2) ** 2 * cmath.exp((-1.0 * I * Gz * L3 * L1) / (L1 - L2)) * i_2_tc(G_par, L2, L1, Gz * L3))
                - ((L1 * J1(G_par * L1) - L2 * J1(G_par * L2)) / G_par))
    elif shape == 14:  # elliptical cone, semi-axes L1, L2, height L3
        Gp = math.sqrt((Gx * L1) ** 2 + (Gy * L2) ** 2)
        if abs(G_mag) < EPS:
            r *= (math.pi * L1 * L2 * L3) / 3.0
        elif abs(Gp) < EPS:
            r *= (1.0 / Gz) * (2.0 * I * math.pi * L1 * L2 * ((1.0 - I * Gz * L3 - cmath.exp(-1.0 * I * Gz * L3))
                                                              / (Gz * L3) ** 2 - 0.5))
        elif abs(Gz) < EPS:
            r *= (2.0 * math.pi * L1 * L2 * L3) * (J1(Gp) / Gp - i_2_gz(Gp))
        else:
            r *= ((2.0 * math.pi * L1 * L2 * I * cmath.exp(-1.0 * I * Gz * L3) * i_2(Gp, Gz * L3)) / Gz
                  - (2.0 * math.pi * I * L1 * L2 * J1(Gp)) / (Gp * Gz))
    elif shape == 15:  # truncated elliptical cone, semi-axes L1, L2, top ratio f = L3 / L1, height L4
        Gp = math.sqrt((Gx * L1) ** 2 + (Gy * L2) ** 2)
        f = L3 / L1
        if abs(G_mag) < EPS:
            r *= (math.pi * L1 * L2 * L4 * (1.0 + f + f ** 2)) / 3.0
        elif abs(Gp) < EPS:
            e = cmath.exp(-1.0 * I * Gz * L4)
            r *= (2.0 * math.pi * I * L1 * L2 * (
                (0.5 * f ** 2 * (e - 1.0))
                + ((f - 1.0) / (Gz * Gz * L4 * L4) * (e * (-1.0 * I * Gz * L4 * f - f + 1.0) + (I * Gz * L4 + f - 1.0)))
                - (0.5 * (1.0 - f ** 2))) / Gz)
        elif abs(Gz) < EPS:
            r *= (2.0 * math.pi * L1 * L2 * L4) * ((f * J1(f * Gp) / Gp) - (1.0 * i_2_etc_gz(Gp, f)) / (1.0 - f)
                                                   + ((J1(Gp) - f * J1(f * Gp)) / ((1.0 - f) * Gp)))
        else:
            r *= ((2.0 * I * math.pi * L1 * L2) / Gz) * (
                (f * (cmath.exp(-1.0 * I * Gz * L4) - 1.0) * J1(f * Gp) / Gp)
                + (cmath.exp(-1.0 * I * Gz * L4 / (1.0 - f)) * i_2_etc(Gp, Gz * L4, f))
                - ((J1(Gp) - f * J1(f * Gp)) / Gp))
    elif shape == 18:  # quantum wire along axis lround(L1 / 10), cross-section L2 x L3
        d = _lround(0.1 * L1)
        cellL = (g0["L1"], g0["L2"], g0["L3"]) if cell == 0 else (g0["SL1"], g0["SL2"], g0["SL3"])
        lens = {0: (cellL[0], L2, L3), 1: (L2, cellL[1], L3), 2: (L2, L3, cellL[2])}.get(d)
        if lens is not None:  # another axis index leaves the prefactor alone, as in the reference
            r *= (lens[0] * sinc_pi((0.5 * Gx * lens[0]) / math.pi) * lens[1] * sinc_pi((0.5 * Gy * lens[1]) / math.pi)
                  * lens[2] * sinc_pi((0.5 * Gz * lens[2]) / math.pi))
    elif shape == 16:
        n = _lround(0.1 * L3)
        r *= sum(prism_segment(Gx, Gy, Gz, s, n, g) for s in range(n))
    elif shape == 17:
        d = _lround(0.1 * L1)
        if cell == 0:
            dims = (g0["L1"], g0["L2"], g0["L3"])
        else:
            dims = (g0["SL1"], g0["SL2"], g0["SL3"])
        if d in (0, 1, 2):  # another axis index leaves the prefactor alone, as in the reference
            lens = list(dims)
            lens[d] = L2
            r *= (lens[0] * sinc_pi((0.5 * Gx * lens[0]) / math.pi) * lens[1]
                  * sinc_pi((0.5 * Gy * lens[1]) / math.pi) * lens[2] * sinc_pi((0.5 * Gz * lens[2]) / math.pi))
    else:
        raise ValueError("unknown shape %d" % shape)
    return r


def chi_table(basis, geo, idx, cell, softening=0, sigma=0.0):
    """chi_s on the (2N-1)^3 grid, index iz + N_zT (iy + N_yT ix)
    (characteristic_functions_reciprocal_space.c:53-80)."""
    Gx, Gy, Gz = basis["G"]
    out = np.empty((len(Gx), len(Gy), len(Gz)), dtype=np.complex128)
    for a, gx in enumerate(Gx):
        for b, gy in enumerate(Gy):
            for c, gz in enumerate(Gz):
                out[a, b, c] = chi(float(gx), float(gy), float(gz), geo, idx, cell, softening, sigma)
    return out

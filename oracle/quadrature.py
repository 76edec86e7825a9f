"""Adaptive Gauss-Kronrod quadrature as GSL's gsl_integration_qag evaluates
the lens integral (test infrastructure).

The reference calls ``gsl_integration_qag(f, 0, 1, EPS_ABS, EPS_REL, LIMIT,
key = 6, ...)`` (``code/source/8_band/characteristic_function_fourier_integrals.c:107-153``,
EPS_ABS = EPS_REL = 1e-4 and LIMIT = 1000 at ``8_band.h:61-63``).  GSL is not
part of the reference checkout (it is an external library, version not
pinned), so its algorithm is restated here from the published QUADPACK
method (R. Piessens, E. de Doncker-Kapenga, C. Ueberhuber, D. Kahaner,
QUADPACK, Springer 1983; GSL documents qag as that routine):

* key 6 is the 61-point Gauss-Kronrod rule (30 Gauss nodes plus 31 Kronrod
  nodes).  The nodes and weights are computed here, not tabulated: the
  Jacobi-Kronrod matrix of D. P. Laurie, "Calculation of Gauss-Kronrod
  quadrature rules", Math. Comp. 66 (1997) 1133-1145, from the Legendre
  recurrence, and its eigen-decomposition (Golub-Welsch);
* the error estimate of one rule application is QUADPACK's:
  err = |K - G| scaled by resasc min(1, (200 err / resasc)^1.5), floored at
  50 eps resabs;
* qag accepts the first application when err <= max(epsabs, epsrel |K|) and
  otherwise bisects the interval with the largest error until the summed error
  meets the tolerance (or LIMIT intervals are used).

For the entire integrands of the lens transform the first application is
accepted, so the reference's value is the 61-point Kronrod sum on [0, 1].
"""

import math

import numpy as np


def _legendre_recurrence(n):
    """Monic Legendre recurrence on [-1, 1]: a_k = 0, b_0 = 2 (total mass), b_k = k^2 / (4 k^2 - 1)."""
    a = np.zeros(n)
    b = np.zeros(n)
    b[0] = 2.0
    k = np.arange(1, n)
    b[1:] = k * k / (4.0 * k * k - 1.0)
    return a, b


def _jacobi_kronrod(n):
    """Laurie's algorithm: recurrence coefficients (a, b) of the (2n+1)-point
    Kronrod extension of the n-point Gauss rule."""
    m = 2 * n + 1
    a0, b0 = _legendre_recurrence(int(math.floor(3 * n / 2.0)) + 2)
    a = np.zeros(m)
    b = np.zeros(m)
    na = int(math.floor(3 * n / 2.0)) + 1
    nb = int(math.ceil(3 * n / 2.0)) + 1
    a[:na] = a0[:na]
    b[:nb] = b0[:nb]
    s = np.zeros(n // 2 + 2)
    t = np.zeros(n // 2 + 2)
    t[1] = b[n + 1]
    for mm in range(0, n - 1):
        acc = 0.0
        for k in range((mm + 1) // 2, -1, -1):
            l = mm - k
            acc += (a[k + n + 1] - a[l]) * t[k + 1] + b[k + n + 1] * s[k] - b[l] * s[k + 1]
            s[k + 1] = acc
        s, t = t, s
    for j in range(n // 2, -1, -1):
        s[j + 1] = s[j]
    for mm in range(n - 1, 2 * n - 2):
        acc = 0.0
        j = 0
        for k in range(mm + 1 - n, (mm - 1) // 2 + 1):
            l = mm - k
            j = n - 1 - l
            acc += -(a[k + n + 1] - a[l]) * t[j + 1] - b[k + n + 1] * s[j + 1] + b[l] * s[j + 2]
            s[j + 1] = acc
        k = (mm + 1) // 2
        if mm % 2 == 0:
            a[k + n + 1] = a[k] + (s[j + 1] - b[k + n + 1] * s[j + 2]) / t[j + 2]
        else:
            b[k + n + 1] = s[j + 1] / s[j + 2]
        s, t = t, s
    a[2 * n] = a[n - 1] - b[2 * n] * s[1] / t[1]
    return a, b


def gauss_kronrod(n):
    """Nodes and weights on [-1, 1] of the (2n+1)-point Kronrod rule and the
    weights of the embedded n-point Gauss rule (on the Gauss nodes, which are
    every second Kronrod node of the sorted list)."""
    a, b = _jacobi_kronrod(n)
    J = np.diag(a) + np.diag(np.sqrt(b[1:]), 1) + np.diag(np.sqrt(b[1:]), -1)
    x, V = np.linalg.eigh(J)
    w = b[0] * V[0, :] ** 2
    xg, wg = np.polynomial.legendre.leggauss(n)
    return x, w, xg, wg


_XK, _WK, _XG, _WG = gauss_kronrod(30)
_EPMACH = np.finfo(np.float64).eps
_UFLOW = np.finfo(np.float64).tiny


def qk61(f, lo, hi):
    """One application on [lo, hi]: (Kronrod result, QUADPACK error estimate,
    resabs, resasc)."""
    c = 0.5 * (lo + hi)
    h = 0.5 * (hi - lo)
    fk = f(c + h * _XK)
    fg = f(c + h * _XG)
    resk = float(np.sum(_WK * fk))
    resg = float(np.sum(_WG * fg))
    reskh = 0.5 * resk
    resabs = float(np.sum(_WK * np.abs(fk))) * abs(h)
    resasc = float(np.sum(_WK * np.abs(fk - reskh))) * abs(h)
    result = resk * h
    err = abs((resk - resg) * h)
    if resasc != 0.0 and err != 0.0:
        err = resasc * min(1.0, (200.0 * err / resasc) ** 1.5)
    if resabs > _UFLOW / (50.0 * _EPMACH):
        err = max(_EPMACH * 50.0 * resabs, err)
    return result, err, resabs, resasc


def qag61(f, lo, hi, epsabs=1.0e-4, epsrel=1.0e-4, limit=1000):
    """gsl_integration_qag with key 6 (61 points).  Returns (result, error)."""
    result, err, resabs, resasc = qk61(f, lo, hi)
    tol = max(epsabs, epsrel * abs(result))
    if (err <= tol and err != resasc) or err == 0.0:
        return result, err
    intervals = [(lo, hi, result, err)]
    total, total_err = result, err
    while total_err > max(epsabs, epsrel * abs(total)) and len(intervals) < limit:
        i = max(range(len(intervals)), key=lambda q: intervals[q][3])
        a, b, r, e = intervals.pop(i)
        m = 0.5 * (a + b)
        r1, e1, _, _ = qk61(f, a, m)
        r2, e2, _, _ = qk61(f, m, b)
        intervals += [(a, m, r1, e1), (m, b, r2, e2)]
        total += r1 + r2 - r
        total_err += e1 + e2 - e
    return sum(iv[2] for iv in intervals), total_err

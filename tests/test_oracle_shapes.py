"""The oracle's shape transforms against direct integration (CPU).

Every shape of characteristic_function_fourier.c is restated in
oracle/shapes.py.  No golden file of the reference holds the curved shapes, so
each transform is checked here against a brute-force midpoint sum of
exp(-i G.r) over the shape's indicator function on a 100^3 grid (the geometry
each formula describes: sphere and ellipsoid about the centre, hemisphere,
cones and pyramids standing on z = 0, cylinder and ring centred in z, regular
N-gon bases given by their inradius).  The grid sum carries a surface
discretisation error of up to about 1.5e-2 of the volume (the ring, with
the largest surface); a wrong term of a formula shows as an error of order 1.
"""

import math

import numpy as np
import pytest

from oracle import inputs, shapes

N = 100
EXT = 40.0
CELL = (100.0, 100.0, 80.0)
G_LIST = [(0.05, 0.03, 0.02), (0.05, 0.0, 0.0), (0.0, 0.0, 0.07), (0.1, -0.05, 0.12)]


def _grid():
    xs = (np.arange(N) + 0.5) / N * 2 * EXT - EXT
    return np.meshgrid(xs, xs, xs, indexing="ij"), (2 * EXT / N) ** 3


def _polygon(n, a_base, a_top, h, X, Y, Z):
    ok = (Z >= 0) & (Z <= h)
    s = a_base + (a_top - a_base) * Z / h
    for k in range(n):
        ang = 2 * math.pi * k / n
        ok &= X * math.cos(ang) + Y * math.sin(ang) <= s
    return ok


def _indicator(sh, L, X, Y, Z):
    r2 = X * X + Y * Y
    if sh == 1:
        return r2 + Z * Z <= L[0] ** 2
    if sh == 2:
        return (X / L[0]) ** 2 + (Y / L[1]) ** 2 + (Z / L[2]) ** 2 <= 1
    if sh == 3:
        return (r2 + Z * Z <= L[0] ** 2) & (Z >= 0)
    if sh == 7:
        return _polygon(int(round(0.1 * L[2])), L[0], 0.0, L[1], X, Y, Z)
    if sh == 8:
        return _polygon(int(round(0.1 * L[3])), L[0], L[1], L[2], X, Y, Z)
    if sh == 9:
        return (r2 <= L[0] ** 2) & (abs(Z) <= L[1] / 2)
    if sh == 10:
        return (r2 <= L[0] ** 2) & (r2 >= L[1] ** 2) & (abs(Z) <= L[2] / 2)
    if sh == 11:
        return (Z >= 0) & (Z <= L[1]) & (r2 <= (L[0] * (1 - Z / L[1])) ** 2)
    if sh == 12:
        return (Z >= 0) & (Z <= L[2]) & (r2 <= (L[0] + (L[1] - L[0]) * Z / L[2]) ** 2)
    if sh == 13:
        return (Z >= 0) & (Z <= L[3]) & (r2 <= (L[0] + (L[1] - L[0]) * Z / L[3]) ** 2) & (r2 >= L[2] ** 2)
    if sh == 14:
        return (Z >= 0) & (Z <= L[2]) & ((X / L[0]) ** 2 + (Y / L[1]) ** 2 <= (1 - Z / L[2]) ** 2)
    if sh == 15:
        f = L[2] / L[0]
        return (Z >= 0) & (Z <= L[3]) & ((X / L[0]) ** 2 + (Y / L[1]) ** 2 <= (1 - (1 - f) * Z / L[3]) ** 2)
    raise ValueError(sh)


@pytest.mark.parametrize("sh,L", [(1, (20, 0, 0, 0)), (2, (20, 15, 10, 0)), (3, (20, 0, 0, 0)), (7, (20, 30, 60, 0)),
                                  (8, (20, 10, 15, 60)), (9, (20, 30.4, 0, 0)), (10, (20, 10, 30.4, 0)),
                                  (11, (20, 30, 0, 0)), (12, (20, 10, 15, 0)), (13, (20, 10, 5, 15)),
                                  (14, (20, 15, 30, 0)), (15, (20, 15, 10, 30))])
def test_shape_transform_matches_direct_integration(sh, L):
    g0 = inputs.empty_geometry()
    g0.update(L1=CELL[0], L2=CELL[1], L3=CELL[2])
    g = inputs.empty_geometry()
    g.update(shape=sh, L1=float(L[0]), L2=float(L[1]), L3=float(L[2]), L4=float(L[3]))
    (X, Y, Z), dv = _grid()
    M = _indicator(sh, L, X, Y, Z)
    vol = CELL[0] * CELL[1] * CELL[2]
    chi0 = shapes.chi(0.0, 0.0, 0.0, [g0, g], 1, 0)
    assert abs(chi0 * vol - M.sum() * dv) <= 2e-2 * chi0.real * vol
    for G in G_LIST:
        direct = np.exp(-1j * (G[0] * X[M] + G[1] * Y[M] + G[2] * Z[M])).sum() * dv / vol
        assert abs(shapes.chi(G[0], G[1], G[2], [g0, g], 1, 0) - direct) <= 2e-2 * abs(chi0), G


def test_quantum_wire_is_a_box():
    g0 = inputs.empty_geometry()
    g0.update(L1=CELL[0], L2=CELL[1], L3=CELL[2])
    g = inputs.empty_geometry()
    g.update(shape=18, L1=10.0, L2=15.0, L3=10.0)  # along y (lround(L1 / 10) = 1), 15 x 10 cross-section
    box = inputs.empty_geometry()
    box.update(shape=0, L1=15.0, L2=CELL[1], L3=10.0)
    for G in G_LIST:
        assert abs(shapes.chi(*G, [g0, g], 1, 0) - shapes.chi(*G, [g0, box], 1, 0)) < 1e-15

"""Commensurate strain and Coulomb cells in the oracle (CPU).

The oracle restates the reference's FFT forms literally:
* strain_reciprocal_space_fft.c:23-362 (and piezo_reciprocal_space_fft.c):
  zero-padded FFT convolution of the strain-cell table with the electronic
  cell's cuboid, sampled at every RL-th wave vector;
* B_coulomb_supercell_fft.c:23-100: B placed on every RCL-th point of the
  Coulomb grid and convolved with the cuboid by FFTs, central block kept.
The GPU evaluates the same linear convolutions as separable sums over the
per-axis cuboid factors (sinc times the softening Gaussian) with the cut-off
that the padded FFT grid implies.  These tests check that the two forms agree,
and that for Coulomb cells the commensurate form equals the free-length form
of B_coulomb_supercell.c with CL = RCL L (its cut-off |GC - G| <= max GC is the
one the FFT grid implies), so the GPU's formulation is pinned to the
reference's steps.
"""

import math

import numpy as np
import pytest

from oracle import coulomb, inputs, shapes, strain


def _cell(L, RL=(1, 1, 1), RCL=(1, 1, 1)):
    g0 = inputs.empty_geometry()
    g0.update(L1=L[0], L2=L[1], L3=L[2], RL1=RL[0], RL2=RL[1], RL3=RL[2], RCL1=RCL[0], RCL2=RCL[1], RCL3=RCL[2])
    for a in range(3):
        g0["SL%d" % (a + 1)] = L[a] * RL[a]
        g0["CL%d" % (a + 1)] = L[a] * RCL[a]
    return [g0]


def _axis_weight(Gv, L, soft, sigma):
    v = L * shapes.sinc_pi((0.5 * Gv * L) / math.pi)
    return v * math.exp(-0.5 * sigma * sigma * Gv * Gv) if soft else v


def _separable_strain(T, basis, sbasis, geo, soft, sigma):
    """The GPU's formulation: T_es(e) = 1/(L1 L2 L3) sum_s prod_a w_a(e_a, s_a) T(s),
    w_a(e, s) = L sinc(GS[q] L / 2) g(GS[q]), q = RL (e - h) - (s - hs) + hs on the strain grid."""
    g0 = geo[0]
    L = (g0["L1"], g0["L2"], g0["L3"])
    RL = (g0["RL1"], g0["RL2"], g0["RL3"])
    W = []
    for a in range(3):
        ne, ns = basis["N_T"][a], sbasis["N_T"][a]
        w = np.zeros((ne, ns))
        for e in range(ne):
            for s in range(ns):
                qq = RL[a] * (e - ne // 2) - (s - ns // 2) + ns // 2
                if 0 <= qq < ns:
                    w[e, s] = _axis_weight(float(sbasis["G"][a][qq]), L[a], soft, sigma)
        W.append(w)
    return np.einsum("xa,yb,zc,abc->xyz", W[0], W[1], W[2], T) / (L[0] * L[1] * L[2])


@pytest.mark.parametrize("RL,N,NS,soft", [((2, 2, 2), (3, 3, 3), (5, 5, 5), 0), ((3, 1, 2), (5, 3, 3), (9, 3, 5), 1),
                                          ((2, 3, 4), (3, 5, 5), (4, 7, 9), 0)])
def test_strain_fft_downsampling_is_the_truncated_separable_sum(RL, N, NS, soft):
    L = (24.0, 20.0, 16.0)
    geo = _cell(L, RL=RL)
    sigma = 0.7
    basis = shapes.make_basis(N, L)
    sbasis = shapes.make_basis(NS, tuple(L[a] * RL[a] for a in range(3)))
    rng = np.random.default_rng(sum(RL) * 10 + sum(NS))
    T = rng.standard_normal(sbasis["N_T"]) + 1j * rng.standard_normal(sbasis["N_T"])
    fft_form = strain.downsample_commensurate(T, basis, sbasis, geo, soft, sigma)
    direct = _separable_strain(T, basis, sbasis, geo, soft, sigma)
    assert fft_form.shape == tuple(basis["N_T"])
    assert np.abs(fft_form - direct).max() <= 1e-13 * np.abs(direct).max()


def test_strain_fft_downsampling_reduces_to_a_copy_for_equal_cells():
    L = (24.0, 20.0, 16.0)
    geo = _cell(L)
    basis = shapes.make_basis((3, 4, 3), L)
    rng = np.random.default_rng(3)
    T = rng.standard_normal(basis["N_T"]) + 1j * rng.standard_normal(basis["N_T"])
    out = strain.downsample_commensurate(T, basis, basis, geo)
    assert np.abs(out - T).max() <= 1e-13 * np.abs(T).max()


def test_strain_grid_check():
    geo = _cell((24.0, 20.0, 16.0), RL=(3, 3, 4))
    # M = 4, 4, 5 with RL 3, 3, 4 needs M_S >= 6, 6, 10 (the reference's example uses 12, 12, 20)
    p = {"N_Gx": 9, "N_Gy": 9, "N_Gz": 11, "N_S_Gx": 25, "N_S_Gy": 25, "N_S_Gz": 41}
    assert strain.strain_grid_too_small(p, geo) == []
    p.update(N_S_Gz=19)
    assert strain.strain_grid_too_small(p, geo) == ["z"]


def _random_b(basis, P, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(basis["N_T"]))
    return rng.standard_normal((P, n)) + 1j * rng.standard_normal((P, n))


@pytest.mark.parametrize("RCL,N,NC", [((1, 2, 2), (3, 4, 3), (4, 7, 5)), ((1, 1, 2), (3, 3, 3), (3, 3, 6)),
                                      ((2, 1, 1), (2, 3, 3), (5, 3, 3))])
def test_coulomb_fft_upsampling_equals_free_lengths(RCL, N, NC):
    L = (60.0, 50.0, 35.0)
    geo = _cell(L, RCL=RCL)
    CL = tuple(L[a] * RCL[a] for a in range(3))
    basis = shapes.make_basis(N, L)
    cb = shapes.make_basis(NC, CL)
    B = _random_b(basis, 4, sum(NC))
    a = coulomb.coulomb_supercell_commensurate(B, basis, cb, geo)
    b = coulomb.coulomb_supercell(B, basis, cb, L, CL)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_coulomb_fft_upsampling_with_softening():
    L = (60.0, 50.0, 35.0)
    RCL = (1, 2, 2)
    geo = _cell(L, RCL=RCL)
    CL = tuple(L[a] * RCL[a] for a in range(3))
    basis = shapes.make_basis((3, 3, 3), L)
    cb = shapes.make_basis((4, 6, 5), CL)
    B = _random_b(basis, 3, 11)
    sigma = 4.0
    got = coulomb.coulomb_supercell_commensurate(B, basis, cb, geo, 1, sigma)
    # free-length weights times the Gaussian of the same wave-vector difference
    W = []
    for a in range(3):
        Gc, Ge = cb["G"][a], basis["G"][a]
        w = np.zeros((len(Gc), len(Ge)))
        for c in range(len(Gc)):
            for g in range(len(Ge)):
                d = Gc[c] - Ge[g]
                if abs(d) < 1e-8:
                    v = L[a]
                elif abs(d) > Gc[-1] + 1e-8:
                    v = 0.0
                else:
                    v = 2.0 * math.sin(d * L[a] / 2.0) / d
                w[c, g] = v * math.exp(-0.5 * sigma * sigma * d * d)
        W.append(w)
    want = np.einsum("xa,yb,zc,pabc->pxyz", W[0], W[1], W[2], B.reshape((3,) + basis["N_T"]))
    want = want.reshape(3, -1) / (L[0] * L[1] * L[2])
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()

"""Input decks (parameters.in / supercell.in) for the workloads this package is
measured on, written in the reference's own file format.

Lengths in the files are in nm, fields in kV/cm (the readers convert to
Angstrom and V/Angstrom).  Material system 3 is Ga(x)In(1-x)P(y)As(1-y): GaAs
is x = 1, y = 0; In(c)Ga(1-c)As is x = 1 - c, y = 0.

  lens_7      InAs lens (r 10 nm, h 3.5 nm) on a 0.5 nm InAs wetting layer in a
              30 x 30 x 20 nm GaAs cell; 7^3 plane waves (N_H = 2744); strain,
              first-order piezo, no field; 4 e + 4 h Kramers pairs.
  pyramid_11  In0.6Ga0.4As truncated pyramid (base 18 nm, top 8 nm, height 5 nm)
              on a 0.6 nm wetting layer in 36 x 36 x 24 nm; 11^3 (N_H = 10648);
              strain, piezo, Fz = 10 kV/cm; 8 e + 8 h pairs; Coulomb cell = ES cell.
  molecule_15 two stacked In0.5Ga0.5As lenses (r 9 / 10 nm, h 3 / 3.5 nm, 4 nm
              GaAs gap between the lower apex and the upper base) in 40 x 40 x 32 nm;
              15^3 (N_H = 27000); strain, first-order piezo; 8 e + 8 h pairs
              (32 eigenpairs).
The wetting-layer placement (centred 0.25 / 0.3 nm below the dot base), the
temperature (300 K) and the lens stacking are choices of this deck.
"""

import os

PARAM_DEFAULTS = dict(
    N_shape=2, M_Gx=3, M_Gy=3, M_Gz=3, Strain_supercell_type=1, M_S_Gx=3, M_S_Gy=3, M_S_Gz=3, N_VB=4, N_CB=4,
    T=300.0, Fx=0, Fy=0, Fz=0, Kx=0, Ky=0, Kz=0, N_line=300, Strain=1, Isotropic=0, Elastic_const=0,
    Elastic_const_order=0, Piezo=1, Eigensolver=1, Overlaps=0, Localisation=0, MME=0, CME=0,
    Coulomb_supercell_type=0, M_C_Gx=3, M_C_Gy=3, M_C_Gz=3, Linescan_100=0, Linescan_010=0, Linescan_001=0,
    Linescan_110=0, Linescan_101=0, Linescan_011=0, Linescan_111=0, Cross_sections=0, N_cross=20,
    Cross_section_100=0, Cross_section_010=0, Cross_section_001=0, Cross_section_m110=0, Cross_section_110=0,
    Cross_section_m101=0, Cross_section_0m11=0, Cross_section_111=0, **{"3D_output": 0}, N_3D=20)


def parameters_text(**kw):
    p = dict(PARAM_DEFAULTS)
    p.update(kw)
    return "".join("%s: %s\n" % (k, v) for k, v in p.items())


def supercell_record(L, material=3, x=1.0, y=0.0, strain_rel=(1, 1, 1), coulomb=None):
    c = coulomb if coulomb is not None else L
    return ("QD shape: 0\nMaterial: %d\nCompos x: %r\nCompos y: %r\n" % (material, x, y) +
            "Length 1: %r\nLength 2: %r\nLength 3: %r\n" % tuple(L) +
            "Strain length 1: %d\nStrain length 2: %d\nStrain length 3: %d\n" % tuple(strain_rel) +
            "Coulomb length 1: %r\nCoulomb length 2: %r\nCoulomb length 3: %r\n\n" % tuple(c))


def shape_record(shape, material, x, y, centre, lengths, euler=(0.0, 0.0, 0.0), embedded=0):
    L = list(lengths) + [0.0] * (5 - len(lengths))
    return ("Embedded: %d\nQD shape: %d\nMaterial: %d\nCompos x: %r\nCompos y: %r\n" % (embedded, shape, material, x, y) +
            "Centre x: %r\nCentre y: %r\nCentre z: %r\n" % tuple(centre) +
            "".join("Length %d: %r\n" % (i + 1, L[i]) for i in range(5)) +
            "Euler alpha angle: %r\nEuler beta angle: %r\nEuler gamma angle: %r\n\n" % tuple(euler))


def lens_7(mg=3):
    params = parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=4, N_CB=4,
                             Piezo=1)
    cell = (supercell_record((30.0, 30.0, 20.0)) +
            shape_record(4, 3, 0.0, 0.0, (0.0, 0.0, -1.75), (10.0, 10.0, 3.5)) +
            shape_record(17, 3, 0.0, 0.0, (0.0, 0.0, -2.0), (2.0, 0.5)))
    return params, cell


def pyramid_11(mg=5, n_states=8, cme=1, height=5.0, half_base=9.0, x=0.4, fz=10.0):
    """The truncated-pyramid deck; height, half_base (nm), the dot's composition
    x (1 - In fraction) and Fz (kV/cm) are the parameters the gradients are
    taken with respect to."""
    params = parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=n_states,
                             N_CB=n_states, Piezo=1, Fz=fz, CME=cme, M_C_Gx=mg, M_C_Gy=mg, M_C_Gz=mg)
    cell = (supercell_record((36.0, 36.0, 24.0)) +
            shape_record(6, 3, x, 0.0, (0.0, 0.0, -2.5), (half_base, half_base, 4.0, height)) +
            shape_record(17, 3, 0.4, 0.0, (0.0, 0.0, -2.8), (2.0, 0.6)))
    return params, cell


def molecule_15(mg=7, n_states=8, cme=0):
    """The benchmark deck; cme > 0 also asks for Coulomb matrix elements on a
    Coulomb cell equal to the electronic cell (mg plane waves per axis)."""
    params = parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=n_states,
                             N_CB=n_states, Piezo=1, CME=cme, M_C_Gx=mg, M_C_Gy=mg, M_C_Gz=mg)
    cell = (supercell_record((40.0, 40.0, 32.0)) +
            shape_record(4, 3, 0.5, 0.0, (0.0, 0.0, -5.25), (9.0, 9.0, 3.0)) +
            shape_record(4, 3, 0.5, 0.0, (0.0, 0.0, 1.75), (10.0, 10.0, 3.5)))
    return params, cell


def batch_lenses(n=64, seed=0):
    """The batched sweep: n lens dots (In(c)Ga(1-c)As on a 0.5 nm wetting layer of
    the same alloy, in a 40 x 40 x 24 nm GaAs cell) with radius U[8, 14] nm,
    height U[2, 5] nm, In fraction c U[0.4, 1.0], Fz U[-50, 50] kV/cm and a
    plane-wave cutoff drawn from {7^3, 9^3, 11^3}, in that draw order per
    instance from numpy.random.default_rng(seed); 4 e + 4 h Kramers pairs each.
    Returns a list of (params, cell, description)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        r = rng.uniform(8.0, 14.0)
        h = rng.uniform(2.0, 5.0)
        c = rng.uniform(0.4, 1.0)
        fz = rng.uniform(-50.0, 50.0)
        mg = int(rng.integers(3, 6))
        x = 1.0 - c
        params = parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=4,
                                 N_CB=4, Piezo=1, Fz=fz)
        cell = (supercell_record((40.0, 40.0, 24.0)) +
                shape_record(4, 3, x, 0.0, (0.0, 0.0, -0.5 * h), (r, r, h)) +
                shape_record(17, 3, x, 0.0, (0.0, 0.0, -0.5 * h - 0.25), (2.0, 0.5)))
        out.append((params, cell, dict(radius=r, height=h, indium=c, fz=fz, mg=mg)))
    return out


DECKS = {"lens_7": lens_7, "pyramid_11": pyramid_11, "molecule_15": molecule_15}


def write_deck(directory, params, cell):
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "parameters.in"), "w") as f:
        f.write(params)
    with open(os.path.join(directory, "supercell.in"), "w") as f:
        f.write(cell)
    return directory

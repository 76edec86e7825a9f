"""Small input decks shared by the parity tests (reference file format)."""

import os

from qudos_b200 import configs as C

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def prism(mg, tmp):
    """The reference's Prism_111 example (rotated hexagonal GaAs prism in AlAs,
    strain, first + second order piezo) at a reduced plane-wave count."""
    src = os.path.join(GOLDEN, "prism_111")
    text = open(os.path.join(src, "parameters.in")).read()
    lines = []
    for ln in text.splitlines():
        k = ln.split(":")[0].strip()
        if k in ("M_Gx", "M_Gy", "M_Gz", "M_S_Gx", "M_S_Gy", "M_S_Gz", "M_C_Gx", "M_C_Gy", "M_C_Gz"):
            ln = "%s: %d" % (k, mg)
        lines.append(ln)
    d = os.path.join(str(tmp), "prism_%d" % mg)
    C.write_deck(d, "\n".join(lines) + "\n", open(os.path.join(src, "supercell.in")).read())
    return d


def lens(mg, tmp):
    return C.write_deck(os.path.join(str(tmp), "lens_%d" % mg), *C.lens_7(mg))


def pyramid(mg, tmp):
    return C.write_deck(os.path.join(str(tmp), "pyr_%d" % mg), *C.pyramid_11(mg, n_states=4))


def molecule(mg, tmp):
    return C.write_deck(os.path.join(str(tmp), "mol_%d" % mg), *C.molecule_15(mg, n_states=4))


def nostrain_k(mg, tmp):
    """No strain; cuboid + pyramid (shape 5) + field along x and a supercell wave vector K."""
    params = C.parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Strain=0, Piezo=0, Fx=25, Fy=-5, Kx=0.02, Ky=0.01, Kz=-0.015)
    cell = (C.supercell_record((20.0, 22.0, 18.0)) +
            C.shape_record(0, 3, 0.3, 0.0, (1.0, -0.5, 0.5), (8.0, 7.0, 4.0)) +
            C.shape_record(5, 3, 0.0, 0.0, (0.0, 0.0, -2.0), (5.0, 4.0, 3.0)))
    return C.write_deck(os.path.join(str(tmp), "nsk_%d" % mg), params, cell)


def isotropic(mg, tmp):
    """Isotropic elastic tensor, second-order piezo only, embedded shape."""
    params = C.parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Isotropic=1, Piezo=3, Fz=-30)
    cell = (C.supercell_record((24.0, 24.0, 20.0)) +
            C.shape_record(0, 3, 0.8, 0.0, (0.0, 0.0, 0.0), (12.0, 12.0, 6.0)) +
            C.shape_record(6, 3, 0.2, 0.0, (0.0, 0.0, -1.5), (5.0, 4.0, 2.0, 3.0), embedded=1))
    return C.write_deck(os.path.join(str(tmp), "iso_%d" % mg), params, cell)


def commensurate(mg, tmp):
    """Commensurate strain cell (Strain_supercell_type 1, RL = 2, 2, 3 with
    M_S = M RL) and Coulomb cell (Coulomb_supercell_type 1, RCL = 1, 2, 2);
    truncated pyramid on a wetting layer, first + second order piezo and
    interface softening (sigma 0.3 nm)."""
    rl = (2, 2, 3)
    params = C.parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg * rl[0], M_S_Gy=mg * rl[1],
                               M_S_Gz=mg * rl[2], N_VB=2, N_CB=1, Piezo=2, CME=4, Coulomb_supercell_type=1,
                               M_C_Gx=mg, M_C_Gy=2 * mg, M_C_Gz=2 * mg, Softening=1, Sigma_softening=0.3)
    cell = (C.supercell_record((20.0, 20.0, 14.0), strain_rel=rl, coulomb=(1, 2, 2)) +
            C.shape_record(6, 3, 0.5, 0.0, (0.0, 0.0, -1.5), (6.0, 6.0, 3.0, 3.0)) +
            C.shape_record(17, 3, 0.5, 0.0, (0.0, 0.0, -1.8), (2.0, 0.5)))
    return C.write_deck(os.path.join(str(tmp), "comm_%d" % mg), params, cell)


def all_shapes(mg, tmp):
    """The thirteen shapes the other decks do not use (sphere, ellipsoid,
    hemisphere, N-sided and truncated N-sided pyramids, cylinder, ring, cone,
    truncated cone, truncated conic ring, elliptical and truncated elliptical
    cones, quantum wire), one with Euler angles, no strain."""
    params = C.parameters_text(N_shape=14, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Strain=0, Piezo=0, Fz=10)
    cell = C.supercell_record((30.0, 30.0, 24.0))
    recs = [(1, (2.0,), (-6.0, -6.0, 4.0)), (2, (2.5, 2.0, 1.5), (6.0, -6.0, 4.0)), (3, (3.0,), (0.0, 0.0, 6.0)),
            (7, (2.0, 3.0, 6.0), (-6.0, 6.0, -3.0)), (8, (2.5, 1.2, 2.0, 5.0), (6.0, 6.0, -3.0)),
            (9, (2.0, 3.0), (-9.0, 0.0, 0.0)), (10, (3.0, 1.5, 2.0), (9.0, 0.0, 0.0)),
            (11, (3.0, 2.5), (0.0, -9.0, -6.0)), (12, (3.0, 1.5, 2.0), (0.0, 9.0, -6.0)),
            (13, (3.0, 2.0, 1.0, 2.5), (-4.0, 0.0, -8.0)), (14, (3.0, 2.0, 2.5), (4.0, 0.0, -8.0)),
            (15, (3.0, 2.0, 1.5, 2.0), (0.0, 0.0, -2.0)), (18, (1.0, 1.5, 1.0), (0.0, 0.0, 9.0))]
    for i, (sh, L, O) in enumerate(recs):
        euler = (20.0, 15.0, 0.0) if sh == 12 else (0.0, 0.0, 0.0)
        cell += C.shape_record(sh, 3, 0.3 + 0.04 * i, 0.0, O, L, euler=euler)
    return C.write_deck(os.path.join(str(tmp), "shapes_%d" % mg), params, cell)


def curved_strain(mg, tmp):
    """Cone, cylinder and sphere dots on a quantum wire, with strain and
    first-order piezo (the strain-cell transforms of the curved shapes and of
    the wire use the strain-cell lengths)."""
    params = C.parameters_text(N_shape=5, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Piezo=1)
    cell = (C.supercell_record((24.0, 24.0, 20.0)) +
            C.shape_record(18, 3, 0.6, 0.0, (0.0, 0.0, -3.0), (0.0, 2.0, 1.0)) +
            C.shape_record(11, 3, 0.4, 0.0, (-5.0, 0.0, -2.5), (3.0, 3.0)) +
            C.shape_record(9, 3, 0.5, 0.0, (5.0, 0.0, -1.0), (2.5, 3.0)) +
            C.shape_record(1, 3, 0.45, 0.0, (0.0, 0.0, 4.0), (2.0,)))
    return C.write_deck(os.path.join(str(tmp), "curved_%d" % mg), params, cell)


def elastic(mg, tmp):
    """Position-dependent elastic constants (Elastic_const 1, two correction
    orders): an InAs lens and a GaP cuboid in GaAs, first + second order piezo."""
    params = C.parameters_text(N_shape=3, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Piezo=2, Elastic_const=1, Elastic_const_order=2)
    cell = (C.supercell_record((22.0, 22.0, 18.0)) +
            C.shape_record(4, 3, 0.0, 0.0, (0.0, 0.0, -1.0), (6.0, 6.0, 3.0)) +
            C.shape_record(0, 3, 1.0, 1.0, (0.0, 0.0, 5.0), (8.0, 8.0, 1.0)))
    return C.write_deck(os.path.join(str(tmp), "elastic_%d" % mg), params, cell)


def elastic_isotropic(mg, tmp):
    """Position-dependent elastic constants with the isotropic elastic tensor,
    one correction order, field along z."""
    params = C.parameters_text(N_shape=2, M_Gx=mg, M_Gy=mg, M_Gz=mg, M_S_Gx=mg, M_S_Gy=mg, M_S_Gz=mg, N_VB=2,
                               N_CB=2, Piezo=1, Isotropic=1, Elastic_const=1, Elastic_const_order=1, Fz=20)
    cell = (C.supercell_record((20.0, 20.0, 16.0)) +
            C.shape_record(6, 3, 0.3, 0.0, (0.0, 0.0, -1.5), (6.0, 6.0, 3.0, 3.0)))
    return C.write_deck(os.path.join(str(tmp), "elastic_iso_%d" % mg), params, cell)


CASES = {"prism": prism, "lens": lens, "pyramid": pyramid, "molecule": molecule, "nostrain_k": nostrain_k,
         "isotropic": isotropic, "commensurate": commensurate, "all_shapes": all_shapes,
         "curved_strain": curved_strain, "elastic": elastic, "elastic_isotropic": elastic_isotropic}

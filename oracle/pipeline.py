"""Oracle end-to-end pipeline in the reference's call order (test infrastructure).

Follows ``code/source/8_band/8_band_main.c:142-763`` for the stages that feed the
solve: inputs, basis sets, material parameters, shape transforms for the strain
and electronic-structure cells, strain, piezo potential, downsampling,
convolutions, then ``eigenstates``.
"""

import numpy as np

from . import eigen, hamiltonian, inputs, materials, shapes, strain


class Problem:
    pass


def prepare(p, geo):
    """Everything up to the Hamiltonian inputs (8_band_main.c:142-723)."""
    geo = inputs.clone(geo)
    pr = Problem()
    pr.p = p
    pr.strain_type = inputs.effective_strain_region_type(p, geo)
    g0 = geo[0]
    K = (p["Kx"], p["Ky"], p["Kz"])
    pr.basis = shapes.make_basis((p["N_Gx"], p["N_Gy"], p["N_Gz"]), (g0["L1"], g0["L2"], g0["L3"]), K)
    pr.params = materials.material_parameters(p["T"], geo, p["Piezo"])
    pr.geo = geo
    ns = p["N_shape"]
    soft, sig = p["Softening"], p["Sigma_softening"]
    include_strain = p["Strain"]
    pr.tables = hamiltonian.Tables([None] * ns)
    if include_strain == 1:
        if pr.strain_type == 1 and strain.strain_grid_too_small(p, geo):
            raise ValueError("M_S is too small for the commensurate strain cell")
        pr.strain_basis = shapes.make_basis((p["N_S_Gx"], p["N_S_Gy"], p["N_S_Gz"]),
                                            (g0["SL1"], g0["SL2"], g0["SL3"]), K)
        chi_s = [None] + [shapes.chi_table(pr.strain_basis, geo, s, 1, soft, sig) for s in range(1, ns)]
        same = all(pr.basis["N"][a] == pr.strain_basis["N"][a] for a in range(3)) and \
            (g0["L1"], g0["L2"], g0["L3"]) == (g0["SL1"], g0["SL2"], g0["SL3"])
        if same:
            chi_es = [None] + [chi_s[s].copy() for s in range(1, ns)]  # main:425-442
        else:
            chi_es = [None] + [shapes.chi_table(pr.basis, geo, s, 0, soft, sig) for s in range(1, ns)]
        eps_s = strain.strain_region(pr.strain_basis, geo, pr.params, chi_s, p["Isotropic"], p["Elastic_const"],
                                     p["Elastic_const_order"])
        if pr.strain_type == 1:  # main:587-600, 634-646
            def down(t):
                return strain.downsample_commensurate(t, pr.basis, pr.strain_basis, geo, soft, sig)
        else:
            def down(t):
                return strain.downsample(t, pr.basis, pr.strain_basis, geo)
        eps = {c: down(eps_s[c]) for c in strain.COMPONENTS}
        phi = None
        if p["Piezo"] != 0:
            phi_s = strain.piezo_region(pr.strain_basis, geo, pr.params, chi_s, eps_s, p["Piezo"])
            phi = down(phi_s)
        conv = strain.convolutions(chi_es, eps, ns)
        pr.tables = hamiltonian.Tables(chi_es, eps, conv, phi)
        pr.chi_strain, pr.eps_strain = chi_s, eps_s
    else:
        chi_es = [None] + [shapes.chi_table(pr.basis, geo, s, 0, soft, sig) for s in range(1, ns)]
        pr.tables = hamiltonian.Tables(chi_es)
    pr.F = (p["Fx"], p["Fy"], p["Fz"])
    Nx, Ny, Nz = pr.basis["N"]
    pr.n_pw = Nx * Ny * Nz
    pr.n_h = 8 * pr.n_pw
    return pr


def assemble(pr, full=False):
    return hamiltonian.assemble(pr.basis, pr.geo, pr.params, pr.tables, pr.F, pr.p["Strain"],
                                pr.p["Piezo"], full=full)


def solve(pr, H=None):
    """eigenstates.c:23-117 with the oracle's zheevr."""
    if H is None:
        H = assemble(pr)
    lo, hi = eigen.index_window(pr.n_pw, pr.p["N_VB"], pr.p["N_CB"])
    w, v = eigen.diagonalise(H, lo, hi)
    return w, v


def energies(pr, w, v):
    """Rows of energies_vb.dat (highest first) and energies_cb.dat."""
    (Ev, Vv), (Ec, Vc) = eigen.collect(w, v, pr.p["N_VB"])
    rows_vb = eigen.energies_rows(Ev, eigen.bloch_character(Vv, pr.n_pw))[::-1]
    rows_cb = eigen.energies_rows(Ec, eigen.bloch_character(Vc, pr.n_pw))
    return rows_vb, rows_cb


def run(directory, overrides=()):
    p, geo = inputs.load(directory, overrides)
    pr = prepare(p, geo)
    w, v = solve(pr)
    return pr, w, v, energies(pr, w, v)


def kramers_sum(rows):
    """Sum consecutive pairs of Bloch columns (the spin-degenerate pairs)."""
    rows = np.asarray(rows)
    return rows[0::2, 1:] + rows[1::2, 1:]

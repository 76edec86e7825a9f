"""Position-dependent elastic constants in the oracle (CPU).

strain_region_reciprocal_space.c:141-418 treats each shape's own elastic
constants perturbatively: an initial term, a zeroth-order term with the shape's
constants, and Elastic_const_order corrections, each the convolution of the
shape's characteristic function with the previous correction times a factor of
the constant differences and the matrix's Green tensor.  Two properties pin
the restatement:
* when every shape has the matrix's constants the treatment reduces to the
  position-independent strain for any number of orders (the zeroth-order
  factor becomes the usual one minus delta_ij and the corrections vanish);
* for an InAs dot in GaAs the corrections shrink order by order.
"""

import numpy as np
import pytest

from oracle import inputs, materials, shapes, strain
from qudos_b200 import configs as C


def _deck(tmp_path, matrix_like):
    x_dot = 1.0 if matrix_like else 0.0  # GaAs (the matrix) or InAs
    params = C.parameters_text(N_shape=2, M_Gx=2, M_Gy=2, M_Gz=2, M_S_Gx=2, M_S_Gy=2, M_S_Gz=2, Piezo=0,
                               Elastic_const=1, Elastic_const_order=3)
    cell = C.supercell_record((20.0, 20.0, 16.0)) + C.shape_record(4, 3, x_dot, 0.0, (0.0, 0.0, -1.0),
                                                                     (6.0, 6.0, 3.0))
    return inputs.load(C.write_deck(str(tmp_path / ("e%d" % matrix_like)), params, cell))


def _setup(tmp_path, matrix_like):
    p, geo = _deck(tmp_path, matrix_like)
    g0 = geo[0]
    basis = shapes.make_basis((p["N_S_Gx"], p["N_S_Gy"], p["N_S_Gz"]), (g0["SL1"], g0["SL2"], g0["SL3"]))
    params = materials.material_parameters(p["T"], geo, p["Piezo"])
    chi = [None] + [shapes.chi_table(basis, geo, s, 1) for s in range(1, len(geo))]
    return basis, geo, params, chi


@pytest.mark.parametrize("isotropic", [0, 1])
def test_matrix_constants_reduce_to_position_independent(tmp_path, isotropic):
    basis, geo, params, chi = _setup(tmp_path, True)
    # the dot's lattice constant differs (a mismatch is needed for any strain), its elastic constants do not
    params[1]["a"] = params[0]["a"] * 1.05
    ref = strain.strain_region(basis, geo, [dict(q) for q in params], chi, isotropic)
    for order in (0, 3):
        got = strain.strain_region(basis, geo, [dict(q) for q in params], chi, isotropic, 1, order)
        for c in strain.COMPONENTS:
            assert np.abs(got[c] - ref[c]).max() <= 1e-14 * max(np.abs(ref[c]).max(), 1e-300), (c, order)


def test_corrections_shrink_order_by_order(tmp_path):
    basis, geo, params, chi = _setup(tmp_path, False)
    eps = [strain.strain_region(basis, geo, [dict(q) for q in params], chi, 0, 1, k) for k in range(4)]
    steps = [max(np.abs(eps[k + 1][c] - eps[k][c]).max() for c in strain.COMPONENTS) for k in range(3)]
    assert steps[0] > 0
    assert steps[1] < 0.5 * steps[0] and steps[2] < 0.5 * steps[1], steps

"""Host-side logic of libqdgpu on the CPU: input readers, material
interpolation, error reporting and the exported C-ABI.  No GPU needed."""

import ctypes
import os
import re

import numpy as np
import pytest

import qudos_b200 as q
from qudos_b200 import lib as L
from oracle import inputs, materials
import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "qudos_b200.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    names = set(re.findall(r"\b(qd_[a-z0-9_]+)\s*\(", hdr))
    names |= {"hamiltonian_8_band", "diagonalise_hamiltonian", "eigenstates", "coulomb_matrix_elements",
              "eigen_gradients_8_band", "eigenstates_batched"}
    missing = [n for n in sorted(names) if not hasattr(L.lib, n)]
    assert not missing, missing
    for g in ("N_H", "na_rows", "characteristic_function_G", "strain_G", "convolutions_char_strain",
              "phi_piezo_G", "include_strain", "include_piezo", "component_run_times", "qd_grad_method"):
        ctypes.c_int.in_dll(L.lib, g)  # global exported


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_inputs_and_materials_match_oracle(name, tmp_path):
    d = cases.CASES[name](2, tmp_path)
    pr = q.Problem(d)
    p, geo = inputs.load(d)
    ns = p["N_shape"]
    om = materials.material_parameters(p["T"], inputs.clone(geo), p["Piezo"])
    cm = pr.materials(ns)
    for s in range(ns):
        for k in om[s]:
            assert cm[s][k] == pytest.approx(om[s][k], rel=0, abs=1e-15), (s, k)
    cg = pr.geometry(ns)
    for s in range(ns):
        for k in ("shape", "embedded", "material", "x", "y", "Ox", "Oy", "Oz", "L1", "L2", "L3", "L4", "SL1", "SL2",
                  "SL3", "CL1", "alpha", "beta", "gamma"):
            assert cg[s][k] == geo[s][k], (s, k)
    n_pw = p["N_Gx"] * p["N_Gy"] * p["N_Gz"]
    assert pr.n_pw == n_pw and pr.n_h == 8 * n_pw
    assert (pr.lo, pr.hi) == (6 * n_pw - 2 * p["N_VB"], 6 * n_pw + 2 * p["N_CB"] - 1)


def test_golden_inputs_parse(tmp_path):
    pr = q.Problem(os.path.join(ROOT, "tests", "golden", "prism_111"))
    assert pr.n_h == 10648 and (pr.lo, pr.hi) == (7978, 7989)
    pr2 = q.Problem(os.path.join(ROOT, "tests", "golden", "prism_111"), ["-M_Gx=2", "-N_VB=2"])
    assert pr2.n_pw == 5 * 11 * 11 and pr2.hi - pr2.lo + 1 == 2 * 2 + 2 * 2


def _write(tmp_path, params, cell):
    (tmp_path / "parameters.in").write_text(params)
    (tmp_path / "supercell.in").write_text(cell)
    return str(tmp_path)


def test_missing_parameter_is_an_error_not_an_exit(tmp_path):
    from qudos_b200 import configs as C
    params = C.parameters_text().replace("Piezo: 1\n", "")
    d = _write(tmp_path, params, C.lens_7()[1])
    with pytest.raises(q.QDError) as e:
        q.Problem(d)
    assert e.value.code == 1 and "Piezo" in str(e.value)


def test_shape_count_mismatch(tmp_path):
    from qudos_b200 import configs as C
    p, c = C.lens_7()
    d = _write(tmp_path, p.replace("N_shape: 3", "N_shape: 4"), c)
    with pytest.raises(q.QDError, match="greater than the number of shapes"):
        q.Problem(d)
    d2 = _write(tmp_path, p.replace("N_shape: 3", "N_shape: 2"), c)
    with pytest.raises(q.QDError, match="less than the number of shapes"):
        q.Problem(d2)


def test_unknown_material_and_missing_file(tmp_path):
    from qudos_b200 import configs as C
    p, c = C.lens_7()
    d = _write(tmp_path, p, c.replace("Material: 3", "Material: 22", 1))
    with pytest.raises(q.QDError, match="material system"):
        q.Problem(d)
    with pytest.raises(q.QDError, match="parameters.in"):
        q.Problem(str(tmp_path / "nowhere"))


def test_malformed_line_and_override(tmp_path):
    from qudos_b200 import configs as C
    p, c = C.lens_7()
    d = _write(tmp_path, p + "this line has no colon\n", c)
    with pytest.raises(q.QDError, match="malformed"):
        q.Problem(d)
    d = _write(tmp_path, p, c)
    with pytest.raises(q.QDError, match="override"):
        q.Problem(d, ["M_Gx=3"])


def test_reference_arm_loads_no_native_code():
    """bench.py --impl reference runs the oracle only: the deck writer and the
    oracle import without loading libqdgpu.so."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import bench; bench.oracle_solve; "
            "from qudos_b200 import configs; import oracle.pipeline; "
            "maps = open('/proc/self/maps').read(); "
            "print(int('qudos_b200.lib' in sys.modules), int('libqdgpu' in maps))" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["0", "0"]


def test_tuning_table_and_cache(tmp_path):
    """The autotuner's cache goes into the library's tuning table; depths
    outside 32..256 or not multiples of 32 are rejected."""
    import json
    from qudos_b200 import autotune
    path = tmp_path / "tuning.json"
    path.write_text(json.dumps({"entries": [{"n_h": 2744, "prec": "mixed", "depth": 128},
                                            {"n_h": 27000, "prec": "mixed", "depth": 256},
                                            {"n_h": 27000, "prec": "fp64", "depth": 192}]}))
    try:
        assert autotune.load(str(path)) == 3
        assert L.lib.qd_tuning_set(L.QD_PREC_MIXED, 1000, 300) == L.QD_ERR_ARG
        assert L.lib.qd_tuning_set(L.QD_PREC_MIXED, 1000, 100) == L.QD_ERR_ARG
        assert L.lib.qd_tuning_set(7, 1000, 128) == L.QD_ERR_ARG
        assert autotune.load(str(tmp_path / "absent.json")) == 0
    finally:
        autotune.load()


@pytest.mark.parametrize("name", ["molecule", "all_shapes"])
def test_material_tangents_match_central_differences(name, tmp_path):
    """qd_material_tangent, the exact d(material parameters)/d(scale) behind the
    Ep and gamma_1 gradients, against central differences of the host material
    function in the scale of the binary table's Ep and gamma_1 columns
    (qd_scale_Ep, qd_scale_gL1); every field that the scale does not move must
    have a zero tangent."""
    d = cases.CASES[name](2, tmp_path)
    p, _ = inputs.load(d)
    pr = q.Problem(d)
    ns = pr.n_shape
    geo = (L.SupercellGeometry * ns)()
    L.check(L.lib.qd_problem_geometry(pr.handle, geo, ns))
    mat_fn = L.lib.qd_material_parameters
    mat_fn.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    tan_fn = L.lib.qd_material_tangent
    tan_fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    scales = {0: ctypes.c_double.in_dll(L.lib, "qd_scale_Ep"), 1: ctypes.c_double.in_dll(L.lib, "qd_scale_gL1")}
    fields = [f for f, _ in L.MaterialParams._fields_]

    def mats(which=None, scale=1.0):
        out = (L.MaterialParams * ns)()
        if which is not None:
            scales[which].value = scale
        try:
            L.check(mat_fn(p["T"], p["Piezo"], ns, ctypes.addressof(geo), ctypes.addressof(out)))
        finally:
            scales[0].value = scales[1].value = 1.0
        return out

    base = mats()
    ref = pr.materials(ns)  # the problem's own materials: same function, same inputs
    for s in range(ns):
        for f in fields:
            assert getattr(base[s], f) == ref[s][f], (s, f)
    h = 1e-5
    for which in (0, 1):
        dm = (L.MaterialParams * ns)()
        L.check(tan_fn(which, ns, ctypes.addressof(geo), ctypes.addressof(base), ctypes.addressof(dm)))
        plus, minus = mats(which, 1.0 + h), mats(which, 1.0 - h)
        moved = 0
        for s in range(ns):
            for f in fields:
                fd = (getattr(plus[s], f) - getattr(minus[s], f)) / (2 * h)
                ex = getattr(dm[s], f)
                scale = max(abs(getattr(base[s], f)), 1e-3)
                assert abs(fd - ex) <= 1e-7 * scale, (which, s, f, fd, ex)
                moved += ex != 0.0
        assert moved > 0

"""ctypes binding of libqdgpu.so (the C-ABI in include/qudos_b200.h).

The library is loaded once, at import.  There is no fallback: if the shared
library is missing or cannot be loaded the import raises.
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqdgpu.so")

QD_OK = 0
QD_ERR = {1: "INPUT", 2: "UNSUPPORTED", 3: "CUDA", 4: "NOMEM", 5: "CONVERGENCE", 6: "TIMEOUT", 7: "ARG"}
QD_PREC_FP64, QD_PREC_MIXED = 0, 1
QD_ERR_ARG = 7
QD_STATIC_TRI_MAX = 65536  # rows of the allocation-free tridiagonal scratch

if not os.path.exists(LIB_PATH):
    raise ImportError("libqdgpu.so is not built: run `python qudos_b200/build.py`")
lib = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)


class QDError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("qudos_b200 error %d (%s): %s" % (code, QD_ERR.get(code, "?"), msg))
        self.code = code


def check(rc):
    if rc != QD_OK:
        raise QDError(rc, lib.qd_last_error_message().decode())
    return rc


class MaterialParams(C.Structure):
    """struct material_params (8_band.h:200)."""
    _fields_ = [(n, C.c_double) for n in (
        "a", "C11", "C12", "C44", "e14", "B114", "B124", "B156", "Eg", "Dso", "Ep", "P", "sc", "g1", "g2", "g3",
        "ac", "av", "b", "d", "Ev_avg", "E_so", "E_lh", "E_hh", "E_cb", "nr")]


class SupercellGeometry(C.Structure):
    """struct supercell_geometry (8_band.h:197)."""
    _fields_ = ([(n, C.c_int) for n in ("shape", "embedded", "material", "material_type", "RL1", "RL2", "RL3",
                                         "RCL1", "RCL2", "RCL3")] +
                [(n, C.c_double) for n in ("x", "y", "Ox", "Oy", "Oz", "L1", "L2", "L3", "L4", "L5", "SL1", "SL2",
                                           "SL3", "CL1", "CL2", "CL3", "alpha", "beta", "gamma")])


class Vector(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class WaveVectors(C.Structure):
    """struct wave_vectors (8_band.h:117-124)."""
    _fields_ = [("N_Gx", C.c_int), ("N_Gy", C.c_int), ("N_Gz", C.c_int), ("N_Gx_T", C.c_int), ("N_Gy_T", C.c_int),
                ("N_Gz_T", C.c_int), ("Gx", C.POINTER(C.c_double)), ("Gy", C.POINTER(C.c_double)),
                ("Gz", C.POINTER(C.c_double)), ("Kx", C.c_double), ("Ky", C.c_double), ("Kz", C.c_double)]


class Eigenstate(C.Structure):
    """struct eigenstate (8_band.h:209-211)."""
    _fields_ = ([("idx_state", C.c_int), ("E", C.c_double)] +
                [(n, C.POINTER(C.c_double)) for n in ("bloch",) + tuple("probability_%d" % i for i in range(1, 9))] +
                [(n, C.c_void_p) for n in ("fourier",) + tuple("F_%d" % i for i in range(1, 9))])


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


vp, i64, ci = C.c_void_p, C.c_int64, C.c_int
_sig("qd_last_error_message", C.c_char_p, [])
_sig("qd_version", ci, [])
_sig("qd_problem_load", ci, [C.c_char_p, C.POINTER(C.c_char_p), ci, C.POINTER(vp)])
_sig("qd_problem_free", None, [vp])
_sig("qd_problem_n_shape", ci, [vp])
_sig("qd_problem_field", ci, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)])
_sig("qd_problem_assemble_dk_dev", ci, [vp, ci, vp, i64, ci, vp])
_sig("qd_momentum_matrix_elements", ci, [vp, vp, ci, ci, vp])
_sig("qd_envelope_functions", ci, [vp, vp, ci, ci, vp, vp, vp, vp, vp])
_sig("qd_launch_count", C.c_longlong, [])
_sig("qd_problem_sizes", ci, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(ci), C.POINTER(ci), C.POINTER(ci),
                              C.POINTER(ci)])
_sig("qd_problem_materials", ci, [vp, C.POINTER(MaterialParams), ci])
_sig("qd_problem_geometry", ci, [vp, C.POINTER(SupercellGeometry), ci])
_sig("qd_problem_build_tables", ci, [vp])
_sig("qd_problem_get_table", ci, [vp, ci, ci, ci, vp, i64])
_sig("qd_problem_assemble_dev", ci, [vp, vp, i64, ci, ci, vp])
_sig("qd_eigh_window_dev", ci, [i64, vp, i64, ci, ci, ci, vp, vp, i64, vp])
_sig("qd_problem_solve", ci, [vp, ci, vp, vp])
_sig("qd_coulomb", ci, [vp, ci, ci, vp, ci, vp, vp, vp, vp])
_sig("qd_last_timings", ci, [C.POINTER(C.c_double), ci])
_sig("qd_stage1_profile", ci, [C.POINTER(C.c_double), ci])
class GradParam(C.Structure):
    _fields_ = [("kind", ci), ("shape", ci), ("index", ci)]


QD_GRAD_LENGTH, QD_GRAD_BASE, QD_GRAD_COMPOSITION, QD_GRAD_FIELD, QD_GRAD_EP, QD_GRAD_GAMMA1 = range(6)
_sig("eigenstates_batched", ci, [C.POINTER(vp), ci, ci, ci, C.POINTER(vp), C.POINTER(vp)])
_sig("eigen_gradients_8_band", ci, [vp, vp, ci, C.POINTER(GradParam), ci, C.c_double, vp])
_sig("qd_tc_work_alloc", ci, [i64, ci, C.POINTER(vp)])
_sig("qd_tc_work_free", None, [vp])
_sig("qd_tc_work_check", ci, [vp])
_sig("qd_tc_xprod", ci, [vp, i64, i64, i64, ci, vp, i64, ci, vp, i64, vp, vp])
_sig("qd_tc_flush", ci, [vp, i64, i64, ci, vp, vp, i64, i64, ci, vp, vp])
_sig("qd_tc_kernel_stats", ci, [ci, C.POINTER(C.c_longlong), C.POINTER(C.c_double), C.POINTER(C.c_double)])
_sig("qd_tc_kernel_launches", ci, [ci, ci, C.POINTER(C.c_double), C.POINTER(C.c_double)])
_sig("qd_gemm_peak", ci, [ci, ci, ci, C.POINTER(C.c_double)])
_sig("qd_tsmm_nn", ci, [ci, ci, ci, ci, C.POINTER(vp), C.POINTER(i64), C.POINTER(vp), C.POINTER(i64), C.POINTER(ci),
                        C.POINTER(ci), C.POINTER(C.c_double), vp, i64, C.c_double, vp])
_sig("qd_tsmm_cn", ci, [ci, ci, vp, i64, ci, vp, i64, ci, vp, i64, vp, C.c_size_t, vp])
_sig("qd_small_cn", ci, [ci, ci, ci, ci, vp, ci, vp, ci, C.c_double, vp, ci, vp])
_sig("qd_tsmm_cn_scratch_bytes", C.c_size_t, [ci, ci, ci, ci])
_sig("qd_set_wait_limits", ci, [C.c_longlong, C.c_longlong, C.c_longlong])
_sig("qd_tuning_set", ci, [ci, C.c_int64, ci])
_sig("qd_hemm_lower_dev", ci, [i64, vp, i64, vp, i64, ci, vp, i64, C.c_double, vp])
_sig("qd_gram_dev", ci, [i64, vp, i64, ci, vp, i64, ci, vp, ci, vp])
_sig("qd_zgemm_small_dev", ci, [i64, vp, i64, ci, vp, ci, ci, vp, i64, C.c_double, vp])
_sig("qd_problem_residuals", ci, [vp, ci, vp, vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_double)])
_sig("qd_last_error_bounds", ci, [vp, vp, ci])
_sig("qd_tridiag_eigvals_noalloc", ci, [vp, ci, ci, ci, ci, vp, vp])
_sig("qd_tridiag_bisect", ci, [vp, ci, ci, ci, ci, vp, vp, vp, vp, vp])
_sig("qd_dev_alloc", ci, [C.c_size_t, C.POINTER(vp)])
_sig("qd_dev_free", ci, [vp])
_sig("qd_memcpy", ci, [vp, vp, C.c_size_t, ci])
_sig("qd_memset", ci, [vp, ci, C.c_size_t])
_sig("qd_host_alloc_pinned", ci, [C.c_size_t, C.POINTER(vp)])
_sig("qd_host_free_pinned", ci, [vp])
_sig("qd_device_synchronize", ci, [])
_sig("qd_device_count", ci, [C.POINTER(ci)])
_sig("qd_set_device", ci, [ci])
_sig("qd_event_create", ci, [C.POINTER(vp)])
_sig("qd_event_record", ci, [vp, vp])
_sig("qd_event_elapsed_ms", ci, [vp, vp, C.POINTER(C.c_float)])
_sig("qd_event_destroy", ci, [vp])
_sig("hamiltonian_8_band", None, [ci, Vector, WaveVectors, C.POINTER(SupercellGeometry), C.POINTER(MaterialParams),
                                  vp])
_sig("diagonalise_hamiltonian", None, [C.POINTER(ci), vp, vp, vp])
_sig("eigenstates", None, [ci, C.POINTER(ci), Vector, WaveVectors, C.POINTER(SupercellGeometry),
                           C.POINTER(MaterialParams), C.POINTER(Eigenstate), C.POINTER(Eigenstate)])


class Complex128(C.Structure):
    """A C double _Complex returned by value (two doubles, returned in SSE registers on x86-64)."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


_sig("hamiltonian_derivative_8_band", None, [ci, ci, WaveVectors, C.POINTER(SupercellGeometry),
                                             C.POINTER(MaterialParams), vp])
_sig("momentum_matrix_element", Complex128, [ci, ci, WaveVectors, C.POINTER(SupercellGeometry),
                                             C.POINTER(MaterialParams), Eigenstate, C.c_int64, Eigenstate, C.c_int64,
                                             C.POINTER(ci)])


_sig("envelope_functions", None, [C.POINTER(SupercellGeometry), C.POINTER(ci), ci, ci, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), WaveVectors, C.POINTER(Eigenstate), ci])


def device_count():
    n = ci(0)
    rc = lib.qd_device_count(C.byref(n))
    return n.value if rc == QD_OK else 0


class DeviceBuffer:
    """Owned device allocation."""

    def __init__(self, nbytes):
        self._free = lib.qd_dev_free  # held: module globals may be gone when collected at exit
        self.ptr = None
        p = vp()
        check(lib.qd_dev_alloc(int(nbytes), C.byref(p)))
        self.ptr = p
        self.nbytes = int(nbytes)

    def free(self):
        p, self.ptr = getattr(self, "ptr", None), None
        if p:
            self._free(p)

    def __del__(self):
        self.free()

    def upload(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        check(lib.qd_memcpy(self.ptr, arr.ctypes.data, arr.nbytes, 1))

    def download(self, arr):
        assert arr.flags.c_contiguous or arr.flags.f_contiguous
        check(lib.qd_memcpy(arr.ctypes.data, self.ptr, arr.nbytes, 2))
        return arr


class Event:
    def __init__(self):
        self._destroy = lib.qd_event_destroy  # held: module globals may be gone when collected at exit
        self.ev = vp()
        check(lib.qd_event_create(C.byref(self.ev)))

    def record(self, stream=None):
        check(lib.qd_event_record(self.ev, stream))

    def elapsed_ms(self, later):
        ms = C.c_float(0)
        check(lib.qd_event_elapsed_ms(self.ev, later.ev, C.byref(ms)))
        return float(ms.value)

    def __del__(self):
        ev, self.ev = getattr(self, "ev", None), None
        if ev:
            self._destroy(ev)


def stage1_profile():
    a = (C.c_double * 8)()
    lib.qd_stage1_profile(a, 8)
    return list(a)


def last_timings():
    a = (C.c_double * 8)()
    lib.qd_last_timings(a, 8)
    return list(a)

"""Python mirror of the QUDOS PWEM solve path on top of libqdgpu.

`Problem` corresponds to one run of the reference's 8_band_pwem.ex up to and
including `eigenstates` (code/source/8_band/8_band_main.c:142-763): the same
`parameters.in` / `supercell.in` files and `-Key=value` overrides, the same
index window and the same outputs (energies, Bloch characters, envelope
Fourier coefficients).  Every numerical step runs in libqdgpu on the GPU.
"""

import ctypes as C
import os

import numpy as np

from . import lib as L

TABLE_CHI, TABLE_STRAIN, TABLE_PHI, TABLE_CONV, TABLE_CHI_S, TABLE_STRAIN_S, TABLE_PHI_S, TABLE_COEF = range(8)


class Problem:
    def __init__(self, directory, overrides=()):
        self._h = C.c_void_p()
        arr = (C.c_char_p * max(1, len(overrides)))(*[o.encode() for o in overrides])
        L.check(L.lib.qd_problem_load(os.fsencode(directory), arr, len(overrides), C.byref(self._h)))
        n_pw, n_h = C.c_int64(), C.c_int64()
        lo, hi, nvb, ncb = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib.qd_problem_sizes(self._h, C.byref(n_pw), C.byref(n_h), C.byref(lo), C.byref(hi),
                                       C.byref(nvb), C.byref(ncb)))
        self.n_pw, self.n_h, self.lo, self.hi = n_pw.value, n_h.value, lo.value, hi.value
        self.n_vb, self.n_cb = nvb.value, ncb.value
        self.m = self.hi - self.lo + 1
        self.n_shape = L.lib.qd_problem_n_shape(self._h)

    def close(self):
        if self._h:
            L.lib.qd_problem_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    def materials(self, n_shape):
        arr = (L.MaterialParams * n_shape)()
        L.check(L.lib.qd_problem_materials(self._h, arr, n_shape))
        return [{f: getattr(a, f) for f, _ in L.MaterialParams._fields_} for a in arr]

    def geometry(self, n_shape):
        arr = (L.SupercellGeometry * n_shape)()
        L.check(L.lib.qd_problem_geometry(self._h, arr, n_shape))
        return [{f: getattr(a, f) for f, _ in L.SupercellGeometry._fields_} for a in arr]

    def build_tables(self):
        L.check(L.lib.qd_problem_build_tables(self._h))

    def table(self, which, s, c, shape):
        out = np.empty(shape, dtype=np.complex128)
        L.check(L.lib.qd_problem_get_table(self._h, which, s, c, out.ctypes.data, out.size))
        return out

    def assemble(self, mode=0, prec=L.QD_PREC_FP64):
        """H on the device, copied back as a numpy array (column-major N_H x N_H)."""
        n = self.n_h
        es = 16 if prec == L.QD_PREC_FP64 else 8
        buf = L.DeviceBuffer(n * n * es)
        L.check(L.lib.qd_memset(buf.ptr, 0, n * n * es))
        L.check(L.lib.qd_problem_assemble_dev(self._h, buf.ptr, n, mode, prec, None))
        L.check(L.lib.qd_device_synchronize())
        H = np.empty((n, n), dtype=np.complex128 if es == 16 else np.complex64, order="F")
        buf.download(H)
        buf.free()
        return H

    def solve(self, prec=L.QD_PREC_FP64):
        """Eigenpairs of the window [lo, hi]: (eigval[M], eigvec N_H x M)."""
        w = np.empty(self.m)
        v = np.empty((self.n_h, self.m), dtype=np.complex128, order="F")
        L.check(L.lib.qd_problem_solve(self._h, prec, w.ctypes.data, v.ctypes.data))
        return w, v

    def residuals(self, w, v):
        """FP64 check of eigenpairs against this problem's H, assembled on the
        device: (||H v_j - w_j v_j|| per state in eV, max |V^H V - I|, max |H_ij|)."""
        v = np.asfortranarray(v, dtype=np.complex128)
        w = np.ascontiguousarray(w, dtype=np.float64)
        m = v.shape[1]
        res = np.zeros(m)
        orth, hn = C.c_double(0), C.c_double(0)
        L.check(L.lib.qd_problem_residuals(self._h, m, w.ctypes.data, v.ctypes.data, res.ctypes.data, C.byref(orth),
                                           C.byref(hn)))
        return res, orth.value, hn.value

    def coulomb(self, v, n_vb_states, n_cb_states, madelung_ranks=1):
        """Coulomb matrix elements of the states v (N_H x M, VB states first)
        with the deck's CME setting (coulomb_matrix_elements.c:24).  Returns
        the reference's four flat arrays hh, ee, eh_direct, eh_exchange."""
        nv, nc = n_vb_states, n_cb_states
        v = np.asfortranarray(v, dtype=np.complex128)
        out = {"hh": np.zeros(nv ** 4, np.complex128), "ee": np.zeros(nc ** 4, np.complex128),
               "eh_direct": np.zeros(nv * nv * nc * nc, np.complex128),
               "eh_exchange": np.zeros(nv * nv * nc * nc, np.complex128)}
        L.check(L.lib.qd_coulomb(self._h, nv, nc, v.ctypes.data, madelung_ranks, out["hh"].ctypes.data,
                                 out["ee"].ctypes.data, out["eh_direct"].ctypes.data, out["eh_exchange"].ctypes.data))
        return out

    def gradients(self, v, params, rel_step=1e-4):
        """Hellmann-Feynman derivatives <psi_n| dH/dp |psi_n> of the states v
        (N_H x M) for params = [(kind, shape, index), ...] (lib.QD_GRAD_*).
        Returns (len(params), M): per nm, per unit composition, per kV/cm or per
        unit relative scale."""
        v = np.asfortranarray(v, dtype=np.complex128)
        m = v.shape[1]
        arr = (L.GradParam * len(params))(*[L.GradParam(*p) for p in params])
        out = np.zeros((len(params), m))
        L.check(L.lib.eigen_gradients_8_band(self._h, v.ctypes.data, m, arr, len(params), rel_step,
                                             out.ctypes.data))
        return out

    def energies(self, w, v):
        """Rows of energies_vb.dat (highest state first) and energies_cb.dat
        (write_energies.c:23-93; Bloch characters bloch_character.c:23-105)."""
        m_vb = 2 * self.n_vb
        a = np.abs(v.reshape(8, self.n_pw, -1)) ** 2  # row = band * n_pw + plane wave
        bl = a.sum(axis=1).T
        rows = np.stack([w, 100.0 * (bl[:, 3] + bl[:, 7]), 100.0 * (bl[:, 2] + bl[:, 6]),
                         100.0 * (bl[:, 1] + bl[:, 5]), 100.0 * (bl[:, 0] + bl[:, 4])], axis=1)
        return rows[:m_vb][::-1], rows[m_vb:]


def last_error_bounds():
    """Per-state FP64 residual norms and Kato-Temple eigenvalue error bounds (eV)
    of the window of the last mixed-precision solve on this host thread."""
    n = L.lib.qd_last_error_bounds(None, None, 0)
    res, bound = np.zeros(n), np.zeros(n)
    if n:
        L.lib.qd_last_error_bounds(res.ctypes.data, bound.ctypes.data, n)
    return res, bound


def solve_batch(problems, prec=L.QD_PREC_MIXED, n_threads=8):
    """Solve independent problems concurrently (eigenstates_batched).  Returns a
    list of (eigval[M], eigvec N_H x M) in the order of `problems`."""
    outs = [(np.empty(p.m), np.empty((p.n_h, p.m), dtype=np.complex128, order="F")) for p in problems]
    n = len(problems)
    hs = (C.c_void_p * n)(*[p.handle.value for p in problems])
    ws = (C.c_void_p * n)(*[o[0].ctypes.data for o in outs])
    vs = (C.c_void_p * n)(*[o[1].ctypes.data for o in outs])
    L.check(L.lib.eigenstates_batched(hs, n, prec, n_threads, ws, vs))
    return outs


def eigh_window_dev(n, H_dev, ld, lo, hi, prec, w_dev, Z_dev, ldz, stream=None):
    L.check(L.lib.qd_eigh_window_dev(n, H_dev, ld, lo, hi, prec, w_dev, Z_dev, ldz, stream))


def write_energies(directory, rows_vb, rows_cb):
    fmt = "%17.10e\t%17.10e\t%17.10e\t%17.10e\t%17.10e\n"
    with open(os.path.join(directory, "energies_vb.dat"), "w") as f:
        f.write("".join(fmt % tuple(r) for r in rows_vb))
    with open(os.path.join(directory, "energies_cb.dat"), "w") as f:
        f.write("".join(fmt % tuple(r) for r in rows_cb))

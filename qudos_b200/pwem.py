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
    def __init__(self, directory, overrides=(), tuned=True):
        """Loads parameters.in / supercell.in from directory.  tuned: put the
        package's autotuner cache into the library's tuning table (once per
        process) before the first solve."""
        # held on the instance: a Problem collected at interpreter exit may
        # find this module's globals already cleared
        self._free = L.lib.qd_problem_free
        if tuned:
            from . import autotune
            autotune.ensure_loaded()
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
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._free(h)

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

    def field(self):
        """(F in V/Angstrom, K in 1/Angstrom) as the reference's routines take them."""
        F, K = (C.c_double * 3)(), (C.c_double * 3)()
        L.check(L.lib.qd_problem_field(self._h, F, K))
        return tuple(F), tuple(K)

    def momentum(self, v, n_vb_states, n_cb_states):
        """Interband momentum matrix elements (8_band_main.c:1578-1680):
        p[pol, c, v] = <vb_(n_vb_states-1-v)| dH/dk_pol |cb_c> in eV Angstrom, pol
        0, 1, 2 = [100], [010], [001]; v holds the VB states first."""
        v = np.asfortranarray(v, dtype=np.complex128)
        out = np.zeros((3, n_cb_states, n_vb_states), dtype=np.complex128)
        L.check(L.lib.qd_momentum_matrix_elements(self._h, v.ctypes.data, n_vb_states, n_cb_states,
                                                  out.ctypes.data))
        return out

    def envelopes(self, v, x, y, z):
        """Band envelopes F (states, 8, points) and |F|^2 of the states v
        (N_H x M) at the points x, y, z (Angstrom), envelope_functions.c:23."""
        v = np.asfortranarray(v, dtype=np.complex128)
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        m, n = v.shape[1], len(x)
        F = np.zeros((m, 8, n), dtype=np.complex128)
        P = np.zeros((m, 8, n))
        L.check(L.lib.qd_envelope_functions(self._h, v.ctypes.data, m, n, x.ctypes.data, y.ctypes.data,
                                            z.ctypes.data, F.ctypes.data, P.ctypes.data))
        return F, P

    def assemble_dk(self, axis, mode=0):
        """dH/dk_axis on the device, copied back (column-major N_H x N_H complex128)."""
        n = self.n_h
        buf = L.DeviceBuffer(n * n * 16)
        L.check(L.lib.qd_memset(buf.ptr, 0, n * n * 16))
        L.check(L.lib.qd_problem_assemble_dk_dev(self._h, axis, buf.ptr, n, mode, None))
        L.check(L.lib.qd_device_synchronize())
        H = np.empty((n, n), dtype=np.complex128, order="F")
        buf.download(H)
        buf.free()
        return H

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


def write_momentum_matrix_elements(directory, mme):
    """momentum_matrix_elements.dat as write_momentum_matrix_elements.c:23-110
    writes it: per (CB state, VB state) row the 1-based indices, then Re, Im
    and |.| of the element for [100], [010], [001], [110] = (p_x + p_y)/sqrt 2
    and [-110] = (-p_x + p_y)/sqrt 2, divided by sqrt(HBSQM / 2) (eV^(1/2));
    a blank line after each CB state."""
    hb = np.sqrt(7.61996 / 2.0)
    n_pol, ncb, nvb = mme.shape
    with open(os.path.join(directory, "momentum_matrix_elements.dat"), "w") as f:
        for c in range(ncb):
            for v in range(nvb):
                px, py, pz = mme[0, c, v] / hb, mme[1, c, v] / hb, mme[2, c, v] / hb
                f.write("%d\t%d\t" % (c + 1, v + 1))
                for z in (px, py, pz, (px + py) / np.sqrt(2.0), (-px + py) / np.sqrt(2.0)):
                    f.write("%17.10e\t%17.10e\t%17.10e\t" % (z.real, z.imag, abs(z)))
                f.write("\n")
            f.write("\n")


LINESCAN_TAGS = ("100", "010", "001", "110", "101", "011", "111")


def write_probability_density(directory, direction, x, y, z, E_vb, prob_vb, E_cb, prob_cb):
    """probability_density_{vb,cb}_<k>_<dir>.dat as write_probability_density.c
    writes them (x, y, z in nm, energy, total / SO / LH / HH / CB densities in
    nm^-3); VB files count from the highest state.  prob_* are (states, 8,
    points) |F_b|^2 from Problem.envelopes; x, y, z in Angstrom."""
    tag = LINESCAN_TAGS[direction]

    def rows(E, p):
        p = 1000.0 * p
        return np.stack([0.1 * np.asarray(x), 0.1 * np.asarray(y), 0.1 * np.asarray(z), np.full(len(x), E),
                         p.sum(axis=0), p[3] + p[7], p[2] + p[6], p[1] + p[5], p[0] + p[4]], axis=1)

    fmt = "\t".join(["%13e"] * 9) + "\n"
    nv = len(E_vb)
    for k in range(nv):
        s = nv - 1 - k
        with open(os.path.join(directory, "probability_density_vb_%d_%s.dat" % (k + 1, tag)), "w") as f:
            f.writelines(fmt % tuple(r) for r in rows(E_vb[s], prob_vb[s]))
    for k in range(len(E_cb)):
        with open(os.path.join(directory, "probability_density_cb_%d_%s.dat" % (k + 1, tag)), "w") as f:
            f.writelines(fmt % tuple(r) for r in rows(E_cb[k], prob_cb[k]))


def write_energies(directory, rows_vb, rows_cb):
    fmt = "%17.10e\t%17.10e\t%17.10e\t%17.10e\t%17.10e\n"
    with open(os.path.join(directory, "energies_vb.dat"), "w") as f:
        f.write("".join(fmt % tuple(r) for r in rows_vb))
    with open(os.path.join(directory, "energies_cb.dat"), "w") as f:
        f.write("".join(fmt % tuple(r) for r in rows_cb))

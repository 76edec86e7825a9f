"""The reference's own routines, called the way its main program calls them.

QUDOS keeps its coefficient tables in global variables
(code/source/8_band/8_band.h:77-110,218-225) and passes the basis, geometry
and material parameters as structs to `hamiltonian_8_band`
(hamiltonian_8_band.c:23), `diagonalise_hamiltonian`
(diagonalise_hamiltonian.c:24), `eigenstates` (eigenstates.c:23) and
`coulomb_matrix_elements` (coulomb_matrix_elements.c:24).  `ReferenceCall`
fills libqdgpu's copies of those globals from host arrays (numpy, C order
iz + N_zT (iy + N_yT ix), the reference's table layout) and makes those calls
through the C ABI with host buffers, as 8_band_main.c:763 and :1822 do.

The tables can come from any source: `from_problem` reads them back from the
library's own GPU table build, `from_tables` takes arrays computed elsewhere.
"""

import ctypes as C

import numpy as np

from . import lib as L

CONV_KEYS = ("char_xx", "char_yy", "char_zz", "char_yz", "char_xz", "char_xy", "char_hydrostatic", "char_biaxial")


class _Chi(C.Structure):
    _fields_ = [("chi", C.c_void_p)]


class _Strain(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("xx", "yy", "zz", "yz", "xz", "xy")]


class _Conv(C.Structure):
    # struct convolution_char_strain (8_band.h:140-144): 32 table pointers, the first 8 read by the solve path
    _fields_ = [(k, C.c_void_p) for k in CONV_KEYS] + [("rest%d" % i, C.c_void_p) for i in range(24)]


class _CME(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("ee", "hh", "eh_direct", "eh_exchange")]


def basis_grid(n_t, length):
    """G_i = (2 pi / L)(i - (N_T - 1)/2), i < N_T (basis_set.c:62-85)."""
    return ((2.0 * np.pi) / length) * (0.5 * (1.0 - n_t) + np.arange(n_t, dtype=np.float64))


class ReferenceCall:
    def __init__(self, N, geo, mat, chi, eps=None, conv=None, phi=None, F=(0.0, 0.0, 0.0), K=(0.0, 0.0, 0.0),
                 include_cme=0, nprocs=1):
        """N: plane waves per axis; geo, mat: per-shape dicts (index 0 = matrix) of
        struct supercell_geometry / struct material_params; chi[s] (s >= 1),
        eps (6 components xx yy zz yz xz xy), conv[s] (8 tables in CONV_KEYS
        order) and phi on the (2N-1)^3 grid; F in V/Angstrom; K in 1/Angstrom."""
        self.N = tuple(int(n) for n in N)
        self.NT = tuple(2 * n - 1 for n in self.N)
        self.n_shape = len(geo)
        self.n_pw = self.N[0] * self.N[1] * self.N[2]
        self.n_h = 8 * self.n_pw
        self.geo, self.mat = geo, mat
        flat = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(-1))  # noqa: E731
        self._chi = [None] + [flat(chi[s]) for s in range(1, self.n_shape)]
        self._eps = [flat(e) for e in eps] if eps is not None else None
        self._conv = ([None] + [[flat(t) for t in conv[s]] for s in range(1, self.n_shape)]) if conv else None
        self._phi = flat(phi) if phi is not None else None
        self.F = L.Vector(*F)
        self._grids = [np.ascontiguousarray(basis_grid(nt, geo[0]["L" + str(a + 1)])) for a, nt in enumerate(self.NT)]
        self.basis = L.WaveVectors(*self.N, *self.NT,
                                   *[g.ctypes.data_as(C.POINTER(C.c_double)) for g in self._grids], *K)
        self.gstruct = (L.SupercellGeometry * self.n_shape)(*[L.SupercellGeometry(**g) for g in geo])
        self.mstruct = (L.MaterialParams * self.n_shape)(*[L.MaterialParams(**m) for m in mat])
        self.include_cme = include_cme
        self.nprocs = nprocs

    @classmethod
    def from_problem(cls, pr):
        """Tables of a loaded qudos_b200.Problem, read back from the GPU build."""
        ns = pr.n_shape
        geo, mat = pr.geometry(ns), pr.materials(ns)
        N = round(pr.n_pw ** (1.0 / 3.0))
        shp = (2 * N - 1,) * 3
        pr.build_tables()
        chi = [None] + [pr.table(0, s, 0, shp) for s in range(1, ns)]

        def optional(fn):  # tables of a disabled stage (no strain, no piezo) do not exist
            try:
                return fn()
            except L.QDError:
                return None

        eps = optional(lambda: [pr.table(1, c, 0, shp) for c in range(6)])
        phi = optional(lambda: pr.table(2, 0, 0, shp)) if eps is not None else None
        conv = optional(lambda: [None] + [[pr.table(3, s, c, shp) for c in range(8)] for s in range(1, ns)])
        F, K = pr.field()
        return cls((N, N, N), geo, mat, chi, eps, conv, phi, F=F, K=K)

    def _install(self):
        lib = L.lib
        ns = self.n_shape
        self._cf = (_Chi * ns)()
        for s in range(1, ns):
            self._cf[s].chi = self._chi[s].ctypes.data
        C.c_void_p.in_dll(lib, "characteristic_function_G").value = C.addressof(self._cf)
        strain_on = self._eps is not None
        C.c_int.in_dll(lib, "include_strain").value = 1 if strain_on else 0
        C.c_int.in_dll(lib, "include_piezo").value = 1 if (strain_on and self._phi is not None) else 0
        if strain_on:
            st = _Strain(*[e.ctypes.data for e in self._eps])
            C.memmove(C.addressof(_Strain.in_dll(lib, "strain_G")), C.addressof(st), C.sizeof(_Strain))
            self._cv = (_Conv * ns)()
            for s in range(1, ns):
                for k, t in zip(CONV_KEYS, self._conv[s]):
                    setattr(self._cv[s], k, t.ctypes.data)
            C.c_void_p.in_dll(lib, "convolutions_char_strain").value = C.addressof(self._cv)
        C.c_void_p.in_dll(lib, "phi_piezo_G").value = self._phi.ctypes.data if self._phi is not None else None
        C.c_int.in_dll(lib, "N_shape").value = ns
        C.c_int64.in_dll(lib, "N_H").value = self.n_h
        C.c_int64.in_dll(lib, "na_rows").value = self.n_h
        C.c_int64.in_dll(lib, "na_cols").value = self.n_h
        C.c_int.in_dll(lib, "nprocs").value = self.nprocs
        C.c_int.in_dll(lib, "myid").value = 0
        C.c_int.in_dll(lib, "PACKED").value = 0
        C.c_int.in_dll(lib, "include_CME").value = self.include_cme

    def hamiltonian(self):
        """hamiltonian_8_band into a zeroed host H (column-major N_H x N_H, lower triangle written)."""
        self._install()
        H = np.zeros((self.n_h, self.n_h), dtype=np.complex128, order="F")
        L.lib.hamiltonian_8_band(self.n_shape, self.F, self.basis, self.gstruct, self.mstruct, H.ctypes.data)
        return H

    def diagonalise(self, H, lo, hi):
        """diagonalise_hamiltonian with the 1-based window [lo + 1, hi + 1]; H is host memory."""
        self._install()
        H = np.asfortranarray(H, dtype=np.complex128)
        M = hi - lo + 1
        idx = (C.c_int * 2)(lo + 1, hi + 1)
        w = np.zeros(self.n_h)
        v = np.zeros((self.n_h, M), dtype=np.complex128, order="F")
        L.lib.diagonalise_hamiltonian(idx, H.ctypes.data, w.ctypes.data, v.ctypes.data)
        return w[:M].copy(), v

    def eigenstates(self, n_vb, n_cb):
        """eigenstates(): the caller allocates every state's .fourier (N_H values),
        as 8_band_main.c:737-751.  Returns (E, vectors) with the 2 n_vb VB states
        first (ascending), then the 2 n_cb CB states, and the raw structs."""
        self._install()
        nstates = (C.c_int * 2)(n_vb, n_cb)
        vb = (L.Eigenstate * (2 * n_vb))()
        cb = (L.Eigenstate * (2 * n_cb))()
        M = 2 * n_vb + 2 * n_cb
        v = np.zeros((self.n_h, M), dtype=np.complex128, order="F")
        for i in range(2 * n_vb):
            vb[i].fourier = v[:, i].ctypes.data
        for i in range(2 * n_cb):
            cb[i].fourier = v[:, 2 * n_vb + i].ctypes.data
        L.lib.eigenstates(self.n_shape, nstates, self.F, self.basis, self.gstruct, self.mstruct, vb, cb)
        E = np.array([vb[i].E for i in range(2 * n_vb)] + [cb[i].E for i in range(2 * n_cb)])
        self._states = (vb, cb, v)
        return E, v

    def hamiltonian_derivative(self, polarisation):
        """hamiltonian_derivative_8_band into a zeroed host array (lower triangle)."""
        self._install()
        H = np.zeros((self.n_h, self.n_h), dtype=np.complex128, order="F")
        L.lib.hamiltonian_derivative_8_band(polarisation, self.n_shape, self.basis, self.gstruct, self.mstruct,
                                            H.ctypes.data)
        return H

    def momentum_matrix_elements(self, v, n_vb, n_cb):
        """The reference's loop (8_band_main.c:1632-1655) over momentum_matrix_element:
        returns p[pol, c, v] for the states v (VB first), valence states from the highest down."""
        self._install()
        C.c_int.in_dll(L.lib, "Polarisation_Indicator").value = -1
        v = np.asfortranarray(v, dtype=np.complex128)
        nv, nc = 2 * n_vb, 2 * n_cb
        states = (L.Eigenstate * (nv + nc))()
        for i in range(nv + nc):
            states[i].fourier = v[:, i].ctypes.data
        nstates = (C.c_int * 2)(n_vb, n_cb)
        out = np.zeros((3, nc, nv), dtype=np.complex128)
        for pol in range(3):
            for c in range(nc):
                for iv in range(nv):
                    j = nv - 1 - iv
                    r = L.lib.momentum_matrix_element(pol, self.n_shape, self.basis, self.gstruct, self.mstruct,
                                                      states[nv + c], nv + c, states[j], j, nstates)
                    out[pol, c, iv] = r.re + 1j * r.im
        return out

    def envelope_functions(self, v, N_states, kind, x, y, z, direction=0):
        """envelope_functions() for the 2 N_states[kind] states v (kind 0 valence,
        1 conduction): the caller allocates F_1..F_8 and probability_1..8 of
        every state (8_band_main.c:824-893); returns (F, prob) as (states, 8, points)."""
        v = np.asfortranarray(v, dtype=np.complex128)
        m, n = v.shape[1], len(x)
        F = np.zeros((m, 8, n), dtype=np.complex128)
        P = np.zeros((m, 8, n))
        st = (L.Eigenstate * m)()
        for s in range(m):
            st[s].fourier = v[:, s].ctypes.data
            for b in range(8):
                setattr(st[s], "F_%d" % (b + 1), F[s, b].ctypes.data)
                setattr(st[s], "probability_%d" % (b + 1), P[s, b].ctypes.data_as(C.POINTER(C.c_double)))
        xs, ys, zs = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        ns = (C.c_int * 2)(*N_states)
        dp = C.POINTER(C.c_double)
        L.lib.envelope_functions(self.gstruct, ns, kind, n, xs.ctypes.data_as(dp), ys.ctypes.data_as(dp),
                                 zs.ctypes.data_as(dp), self.basis, st, direction)
        return F, P

    def coulomb(self, NC, v, n_vb, n_cb, coulomb_region_type=0):
        """coulomb_matrix_elements for the states v (N_H x (2 n_vb + 2 n_cb), VB
        first) on a Coulomb cell with NC plane waves per axis and lengths
        geo[0]['CL1..3']; arrays sized as 8_band_main.c:1752-1775."""
        self._install()
        nv, nc = 2 * n_vb, 2 * n_cb
        v = np.asfortranarray(v, dtype=np.complex128)
        vb = (L.Eigenstate * nv)()
        cb = (L.Eigenstate * nc)()
        for i in range(nv):
            vb[i].fourier = v[:, i].ctypes.data
        for i in range(nc):
            cb[i].fourier = v[:, nv + i].ctypes.data
        NCT = tuple(2 * n - 1 for n in NC)
        cgrids = [np.ascontiguousarray(basis_grid(nt, self.geo[0]["CL" + str(a + 1)])) for a, nt in enumerate(NCT)]
        cbasis = L.WaveVectors(*NC, *NCT, *[g.ctypes.data_as(C.POINTER(C.c_double)) for g in cgrids], 0.0, 0.0, 0.0)
        out = {"hh": np.zeros(nv ** 4, np.complex128), "ee": np.zeros(nc ** 4, np.complex128),
               "eh_direct": np.zeros(nv * nv * nc * nc, np.complex128),
               "eh_exchange": np.zeros(nv * nv * nc * nc, np.complex128)}
        cme = _CME(out["ee"].ctypes.data, out["hh"].ctypes.data, out["eh_direct"].ctypes.data,
                   out["eh_exchange"].ctypes.data)
        nstates = (C.c_int * 2)(n_vb, n_cb)
        L.lib.coulomb_matrix_elements(self.basis, cbasis, self.gstruct, self.mstruct, nstates, vb, cb, cme,
                                      coulomb_region_type)
        return out


def signatures():
    """ctypes signature of coulomb_matrix_elements (the other three are set in lib.py)."""
    L.lib.coulomb_matrix_elements.restype = None
    L.lib.coulomb_matrix_elements.argtypes = [L.WaveVectors, L.WaveVectors, C.POINTER(L.SupercellGeometry),
                                              C.POINTER(L.MaterialParams), C.POINTER(C.c_int),
                                              C.POINTER(L.Eigenstate), C.POINTER(L.Eigenstate), _CME, C.c_int]


signatures()

/*
 * qudos_b200 -- B200 (sm_100a) implementation of the QUDOS plane-wave (PWEM)
 * solve path: 8-band k.p supercell Hamiltonian assembly, partial dense
 * Hermitian eigensolve for the states nearest the gap, and the FFT-based
 * Coulomb matrix elements.
 *
 * Two layers are exported from libqdgpu.so:
 *
 *  1. The reference's own routines, same names, same arguments, same global
 *     state (QUDOS code/source/8_band/8_band.h).  They run on the GPU.  The
 *     reference's globals are defined here as weak symbols so that the
 *     reference's 8_band_main.c, linked against this library, provides them.
 *
 *  2. Status-returning entry points with plain pointers and sizes (prefix
 *     qd_), used by the driver program, the Python binding and the tests.
 *     They never exit the process; they return QD_OK or a QD_ERR_* code and
 *     qd_last_error_message() describes the failure.
 *
 * Only one GPU is used (the current CUDA device).  Calls are not re-entrant
 * (the reference keeps global state); one call at a time per process.
 */
#ifndef QUDOS_B200_H
#define QUDOS_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
typedef struct { double re, im; } qd_complex128;
typedef struct { float re, im; } qd_complex64;
#else
#include <complex.h>
typedef double _Complex qd_complex128;
typedef float _Complex qd_complex64;
#endif

/* ------------------------------------------------------------------------- */
/* Reference ABI types (layout identical to code/source/8_band/8_band.h)      */
/* ------------------------------------------------------------------------- */
#ifndef QD_NO_REFERENCE_TYPES
/* 8_band.h:117-124 */
struct wave_vectors {
    int N_Gx, N_Gy, N_Gz;
    int N_Gx_T, N_Gy_T, N_Gz_T;
    double *Gx, *Gy, *Gz;
    double Kx, Ky, Kz;
};
/* 8_band.h:126 */
struct characteristic_functions { qd_complex128 *chi; };
/* 8_band.h:130 */
struct vector { double x, y, z; };
/* 8_band.h:134-138 */
struct strain_tensor { qd_complex128 *xx, *yy, *zz, *yz, *xz, *xy; };
/* 8_band.h:140-144 (only the first eight tables are read by the solve path) */
struct convolution_char_strain {
    qd_complex128 *char_xx, *char_yy, *char_zz, *char_yz, *char_xz, *char_xy, *char_hydrostatic,
        *char_biaxial, *xx_yz, *yy_yz, *zz_yz, *xy_xz, *yy_xz, *xx_xz, *zz_xz, *xy_yz, *zz_xy,
        *xx_xy, *yy_xy, *xz_yz, *char_xx_yz, *char_yy_yz, *char_zz_yz, *char_xy_xz, *char_yy_xz,
        *char_xx_xz, *char_zz_xz, *char_xy_yz, *char_zz_xy, *char_xx_xy, *char_yy_xy, *char_xz_yz;
};
/* 8_band.h:146-150 */
struct piezo_potential { qd_complex128 *pz; };
/* 8_band.h:170-174 */
struct coulomb_matrix_element { qd_complex128 *ee, *hh, *eh_direct, *eh_exchange; };
/* 8_band.h:190-194 */
struct timing {
    double char_s_grid, char_es_grid, strain_s_grid, piezo_s_grid, strain_es_grid, piezo_es_grid,
        conv, ham_elements, ham_diag, eig, bloch, overlaps, car_loc, mme, linescan, cross_section,
        real_3D, cme_B, cme_I, cme_total, total;
};
/* 8_band.h:197 */
struct supercell_geometry {
    int shape, embedded, material, material_type, RL1, RL2, RL3, RCL1, RCL2, RCL3;
    double x, y, Ox, Oy, Oz, L1, L2, L3, L4, L5, SL1, SL2, SL3, CL1, CL2, CL3, alpha, beta, gamma;
};
/* 8_band.h:200 */
struct material_params {
    double a, C11, C12, C44, e14, B114, B124, B156, Eg, Dso, Ep, P, sc, g1, g2, g3, ac, av, b, d,
        Ev_avg, E_so, E_lh, E_hh, E_cb, nr;
};
/* 8_band.h:209-211 */
struct eigenstate {
    int idx_state;
    double E, *bloch, *probability_1, *probability_2, *probability_3, *probability_4,
        *probability_5, *probability_6, *probability_7, *probability_8;
    qd_complex128 *fourier, *F_1, *F_2, *F_3, *F_4, *F_5, *F_6, *F_7, *F_8;
};

/* ------------------------------------------------------------------------- */
/* Reference global state read by the solve path (8_band.h:77-110,218-225).   */
/* Weak definitions live in the library.                                      */
/* ------------------------------------------------------------------------- */
extern int N_shape, isotropic, softening, include_strain, include_piezo, include_CME, PACKED;
extern double sigma_softening; /* 8_band.h:90; read by coulomb_matrix_elements for commensurate cells */
extern int myid, nprocs;
extern int64_t N_H, na_rows, na_cols, na_rowsz, na_colsz, np_rows, np_cols, my_prow, my_pcol,
    block_size;
extern struct characteristic_functions *characteristic_function_G;
extern struct strain_tensor strain_G;
extern struct convolution_char_strain *convolutions_char_strain;
extern struct piezo_potential phi_piezo_G;
extern struct timing component_run_times;

/* --- Reference routines, GPU implementations ------------------------------ */
/* Replaces code/source/8_band/hamiltonian_8_band.c:23.  Writes the lower
 * triangle of the column-major N_H x N_H Hamiltonian into the caller's H
 * (host memory, leading dimension na_rows = N_H); the strict upper triangle
 * is not written.  Reads characteristic_function_G, strain_G,
 * convolutions_char_strain, phi_piezo_G, include_strain, include_piezo. */
void hamiltonian_8_band(int N_shape, struct vector F, struct wave_vectors basis,
                        struct supercell_geometry *supercell, struct material_params *parameters,
                        qd_complex128 *H);

/* Replaces code/source/8_band/diagonalise_hamiltonian.c:24 (zheevr with
 * RANGE='I', UPLO='L').  idx_eig holds the 1-based window [il, iu]; eigval
 * receives the iu-il+1 eigenvalues in ascending order, eigvec the
 * eigenvectors (N_H x (iu-il+1), column-major).  H (lower triangle) is read. */
void diagonalise_hamiltonian(int *idx_eig, qd_complex128 *H, double *eigval, qd_complex128 *eigvec);

/* Replaces code/source/8_band/eigenstates.c:23.  Assembles H on the GPU from
 * the global coefficient tables, solves the index window
 * [6 N_PW - 2 N_vb, 6 N_PW + 2 N_cb - 1] and fills eigenstate_vb[0..2N_vb-1]
 * and eigenstate_cb[0..2N_cb-1] (.E and .fourier, which the caller allocates
 * with na_rows elements).  H never leaves the device. */
void eigenstates(int N_shape, int *N_states, struct vector F, struct wave_vectors basis,
                 struct supercell_geometry *supercell, struct material_params *parameters,
                 struct eigenstate *eigenstate_vb, struct eigenstate *eigenstate_cb);

/* Replaces code/source/8_band/coulomb_matrix_elements.c:24.  include_CME 1-4
 * (1: the Fourier-space integrals only; 2: plus the Madelung monopole term;
 * 3: plus dipole; 4: plus quadrupole, coulomb_matrix_elements.c:250-557), a
 * free Coulomb cell (coulomb_region_type 0) equal to or larger than the
 * electronic-structure cell, or a commensurate one (coulomb_region_type 1,
 * supercell[0].CL* = RCL* L*; with `softening` set, the cell's cuboid is
 * softened by `sigma_softening` as in B_coulomb_supercell_fft.c), with
 * coulomb_basis.N_G* plane waves per axis.  The real-space Madelung sum
 * follows the reference's split over the `nprocs` global.  CME arrays are
 * allocated by the caller with the sizes of 8_band_main.c:1752-1775. */
void coulomb_matrix_elements(struct wave_vectors basis, struct wave_vectors coulomb_basis,
                             struct supercell_geometry *supercell,
                             struct material_params *parameters, int *N_states,
                             struct eigenstate *eigenstate_vb, struct eigenstate *eigenstate_cb,
                             struct coulomb_matrix_element CME, int coulomb_region_type);

/* Globals of the momentum-matrix-element stage (8_band.h): include_MME,
 * Polarisation_Indicator (the polarisation whose dH/dk is current),
 * Num_Possible_Polarisations, and the reference's host work arrays dH_dk and
 * yV, which this library leaves unwritten (it keeps both on the device). */
extern int include_MME, Polarisation_Indicator, Num_Possible_Polarisations;
extern qd_complex128 *dH_dk, *yV;

/* Replaces code/source/8_band/hamiltonian_derivative_8_band.c:23.  dH/dk
 * along [100], [010] or [001] (polarisation 0, 1, 2) into the caller's host
 * H_dk, lower triangle, leading dimension na_rows = N_H, from the same global
 * coefficient tables as hamiltonian_8_band. */
void hamiltonian_derivative_8_band(int polarisation, int N_shape, struct wave_vectors basis,
                                   struct supercell_geometry *supercell, struct material_params *parameters,
                                   qd_complex128 *H_dk);

/* Replaces code/source/8_band/momentum_matrix_element.c:24: returns
 * <psi_2| dH/dk_polarisation |psi_1> (eV Angstrom).  dH/dk is rebuilt on the
 * device when Polarisation_Indicator differs from polarisation; dH/dk psi_1
 * is recomputed when eigenstate_2_idx == 2 N_states[0] - 1 (the first valence
 * state of the reference's loop, 8_band_main.c:1635-1655) and reused for the
 * other valence states. */
qd_complex128 momentum_matrix_element(int polarisation, int N_shape, struct wave_vectors basis,
                                      struct supercell_geometry *supercell, struct material_params *parameters,
                                      struct eigenstate eigenstate_1, int64_t eigenstate_1_idx,
                                      struct eigenstate eigenstate_2, int64_t eigenstate_2_idx, int *N_states);

/* Replaces code/source/8_band/envelope_functions.c:23.  For the 2 N_states[type]
 * states of `eigenstate` (type 0 valence, 1 conduction) fills F_1..F_8 (the
 * envelope of each Bloch band, sum_G a_G exp(i (G + K).r) / sqrt(L1 L2 L3))
 * and probability_1..probability_8 = |F_b|^2, each caller-allocated with
 * N_grid entries, at the points (x, y, z) in Angstrom; `direction` only names
 * the scan for the output writers. */
void envelope_functions(struct supercell_geometry *supercell, int *N_states, int type, int N_grid, double *x,
                        double *y, double *z, struct wave_vectors basis, struct eigenstate *eigenstate,
                        int direction);
#endif /* QD_NO_REFERENCE_TYPES */

/* ------------------------------------------------------------------------- */
/* Status-returning API                                                       */
/* ------------------------------------------------------------------------- */
enum {
    QD_OK = 0,
    QD_ERR_INPUT = 1,        /* malformed or missing input file / key          */
    QD_ERR_UNSUPPORTED = 2,  /* option outside the implemented path            */
    QD_ERR_CUDA = 3,         /* CUDA runtime / device error                     */
    QD_ERR_NOMEM = 4,        /* host or device allocation failed               */
    QD_ERR_CONVERGENCE = 5,  /* eigensolver failed to converge                 */
    QD_ERR_TIMEOUT = 6,      /* a bounded device-side wait ran out              */
    QD_ERR_ARG = 7           /* invalid argument                               */
};
enum { QD_PREC_FP64 = 0, QD_PREC_MIXED = 1 };

const char *qd_last_error_message(void);
int qd_version(void);

typedef struct qd_problem qd_problem;

/* Parse parameters.in and supercell.in in `dir`; `overrides` are CLI-style
 * "-Key=value" strings (read_command_line_input.c).  Computes the basis sets
 * and material parameters on the host. */
int qd_problem_load(const char *dir, const char *const *overrides, int n_overrides, qd_problem **out);
void qd_problem_free(qd_problem *pr);
int qd_problem_n_shape(const qd_problem *pr);
/* Applied field F (V/Angstrom) and Bloch wave vector K (1/Angstrom) of a
 * loaded problem, in the units the reference's routines take them. */
int qd_problem_field(const qd_problem *pr, double F[3], double K[3]);
/* Number of libqdgpu kernel launches since the library was loaded (library
 * GEMMs from cuBLAS not included). */
long long qd_launch_count(void);
/* Sizes: n_pw = N_Gx N_Gy N_Gz, n_h = 8 n_pw, window [lo, hi] 0-based. */
int qd_problem_sizes(const qd_problem *pr, int64_t *n_pw, int64_t *n_h, int *lo, int *hi,
                     int *n_vb, int *n_cb);
/* Copies of the host-side set-up for checking: per-shape material parameters
 * (n_shape structs) and geometry. */
int qd_problem_materials(const qd_problem *pr, struct material_params *out, int n_shape);
int qd_problem_geometry(const qd_problem *pr, struct supercell_geometry *out, int n_shape);

/* Build every coefficient table on the GPU (shape transforms, strain, piezo
 * potential, downsampling, convolutions, fused per-difference coefficients). */
int qd_problem_build_tables(qd_problem *pr);
/* Copy a table to host memory.  which: 0 chi (shape s), 1 strain component s
 * (0..5 = xx yy zz yz xz xy), 2 piezo potential, 3 convolution (shape s,
 * component c = 0..7 with 6 hydrostatic, 7 biaxial), 4 strain-cell chi,
 * 5 strain-cell strain component s, 6 strain-cell piezo potential.
 * out holds n_T elements (the grid of that cell). */
int qd_problem_get_table(const qd_problem *pr, int which, int s, int c, qd_complex128 *out, int64_t n);

/* Assemble H on the device.  mode 0: lower triangle only (the reference's
 * layout), mode 1: full Hermitian.  H_dev is column-major N_H x N_H with leading
 * dimension ld (>= N_H); complex128 (prec FP64) or complex64 (prec MIXED). */
int qd_problem_assemble_dev(qd_problem *pr, void *H_dev, int64_t ld, int mode, int prec, void *stream);

/* Eigenpairs of the problem's index window, H on the device (lower triangle,
 * complex128, destroyed).  eigval_dev (M doubles) / eigvec_dev (N_H x M
 * complex128) are device pointers.  prec QD_PREC_MIXED reduces a complex64
 * copy on the tensor cores and refines in FP64 against H. */
int qd_eigh_window_dev(int64_t n, void *H_dev, int64_t ld, int lo, int hi, int prec,
                       double *eigval_dev, void *eigvec_dev, int64_t ldz, void *stream);

/* Full solve for a loaded problem with host outputs: tables, assembly,
 * eigensolve; eigval (M) and eigvec (N_H x M) in host memory. */
int qd_problem_solve(qd_problem *pr, int prec, double *eigval, qd_complex128 *eigvec);

/* Coulomb matrix elements (coulomb_matrix_elements.c:24, free or
 * commensurate Coulomb cells as the deck's Coulomb_supercell_type says, the
 * problem's CME setting 1..4) for n_vb_states + n_cb_states
 * states (eigvec_host: N_H x M_c, VB states first, as eigenstates orders
 * them) into the reference's four arrays (sizes of 8_band_main.c:1752-1755;
 * elements outside the reference's computed set are zero).  The real-space
 * part of the Madelung sum follows the reference's split over
 * madelung_ranks MPI ranks (its value depends on the rank count). */
int qd_coulomb(qd_problem *pr, int n_vb_states, int n_cb_states, const qd_complex128 *eigvec_host,
               int madelung_ranks, qd_complex128 *hh, qd_complex128 *ee, qd_complex128 *eh_direct,
               qd_complex128 *eh_exchange);

/* dH/dk_axis (axis 0, 1, 2: [100], [010], [001]) of a loaded problem on the
 * device, complex128, lower triangle (mode 0) or full Hermitian (mode 1). */
int qd_problem_assemble_dk_dev(qd_problem *pr, int axis, void *H_dev, int64_t ld, int mode, void *stream);

/* Interband momentum matrix elements of a loaded problem (the loop of
 * 8_band_main.c:1578-1680 over momentum_matrix_element.c:24): eigvec_host
 * holds the window's states, n_vb_states valence states first (ascending)
 * then n_cb_states conduction states, N_H each.
 * mme[(pol * n_cb_states + c) * n_vb_states + v] = <vb_{n_vb_states-1-v}|
 * dH/dk_pol |cb_c> in eV Angstrom (valence states counted from the highest,
 * as the reference does).  All pairs of a polarisation come from one dH/dk
 * assembled on the device, one product with the conduction states and one
 * reduction. */
int qd_momentum_matrix_elements(qd_problem *pr, const qd_complex128 *eigvec_host, int n_vb_states, int n_cb_states,
                                qd_complex128 *mme);

/* Real-space envelopes of m host states (N_H x m) of a loaded problem at
 * n_grid points (x, y, z in Angstrom): F and prob (host, either may be NULL)
 * receive [state][band][point] values of the band envelopes and of |F|^2. */
int qd_envelope_functions(qd_problem *pr, const qd_complex128 *eigvec_host, int m, int n_grid, const double *x,
                          const double *y, const double *z, qd_complex128 *F, double *prob);

/* Device plumbing for callers without their own CUDA binding.  qd_memcpy kind:
 * 1 host->device, 2 device->host, 3 device->device.  Events time work on a
 * stream (NULL = default stream). */
int qd_dev_alloc(size_t bytes, void **out);
int qd_dev_free(void *p);
int qd_memcpy(void *dst, const void *src, size_t bytes, int kind);
int qd_memset(void *dst, int value, size_t bytes);
int qd_host_alloc_pinned(size_t bytes, void **out);
int qd_host_free_pinned(void *p);
int qd_device_synchronize(void);
int qd_device_count(int *n);
int qd_set_device(int dev);
int qd_event_create(void **ev);
int qd_event_record(void *ev, void *stream);
int qd_event_elapsed_ms(void *ev0, void *ev1, float *ms);
int qd_event_destroy(void *ev);
/* The solve path keeps its device workspace in the device's stream-ordered
 * memory pool between calls; this returns the cached memory to the driver. */
int qd_trim_pool(void);

/* Limits of the library's bounded device-side waits, for the current device
 * (a negative value restores that limit's default):
 *   barrier_polls  polls of the panel factorisation's grid barrier (default
 *                  2^26, about three seconds);
 *   sweep_polls    polls of a bulge-chasing sweep waiting on the previous one
 *                  (default 2^25);
 *   pipeline_ns    nanoseconds a tensor-core kernel's pipeline stage waits
 *                  (default 2e9).
 * A wait that runs out makes the call return QD_ERR_TIMEOUT; the kernels exit
 * cleanly and the device stays usable.  Waits that drain a kernel's own copies
 * in flight before it exits keep a fixed 2 s bound. */
int qd_set_wait_limits(long long barrier_polls, long long sweep_polls, long long pipeline_ns);

/* Stage timings of the last qd_problem_solve / qd_eigh_window_dev call (ms):
 * [0] assembly, [1] band reduction, [2] bulge chasing, [3] bisection,
 * [4] inverse iteration, [5] back-transform, [6] refinement. */
int qd_last_timings(double *ms, int n);
/* With QD_PROFILE=1 in the environment: per-step times (ms) of the last
 * dense->band reduction: [0] panel refresh, [1] panel QR, [2] T and V T,
 * [3] X = A22 V T, [4] pending-update corrections, [5] W, [6] append,
 * [7] trailing rank-2K updates.  Adds one event per step boundary. */
int qd_stage1_profile(double *ms, int n);

/* Batched solves of independent problems (no counterpart in the reference):
 * problems[k] is solved as by qd_problem_solve(problems[k], prec, eigval[k],
 * eigvec[k]) (host outputs of M_k and N_H,k x M_k values).  Up to n_threads
 * solves run at once, each from its own host thread on its own stream,
 * largest instances first, so that small latency-bound solves overlap on the
 * GPU.  Each worker's kernels size their grids to a share of the SMs (twice
 * the even split, at least 16; the environment's QD_BATCH_SMS sets it, 0 for
 * the whole GPU).  Returns the first failure. */
int eigenstates_batched(qd_problem **problems, int n, int prec, int n_threads, double *const *eigval,
                        qd_complex128 *const *eigvec);

/* Tuning table of the dense->band reduction: for solves of order <= n_h_max
 * in precision prec, aggregate `agg` columns (a multiple of 32, 32..256) of
 * Householder panels before each rank-2K trailing update.  The entry with the
 * smallest bound >= N_H applies; without one, the environment's QD_AGG or 256.
 * n_h_max <= 0 clears the table.  Set it before the solves that should use it;
 * the Python package fills it from the cache its autotuner writes
 * (qudos_b200/autotune.py).  No counterpart in the reference. */
int qd_tuning_set(int prec, int64_t n_h_max, int agg);

/* Hellmann-Feynman gradients dE_n/dp = <psi_n| dH/dp |psi_n> of the states in
 * eigvec_host (N_H x n_states, host, normalised eigenvectors of the problem's
 * H) with respect to the parameters in params:
 *   QD_GRAD_LENGTH       Length `index` (1..5) of shape `shape`   per nm
 *   QD_GRAD_BASE         Lengths 1 and 2 of shape `shape` together per nm
 *   QD_GRAD_COMPOSITION  composition x of shape `shape`           per unit x
 *   QD_GRAD_FIELD        field component `index` (0 x, 1 y, 2 z)  per kV/cm
 *   QD_GRAD_EP           relative scale of the binary-table Ep     per unit scale
 *   QD_GRAD_GAMMA1       relative scale of the binary-table gamma_1 per unit scale
 * H is linear in the per-difference coefficient tables, so dH/dp is the
 * Hamiltonian of dcoef/dp.  For the field and the Ep and gamma_1 scales that
 * table derivative is exact (the table is linear in the field and in the
 * material parameters, whose derivatives are closed forms).  A length moves
 * only its shape's transform chi: dchi/dL is a fourth-order central
 * difference of the closed-form transform, and the table, a polynomial in
 * chi, is differentiated along it exactly by builds at chi +- dir (and
 * +- 2 dir when second-order piezo or position-dependent elastic constants
 * raise its degree).  Composition moves only the shape's material
 * parameters, in which the table is a polynomial too: dmat/dx is a
 * fourth-order central difference of the host material function and the
 * table is differentiated along it the same way.
 * Steps: rel_step times the parameter's magnitude, with a floor (rel_step <= 0
 * selects 1e-4).
 * The contraction never forms dH: every band function is a bilinear form in
 * G + K and G' + K, so <psi|dH|psi> = Re sum_f sum_D dcoef_f(D) C_f(D) with
 * C_f the reciprocal-space correlations of the k-weighted envelopes, computed
 * once per state by FFT; each parameter then costs one dot product.  No
 * counterpart in the reference.
 * dEdp[k * n_states + n] receives the derivative of state n for parameter k.
 * qd_grad_method selects the contraction: 0 (default) the FFT correlations,
 * 1 the direct sum over the lower triangle of dH (an independent check). */
extern int qd_grad_method;
enum {
    QD_GRAD_LENGTH = 0,
    QD_GRAD_BASE = 1,
    QD_GRAD_COMPOSITION = 2,
    QD_GRAD_FIELD = 3,
    QD_GRAD_EP = 4,
    QD_GRAD_GAMMA1 = 5
};
typedef struct { int kind, shape, index; } qd_grad_param;
int eigen_gradients_8_band(qd_problem *pr, const qd_complex128 *eigvec_host, int n_states,
                           const qd_grad_param *params, int n_params, double rel_step, double *dEdp);

/* Tensor-core building blocks of the mixed-precision reduction (tcgen05
 * kind::tf32 with a 3xTF32 hi/lo split, FP32 accumulation), exposed for
 * tests.  All pointers are device pointers to column-major complex64 data.
 *   qd_tc_xprod: X[0:m, 0:nb] = A[off:off+m, off:off+m] * VT for a full
 *     Hermitian n x n matrix A (lda even, off even), VT m x nb, nb <= 32.
 *   qd_tc_flush: A[off:, off:] (mt x mt) -= P Q^H, P = [V W], Q = [W V]
 *     with rows voff..voff+mt-1 and the first K columns of V and W.
 * Work buffers serve matrices up to n rows and K <= kmax; qd_tc_work_check
 * reports (and clears) a timed-out wait inside the kernels. */
typedef struct QdTcWork QdTcWork;
int qd_tc_work_alloc(int64_t n, int kmax, QdTcWork **out);
void qd_tc_work_free(QdTcWork *w);
int qd_tc_work_check(QdTcWork *w);
int qd_tc_xprod(const void *A, int64_t lda, int64_t n, int64_t off, int m, const void *VT, int64_t ldvt, int nb,
                void *X, int64_t ldx, QdTcWork *w, void *stream);
int qd_tc_flush(void *A, int64_t lda, int64_t off, int mt, const void *V, const void *W, int64_t ldv, int64_t voff,
                int K, QdTcWork *w, void *stream);

/* Per-kernel device time of the tensor-core building blocks since the last
 * call (CUDA events around every launch, on the launching stream): which 0
 * is the X product (work = bytes of the trailing matrix read, 8 m^2 per
 * launch), 1 the Hermitian rank-2K trailing update (work = 8 mt (mt+1) K
 * flops per launch).  Synchronises the device and resets the counters. */
int qd_tc_kernel_stats(int which, long long *launches, double *ms, double *work);
/* Per-launch device time (ms) and algorithmic work of the same kernels since the
 * last qd_tc_kernel_stats reset (up to cap launches); returns the count. */
int qd_tc_kernel_launches(int which, int cap, double *ms, double *work);

/* Throughput (TFLOP/s) of a plain cuBLAS n^3 GEMM: kind 0 DGEMM (FP64), 1
 * SGEMM on TF32 tensor cores, 2 ZGEMM; `reps` timed launches after one
 * warm-up.  Used for the roofline denominators that are not measured
 * elsewhere. */
int qd_gemm_peak(int kind, int n, int reps, double *tflops);

/* FP64 building blocks of the solver's last stage, exposed for checking
 * (device pointers, column-major complex128):
 *   qd_hemm_lower_dev   Y = H X + beta Y, H Hermitian n x n with its lower
 *                       triangle stored (the reference's layout), X n x k;
 *   qd_gram_dev         C = A^H B (ka x kb) reduced over n rows;
 *   qd_zgemm_small_dev  Y = Z C + beta Y, C small (k x k2);
 *   qd_residual_norms_dev  res[j] = ||R[:, j] - w[j] Z[:, j]||. */
int qd_hemm_lower_dev(int64_t n, const void *H, int64_t ld, const void *X, int64_t ldx, int k, void *Y, int64_t ldy,
                      double beta, void *stream);
int qd_gram_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb, void *C, int ldc,
                void *stream);
int qd_zgemm_small_dev(int64_t n, const void *Z, int64_t ldz, int k, const void *C, int ldc, int k2, void *Y,
                       int64_t ldy, double beta, void *stream);
int qd_residual_norms_dev(int64_t n, const void *R, int64_t ldr, const void *Z, int64_t ldz, const double *w_dev,
                          int m, double *res_dev, void *stream);

/* Tall-and-skinny products of the panel steps (device pointers, column-major;
 * fp32 != 0 selects complex64, else complex128):
 *   qd_tsmm_nn  C[m x nc] = beta C + sum_t alpha[t] A[t] op(B[t]), nterms 1 or
 *               2, nc <= 64; op(B) = B (K x nc, ldb) when btrans[t] == 0, else
 *               B^H of an nc x K block;
 *   qd_tsmm_cn  C[k1 x nc] = A^H B reduced over m rows, k1 <= 256 with
 *               nc <= 32 or k1 <= 64 with nc <= 64; scratch holds
 *               scratch_bytes >= qd_tsmm_cn_scratch_bytes(m, k1, nc, 8 or 16)
 *               of partial sums (QD_ERR_ARG when too small), which are
 *               added in FP64 in a fixed order;
 *   qd_small_cn C[n1 x n2] = alpha A^H B for k x n1, k x n2 inputs, k, n1, n2 <= 32. */
int qd_tsmm_nn(int fp32, int m, int nc, int nterms, const void *const *A, const int64_t *lda, const void *const *B,
               const int64_t *ldb, const int *K, const int *btrans, const double *alpha, void *C, int64_t ldc,
               double beta, void *stream);
int qd_tsmm_cn(int fp32, int m, const void *A, int64_t lda, int k1, const void *B, int64_t ldb, int nc, void *C,
               int64_t ldc, void *scratch, size_t scratch_bytes, void *stream);
int qd_small_cn(int fp32, int k, int n1, int n2, const void *A, int lda, const void *B, int ldb, double alpha,
                void *C, int ldc, void *stream);
size_t qd_tsmm_cn_scratch_bytes(int m, int k1, int nc, int elem_bytes);

/* Residual check of host eigenpairs (m values, N_H x m vectors) of a loaded
 * problem against its H, assembled on the device in FP64:
 * res[j] = ||H z_j - w_j z_j|| (eV), *orth = max |(Z^H Z - I)_ij|,
 * *hnorm = max |H_ij|. */
int qd_problem_residuals(qd_problem *pr, int m, const double *eigval, const void *eigvec, double *res, double *orth,
                         double *hnorm);

/* Error bounds of the last mixed-precision solve on the calling thread, per
 * window state: residual[i] = ||H x_i - theta_i x_i|| in FP64 and
 * bound[i] = ||r||^2 / delta (Kato-Temple), delta the distance from theta_i to
 * the nearest Ritz value outside its degenerate group.  The mixed solve
 * returns QD_ERR_CONVERGENCE when a bound exceeds QD_BOUND_TOL (eV, default
 * 1e-6).  Returns the number of states (either pointer may be NULL). */
int qd_last_error_bounds(double *residual, double *bound, int n);

/* Allocation-free eigenvalues of a Hermitian tridiagonal matrix for the index
 * window [lo, hi] (0-based, ascending), by the same Sturm-count multisection
 * as the solver's bisection stage.  No reference counterpart: it is for
 * callers that cannot call cudaMalloc, such as a host program whose device
 * memory belongs to another allocator (a framework's caching pool, a fixed
 * per-process budget) and which hands this library only its own buffers.
 *   AB: device, band storage with ldb >= 2; AB[j*ldb] is the diagonal entry
 *       (real part used), AB[1 + j*ldb] the sub-diagonal entry (j, j+1).
 *   w:  device, hi - lo + 1 doubles.
 * Scratch is a file-scope device array for n <= QD_STATIC_TRI_MAX rows
 * (1 MB, held by every GPU that loads the library until exit); larger n
 * returns QD_ERR_ARG.  Every call on a device shares that scratch, so calls
 * that overlap on the GPU (several streams or host threads) race and must be
 * serialised by the caller.  The first call on each device resolves the
 * scratch address (cudaGetSymbolAddress, with that device current); make that
 * first call before any stream capture. */
#define QD_STATIC_TRI_MAX 65536
int qd_tridiag_eigvals_noalloc(const void *AB, int ldb, int n, int lo, int hi, double *w, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* QUDOS_B200_H */

/* C entry points of libqdgpu: error state, problem set-up from the reference's
 * input files, the status-returning qd_* API and the reference-named routines
 * (hamiltonian_8_band, diagonalise_hamiltonian, eigenstates,
 * coulomb_matrix_elements) with the reference's global state. */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <dlfcn.h>

#include <cublas_v2.h>
#include <cuda_runtime_api.h>

#include "qd_internal.h"

/* ------------------------------------------------------------------------- */
/* Reference global state (8_band_main.c:36-65).  Weak, so that the           */
/* reference's own definitions win when its main program links this library. */
/* ------------------------------------------------------------------------- */
#define QD_WEAK __attribute__((weak))
QD_WEAK int N_shape = 0;
QD_WEAK int isotropic = 0;
QD_WEAK int softening = 0;
QD_WEAK double sigma_softening = 0.0;
QD_WEAK int include_strain = 0;
QD_WEAK int include_piezo = 0;
QD_WEAK int include_CME = 0;
QD_WEAK int PACKED = 0;
QD_WEAK int myid = 0;
QD_WEAK int nprocs = 1;
QD_WEAK int64_t N_H = 0, na_rows = 0, na_cols = 0, na_rowsz = 0, na_colsz = 0, np_rows = 1, np_cols = 1, my_prow = 0,
                my_pcol = 0, block_size = 0;
QD_WEAK struct characteristic_functions *characteristic_function_G = NULL;
QD_WEAK struct strain_tensor strain_G = {0};
QD_WEAK struct convolution_char_strain *convolutions_char_strain = NULL;
QD_WEAK struct piezo_potential phi_piezo_G = {0};
QD_WEAK struct timing component_run_times = {0};
QD_WEAK int include_MME = 0;
QD_WEAK int Polarisation_Indicator = -1;
QD_WEAK int Num_Possible_Polarisations = 3;
QD_WEAK qd_complex128 *dH_dk = NULL;
QD_WEAK qd_complex128 *yV = NULL;

/* ------------------------------------------------------------------------- */
/* errors                                                                    */
/* ------------------------------------------------------------------------- */
static __thread char g_err[512];
static __thread int g_err_code;

int qd_set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    g_err_code = code;
    return code;
}

const char *qd_last_error_message(void) { return g_err; }
int qd_version(void) { return 1; }

/* Number of this library's own kernel launches since load (cuBLAS calls not
 * included); read by callers that report how much of a step ran in our kernels. */
static long long g_launches = 0;
void qd_count_launch(int n) { __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED); }
long long qd_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int qd_stage1_set_wait_limit(long long polls);
int qd_stage2_set_wait_limit(long long polls);
int qd_tc_set_wait_limit(long long ns);

int qd_set_wait_limits(long long barrier_polls, long long sweep_polls, long long pipeline_ns) {
    int rc = qd_stage1_set_wait_limit(barrier_polls);
    if (rc == QD_OK) rc = qd_stage2_set_wait_limit(sweep_polls);
    if (rc == QD_OK) rc = qd_tc_set_wait_limit(pipeline_ns);
    return rc;
}

/* Stream-ordered pool allocations of the solve path.  The first use on a
 * device raises the release threshold of its default pool so that freed
 * workspace stays mapped for the next solve; qd_trim_pool() hands it back. */
static int g_pool_ready[64];
int qd_pool_alloc(void **p, size_t bytes, void *stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev >= 0 && dev < 64 && !g_pool_ready[dev]) {
        cudaMemPool_t pool;
        e = cudaDeviceGetDefaultMemPool(&pool, dev);
        if (e != cudaSuccess) return (int)e;
        unsigned long long keep = ~0ull;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return (int)e;
        g_pool_ready[dev] = 1;
    }
    return (int)cudaMallocAsync(p, bytes ? bytes : 16, (cudaStream_t)stream);
}
void qd_pool_free(void *p, void *stream) {
    if (p) cudaFreeAsync(p, (cudaStream_t)stream);
}
int qd_trim_pool(void) {
    int dev = 0;
    cudaMemPool_t pool;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetDefaultMemPool(&pool, dev);
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(pool, 0);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "qd_trim_pool: %s", cudaGetErrorString(e));
    return QD_OK;
}

/* Device-memory, copy and event helpers so that callers without a CUDA
 * toolkit binding (ctypes, Fortran, ...) can drive the device-resident entry
 * points. */
int qd_dev_alloc(size_t bytes, void **out) {
    cudaError_t e = cudaMalloc(out, bytes ? bytes : 16);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    return QD_OK;
}
int qd_dev_free(void *p) {
    if (p) cudaFree(p);
    return QD_OK;
}
int qd_memcpy(void *dst, const void *src, size_t bytes, int kind) {
    /* kind: 1 host->device, 2 device->host, 3 device->device */
    enum cudaMemcpyKind k = kind == 1 ? cudaMemcpyHostToDevice : kind == 2 ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaMemcpy(dst, src, bytes, k);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_memset(void *dst, int value, size_t bytes) {
    cudaError_t e = cudaMemset(dst, value, bytes);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_host_alloc_pinned(size_t bytes, void **out) {
    cudaError_t e = cudaMallocHost(out, bytes ? bytes : 16);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_NOMEM, "cudaMallocHost(%zu): %s", bytes, cudaGetErrorString(e));
    return QD_OK;
}
int qd_host_free_pinned(void *p) {
    if (p) cudaFreeHost(p);
    return QD_OK;
}
int qd_device_synchronize(void) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "device: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_device_count(int *n) {
    cudaError_t e = cudaGetDeviceCount(n);
    if (e != cudaSuccess) {
        *n = 0;
        return qd_set_error(QD_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    return QD_OK;
}
int qd_set_device(int dev) {
    cudaError_t e = cudaSetDevice(dev);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_event_create(void **ev) {
    cudaError_t e = cudaEventCreate((cudaEvent_t *)ev);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaEventCreate: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_event_record(void *ev, void *stream) {
    cudaError_t e = cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaEventRecord: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_event_elapsed_ms(void *ev0, void *ev1, float *ms) {
    cudaError_t e = cudaEventSynchronize((cudaEvent_t)ev1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, (cudaEvent_t)ev0, (cudaEvent_t)ev1);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "cudaEventElapsedTime: %s", cudaGetErrorString(e));
    return QD_OK;
}
int qd_event_destroy(void *ev) {
    if (ev) cudaEventDestroy((cudaEvent_t)ev);
    return QD_OK;
}

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess)                                                                  \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)
#define RC(x)                         \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != QD_OK) return rc_; \
    } while (0)

/* one handle per host thread: concurrent solves on several threads each drive
 * their own per-thread default stream */
static __thread cublasHandle_t g_cublas = NULL;
cublasHandle_t qd_cublas(void) {
    if (!g_cublas) {
        cublasCreate(&g_cublas);
        /* FP32 emulation on the tensor cores needs cuBLAS >= 12.9; looked up at run
         * time so that an older cuBLAS already loaded in the process still works
         * (the complex64 products then run in plain FP32). */
        typedef cublasStatus_t (*set_strategy_fn)(cublasHandle_t, int);
        set_strategy_fn f = (set_strategy_fn)dlsym(RTLD_DEFAULT, "cublasSetEmulationStrategy");
        if (f) f(g_cublas, 2 /* CUBLAS_EMULATION_STRATEGY_EAGER */);
        cublasSetStream(g_cublas, cudaStreamPerThread);
    }
    return g_cublas;
}

/* complex64 GEMM arithmetic of the mixed path: 3 = the library's tcgen05
 * 3xTF32 kernels (default); 2, 1, 0 = cuBLAS CGEMM with FP32 emulated by BF16x9,
 * with TF32, or in plain FP32 (for comparison).  QD_MIXED_GEMM overrides. */
int qd_mixed_gemm_mode(void) {
    const char *s = getenv("QD_MIXED_GEMM");
    return s ? atoi(s) : 3;
}

void qd_set_timing(int i, double ms);

/* ------------------------------------------------------------------------- */
/* problem set-up                                                            */
/* ------------------------------------------------------------------------- */
static char *read_file(const char *dir, const char *name) {
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s", dir, name);
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)n + 1);
    if (buf && fread(buf, 1, (size_t)n, f) != (size_t)n) {
        free(buf);
        buf = NULL;
    }
    if (buf) buf[n] = 0;
    fclose(f);
    return buf;
}

static int setup_problem(struct qd_problem *pr) {
    qd_params *p = &pr->p;
    if (p->n_shape < 1) return qd_set_error(QD_ERR_INPUT, "N_shape must be >= 1");
    for (int a = 0; a < 3; a++)
        if (p->N[a] < 1) return qd_set_error(QD_ERR_INPUT, "number of plane waves must be >= 1");
    struct supercell_geometry *g0 = &pr->geo[0];
    double L[3] = {g0->L1, g0->L2, g0->L3}, SL[3] = {g0->SL1, g0->SL2, g0->SL3};
    /* 8_band_main.c:195-200 */
    if (p->strain_type == 1 && g0->RL1 == 1 && g0->RL2 == 1 && g0->RL3 == 1 && p->N[0] == p->NS[0] &&
        p->N[1] == p->NS[1] && p->N[2] == p->NS[2])
        p->strain_type = 0;
    RC(qd_material_parameters(p->T, p->piezo, p->n_shape, pr->geo, pr->mat));
    pr->nT = 1;
    pr->nTS = 1;
    pr->n_pw = 1;
    for (int a = 0; a < 3; a++) {
        pr->NT[a] = 2 * p->N[a] - 1;
        pr->nT *= pr->NT[a];
        pr->n_pw *= p->N[a];
        pr->G[a] = (double *)malloc(sizeof(double) * pr->NT[a]);
        qd_basis_grid(pr->NT[a], L[a], pr->G[a]);
        if (p->strain) {
            pr->NTS[a] = 2 * p->NS[a] - 1;
            pr->nTS *= pr->NTS[a];
            pr->GS[a] = (double *)malloc(sizeof(double) * pr->NTS[a]);
            qd_basis_grid(pr->NTS[a], SL[a], pr->GS[a]);
        }
    }
    pr->n_h = 8 * pr->n_pw;
    pr->same_cells = p->strain && p->N[0] == p->NS[0] && p->N[1] == p->NS[1] && p->N[2] == p->NS[2] && L[0] == SL[0] &&
                     L[1] == SL[1] && L[2] == SL[2];
    /* eigenstates.c:29-36 (0-based) */
    int idx_cb_min = (QD_N_BAND - 2) * (int)pr->n_pw;
    pr->lo = idx_cb_min - 2 * p->n_vb;
    pr->hi = idx_cb_min + 2 * p->n_cb - 1;
    if (pr->lo < 0 || pr->hi >= pr->n_h || pr->lo > pr->hi)
        return qd_set_error(QD_ERR_INPUT, "eigenstate window outside the spectrum");
    return QD_OK;
}

int qd_problem_load(const char *dir, const char *const *overrides, int n_overrides, qd_problem **out) {
    *out = NULL;
    char *ptext = read_file(dir, "parameters.in");
    if (!ptext) return qd_set_error(QD_ERR_INPUT, "Error. Failed to open parameters.in file.");
    struct qd_problem *pr = (struct qd_problem *)calloc(1, sizeof(struct qd_problem));
    int rc = qd_read_parameters_text(ptext, &pr->p, NULL);
    free(ptext);
    for (int i = 0; rc == QD_OK && i < n_overrides; i++) rc = qd_apply_override(&pr->p, overrides[i]);
    if (rc) {
        free(pr);
        return rc;
    }
    char *stext = read_file(dir, "supercell.in");
    if (!stext) {
        free(pr);
        return qd_set_error(QD_ERR_INPUT, "Error. Failed to open supercell.in file.");
    }
    pr->geo = (struct supercell_geometry *)calloc((size_t)pr->p.n_shape, sizeof(struct supercell_geometry));
    pr->mat = (struct material_params *)calloc((size_t)pr->p.n_shape, sizeof(struct material_params));
    rc = qd_read_supercell_text(stext, &pr->p, pr->geo);
    free(stext);
    if (rc == QD_OK) rc = setup_problem(pr);
    if (rc) {
        qd_problem_free(pr);
        return rc;
    }
    *out = pr;
    return QD_OK;
}

void qd_problem_free(qd_problem *pr) {
    if (!pr) return;
    for (int a = 0; a < 3; a++) {
        free(pr->G[a]);
        free(pr->GS[a]);
        if (pr->d_G[a]) qd_pool_free(pr->d_G[a], NULL);
        if (pr->d_GS[a]) qd_pool_free(pr->d_GS[a], NULL);
    }
    void *dev[] = {pr->d_geo, pr->d_mat, pr->d_chi_s, pr->d_eps_s, pr->d_phi_s, pr->d_chi,
                   pr->d_eps, pr->d_phi, pr->d_conv, pr->d_coef};
    for (size_t i = 0; i < sizeof(dev) / sizeof(dev[0]); i++)
        if (dev[i]) qd_pool_free(dev[i], NULL);
    free(pr->geo);
    free(pr->mat);
    free(pr);
}

int qd_problem_field(const qd_problem *pr, double F[3], double K[3]) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    for (int a = 0; a < 3; a++) {
        if (F) F[a] = pr->p.F[a];
        if (K) K[a] = pr->p.K[a];
    }
    return QD_OK;
}

int qd_problem_n_shape(const qd_problem *pr) { return pr ? pr->p.n_shape : 0; }

int qd_problem_sizes(const qd_problem *pr, int64_t *n_pw, int64_t *n_h, int *lo, int *hi, int *n_vb, int *n_cb) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    if (n_pw) *n_pw = pr->n_pw;
    if (n_h) *n_h = pr->n_h;
    if (lo) *lo = pr->lo;
    if (hi) *hi = pr->hi;
    if (n_vb) *n_vb = pr->p.n_vb;
    if (n_cb) *n_cb = pr->p.n_cb;
    return QD_OK;
}

int qd_problem_materials(const qd_problem *pr, struct material_params *out, int n) {
    if (!pr || n != pr->p.n_shape) return qd_set_error(QD_ERR_ARG, "n_shape mismatch");
    memcpy(out, pr->mat, sizeof(*out) * (size_t)n);
    return QD_OK;
}

int qd_problem_geometry(const qd_problem *pr, struct supercell_geometry *out, int n) {
    if (!pr || n != pr->p.n_shape) return qd_set_error(QD_ERR_ARG, "n_shape mismatch");
    memcpy(out, pr->geo, sizeof(*out) * (size_t)n);
    return QD_OK;
}

int qd_problem_build_tables(qd_problem *pr) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    if (pr->tables_ready) return QD_OK;
    return qd_tables_build_dev(pr);
}

int qd_problem_get_table(const qd_problem *pr, int which, int s, int c, qd_complex128 *out, int64_t n) {
    if (!pr || !pr->tables_ready) return qd_set_error(QD_ERR_ARG, "tables not built");
    const void *src = NULL;
    int64_t nt = (which >= 4) ? pr->nTS : pr->nT;
    if (n != nt) return qd_set_error(QD_ERR_ARG, "table size %lld != %lld", (long long)n, (long long)nt);
    int ns = pr->p.n_shape;
    switch (which) {
        case 0: if (s < 1 || s >= ns) break; src = (const qd_complex128 *)pr->d_chi + (int64_t)s * nt; break;
        case 1: if (!pr->d_eps || s < 0 || s > 5) break; src = (const qd_complex128 *)pr->d_eps + (int64_t)s * nt; break;
        case 2: src = pr->d_phi; break;
        case 3: if (!pr->d_conv || s < 1 || s >= ns || c < 0 || c > 7) break;
            src = (const qd_complex128 *)pr->d_conv + ((int64_t)s * 8 + c) * nt; break;
        case 4: if (!pr->d_chi_s || s < 1 || s >= ns) break; src = (const qd_complex128 *)pr->d_chi_s + (int64_t)s * nt; break;
        case 5: if (!pr->d_eps_s || s < 0 || s > 5) break; src = (const qd_complex128 *)pr->d_eps_s + (int64_t)s * nt; break;
        case 6: src = pr->d_phi_s; break;
        case 7: if (c < 0 || c >= QD_N_COEF) break; src = (const qd_complex128 *)pr->d_coef + (int64_t)c * nt; break;
        default: break;
    }
    if (!src) return qd_set_error(QD_ERR_ARG, "table (%d, %d, %d) not available", which, s, c);
    CK(cudaMemcpy(out, src, sizeof(qd_complex128) * (size_t)nt, cudaMemcpyDeviceToHost));
    return QD_OK;
}

int qd_problem_assemble_dev(qd_problem *pr, void *H_dev, int64_t ld, int mode, int prec, void *stream) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    RC(qd_problem_build_tables(pr));
    return qd_assemble_launch(pr->d_coef, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->p.N, pr->p.K, H_dev, ld, mode, prec,
                              stream);
}

int qd_eigh_window_dev(int64_t n, void *H_dev, int64_t ld, int lo, int hi, int prec, double *eigval_dev,
                       void *eigvec_dev, int64_t ldz, void *stream) {
    return qd_eigh_window(n, H_dev, ld, lo, hi, prec, eigval_dev, eigvec_dev, ldz, stream);
}

int qd_problem_solve(qd_problem *pr, int prec, double *eigval, qd_complex128 *eigvec) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    RC(qd_problem_build_tables(pr));
    int64_t n = pr->n_h;
    int M = pr->hi - pr->lo + 1;
    void *H = NULL, *Z = NULL;
    double *w = NULL;
    CK((cudaError_t)qd_pool_alloc((void **)&H, sizeof(qd_complex128) * (size_t)n * (size_t)n, NULL));
    CK((cudaError_t)qd_pool_alloc((void **)&Z, sizeof(qd_complex128) * (size_t)n * (size_t)M, NULL));
    CK((cudaError_t)qd_pool_alloc((void **)&w, sizeof(double) * (size_t)M, NULL));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    int rc = qd_problem_assemble_dev(pr, H, n, 0, QD_PREC_FP64, NULL);
    cudaEventRecord(e1, 0);
    if (rc == QD_OK) rc = qd_eigh_window(n, H, n, pr->lo, pr->hi, prec, w, Z, n, NULL);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    qd_set_timing(0, ms);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == QD_OK) {
        cudaError_t e = cudaMemcpy(eigval, w, sizeof(double) * (size_t)M, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(eigvec, Z, sizeof(qd_complex128) * (size_t)n * (size_t)M, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = qd_set_error(QD_ERR_CUDA, "copy-out: %s", cudaGetErrorString(e));
    }
    qd_pool_free(H, NULL);
    qd_pool_free(Z, NULL);
    qd_pool_free(w, NULL);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Reference-named routines                                                  */
/* ------------------------------------------------------------------------- */
static double wall_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static int env_precision(void) {
    const char *s = getenv("QD_PRECISION");
    return (s && (!strcmp(s, "mixed") || !strcmp(s, "1"))) ? QD_PREC_MIXED : QD_PREC_FP64;
}

static void die(const char *where, int rc) {
    /* The reference prints a message and aborts (diagonalise_hamiltonian.c:279-293). */
    printf("%s failed (%d): %s\n", where, rc, qd_last_error_message());
    fflush(stdout);
    exit(1);
}

static int check_single_rank(void) {
    if (nprocs != 1 || PACKED)
        return qd_set_error(QD_ERR_UNSUPPORTED, "the GPU solve path runs as a single process with PACKED = 0");
    return QD_OK;
}

/* Uploads the reference's global tables, fuses them and assembles H on the device. */
static int assemble_from_globals(int n_shape, struct vector F, struct wave_vectors basis,
                                 struct supercell_geometry *supercell, struct material_params *parameters, void *H_dev,
                                 int64_t ld, int dk_axis) {
    int N[3] = {basis.N_Gx, basis.N_Gy, basis.N_Gz};
    const qd_complex128 *chi[1024];
    const qd_complex128 *eps[6];
    const qd_complex128 **conv8 = NULL;
    if (n_shape > 1024) return qd_set_error(QD_ERR_UNSUPPORTED, "more than 1024 shapes");
    chi[0] = NULL;
    for (int s = 1; s < n_shape; s++) chi[s] = characteristic_function_G[s].chi;
    int strain_on = include_strain != 0;
    int piezo_on = strain_on && include_piezo != 0;
    if (strain_on) {
        eps[0] = strain_G.xx; eps[1] = strain_G.yy; eps[2] = strain_G.zz;
        eps[3] = strain_G.yz; eps[4] = strain_G.xz; eps[5] = strain_G.xy;
        conv8 = (const qd_complex128 **)calloc((size_t)n_shape * 8, sizeof(*conv8));
        for (int s = 1; s < n_shape; s++) {
            const struct convolution_char_strain *c = &convolutions_char_strain[s];
            conv8[s * 8 + 0] = c->char_xx; conv8[s * 8 + 1] = c->char_yy; conv8[s * 8 + 2] = c->char_zz;
            conv8[s * 8 + 3] = c->char_yz; conv8[s * 8 + 4] = c->char_xz; conv8[s * 8 + 5] = c->char_xy;
            conv8[s * 8 + 6] = c->char_hydrostatic; conv8[s * 8 + 7] = c->char_biaxial;
        }
    }
    double Fv[3] = {F.x, F.y, F.z};
    void *d_coef = NULL;
    double *d_G = NULL;
    int rc = qd_coef_from_host_tables(n_shape, N, basis.Gx, basis.Gy, basis.Gz, basis.Kx, basis.Ky, basis.Kz, Fv,
                                      supercell, parameters, strain_on, piezo_on, chi, eps,
                                      piezo_on ? phi_piezo_G.pz : NULL, conv8, &d_coef, &d_G);
    free(conv8);
    if (rc) return rc;
    int NT[3] = {2 * N[0] - 1, 2 * N[1] - 1, 2 * N[2] - 1};
    double K[3] = {basis.Kx, basis.Ky, basis.Kz};
    rc = dk_axis < 0 ? qd_assemble_launch(d_coef, d_G, d_G + NT[0], d_G + NT[0] + NT[1], N, K, H_dev, ld, 0,
                                          QD_PREC_FP64, NULL)
                     : qd_assemble_dk_launch(d_coef, d_G, d_G + NT[0], d_G + NT[0] + NT[1], N, K, dk_axis, H_dev, ld,
                                             0, NULL);
    if (rc == QD_OK && cudaDeviceSynchronize() != cudaSuccess) rc = qd_set_error(QD_ERR_CUDA, "assembly failed");
    qd_pool_free(d_coef, NULL);
    qd_pool_free(d_G, NULL);
    return rc;
}

void hamiltonian_8_band(int n_shape, struct vector F, struct wave_vectors basis, struct supercell_geometry *supercell,
                        struct material_params *parameters, qd_complex128 *H) {
    int rc = check_single_rank();
    int64_t n = (int64_t)8 * basis.N_Gx * basis.N_Gy * basis.N_Gz;
    int64_t ld = na_rows > 0 ? na_rows : n;
    void *Hd = NULL;
    if (rc == QD_OK && qd_pool_alloc(&Hd, sizeof(qd_complex128) * (size_t)ld * (size_t)n, NULL) != 0)
        rc = qd_set_error(QD_ERR_NOMEM, "device H");
    if (rc == QD_OK) rc = assemble_from_globals(n_shape, F, basis, supercell, parameters, Hd, ld, -1);
    /* copy the lower triangle column by column; the caller's strict upper triangle is left as it was */
    for (int64_t c = 0; rc == QD_OK && c < n; c++) {
        cudaError_t e = cudaMemcpy(H + c + c * ld, (qd_complex128 *)Hd + c + c * ld, sizeof(qd_complex128) * (size_t)(n - c),
                                   cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = qd_set_error(QD_ERR_CUDA, "copy-out: %s", cudaGetErrorString(e));
    }
    if (Hd) qd_pool_free(Hd, NULL);
    if (rc) die("hamiltonian_8_band", rc);
}

void diagonalise_hamiltonian(int *idx_eig, qd_complex128 *H, double *eigval, qd_complex128 *eigvec) {
    int rc = check_single_rank();
    int64_t n = N_H;
    int64_t ld = na_rows > 0 ? na_rows : n;
    int lo = idx_eig[0] - 1, hi = idx_eig[1] - 1, M = hi - lo + 1;
    void *Hd = NULL, *Zd = NULL;
    double *wd = NULL;
    if (rc == QD_OK && (qd_pool_alloc(&Hd, sizeof(qd_complex128) * (size_t)ld * (size_t)n, NULL) != 0 ||
                        qd_pool_alloc(&Zd, sizeof(qd_complex128) * (size_t)n * (size_t)M, NULL) != 0 ||
                        qd_pool_alloc((void **)&wd, sizeof(double) * (size_t)M, NULL) != 0))
        rc = qd_set_error(QD_ERR_NOMEM, "device buffers");
    if (rc == QD_OK && cudaMemcpy(Hd, H, sizeof(qd_complex128) * (size_t)ld * (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "copy-in");
    if (rc == QD_OK) rc = qd_eigh_window(n, Hd, ld, lo, hi, env_precision(), wd, Zd, n, NULL);
    if (rc == QD_OK && (cudaMemcpy(eigval, wd, sizeof(double) * (size_t)M, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(eigvec, Zd, sizeof(qd_complex128) * (size_t)n * (size_t)M, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = qd_set_error(QD_ERR_CUDA, "copy-out");
    qd_pool_free(Hd, NULL);
    qd_pool_free(Zd, NULL);
    qd_pool_free(wd, NULL);
    if (rc) die("diagonalise_hamiltonian", rc);
}

void eigenstates(int n_shape, int *N_states, struct vector F, struct wave_vectors basis,
                 struct supercell_geometry *supercell, struct material_params *parameters,
                 struct eigenstate *eigenstate_vb, struct eigenstate *eigenstate_cb) {
    int rc = check_single_rank();
    int64_t npw = (int64_t)basis.N_Gx * basis.N_Gy * basis.N_Gz, n = 8 * npw;
    int idx_cb_min = (QD_N_BAND - 2) * (int)npw; /* eigenstates.c:29-36 */
    int lo = idx_cb_min - 2 * N_states[0], hi = idx_cb_min + 2 * N_states[1] - 1, M = hi - lo + 1;
    void *Hd = NULL, *Zd = NULL;
    double *wd = NULL;
    if (rc == QD_OK && (qd_pool_alloc(&Hd, sizeof(qd_complex128) * (size_t)n * (size_t)n, NULL) != 0 ||
                        qd_pool_alloc(&Zd, sizeof(qd_complex128) * (size_t)n * (size_t)M, NULL) != 0 ||
                        qd_pool_alloc((void **)&wd, sizeof(double) * (size_t)M, NULL) != 0))
        rc = qd_set_error(QD_ERR_NOMEM, "device buffers");
    double t0 = wall_s();
    if (rc == QD_OK) rc = assemble_from_globals(n_shape, F, basis, supercell, parameters, Hd, n, -1);
    double t1 = wall_s();
    if (rc == QD_OK) rc = qd_eigh_window(n, Hd, n, lo, hi, env_precision(), wd, Zd, n, NULL);
    double t2 = wall_s();
    component_run_times.ham_elements = t1 - t0;
    component_run_times.ham_diag = t2 - t1;
    double *w = (double *)malloc(sizeof(double) * (size_t)M);
    if (rc == QD_OK && cudaMemcpy(w, wd, sizeof(double) * (size_t)M, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "copy-out");
    /* collect_eigenstates.c:23-75 */
    for (int s = 0; rc == QD_OK && s < M; s++) {
        struct eigenstate *es = s < 2 * N_states[0] ? &eigenstate_vb[s] : &eigenstate_cb[s - 2 * N_states[0]];
        es->E = w[s];
        if (cudaMemcpy(es->fourier, (qd_complex128 *)Zd + (int64_t)s * n, sizeof(qd_complex128) * (size_t)n,
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = qd_set_error(QD_ERR_CUDA, "copy-out");
    }
    free(w);
    qd_pool_free(Hd, NULL);
    qd_pool_free(Zd, NULL);
    qd_pool_free(wd, NULL);
    if (rc) die("eigenstates", rc);
}

void coulomb_matrix_elements(struct wave_vectors basis, struct wave_vectors coulomb_basis,
                             struct supercell_geometry *supercell, struct material_params *parameters, int *N_states,
                             struct eigenstate *eigenstate_vb, struct eigenstate *eigenstate_cb,
                             struct coulomb_matrix_element CME, int coulomb_region_type);

/* ------------------------------------------------------------------------- */
/* Hellmann-Feynman gradients of the window's eigenvalues                     */
/* ------------------------------------------------------------------------- */
int qd_coef_diff(const void *plus, const void *minus, int64_t n, double scale, void *d, void *stream);
int qd_coef_diff4(const void *p1, const void *m1, const void *p2, const void *m2, int64_t n, double scale, void *d,
                  void *stream);
int qd_chi_direction(struct qd_problem *pr, int s, const struct supercell_geometry *geo4, void **dir_s, void **dir);
int qd_grad_contract(const void *d_dcoef, const double *d_Gx, const double *d_Gy, const double *d_Gz, const int N[3],
                     const double K[3], const void *psi, int64_t ldz, int m, double *out_dev, void *stream);

/* Every device table of the problem is freed (the next build allocates anew). */
static void release_tables(qd_problem *pr) {
    for (int a = 0; a < 3; a++) {
        if (pr->d_G[a]) qd_pool_free(pr->d_G[a], NULL);
        if (pr->d_GS[a]) qd_pool_free(pr->d_GS[a], NULL);
        pr->d_G[a] = NULL;
        pr->d_GS[a] = NULL;
    }
    void **dev[] = {&pr->d_geo, &pr->d_mat, &pr->d_chi_s, &pr->d_eps_s, &pr->d_phi_s, &pr->d_chi,
                    &pr->d_eps, &pr->d_phi, &pr->d_conv, &pr->d_coef};
    for (size_t i = 0; i < sizeof(dev) / sizeof(dev[0]); i++) {
        if (*dev[i]) qd_pool_free(*dev[i], NULL);
        *dev[i] = NULL;
    }
    pr->tables_ready = 0;
}

static double *grad_length(struct supercell_geometry *g, int k) {
    switch (k) {
        case 1: return &g->L1;
        case 2: return &g->L2;
        case 3: return &g->L3;
        case 4: return &g->L4;
        case 5: return &g->L5;
        default: return NULL;
    }
}

/* Apply value offset `delta` (internal units) to parameter q; materials are
 * re-evaluated.  Returns the parameter's current value through *value. */
static int grad_apply(qd_problem *pr, const qd_grad_param *q, double delta, double *value) {
    struct supercell_geometry *g = NULL;
    if (q->kind <= QD_GRAD_COMPOSITION) {
        if (q->shape < 1 || q->shape >= pr->p.n_shape)
            return qd_set_error(QD_ERR_ARG, "gradient parameter: shape index %d out of range", q->shape);
        g = &pr->geo[q->shape];
    }
    double *x = NULL;
    switch (q->kind) {
        case QD_GRAD_LENGTH:
            x = grad_length(g, q->index);
            if (!x) return qd_set_error(QD_ERR_ARG, "gradient parameter: length index %d not in 1..5", q->index);
            break;
        case QD_GRAD_BASE:
            g->L2 += delta;
            x = &g->L1;
            break;
        case QD_GRAD_COMPOSITION: x = &g->x; break;
        case QD_GRAD_FIELD:
            if (q->index < 0 || q->index > 2) return qd_set_error(QD_ERR_ARG, "field component %d", q->index);
            x = &pr->p.F[q->index];
            break;
        case QD_GRAD_EP: x = &qd_scale_Ep; break;
        case QD_GRAD_GAMMA1: x = &qd_scale_gL1; break;
        default: return qd_set_error(QD_ERR_ARG, "gradient parameter kind %d", q->kind);
    }
    *x += delta;
    if (value) *value = *x;
    return qd_material_parameters(pr->p.T, pr->p.piezo, pr->p.n_shape, pr->geo, pr->mat);
}

/* Step floor (internal units) and the factor from the internal derivative to
 * the reported one (per nm, per unit composition, per kV/cm, per unit scale). */
static void grad_units(int kind, double *floor_, double *to_user) {
    switch (kind) {
        case QD_GRAD_LENGTH:
        case QD_GRAD_BASE: *floor_ = 10.0; *to_user = 10.0; break;        /* Angstrom -> per nm */
        case QD_GRAD_COMPOSITION: *floor_ = 0.1; *to_user = 1.0; break;
        case QD_GRAD_FIELD: *floor_ = 1.0e-5; *to_user = 1.0e-5; break;   /* V/Angstrom -> per kV/cm */
        default: *floor_ = 1.0; *to_user = 1.0; break;                     /* relative scales */
    }
}

static __thread int g_sm_budget = 0;
int qd_sm_budget(int nsm) { return g_sm_budget > 0 && g_sm_budget < nsm ? g_sm_budget : nsm; }
void qd_set_sm_budget(int n) { g_sm_budget = n > 0 ? n : 0; }

/* Contraction used by eigen_gradients_8_band: 0 = reciprocal-space
 * correlations by FFT (default), 1 = the direct sum over the lower triangle of
 * dH (an independent check). */
int qd_grad_method = 0;

int qd_material_tangent(int which, int n_shape, const struct supercell_geometry *geo,
                        const struct material_params *mat, struct material_params *dmat);
int qd_tables_tangent_dev(struct qd_problem *pr, const struct material_params *dmat, const double dF[3], void *dcoef);

int qd_grad_corr_tables(const double *d_Gx, const double *d_Gy, const double *d_Gz, const int N[3], const double K[3],
                        const void *psi, int64_t ldz, int m, void **C_out, int P_out[3], void *stream);
int qd_grad_corr_dot(const void *d_dcoef, const int N[3], const void *C, const int P[3], int m, double *out_dev,
                     void *stream);

int eigen_gradients_8_band(qd_problem *pr, const qd_complex128 *eigvec_host, int n_states,
                           const qd_grad_param *params, int n_params, double rel_step, double *dEdp) {
    if (!pr || !eigvec_host || !params || !dEdp || n_states < 1 || n_params < 1)
        return qd_set_error(QD_ERR_ARG, "eigen_gradients_8_band: bad arguments");
    if (!(rel_step > 0.0)) rel_step = 1e-4;
    RC(qd_problem_build_tables(pr));
    const int64_t nt = pr->nT, ncoef = (int64_t)QD_N_COEF * nt, nh = pr->n_h;
    void *Z = NULL, *dplus = NULL, *dminus = NULL, *dcoef = NULL, *dplus2 = NULL, *dminus2 = NULL;
    double *out = NULL;
    int rc = QD_OK;
    if (qd_pool_alloc(&Z, sizeof(qd_complex128) * (size_t)nh * n_states, NULL) ||
        qd_pool_alloc(&dplus, sizeof(qd_complex128) * (size_t)ncoef, NULL) ||
        qd_pool_alloc(&dminus, sizeof(qd_complex128) * (size_t)ncoef, NULL) ||
        qd_pool_alloc(&dcoef, sizeof(qd_complex128) * (size_t)ncoef, NULL) ||
        qd_pool_alloc((void **)&out, sizeof(double) * (size_t)n_params * n_states, NULL))
        rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band: work buffers");
    if (rc == QD_OK && cudaMemcpy(Z, eigvec_host, sizeof(qd_complex128) * (size_t)nh * n_states,
                                  cudaMemcpyHostToDevice) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "eigen_gradients_8_band: eigenvector upload");
    /* correlation tables of the states, shared by every parameter */
    void *corr = NULL;
    int P[3] = {0, 0, 0};
    const int direct = qd_grad_method == 1;
    if (rc == QD_OK && !direct)
        rc = qd_grad_corr_tables(pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->p.N, pr->p.K, Z, nh, n_states, &corr, P, NULL);
    /* originals, restored exactly after each parameter */
    const int ns = pr->p.n_shape;
    struct supercell_geometry *geo0 = (struct supercell_geometry *)malloc(sizeof(*geo0) * ns);
    qd_params p0 = pr->p;
    const double sEp = qd_scale_Ep, sg1 = qd_scale_gL1;
    struct material_params *dmat = (struct material_params *)malloc(sizeof(*dmat) * ns);
    if (!geo0 || !dmat) rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band");
    else memcpy(geo0, pr->geo, sizeof(*geo0) * ns);
    /* Two passes: first the parameters whose derivative table is exact (the
     * table is linear in the field and in the material parameters, so it is
     * the fused sum of the tangents, taken on the problem's own tables), then
     * those that move the shapes or the composition (central difference of two
     * table builds; they leave the tables rebuilt at a perturbed point). */
    for (int pass = 0; pass < 2 && rc == QD_OK; pass++)
        for (int k = 0; rc == QD_OK && k < n_params; k++) {
            const qd_grad_param *q = &params[k];
            const int exact = q->kind == QD_GRAD_FIELD || q->kind == QD_GRAD_EP || q->kind == QD_GRAD_GAMMA1;
            if (exact != (pass == 0)) continue;
            if (exact) {
                double dF[3] = {0.0, 0.0, 0.0};
                if (q->kind == QD_GRAD_FIELD) {
                    if (q->index < 0 || q->index > 2) {
                        rc = qd_set_error(QD_ERR_ARG, "field component %d", q->index);
                        break;
                    }
                    dF[q->index] = 1.0;
                    memset(dmat, 0, sizeof(*dmat) * ns);
                } else if ((rc = qd_material_tangent(q->kind == QD_GRAD_EP ? 0 : 1, ns, pr->geo, pr->mat, dmat))) {
                    break;
                }
                if ((rc = qd_tables_tangent_dev(pr, dmat, dF, dcoef))) break;
            } else if (q->kind == QD_GRAD_LENGTH || q->kind == QD_GRAD_BASE) {
                /* A length moves only chi of its shape.  dchi/dL: fourth-order central difference
                 * of the closed-form transforms (steps +-h, +-2h).  The table is a polynomial in chi
                 * (strain linear, convolutions and first-order piezo quadratic, second-order piezo
                 * and the position-dependent elastic series of higher degree), so its derivative
                 * along dir = h dchi/dL is taken exactly by builds at chi + t dir: t = +-1 (exact to
                 * degree 2), or +-1, +-2 (exact to degree 4) when second-order piezo or
                 * position-dependent elastic constants raise the degree. */
                double v0 = 0.0, floor_ = 1.0, to_user = 1.0, dummy;
                if ((rc = grad_apply(pr, q, 0.0, &v0))) break;
                grad_units(q->kind, &floor_, &to_user);
                const double h = rel_step * (fabs(v0) > floor_ ? fabs(v0) : floor_);
                struct supercell_geometry *g4 = (struct supercell_geometry *)malloc(sizeof(*g4) * 4 * (size_t)ns);
                if (!g4) {
                    rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band");
                    break;
                }
                const double del[4] = {2.0 * h, h, -h, -2.0 * h};
                for (int k4 = 0; rc == QD_OK && k4 < 4; k4++) {
                    rc = grad_apply(pr, q, del[k4], &dummy);
                    memcpy(g4 + (size_t)k4 * ns, pr->geo, sizeof(*g4) * ns);
                    memcpy(pr->geo, geo0, sizeof(*geo0) * ns);
                    pr->p = p0;
                    if (rc == QD_OK) rc = qd_material_parameters(pr->p.T, pr->p.piezo, ns, pr->geo, pr->mat);
                }
                void *dir_s = NULL, *dir = NULL;
                if (rc == QD_OK) rc = qd_chi_direction(pr, q->shape, g4, &dir_s, &dir);
                free(g4);
                const int four = pr->p.piezo >= 2 || pr->p.elastic_const != 0;
                if (rc == QD_OK && four && !dplus2 &&
                    (qd_pool_alloc(&dplus2, sizeof(qd_complex128) * (size_t)ncoef, NULL) ||
                     qd_pool_alloc(&dminus2, sizeof(qd_complex128) * (size_t)ncoef, NULL)))
                    rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band: work buffers");
                const double ts[4] = {1.0, -1.0, 2.0, -2.0};
                void *outs[4] = {dplus, dminus, dplus2, dminus2};
                pr->chi_dir_shape = q->shape;
                pr->d_chi_dir_s = dir_s;
                pr->d_chi_dir = dir;
                for (int k4 = 0; rc == QD_OK && k4 < (four ? 4 : 2); k4++) {
                    pr->chi_dir_t = ts[k4];
                    release_tables(pr);
                    if ((rc = qd_tables_build_dev(pr))) break;
                    if (cudaMemcpy(outs[k4], pr->d_coef, sizeof(qd_complex128) * (size_t)ncoef,
                                   cudaMemcpyDeviceToDevice) != cudaSuccess)
                        rc = qd_set_error(QD_ERR_CUDA, "eigen_gradients_8_band: table copy");
                }
                pr->chi_dir_t = 0.0;
                pr->d_chi_dir_s = pr->d_chi_dir = NULL;
                qd_pool_free(dir_s, NULL);
                qd_pool_free(dir, NULL);
                if (rc) break;
                rc = four ? qd_coef_diff4(dplus, dminus, dplus2, dminus2, ncoef, 1.0 / (12.0 * h), dcoef, NULL)
                          : qd_coef_diff(dplus, dminus, ncoef, 1.0 / (2.0 * h), dcoef, NULL);
                if (rc) break;
            } else if (q->kind == QD_GRAD_COMPOSITION) {
                /* The composition moves only the composed shape's material parameters, and for a
                 * fixed geometry the table is a polynomial in them (the mismatch (a_emb - a_s) /
                 * a_matrix is linear in a_s; band parameters, P and deformation potentials enter
                 * linearly, products with the strain give degree two, second-order piezo and the
                 * position-dependent elastic series more).  dmat/dx: fourth-order central
                 * difference of the host material function (steps +-h, +-2h); the table's
                 * derivative along dmat is then exact from builds at mat +- t dmat. */
                double v0 = 0.0, floor_ = 1.0, to_user = 1.0, dummy;
                if ((rc = grad_apply(pr, q, 0.0, &v0))) break;
                grad_units(q->kind, &floor_, &to_user);
                const double h = rel_step * (fabs(v0) > floor_ ? fabs(v0) : floor_);
                const size_t nd = sizeof(struct material_params) / sizeof(double);
                double *m4 = (double *)malloc(sizeof(struct material_params) * 5 * (size_t)ns);
                if (!m4) {
                    rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band");
                    break;
                }
                double *mat0 = m4 + 4 * nd * (size_t)ns;
                const double del[4] = {2.0 * h, h, -h, -2.0 * h};
                for (int k4 = 0; rc == QD_OK && k4 < 4; k4++) {
                    rc = grad_apply(pr, q, del[k4], &dummy);
                    memcpy(m4 + (size_t)k4 * nd * ns, pr->mat, sizeof(struct material_params) * ns);
                    memcpy(pr->geo, geo0, sizeof(*geo0) * ns);
                    pr->p = p0;
                    if (rc == QD_OK) rc = qd_material_parameters(pr->p.T, pr->p.piezo, ns, pr->geo, pr->mat);
                }
                if (rc == QD_OK) memcpy(mat0, pr->mat, sizeof(struct material_params) * ns);
                const int four = pr->p.piezo >= 2 || pr->p.elastic_const != 0;
                if (rc == QD_OK && four && !dplus2 &&
                    (qd_pool_alloc(&dplus2, sizeof(qd_complex128) * (size_t)ncoef, NULL) ||
                     qd_pool_alloc(&dminus2, sizeof(qd_complex128) * (size_t)ncoef, NULL)))
                    rc = qd_set_error(QD_ERR_NOMEM, "eigen_gradients_8_band: work buffers");
                const double ts[4] = {1.0, -1.0, 2.0, -2.0};
                void *outs[4] = {dplus, dminus, dplus2, dminus2};
                for (int k4 = 0; rc == QD_OK && k4 < (four ? 4 : 2); k4++) {
                    double *mp = (double *)pr->mat;
                    for (size_t e = 0; e < nd * (size_t)ns; e++) {
                        const size_t o = e;  /* field e % nd of shape e / nd */
                        const double dm = (-m4[o] + 8.0 * m4[nd * ns + o] - 8.0 * m4[2 * nd * ns + o] +
                                           m4[3 * nd * ns + o]) / 12.0;
                        mp[e] = mat0[e] + ts[k4] * dm;
                    }
                    release_tables(pr);
                    if ((rc = qd_tables_build_dev(pr))) break;
                    if (cudaMemcpy(outs[k4], pr->d_coef, sizeof(qd_complex128) * (size_t)ncoef,
                                   cudaMemcpyDeviceToDevice) != cudaSuccess)
                        rc = qd_set_error(QD_ERR_CUDA, "eigen_gradients_8_band: table copy");
                }
                memcpy(pr->mat, mat0, sizeof(struct material_params) * ns);
                free(m4);
                if (rc) break;
                rc = four ? qd_coef_diff4(dplus, dminus, dplus2, dminus2, ncoef, 1.0 / (12.0 * h), dcoef, NULL)
                          : qd_coef_diff(dplus, dminus, ncoef, 1.0 / (2.0 * h), dcoef, NULL);
                if (rc) break;
            } else {
                double v0 = 0.0, floor_ = 1.0, to_user = 1.0;
                if ((rc = grad_apply(pr, q, 0.0, &v0))) break;
                grad_units(q->kind, &floor_, &to_user);
                const double h = rel_step * (fabs(v0) > floor_ ? fabs(v0) : floor_);
                for (int side = 0; rc == QD_OK && side < 2; side++) {
                    double dummy;
                    if ((rc = grad_apply(pr, q, side == 0 ? h : -h, &dummy))) break;
                    release_tables(pr);
                    if ((rc = qd_tables_build_dev(pr))) break;
                    if (cudaMemcpy(side == 0 ? dplus : dminus, pr->d_coef, sizeof(qd_complex128) * (size_t)ncoef,
                                   cudaMemcpyDeviceToDevice) != cudaSuccess)
                        rc = qd_set_error(QD_ERR_CUDA, "eigen_gradients_8_band: table copy");
                    /* back to the exact original values before the other side */
                    memcpy(pr->geo, geo0, sizeof(*geo0) * ns);
                    pr->p = p0;
                    qd_scale_Ep = sEp;
                    qd_scale_gL1 = sg1;
                    if (rc == QD_OK) rc = qd_material_parameters(pr->p.T, pr->p.piezo, ns, pr->geo, pr->mat);
                }
                if (rc) break;
                if ((rc = qd_coef_diff(dplus, dminus, ncoef, 1.0 / (2.0 * h), dcoef, NULL))) break;
            }
            if (direct)
                rc = qd_grad_contract(dcoef, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->p.N, pr->p.K, Z, nh, n_states,
                                      out + (size_t)k * n_states, NULL);
            else
                rc = qd_grad_corr_dot(dcoef, pr->p.N, corr, P, n_states, out + (size_t)k * n_states, NULL);
        }
    free(dmat);
    /* the problem's own tables again */
    if (geo0) {
        memcpy(pr->geo, geo0, sizeof(*geo0) * ns);
        free(geo0);
    }
    pr->p = p0;
    qd_scale_Ep = sEp;
    qd_scale_gL1 = sg1;
    int rc2 = qd_material_parameters(pr->p.T, pr->p.piezo, ns, pr->geo, pr->mat);
    release_tables(pr);
    if (rc2 == QD_OK) rc2 = qd_tables_build_dev(pr);
    if (rc == QD_OK) rc = rc2;
    if (rc == QD_OK) {
        if (cudaMemcpy(dEdp, out, sizeof(double) * (size_t)n_params * n_states, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = qd_set_error(QD_ERR_CUDA, "eigen_gradients_8_band: copy-out");
        for (int k = 0; rc == QD_OK && k < n_params; k++) {
            double floor_, to_user;
            grad_units(params[k].kind, &floor_, &to_user);
            for (int s = 0; s < n_states; s++) dEdp[(size_t)k * n_states + s] *= to_user;
        }
    }
    void *bufs[] = {Z, dplus, dminus, dcoef, out, corr, dplus2, dminus2};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        if (bufs[i]) qd_pool_free(bufs[i], NULL);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Momentum matrix elements <vb| dH/dk_a |cb>                                 */
/* ------------------------------------------------------------------------- */
int qd_problem_assemble_dk_dev(qd_problem *pr, int axis, void *H_dev, int64_t ld, int mode, void *stream) {
    if (!pr) return qd_set_error(QD_ERR_ARG, "null problem");
    RC(qd_problem_build_tables(pr));
    return qd_assemble_dk_launch(pr->d_coef, pr->d_G[0], pr->d_G[1], pr->d_G[2], pr->p.N, pr->p.K, axis, H_dev, ld,
                                 mode, stream);
}

int qd_momentum_matrix_elements(qd_problem *pr, const qd_complex128 *eigvec_host, int n_vb_states, int n_cb_states,
                                qd_complex128 *mme) {
    if (!pr || !eigvec_host || !mme || n_vb_states < 1 || n_cb_states < 1)
        return qd_set_error(QD_ERR_ARG, "qd_momentum_matrix_elements: bad arguments");
    RC(qd_problem_build_tables(pr));
    const int64_t n = pr->n_h;
    const int M = n_vb_states + n_cb_states;
    void *dH = NULL, *Z = NULL, *Y = NULL, *G = NULL;
    int rc = QD_OK;
    if (qd_pool_alloc(&dH, sizeof(qd_complex128) * (size_t)n * (size_t)n, NULL) ||
        qd_pool_alloc(&Z, sizeof(qd_complex128) * (size_t)n * M, NULL) ||
        qd_pool_alloc(&Y, sizeof(qd_complex128) * (size_t)n * n_cb_states, NULL) ||
        qd_pool_alloc(&G, sizeof(qd_complex128) * (size_t)n_vb_states * n_cb_states, NULL))
        rc = qd_set_error(QD_ERR_NOMEM, "qd_momentum_matrix_elements: device buffers");
    if (rc == QD_OK && cudaMemcpy(Z, eigvec_host, sizeof(qd_complex128) * (size_t)n * M, cudaMemcpyHostToDevice) !=
                           cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "qd_momentum_matrix_elements: upload");
    qd_complex128 *g = (qd_complex128 *)malloc(sizeof(qd_complex128) * (size_t)n_vb_states * n_cb_states);
    if (rc == QD_OK && !g) rc = qd_set_error(QD_ERR_NOMEM, "qd_momentum_matrix_elements");
    const qd_complex128 *Zcb = (const qd_complex128 *)Z + (size_t)n * n_vb_states;
    for (int a = 0; rc == QD_OK && a < 3; a++) {
        /* momentum_matrix_element.c:81 (zhemv) and :97 (zdotc), all pairs at once */
        if ((rc = qd_problem_assemble_dk_dev(pr, a, dH, n, 0, NULL))) break;
        if ((rc = qd_hemm_lower_dev(n, dH, n, Zcb, n, n_cb_states, Y, n, 0.0, NULL))) break;
        if ((rc = qd_gram_dev(n, Z, n, n_vb_states, Y, n, n_cb_states, G, n_vb_states, NULL))) break;
        if (cudaMemcpy(g, G, sizeof(qd_complex128) * (size_t)n_vb_states * n_cb_states, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
            rc = qd_set_error(QD_ERR_CUDA, "qd_momentum_matrix_elements: copy-out");
            break;
        }
        /* 8_band_main.c:1647: [pol][cb][vb], valence states from the highest down */
        for (int c = 0; c < n_cb_states; c++)
            for (int v = 0; v < n_vb_states; v++)
                mme[((size_t)a * n_cb_states + c) * n_vb_states + v] = g[(n_vb_states - 1 - v) + (size_t)c * n_vb_states];
    }
    free(g);
    void *bufs[] = {dH, Z, Y, G};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); i++)
        if (bufs[i]) qd_pool_free(bufs[i], NULL);
    return rc;
}

/* Replaces code/source/8_band/hamiltonian_derivative_8_band.c:23: dH/dk for
 * polarisation 0, 1, 2 ([100], [010], [001]) into the caller's host H_dk
 * (lower triangle, leading dimension na_rows), from the reference's globals. */
void hamiltonian_derivative_8_band(int polarisation, int n_shape, struct wave_vectors basis,
                                   struct supercell_geometry *supercell, struct material_params *parameters,
                                   qd_complex128 *H_dk) {
    int rc = check_single_rank();
    int64_t n = (int64_t)8 * basis.N_Gx * basis.N_Gy * basis.N_Gz;
    int64_t ld = na_rows > 0 ? na_rows : n;
    void *Hd = NULL;
    if (rc == QD_OK && qd_pool_alloc(&Hd, sizeof(qd_complex128) * (size_t)ld * (size_t)n, NULL) != 0)
        rc = qd_set_error(QD_ERR_NOMEM, "device dH/dk");
    struct vector F0 = {0.0, 0.0, 0.0};
    if (rc == QD_OK) rc = assemble_from_globals(n_shape, F0, basis, supercell, parameters, Hd, ld, polarisation);
    for (int64_t c = 0; rc == QD_OK && c < n; c++) {
        cudaError_t e = cudaMemcpy(H_dk + c + c * ld, (qd_complex128 *)Hd + c + c * ld,
                                   sizeof(qd_complex128) * (size_t)(n - c), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = qd_set_error(QD_ERR_CUDA, "copy-out: %s", cudaGetErrorString(e));
    }
    if (Hd) qd_pool_free(Hd, NULL);
    if (rc) die("hamiltonian_derivative_8_band", rc);
}

/* Device state of momentum_matrix_element between calls: dH/dk of the
 * current polarisation (Polarisation_Indicator), the product y = dH/dk psi_1
 * of the last conduction state and a staging vector for psi_2. */
static struct {
    void *dH, *psi, *y, *r;
    int64_t n;
    int pol;
} g_mme = {NULL, NULL, NULL, NULL, 0, -1};

/* Replaces code/source/8_band/momentum_matrix_element.c:24.  Same contract:
 * dH/dk is rebuilt when Polarisation_Indicator differs from polarisation,
 * y = dH/dk psi_1 is recomputed when eigenstate_2_idx is the first valence
 * state (2 N_states[0] - 1) and otherwise reused, and the result is
 * psi_2^H y.  dH/dk and y stay on the device; the reference's host arrays
 * dH_dk and yV are not written. */
qd_complex128 momentum_matrix_element(int polarisation, int n_shape, struct wave_vectors basis,
                                      struct supercell_geometry *supercell, struct material_params *parameters,
                                      struct eigenstate eigenstate_1, int64_t eigenstate_1_idx,
                                      struct eigenstate eigenstate_2, int64_t eigenstate_2_idx, int *N_states) {
    (void)eigenstate_1_idx;
    int rc = check_single_rank();
    const int64_t n = (int64_t)8 * basis.N_Gx * basis.N_Gy * basis.N_Gz;
    if (rc == QD_OK && g_mme.n != n) {
        void *p[] = {g_mme.dH, g_mme.psi, g_mme.y, g_mme.r};
        for (int i = 0; i < 4; i++)
            if (p[i]) cudaFree(p[i]);
        g_mme.dH = g_mme.psi = g_mme.y = g_mme.r = NULL;
        if (cudaMalloc(&g_mme.dH, sizeof(qd_complex128) * (size_t)n * (size_t)n) != cudaSuccess ||
            cudaMalloc(&g_mme.psi, sizeof(qd_complex128) * (size_t)n) != cudaSuccess ||
            cudaMalloc(&g_mme.y, sizeof(qd_complex128) * (size_t)n) != cudaSuccess ||
            cudaMalloc(&g_mme.r, sizeof(qd_complex128)) != cudaSuccess)
            rc = qd_set_error(QD_ERR_NOMEM, "momentum_matrix_element: device buffers");
        g_mme.n = rc == QD_OK ? n : 0;
        g_mme.pol = -1;
        Polarisation_Indicator = -1;
    }
    if (rc == QD_OK && (Polarisation_Indicator != polarisation || g_mme.pol != polarisation)) {
        struct vector F0 = {0.0, 0.0, 0.0};
        rc = assemble_from_globals(n_shape, F0, basis, supercell, parameters, g_mme.dH, n, polarisation);
        if (rc == QD_OK) {
            Polarisation_Indicator = polarisation;
            g_mme.pol = polarisation;
        }
    }
    if (rc == QD_OK && eigenstate_2_idx == 2 * (int64_t)N_states[0] - 1) {
        if (cudaMemcpy(g_mme.psi, eigenstate_1.fourier, sizeof(qd_complex128) * (size_t)n, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            rc = qd_set_error(QD_ERR_CUDA, "momentum_matrix_element: upload");
        if (rc == QD_OK) rc = qd_hemm_lower_dev(n, g_mme.dH, n, g_mme.psi, n, 1, g_mme.y, n, 0.0, NULL);
    }
    qd_complex128 result;
    memset(&result, 0, sizeof(result));
    if (rc == QD_OK &&
        cudaMemcpy(g_mme.psi, eigenstate_2.fourier, sizeof(qd_complex128) * (size_t)n, cudaMemcpyHostToDevice) !=
            cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "momentum_matrix_element: upload");
    if (rc == QD_OK) rc = qd_gram_dev(n, g_mme.psi, n, 1, g_mme.y, n, 1, g_mme.r, 1, NULL);
    if (rc == QD_OK && cudaMemcpy(&result, g_mme.r, sizeof(result), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "momentum_matrix_element: copy-out");
    if (rc) die("momentum_matrix_element", rc);
    return result;
}

/* ------------------------------------------------------------------------- */
/* Real-space envelope functions (envelope_functions.c:23-220)                */
/* ------------------------------------------------------------------------- */
int qd_envelope_dev(const int N[3], const double *d_Gx, const double *d_Gy, const double *d_Gz, const double K[3],
                    double volume, const void *Z, int64_t ldz, int m, int n_grid, const double *x, const double *y,
                    const double *z, void *F, double *prob, void *stream);

/* Host-side driver shared by the qd_ entry point and the reference-named one:
 * G grids and points are host arrays, states host N_H x m; outputs host
 * [state][band][point] (either may be NULL). */
static int envelopes_host(const int N[3], const double *const G[3], const double K[3], double volume,
                          const qd_complex128 *Zh, int64_t ldz, int m, int n_grid, const double *x, const double *y,
                          const double *z, qd_complex128 *F, double *prob) {
    const int64_t npw = (int64_t)N[0] * N[1] * N[2], nh = 8 * npw;
    const int NT[3] = {2 * N[0] - 1, 2 * N[1] - 1, 2 * N[2] - 1};
    double *dG = NULL, *dp = NULL, *dprob = NULL;
    void *dZ = NULL, *dF = NULL;
    int rc = QD_OK;
    const size_t nout = (size_t)m * 8 * n_grid;
    if (cudaMalloc((void **)&dG, sizeof(double) * (NT[0] + NT[1] + NT[2])) != cudaSuccess ||
        cudaMalloc((void **)&dp, sizeof(double) * 3 * (size_t)n_grid) != cudaSuccess ||
        cudaMalloc(&dZ, sizeof(qd_complex128) * (size_t)nh * m) != cudaSuccess ||
        (F && cudaMalloc(&dF, sizeof(qd_complex128) * nout) != cudaSuccess) ||
        (prob && cudaMalloc((void **)&dprob, sizeof(double) * nout) != cudaSuccess))
        rc = qd_set_error(QD_ERR_NOMEM, "envelope functions: device buffers");
    for (int a = 0, o = 0; rc == QD_OK && a < 3; o += NT[a], a++)
        if (cudaMemcpy(dG + o, G[a], sizeof(double) * NT[a], cudaMemcpyHostToDevice) != cudaSuccess)
            rc = qd_set_error(QD_ERR_CUDA, "envelope functions: upload");
    if (rc == QD_OK && (cudaMemcpy(dp, x, sizeof(double) * n_grid, cudaMemcpyHostToDevice) != cudaSuccess ||
                        cudaMemcpy(dp + n_grid, y, sizeof(double) * n_grid, cudaMemcpyHostToDevice) != cudaSuccess ||
                        cudaMemcpy(dp + 2 * (size_t)n_grid, z, sizeof(double) * n_grid, cudaMemcpyHostToDevice) !=
                            cudaSuccess ||
                        cudaMemcpy2D(dZ, sizeof(qd_complex128) * nh, Zh, sizeof(qd_complex128) * ldz,
                                     sizeof(qd_complex128) * nh, m, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = qd_set_error(QD_ERR_CUDA, "envelope functions: upload");
    if (rc == QD_OK)
        rc = qd_envelope_dev(N, dG, dG + NT[0], dG + NT[0] + NT[1], K, volume, dZ, nh, m, n_grid, dp, dp + n_grid,
                             dp + 2 * (size_t)n_grid, dF, dprob, NULL);
    if (rc == QD_OK && F && cudaMemcpy(F, dF, sizeof(qd_complex128) * nout, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "envelope functions: copy-out");
    if (rc == QD_OK && prob && cudaMemcpy(prob, dprob, sizeof(double) * nout, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = qd_set_error(QD_ERR_CUDA, "envelope functions: copy-out");
    cudaFree(dG);
    cudaFree(dp);
    cudaFree(dZ);
    cudaFree(dF);
    cudaFree(dprob);
    return rc;
}

int qd_envelope_functions(qd_problem *pr, const qd_complex128 *eigvec_host, int m, int n_grid, const double *x,
                          const double *y, const double *z, qd_complex128 *F, double *prob) {
    if (!pr || !eigvec_host || m < 1 || n_grid < 1 || !x || !y || !z)
        return qd_set_error(QD_ERR_ARG, "qd_envelope_functions: bad arguments");
    const double vol = pr->geo[0].L1 * pr->geo[0].L2 * pr->geo[0].L3;
    const double *G[3] = {pr->G[0], pr->G[1], pr->G[2]};
    return envelopes_host(pr->p.N, G, pr->p.K, vol, eigvec_host, pr->n_h, m, n_grid, x, y, z, F, prob);
}

/* Replaces code/source/8_band/envelope_functions.c:23.  For the 2 N_states[type]
 * states of eigenstate (type 0 valence, 1 conduction) fills F_1..F_8 and
 * probability_1..probability_8 (caller-allocated, N_grid each) at the points
 * (x, y, z) in Angstrom.  `direction` only names the scan for the writers. */
void envelope_functions(struct supercell_geometry *supercell, int *N_states, int type, int N_grid, double *x,
                        double *y, double *z, struct wave_vectors basis, struct eigenstate *eigenstate,
                        int direction) {
    (void)direction;
    int rc = check_single_rank();
    const int m = 2 * N_states[type];
    const int N[3] = {basis.N_Gx, basis.N_Gy, basis.N_Gz};
    const int64_t nh = (int64_t)8 * N[0] * N[1] * N[2];
    const double *G[3] = {basis.Gx, basis.Gy, basis.Gz};
    const double K[3] = {basis.Kx, basis.Ky, basis.Kz};
    const double vol = supercell[0].L1 * supercell[0].L2 * supercell[0].L3;
    qd_complex128 *Z = NULL, *F = NULL;
    double *prob = NULL;
    const size_t nout = (size_t)m * 8 * N_grid;
    if (rc == QD_OK && (!(Z = (qd_complex128 *)malloc(sizeof(qd_complex128) * (size_t)nh * m)) ||
                        !(F = (qd_complex128 *)malloc(sizeof(qd_complex128) * nout)) ||
                        !(prob = (double *)malloc(sizeof(double) * nout))))
        rc = qd_set_error(QD_ERR_NOMEM, "envelope_functions: host buffers");
    for (int s = 0; rc == QD_OK && s < m; s++) memcpy(Z + (size_t)s * nh, eigenstate[s].fourier, sizeof(qd_complex128) * nh);
    if (rc == QD_OK) rc = envelopes_host(N, G, K, vol, Z, nh, m, N_grid, x, y, z, F, prob);
    for (int s = 0; rc == QD_OK && s < m; s++) {
        qd_complex128 *Fb[8] = {eigenstate[s].F_1, eigenstate[s].F_2, eigenstate[s].F_3, eigenstate[s].F_4,
                                eigenstate[s].F_5, eigenstate[s].F_6, eigenstate[s].F_7, eigenstate[s].F_8};
        double *Pb[8] = {eigenstate[s].probability_1, eigenstate[s].probability_2, eigenstate[s].probability_3,
                         eigenstate[s].probability_4, eigenstate[s].probability_5, eigenstate[s].probability_6,
                         eigenstate[s].probability_7, eigenstate[s].probability_8};
        for (int b = 0; b < 8; b++) {
            if (Fb[b]) memcpy(Fb[b], F + ((size_t)s * 8 + b) * N_grid, sizeof(qd_complex128) * N_grid);
            if (Pb[b]) memcpy(Pb[b], prob + ((size_t)s * 8 + b) * N_grid, sizeof(double) * N_grid);
        }
    }
    free(Z);
    free(F);
    free(prob);
    if (rc) die("envelope_functions", rc);
}

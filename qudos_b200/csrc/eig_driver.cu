// Partial Hermitian eigensolver for an index window [lo, hi] (the zheevr
// RANGE='I' call of diagonalise_hamiltonian.c:55-77), on one GPU.
//
// FP64 path:  stage 1 (dense -> band, FP64) -> stage 2 (band -> tridiagonal)
//             -> bisection for [lo, hi] -> band inverse iteration -> Q1 back-transform.
// Mixed path: stage 1 on a complex64 copy (tensor-core CGEMMs) -> stage 2,
//             bisection and inverse iteration in FP64 on that band for
//             [lo - g, hi + g] (g guard states on each side) -> complex64
//             back-transform -> one FP64 Rayleigh-Ritz step against the FP64 H
//             (Y = H X with ZHEMM, k x k generalized Hermitian eigenproblem by
//             Cholesky + Jacobi in one block) -> the window's eigenpairs.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "eig_common.cuh"
#include "qd_internal.h"

typedef cpx<double> zd;

extern "C" int qd_stage1_alloc(int64_t n, int b, int elem_bytes, Stage1Work *w, cudaStream_t st);
extern "C" void qd_stage1_free(Stage1Work *w, cudaStream_t st);
extern "C" int qd_stage1_run(void *A, int64_t n, int64_t lda, int b, int fp32, Stage1Work *w, void *stream);
extern "C" int qd_extract_band(const void *A, int64_t n, int64_t lda, int b, int fp32, const Stage1Work *w,
                               double2 *AB, int ldb, void *stream);
extern "C" int qd_stage1_backtransform(const void *A, int64_t n, int64_t lda, int b, int fp32, const Stage1Work *w,
                                       void *Z, int64_t ldz, int mz, void *stream);
extern "C" int qd_hb2st(double2 *AB, int ldb, int n, int b, int *progress, int *err, void *stream);
extern "C" int qd_tridiag_bisect(const double2 *AB, int ldb, int n, int lo, int hi, double *d, double *e2,
                                 double *bounds, double *w, void *stream);
extern "C" int qd_band_invit(const double2 *AB0, int ldb, int n, int b, const double *lam_dev, int ngroups,
                             const int *gstart_dev, const int *gsize_dev, double2 *Lw, double2 *Uw, int *ipivw,
                             double2 *Z, int64_t ldz, double bnorm, double2 *ywork, void *stream);
extern "C" cublasHandle_t qd_cublas(void);
extern "C" int qd_hemm_lower_dev(int64_t n, const void *H, int64_t ld, const void *X, int64_t ldx, int k, void *Y,
                                 int64_t ldy, double beta, void *stream);
extern "C" int qd_gram_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb, void *C,
                           int ldc, void *stream);
extern "C" int qd_zgemm_small_dev(int64_t n, const void *Z, int64_t ldz, int k, const void *Cm, int ldc, int k2,
                                  void *Y, int64_t ldy, double beta, void *stream);
extern "C" int qd_residual_norms_dev(int64_t n, const void *R, int64_t ldr, const void *Z, int64_t ldz,
                                     const double *w_dev, int m, double *res_dev, void *stream);

static thread_local double g_timings[8];  // per host thread (concurrent batched solves)
extern "C" int qd_last_timings(double *ms, int n) {
    for (int i = 0; i < n && i < 8; i++) ms[i] = g_timings[i];
    return QD_OK;
}
extern "C" void qd_set_timing(int i, double ms) {
    if (i >= 0 && i < 8) g_timings[i] = ms;
}

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)
#define BLAS_OK(x)                                                                                   \
    do {                                                                                             \
        cublasStatus_t s_ = (x);                                                                     \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                             \
            return qd_set_error(QD_ERR_CUDA, "%s:%d cuBLAS status %d", __FILE__, __LINE__, (int)s_); \
    } while (0)
#define RC(x)                         \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != QD_OK) return rc_; \
    } while (0)

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
// Full Hermitian complex64 copy of a complex128 lower triangle, by 32 x 32
// tiles of the lower triangle: tile (I, J), I >= J, is read once (coalesced
// down its columns), written to (I, J) and, conjugate-transposed through
// shared memory, to (J, I), so that both stores are coalesced too.  Only the
// lower triangle is read; the diagonal comes out real.
__global__ void __launch_bounds__(256) lower64_to_full32_kernel(const double2 *__restrict__ H, int64_t ld, int n,
                                                                float2 *__restrict__ H32, int64_t ld32) {
    __shared__ float2 tile[32][33];
    const int T = (n + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32 threads
    for (int64_t item = blockIdx.x; item < (int64_t)T * (T + 1) / 2; item += gridDim.x) {
        // item -> (I, J), I >= J: I (I + 1) / 2 <= item < (I + 1) (I + 2) / 2
        int I = (int)((sqrt(8.0 * (double)item + 1.0) - 1.0) * 0.5);
        while ((int64_t)I * (I + 1) / 2 > item) I--;
        while ((int64_t)(I + 1) * (I + 2) / 2 <= item) I++;
        const int J = (int)(item - (int64_t)I * (I + 1) / 2);
        const int r0 = 32 * I, c0 = 32 * J;
        // tile[a][b] holds element (r0 + b, c0 + a)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int row = r0 + tx, col = c0 + ty + 8 * k;
            float2 v = make_float2(0.f, 0.f);
            if (row < n && col < n && row >= col) {
                const double2 h = H[row + (int64_t)col * ld];
                v = make_float2((float)h.x, row == col ? 0.f : (float)h.y);
                H32[row + (int64_t)col * ld32] = v;
            }
            tile[ty + 8 * k][tx] = v;
        }
        __syncthreads();
        // strictly upper element (c0 + tx, r0 + ty + 8 k) = conj(element (r0 + ty + 8 k, c0 + tx))
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int row = c0 + tx, col = r0 + ty + 8 * k;
            if (row < n && col < n && row < col) {
                const float2 v = tile[tx][ty + 8 * k];
                H32[row + (int64_t)col * ld32] = make_float2(v.x, -v.y);
            }
        }
        __syncthreads();
    }
}

__global__ void c128_to_c64_kernel(const double2 *a, int64_t lda, float2 *b, int64_t ldb, int64_t n) {
    int64_t col = blockIdx.y;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 v = a[i + col * lda];
        b[i + col * ldb] = make_float2((float)v.x, (float)v.y);
    }
}
__global__ void c64_to_c128_kernel(const float2 *a, int64_t lda, double2 *b, int64_t ldb, int64_t n) {
    int64_t col = blockIdx.y;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 v = a[i + col * lda];
        b[i + col * ldb] = make_double2((double)v.x, (double)v.y);
    }
}

// Max |B_ij| of the band (a norm estimate for the inverse-iteration pivot floor).
__global__ void band_absmax_kernel(const double2 *AB, int ldb, int64_t n, int b, unsigned long long *out) {
    double m = 0.0;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        for (int d = 0; d <= b; d++) {
            double2 v = AB[d + j * ldb];
            m = fmax(m, sqrt(v.x * v.x + v.y * v.y));
        }
    atomicMax(out, (unsigned long long)__double_as_longlong(m));  // non-negative doubles order as integers
}

// Rayleigh-Ritz on k vectors: S = X^H X, A = X^H (H X) (k x k, column-major,
// global).  Solves A c = theta S c: S = L L^H, A' = L^-1 A L^-H, Jacobi on A',
// C = L^-H C'.  theta ascending.  One block.
__global__ void __launch_bounds__(256) small_rr_kernel(int k, double2 *S, double2 *A, double2 *C, double *theta,
                                                       int *info) {
    __shared__ double scratch[33];
    // Cholesky S = L L^H (lower, in place)
    for (int j = 0; j < k; j++) {
        __syncthreads();
        if (threadIdx.x == 0) {
            double d = S[j + j * k].x;
            for (int p = 0; p < j; p++) d -= S[j + p * k].x * S[j + p * k].x + S[j + p * k].y * S[j + p * k].y;
            if (!(d > 0.0)) { *info = 1; d = 1e-300; }
            S[j + j * k] = make_double2(sqrt(d), 0.0);
        }
        __syncthreads();
        double ljj = S[j + j * k].x;
        for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) {
            double2 s = S[i + j * k];
            for (int p = 0; p < j; p++) {  // s -= L[i,p] conj(L[j,p])
                double2 a = S[i + p * k], b = S[j + p * k];
                s.x -= a.x * b.x + a.y * b.y;
                s.y -= a.y * b.x - a.x * b.y;
            }
            S[i + j * k] = make_double2(s.x / ljj, s.y / ljj);
        }
    }
    __syncthreads();
    // A <- L^-1 A (forward substitution on each column), then A <- A L^-H (on rows)
    for (int c = threadIdx.x; c < k; c += blockDim.x) {
        for (int i = 0; i < k; i++) {
            double2 s = A[i + c * k];
            for (int p = 0; p < i; p++) {
                double2 l = S[i + p * k], a = A[p + c * k];
                s.x -= l.x * a.x - l.y * a.y;
                s.y -= l.x * a.y + l.y * a.x;
            }
            double d = S[i + i * k].x;
            A[i + c * k] = make_double2(s.x / d, s.y / d);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < k; r += blockDim.x) {
        // row r: x L^H = a  ->  x_i = (a_i - sum_{p<i} x_p conj(L[i,p])) / L[i,i]
        for (int i = 0; i < k; i++) {
            double2 s = A[r + i * k];
            for (int p = 0; p < i; p++) {
                double2 x = A[r + p * k], l = S[i + p * k];
                s.x -= x.x * l.x + x.y * l.y;
                s.y -= x.y * l.x - x.x * l.y;
            }
            double d = S[i + i * k].x;
            A[r + i * k] = make_double2(s.x / d, s.y / d);
        }
    }
    __syncthreads();
    // symmetrize, C' = I
    for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
        int i = idx % k, j = idx / k;
        if (i > j) {
            double2 a = A[i + j * k], b = A[j + i * k];
            double2 m = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
            A[i + j * k] = m;
            A[j + i * k] = make_double2(m.x, -m.y);
        } else if (i == j) {
            A[i + i * k].y = 0.0;
        }
        C[idx] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    // cyclic Jacobi with round-robin pairing (k padded to even)
    int kk = k + (k & 1);
    __shared__ int pp[128], qq[128];
    __shared__ double jc[64], js[64], jpr[64], jpi[64];  // rotation per pair: c, s, e^{-i phi}
    for (int sweep = 0; sweep < 30; sweep++) {
        double off = 0.0;
        for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
            int i = idx % k, j = idx / k;
            if (i != j) off += A[idx].x * A[idx].x + A[idx].y * A[idx].y;
        }
        off = block_sum(off, scratch);
        double dn = 0.0;
        for (int i = threadIdx.x; i < k; i += blockDim.x) dn += A[i + i * k].x * A[i + i * k].x;
        dn = block_sum(dn, scratch);
        if (off <= 1e-30 * dn || off == 0.0) break;
        for (int round = 0; round < kk - 1; round++) {
            // pairs: position 0 fixed, others rotate
            for (int t = threadIdx.x; t < kk / 2; t += blockDim.x) {
                int a = t == 0 ? 0 : 1 + (t - 1 + round) % (kk - 1);
                int bpos = kk - 1 - t;
                int b = 1 + (bpos - 1 + round) % (kk - 1);
                int p = a < b ? a : b, q = a < b ? b : a;
                pp[t] = p;
                qq[t] = q;
                double c = 1.0, s = 0.0, er = 1.0, ei = 0.0;
                if (q < k) {
                    double app = A[p + p * k].x, aqq = A[q + q * k].x;
                    double2 apq = A[p + q * k];
                    double mag = sqrt(apq.x * apq.x + apq.y * apq.y);
                    if (mag > 1e-300) {
                        er = apq.x / mag;   // e^{-i phi} with phi = arg(apq): (cos phi, -sin phi)
                        ei = -apq.y / mag;
                        double th = (aqq - app) / (2.0 * mag);
                        double t_ = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t_ * t_ + 1.0);
                        s = t_ * c;
                    }
                }
                jc[t] = c; js[t] = s; jpr[t] = er; jpi[t] = ei;
            }
            __syncthreads();
            // rows: A <- J^H A  with J = [[c, s], [-s e, c e]] on (p, q), e = e^{-i phi}
            for (int idx = threadIdx.x; idx < (kk / 2) * k; idx += blockDim.x) {
                int t = idx / k, col = idx % k;
                int p = pp[t], q = qq[t];
                if (q >= k) continue;
                double c = jc[t], s = js[t], er = jpr[t], ei = jpi[t];
                double2 ap = A[p + col * k], aq = A[q + col * k];
                // conj(j21) = -s conj(e), conj(j22) = c conj(e); conj(e) = (er, -ei)
                double2 eq = make_double2(er * aq.x + ei * aq.y, er * aq.y - ei * aq.x);  // conj(e) * aq
                A[p + col * k] = make_double2(c * ap.x - s * eq.x, c * ap.y - s * eq.y);
                A[q + col * k] = make_double2(s * ap.x + c * eq.x, s * ap.y + c * eq.y);
            }
            __syncthreads();
            // columns: A <- A J, C <- C J
            for (int idx = threadIdx.x; idx < (kk / 2) * k * 2; idx += blockDim.x) {
                int which = idx / ((kk / 2) * k);
                int r2 = idx % ((kk / 2) * k);
                int t = r2 / k, row = r2 % k;
                int p = pp[t], q = qq[t];
                if (q >= k) continue;
                double c = jc[t], s = js[t], er = jpr[t], ei = jpi[t];
                double2 *M = which == 0 ? A : C;
                double2 xp = M[row + p * k], xq = M[row + q * k];
                // new_p = xp c + xq (-s e) ; new_q = xp s + xq (c e)
                double2 xe = make_double2(xq.x * er - xq.y * ei, xq.x * ei + xq.y * er);  // xq * e
                M[row + p * k] = make_double2(c * xp.x - s * xe.x, c * xp.y - s * xe.y);
                M[row + q * k] = make_double2(s * xp.x + c * xe.x, s * xp.y + c * xe.y);
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // sort ascending (selection sort on thread 0), permute C' columns
    if (threadIdx.x == 0) {
        for (int i = 0; i < k; i++) theta[i] = A[i + i * k].x;
        for (int i = 0; i < k; i++) {
            int m = i;
            for (int j = i + 1; j < k; j++)
                if (theta[j] < theta[m]) m = j;
            if (m != i) {
                double t = theta[i]; theta[i] = theta[m]; theta[m] = t;
                for (int r = 0; r < k; r++) {
                    double2 x = C[r + i * k]; C[r + i * k] = C[r + m * k]; C[r + m * k] = x;
                }
            }
        }
    }
    __syncthreads();
    // C <- L^-H C'  (back substitution with L^H)
    for (int c = threadIdx.x; c < k; c += blockDim.x) {
        for (int i = k - 1; i >= 0; i--) {
            double2 s = C[i + c * k];
            for (int p = i + 1; p < k; p++) {  // (L^H)[i,p] = conj(L[p,i])
                double2 l = S[p + i * k], x = C[p + c * k];
                s.x -= l.x * x.x + l.y * x.y;
                s.y -= l.x * x.y - l.y * x.x;
            }
            double d = S[i + i * k].x;
            C[i + c * k] = make_double2(s.x / d, s.y / d);
        }
    }
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
struct Timer {
    cudaEvent_t e[10];
    int n = 0;
    cudaStream_t st;
    explicit Timer(cudaStream_t s) : st(s) {
        for (int i = 0; i < 10; i++) cudaEventCreate(&e[i]);
    }
    ~Timer() {
        for (int i = 0; i < 10; i++) cudaEventDestroy(e[i]);
    }
    void mark() {
        if (n < 10) cudaEventRecord(e[n++], st);
    }
    double ms(int a, int b) {
        float t = 0;
        cudaEventElapsedTime(&t, e[a], e[b]);
        return t;
    }
};

static int block_size_default() {
    const char *s = getenv("QD_BAND");
    int b = s ? atoi(s) : 32;
    if (b < 8) b = 8;
    if (b > 32) b = 32;
    return b;
}

// Per-state error bounds of the last mixed-precision solve (eV): the FP64
// residual norm ||H x - theta x|| of each window state and the Kato-Temple
// bound ||r||^2 / delta on |lambda - theta|, delta being the distance from
// theta to the nearest Ritz value outside its degenerate group (the guard
// states supply the neighbours of the window's edges).
static thread_local std::vector<double> g_res, g_bound;

extern "C" int qd_last_error_bounds(double *residual, double *bound, int n) {
    for (int i = 0; i < n && i < (int)g_res.size(); i++) {
        if (residual) residual[i] = g_res[i];
        if (bound) bound[i] = g_bound[i];
    }
    return (int)g_res.size();
}

// Largest bound accepted before the solve reports QD_ERR_CONVERGENCE (eV).
static double bound_tolerance(void) {
    const char *s = getenv("QD_BOUND_TOL");
    return s ? atof(s) : 1.0e-6;
}

static int window_error_bounds(const double *theta, int k, int off, int M, const double *res, int guard_below,
                               int guard_above) {
    g_res.assign(res, res + M);
    g_bound.assign(M, 0.0);
    double worst = 0.0;
    int iw = -1;
    for (int i = 0; i < M; i++) {
        const double t = theta[off + i];
        const double deg = 1e-9 * (fabs(t) > 1.0 ? fabs(t) : 1.0);
        double delta = INFINITY;
        for (int j = 0; j < k; j++)
            if (fabs(theta[j] - t) > deg && fabs(theta[j] - t) < delta) delta = fabs(theta[j] - t);
        // an edge state with no Ritz value beyond it in the basis has no neighbour there to bound against
        const bool edge_lo = off + i == 0 && guard_below, edge_hi = off + i == k - 1 && guard_above;
        double b = (edge_lo || edge_hi || !isfinite(delta)) ? INFINITY : res[i] * res[i] / delta;
        // the degenerate group's residual is the root sum of squares of its members'
        double rg = 0.0;
        for (int j = 0; j < M; j++)
            if (fabs(theta[off + j] - t) <= deg) rg += res[j] * res[j];
        if (isfinite(b)) b = rg / delta;
        g_bound[i] = b;
        if (!(b <= worst)) {
            worst = b;
            iw = i;
        }
    }
    if (!(worst <= bound_tolerance()))
        return qd_set_error(QD_ERR_CONVERGENCE,
                            "mixed-precision refinement: error bound %.3g eV of window state %d above %.3g eV "
                            "(residual %.3g eV); raise QD_GUARD",
                            worst, iw, bound_tolerance(), iw >= 0 ? res[iw] : 0.0);
    return QD_OK;
}

extern "C" int qd_mixed_guard(void) {
    const char *s = getenv("QD_GUARD");
    return s ? atoi(s) : 8;
}

extern "C" int qd_eigh_window(int64_t n, void *H, int64_t ld, int lo, int hi, int prec, double *w_dev, void *Z_dev,
                              int64_t ldz, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (lo < 0 || hi >= n || lo > hi) return qd_set_error(QD_ERR_ARG, "bad eigenvalue window [%d, %d] for n=%lld", lo, hi, (long long)n);
    if (n > 0x7fffffff / 2) return qd_set_error(QD_ERR_UNSUPPORTED, "matrix too large");
    int b = block_size_default();
    if (b > n - 1) b = (int)(n > 2 ? n - 1 : 1);
    const int mixed = prec == QD_PREC_MIXED;
    int g = mixed ? qd_mixed_guard() : 0;
    int lo2 = lo - g < 0 ? 0 : lo - g, hi2 = hi + g > n - 1 ? (int)n - 1 : hi + g;
    int k = hi2 - lo2 + 1, M = hi - lo + 1;
    if (mixed && k > 128)
        return qd_set_error(QD_ERR_UNSUPPORTED, "mixed precision: window plus guard states above 128 (%d)", k);
    int ldb = 2 * b + 1;
    Timer tm(st);
    tm.mark();  // 0
    // ---- stage 1
    void *A = H;
    int64_t lda = ld;
    float2 *H32 = nullptr;
    if (mixed) {
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&H32, sizeof(float2) * n * n, st));
        qd_count_launch(1);
        lower64_to_full32_kernel<<<148 * 8, 256, 0, st>>>((const double2 *)H, ld, (int)n, H32, n);
        CUDA_OK(cudaGetLastError());
        A = H32;
        lda = n;
    }
    Stage1Work w1;
    RC(qd_stage1_alloc(n, b, mixed ? 8 : 16, &w1, st));
    RC(qd_stage1_run(A, n, lda, b, mixed, &w1, st));
    tm.mark();  // 1
    // ---- band, stage 2, bisection
    double2 *AB, *AB0, *Zb;
    double *d, *e2, *bounds, *lam;
    int *progress, *err;
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&AB, sizeof(double2) * n * ldb, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&AB0, sizeof(double2) * n * ldb, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&d, sizeof(double) * n, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&e2, sizeof(double) * n, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&bounds, sizeof(double) * 4, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&lam, sizeof(double) * k, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&progress, sizeof(int) * n, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&err, sizeof(int), st));
    RC(qd_extract_band(A, n, lda, b, mixed, &w1, AB, ldb, st));
    CUDA_OK(cudaMemcpyAsync(AB0, AB, sizeof(double2) * n * ldb, cudaMemcpyDeviceToDevice, st));
    RC(qd_hb2st(AB, ldb, (int)n, b, progress, err, st));
    int herr = 0;
    CUDA_OK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (herr) return qd_set_error(QD_ERR_TIMEOUT, "band reduction: wait on the previous sweep ran out");
    tm.mark();  // 2
    RC(qd_tridiag_bisect(AB, ldb, (int)n, lo2, hi2, d, e2, bounds, lam, st));
    std::vector<double> lam_h(k);
    CUDA_OK(cudaMemcpyAsync(lam_h.data(), lam, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    unsigned long long *dmax;
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&dmax, sizeof(unsigned long long), st));
    CUDA_OK(cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), st));
    qd_count_launch(1);
    band_absmax_kernel<<<64, 256, 0, st>>>(AB0, ldb, n, b, dmax);
    unsigned long long bm_bits = 0;
    CUDA_OK(cudaMemcpyAsync(&bm_bits, dmax, sizeof(bm_bits), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    tm.mark();  // 3
    double bnorm;
    memcpy(&bnorm, &bm_bits, sizeof(double));
    bnorm *= (double)(2 * b + 1);
    // Numerically degenerate eigenvalues (within 1e-10 of the band's norm: the
    // Kramers pairs, and any accidental degeneracy on top of them) form one
    // group of up to 64: one block factorises the band once at the group's
    // shift and orthogonalises the group's vectors, which span the degenerate
    // subspace.  Distinct eigenvalues keep their own shifts; two inverse
    // iterations leave an overlap of about eps |B| / gap between them.
    std::vector<int> gs, gz;
    double tol_deg = 1e-10 * (bnorm > 1.0 ? bnorm : 1.0);
    for (int i = 0; i < k; i++) {
        if (i > 0 && fabs(lam_h[i] - lam_h[i - 1]) <= tol_deg && gz.back() < 64) gz.back()++;
        else { gs.push_back(i); gz.push_back(1); }
    }
    int ng = (int)gs.size();
    int *gs_d, *gz_d, *ipiv;
    double2 *Lw, *Uw, *yw;
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&gs_d, sizeof(int) * ng, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&gz_d, sizeof(int) * ng, st));
    CUDA_OK(cudaMemcpyAsync(gs_d, gs.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(gz_d, gz.data(), sizeof(int) * ng, cudaMemcpyHostToDevice, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Lw, sizeof(double2) * (size_t)ng * n * b, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Uw, sizeof(double2) * (size_t)ng * n * (2 * b + 1), st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&ipiv, sizeof(int) * (size_t)ng * n, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&yw, sizeof(double2) * (size_t)ng * 8 * n, st));
    CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Zb, sizeof(double2) * n * k, st));
    RC(qd_band_invit(AB0, ldb, (int)n, b, lam, ng, gs_d, gz_d, Lw, Uw, ipiv, Zb, n, bnorm, yw, st));
    tm.mark();  // 4
    // ---- back-transform
    if (!mixed) {
        RC(qd_stage1_backtransform(A, n, lda, b, 0, &w1, Zb, n, k, st));
        tm.mark();  // 5
        CUDA_OK(cudaMemcpy2DAsync(Z_dev, sizeof(double2) * ldz, Zb, sizeof(double2) * n, sizeof(double2) * n, M,
                                  cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(w_dev, lam, sizeof(double) * M, cudaMemcpyDeviceToDevice, st));
        tm.mark();  // 6
    } else {
        float2 *Z32;
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Z32, sizeof(float2) * n * k, st));
        qd_count_launch(4);
        c128_to_c64_kernel<<<dim3(64, k), 256, 0, st>>>(Zb, n, Z32, n, n);
        RC(qd_stage1_backtransform(A, n, lda, b, 1, &w1, Z32, n, k, st));
        c64_to_c128_kernel<<<dim3(64, k), 256, 0, st>>>(Z32, n, Zb, n, n);
        CUDA_OK(cudaGetLastError());
        tm.mark();  // 5
        // ---- FP64 Rayleigh-Ritz against H (lower triangle, complex128)
        double2 *Y, *S, *Ak, *C, *Xn, *YC;
        double *theta, *res;
        int *info;
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Y, sizeof(double2) * n * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Xn, sizeof(double2) * n * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&YC, sizeof(double2) * n * M, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&S, sizeof(double2) * k * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&Ak, sizeof(double2) * k * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&C, sizeof(double2) * k * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&theta, sizeof(double) * k, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&res, sizeof(double) * M, st));
        CUDA_OK((cudaError_t)qd_pool_alloc((void **)&info, sizeof(int), st));
        CUDA_OK(cudaMemsetAsync(info, 0, sizeof(int), st));
        RC(qd_hemm_lower_dev(n, H, ld, Zb, n, k, Y, n, 0.0, st));     // Y = H Z
        RC(qd_gram_dev(n, Zb, n, k, Zb, n, k, S, k, st));               // S = Z^H Z
        RC(qd_gram_dev(n, Zb, n, k, Y, n, k, Ak, k, st));               // A = Z^H H Z
        qd_count_launch(1);
        small_rr_kernel<<<1, 256, 0, st>>>(k, S, Ak, C, theta, info);
        CUDA_OK(cudaGetLastError());
        RC(qd_zgemm_small_dev(n, Zb, n, k, C, k, k, Xn, n, 0.0, st));   // X = Z C
        // residuals of the window's Ritz pairs: H X - X Theta = (H Z) C - X Theta
        const int off = lo - lo2;
        RC(qd_zgemm_small_dev(n, Y, n, k, C + (int64_t)off * k, k, M, YC, n, 0.0, st));
        RC(qd_residual_norms_dev(n, YC, n, Xn + (int64_t)off * n, n, theta + off, M, res, st));
        CUDA_OK(cudaMemcpy2DAsync(Z_dev, sizeof(double2) * ldz, Xn + (int64_t)off * n, sizeof(double2) * n,
                                  sizeof(double2) * n, M, cudaMemcpyDeviceToDevice, st));
        CUDA_OK(cudaMemcpyAsync(w_dev, theta + off, sizeof(double) * M, cudaMemcpyDeviceToDevice, st));
        int hinfo = 0;
        std::vector<double> th_h(k), res_h(M);
        CUDA_OK(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(th_h.data(), theta, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(res_h.data(), res, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
        tm.mark();  // 6
        CUDA_OK(cudaStreamSynchronize(st));
        void *rr_bufs[] = {Y, Xn, YC, S, Ak, C, theta, res, info, Z32};
        for (void *p : rr_bufs) qd_pool_free(p, st);
        if (!hinfo) {
            int brc = window_error_bounds(th_h.data(), k, off, M, res_h.data(), lo2 > 0 || off > 0,
                                          hi2 < n - 1 || off + M < k);
            if (brc) return brc;
        }
        if (hinfo) return qd_set_error(QD_ERR_CONVERGENCE, "Rayleigh-Ritz: Gram matrix not positive definite");
    }
    CUDA_OK(cudaStreamSynchronize(st));
    g_timings[1] = tm.ms(0, 1);
    g_timings[2] = tm.ms(1, 2);
    g_timings[3] = tm.ms(2, 3);
    g_timings[4] = tm.ms(3, 4);
    g_timings[5] = tm.ms(4, 5);
    g_timings[6] = tm.ms(5, 6);
    void *bufs[] = {AB, AB0, d, e2, bounds, lam, progress, err, dmax, gs_d, gz_d, Lw, Uw, ipiv, yw, Zb, H32};
    for (void *p : bufs)
        if (p) qd_pool_free(p, st);
    qd_stage1_free(&w1, st);
    return QD_OK;
}

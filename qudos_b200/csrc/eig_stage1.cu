// Stage 1 of the eigensolver: dense Hermitian -> band (half bandwidth b) by
// blocked Householder reflections, and the matching back-transformation of the
// wanted eigenvectors.  Replaces the zhetrd part of LAPACK zheevr called by
// diagonalise_hamiltonian.c:73.
//
// Panels of b columns are reduced left to right.  For panel k (columns
// k..k+b-1, rows k+b..N-1):
//   * panel_qr_kernel: Householder QR of the tall panel in one cooperative
//     launch.  Each block keeps its slice of rows in shared memory for all b
//     columns.  Per column there is exactly one bounded grid arrival (a
//     counter that only grows): the column norm and the dot products with the
//     remaining columns are formed from the unscaled column
//     (w_c = A[j,c] + conj(s) x^H A_c), accumulated in the pass that applies
//     the previous reflector, double-buffered in global scratch and reduced by
//     whole warps.
//   * T of the compact WY form I - V T V^H from the Gram matrix V^H V (GEMM)
//     and the tau's (form_t_kernel).
//   * delayed trailing update: the two-sided update A22 <- Q^H A22 Q is written
//     as A22 -= V W^H + W V^H with W = X - 1/2 V (T^H V^H X), X = A22 V T.  The
//     (V, W) pairs of up to `agg` columns are accumulated and applied to the
//     trailing matrix in one rank-2*agg update; in between, the next panel's
//     columns and X are corrected for the pending terms with thin GEMMs.
//     FP64: ZHEMM/ZHER2K on the lower triangle.  complex64 (mixed path): the
//     full matrix; X and the rank-2*agg update run in the tcgen05 3xTF32
//     kernels of tc_gemm.cu, the thin products in cuBLAS CGEMM.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "eig_common.cuh"
#include "qd_internal.h"

// Polls before a panel's grid-barrier wait gives up (set at run time by
// qd_set_wait_limits; the default is about three seconds of polling).
#define QD_BAR_LIMIT_DEFAULT (1LL << 26)
__device__ long long g_bar_limit = QD_BAR_LIMIT_DEFAULT;

// ---------------------------------------------------------------------------
// panel QR
// ---------------------------------------------------------------------------
// Partial sums of column jj over this block's rows r > jj: slot 0 = |x|^2, slot
// c (> jj) = x^H A_c.  The owner of row jj publishes that row (columns >= jj).
template <typename R>
__device__ void panel_partials(const cpx<R> *tile, int chunk, int r0, int rows, int nb, int jj, double2 *red_blk,
                               double2 *rowbuf) {  // nb = number of panel columns
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int slot = w; slot < nb - jj; slot += nw) {
        int c = slot == 0 ? jj : jj + slot;
        double sr = 0.0, si = 0.0;
        for (int rr = lane; rr < rows; rr += 32) {
            if (r0 + rr <= jj) continue;
            cpx<R> x = tile[jj * chunk + rr];
            if (slot == 0) {
                sr += (double)x.re * x.re + (double)x.im * x.im;
            } else {
                cpx<R> a = tile[c * chunk + rr];
                sr += (double)x.re * a.re + (double)x.im * a.im;
                si += (double)x.re * a.im - (double)x.im * a.re;
            }
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) __stcg(&red_blk[slot == 0 ? 0 : c], make_double2(sr, si));
    }
    if (jj >= r0 && jj < r0 + rows) {
        int rr = jj - r0;
        for (int c = jj + threadIdx.x; c < nb; c += blockDim.x) {
            cpx<R> a = tile[c * chunk + rr];
            __stcg(&rowbuf[c], make_double2((double)a.re, (double)a.im));
        }
    }
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide arrival on a counter that only grows (zeroed by the host before the
// launch): barrier number j completes when the counter reaches (j + 1) * G.  The
// block barrier plus the release add publish every thread's prior stores; the
// acquire poll is bounded.
__device__ __forceinline__ bool grid_arrive_wait(unsigned *ctr, unsigned target, int *err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        asm volatile("fence.acq_rel.gpu;\n\tred.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(ctr) : "memory");
        long long it = 0;
        const long long limit = g_bar_limit;
        while (ld_acquire_u32(ctr) < target) {
            if (++it > limit || *(volatile int *)err) {
                atomicExch(err, 6);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
    }
    __syncthreads();
    return ok != 0;
}

// Panel QR.  Per reflector j: one grid arrival, then every block reduces the
// column's partial sums, forms the Householder scalars and updates its rows.
// The update does column j+1 first; the remaining columns are updated in one
// pass that also accumulates column j+1's partial sums for the next reflector
// (warps over columns, lanes over rows: no index division).
template <typename R>
__global__ void __launch_bounds__(256) panel_qr_kernel(cpx<R> *A, int64_t lda, int m, int nb, int nref, int chunk,
                                                       cpx<R> *Rout, cpx<R> *tau_out, double2 *red,
                                                       double2 *rowbuf, unsigned *bar, int *err) {
    // nb panel columns, nref = min(m, nb) reflectors (a short panel still spans all nb columns)
    extern __shared__ unsigned char smem_raw[];
    cpx<R> *tile = (cpx<R> *)smem_raw;  // [nb][chunk]
    __shared__ double2 s_red[64];
    __shared__ double2 s_w[64];
    __shared__ double2 s_row[64];  // row j of the panel, columns j ..
    __shared__ double s_beta;
    __shared__ double2 s_tau, s_scale;
    const unsigned G = gridDim.x;
    const int r0 = blockIdx.x * chunk;
    const int rows = max(0, min(m, r0 + chunk) - r0);
    const int stride = nb + 1;  // double2 slots per block per buffer
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int c = w; c < nb; c += nw)
        for (int rr = lane; rr < rows; rr += 32) tile[c * chunk + rr] = A[(int64_t)(r0 + rr) + (int64_t)c * lda];
    __syncthreads();
    panel_partials<R>(tile, chunk, r0, rows, nb, 0, red + (size_t)blockIdx.x * stride, rowbuf);
    for (int j = 0; j < nref; j++) {
        const int buf = j & 1;
        double2 *redb = red + (size_t)buf * G * stride;
        double2 *rowb = rowbuf + (size_t)buf * nb;
        if (!grid_arrive_wait(bar, (unsigned)(j + 1) * G, err)) return;
        // ---- reduce the partials of column j over all blocks (one warp per value);
        //      row j is fetched in the same round trip
        const double2 rv = (int)threadIdx.x < nb - j ? __ldcg(&rowb[j + threadIdx.x]) : make_double2(0.0, 0.0);
        for (int slot = w; slot < nb - j; slot += nw) {
            int sidx = slot == 0 ? 0 : j + slot;
            double sr = 0.0, si = 0.0;
            for (unsigned q = lane; q < G; q += 32) {
                double2 v = __ldcg(&redb[(size_t)q * stride + sidx]);
                sr += v.x;
                si += v.y;
            }
            sr = warp_sum(sr);
            si = warp_sum(si);
            if (lane == 0) s_red[slot] = make_double2(sr, si);
        }
        if ((int)threadIdx.x < nb - j) s_row[threadIdx.x] = rv;
        __syncthreads();
        // ---- Householder scalars (LAPACK zlarfg conventions)
        if (threadIdx.x == 0) {
            double sig = s_red[0].x;
            double2 a = s_row[0];
            double ar = a.x, ai = a.y;
            if (sig == 0.0 && ai == 0.0) {
                s_tau = make_double2(0.0, 0.0);
                s_beta = ar;
                s_scale = make_double2(0.0, 0.0);
            } else {
                double beta = -copysign(sqrt(ar * ar + ai * ai + sig), ar);
                s_beta = beta;
                s_tau = make_double2((beta - ar) / beta, -ai / beta);
                double dr = ar - beta, di = ai, den = dr * dr + di * di;
                s_scale = make_double2(dr / den, -di / den);  // 1 / (alpha - beta)
            }
        }
        __syncthreads();
        // ---- w_c = A[j,c] + conj(scale) (x^H A_c);  s_w = conj(tau) w_c
        for (int c = j + 1 + threadIdx.x; c < nb; c += blockDim.x) {
            double2 a = s_row[c - j];
            double2 d = s_red[c - j];
            double sr = s_scale.x, si = -s_scale.y;  // conj(scale)
            double wr = a.x + sr * d.x - si * d.y, wi = a.y + sr * d.y + si * d.x;
            double tr = s_tau.x, ti = -s_tau.y;      // conj(tau)
            s_w[c] = make_double2(tr * wr - ti * wi, tr * wi + ti * wr);
        }
        __syncthreads();
        // ---- A[r, c] -= v_r s_w[c] for r >= j, c > j  (v_j = 1, v_r = scale x_r for r > j)
        const cpx<R> scale = mk<R>((R)s_scale.x, (R)s_scale.y);
        const bool nextp = j + 1 < nref;
        if (j + 1 < nb) {
            const cpx<R> tw = mk<R>((R)s_w[j + 1].x, (R)s_w[j + 1].y);
            for (int rr = threadIdx.x; rr < rows; rr += blockDim.x) {
                const int r = r0 + rr;
                if (r < j) continue;
                cpx<R> v = (r == j) ? mk<R>(1, 0) : cmul(tile[j * chunk + rr], scale);
                tile[(j + 1) * chunk + rr] = csub(tile[(j + 1) * chunk + rr], cmul(v, tw));
            }
        }
        __syncthreads();
        double2 *redn = red + (size_t)((j + 1) & 1) * G * stride + (size_t)blockIdx.x * stride;
        for (int c = j + 1 + w; c < nb; c += nw) {
            const bool upd = c > j + 1;
            const cpx<R> tw = upd ? mk<R>((R)s_w[c].x, (R)s_w[c].y) : mk<R>(0, 0);
            double sr = 0.0, si = 0.0;
            for (int rr = lane; rr < rows; rr += 32) {
                const int r = r0 + rr;
                cpx<R> a = tile[c * chunk + rr];
                if (upd && r >= j) {
                    cpx<R> v = (r == j) ? mk<R>(1, 0) : cmul(tile[j * chunk + rr], scale);
                    a = csub(a, cmul(v, tw));
                    tile[c * chunk + rr] = a;
                }
                if (nextp && r > j + 1) {
                    cpx<R> x = tile[(j + 1) * chunk + rr];
                    if (!upd) {
                        sr += (double)x.re * x.re + (double)x.im * x.im;
                    } else {
                        sr += (double)x.re * a.re + (double)x.im * a.im;
                        si += (double)x.re * a.im - (double)x.im * a.re;
                    }
                }
            }
            if (nextp) {
                sr = warp_sum(sr);
                si = warp_sum(si);
                if (lane == 0) __stcg(&redn[upd ? c : 0], make_double2(sr, si));
            }
        }
        __syncthreads();
        // ---- column j becomes v (explicit); row j of R is final; row j+1 is published
        for (int rr = threadIdx.x; rr < rows; rr += blockDim.x)
            if (r0 + rr > j) tile[j * chunk + rr] = cmul(tile[j * chunk + rr], scale);
        if (j >= r0 && j < r0 + rows) {
            int rr = j - r0;
            for (int c = j + threadIdx.x; c < nb; c += blockDim.x) {
                cpx<R> val = (c == j) ? mk<R>((R)s_beta, 0) : tile[c * chunk + rr];
                Rout[j + (int64_t)c * nb] = val;
                tile[c * chunk + rr] = (c == j) ? mk<R>(1, 0) : mk<R>(0, 0);
            }
            if (threadIdx.x == 0) tau_out[j] = mk<R>((R)s_tau.x, (R)s_tau.y);
        }
        if (nextp && j + 1 >= r0 && j + 1 < r0 + rows) {
            int rr = j + 1 - r0;
            double2 *rown = rowbuf + (size_t)((j + 1) & 1) * nb;
            for (int c = j + 1 + threadIdx.x; c < nb; c += blockDim.x) {
                cpx<R> a = tile[c * chunk + rr];
                __stcg(&rown[c], make_double2((double)a.re, (double)a.im));
            }
        }
    }
    __syncthreads();
    for (int c = w; c < nref; c += nw)
        for (int rr = lane; rr < rows; rr += 32) {
            const int r = r0 + rr;
            cpx<R> v = tile[c * chunk + rr];
            if (r < c) v = mk<R>(0, 0);
            A[(int64_t)r + (int64_t)c * lda] = v;
        }
}

// T of the compact WY form (LAPACK zlarft, forward, columnwise):
// T[i,i] = tau_i, T[0:i, i] = -tau_i T[0:i, 0:i] (V^H V)[0:i, i].  One block of
// nb <= 32 warps; the Gram matrix is staged in shared memory first (dynamic:
// 2 nb^2 double2).  Column i depends on the columns before it, so the columns
// are formed in order, but each entry T[p, i] of a column is one warp's
// shuffle-reduced dot product over q in [p, i), so a column costs one reduction
// and one block barrier instead of a serial loop per thread.
template <typename R>
__global__ void form_t_kernel(const cpx<R> *gram, int ldg, const cpx<R> *tau, cpx<R> *T, int ldt, int nb) {
    extern __shared__ double2 ft_smem[];
    double2 *Tl = ft_smem;            // nb x nb
    double2 *Gs = ft_smem + nb * nb;  // nb x nb
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        int p = idx % nb, q = idx / nb;
        Tl[idx] = p == q ? make_double2((double)tau[p].re, (double)tau[p].im) : make_double2(0.0, 0.0);
        cpx<R> g = gram[p + (int64_t)q * ldg];
        Gs[idx] = make_double2((double)g.re, (double)g.im);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = 1; i < nb; i++) {
        if (w < i) {  // entry p = w of column i
            const int p = w;
            const int q = p + lane;
            double sr = 0.0, si = 0.0;
            if (q < i) {
                const double2 a = Tl[p + q * nb], g = Gs[q + i * nb];
                sr = a.x * g.x - a.y * g.y;
                si = a.x * g.y + a.y * g.x;
            }
            for (int o = 16; o > 0; o >>= 1) {
                sr += __shfl_xor_sync(0xffffffffu, sr, o);
                si += __shfl_xor_sync(0xffffffffu, si, o);
            }
            if (lane == 0) {
                const double2 t = Tl[i + i * nb];
                Tl[p + i * nb] = make_double2(-(t.x * sr - t.y * si), -(t.x * si + t.y * sr));
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        int p = idx % nb, q = idx / nb;
        T[p + (int64_t)q * ldt] = mk<R>((R)Tl[idx].x, (R)Tl[idx].y);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
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

extern "C" int qd_stage1_set_wait_limit(long long polls) {
    const long long v = polls < 0 ? QD_BAR_LIMIT_DEFAULT : polls;
    CUDA_OK(cudaMemcpyToSymbol(g_bar_limit, &v, sizeof(v)));
    return QD_OK;
}

static int n_panels(int64_t n, int b) {
    int c = 0;
    for (int64_t k = 0; k + b < n; k += b) c++;
    return c;
}

extern "C" cublasHandle_t qd_cublas(void);
extern "C" int qd_mixed_gemm_mode(void);
extern "C" int qd_tsmm_nn(int fp32, int m, int nc, int nterms, const void *const *A, const int64_t *lda,
                          const void *const *B, const int64_t *ldb, const int *K, const int *btrans,
                          const double *alpha, void *C, int64_t ldc, double beta, void *stream);
extern "C" int qd_tsmm_cn(int fp32, int m, const void *A, int64_t lda, int k1, const void *B, int64_t ldb, int nc,
                          void *C, int64_t ldc, void *scratch, size_t scratch_bytes, void *stream);
extern "C" int qd_small_cn(int fp32, int k, int n1, int n2, const void *A, int lda, const void *B, int ldb,
                           double alpha, void *C, int ldc, void *stream);
extern "C" size_t qd_tsmm_cn_scratch_bytes(int m, int k1, int nc, int elem_bytes);

// One- or two-term tall product C[m x nc] = beta C + sum alpha_t A_t op(B_t),
// up to 64 output columns per launch.
template <typename T>
static int nn(cudaStream_t st, int m, int nc, const T *A0, int64_t lda0, const T *B0, int64_t ldb0, int K0, int bt0,
              double al0, T *C, int64_t ldc, double beta, const T *A1 = nullptr, int64_t lda1 = 0,
              const T *B1 = nullptr, int64_t ldb1 = 0, int K1 = 0, int bt1 = 0, double al1 = 0.0) {
    const void *A[2] = {A0, A1}, *B[2] = {B0, B1};
    int64_t la[2] = {lda0, lda1}, lb[2] = {ldb0, ldb1};
    int K[2] = {K0, K1}, bt[2] = {bt0, bt1};
    double al[2] = {al0, al1};
    const int fp32 = sizeof(T) == 8;
    for (int c0 = 0; c0 < nc; c0 += 64) {
        const int w = nc - c0 < 64 ? nc - c0 : 64;
        const void *Bc[2];
        for (int t = 0; t < 2; t++)
            Bc[t] = B[t] ? (const void *)((const T *)B[t] + (bt[t] ? c0 : c0 * lb[t])) : nullptr;
        int rc = qd_tsmm_nn(fp32, m, w, A1 ? 2 : 1, A, la, Bc, lb, K, bt, al, C + c0 * ldc, ldc, beta, st);
        if (rc) return rc;
    }
    return QD_OK;
}
// C[k1 x nc] = A[m x k1]^H B[m x nc] (k1 <= 256): 64 output columns per launch
// when k1 <= 64, else 32.  part holds part_bytes of partial sums.
template <typename T>
static int cn(cudaStream_t st, int m, const T *A, int64_t lda, int k1, const T *B, int64_t ldb, int nc, T *C,
              int64_t ldc, void *part, size_t part_bytes) {
    const int fp32 = sizeof(T) == 8;
    const int cw = k1 <= 64 ? 64 : 32;
    for (int c0 = 0; c0 < nc; c0 += cw) {
        const int w = nc - c0 < cw ? nc - c0 : cw;
        int rc = qd_tsmm_cn(fp32, m, A, lda, k1, B + c0 * ldb, ldb, w, C + c0 * ldc, ldc, part, part_bytes, st);
        if (rc) return rc;
    }
    return QD_OK;
}
extern "C" int qd_tc_work_alloc_on(int64_t n, int kmax, QdTcWork **out, cudaStream_t st);
extern "C" void qd_tc_work_free_on(QdTcWork *w, cudaStream_t st);


// typed cuBLAS wrappers --------------------------------------------------------
template <typename T> struct Blas;
template <> struct Blas<cuDoubleComplex> {
    typedef double R;
    static cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k,
                               const cuDoubleComplex *al, const cuDoubleComplex *A, int64_t lda,
                               const cuDoubleComplex *B, int64_t ldb, const cuDoubleComplex *be, cuDoubleComplex *C,
                               int64_t ldc) {
        return cublasZgemm(h, a, b, m, n, k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
    }
    // big products (X = A22 V T; trailing updates): FP64 tensor cores through cuBLAS
    static cublasStatus_t big(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k,
                              const cuDoubleComplex *al, const cuDoubleComplex *A, int64_t lda,
                              const cuDoubleComplex *B, int64_t ldb, const cuDoubleComplex *be, cuDoubleComplex *C,
                              int64_t ldc) {
        return gemm(h, a, b, m, n, k, al, A, lda, B, ldb, be, C, ldc);
    }
};
template <> struct Blas<cuComplex> {
    typedef float R;
    static cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k,
                               const cuComplex *al, const cuComplex *A, int64_t lda, const cuComplex *B, int64_t ldb,
                               const cuComplex *be, cuComplex *C, int64_t ldc) {
        return cublasCgemm(h, a, b, m, n, k, al, A, (int)lda, B, (int)ldb, be, C, (int)ldc);
    }
    static cublasStatus_t big(cublasHandle_t h, cublasOperation_t a, cublasOperation_t b, int m, int n, int k,
                              const cuComplex *al, const cuComplex *A, int64_t lda, const cuComplex *B, int64_t ldb,
                              const cuComplex *be, cuComplex *C, int64_t ldc) {
        int mode = qd_mixed_gemm_mode();
        cublasComputeType_t ct = mode == 2 ? CUBLAS_COMPUTE_32F_EMULATED_16BFX9
                                 : mode == 1 ? CUBLAS_COMPUTE_32F_FAST_TF32
                                             : CUBLAS_COMPUTE_32F;
        cublasStatus_t s = cublasGemmEx(h, a, b, m, n, k, al, A, CUDA_C_32F, (int)lda, B, CUDA_C_32F, (int)ldb, be, C,
                                        CUDA_C_32F, (int)ldc, ct, CUBLAS_GEMM_DEFAULT);
        if (s != CUBLAS_STATUS_SUCCESS && mode != 0)
            s = cublasGemmEx(h, a, b, m, n, k, al, A, CUDA_C_32F, (int)lda, B, CUDA_C_32F, (int)ldb, be, C, CUDA_C_32F,
                             (int)ldc, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
        return s;
    }
};

template <typename T>
static T cval(double re, double im) {
    T z;
    z.x = (typename Blas<T>::R)re;
    z.y = (typename Blas<T>::R)im;
    return z;
}

template <typename T>
static int launch_panel(T *P, int64_t lda, int m, int nb, int nref, T *Rp, T *taup, Stage1Work &w, cudaStream_t st) {
    typedef typename Blas<T>::R R;
    static int nsm = 0;
    if (!nsm) {
        int dev;
        CUDA_OK(cudaGetDevice(&dev));
        CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    }
    int G = (m + 63) / 64;
    if (G > qd_sm_budget(nsm)) G = qd_sm_budget(nsm);
    if (G < 1) G = 1;
    int chunk = (m + G - 1) / G;
    size_t smem = (size_t)chunk * nb * sizeof(cpx<R>);
    if (smem > 200 * 1024) return qd_set_error(QD_ERR_UNSUPPORTED, "panel slice too large (%d rows)", chunk);
    static int configured[2] = {0, 0};
    int ti = sizeof(R) == 8 ? 0 : 1;
    if (!configured[ti]) {
        CUDA_OK(cudaFuncSetAttribute(panel_qr_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        configured[ti] = 1;
    }
    CUDA_OK(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), st));
    cpx<R> *Pp = (cpx<R> *)P, *Rpp = (cpx<R> *)Rp, *tp = (cpx<R> *)taup;
    void *args[] = {&Pp, &lda, &m, &nb, &nref, &chunk, &Rpp, &tp, &w.red, &w.rowbuf, &w.bar, &w.err};
    qd_count_launch(1);
    CUDA_OK(cudaLaunchCooperativeKernel((void *)panel_qr_kernel<R>, dim3(G), dim3(256), args, smem, st));
    return QD_OK;
}

// Stage 1 for element type T (cuDoubleComplex: lower triangle; cuComplex: full matrix).
// Opt-in breakdown of the reduction (QD_PROFILE=1): events recorded at the
// boundaries of the steps of every panel, summed per step after the stage.
// Steps: 0 panel refresh, 1 panel QR, 2 T and VT, 3 X = A22 VT,
// 4 pending-update corrections, 5 W, 6 append, 7 trailing update.
namespace {
struct StageProfile {
    int on = -1;
    std::vector<cudaEvent_t> ev;
    std::vector<int> step;
    int used = 0;
    double ms[8] = {0};
};
thread_local StageProfile g_prof;
void prof_mark(int stepid, cudaStream_t st) {
    if (g_prof.on < 0) {
        const char *e = getenv("QD_PROFILE");
        g_prof.on = e && atoi(e) > 0;
    }
    if (!g_prof.on) return;
    if (g_prof.used == (int)g_prof.ev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        g_prof.ev.push_back(e);
        g_prof.step.push_back(0);
    }
    cudaEventRecord(g_prof.ev[g_prof.used], st);
    g_prof.step[g_prof.used++] = stepid;
}
void prof_collect(cudaStream_t st) {
    if (g_prof.on <= 0) return;
    prof_mark(-1, st);
    cudaStreamSynchronize(st);
    for (int i = 0; i < 8; i++) g_prof.ms[i] = 0;
    for (int i = 0; i + 1 < g_prof.used; i++) {
        float t = 0;
        cudaEventElapsedTime(&t, g_prof.ev[i], g_prof.ev[i + 1]);
        if (g_prof.step[i] >= 0) g_prof.ms[g_prof.step[i]] += t;
    }
    g_prof.used = 0;
}
}  // namespace

// Per-step times (ms) of the last dense->band reduction when QD_PROFILE=1.
extern "C" int qd_stage1_profile(double *ms, int n) {
    for (int i = 0; i < n && i < 8; i++) ms[i] = g_prof.ms[i];
    return QD_OK;
}

template <typename T>
static int stage1(T *A, int64_t n, int64_t lda, int b, Stage1Work &w, cudaStream_t st) {
    typedef typename Blas<T>::R R;
    const bool full = sizeof(R) == 4;
    cublasHandle_t h = qd_cublas();
    BLAS_OK(cublasSetStream(h, st ? st : cudaStreamPerThread));
    const T one = cval<T>(1, 0), zero = cval<T>(0, 0), mone = cval<T>(-1, 0);
    const cublasOperation_t N_ = CUBLAS_OP_N, C_ = CUBLAS_OP_C;
    T *Vacc = (T *)w.Vacc, *Wacc = (T *)w.Wacc;
    const int64_t ldv = w.ldv;
    int64_t k0 = 0;  // start row/column of the current aggregation window
    int K = 0;       // accumulated reflector columns
    int p = 0;
    for (int64_t k = 0; k + b < n; k += b, p++) {
        int m = (int)(n - k - b), nb = b < m ? b : m;
        int64_t off = k - k0;
        T *Tp = (T *)w.Tall + (int64_t)p * b * b;
        T *Rp = (T *)w.Rall + (int64_t)p * b * b;
        T *Pcol = A + k + k * lda;  // rows k.., columns k..k+nb-1
        // 1. bring the panel's b columns up to date with the pending (V, W) terms
        prof_mark(0, st);
        if (K > 0)  // P -= V Wb^H + W Vb^H
            RC(nn<T>(st, (int)(n - k), b, Vacc + off, ldv, Wacc + off, ldv, K, 1, -1.0, Pcol, lda, 1.0, Wacc + off,
                     ldv, Vacc + off, ldv, K, 1, -1.0));
        // 2. panel QR -> V (explicit, in place), tau, R; nb = min(b, m) reflectors over all b columns
        T *P = A + (k + b) + k * lda;
        prof_mark(1, st);
        CUDA_OK(cudaMemsetAsync(Rp, 0, sizeof(T) * b * b, st));
        RC(launch_panel<T>(P, lda, m, b, nb, Rp, (T *)w.tau, w, st));
        // 3. T from the Gram matrix
        prof_mark(2, st);
        RC(cn<T>(st, m, P, lda, nb, P, lda, nb, (T *)w.gram, b, w.part, w.part_bytes));
        qd_count_launch(1);
        {
            static int ft_configured[2] = {0, 0};
            const int ti = sizeof(R) == 8 ? 0 : 1;
            if (!ft_configured[ti]) {  // nb <= 48: up to 72 KB
                CUDA_OK(cudaFuncSetAttribute(form_t_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             2 * 48 * 48 * (int)sizeof(double2)));
                ft_configured[ti] = 1;
            }
        }
        form_t_kernel<R><<<1, 32 * nb, 2 * nb * nb * sizeof(double2), st>>>((const cpx<R> *)w.gram, b,
                                                                        (const cpx<R> *)w.tau, (cpx<R> *)Tp, b, nb);
        CUDA_OK(cudaGetLastError());
        // 4. VT = V T ; 5. X = A22 VT (stale A22 + pending terms), written straight into Wacc
        T *VT = (T *)w.VT;
        T *X = Wacc + (off + b) + (int64_t)K * ldv;
        T *A22 = A + (k + b) + (k + b) * lda;
        RC(nn<T>(st, m, nb, P, lda, Tp, b, nb, 0, 1.0, VT, m, 0.0));
        prof_mark(3, st);
        if (full && w.tc) {
            RC(qd_tc_xprod(A, lda, n, k + b, m, VT, m, nb, X, ldv, w.tc, st));
        } else if (full) {
            BLAS_OK(Blas<T>::big(h, N_, N_, m, nb, m, &one, A22, lda, VT, m, &zero, X, ldv));
        } else {
            BLAS_OK(cublasZhemm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, m, nb, (const cuDoubleComplex *)&one,
                                (const cuDoubleComplex *)A22, (int)lda, (const cuDoubleComplex *)VT, m,
                                (const cuDoubleComplex *)&zero, (cuDoubleComplex *)X, (int)ldv));
        }
        prof_mark(4, st);
        if (K > 0) {
            T *S1 = (T *)w.S1, *S2 = (T *)w.S2;
            RC(cn<T>(st, m, Wacc + off + b, ldv, K, VT, m, nb, S1, w.agg, w.part, w.part_bytes));
            RC(cn<T>(st, m, Vacc + off + b, ldv, K, VT, m, nb, S2, w.agg, w.part, w.part_bytes));
            RC(nn<T>(st, m, nb, Vacc + off + b, ldv, S1, w.agg, K, 0, -1.0, X, ldv, 1.0, Wacc + off + b, ldv, S2,
                     w.agg, K, 0, -1.0));
        }
        // 6. W = X - 1/2 V (T^H V^H X)
        prof_mark(5, st);
        RC(cn<T>(st, m, P, lda, nb, X, ldv, nb, (T *)w.M, b, w.part, w.part_bytes));
        RC(qd_small_cn(sizeof(T) == 8, nb, nb, nb, Tp, b, w.M, b, 1.0, w.Y, b, st));
        RC(nn<T>(st, m, nb, P, lda, (T *)w.Y, b, nb, 0, -0.5, X, ldv, 1.0));
        // 7. append V (zero above its first row) to Vacc; W already sits in Wacc
        prof_mark(6, st);
        CUDA_OK(cudaMemset2DAsync(Vacc + (int64_t)K * ldv, sizeof(T) * ldv, 0, sizeof(T) * (off + b), nb, st));
        CUDA_OK(cudaMemset2DAsync(Wacc + (int64_t)K * ldv, sizeof(T) * ldv, 0, sizeof(T) * (off + b), nb, st));
        CUDA_OK(cudaMemcpy2DAsync(Vacc + (off + b) + (int64_t)K * ldv, sizeof(T) * ldv, P, sizeof(T) * lda,
                                  sizeof(T) * m, nb, cudaMemcpyDeviceToDevice, st));
        K += nb;
        // 8. flush: trailing matrix from the next panel on
        int64_t kn = k + b;
        bool last = !(kn + b < n);
        if (K + b > w.agg || last) {
            prof_mark(7, st);
            int mt = (int)(n - kn);
            int64_t offn = kn - k0;
            T *At = A + kn + kn * lda;
            if (full && w.tc) {
                RC(qd_tc_flush(A, lda, kn, mt, Vacc, Wacc, ldv, offn, K, w.tc, st));
            } else if (full) {
                BLAS_OK(Blas<T>::big(h, N_, C_, mt, mt, K, &mone, Vacc + offn, ldv, Wacc + offn, ldv, &one, At, lda));
                BLAS_OK(Blas<T>::big(h, N_, C_, mt, mt, K, &mone, Wacc + offn, ldv, Vacc + offn, ldv, &one, At, lda));
            } else {
                const double done = 1.0;
                BLAS_OK(cublasZher2k(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, mt, K, (const cuDoubleComplex *)&mone,
                                     (const cuDoubleComplex *)(Vacc + offn), (int)ldv,
                                     (const cuDoubleComplex *)(Wacc + offn), (int)ldv, &done, (cuDoubleComplex *)At,
                                     (int)lda));
            }
            k0 = kn;
            K = 0;
        }
    }
    prof_collect(st);
    return QD_OK;
}

// Tuning table of the aggregation depth (columns of the rank-2K update per
// flush), per element size (8: mixed path, 16: FP64) and matrix-size bound;
// written by qd_tuning_set (the package's autotuner fills it from its cache).
namespace {
constexpr int TUNE_MAX = 64;
struct TuneEntry {
    int64_t n_max;
    int elem_bytes, agg;
};
TuneEntry g_tune[TUNE_MAX];
int g_ntune = 0;
}  // namespace

// Adds (or replaces) the aggregation depth for matrices of order <= n_h_max
// solved in precision prec; n_h_max <= 0 clears the table.  Call before the
// solves that should use it (the table is read when a solve sets up).
extern "C" int qd_tuning_set(int prec, int64_t n_h_max, int agg) {
    if (n_h_max <= 0) {
        g_ntune = 0;
        return QD_OK;
    }
    if (prec != QD_PREC_FP64 && prec != QD_PREC_MIXED) return qd_set_error(QD_ERR_ARG, "qd_tuning_set: precision");
    if (agg < 32 || agg > 256 || agg % 32) return qd_set_error(QD_ERR_ARG, "qd_tuning_set: depth %d (32..256, multiple of 32)", agg);
    const int eb = prec == QD_PREC_MIXED ? 8 : 16;
    for (int i = 0; i < g_ntune; i++)
        if (g_tune[i].n_max == n_h_max && g_tune[i].elem_bytes == eb) {
            g_tune[i].agg = agg;
            return QD_OK;
        }
    if (g_ntune == TUNE_MAX) return qd_set_error(QD_ERR_ARG, "qd_tuning_set: table full");
    g_tune[g_ntune++] = {n_h_max, eb, agg};
    return QD_OK;
}

// Depth for an order-n solve: the entry with the smallest bound >= n, else
// QD_AGG from the environment, else 256.
static int tuned_agg(int64_t n, int elem_bytes) {
    int best = -1;
    for (int i = 0; i < g_ntune; i++)
        if (g_tune[i].elem_bytes == elem_bytes && g_tune[i].n_max >= n &&
            (best < 0 || g_tune[i].n_max < g_tune[best].n_max))
            best = i;
    if (best >= 0) return g_tune[best].agg;
    const char *s = getenv("QD_AGG");
    return s ? atoi(s) : 256;
}

extern "C" int qd_stage1_alloc(int64_t n, int b, int elem_bytes, Stage1Work *w, cudaStream_t st) {
    w->tc = nullptr;
    w->npanels = n_panels(n, b);
    int agg = tuned_agg(n, elem_bytes);
    if (agg < b) agg = b;
    agg = (agg / b) * b;
    w->agg = agg;
    w->ldv = n;
    size_t eb = (size_t)elem_bytes;
    void **bufs[] = {&w->VT, &w->X, &w->M, &w->Y, &w->Tall, &w->Rall, &w->Vacc, &w->Wacc, &w->S1, &w->S2, &w->gram,
                     &w->tau, &w->part};
    size_t sizes[] = {eb * n * b, eb * 16, eb * b * b, eb * b * b, eb * (size_t)(w->npanels + 1) * b * b,
                      eb * (size_t)(w->npanels + 1) * b * b, eb * n * agg, eb * n * agg, eb * agg * b,
                      eb * agg * b, eb * b * b, eb * b, qd_tsmm_cn_scratch_bytes((int)n, agg, 32, (int)eb)};
    w->part_bytes = sizes[12];
    for (size_t i = 0; i < sizeof(sizes) / sizeof(sizes[0]); i++)
        if (qd_pool_alloc(bufs[i], sizes[i], st) != 0) return qd_set_error(QD_ERR_NOMEM, "stage-1 workspace");
    int dev, nsm;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (qd_pool_alloc((void **)&w->red, sizeof(double2) * 2 * (size_t)nsm * (b + 1), st) != 0 ||
        qd_pool_alloc((void **)&w->rowbuf, sizeof(double2) * 2 * (size_t)b, st) != 0 ||
        qd_pool_alloc((void **)&w->bar, 4 * sizeof(unsigned), st) != 0 ||
        qd_pool_alloc((void **)&w->err, sizeof(int), st) != 0)
        return qd_set_error(QD_ERR_NOMEM, "stage-1 scratch allocation failed");
    CUDA_OK(cudaMemsetAsync(w->err, 0, sizeof(int), st));
    w->tc = nullptr;
    if (elem_bytes == 8 && qd_mixed_gemm_mode() == 3 && (b % 2) == 0 && (n % 2) == 0) {
        int rc = qd_tc_work_alloc_on(n, agg, &w->tc, st);
        if (rc) return rc;
    }
    return QD_OK;
}

extern "C" void qd_stage1_free(Stage1Work *w, cudaStream_t st) {
    void *p[] = {w->VT, w->X, w->M, w->Y, w->Tall, w->Rall, w->Vacc, w->Wacc, w->S1, w->S2, w->gram, w->tau,
                 w->part, w->red, w->rowbuf, w->bar, w->err};
    for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); i++) qd_pool_free(p[i], st);
    if (w->tc) qd_tc_work_free_on(w->tc, st);
    w->tc = nullptr;
}

extern "C" int qd_stage1_run(void *A, int64_t n, int64_t lda, int b, int fp32, Stage1Work *w, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (b > 32) return qd_set_error(QD_ERR_UNSUPPORTED, "band width above 32");
    int rc = fp32 ? stage1<cuComplex>((cuComplex *)A, n, lda, b, *w, st)
                  : stage1<cuDoubleComplex>((cuDoubleComplex *)A, n, lda, b, *w, st);
    if (rc) return rc;
    int herr = 0;
    CUDA_OK(cudaMemcpyAsync(&herr, w->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (herr) return qd_set_error(QD_ERR_TIMEOUT, "panel factorisation: grid barrier wait ran out");
    if (w->tc) return qd_tc_work_check(w->tc);
    return QD_OK;
}

// Band extraction: AB[d + j*ldb] = A(j+d, j) for 0 <= d <= b, zero for b < d < ldb.
// Diagonal blocks come from A, the blocks below the diagonal from the panels' R.
template <typename R>
__global__ void extract_band_kernel(const cpx<R> *A, int64_t lda, int64_t n, int b, const cpx<R> *Rall, double2 *AB,
                                    int ldb) {
    int64_t j = blockIdx.x;
    if (j >= n) return;
    int64_t k = (j / b) * b;  // block start
    for (int d = threadIdx.x; d < ldb; d += blockDim.x) {
        int64_t i = j + d;
        double2 v = make_double2(0.0, 0.0);
        if (i < n && d <= b) {
            if (i < k + b) {
                cpx<R> a = A[i + j * lda];
                v = make_double2((double)a.re, (double)a.im);
            } else {
                int64_t pr = i - (k + b), pc = j - k;
                int64_t p = k / b;
                if (pr <= pc && k + b < n) {
                    cpx<R> a = Rall[p * (int64_t)b * b + pr + pc * b];
                    v = make_double2((double)a.re, (double)a.im);
                }
            }
            if (d == 0) v.y = 0.0;
        }
        AB[d + j * (int64_t)ldb] = v;
    }
}

extern "C" int qd_extract_band(const void *A, int64_t n, int64_t lda, int b, int fp32, const Stage1Work *w,
                               double2 *AB, int ldb, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    qd_count_launch(1);
    if (fp32)
        extract_band_kernel<float><<<(unsigned)n, 64, 0, st>>>((const cpx<float> *)A, lda, n, b,
                                                               (const cpx<float> *)w->Rall, AB, ldb);
    else
        extract_band_kernel<double><<<(unsigned)n, 64, 0, st>>>((const cpx<double> *)A, lda, n, b,
                                                                (const cpx<double> *)w->Rall, AB, ldb);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// Back-transformation Z <- Q1 Z, panels in reverse order:
// Z[k+b:, :] -= V (T (V^H Z[k+b:, :])).  Z is n x mz (ldz), same precision as A.
template <typename T>
static int backtransform(const T *A, int64_t n, int64_t lda, int b, const Stage1Work *w, T *Z, int64_t ldz, int mz,
                         cudaStream_t st) {
    for (int p = w->npanels - 1; p >= 0; p--) {
        int64_t k = (int64_t)p * b;
        int m = (int)(n - k - b), nb = b < m ? b : m;
        const T *V = A + (k + b) + k * lda;
        const T *Tm = (const T *)w->Tall + (int64_t)p * b * b;
        T *Zs = Z + (k + b);
        T *M = (T *)w->VT, *Y = (T *)w->Vacc;
        RC(cn<T>(st, m, V, lda, nb, Zs, ldz, mz, M, nb, w->part, w->part_bytes));     // M = V^H Z
        RC(nn<T>(st, nb, mz, Tm, b, M, nb, nb, 0, 1.0, Y, nb, 0.0));    // Y = T M
        RC(nn<T>(st, m, mz, V, lda, Y, nb, nb, 0, -1.0, Zs, ldz, 1.0));  // Z -= V Y
    }
    return QD_OK;
}

extern "C" int qd_stage1_backtransform(const void *A, int64_t n, int64_t lda, int b, int fp32, const Stage1Work *w,
                                       void *Z, int64_t ldz, int mz, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (fp32) return backtransform<cuComplex>((const cuComplex *)A, n, lda, b, w, (cuComplex *)Z, ldz, mz, st);
    return backtransform<cuDoubleComplex>((const cuDoubleComplex *)A, n, lda, b, w, (cuDoubleComplex *)Z, ldz, mz, st);
}

// Uniform values in [-1, 1) from a 64-bit integer hash of the index
// (splitmix64 finaliser), so that the peak GEMM runs on dense nonzero data.
__global__ void fill_uniform_kernel(double *d, float *f, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long z = i + 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const double v = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
        if (d) d[i] = v;
        if (f) f[i] = (float)v;
    }
}

// Throughput of a plain cuBLAS GEMM (the denominators of the roofline
// fractions that the measured-peak file does not hold): kind 0 DGEMM (FP64),
// 1 SGEMM with TF32 tensor-core inputs, 2 ZGEMM.  n x n x n on operands
// filled with uniform random values, `reps` timed back-to-back launches after
// one warm-up; returns TFLOP/s (2 n^3 per real GEMM, 8 n^3 per complex GEMM).
extern "C" int qd_gemm_peak(int kind, int n, int reps, double *tflops) {
    if (kind < 0 || kind > 2 || n < 64 || reps < 1) return qd_set_error(QD_ERR_ARG, "qd_gemm_peak: bad arguments");
    cublasHandle_t h = qd_cublas();
    if (!h) return qd_set_error(QD_ERR_CUDA, "cuBLAS unavailable");
    size_t es = kind == 0 ? 8 : kind == 1 ? 4 : 16;
    void *A = nullptr, *B = nullptr, *C = nullptr;
    size_t bytes = es * (size_t)n * n;
    if (cudaMalloc(&A, bytes) != cudaSuccess || cudaMalloc(&B, bytes) != cudaSuccess ||
        cudaMalloc(&C, bytes) != cudaSuccess) {
        cudaFree(A);
        cudaFree(B);
        cudaGetLastError();
        return qd_set_error(QD_ERR_NOMEM, "qd_gemm_peak");
    }
    const size_t nel = bytes / (kind == 1 ? 4 : 8);
    fill_uniform_kernel<<<148 * 8, 256, 0, cudaStreamPerThread>>>(kind == 1 ? nullptr : (double *)A,
                                                                   kind == 1 ? (float *)A : nullptr, nel);
    fill_uniform_kernel<<<148 * 8, 256, 0, cudaStreamPerThread>>>(kind == 1 ? nullptr : (double *)B,
                                                                   kind == 1 ? (float *)B : nullptr, nel);
    BLAS_OK(cublasSetStream(h, cudaStreamPerThread));
    const double d1 = 1.0, d0 = 0.0;
    const float f1 = 1.0f, f0 = 0.0f;
    const cuDoubleComplex z1 = {1, 0}, z0 = {0, 0};
    auto run = [&]() -> cublasStatus_t {
        if (kind == 0)
            return cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &d1, (double *)A, n, (double *)B, n, &d0,
                               (double *)C, n);
        if (kind == 1)
            return cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &f1, A, CUDA_R_32F, n, B, CUDA_R_32F, n, &f0, C,
                                CUDA_R_32F, n, CUBLAS_COMPUTE_32F_FAST_TF32, CUBLAS_GEMM_DEFAULT);
        return cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &z1, (cuDoubleComplex *)A, n, (cuDoubleComplex *)B, n,
                           &z0, (cuDoubleComplex *)C, n);
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cublasStatus_t st = run();
    cudaEventRecord(e0, cudaStreamPerThread);
    for (int r = 0; r < reps && st == CUBLAS_STATUS_SUCCESS; r++) st = run();
    cudaEventRecord(e1, cudaStreamPerThread);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(A);
    cudaFree(B);
    cudaFree(C);
    if (st != CUBLAS_STATUS_SUCCESS) return qd_set_error(QD_ERR_CUDA, "qd_gemm_peak: cuBLAS status %d", (int)st);
    double flop = (kind == 2 ? 8.0 : 2.0) * (double)n * n * n * reps;
    *tflops = flop / (ms * 1e-3) / 1e12;
    return QD_OK;
}

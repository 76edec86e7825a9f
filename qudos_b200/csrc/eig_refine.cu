// FP64 products of the eigensolver's final stage: H times a block of vectors
// with H Hermitian in the reference's lower-triangle storage, the small Gram
// products Z^H Y, and Z C with a small C.  They serve the Rayleigh-Ritz step
// of the mixed path and the residual check ||H z - lambda z|| of both paths.
//
// The block widths are small (k <= 64 columns) and the row count large
// (N_H up to 27000), so:
//   * hemm_lower_kernel: one CTA per 64-row tile of the output, the full row
//     of H streamed through shared memory in 16-column chunks.  A chunk left
//     of the diagonal is read straight from the stored lower triangle (rows
//     contiguous), a chunk right of it from the transposed lower triangle
//     (A[i, j] = conj(L[j, i]), columns contiguous); only chunks that cross the
//     diagonal pick per element.  Every output tile does the same amount of
//     work, so the grid needs no balancing.
//   * gram_kernel: C = A^H B reduced over row slices, one CTA per slice, FP64
//     atomics into the zeroed k x k result.
//   * zgemm_small_kernel: Y = Z C (+ beta Y) with C (k x k2) in shared memory.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "qd_internal.h"

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr int HM_TM = 64;   // output rows per CTA
constexpr int HM_JC = 16;   // columns of H per shared-memory chunk
constexpr int HM_THREADS = 128;

__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}

// Y[0:n, 0:k] = A X (+ beta Y), A Hermitian (lower triangle stored, diagonal
// taken as real).  Thread (tr, tc): rows tr + 16 r (r < 4), columns tc + 8 c.
template <int KC>
__global__ void __launch_bounds__(HM_THREADS) hemm_lower_kernel(const double2 *__restrict__ A, int64_t lda, int n,
                                                                const double2 *__restrict__ X, int64_t ldx, int k,
                                                                double2 *__restrict__ Y, int64_t ldy, double beta) {
    constexpr int NCOL = KC / 8;
    __shared__ double2 As[HM_JC][HM_TM + 1];
    __shared__ double2 Xs[HM_JC][KC];
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    const int i0 = blockIdx.x * HM_TM;
    double2 acc[4][NCOL];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < NCOL; c++) acc[r][c] = make_double2(0.0, 0.0);

    for (int j0 = 0; j0 < n; j0 += HM_JC) {
        if (j0 + HM_JC <= i0) {
            // strictly below the diagonal: A[i, j] = L[i, j], rows contiguous
            for (int e = threadIdx.x; e < HM_JC * HM_TM; e += HM_THREADS) {
                const int j = e / HM_TM, i = e % HM_TM;
                const int gi = i0 + i, gj = j0 + j;
                As[j][i] = gi < n ? A[gi + (int64_t)gj * lda] : make_double2(0.0, 0.0);
            }
        } else if (j0 >= i0 + HM_TM) {
            // strictly above: A[i, j] = conj(L[j, i]), columns of L contiguous over j
            for (int e = threadIdx.x; e < HM_JC * HM_TM; e += HM_THREADS) {
                const int i = e / HM_JC, j = e % HM_JC;
                const int gi = i0 + i, gj = j0 + j;
                double2 v = make_double2(0.0, 0.0);
                if (gi < n && gj < n) {
                    v = A[gj + (int64_t)gi * lda];
                    v.y = -v.y;
                }
                As[j][i] = v;
            }
        } else {
            for (int e = threadIdx.x; e < HM_JC * HM_TM; e += HM_THREADS) {
                const int j = e / HM_TM, i = e % HM_TM;
                const int gi = i0 + i, gj = j0 + j;
                double2 v = make_double2(0.0, 0.0);
                if (gi < n && gj < n) {
                    if (gi > gj) {
                        v = A[gi + (int64_t)gj * lda];
                    } else if (gi < gj) {
                        v = A[gj + (int64_t)gi * lda];
                        v.y = -v.y;
                    } else {
                        v = make_double2(A[gi + (int64_t)gi * lda].x, 0.0);
                    }
                }
                As[j][i] = v;
            }
        }
        for (int e = threadIdx.x; e < HM_JC * KC; e += HM_THREADS) {
            const int j = e % HM_JC, c = e / HM_JC;
            const int gj = j0 + j;
            Xs[j][c] = (gj < n && c < k) ? X[gj + (int64_t)c * ldx] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll 4
        for (int j = 0; j < HM_JC; j++) {
            double2 a[4], x[NCOL];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = As[j][tr + 16 * r];
#pragma unroll
            for (int c = 0; c < NCOL; c++) x[c] = Xs[j][tc + 8 * c];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int c = 0; c < NCOL; c++) acc[r][c] = cfma(acc[r][c], a[r], x[c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int gi = i0 + tr + 16 * r;
        if (gi >= n) continue;
#pragma unroll
        for (int c = 0; c < NCOL; c++) {
            const int col = tc + 8 * c;
            if (col >= k) continue;
            double2 *y = Y + gi + (int64_t)col * ldy;
            double2 v = acc[r][c];
            if (beta != 0.0) {
                const double2 o = *y;
                v.x += beta * o.x;
                v.y += beta * o.y;
            }
            *y = v;
        }
    }
}

// C[0:ka, 0:kb] += A^H B (or A^T B with CONJ_A false) over rows [slice),
// A n x ka, B n x kb (ka, kb <= 64).
// The slice's rows go through shared memory 16 at a time; thread t owns the
// outputs t, t + 256, ... of the ka x kb result.
constexpr int GR_ROWS = 16;
template <bool CONJ_A>
__global__ void __launch_bounds__(256) gram_kernel(const double2 *__restrict__ A, int64_t lda, int ka,
                                                   const double2 *__restrict__ B, int64_t ldb, int kb, int n,
                                                   int rows_per_cta, double *__restrict__ C /* interleaved re, im */,
                                                   int ldc) {
    __shared__ double2 As[GR_ROWS][65];
    __shared__ double2 Bs[GR_ROWS][65];
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    const int nout = ka * kb;
    double2 acc[16];
#pragma unroll
    for (int q = 0; q < 16; q++) acc[q] = make_double2(0.0, 0.0);
    for (int rb = r0; rb < r1; rb += GR_ROWS) {
        for (int e = threadIdx.x; e < GR_ROWS * 64; e += 256) {
            const int r = e % GR_ROWS, c = e / GR_ROWS;
            const int gr = rb + r;
            As[r][c] = (gr < r1 && c < ka) ? A[gr + (int64_t)c * lda] : make_double2(0.0, 0.0);
            Bs[r][c] = (gr < r1 && c < kb) ? B[gr + (int64_t)c * ldb] : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int o = threadIdx.x + 256 * q;
            if (o < nout) {
                const int i = o % ka, j = o / ka;
                double2 s = acc[q];
#pragma unroll 8
                for (int r = 0; r < GR_ROWS; r++) {
                    double2 a = As[r][i];
                    const double2 b = Bs[r][j];  // conj(a) b, or a b
                    if (!CONJ_A) a.y = -a.y;
                    s.x = fma(a.x, b.x, s.x);
                    s.x = fma(a.y, b.y, s.x);
                    s.y = fma(a.x, b.y, s.y);
                    s.y = fma(-a.y, b.x, s.y);
                }
                acc[q] = s;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int o = threadIdx.x + 256 * q;
        if (o < nout) {
            const int i = o % ka, j = o / ka;
            atomicAdd(&C[2 * (i + (int64_t)j * ldc)], acc[q].x);
            atomicAdd(&C[2 * (i + (int64_t)j * ldc) + 1], acc[q].y);
        }
    }
}

// Y[0:n, 0:k2] = Z[0:n, 0:k] C[0:k, 0:k2] + beta Y, C (ldc) staged in shared memory.
__global__ void __launch_bounds__(256) zgemm_small_kernel(const double2 *__restrict__ Z, int64_t ldz, int n, int k,
                                                          const double2 *__restrict__ Cm, int ldc, int k2,
                                                          double2 *__restrict__ Y, int64_t ldy, double beta) {
    extern __shared__ double2 Cs[];  // k x k2
    for (int e = threadIdx.x; e < k * k2; e += blockDim.x) Cs[e] = Cm[(e % k) + (int64_t)(e / k) * ldc];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c0 = 0; c0 < k2; c0 += 8) {
        double2 acc[8];
#pragma unroll
        for (int c = 0; c < 8; c++) acc[c] = make_double2(0.0, 0.0);
        for (int p = 0; p < k; p++) {
            const double2 z = Z[i + (int64_t)p * ldz];
#pragma unroll
            for (int c = 0; c < 8; c++)
                if (c0 + c < k2) acc[c] = cfma(acc[c], z, Cs[p + (c0 + c) * k]);
        }
#pragma unroll
        for (int c = 0; c < 8; c++) {
            if (c0 + c >= k2) break;
            double2 *y = Y + i + (int64_t)(c0 + c) * ldy;
            double2 v = acc[c];
            if (beta != 0.0) {
                const double2 o = *y;
                v.x += beta * o.x;
                v.y += beta * o.y;
            }
            *y = v;
        }
    }
}

// res[j] = || Y[:, j] - w[j] Z[:, j] ||_2 over all rows (one CTA per column).
__global__ void __launch_bounds__(256) residual_norm_kernel(const double2 *__restrict__ Y, int64_t ldy,
                                                            const double2 *__restrict__ Z, int64_t ldz,
                                                            const double *__restrict__ w, int n, double *res) {
    __shared__ double red[33];
    const int j = blockIdx.x;
    const double lam = w[j];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 y = Y[i + (int64_t)j * ldy], z = Z[i + (int64_t)j * ldz];
        const double rx = y.x - lam * z.x, ry = y.y - lam * z.y;
        s += rx * rx + ry * ry;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
        res[j] = sqrt(t);
    }
}

// max |L_ij| over the stored lower triangle (non-negative doubles order as integers).
__global__ void lower_absmax_kernel(const double2 *__restrict__ A, int64_t lda, int n, unsigned long long *out) {
    double m = 0.0;
    for (int j = blockIdx.x; j < n; j += gridDim.x)
        for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
            const double2 v = A[i + (int64_t)j * lda];
            m = fmax(m, sqrt(v.x * v.x + v.y * v.y));
        }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

}  // namespace

static int hemm_launch(int64_t n, const double2 *A, int64_t ld, const double2 *Xp, int64_t ldx, int k, double2 *Yp,
                       int64_t ldy, double beta, cudaStream_t st) {
    const unsigned grid = (unsigned)((n + HM_TM - 1) / HM_TM);
    qd_count_launch(1);
    if (k <= 16)
        hemm_lower_kernel<16><<<grid, HM_THREADS, 0, st>>>(A, ld, (int)n, Xp, ldx, k, Yp, ldy, beta);
    else if (k <= 32)
        hemm_lower_kernel<32><<<grid, HM_THREADS, 0, st>>>(A, ld, (int)n, Xp, ldx, k, Yp, ldy, beta);
    else if (k <= 48)
        hemm_lower_kernel<48><<<grid, HM_THREADS, 0, st>>>(A, ld, (int)n, Xp, ldx, k, Yp, ldy, beta);
    else
        hemm_lower_kernel<64><<<grid, HM_THREADS, 0, st>>>(A, ld, (int)n, Xp, ldx, k, Yp, ldy, beta);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// Y = H X + beta Y; H Hermitian n x n (lower triangle, complex128, ld), X and Y
// n x k.  Blocks of more than 64 columns are done 64 at a time.
extern "C" int qd_hemm_lower_dev(int64_t n, const void *H, int64_t ld, const void *X, int64_t ldx, int k, void *Y,
                                 int64_t ldy, double beta, void *stream) {
    if (n < 1 || k < 1 || ld < n || ldx < n || ldy < n || n > 0x7fffffff)
        return qd_set_error(QD_ERR_ARG, "qd_hemm_lower_dev: bad sizes (n=%lld, k=%d)", (long long)n, k);
    for (int c0 = 0; c0 < k; c0 += 64) {
        const int kc = k - c0 < 64 ? k - c0 : 64;
        int rc = hemm_launch(n, (const double2 *)H, ld, (const double2 *)X + (int64_t)c0 * ldx, ldx, kc,
                             (double2 *)Y + (int64_t)c0 * ldy, ldy, beta, (cudaStream_t)stream);
        if (rc) return rc;
    }
    return QD_OK;
}

// C (ka x kb, ldc, device, complex128) = A^H B (conj_a != 0) or A^T B over n
// rows; C is overwritten.  Output blocks of up to 64 x 64 are reduced one
// launch each.
extern "C" int qd_gram_ex_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb,
                              void *C, int ldc, int conj_a, void *stream) {
    if (n < 1 || ka < 1 || kb < 1 || ldc < ka || n > 0x7fffffff) return qd_set_error(QD_ERR_ARG, "qd_gram_dev: bad sizes");
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(cudaMemset2DAsync(C, sizeof(double2) * (size_t)ldc, 0, sizeof(double2) * (size_t)ka, kb, st));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int64_t slices = 2 * (int64_t)qd_sm_budget(nsm);
    int64_t rows = (n + slices - 1) / slices;
    rows = ((rows + GR_ROWS - 1) / GR_ROWS) * GR_ROWS;
    const unsigned grid = (unsigned)((n + rows - 1) / rows);
    for (int j0 = 0; j0 < kb; j0 += 64)
        for (int i0 = 0; i0 < ka; i0 += 64) {
            const int kai = ka - i0 < 64 ? ka - i0 : 64, kbj = kb - j0 < 64 ? kb - j0 : 64;
            const double2 *Ab = (const double2 *)A + (int64_t)i0 * lda, *Bb = (const double2 *)B + (int64_t)j0 * ldb;
            double *Cb = (double *)((double2 *)C + i0 + (int64_t)j0 * ldc);
            qd_count_launch(1);
            if (conj_a)
                gram_kernel<true><<<grid, 256, 0, st>>>(Ab, lda, kai, Bb, ldb, kbj, (int)n, (int)rows, Cb, ldc);
            else
                gram_kernel<false><<<grid, 256, 0, st>>>(Ab, lda, kai, Bb, ldb, kbj, (int)n, (int)rows, Cb, ldc);
            CUDA_OK(cudaGetLastError());
        }
    return QD_OK;
}

// C (ka x kb) = A^H B over n rows.
extern "C" int qd_gram_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb, void *C,
                           int ldc, void *stream) {
    return qd_gram_ex_dev(n, A, lda, ka, B, ldb, kb, C, ldc, 1, stream);
}

// Y = Z C + beta Y (Z n x k, C k x k2 on the device with leading dimension ldc).
extern "C" int qd_zgemm_small_dev(int64_t n, const void *Z, int64_t ldz, int k, const void *Cm, int ldc, int k2,
                                  void *Y, int64_t ldy, double beta, void *stream) {
    if (n < 1 || k < 1 || k2 < 1 || ldc < k || n > 0x7fffffff) return qd_set_error(QD_ERR_ARG, "qd_zgemm_small_dev: bad sizes");
    cudaStream_t st = (cudaStream_t)stream;
    static int configured = 0;
    if (!configured) {
        CUDA_OK(cudaFuncSetAttribute(zgemm_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 64 * 16));
        configured = 1;
    }
    for (int c0 = 0; c0 < k2; c0 += 64) {
        const int kc = k2 - c0 < 64 ? k2 - c0 : 64;
        for (int p0 = 0; p0 < k; p0 += 64) {
            const int kp = k - p0 < 64 ? k - p0 : 64;
            const size_t smem = sizeof(double2) * (size_t)kp * kc;
            qd_count_launch(1);
            zgemm_small_kernel<<<(unsigned)((n + 255) / 256), 256, smem, st>>>(
                (const double2 *)Z + (int64_t)p0 * ldz, ldz, (int)n, kp, (const double2 *)Cm + p0 + (int64_t)c0 * ldc,
                ldc, kc, (double2 *)Y + (int64_t)c0 * ldy, ldy, p0 == 0 ? beta : 1.0);
            CUDA_OK(cudaGetLastError());
        }
    }
    return QD_OK;
}

// Residual norms ||H z_j - w_j z_j|| (res_dev, m doubles) and the Gram matrix
// Z^H Z (gram_dev, m x m complex128) of m device vectors against H
// (lower triangle, complex128, device).  Y_dev is n x m complex128 work.
extern "C" int qd_eig_residuals_dev(int64_t n, const void *H, int64_t ld, const void *Z, int64_t ldz,
                                    const double *w_dev, int m, void *Y_dev, double *res_dev, void *gram_dev,
                                    void *stream) {
    int rc = qd_hemm_lower_dev(n, H, ld, Z, ldz, m, Y_dev, n, 0.0, stream);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    qd_count_launch(1);
    residual_norm_kernel<<<m, 256, 0, st>>>((const double2 *)Y_dev, n, (const double2 *)Z, ldz, w_dev, (int)n,
                                            res_dev);
    CUDA_OK(cudaGetLastError());
    return qd_gram_dev(n, Z, ldz, m, Z, ldz, m, gram_dev, m, stream);
}

// res[j] = || R[:, j] - w[j] Z[:, j] || for m columns.
extern "C" int qd_residual_norms_dev(int64_t n, const void *R, int64_t ldr, const void *Z, int64_t ldz,
                                     const double *w_dev, int m, double *res_dev, void *stream) {
    if (n < 1 || m < 1 || n > 0x7fffffff) return qd_set_error(QD_ERR_ARG, "qd_residual_norms_dev: bad sizes");
    qd_count_launch(1);
    residual_norm_kernel<<<m, 256, 0, (cudaStream_t)stream>>>((const double2 *)R, ldr, (const double2 *)Z, ldz, w_dev,
                                                              (int)n, res_dev);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// Residual check of host eigenpairs of a loaded problem: H is assembled on
// the device (lower triangle, FP64) and the m pairs (eigval_host,
// eigvec_host N_H x m) are checked against it.  res_host[j] = ||H z - w z||
// (eV), *orth_host = max |(Z^H Z - I)_ij|, *hnorm_host = max |H_ij|.
extern "C" int qd_problem_residuals(qd_problem *pr, int m, const double *eigval_host, const void *eigvec_host,
                                    double *res_host, double *orth_host, double *hnorm_host) {
    if (!pr || m < 1 || !eigval_host || !eigvec_host || !res_host || !orth_host)
        return qd_set_error(QD_ERR_ARG, "qd_problem_residuals: bad arguments");
    int rc = qd_problem_build_tables(pr);
    if (rc) return rc;
    const int64_t n = pr->n_h;
    void *H = nullptr, *Z = nullptr, *Y = nullptr, *G = nullptr;
    double *w = nullptr, *res = nullptr;
    if (cudaMalloc(&H, sizeof(double2) * (size_t)n * n) != cudaSuccess ||
        cudaMalloc(&Z, sizeof(double2) * (size_t)n * m) != cudaSuccess ||
        cudaMalloc(&Y, sizeof(double2) * (size_t)n * m) != cudaSuccess ||
        cudaMalloc(&G, sizeof(double2) * (size_t)m * m) != cudaSuccess ||
        cudaMalloc((void **)&w, sizeof(double) * m) != cudaSuccess ||
        cudaMalloc((void **)&res, sizeof(double) * m) != cudaSuccess) {
        rc = qd_set_error(QD_ERR_NOMEM, "qd_problem_residuals: device buffers");
    }
    if (rc == QD_OK) rc = qd_problem_assemble_dev(pr, H, n, 0, QD_PREC_FP64, nullptr);
    if (rc == QD_OK && (cudaMemcpy(Z, eigvec_host, sizeof(double2) * (size_t)n * m, cudaMemcpyHostToDevice) !=
                            cudaSuccess ||
                        cudaMemcpy(w, eigval_host, sizeof(double) * m, cudaMemcpyHostToDevice) != cudaSuccess))
        rc = qd_set_error(QD_ERR_CUDA, "qd_problem_residuals: upload");
    if (rc == QD_OK) rc = qd_eig_residuals_dev(n, H, n, Z, n, w, m, Y, res, G, nullptr);
    double2 *gh = (double2 *)malloc(sizeof(double2) * (size_t)m * m);
    if (rc == QD_OK && (cudaMemcpy(res_host, res, sizeof(double) * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
                        cudaMemcpy(gh, G, sizeof(double2) * (size_t)m * m, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = qd_set_error(QD_ERR_CUDA, "qd_problem_residuals: copy-out");
    if (rc == QD_OK) {
        double o = 0.0;
        for (int j = 0; j < m; j++)
            for (int i = 0; i < m; i++) {
                double2 g = gh[i + (size_t)j * m];
                double d = hypot(g.x - (i == j ? 1.0 : 0.0), g.y);
                if (d > o) o = d;
            }
        *orth_host = o;
    }
    if (rc == QD_OK && hnorm_host) {
        unsigned long long *mx = nullptr, bits = 0;
        if (cudaMalloc((void **)&mx, sizeof(*mx)) != cudaSuccess || cudaMemset(mx, 0, sizeof(*mx)) != cudaSuccess)
            rc = qd_set_error(QD_ERR_NOMEM, "qd_problem_residuals: norm");
        if (rc == QD_OK) {
            qd_count_launch(1);
            lower_absmax_kernel<<<1024, 256>>>((const double2 *)H, n, (int)n, mx);
            if (cudaMemcpy(&bits, mx, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = qd_set_error(QD_ERR_CUDA, "qd_problem_residuals: norm");
        }
        cudaFree(mx);
        double v;
        memcpy(&v, &bits, sizeof(v));
        *hnorm_host = v;
    }
    free(gh);
    cudaFree(H);
    cudaFree(Z);
    cudaFree(Y);
    cudaFree(G);
    cudaFree(w);
    cudaFree(res);
    return rc;
}

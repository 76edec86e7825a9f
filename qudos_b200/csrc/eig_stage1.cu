// Stage 1 of the eigensolver: dense Hermitian -> band (half bandwidth b) by
// blocked Householder reflections, and the matching back-transformation of the
// wanted eigenvectors.  Replaces the zhetrd part of LAPACK zheevr called by
// diagonalise_hamiltonian.c:73.
//
// For each panel (columns k..k+b-1, rows k+b..N-1):
//   * panel_qr_kernel: Householder QR of the tall panel in one cooperative
//     launch.  Each block keeps its slice of rows in shared memory for all b
//     columns; every column needs one norm reduction and one reduction of the
//     b-j column dot products across blocks (two bounded grid barriers).  The
//     block reflector I - V T V^H (compact WY, T upper triangular) and R are
//     written out; V is stored explicitly in the panel's place in A.
//   * trailing update A22 <- Q^H A22 Q with X = A22 V T, W = X - 1/2 V (T^H V^H X),
//     A22 -= V W^H + W V^H: FP64 with ZHEMM/ZHER2K on the lower triangle; the
//     complex64 path keeps the full matrix and runs the three products as CGEMMs
//     on the tensor cores (FP32 emulated with BF16x9, FP32 accumulation).
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "eig_common.cuh"
#include "qd_internal.h"

#define QD_BAR_LIMIT (1LL << 26)

template <typename R>
__global__ void __launch_bounds__(256) panel_qr_kernel(cpx<R> *A, int64_t lda, int m, int nb, int chunk,
                                                       cpx<R> *Rout, cpx<R> *Tout, double *red, unsigned *bar,
                                                       int *err) {
    extern __shared__ unsigned char smem_raw[];
    cpx<R> *tile = (cpx<R> *)smem_raw;  // [nb][chunk]
    __shared__ double scratch[33];
    __shared__ double s_sig;
    __shared__ cpx<double> s_alpha, s_tau, s_scale;
    __shared__ double s_beta;
    __shared__ int s_zero;
    const unsigned G = gridDim.x;
    const int r0 = blockIdx.x * chunk;
    const int rows = max(0, min(m, r0 + chunk) - r0);
    // scratch in global memory: [G] norms, then [G][nb] complex dots, alpha slot, [G][nb][nb] gram
    double *red_norm = red;
    double *red_dot = red + G;                      // 2 doubles per entry
    double *alpha_slot = red_dot + 2 * (size_t)G * nb;  // 2 doubles
    double *red_gram = alpha_slot + 2;               // 2 * nb * nb per block
    for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
        int c = idx / rows, rr = idx % rows;
        tile[c * chunk + rr] = A[(int64_t)(r0 + rr) + (int64_t)c * lda];
    }
    __syncthreads();
    for (int j = 0; j < nb; j++) {
        // ---- phase A: partial |x|^2 over rows > j; the owner of row j publishes alpha
        double s = 0.0;
        for (int rr = threadIdx.x; rr < rows; rr += blockDim.x)
            if (r0 + rr > j) s += (double)cabs2(tile[j * chunk + rr]);
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) {
            __stcg(&red_norm[blockIdx.x], s);
            if (j >= r0 && j < r0 + rows) {
                cpx<R> a = tile[j * chunk + (j - r0)];
                __stcg(&alpha_slot[0], (double)a.re);
                __stcg(&alpha_slot[1], (double)a.im);
            }
        }
        if (!grid_barrier(bar, G, err, QD_BAR_LIMIT)) return;
        // ---- phase B: Householder vector (LAPACK zlarfg conventions)
        if (threadIdx.x == 0) {
            double sig = 0.0;
            for (unsigned c = 0; c < G; c++) sig += __ldcg(&red_norm[c]);
            double ar = __ldcg(&alpha_slot[0]), ai = __ldcg(&alpha_slot[1]);
            s_sig = sig;
            s_alpha.re = ar;
            s_alpha.im = ai;
            if (sig == 0.0 && ai == 0.0) {
                s_zero = 1;
                s_tau.re = 0.0; s_tau.im = 0.0;
                s_beta = ar;
                s_scale.re = 0.0; s_scale.im = 0.0;
            } else {
                s_zero = 0;
                double beta = -copysign(sqrt(ar * ar + ai * ai + sig), ar);
                s_beta = beta;
                s_tau.re = (beta - ar) / beta;
                s_tau.im = -ai / beta;
                // scale = 1 / (alpha - beta)
                double dr = ar - beta, di = ai, den = dr * dr + di * di;
                s_scale.re = dr / den;
                s_scale.im = -di / den;
            }
        }
        __syncthreads();
        const cpx<R> scale = mk<R>((R)s_scale.re, (R)s_scale.im);
        for (int rr = threadIdx.x; rr < rows; rr += blockDim.x) {
            int r = r0 + rr;
            if (r > j) tile[j * chunk + rr] = s_zero ? mk<R>(0, 0) : cmul(tile[j * chunk + rr], scale);
        }
        __syncthreads();
        // partial dots w_c = sum_{r >= j} conj(v_r) A[r, c], v_j = 1
        {
            int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int c = j + 1 + w; c < nb; c += nw) {
                double sr = 0.0, si = 0.0;
                for (int rr = lane; rr < rows; rr += 32) {
                    int r = r0 + rr;
                    if (r < j) continue;
                    cpx<R> v = (r == j) ? mk<R>(1, 0) : tile[j * chunk + rr];
                    cpx<R> a = tile[c * chunk + rr];
                    sr += (double)v.re * a.re + (double)v.im * a.im;
                    si += (double)v.re * a.im - (double)v.im * a.re;
                }
                sr = warp_sum(sr);
                si = warp_sum(si);
                if (lane == 0) {
                    __stcg(&red_dot[2 * ((size_t)blockIdx.x * nb + c)], sr);
                    __stcg(&red_dot[2 * ((size_t)blockIdx.x * nb + c) + 1], si);
                }
            }
        }
        if (!grid_barrier(bar, G, err, QD_BAR_LIMIT)) return;
        // ---- phase C: A[r, c] -= conj(tau) v_r w_c for r >= j, c > j
        __shared__ double s_w[2 * 64];
        for (int c = j + 1 + threadIdx.x; c < nb; c += blockDim.x) {
            double sr = 0.0, si = 0.0;
            for (unsigned q = 0; q < G; q++) {
                sr += __ldcg(&red_dot[2 * ((size_t)q * nb + c)]);
                si += __ldcg(&red_dot[2 * ((size_t)q * nb + c) + 1]);
            }
            // conj(tau) * w
            double tr = s_tau.re, ti = -s_tau.im;
            s_w[2 * c] = tr * sr - ti * si;
            s_w[2 * c + 1] = tr * si + ti * sr;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < rows * (nb - j - 1); idx += blockDim.x) {
            int c = j + 1 + idx / rows, rr = idx % rows;
            int r = r0 + rr;
            if (r < j) continue;
            cpx<R> v = (r == j) ? mk<R>(1, 0) : tile[j * chunk + rr];
            cpx<R> tw = mk<R>((R)s_w[2 * c], (R)s_w[2 * c + 1]);
            tile[c * chunk + rr] = csub(tile[c * chunk + rr], cmul(v, tw));
        }
        __syncthreads();
        // row j of R is final: record it, and store the explicit V (1 on the diagonal, 0 above)
        if (j >= r0 && j < r0 + rows) {
            int rr = j - r0;
            for (int c = j + threadIdx.x; c < nb; c += blockDim.x) {
                cpx<R> val = (c == j) ? mk<R>((R)s_beta, 0) : tile[c * chunk + rr];
                Rout[j + (int64_t)c * nb] = val;
                tile[c * chunk + rr] = (c == j) ? mk<R>(1, 0) : mk<R>(0, 0);
            }
            if (threadIdx.x == 0) {
                __stcg(&Tout[j + (int64_t)j * nb].re, (R)s_tau.re);  // diagonal of T
                __stcg(&Tout[j + (int64_t)j * nb].im, (R)s_tau.im);
            }
        }
        __syncthreads();
    }
    // rows above their diagonal inside this slice are zero in V (r < c); write V back
    for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
        int c = idx / rows, rr = idx % rows;
        int r = r0 + rr;
        cpx<R> v = tile[c * chunk + rr];
        if (r < c) v = mk<R>(0, 0);
        A[(int64_t)r + (int64_t)c * lda] = v;
    }
    // Gram matrix V^H V (partial per block)
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        int p = idx / nb, q = idx % nb;
        double sr = 0.0, si = 0.0;
        if (p < q) {
            for (int rr = 0; rr < rows; rr++) {
                int r = r0 + rr;
                cpx<R> a = (r < p) ? mk<R>(0, 0) : tile[p * chunk + rr];
                cpx<R> b = (r < q) ? mk<R>(0, 0) : tile[q * chunk + rr];
                sr += (double)a.re * b.re + (double)a.im * b.im;
                si += (double)a.re * b.im - (double)a.im * b.re;
            }
        }
        __stcg(&red_gram[2 * ((size_t)blockIdx.x * nb * nb + idx)], sr);
        __stcg(&red_gram[2 * ((size_t)blockIdx.x * nb * nb + idx) + 1], si);
    }
    if (!grid_barrier(bar, G, err, QD_BAR_LIMIT)) return;
    if (blockIdx.x != 0) return;
    // T (LAPACK zlarft, forward, columnwise): T[0:i, i] = -tau_i T[0:i, 0:i] (V^H V)[0:i, i]
    double *gram = (double *)smem_raw;       // nb*nb complex, row-major [p][q]
    double *Tl = gram + 2 * nb * nb;         // nb*nb complex, column-major
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        double sr = 0.0, si = 0.0;
        for (unsigned q = 0; q < G; q++) {
            sr += __ldcg(&red_gram[2 * ((size_t)q * nb * nb + idx)]);
            si += __ldcg(&red_gram[2 * ((size_t)q * nb * nb + idx) + 1]);
        }
        gram[2 * idx] = sr;
        gram[2 * idx + 1] = si;
    }
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
        int p = idx % nb, q = idx / nb;
        double tr = 0.0, ti = 0.0;
        if (p == q) {
            tr = (double)__ldcg(&Tout[p + (int64_t)q * nb].re);
            ti = (double)__ldcg(&Tout[p + (int64_t)q * nb].im);
        }
        Tl[2 * idx] = tr;
        Tl[2 * idx + 1] = ti;
    }
    __syncthreads();
    for (int i = 1; i < nb; i++) {
        double tr = Tl[2 * (i + i * nb)], ti = Tl[2 * (i + i * nb) + 1];
        for (int p = threadIdx.x; p < i; p += blockDim.x) {
            double sr = 0.0, si = 0.0;
            for (int q = p; q < i; q++) {  // T upper triangular
                double a_r = Tl[2 * (p + q * nb)], a_i = Tl[2 * (p + q * nb) + 1];
                double g_r = gram[2 * (q * nb + i)], g_i = gram[2 * (q * nb + i) + 1];
                sr += a_r * g_r - a_i * g_i;
                si += a_r * g_i + a_i * g_r;
            }
            Tl[2 * (p + i * nb)] = -(tr * sr - ti * si);
            Tl[2 * (p + i * nb) + 1] = -(tr * si + ti * sr);
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x)
        Tout[idx] = mk<R>((R)Tl[2 * idx], (R)Tl[2 * idx + 1]);
}

// ----------------------------------------------------------------------------
// Host driver
// ----------------------------------------------------------------------------
#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)
#define BLAS_OK(x)                                                                          \
    do {                                                                                    \
        cublasStatus_t s_ = (x);                                                            \
        if (s_ != CUBLAS_STATUS_SUCCESS)                                                    \
            return qd_set_error(QD_ERR_CUDA, "%s:%d cuBLAS status %d", __FILE__, __LINE__, (int)s_); \
    } while (0)

struct Stage1Work {
    void *VT, *X, *M, *Y, *Tall, *Rall;  // VT, X: n x b; M, Y: b x b; Tall/Rall: npanels x b x b
    double *red;
    unsigned *bar;
    int *err;
    int npanels;
};

static int n_panels(int64_t n, int b) {
    int c = 0;
    for (int64_t k = 0; k + b < n; k += b) c++;
    return c;
}

extern "C" cublasHandle_t qd_cublas(void);
extern "C" int qd_mixed_gemm_mode(void);

template <typename R>
static int launch_panel(cpx<R> *P, int64_t lda, int m, int nb, cpx<R> *Rp, cpx<R> *Tp, Stage1Work &w,
                        cudaStream_t st) {
    int dev;
    CUDA_OK(cudaGetDevice(&dev));
    int nsm;
    CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int G = (int)((m + 31) / 32);
    if (G > nsm) G = nsm;
    if (G < 1) G = 1;
    int chunk = (m + G - 1) / G;
    size_t smem = (size_t)chunk * nb * sizeof(cpx<R>);
    size_t smem_need = smem > (size_t)nb * nb * 32 ? smem : (size_t)nb * nb * 32;
    static size_t configured[2] = {0, 0};
    int ti = sizeof(R) == 8 ? 0 : 1;
    if (smem_need > configured[ti]) {
        CUDA_OK(cudaFuncSetAttribute(panel_qr_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(200 * 1024)));
        configured[ti] = 200 * 1024;
    }
    if (smem_need > 200 * 1024) return qd_set_error(QD_ERR_UNSUPPORTED, "panel slice too large (%d rows)", chunk);
    CUDA_OK(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), st));
    void *args[] = {&P, &lda, &m, &nb, &chunk, &Rp, &Tp, &w.red, &w.bar, &w.err};
    CUDA_OK(cudaLaunchCooperativeKernel((void *)panel_qr_kernel<R>, dim3(G), dim3(256), args, smem_need, st));
    return QD_OK;
}

// FP64: A lower triangle (complex128, lda), reduced in place to band form.
static int stage1_fp64(cuDoubleComplex *A, int64_t n, int64_t lda, int b, Stage1Work &w, cudaStream_t st) {
    cublasHandle_t h = qd_cublas();
    BLAS_OK(cublasSetStream(h, st));
    const cuDoubleComplex one = {1, 0}, zero = {0, 0}, mone = {-1, 0}, mhalf = {-0.5, 0};
    int p = 0;
    for (int64_t k = 0; k + b < n; k += b, p++) {
        int m = (int)(n - k - b), nb = b < m ? b : m;
        cuDoubleComplex *P = A + (k + b) + k * lda;
        cuDoubleComplex *Tp = (cuDoubleComplex *)w.Tall + (int64_t)p * b * b;
        cuDoubleComplex *Rp = (cuDoubleComplex *)w.Rall + (int64_t)p * b * b;
        CUDA_OK(cudaMemsetAsync(Tp, 0, sizeof(cuDoubleComplex) * b * b, st));
        CUDA_OK(cudaMemsetAsync(Rp, 0, sizeof(cuDoubleComplex) * b * b, st));
        int rc = launch_panel<double>((cpx<double> *)P, lda, m, nb, (cpx<double> *)Rp, (cpx<double> *)Tp, w, st);
        if (rc) return rc;
        cuDoubleComplex *A22 = A + (k + b) + (k + b) * lda;
        cuDoubleComplex *VT = (cuDoubleComplex *)w.VT, *X = (cuDoubleComplex *)w.X, *M = (cuDoubleComplex *)w.M,
                        *Y = (cuDoubleComplex *)w.Y;
        // VT = V T ; X = A22 VT
        BLAS_OK(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &one, P, lda, Tp, b, &zero, VT, m));
        BLAS_OK(cublasZhemm(h, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, m, nb, &one, A22, lda, VT, m, &zero, X, m));
        // M = V^H X ; Y = T^H M ; X = X - 1/2 V Y
        BLAS_OK(cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, nb, m, &one, P, lda, X, m, &zero, M, b));
        BLAS_OK(cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, nb, nb, &one, Tp, b, M, b, &zero, Y, b));
        BLAS_OK(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &mhalf, P, lda, Y, b, &one, X, m));
        // A22 -= V X^H + X V^H
        const double dmone = -1.0, done = 1.0;
        (void)dmone;
        BLAS_OK(cublasZher2k(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, m, nb, &mone, P, lda, X, m, &done, A22, lda));
    }
    return QD_OK;
}

// complex64, full Hermitian storage: the three products as CGEMMs on the tensor cores.
static int cgemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
                 const cuComplex *alpha, const cuComplex *A, int64_t lda, const cuComplex *B, int64_t ldb,
                 const cuComplex *beta, cuComplex *C, int64_t ldc) {
    int mode = qd_mixed_gemm_mode();
    cublasComputeType_t ct = mode == 2 ? CUBLAS_COMPUTE_32F_EMULATED_16BFX9
                             : mode == 1 ? CUBLAS_COMPUTE_32F_FAST_TF32
                                         : CUBLAS_COMPUTE_32F;
    cublasStatus_t s = cublasGemmEx(h, ta, tb, m, n, k, alpha, A, CUDA_C_32F, (int)lda, B, CUDA_C_32F, (int)ldb, beta,
                                    C, CUDA_C_32F, (int)ldc, ct, CUBLAS_GEMM_DEFAULT);
    if (s == CUBLAS_STATUS_NOT_SUPPORTED && mode == 2)
        s = cublasGemmEx(h, ta, tb, m, n, k, alpha, A, CUDA_C_32F, (int)lda, B, CUDA_C_32F, (int)ldb, beta, C,
                         CUDA_C_32F, (int)ldc, CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT);
    BLAS_OK(s);
    return QD_OK;
}

static int stage1_fp32(cuComplex *A, int64_t n, int64_t lda, int b, Stage1Work &w, cudaStream_t st) {
    cublasHandle_t h = qd_cublas();
    BLAS_OK(cublasSetStream(h, st));
    const cuComplex one = {1, 0}, zero = {0, 0}, mone = {-1, 0}, mhalf = {-0.5f, 0};
    int p = 0;
    for (int64_t k = 0; k + b < n; k += b, p++) {
        int m = (int)(n - k - b), nb = b < m ? b : m;
        cuComplex *P = A + (k + b) + k * lda;
        cuComplex *Tp = (cuComplex *)w.Tall + (int64_t)p * b * b;
        cuComplex *Rp = (cuComplex *)w.Rall + (int64_t)p * b * b;
        CUDA_OK(cudaMemsetAsync(Tp, 0, sizeof(cuComplex) * b * b, st));
        CUDA_OK(cudaMemsetAsync(Rp, 0, sizeof(cuComplex) * b * b, st));
        int rc = launch_panel<float>((cpx<float> *)P, lda, m, nb, (cpx<float> *)Rp, (cpx<float> *)Tp, w, st);
        if (rc) return rc;
        cuComplex *A22 = A + (k + b) + (k + b) * lda;
        cuComplex *VT = (cuComplex *)w.VT, *X = (cuComplex *)w.X, *M = (cuComplex *)w.M, *Y = (cuComplex *)w.Y;
        BLAS_OK(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &one, P, (int)lda, Tp, b, &zero, VT, m));
        rc = cgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, m, &one, A22, lda, VT, m, &zero, X, m);
        if (rc) return rc;
        BLAS_OK(cublasCgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, nb, m, &one, P, (int)lda, X, m, &zero, M, b));
        BLAS_OK(cublasCgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, nb, nb, &one, Tp, b, M, b, &zero, Y, b));
        BLAS_OK(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &mhalf, P, (int)lda, Y, b, &one, X, m));
        // A22 -= V X^H + X V^H on the full matrix: two products of inner dimension nb
        rc = cgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, m, m, nb, &mone, P, lda, X, m, &one, A22, lda);
        if (rc) return rc;
        rc = cgemm(h, CUBLAS_OP_N, CUBLAS_OP_C, m, m, nb, &mone, X, m, P, lda, &one, A22, lda);
        if (rc) return rc;
    }
    return QD_OK;
}

extern "C" int qd_stage1_alloc(int64_t n, int b, int elem_bytes, Stage1Work *w) {
    w->npanels = n_panels(n, b);
    size_t eb = (size_t)elem_bytes;
    if (cudaMalloc(&w->VT, eb * n * b) != cudaSuccess || cudaMalloc(&w->X, eb * n * b) != cudaSuccess ||
        cudaMalloc(&w->M, eb * b * b) != cudaSuccess || cudaMalloc(&w->Y, eb * b * b) != cudaSuccess ||
        cudaMalloc(&w->Tall, eb * (size_t)(w->npanels + 1) * b * b) != cudaSuccess ||
        cudaMalloc(&w->Rall, eb * (size_t)(w->npanels + 1) * b * b) != cudaSuccess)
        return qd_set_error(QD_ERR_NOMEM, "stage-1 workspace allocation failed");
    int dev, nsm;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    size_t red_doubles = (size_t)nsm * (1 + 2 * b + 2 * b * b) + 8;
    if (cudaMalloc(&w->red, sizeof(double) * red_doubles) != cudaSuccess ||
        cudaMalloc(&w->bar, 4 * sizeof(unsigned)) != cudaSuccess || cudaMalloc(&w->err, sizeof(int)) != cudaSuccess)
        return qd_set_error(QD_ERR_NOMEM, "stage-1 scratch allocation failed");
    cudaMemset(w->err, 0, sizeof(int));
    return QD_OK;
}

extern "C" void qd_stage1_free(Stage1Work *w) {
    cudaFree(w->VT); cudaFree(w->X); cudaFree(w->M); cudaFree(w->Y);
    cudaFree(w->Tall); cudaFree(w->Rall); cudaFree(w->red); cudaFree(w->bar); cudaFree(w->err);
}

extern "C" int qd_stage1_run(void *A, int64_t n, int64_t lda, int b, int fp32, Stage1Work *w, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    int rc = fp32 ? stage1_fp32((cuComplex *)A, n, lda, b, *w, st) : stage1_fp64((cuDoubleComplex *)A, n, lda, b, *w, st);
    if (rc) return rc;
    int herr = 0;
    CUDA_OK(cudaMemcpyAsync(&herr, w->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (herr) return qd_set_error(QD_ERR_TIMEOUT, "panel factorisation: grid barrier wait ran out");
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
                // R block of panel p = k/b: R[pr][pc], pr = i - (k+b), pc = j - k, nonzero for pr <= pc
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
    if (fp32)
        extract_band_kernel<float><<<(unsigned)n, 64, 0, st>>>((const cpx<float> *)A, lda, n, b,
                                                               (const cpx<float> *)w->Rall, AB, ldb);
    else
        extract_band_kernel<double><<<(unsigned)n, 64, 0, st>>>((const cpx<double> *)A, lda, n, b,
                                                                (const cpx<double> *)w->Rall, AB, ldb);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// Back-transformation Z <- Q1 Z = H_1 H_2 ... Z, panels in reverse order:
// Z[k+b:, :] -= V (T (V^H Z[k+b:, :])).  Z is n x mz (ldz), same precision as A.
extern "C" int qd_stage1_backtransform(const void *A, int64_t n, int64_t lda, int b, int fp32, const Stage1Work *w,
                                       void *Z, int64_t ldz, int mz, void *stream) {
    cublasHandle_t h = qd_cublas();
    BLAS_OK(cublasSetStream(h, (cudaStream_t)stream));
    int np = w->npanels;
    for (int p = np - 1; p >= 0; p--) {
        int64_t k = (int64_t)p * b;
        int m = (int)(n - k - b), nb = b < m ? b : m;
        if (fp32) {
            const cuComplex one = {1, 0}, zero = {0, 0}, mone = {-1, 0};
            const cuComplex *V = (const cuComplex *)A + (k + b) + k * lda;
            const cuComplex *T = (const cuComplex *)w->Tall + (int64_t)p * b * b;
            cuComplex *Zs = (cuComplex *)Z + (k + b);
            cuComplex *M = (cuComplex *)w->VT, *Y = (cuComplex *)w->X;
            BLAS_OK(cublasCgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, mz, m, &one, V, (int)lda, Zs, (int)ldz, &zero, M, nb));
            BLAS_OK(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nb, mz, nb, &one, T, b, M, nb, &zero, Y, nb));
            BLAS_OK(cublasCgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, mz, nb, &mone, V, (int)lda, Y, nb, &one, Zs, (int)ldz));
        } else {
            const cuDoubleComplex one = {1, 0}, zero = {0, 0}, mone = {-1, 0};
            const cuDoubleComplex *V = (const cuDoubleComplex *)A + (k + b) + k * lda;
            const cuDoubleComplex *T = (const cuDoubleComplex *)w->Tall + (int64_t)p * b * b;
            cuDoubleComplex *Zs = (cuDoubleComplex *)Z + (k + b);
            cuDoubleComplex *M = (cuDoubleComplex *)w->VT, *Y = (cuDoubleComplex *)w->X;
            BLAS_OK(cublasZgemm(h, CUBLAS_OP_C, CUBLAS_OP_N, nb, mz, m, &one, V, lda, Zs, ldz, &zero, M, nb));
            BLAS_OK(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, nb, mz, nb, &one, T, b, M, nb, &zero, Y, nb));
            BLAS_OK(cublasZgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, m, mz, nb, &mone, V, lda, Y, nb, &one, Zs, ldz));
        }
    }
    return QD_OK;
}

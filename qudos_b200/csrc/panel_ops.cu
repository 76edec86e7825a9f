// Tall-and-skinny products of the dense -> band reduction (eig_stage1.cu) and
// of the back-transformation, for complex64 (mixed path) and complex128
// (FP64 path) data.  Every product of a panel step has one long dimension
// (the m rows of the trailing matrix) and short others (the b = 32 panel
// columns and the K <= 256 pending reflector columns):
//
//   tsmm_nn  C[m x nc] = beta C + sum_t alpha_t A_t[m x K_t] op(B_t)[K_t x nc],
//            nc <= 64
//            (up to two terms; op(B) is B or B^H of an nc x K block).  One CTA
//            per 128-row tile; the K dimension is streamed through shared
//            memory in chunks of 16.  Serves the panel refresh
//            (P -= V Wb^H + W Vb^H), V T, the corrections (X -= V S1 + W S2),
//            W = X - 1/2 V Y and the back-transformation (Z -= V Y).
//   tsmm_cn  C[k1 x nc] = A[m x k1]^H B[m x nc], k1 <= 256 with nc <= 32, or
//            k1 <= 64 with nc <= 64: the rows
//            are split into slices, each CTA accumulates its slice in the
//            working precision, writes the partial, and a second kernel sums
//            the partials in FP64 (a fixed order, so results do not depend on
//            scheduling).  Serves the Gram matrix V^H V, [W V]^H VT, V^H X and
//            V^H Z.
//   small_cn C[n1 x n2] = A[k x n1]^H B[k x n2] for matrices of up to 32 x 32 (T^H M).
#include <cuda_runtime.h>
#include <stdint.h>

#include "eig_common.cuh"
#include "qd_internal.h"

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

namespace {

template <typename R>
struct TsTerm {
    const cpx<R> *A;
    int64_t lda;
    const cpx<R> *B;
    int64_t ldb;
    int K;
    int btrans;  // 0: B is K x nc (ldb); 1: op(B) = B^H with B stored nc x K (ldb)
    R alpha;
};

template <typename R>
__device__ __forceinline__ cpx<R> cfma_(cpx<R> acc, cpx<R> a, cpx<R> b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
    return acc;
}

// Thread (tx, ty): rows tx + 32 i (i < RI, a tile of 32 RI rows), columns
// NJ ty + j (j < NJ), NJ = NCW / 8 for an output width of NCW = 32 or 64.
// The K dimension of both terms is one sequence of chunks; the next chunk's
// global loads are issued into registers before the current chunk is
// multiplied, so their latency overlaps the arithmetic.
template <typename R, int NCW, int RI>
__global__ void __launch_bounds__(256) tsmm_nn_kernel(int m, int nc, TsTerm<R> t0, TsTerm<R> t1, int nterms,
                                                      cpx<R> *C, int64_t ldc, R beta) {
    // K chunk of 16 (8 for complex128 at 64 columns, to stay within 48 KB of static shared memory)
    constexpr int TM = 32 * RI, NJ = NCW / 8, KC = (sizeof(R) == 8 && NCW == 64) ? 8 : 16;
    constexpr int LA = KC * TM / 256, LB = (KC * NCW + 255) / 256;
    __shared__ cpx<R> As[KC][TM];
    __shared__ cpx<R> Bs[KC][NCW + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int r0 = blockIdx.x * TM;
    const int nch0 = (t0.K + KC - 1) / KC, nch = nch0 + (nterms > 1 ? (t1.K + KC - 1) / KC : 0);
    cpx<R> acc[RI][NJ];
#pragma unroll
    for (int i = 0; i < RI; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++) acc[i][j] = mk<R>(0, 0);
    cpx<R> ra[LA], rb[LB];
    auto fetch = [&](int ch) {
        const TsTerm<R> &T = ch < nch0 ? t0 : t1;
        const int p0 = (ch < nch0 ? ch : ch - nch0) * KC;
#pragma unroll
        for (int l = 0; l < LA; l++) {
            const int e = threadIdx.x + 256 * l;
            const int r = e % TM, p = e / TM;
            const int gr = r0 + r, gp = p0 + p;
            ra[l] = (gr < m && gp < T.K) ? T.A[gr + (int64_t)gp * T.lda] : mk<R>(0, 0);
        }
#pragma unroll
        for (int l = 0; l < LB; l++) {
            const int e = threadIdx.x + 256 * l;
            cpx<R> v = mk<R>(0, 0);
            if (e < KC * NCW) {
                if (!T.btrans) {
                    const int p = e % KC, c = e / KC;
                    if (p0 + p < T.K && c < nc) v = T.B[(p0 + p) + (int64_t)c * T.ldb];
                } else {
                    const int c = e % NCW, p = e / NCW;
                    if (p0 + p < T.K && c < nc) v = cconj(T.B[c + (int64_t)(p0 + p) * T.ldb]);
                }
            }
            rb[l] = mk<R>(T.alpha * v.re, T.alpha * v.im);
        }
    };
    if (nch > 0) fetch(0);
    for (int ch = 0; ch < nch; ch++) {
        __syncthreads();
#pragma unroll
        for (int l = 0; l < LA; l++) {
            const int e = threadIdx.x + 256 * l;
            As[e / TM][e % TM] = ra[l];
        }
        const TsTerm<R> &T = ch < nch0 ? t0 : t1;
#pragma unroll
        for (int l = 0; l < LB; l++) {
            const int e = threadIdx.x + 256 * l;
            if (e < KC * NCW) {
                if (!T.btrans) Bs[e % KC][e / KC] = rb[l];
                else Bs[e / NCW][e % NCW] = rb[l];
            }
        }
        __syncthreads();
        if (ch + 1 < nch) fetch(ch + 1);
#pragma unroll 4
        for (int p = 0; p < KC; p++) {
            cpx<R> a[RI], b[NJ];
#pragma unroll
            for (int i = 0; i < RI; i++) a[i] = As[p][tx + 32 * i];
#pragma unroll
            for (int j = 0; j < NJ; j++) b[j] = Bs[p][NJ * ty + j];
#pragma unroll
            for (int i = 0; i < RI; i++)
#pragma unroll
                for (int j = 0; j < NJ; j++) acc[i][j] = cfma_(acc[i][j], a[i], b[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < RI; i++) {
        const int gr = r0 + tx + 32 * i;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int c = NJ * ty + j;
            if (c >= nc) continue;
            cpx<R> *p = C + gr + (int64_t)c * ldc;
            cpx<R> v = acc[i][j];
            if (beta != (R)0) {
                const cpx<R> o = *p;
                v.re = fma(beta, o.re, v.re);
                v.im = fma(beta, o.im, v.im);
            }
            *p = v;
        }
    }
}

constexpr int CN_RC = 32;  // rows per shared-memory chunk

// Partial A^H B over one slice of rows.  Thread (ti, tj): outputs i = ti + 32 u
// (u < KU), j = NV tj + v (v < NV), NV = NCW / 8 for NCW = 32 or 64 output
// columns.  Partials: part[slice][j * k1 + i].
template <typename R, int KU, int NCW>
__global__ void __launch_bounds__(256) tsmm_cn_kernel(int m, const cpx<R> *__restrict__ A, int64_t lda, int k1,
                                                      const cpx<R> *__restrict__ B, int64_t ldb, int nc,
                                                      int rows_per_slice, cpx<R> *__restrict__ part) {
    // rows padded by one element so that the row-wise (coalesced) global loads
    // of a warp land in distinct banks
    constexpr int KW = 32 * KU + 1, BW = NCW + 1, NV = NCW / 8;
    extern __shared__ unsigned char cn_smem[];
    cpx<R> *As = (cpx<R> *)cn_smem;  // [CN_RC][KW]
    cpx<R> *Bs = As + CN_RC * KW;    // [CN_RC][BW]
    const int ti = threadIdx.x & 31, tj = threadIdx.x >> 5;
    const int r0 = blockIdx.x * rows_per_slice, r1 = min(m, r0 + rows_per_slice);
    cpx<R> acc[KU][NV];
#pragma unroll
    for (int u = 0; u < KU; u++)
#pragma unroll
        for (int v = 0; v < NV; v++) acc[u][v] = mk<R>(0, 0);
    for (int rb = r0; rb < r1; rb += CN_RC) {
        for (int e = threadIdx.x; e < CN_RC * 32 * KU; e += 256) {
            const int r = e % CN_RC, i = e / CN_RC;
            As[r * KW + i] = (rb + r < r1 && i < k1) ? A[(rb + r) + (int64_t)i * lda] : mk<R>(0, 0);
        }
        for (int e = threadIdx.x; e < CN_RC * NCW; e += 256) {
            const int r = e % CN_RC, j = e / CN_RC;
            Bs[r * BW + j] = (rb + r < r1 && j < nc) ? B[(rb + r) + (int64_t)j * ldb] : mk<R>(0, 0);
        }
        __syncthreads();
#pragma unroll 2
        for (int r = 0; r < CN_RC; r++) {
            cpx<R> a[KU], b[NV];
#pragma unroll
            for (int u = 0; u < KU; u++) a[u] = cconj(As[r * KW + ti + 32 * u]);
#pragma unroll
            for (int v = 0; v < NV; v++) b[v] = Bs[r * BW + NV * tj + v];
#pragma unroll
            for (int u = 0; u < KU; u++)
#pragma unroll
                for (int v = 0; v < NV; v++) acc[u][v] = cfma_(acc[u][v], a[u], b[v]);
        }
        __syncthreads();
    }
    cpx<R> *P = part + (int64_t)blockIdx.x * k1 * nc;
#pragma unroll
    for (int u = 0; u < KU; u++) {
        const int i = ti + 32 * u;
        if (i >= k1) continue;
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const int j = NV * tj + v;
            if (j < nc) P[(int64_t)j * k1 + i] = acc[u][v];
        }
    }
}

// C[i + j ldc] = sum over slices of part[s][j k1 + i] in FP64: one warp per
// output, lane l adds the slices l, l + 32, ..., then a fixed shuffle tree
// (the same order on every run).
template <typename R>
__global__ void __launch_bounds__(256) cn_reduce_kernel(const cpx<R> *__restrict__ part, int slices, int k1, int nc,
                                                        cpx<R> *C, int64_t ldc) {
    const int o = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (o >= k1 * nc) return;
    double sr = 0.0, si = 0.0;
    for (int s = lane; s < slices; s += 32) {
        const cpx<R> v = part[(int64_t)s * k1 * nc + o];
        sr += (double)v.re;
        si += (double)v.im;
    }
    for (int d = 16; d > 0; d >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, d);
        si += __shfl_xor_sync(0xffffffffu, si, d);
    }
    if (lane == 0) C[(o % k1) + (int64_t)(o / k1) * ldc] = mk<R>((R)sr, (R)si);
}

// C[n1 x n2] = alpha A[k x n1]^H B[k x n2], small (one CTA; k, n1, n2 <= 32;
// both factors staged in shared memory, FP64 sums).
template <typename R>
__global__ void __launch_bounds__(1024) small_cn_kernel(int k, int n1, int n2, const cpx<R> *A, int lda,
                                                        const cpx<R> *B, int ldb, R alpha, cpx<R> *C, int ldc) {
    __shared__ cpx<R> As[32][33], Bs[32][33];
    for (int e = threadIdx.x; e < k * n1; e += blockDim.x) As[e / k][e % k] = A[(e % k) + (e / k) * lda];
    for (int e = threadIdx.x; e < k * n2; e += blockDim.x) Bs[e / k][e % k] = B[(e % k) + (e / k) * ldb];
    __syncthreads();
    for (int o = threadIdx.x; o < n1 * n2; o += blockDim.x) {
        const int i = o % n1, j = o / n1;
        double sr = 0.0, si = 0.0;
        for (int p = 0; p < k; p++) {
            const cpx<R> a = As[i][p], b = Bs[j][p];
            sr += (double)a.re * b.re + (double)a.im * b.im;
            si += (double)a.re * b.im - (double)a.im * b.re;
        }
        C[i + j * ldc] = mk<R>((R)(alpha * sr), (R)(alpha * si));
    }
}

int g_nsm = 0;
int nsm() {
    if (!g_nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
        if (g_nsm < 1) g_nsm = 148;
    }
    return qd_sm_budget(g_nsm);
}

// Rows per slice and slice count of tsmm_cn for m rows and k1 outputs per
// column: up to four CTAs per SM for narrow products (so that loads of some
// CTAs overlap the arithmetic of others), one for the widest, at least 64
// rows each.
void cn_slices(int m, int k1, int *rows, int *slices) {
    int s = nsm() * (k1 <= 64 ? 4 : k1 <= 128 ? 2 : 1);
    int r = (m + s - 1) / s;
    if (r < 64) r = 64;
    r = ((r + CN_RC - 1) / CN_RC) * CN_RC;
    *rows = r;
    *slices = (m + r - 1) / r;
}

template <typename R>
int tsmm_nn(int m, int nc, int nterms, const TsTerm<R> *terms, cpx<R> *C, int64_t ldc, R beta, cudaStream_t st) {
    if (m <= 0 || nc <= 0) return QD_OK;
    if (nc > 64) return qd_set_error(QD_ERR_ARG, "tsmm_nn: %d columns above 64", nc);
    TsTerm<R> t1 = nterms > 1 ? terms[1] : terms[0];
    qd_count_launch(1);
    // rows per CTA: 128 while that still gives two CTAs per SM, else 64 or 32
    const int ri = m >= 2 * 128 * nsm() ? 4 : m >= 2 * 64 * nsm() ? 2 : 1;
    const unsigned grid = (unsigned)((m + 32 * ri - 1) / (32 * ri));
#define QD_NN(W, RI) tsmm_nn_kernel<R, W, RI><<<grid, 256, 0, st>>>(m, nc, terms[0], t1, nterms, C, ldc, beta)
    if (nc <= 32) {
        if (ri == 4) QD_NN(32, 4);
        else if (ri == 2) QD_NN(32, 2);
        else QD_NN(32, 1);
    } else {
        if (ri == 4) QD_NN(64, 4);
        else if (ri == 2) QD_NN(64, 2);
        else QD_NN(64, 1);
    }
#undef QD_NN
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

template <typename R, int KU, int NCW = 32>
int cn_launch(int slices, cudaStream_t st, int m, const cpx<R> *A, int64_t lda, int k1, const cpx<R> *B,
              int64_t ldb, int nc, int rows, cpx<R> *scratch) {
    const size_t smem = sizeof(cpx<R>) * (size_t)CN_RC * (32 * KU + 1 + NCW + 1);
    static int cfg = 0;
    if (!cfg) {
        CUDA_OK(cudaFuncSetAttribute(tsmm_cn_kernel<R, KU, NCW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
        cfg = 1;
    }
    tsmm_cn_kernel<R, KU, NCW><<<slices, 256, smem, st>>>(m, A, lda, k1, B, ldb, nc, rows, scratch);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

template <typename R>
int tsmm_cn(int m, const cpx<R> *A, int64_t lda, int k1, const cpx<R> *B, int64_t ldb, int nc, cpx<R> *C,
            int64_t ldc, cpx<R> *scratch, size_t scratch_bytes, cudaStream_t st) {
    if (k1 <= 0 || nc <= 0) return QD_OK;
    if (k1 > 256 || nc > 64 || (nc > 32 && k1 > 64))
        return qd_set_error(QD_ERR_ARG, "tsmm_cn: %d x %d outputs (at most 256 x 32 or 64 x 64)", k1, nc);
    if (m <= 0) {
        CUDA_OK(cudaMemset2DAsync(C, sizeof(cpx<R>) * ldc, 0, sizeof(cpx<R>) * k1, nc, st));
        return QD_OK;
    }
    int rows, slices;
    cn_slices(m, k1, &rows, &slices);
    if ((size_t)slices * k1 * nc * sizeof(cpx<R>) > scratch_bytes)
        return qd_set_error(QD_ERR_ARG, "tsmm_cn: scratch of %zu bytes below the %zu needed", scratch_bytes,
                            (size_t)slices * k1 * nc * sizeof(cpx<R>));
    const int ku = (k1 + 31) / 32;
    qd_count_launch(2);
    int rc = QD_OK;
    if (nc > 32) {
        rc = ku == 1 ? cn_launch<R, 1, 64>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch)
                     : cn_launch<R, 2, 64>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch);
    } else {
        switch (ku) {
            case 1: rc = cn_launch<R, 1>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 2: rc = cn_launch<R, 2>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 3: rc = cn_launch<R, 3>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 4: rc = cn_launch<R, 4>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 5: rc = cn_launch<R, 5>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 6: rc = cn_launch<R, 6>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            case 7: rc = cn_launch<R, 7>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
            default: rc = cn_launch<R, 8>(slices, st, m, A, lda, k1, B, ldb, nc, rows, scratch); break;
        }
    }
    if (rc) return rc;
    const int nout = k1 * nc;
    cn_reduce_kernel<R><<<(nout + 7) / 8, 256, 0, st>>>(scratch, slices, k1, nc, C, ldc);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

template <typename R>
int small_cn(int k, int n1, int n2, const cpx<R> *A, int lda, const cpx<R> *B, int ldb, R alpha, cpx<R> *C, int ldc,
             cudaStream_t st) {
    if (k < 1 || n1 < 1 || n2 < 1 || k > 32 || n1 > 32 || n2 > 32)
        return qd_set_error(QD_ERR_ARG, "small_cn: sizes above 32");
    qd_count_launch(1);
    small_cn_kernel<R><<<1, 1024, 0, st>>>(k, n1, n2, A, lda, B, ldb, alpha, C, ldc);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

}  // namespace

// Partial-sum scratch (bytes) that qd_tsmm_cn needs for any row count up to m
// and any product of at most k1 x nc outputs.  The slice count is not
// monotonic in m (slices are rounded to whole shared-memory chunks), so the
// bound is taken over every m' <= m: at most four slices per SM, and at most
// ceil(m / 64).
extern "C" size_t qd_tsmm_cn_scratch_bytes(int m, int k1, int nc, int elem_bytes) {
    int64_t smax = 4 * (int64_t)nsm();
    const int64_t by_rows = ((int64_t)(m > 0 ? m : 1) + 63) / 64;
    if (by_rows < smax) smax = by_rows;
    return (size_t)smax * k1 * nc * elem_bytes;
}

// C-linkage entry points for both precisions (fp32 != 0: complex64).  Terms
// are passed as arrays of pointers and sizes; alpha is real.
extern "C" int qd_tsmm_nn(int fp32, int m, int nc, int nterms, const void *const *A, const int64_t *lda,
                          const void *const *B, const int64_t *ldb, const int *K, const int *btrans,
                          const double *alpha, void *C, int64_t ldc, double beta, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (nterms < 1 || nterms > 2) return qd_set_error(QD_ERR_ARG, "tsmm_nn: 1 or 2 terms");
    if (fp32) {
        TsTerm<float> t[2];
        for (int i = 0; i < nterms; i++)
            t[i] = {(const cpx<float> *)A[i], lda[i], (const cpx<float> *)B[i], ldb[i], K[i], btrans[i],
                    (float)alpha[i]};
        return tsmm_nn<float>(m, nc, nterms, t, (cpx<float> *)C, ldc, (float)beta, st);
    }
    TsTerm<double> t[2];
    for (int i = 0; i < nterms; i++)
        t[i] = {(const cpx<double> *)A[i], lda[i], (const cpx<double> *)B[i], ldb[i], K[i], btrans[i], alpha[i]};
    return tsmm_nn<double>(m, nc, nterms, t, (cpx<double> *)C, ldc, beta, st);
}

extern "C" int qd_tsmm_cn(int fp32, int m, const void *A, int64_t lda, int k1, const void *B, int64_t ldb, int nc,
                          void *C, int64_t ldc, void *scratch, size_t scratch_bytes, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (fp32)
        return tsmm_cn<float>(m, (const cpx<float> *)A, lda, k1, (const cpx<float> *)B, ldb, nc, (cpx<float> *)C, ldc,
                              (cpx<float> *)scratch, scratch_bytes, st);
    return tsmm_cn<double>(m, (const cpx<double> *)A, lda, k1, (const cpx<double> *)B, ldb, nc, (cpx<double> *)C, ldc,
                           (cpx<double> *)scratch, scratch_bytes, st);
}

extern "C" int qd_small_cn(int fp32, int k, int n1, int n2, const void *A, int lda, const void *B, int ldb,
                           double alpha, void *C, int ldc, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (fp32)
        return small_cn<float>(k, n1, n2, (const cpx<float> *)A, lda, (const cpx<float> *)B, ldb, (float)alpha,
                               (cpx<float> *)C, ldc, st);
    return small_cn<double>(k, n1, n2, (const cpx<double> *)A, lda, (const cpx<double> *)B, ldb, alpha,
                            (cpx<double> *)C, ldc, st);
}

// Stage 2 of the eigensolver and the tridiagonal / band eigenvector steps.
//
//  * hb2st_kernel: Hermitian band (half bandwidth b) -> real-diagonal
//    tridiagonal by Householder bulge chasing, eigenvalues only.  Sweep s
//    annihilates column s below the subdiagonal and chases the bulge down the
//    band in tasks of b rows.  Sweeps run concurrently in a persistent
//    cooperative kernel.  Task k >= 1 of sweep s reads and writes the block
//    E = A[s+kb+1 .. s+(k+1)b, s+(k-1)b+1 .. s+kb] and the diagonal block
//    D = A[s+kb+1 .. s+(k+1)b]^2 (task 0: column s and D = A[s+1 .. s+b]^2).
//    Task k+1 of sweep s-1 overlaps these (its D shares index s+(k+1)b and its
//    E the last row of D); task k+2 starts at row s+(k+2)b and column
//    s+(k+1)b and is disjoint.  So task k may start once sweep s-1 has finished
//    tasks 0..k+1 (progress counter >= k+2).  The wait is bounded.
//  * bisect_kernel: eigenvalues of the tridiagonal matrix with indices [lo, hi]
//    by multisection on Sturm counts (one warp per eigenvalue, 32 shifts per
//    step).  Selecting by index reproduces zheevr's RANGE='I' window.
//  * band_invit_kernel: eigenvectors of the band matrix by inverse iteration:
//    LU with partial pivoting of (B - lambda I) in a shared-memory window that
//    slides down the band, then three solves with the starting block of the
//    whole group of (numerically) degenerate eigenvalues and Gram-Schmidt within
//    the group (Kramers pairs are exactly degenerate).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "eig_common.cuh"
#include "qd_internal.h"

typedef cpx<double> zd;

// Polls before a wait on the previous sweep gives up (set at run time by
// qd_set_wait_limits; the default is about a second and a half of polling).
#define QD_SPIN_LIMIT_DEFAULT (1LL << 25)
__device__ long long g_spin_limit = QD_SPIN_LIMIT_DEFAULT;
#define PROGRESS_DONE 0x7fffffff
#define QD_INVIT_ITERS 2

__device__ __forceinline__ zd ldab(const double2 *AB, int ldb, int64_t i, int64_t j) {  // i >= j
    double2 v = __ldcg(&AB[(i - j) + j * (int64_t)ldb]);
    return mk<double>(v.x, v.y);
}
__device__ __forceinline__ void stab(double2 *AB, int ldb, int64_t i, int64_t j, zd v) {
    __stcg(&AB[(i - j) + j * (int64_t)ldb], make_double2(v.re, v.im));
}

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ bool wait_progress(const int *progress, int s_prev, int need, int *err) {
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        long long it = 0;
        const long long limit = g_spin_limit;
        while (ld_acquire(progress + s_prev) < need) {
            if (++it > limit || *(volatile int *)err) {
                atomicExch(err, QD_ERR_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
    }
    __syncthreads();
    return ok != 0;
}

// The block barrier orders every thread's stores before thread 0's release
// store (release at gpu scope is cumulative over what thread 0 has observed).
__device__ __forceinline__ void publish(int *progress, int s, int val) {
    __syncthreads();
    if (threadIdx.x == 0) st_release(progress + s, val);
}

// ---------------------------------------------------------------------------
// Warp-register helpers for the bulge chasing.  Blocks are at most 32 x 32;
// lane r holds row r, warp w holds the columns w + 8 i (i = 0..3).
// ---------------------------------------------------------------------------
#define HB_NW 8  // warps per block
#define HB_NC 4  // columns per thread (32 / HB_NW)

__device__ __forceinline__ zd shfl_z(zd a, int src) {
    return mk<double>(__shfl_sync(0xffffffffu, a.re, src), __shfl_sync(0xffffffffu, a.im, src));
}
__device__ __forceinline__ zd warp_sum_z(zd a) {
    for (int o = 16; o > 0; o >>= 1) {
        a.re += __shfl_xor_sync(0xffffffffu, a.re, o);
        a.im += __shfl_xor_sync(0xffffffffu, a.im, o);
    }
    return a;
}

// Householder reflector of the warp-distributed vector x (lane r holds x[r],
// zero for r >= len), zlarfg conventions: H^H x = beta e_0 with
// H = I - tau v v^H, v[0] = 1.  Every lane returns its v[r]; beta and tau are
// the same in all lanes.
__device__ __forceinline__ zd larfg_lanes(zd x, int len, double *beta_out, zd *tau_out) {
    const int r = threadIdx.x & 31;
    double s = warp_sum(r >= 1 && r < len ? cabs2(x) : 0.0);
    zd alpha = shfl_z(x, 0);
    double beta;
    zd tau, scale;
    if (s == 0.0 && alpha.im == 0.0) {
        beta = alpha.re;
        tau = mk<double>(0, 0);
        scale = mk<double>(0, 0);
    } else {
        beta = -copysign(sqrt(alpha.re * alpha.re + alpha.im * alpha.im + s), alpha.re);
        tau = mk<double>((beta - alpha.re) / beta, -alpha.im / beta);
        double dr = alpha.re - beta, di = alpha.im, den = dr * dr + di * di;
        scale = mk<double>(dr / den, -di / den);
    }
    *beta_out = beta;
    *tau_out = tau;
    if (r == 0) return mk<double>(1, 0);
    return r < len ? cmul(x, scale) : mk<double>(0, 0);
}

// Loads the Hermitian diagonal block D = A[r0 .. r0+len-1]^2 from the lower band.
__device__ __forceinline__ void load_diag_block(zd (&D)[HB_NC], const double2 *AB, int ldb, int64_t r0, int len) {
    const int r = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < HB_NC; i++) {
        int c = w + HB_NW * i;
        D[i] = mk<double>(0, 0);
        if (r < len && c < len) D[i] = r >= c ? ldab(AB, ldb, r0 + r, r0 + c) : cconj(ldab(AB, ldb, r0 + c, r0 + r));
    }
}

// Two-sided update D <- H^H D H with H = I - tau v v^H, given the partial sums
// of D v over this warp's columns; stores the lower triangle at (r0, r0).
// part: HB_NW x 32 shared scratch.  vr = v[r], vc[i] = v[w + 8 i].
__device__ __forceinline__ void diag_update_store(const zd (&D)[HB_NC], zd dv_part, zd vr, const zd (&vc)[HB_NC],
                                                  zd tau, int len, zd (*part)[32], double2 *AB, int ldb, int64_t r0) {
    const int r = threadIdx.x & 31, w = threadIdx.x >> 5;
    part[w][r] = dv_part;
    __syncthreads();
    zd u = mk<double>(0, 0);
#pragma unroll
    for (int q = 0; q < HB_NW; q++) u = cadd(u, part[q][r]);
    u = cmul(tau, u);  // u = tau D v
    double c = warp_sum(cmulc(tau, cmulc(vr, u)).re);  // Re(conj(tau) v^H u)
    u = csub(u, mk<double>(0.5 * c * vr.re, 0.5 * c * vr.im));
#pragma unroll
    for (int i = 0; i < HB_NC; i++) {
        int col = w + HB_NW * i;
        zd uc = shfl_z(u, col);
        zd val = csub(D[i], cadd(cmul(vr, cconj(uc)), cmul(u, cconj(vc[i]))));
        if (r == col) val.im = 0.0;
        if (r < len && col < len && r >= col) stab(AB, ldb, r0 + r, r0 + col, val);
    }
}

// Bulge chasing, one sweep per block at a time.  Task 0 of sweep s annihilates
// column s below the subdiagonal: v from A[s+1 .., s], then the two-sided update
// of D = A[s+1 .. s+b]^2.  Task k >= 1 applies the previous reflector to
// E = A[J1 .. J2, st .. ed] from the right, annihilates E[:, 0] below its first
// row with a new reflector applied from the left to E and two-sided to
// D = A[J1 .. J2]^2.  E and D live in registers; every warp forms the reflector
// itself from its own copy of the first column, so a task has two block
// barriers (the row sums E v and D v cross the warps).
__global__ void __launch_bounds__(256, 3) hb2st_kernel(double2 *AB, int ldb, int n, int b, int *progress, int *err) {
    __shared__ zd partA[HB_NW][32];
    __shared__ zd partB[HB_NW][32];
    const int r = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int s = blockIdx.x; s < n - 1; s += gridDim.x) {
        if (s > 0 && !wait_progress(progress, s - 1, 2, err)) return;
        int st = s + 1, ed = min(s + b, n - 1), len = ed - st + 1;
        zd D[HB_NC], E[HB_NC], vc[HB_NC];
        zd x = r < len ? ldab(AB, ldb, st + r, s) : mk<double>(0, 0);
        load_diag_block(D, AB, ldb, st, len);
        double beta;
        zd tau;
        zd vr = larfg_lanes(x, len, &beta, &tau);
        if (w == 0 && r < len) stab(AB, ldb, st + r, s, r == 0 ? mk<double>(beta, 0.0) : mk<double>(0, 0));
        zd dv = mk<double>(0, 0);
#pragma unroll
        for (int i = 0; i < HB_NC; i++) {
            vc[i] = shfl_z(vr, w + HB_NW * i);
            dv = cadd(dv, cmul(D[i], vc[i]));
        }
        diag_update_store(D, dv, vr, vc, tau, len, partB, AB, ldb, st);
        publish(progress, s, 1);
        int k = 1;
        while (true) {
            int J1 = ed + 1;
            if (J1 > n - 1) break;
            int J2 = min(ed + b, n - 1), lm = J2 - J1 + 1;
            if (s > 0 && !wait_progress(progress, s - 1, k + 2, err)) return;
            // all loads of the task in flight at once
            zd e0 = r < lm ? ldab(AB, ldb, J1 + r, st) : mk<double>(0, 0);  // E[:, 0], every warp
#pragma unroll
            for (int i = 0; i < HB_NC; i++) {
                int c = w + HB_NW * i;
                E[i] = r < lm && c < len ? ldab(AB, ldb, J1 + r, st + c) : mk<double>(0, 0);
            }
            load_diag_block(D, AB, ldb, J1, lm);
            // right application of the previous reflector: E <- E - (tau E v) v^H
            zd ev = mk<double>(0, 0);
#pragma unroll
            for (int i = 0; i < HB_NC; i++) ev = cadd(ev, cmul(E[i], vc[i]));
            partA[w][r] = ev;
            __syncthreads();
            zd wr = mk<double>(0, 0);
#pragma unroll
            for (int q = 0; q < HB_NW; q++) wr = cadd(wr, partA[q][r]);
            wr = cmul(tau, wr);
#pragma unroll
            for (int i = 0; i < HB_NC; i++) E[i] = csub(E[i], cmul(wr, cconj(vc[i])));
            e0 = csub(e0, wr);  // v[0] = 1
            // new reflector from the updated first column (formed in every warp)
            double beta2;
            zd tau2;
            zd v2r = larfg_lanes(e0, lm, &beta2, &tau2);
            zd v2c[HB_NC];
            zd dv2 = mk<double>(0, 0);
#pragma unroll
            for (int i = 0; i < HB_NC; i++) {
                v2c[i] = shfl_z(v2r, w + HB_NW * i);
                dv2 = cadd(dv2, cmul(D[i], v2c[i]));
            }
            // left application to E: E <- E - v2 (conj(tau2) v2^H E), column 0 -> beta2 e_0
#pragma unroll
            for (int i = 0; i < HB_NC; i++) {
                int c = w + HB_NW * i;
                zd wl = warp_sum_z(cmulc(v2r, E[i]));
                wl = cmul(cconj(tau2), wl);
                if (r < lm && c < len) {
                    zd val;
                    if (c == 0) val = r == 0 ? mk<double>(beta2, 0.0) : mk<double>(0, 0);
                    else val = csub(E[i], cmul(v2r, wl));
                    stab(AB, ldb, J1 + r, st + c, val);
                }
            }
            diag_update_store(D, dv2, v2r, v2c, tau2, lm, partB, AB, ldb, J1);
#pragma unroll
            for (int i = 0; i < HB_NC; i++) vc[i] = v2c[i];
            tau = tau2;
            st = J1;
            ed = J2;
            len = lm;
            k++;
            publish(progress, s, k);
        }
        publish(progress, s, PROGRESS_DONE);
    }
}

// d[i] = AB(i, i) (real), e[i] = |AB(i+1, i)|^2 (squared off-diagonal moduli)
__global__ void tri_extract_kernel(const double2 *AB, int ldb, int n, double *d, double *e2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    d[i] = AB[(int64_t)i * ldb].x;
    if (i < n - 1) {
        double2 e = AB[1 + (int64_t)i * ldb];
        e2[i] = e.x * e.x + e.y * e.y;
    }
}

// Gershgorin bounds and the pivot floor (LAPACK dlaebz/dstebz conventions)
__global__ void gersh_kernel(const double *d, const double *e2, int n, double *out /*gl, gu, pivmin*/) {
    double gl = 1e300, gu = -1e300, emax = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double r = (i > 0 ? sqrt(e2[i - 1]) : 0.0) + (i < n - 1 ? sqrt(e2[i]) : 0.0);
        gl = fmin(gl, d[i] - r);
        gu = fmax(gu, d[i] + r);
        if (i < n - 1) emax = fmax(emax, e2[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        gl = fmin(gl, __shfl_xor_sync(0xffffffffu, gl, o));
        gu = fmax(gu, __shfl_xor_sync(0xffffffffu, gu, o));
        emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    }
    __shared__ double sg[3][32];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { sg[0][w] = gl; sg[1][w] = gu; sg[2][w] = emax; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < (int)(blockDim.x >> 5); q++) {
            gl = fmin(gl, sg[0][q]); gu = fmax(gu, sg[1][q]); emax = fmax(emax, sg[2][q]);
        }
        double tnorm = fmax(fabs(gl), fabs(gu));
        double pad = 2.1 * 2.220446049250313e-16 * tnorm * n;
        out[0] = gl - pad;
        out[1] = gu + pad;
        out[2] = 2.2250738585072014e-308 * fmax(1.0, emax);
    }
}

__device__ int sturm_count(const double *d, const double *e2, int n, double x, double pivmin) {
    int c = 0;
    double q = d[0] - x;
    if (fabs(q) <= pivmin) q = -pivmin;
    c += q < 0.0;
    for (int i = 1; i < n; i++) {
        q = d[i] - x - e2[i - 1] / q;
        if (fabs(q) <= pivmin) q = -pivmin;
        c += q < 0.0;
    }
    return c;
}

// One warp per wanted index k in [lo, hi]: interval [a, b] with count(a) <= k < count(b).
__global__ void bisect_kernel(const double *d, const double *e2, int n, int lo, int hi, const double *bounds,
                              double *w) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int k = lo + warp;
    if (k > hi) return;
    double a = bounds[0], bnd = bounds[1], pivmin = bounds[2];
    for (int it = 0; it < 64; it++) {
        double width = bnd - a;
        double tol = 2.0 * 2.220446049250313e-16 * fmax(fabs(a), fabs(bnd)) + 4.0 * pivmin;
        if (width <= tol) break;
        double x = a + width * (double)(lane + 1) / 33.0;
        int c = sturm_count(d, e2, n, x, pivmin);
        unsigned above = __ballot_sync(0xffffffffu, c > k);
        int first = above ? __ffs(above) - 1 : 32;  // smallest lane with count > k
        double na = first == 0 ? a : a + width * (double)first / 33.0;
        double nb = first == 32 ? bnd : a + width * (double)(first + 1) / 33.0;
        a = na;
        bnd = nb;
    }
    if (lane == 0) w[k - lo] = 0.5 * (a + bnd);
}

// ---------------------------------------------------------------------------
// Band inverse iteration.  One block per group of degenerate eigenvalues.
// B is the Hermitian band before stage 2 (AB0, lower, offsets 0..b, ldb).
// Workspace per group: L (n x b), U (n x (2b+1)), ipiv (n).
// ---------------------------------------------------------------------------
__device__ __forceinline__ zd band_val(const double2 *AB, int ldb, int b, int n, int64_t i, int64_t c, double lam) {
    if (i < 0 || c < 0 || i >= n || c >= n) return mk<double>(0, 0);
    int64_t d = i - c;
    zd v;
    if (d >= 0) {
        if (d > b) return mk<double>(0, 0);
        double2 x = AB[d + c * (int64_t)ldb];
        v = mk<double>(x.x, x.y);
    } else {
        if (-d > b) return mk<double>(0, 0);
        double2 x = AB[-d + i * (int64_t)ldb];
        v = mk<double>(x.x, -x.y);
    }
    if (d == 0) v.re -= lam;
    return v;
}

#define IW_ROWS 64
#define IW_COLS 128
#define IW(i, c) ((((i) & (IW_ROWS - 1)) * IW_COLS) + ((c) & (IW_COLS - 1)))

__global__ void __launch_bounds__(256) band_invit_kernel(const double2 *AB, int ldb, int n, int b, const double *lam,
                                                         const int *group_start, const int *group_size, double2 *Lw,
                                                         double2 *Uw, int *ipivw, double2 *Z, int64_t ldz,
                                                         double bnorm, double2 *ywork) {
    extern __shared__ unsigned char sm_raw[];
    const int cols = 2 * b + 1;
    // Circular window of the banded LU, 64 row slots x 128 column slots (b <= 32):
    // (i, c) lives in W[IW(i, c)].  The live rows j..j+b and columns j..j+2b
    // never share a slot with the row and column that enter at step j.
    zd *W = (zd *)sm_raw;
    zd *lcol = W + IW_ROWS * IW_COLS;  // b multipliers of the current step
    __shared__ double scratch[33];
    __shared__ int s_piv;
    __shared__ zd s_inv;
    int g = blockIdx.x;
    int m0 = group_start[g], gs = group_size[g];
    double lambda = lam[m0];
    double2 *L = Lw + (int64_t)g * n * b;
    double2 *U = Uw + (int64_t)g * n * cols;
    int *ipiv = ipivw + (int64_t)g * n;
    for (int idx = threadIdx.x; idx < (b + 1) * cols; idx += blockDim.x) {
        int i = idx / cols, c = idx % cols;
        W[IW(i, c)] = band_val(AB, ldb, b, n, i, c, lambda);
    }
    // Values entering at step j (original matrix entries, so fetched one step
    // ahead): thread t < 2b+1 holds (j+b+1, j+1+t), thread 2b+1+k (k < b)
    // holds (j+1+k, j+2b+1).
    auto incoming = [&](int j) -> zd {
        const int t = threadIdx.x;
        if (t < cols) return band_val(AB, ldb, b, n, j + b + 1, j + 1 + t, lambda);
        if (t < cols + b) return band_val(AB, ldb, b, n, j + 1 + (t - cols), j + 2 * b + 1, lambda);
        return mk<double>(0, 0);
    };
    zd in_next = incoming(0);
    __syncthreads();
    const double tiny = 2.220446049250313e-16 * bnorm;
    for (int j = 0; j < n; j++) {
        int imax = min(j + b, n - 1), cmax = min(j + 2 * b, n - 1);
        const zd in_cur = in_next;
        if (j + 1 < n) in_next = incoming(j + 1);
        if (threadIdx.x < 32) {
            // pivot search in column j, rows j..imax
            double best = -1.0;
            int bi = j;
            for (int i = j + threadIdx.x; i <= imax; i += 32) {
                double a = cabs2(W[IW(i, j)]);
                if (a > best) { best = a; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (threadIdx.x == 0) s_piv = bi;
            __syncwarp();
            int p = bi;
            if (p != j) {
                for (int c = j + threadIdx.x; c <= cmax; c += 32) {
                    zd t = W[IW(j, c)];
                    W[IW(j, c)] = W[IW(p, c)];
                    W[IW(p, c)] = t;
                }
            }
            __syncwarp();
            if (threadIdx.x == 0) {
                zd piv = W[IW(j, j)];
                double a2 = cabs2(piv);
                if (a2 < tiny * tiny) {
                    piv = mk<double>(tiny, 0.0);
                    W[IW(j, j)] = piv;
                    a2 = tiny * tiny;
                }
                s_inv = mk<double>(piv.re / a2, -piv.im / a2);
            }
            __syncwarp();
            for (int i = j + 1 + threadIdx.x; i <= imax; i += 32) {
                zd l = cmul(W[IW(i, j)], s_inv);
                lcol[i - j - 1] = l;
                L[(int64_t)j * b + (i - j - 1)] = make_double2(l.re, l.im);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) ipiv[j] = s_piv;
        // U row j, the rank-1 update of the live window (lanes along columns,
        // four row groups) and the entering row and column, all in one phase
        for (int c = j + threadIdx.x; c < j + cols; c += blockDim.x) {
            zd u = c <= cmax ? W[IW(j, c)] : mk<double>(0, 0);
            U[(int64_t)j * cols + (c - j)] = make_double2(u.re, u.im);
        }
        const int nr = imax - j, nc = cmax - j;
        {
            const int cc = threadIdx.x & 63, rg = threadIdx.x >> 6;
            if (cc < nc) {
                const int c = j + 1 + cc;
                const zd top = W[IW(j, c)];
                for (int ri = rg; ri < nr; ri += 4) {
                    zd *a = &W[IW(j + 1 + ri, c)];
                    *a = csub(*a, cmul(lcol[ri], top));
                }
            }
        }
        if ((int)threadIdx.x < cols) W[IW(j + b + 1, j + 1 + threadIdx.x)] = in_cur;
        else if ((int)threadIdx.x < cols + b) W[IW(j + 1 + (threadIdx.x - cols), j + 2 * b + 1)] = in_cur;
        __syncthreads();
    }
    // ---- inverse iteration on the group's block of vectors (one warp per vector).
    // The forward and backward sweeps keep their active windows (b+1 and 2b+1
    // entries) in per-warp circular buffers in shared memory.
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    zd *fb = lcol + b + warp * 192;  // 64 slots forward window
    zd *bb = fb + 64;                // 128 slots backward window
    for (int it = 0; it < QD_INVIT_ITERS; it++) {
        for (int q = warp; q < gs; q += nwarp) {
            double2 *y = ywork + ((int64_t)blockIdx.x * 8 + warp) * n;
            double2 *x = Z + (int64_t)(m0 + q) * ldz;
            auto rhs = [&](int i) -> zd {
                if (it == 0) {
                    unsigned h = (unsigned)(i * 2654435761u) ^ (unsigned)((m0 + q + 1) * 40503u);
                    h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
                    unsigned h2 = h * 2246822519u + 374761393u;
                    return mk<double>((double)(h & 0xffff) / 65536.0 - 0.5, (double)(h2 & 0xffff) / 65536.0 - 0.5);
                }
                double2 t = x[i];
                return mk<double>(t.x, t.y);
            };
            for (int i = lane; i <= b && i < n; i += 32) fb[i & 63] = rhs(i);
            __syncwarp();
            // forward: P and L (the next step's pivot and multipliers are fetched ahead)
            int p_next = ipiv[0];
            double2 l_next = lane < b ? L[lane] : make_double2(0.0, 0.0);
            for (int j = 0; j < n; j++) {
                int p = p_next;
                double2 l = l_next;
                if (j + 1 < n) {
                    p_next = ipiv[j + 1];
                    if (lane < b) l_next = L[(int64_t)(j + 1) * b + lane];
                }
                if (lane == 0 && p != j) {
                    zd t = fb[j & 63];
                    fb[j & 63] = fb[p & 63];
                    fb[p & 63] = t;
                }
                __syncwarp();
                zd yj = fb[j & 63];
                int i = j + 1 + lane;
                if (lane < b && i < n) fb[i & 63] = csub(fb[i & 63], cmul(mk<double>(l.x, l.y), yj));
                if (lane == 0) y[j] = make_double2(yj.re, yj.im);
                if (lane == 1 && j + b + 1 < n) fb[(j + b + 1) & 63] = rhs(j + b + 1);
                __syncwarp();
            }
            // backward: U x = y (row j of U fetched one step ahead)
            auto urow = [&](int j, double2 &u0, double2 &u1, double2 &ud, double2 &yy) {
                int c0 = j + 1 + lane, c1 = j + 33 + lane, cend = min(j + 2 * b, n - 1);
                u0 = c0 <= cend ? U[(int64_t)j * cols + (c0 - j)] : make_double2(0.0, 0.0);
                u1 = c1 <= cend ? U[(int64_t)j * cols + (c1 - j)] : make_double2(0.0, 0.0);
                ud = U[(int64_t)j * cols];
                yy = y[j];
            };
            double2 nu0, nu1, nud, nyy;
            urow(n - 1, nu0, nu1, nud, nyy);
            for (int j = n - 1; j >= 0; j--) {
                double2 u0 = nu0, u1 = nu1, ud = nud, yy = nyy;
                if (j > 0) urow(j - 1, nu0, nu1, nud, nyy);
                int c0 = j + 1 + lane, c1 = j + 33 + lane;
                int cend = min(j + 2 * b, n - 1);
                zd x0 = c0 <= cend ? bb[c0 & 127] : mk<double>(0, 0);
                zd x1 = c1 <= cend ? bb[c1 & 127] : mk<double>(0, 0);
                double sr = u0.x * x0.re - u0.y * x0.im + u1.x * x1.re - u1.y * x1.im;
                double si = u0.x * x0.im + u0.y * x0.re + u1.x * x1.im + u1.y * x1.re;
                sr = warp_sum(sr);
                si = warp_sum(si);
                if (lane == 0) {
                    double rr = yy.x - sr, ri = yy.y - si;
                    double den = ud.x * ud.x + ud.y * ud.y;
                    zd xj = mk<double>((rr * ud.x + ri * ud.y) / den, (ri * ud.x - rr * ud.y) / den);
                    bb[j & 127] = xj;
                    x[j] = make_double2(xj.re, xj.im);
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // modified Gram-Schmidt within the group (block-wide reductions)
        for (int q = 0; q < gs; q++) {
            double2 *xq = Z + (int64_t)(m0 + q) * ldz;
            for (int p = 0; p < q; p++) {
                double2 *xp = Z + (int64_t)(m0 + p) * ldz;
                double sr = 0.0, si = 0.0;
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    double2 a = xp[i], c = xq[i];
                    sr += a.x * c.x + a.y * c.y;
                    si += a.x * c.y - a.y * c.x;
                }
                sr = block_sum(sr, scratch);
                si = block_sum(si, scratch);
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    double2 a = xp[i], c = xq[i];
                    c.x -= sr * a.x - si * a.y;
                    c.y -= sr * a.y + si * a.x;
                    xq[i] = c;
                }
                __syncthreads();
            }
            double nn = 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) nn += xq[i].x * xq[i].x + xq[i].y * xq[i].y;
            nn = block_sum(nn, scratch);
            double inv = nn > 0.0 ? 1.0 / sqrt(nn) : 0.0;
            for (int i = threadIdx.x; i < n; i += blockDim.x) xq[i] = make_double2(xq[i].x * inv, xq[i].y * inv);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Host wrappers
// ---------------------------------------------------------------------------
#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int qd_stage2_set_wait_limit(long long polls) {
    const long long v = polls < 0 ? QD_SPIN_LIMIT_DEFAULT : polls;
    CUDA_OK(cudaMemcpyToSymbol(g_spin_limit, &v, sizeof(v)));
    return QD_OK;
}

extern "C" int qd_hb2st(double2 *AB, int ldb, int n, int b, int *progress, int *err, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    int dev, nsm, per_sm = 0;
    CUDA_OK(cudaGetDevice(&dev));
    CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CUDA_OK(cudaMemsetAsync(progress, 0, sizeof(int) * (size_t)n, st));
    CUDA_OK(cudaMemsetAsync(err, 0, sizeof(int), st));
    if (b < 1 || b > 32) return qd_set_error(QD_ERR_UNSUPPORTED, "bulge chasing needs 1 <= b <= 32");
    void *args[] = {&AB, &ldb, &n, &b, &progress, &err};
    const size_t smem = 0;
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hb2st_kernel, 256, smem));
    if (per_sm < 1) return qd_set_error(QD_ERR_CUDA, "hb2st kernel does not fit on an SM");
    int G = qd_sm_budget(nsm) * per_sm;
    int useful = n / (2 * b) + 2;  // concurrent sweeps are limited by the 2-task lag
    if (G > useful) G = useful;
    if (G > n - 1) G = n - 1;
    if (G < 1) G = 1;
    qd_count_launch(1);
    CUDA_OK(cudaLaunchCooperativeKernel((void *)hb2st_kernel, dim3(G), dim3(256), args, smem, st));
    return QD_OK;
}

extern "C" int qd_tridiag_bisect(const double2 *AB, int ldb, int n, int lo, int hi, double *d, double *e2,
                                 double *bounds, double *w, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    qd_count_launch(3);
    tri_extract_kernel<<<(n + 255) / 256, 256, 0, st>>>(AB, ldb, n, d, e2);
    gersh_kernel<<<1, 1024, 0, st>>>(d, e2, n, bounds);
    int m = hi - lo + 1;
    bisect_kernel<<<(m * 32 + 127) / 128, 128, 0, st>>>(d, e2, n, lo, hi, bounds, w);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

extern "C" int qd_band_invit(const double2 *AB0, int ldb, int n, int b, const double *lam_dev, int ngroups,
                             const int *gstart_dev, const int *gsize_dev, double2 *Lw, double2 *Uw, int *ipivw,
                             double2 *Z, int64_t ldz, double bnorm, double2 *ywork, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (b < 1 || b > 32) return qd_set_error(QD_ERR_UNSUPPORTED, "band inverse iteration needs 1 <= b <= 32");
    size_t smem = (size_t)(IW_ROWS * IW_COLS + b + 8 * 192) * sizeof(zd);
    CUDA_OK(cudaFuncSetAttribute(band_invit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    qd_count_launch(1);
    band_invit_kernel<<<ngroups, 256, smem, st>>>(AB0, ldb, n, b, lam_dev, gstart_dev, gsize_dev, Lw, Uw, ipivw, Z,
                                                  ldz, bnorm, ywork);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of qd_tridiag_bisect for callers that may not
// allocate device memory (see the declaration in qudos_b200.h).  The
// per-call scratch (diagonal, squared off-diagonal, Gershgorin bounds) lives
// in file-scope device arrays sized for QD_STATIC_TRI_MAX rows; the kernels
// and their launch shapes are those of qd_tridiag_bisect.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_static_tri_d[QD_STATIC_TRI_MAX];
static __device__ __align__(256) double g_static_tri_e2[QD_STATIC_TRI_MAX];
static __device__ __align__(256) double g_static_tri_bounds[4];

#define QD_STATIC_MAX_DEVICES 64
static double *g_static_addr[QD_STATIC_MAX_DEVICES][3];

extern "C" int qd_tridiag_eigvals_noalloc(const void *ABv, int ldb, int n, int lo, int hi, double *w,
                                          void *stream) {
    const double2 *AB = (const double2 *)ABv;
    if (n < 1 || n > QD_STATIC_TRI_MAX)
        return qd_set_error(QD_ERR_ARG, "qd_tridiag_eigvals_noalloc: n = %d outside [1, %d]", n, QD_STATIC_TRI_MAX);
    if (ldb < 2 || lo < 0 || hi < lo || hi >= n || !AB || !w)
        return qd_set_error(QD_ERR_ARG, "qd_tridiag_eigvals_noalloc: bad arguments (ldb %d, window [%d, %d])", ldb,
                            lo, hi);
    int dev = 0;
    CUDA_OK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= QD_STATIC_MAX_DEVICES)
        return qd_set_error(QD_ERR_ARG, "qd_tridiag_eigvals_noalloc: device %d not supported", dev);
    double **a = g_static_addr[dev];
    double *d0 = __atomic_load_n(&a[0], __ATOMIC_ACQUIRE);
    if (!d0) {  // first call on this device: resolve the scratch addresses once
        void *p0 = nullptr, *p1 = nullptr, *p2 = nullptr;
        CUDA_OK(cudaGetSymbolAddress(&p0, g_static_tri_d));
        CUDA_OK(cudaGetSymbolAddress(&p1, g_static_tri_e2));
        CUDA_OK(cudaGetSymbolAddress(&p2, g_static_tri_bounds));
        // a[1] and a[2] are published by the release store of a[0]; a thread
        // that sees a[0] through the acquire load above also sees them
        __atomic_store_n(&a[1], (double *)p1, __ATOMIC_RELAXED);
        __atomic_store_n(&a[2], (double *)p2, __ATOMIC_RELAXED);
        __atomic_store_n(&a[0], (double *)p0, __ATOMIC_RELEASE);
        d0 = (double *)p0;
    }
    double *e2s = __atomic_load_n(&a[1], __ATOMIC_RELAXED), *bnds = __atomic_load_n(&a[2], __ATOMIC_RELAXED);
    // Every scratch element that is read is written first in the same call
    // (d and e2 for the n rows by tri_extract_kernel, the bounds by
    // gersh_kernel), so nothing needs clearing.
    cudaStream_t st = (cudaStream_t)stream;
    qd_count_launch(3);
    tri_extract_kernel<<<(n + 255) / 256, 256, 0, st>>>(AB, ldb, n, d0, e2s);
    gersh_kernel<<<1, 1024, 0, st>>>(d0, e2s, n, bnds);
    int m = hi - lo + 1;
    bisect_kernel<<<(m * 32 + 127) / 128, 128, 0, st>>>(d0, e2s, n, lo, hi, bnds, w);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// Real-space envelope functions of plane-wave eigenstates
// (code/source/8_band/envelope_functions.c:23-220):
//   F_b(r) = sum_G a_{b, G} exp(i (G + K) . r) / sqrt(L1 L2 L3),  b = 1..8,
// and the band-resolved probability densities |F_b(r)|^2, at arbitrary
// points r (line scans, cross-sections and 3-D grids of the reference's
// real_space_grid_* routines).
//
// One CTA per (point, state): the threads stride over the plane waves, each
// evaluates its phase once and accumulates all eight band components, and a
// block reduction gives the eight sums.  The coefficient reads of a warp are
// 32 consecutive rows of one band of the state (coalesced).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "qd_internal.h"

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr int ENV_THREADS = 256;

struct EnvGeom {
    int N[3], off[3];
    const double *G[3];
    double K[3];
    double inv_sqrt_vol;
};

__global__ void __launch_bounds__(ENV_THREADS) envelope_kernel(EnvGeom g, const double2 *__restrict__ Z, int64_t ldz,
                                                               int npw, const double *__restrict__ x,
                                                               const double *__restrict__ y,
                                                               const double *__restrict__ z, int n_grid,
                                                               double2 *__restrict__ F, double *__restrict__ prob) {
    __shared__ double red[ENV_THREADS / 32][16];
    const int p = blockIdx.x, s = blockIdx.y;
    const double rx = x[p], ry = y[p], rz = z[p];
    const double2 *zs = Z + (int64_t)s * ldz;
    double acc[16];
#pragma unroll
    for (int b = 0; b < 16; b++) acc[b] = 0.0;
    const int nyz = g.N[1] * g.N[2];
    for (int pw = threadIdx.x; pw < npw; pw += ENV_THREADS) {
        const int ix = pw / nyz, iy = (pw / g.N[2]) % g.N[1], iz = pw % g.N[2];
        const double arg = (g.G[0][g.off[0] + ix] + g.K[0]) * rx + (g.G[1][g.off[1] + iy] + g.K[1]) * ry +
                           (g.G[2][g.off[2] + iz] + g.K[2]) * rz;
        double sn, cs;
        sincos(arg, &sn, &cs);
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const double2 a = zs[(int64_t)b * npw + pw];
            acc[2 * b] += a.x * cs - a.y * sn;
            acc[2 * b + 1] += a.x * sn + a.y * cs;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int b = 0; b < 16; b++) {
        double v = acc[b];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[w][b] = v;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int b = threadIdx.x;
        double re = 0.0, im = 0.0;
        for (int q = 0; q < ENV_THREADS / 32; q++) {
            re += red[q][2 * b];
            im += red[q][2 * b + 1];
        }
        re *= g.inv_sqrt_vol;
        im *= g.inv_sqrt_vol;
        const int64_t o = ((int64_t)s * 8 + b) * n_grid + p;
        if (F) F[o] = make_double2(re, im);
        if (prob) prob[o] = re * re + im * im;
    }
}

}  // namespace

// Device envelopes: Z (N_H x m, device), points x, y, z (n_grid each, device,
// Angstrom), G grids (device, 2N-1 per axis), outputs F and prob (device,
// [state][band][point]; either may be null).
extern "C" int qd_envelope_dev(const int N[3], const double *d_Gx, const double *d_Gy, const double *d_Gz,
                               const double K[3], double volume, const void *Z, int64_t ldz, int m, int n_grid,
                               const double *x, const double *y, const double *z, void *F, double *prob,
                               void *stream) {
    if (m < 1 || n_grid < 1 || volume <= 0.0 || m > 65535)
        return qd_set_error(QD_ERR_ARG, "qd_envelope_dev: bad sizes (m %d, points %d)", m, n_grid);
    EnvGeom g;
    for (int a = 0; a < 3; a++) {
        g.N[a] = N[a];
        g.off[a] = (2 * N[a] - 1) / 2 - N[a] / 2;
        g.K[a] = K[a];
    }
    g.G[0] = d_Gx;
    g.G[1] = d_Gy;
    g.G[2] = d_Gz;
    g.inv_sqrt_vol = 1.0 / sqrt(volume);
    const int npw = N[0] * N[1] * N[2];
    qd_count_launch(1);
    envelope_kernel<<<dim3((unsigned)n_grid, (unsigned)m), ENV_THREADS, 0, (cudaStream_t)stream>>>(
        g, (const double2 *)Z, ldz, npw, x, y, z, n_grid, (double2 *)F, prob);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

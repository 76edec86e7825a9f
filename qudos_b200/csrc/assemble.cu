// 8-band supercell Hamiltonian assembly (hamiltonian_8_band.c:23-500 with the
// band functions of hamiltonian_8_band_matrix_elements.c:27-969).
//
// Every element H[(b1,G1),(b2,G2)] is a band-dependent polynomial in G1 and G2
// whose coefficients depend only on the difference G1 - G2.  Those coefficients
// are precomputed once per difference (fused_coef_kernel, 28 complex fields,
// field-major so a warp's gathers are contiguous); this kernel then only
// evaluates the polynomial and streams the result out.  It is bound by the
// HBM write of H: 16 bytes per element (complex128), 8 (complex64), 24 (both).
//
// Layout: column-major, H[row + ld * col], row = band * N_PW + (ix N_y + iy) N_z + iz.
// mode 0 writes the lower triangle only (the reference's layout; the strict upper
// triangle of the caller's buffer is not touched); mode 1 writes both triangles
// (upper = conjugate transpose, evaluated directly so every store stays coalesced).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "qd_complex.cuh"
#include "qd_internal.h"

namespace {

enum { F_ZERO = 0, F_ECB, F_EHH, F_ELH, F_ESO, F_Q, F_R, F_RC, F_S, F_SC, F_TP, F_TM, F_U };

// (row band, column band) for row band >= column band, 0-based (hamiltonian_8_band.c:78-492)
__constant__ signed char c_func[8][8];
__constant__ double c_fac[8][8];

struct Ctx {
    const double2 *__restrict__ coef;
    int64_t nT;
    const double *__restrict__ G[3];
    int N[3], NT[3], off[3];
    double K[3];
};

__device__ __forceinline__ zc ld(const Ctx &c, int k, int64_t t) { return zc(__ldg(&c.coef[k * c.nT + t])); }

__device__ zc band_element(const Ctx &c, int rb, int cb, const int r[3], const int q[3]) {
    int f = c_func[rb][cb];
    if (f == F_ZERO) return zc(0.0);
    int64_t t = ((int64_t)(r[0] - q[0] + c.NT[0] / 2) * c.NT[1] + (r[1] - q[1] + c.NT[1] / 2)) * c.NT[2] +
                (r[2] - q[2] + c.NT[2] / 2);
    double g1x = c.G[0][c.off[0] + r[0]], g1y = c.G[1][c.off[1] + r[1]], g1z = c.G[2][c.off[2] + r[2]];
    double g2x = c.G[0][c.off[0] + q[0]], g2y = c.G[1][c.off[1] + q[1]], g2z = c.G[2][c.off[2] + q[2]];
    double Kx = c.K[0], Ky = c.K[1], Kz = c.K[2];
    double kinx = g1x * g2x + Kx * (g1x + g2x), kiny = g1y * g2y + Ky * (g1y + g2y),
           kinz = g1z * g2z + Kz * (g1z + g2z);
    const double H2 = 0.5 * QD_HBSQM;
    zc v;
    switch (f) {
        case F_ECB:
            v = ld(c, 0, t) + H2 * ld(c, 1, t) * (kinx + kiny + kinz + Kx * Kx + Ky * Ky + Kz * Kz) + ld(c, 13, t);
            break;
        case F_EHH:
            v = ld(c, 2, t) - H2 * ld(c, 3, t) * (kinx + kiny + Kx * Kx + Ky * Ky) -
                H2 * ld(c, 4, t) * (kinz + Kz * Kz) + ld(c, 14, t);
            break;
        case F_ELH:
            v = ld(c, 5, t) - H2 * ld(c, 6, t) * (kinx + kiny + Kx * Kx + Ky * Ky) -
                H2 * ld(c, 7, t) * (kinz + Kz * Kz) + ld(c, 15, t);
            break;
        case F_ESO:
            v = ld(c, 8, t) - H2 * ld(c, 9, t) * (kinx + kiny + kinz + Kx * Kx + Ky * Ky + Kz * Kz) + ld(c, 16, t);
            break;
        case F_Q: {
            zc g2 = ld(c, 10, t);
            v = (-sqrt(0.5) * QD_HBSQM) * g2 * (kinx + kiny + Kx * Kx + Ky * Ky) +
                (sqrt(2.0) * QD_HBSQM) * g2 * (kinz + Kz * Kz) + ld(c, 17, t);
            break;
        }
        case F_R:
        case F_RC: {
            double sg = f == F_R ? -1.0 : 1.0;
            double a = 0.5 * sqrt(3.0) * QD_HBSQM;
            zc kin = a * ld(c, 10, t) * (kinx - kiny + Kx * Kx - Ky * Ky);
            zc off = (sg * a) * ld(c, 11, t) * ((g1x + Kx) * (g2y + Ky) + (g1y + Ky) * (g2x + Kx));
            zc rd = ld(c, 19, t);
            v = kin + I_times(off) + ld(c, 18, t) - sg * I_times(rd);
            break;
        }
        case F_S:
        case F_SC: {
            double sg = f == F_S ? -1.0 : 1.0;
            double a = 0.5 * sqrt(1.5) * QD_HBSQM;
            zc g3 = ld(c, 11, t);
            zc re = a * g3 * ((g1x + Kx) * (g2z + Kz) + (g1z + Kz) * (g2x + Kx));
            zc im = (sg * a) * g3 * ((g1y + Ky) * (g2z + Kz) + (g1z + Kz) * (g2y + Ky));
            zc sxz = ld(c, 20, t), syz = ld(c, 21, t);
            v = re + I_times(im) - sqrt(0.5) * (sxz + sg * I_times(syz));
            break;
        }
        case F_TP:
        case F_TM: {
            double sg = f == F_TP ? 1.0 : -1.0;
            double kx = g1x + g2x + 2 * Kx, ky = g1y + g2y + 2 * Ky, kz = g1z + g2z + 2 * Kz;
            zc P = ld(c, 12, t);
            zc Txx = ld(c, 22, t), Txy = ld(c, 23, t), Tyy = ld(c, 24, t), Txz = ld(c, 25, t), Tyz = ld(c, 26, t);
            double c6 = -0.5 / sqrt(6.0);
            zc s = (Txx + sg * I_times(Txy)) * kx + (Txy + sg * I_times(Tyy)) * ky + (Txz + sg * I_times(Tyz)) * kz;
            v = (P * kx) / (2.0 * sqrt(6.0)) + sg * I_times(P * ky) / (2.0 * sqrt(6.0)) + c6 * s;
            break;
        }
        case F_U: {
            double kx = g1x + g2x + 2 * Kx, ky = g1y + g2y + 2 * Ky, kz = g1z + g2z + 2 * Kz;
            zc P = ld(c, 12, t);
            double c3 = -0.5 / sqrt(3.0);
            v = (P * kz) / (2.0 * sqrt(3.0)) + c3 * (ld(c, 25, t) * kx + ld(c, 26, t) * ky + ld(c, 27, t) * kz);
            break;
        }
    }
    return c_fac[rb][cb] * v;
}

// Band-block map of hamiltonian_8_band.c:78-492 as compile-time functions of
// (row band, column band), row band >= column band, 0-based; the same table
// as upload_block_map below, in a form the unrolled block loop folds away.
__host__ __device__ constexpr int bfunc(int rb, int cb) {
    switch (rb * 8 + cb) {
        case 0: return F_ECB;  case 8: return F_TM;  case 16: return F_U;   case 24: return F_U;
        case 48: return F_TP;  case 56: return F_TP;
        case 9: return F_EHH;  case 17: return F_SC; case 25: return F_SC;  case 49: return F_RC; case 57: return F_RC;
        case 18: return F_ELH; case 26: return F_Q;  case 34: return F_TP;  case 42: return F_RC; case 58: return F_SC;
        case 27: return F_ESO; case 35: return F_TP; case 43: return F_RC;  case 51: return F_SC;
        case 36: return F_ECB; case 44: return F_TP; case 52: return F_U;   case 60: return F_U;
        case 45: return F_EHH; case 53: return F_S;  case 61: return F_S;
        case 54: return F_ELH; case 62: return F_Q;
        case 63: return F_ESO;
        default: return F_ZERO;
    }
}
__host__ __device__ constexpr double bfac(int rb, int cb) {
    switch (rb * 8 + cb) {
        case 8: return -1.7320508075688772;   case 16: return 1.4142135623730951; case 24: return -1.0;
        case 48: return -1.0;                 case 56: return -1.4142135623730951;
        case 17: return 1.4142135623730951;  case 25: return -1.0; case 49: return -1.0; case 57: return -1.4142135623730951;
        case 58: return 1.7320508075688772;
        case 35: return 1.4142135623730951;  case 43: return 1.4142135623730951; case 51: return -1.7320508075688772;
        case 44: return -1.7320508075688772; case 52: return 1.4142135623730951; case 60: return -1.0;
        case 53: return 1.4142135623730951;  case 61: return -1.0;
        default: return 1.0;
    }
}

// All twelve band functions of one (row plane wave, column plane wave) pair:
// v[F_*], from the fused coefficients at difference index t (each field
// loaded once) and the two plane waves' G (g1: row, g2: column).
__device__ __forceinline__ void band_values(const Ctx &c, int64_t t, const double g1[3], const double g2[3],
                                            zc (&v)[13]) {
    const double Kx = c.K[0], Ky = c.K[1], Kz = c.K[2];
    const double g1x = g1[0], g1y = g1[1], g1z = g1[2], g2x = g2[0], g2y = g2[1], g2z = g2[2];
    const double kinx = g1x * g2x + Kx * (g1x + g2x), kiny = g1y * g2y + Ky * (g1y + g2y),
                 kinz = g1z * g2z + Kz * (g1z + g2z);
    const double kxy = kinx + kiny + Kx * Kx + Ky * Ky, kzz = kinz + Kz * Kz, kall = kxy + kzz;
    const double H2 = 0.5 * QD_HBSQM;
    const zc f10 = ld(c, 10, t), f11 = ld(c, 11, t), P = ld(c, 12, t);
    v[F_ZERO] = zc(0.0);
    v[F_ECB] = ld(c, 0, t) + H2 * ld(c, 1, t) * kall + ld(c, 13, t);
    v[F_EHH] = ld(c, 2, t) - H2 * ld(c, 3, t) * kxy - H2 * ld(c, 4, t) * kzz + ld(c, 14, t);
    v[F_ELH] = ld(c, 5, t) - H2 * ld(c, 6, t) * kxy - H2 * ld(c, 7, t) * kzz + ld(c, 15, t);
    v[F_ESO] = ld(c, 8, t) - H2 * ld(c, 9, t) * kall + ld(c, 16, t);
    v[F_Q] = (-sqrt(0.5) * QD_HBSQM) * f10 * kxy + (sqrt(2.0) * QD_HBSQM) * f10 * kzz + ld(c, 17, t);
    {
        const double a = 0.5 * sqrt(3.0) * QD_HBSQM;
        const zc kin = a * f10 * (kinx - kiny + Kx * Kx - Ky * Ky);
        const zc off = a * f11 * ((g1x + Kx) * (g2y + Ky) + (g1y + Ky) * (g2x + Kx));
        const zc r18 = ld(c, 18, t), rd = ld(c, 19, t);
        v[F_R] = kin - I_times(off) + r18 + I_times(rd);   // sg = -1
        v[F_RC] = kin + I_times(off) + r18 - I_times(rd);  // sg = +1
    }
    {
        const double a = 0.5 * sqrt(1.5) * QD_HBSQM;
        const zc re = a * f11 * ((g1x + Kx) * (g2z + Kz) + (g1z + Kz) * (g2x + Kx));
        const zc im = a * f11 * ((g1y + Ky) * (g2z + Kz) + (g1z + Kz) * (g2y + Ky));
        const zc sxz = ld(c, 20, t), syz = ld(c, 21, t);
        v[F_S] = re - I_times(im) - sqrt(0.5) * (sxz - I_times(syz));
        v[F_SC] = re + I_times(im) - sqrt(0.5) * (sxz + I_times(syz));
    }
    {
        const double kx = g1x + g2x + 2 * Kx, ky = g1y + g2y + 2 * Ky, kz = g1z + g2z + 2 * Kz;
        const zc Txx = ld(c, 22, t), Txy = ld(c, 23, t), Tyy = ld(c, 24, t), Txz = ld(c, 25, t), Tyz = ld(c, 26, t);
        const double c6 = -0.5 / sqrt(6.0), i26 = 1.0 / (2.0 * sqrt(6.0));
        const zc base = Txx * kx + Txy * ky + Txz * kz;  // part of the strain sum without the +-i factor
        const zc sI = Txy * kx + Tyy * ky + Tyz * kz;    // part multiplied by +-i
        const zc p0 = (P * kx) * i26, p1 = I_times(P * ky) * i26;
        v[F_TP] = p0 + p1 + c6 * (base + I_times(sI));
        v[F_TM] = p0 - p1 + c6 * (base - I_times(sI));
        const double c3 = -0.5 / sqrt(3.0);
        v[F_U] = (P * kz) / (2.0 * sqrt(3.0)) + c3 * (Txz * kx + Tyz * ky + ld(c, 27, t) * kz);
    }
}

// Derivatives of the twelve band functions with respect to the Bloch wave
// vector component K_ax (the momentum operator of the momentum matrix
// elements, hamiltonian_derivative_8_band_matrix_elements.c:27-969).  The band
// functions are polynomials of degree two in K, so with s = G1 + G2 + 2K the
// derivative of every (G1 + K)_a (G2 + K)_b term is exact and constant terms
// drop out.
__device__ __forceinline__ void band_derivs(const Ctx &c, int64_t t, const double g1[3], const double g2[3], int ax,
                                            zc (&v)[13]) {
    const double K[3] = {c.K[0], c.K[1], c.K[2]};
    double sv[3];
#pragma unroll
    for (int a = 0; a < 3; a++) sv[a] = g1[a] + g2[a] + 2.0 * K[a];
    const double sx = sv[0], sy = sv[1], sz = sv[2], sa = sv[ax];
    const double H2 = 0.5 * QD_HBSQM;
    const zc f10 = ld(c, 10, t), f11 = ld(c, 11, t), P = ld(c, 12, t);
    v[F_ZERO] = zc(0.0);
    v[F_ECB] = H2 * ld(c, 1, t) * sa;
    v[F_EHH] = -H2 * (ax < 2 ? ld(c, 3, t) : ld(c, 4, t)) * sa;
    v[F_ELH] = -H2 * (ax < 2 ? ld(c, 6, t) : ld(c, 7, t)) * sa;
    v[F_ESO] = -H2 * ld(c, 9, t) * sa;
    v[F_Q] = (ax < 2 ? -sqrt(0.5) * QD_HBSQM : sqrt(2.0) * QD_HBSQM) * f10 * sa;
    {
        const double a = 0.5 * sqrt(3.0) * QD_HBSQM;
        const zc kin = ax == 0 ? a * f10 * sx : ax == 1 ? -a * f10 * sy : zc(0.0);
        const zc off = ax == 0 ? a * f11 * sy : ax == 1 ? a * f11 * sx : zc(0.0);
        v[F_R] = kin - I_times(off);
        v[F_RC] = kin + I_times(off);
    }
    {
        const double a = 0.5 * sqrt(1.5) * QD_HBSQM;
        const zc re = ax == 0 ? a * f11 * sz : ax == 2 ? a * f11 * sx : zc(0.0);
        const zc im = ax == 1 ? a * f11 * sz : ax == 2 ? a * f11 * sy : zc(0.0);
        v[F_S] = re - I_times(im);
        v[F_SC] = re + I_times(im);
    }
    {
        // d kx / d Kx = 2 for the linear terms in kx = G1x + G2x + 2 Kx
        const zc Txx = ld(c, 22, t), Txy = ld(c, 23, t), Tyy = ld(c, 24, t), Txz = ld(c, 25, t), Tyz = ld(c, 26, t);
        const double c6 = -0.5 / sqrt(6.0), i26 = 1.0 / (2.0 * sqrt(6.0)), c3 = -0.5 / sqrt(3.0);
        const zc base = ax == 0 ? Txx : ax == 1 ? Txy : Txz;
        const zc sI = ax == 0 ? Txy : ax == 1 ? Tyy : Tyz;
        const zc p0 = ax == 0 ? 2.0 * i26 * P : zc(0.0);
        const zc p1 = ax == 1 ? I_times(2.0 * i26 * P) : zc(0.0);
        v[F_TP] = p0 + p1 + (2.0 * c6) * (base + I_times(sI));
        v[F_TM] = p0 - p1 + (2.0 * c6) * (base - I_times(sI));
        const zc tz = ax == 0 ? Txz : ax == 1 ? Tyz : ld(c, 27, t);
        v[F_U] = (ax == 2 ? (2.0 / (2.0 * sqrt(3.0))) * P : zc(0.0)) + (2.0 * c3) * tz;
    }
}

__device__ __forceinline__ int64_t diff_index(const Ctx &c, const int r[3], const int q[3]) {
    return ((int64_t)(r[0] - q[0] + c.NT[0] / 2) * c.NT[1] + (r[1] - q[1] + c.NT[1] / 2)) * c.NT[2] +
           (r[2] - q[2] + c.NT[2] / 2);
}

// One thread per (row plane wave r, column plane wave q): the twelve band
// functions are evaluated once for the pair (twice when an output needs the
// upper triangle: the upper elements are conjugates of the lower ones of the
// pair (q, r)), and the 8 x 8 band block is written out.  Threads of a warp
// hold 32 consecutive r for one q, so every store of a band block is 32
// consecutive elements of one column.  Stores: complex128 into H64 (lower
// triangle, or full with F64), complex64 into H32 (lower or full with F32).
// DAX >= 0 writes dH/dK_DAX instead of H (same layout and symmetry).
template <bool W64, bool F64, bool W32, bool F32, int DAX = -1>
__global__ void __launch_bounds__(256) assemble_pw_kernel(Ctx c, int npw, double2 *__restrict__ H64, int64_t ld64,
                                                          float2 *__restrict__ H32, int64_t ld32) {
    const int r = blockIdx.x * 32 + threadIdx.x;
    const int q = blockIdx.y * 8 + threadIdx.y;
    if (r >= npw || q >= npw) return;
    const int nyz = c.N[1] * c.N[2];
    const int ir[3] = {r / nyz, (r / c.N[2]) % c.N[1], r % c.N[2]};
    const int iq[3] = {q / nyz, (q / c.N[2]) % c.N[1], q % c.N[2]};
    double g1[3], g2[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        g1[a] = __ldg(&c.G[a][c.off[a] + ir[a]]);
        g2[a] = __ldg(&c.G[a][c.off[a] + iq[a]]);
    }
    zc v[13], u[13];
    constexpr bool need_upper = (W64 && F64) || (W32 && F32);
    if (DAX < 0) {
        band_values(c, diff_index(c, ir, iq), g1, g2, v);
        if (need_upper) band_values(c, diff_index(c, iq, ir), g2, g1, u);
    } else {
        band_derivs(c, diff_index(c, ir, iq), g1, g2, DAX, v);
        if (need_upper) band_derivs(c, diff_index(c, iq, ir), g2, g1, DAX, u);
    }
#pragma unroll
    for (int cb = 0; cb < 8; cb++) {
#pragma unroll
        for (int rb = 0; rb < 8; rb++) {
            const int64_t row = (int64_t)rb * npw + r, col = (int64_t)cb * npw + q;
            const bool lower = rb > cb || (rb == cb && r >= q);
            zc val;
            if (lower) {
                val = bfac(rb, cb) * v[bfunc(rb, cb)];
            } else {
                if (!need_upper) continue;
                val = conj(bfac(cb, rb) * u[bfunc(cb, rb)]);
            }
            if (W64 && (lower || F64)) __stcs(&H64[row + ld64 * col], val.d2());
            if (W32 && (lower || F32)) __stcs(&H32[row + ld32 * col], make_float2((float)val.re, (float)val.im));
        }
    }
}

template <bool W64, bool F64, bool W32, bool F32, int DAX = -1>
int launch_pw(const Ctx &c, int npw, double2 *H64, int64_t ld64, float2 *H32, int64_t ld32, cudaStream_t st) {
    dim3 grid((unsigned)((npw + 31) / 32), (unsigned)((npw + 7) / 8)), block(32, 8);
    qd_count_launch(1);
    assemble_pw_kernel<W64, F64, W32, F32, DAX><<<grid, block, 0, st>>>(c, npw, H64, ld64, H32, ld32);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "assemble launch: %s", cudaGetErrorString(e));
    return QD_OK;
}

int upload_block_map() {
    static int done = 0;
    if (done) return QD_OK;
    signed char fn[8][8] = {{0}};
    double fac[8][8] = {{0}};
    const double s2 = sqrt(2.0), s3 = sqrt(3.0);
    struct E { int r, c, f; double a; } m[] = {
        {1, 1, F_ECB, 1}, {2, 1, F_TM, -s3}, {3, 1, F_U, s2}, {4, 1, F_U, -1}, {7, 1, F_TP, -1}, {8, 1, F_TP, -s2},
        {2, 2, F_EHH, 1}, {3, 2, F_SC, s2}, {4, 2, F_SC, -1}, {7, 2, F_RC, -1}, {8, 2, F_RC, -s2},
        {3, 3, F_ELH, 1}, {4, 3, F_Q, 1}, {5, 3, F_TP, 1}, {6, 3, F_RC, 1}, {8, 3, F_SC, s3},
        {4, 4, F_ESO, 1}, {5, 4, F_TP, s2}, {6, 4, F_RC, s2}, {7, 4, F_SC, -s3},
        {5, 5, F_ECB, 1}, {6, 5, F_TP, -s3}, {7, 5, F_U, s2}, {8, 5, F_U, -1},
        {6, 6, F_EHH, 1}, {7, 6, F_S, s2}, {8, 6, F_S, -1},
        {7, 7, F_ELH, 1}, {8, 7, F_Q, 1},
        {8, 8, F_ESO, 1}};
    for (auto &e : m) {
        fn[e.r - 1][e.c - 1] = (signed char)e.f;
        fac[e.r - 1][e.c - 1] = e.a;
    }
    if (cudaMemcpyToSymbol(c_func, fn, sizeof(fn)) != cudaSuccess) return QD_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_fac, fac, sizeof(fac)) != cudaSuccess) return QD_ERR_CUDA;
    done = 1;
    return QD_OK;
}

}  // namespace

extern "C" int qd_assemble_launch(const void *d_coef, const double *d_Gx, const double *d_Gy, const double *d_Gz,
                                  const int N[3], const double K[3], void *H, int64_t ld, int mode, int prec,
                                  void *stream) {
    if (upload_block_map() != QD_OK) return qd_set_error(QD_ERR_CUDA, "block map upload failed");
    Ctx c;
    c.coef = (const double2 *)d_coef;
    c.G[0] = d_Gx; c.G[1] = d_Gy; c.G[2] = d_Gz;
    for (int a = 0; a < 3; a++) {
        c.N[a] = N[a];
        c.NT[a] = 2 * N[a] - 1;
        c.off[a] = c.NT[a] / 2 - N[a] / 2;
        c.K[a] = K[a];
    }
    c.nT = (int64_t)c.NT[0] * c.NT[1] * c.NT[2];
    int64_t npw = (int64_t)N[0] * N[1] * N[2], nh = 8 * npw;
    if (ld < nh) return qd_set_error(QD_ERR_ARG, "leading dimension %lld < N_H %lld", (long long)ld, (long long)nh);
    cudaStream_t st = (cudaStream_t)stream;
    const int full = mode == 1;
    if (prec == QD_PREC_FP64)
        return full ? launch_pw<true, true, false, false>(c, (int)npw, (double2 *)H, ld, nullptr, 0, st)
                    : launch_pw<true, false, false, false>(c, (int)npw, (double2 *)H, ld, nullptr, 0, st);
    if (prec == QD_PREC_MIXED)
        return full ? launch_pw<false, false, true, true>(c, (int)npw, nullptr, 0, (float2 *)H, ld, st)
                    : launch_pw<false, false, true, false>(c, (int)npw, nullptr, 0, (float2 *)H, ld, st);
    return qd_set_error(QD_ERR_ARG, "unknown precision %d", prec);
}

// dH/dK_axis (axis 0, 1, 2), complex128, lower triangle (mode 0) or full
// Hermitian (mode 1) into H (ld), from the problem's coefficient table.
extern "C" int qd_assemble_dk_launch(const void *d_coef, const double *d_Gx, const double *d_Gy, const double *d_Gz,
                                     const int N[3], const double K[3], int axis, void *H, int64_t ld, int mode,
                                     void *stream) {
    if (upload_block_map() != QD_OK) return qd_set_error(QD_ERR_CUDA, "block map upload failed");
    if (axis < 0 || axis > 2) return qd_set_error(QD_ERR_ARG, "derivative axis %d not in 0..2", axis);
    Ctx c;
    c.coef = (const double2 *)d_coef;
    c.G[0] = d_Gx; c.G[1] = d_Gy; c.G[2] = d_Gz;
    for (int a = 0; a < 3; a++) {
        c.N[a] = N[a];
        c.NT[a] = 2 * N[a] - 1;
        c.off[a] = c.NT[a] / 2 - N[a] / 2;
        c.K[a] = K[a];
    }
    c.nT = (int64_t)c.NT[0] * c.NT[1] * c.NT[2];
    const int64_t npw = (int64_t)N[0] * N[1] * N[2];
    if (ld < 8 * npw) return qd_set_error(QD_ERR_ARG, "leading dimension below N_H");
    cudaStream_t st = (cudaStream_t)stream;
    double2 *Hd = (double2 *)H;
    if (mode == 1) {
        if (axis == 0) return launch_pw<true, true, false, false, 0>(c, (int)npw, Hd, ld, nullptr, 0, st);
        if (axis == 1) return launch_pw<true, true, false, false, 1>(c, (int)npw, Hd, ld, nullptr, 0, st);
        return launch_pw<true, true, false, false, 2>(c, (int)npw, Hd, ld, nullptr, 0, st);
    }
    if (axis == 0) return launch_pw<true, false, false, false, 0>(c, (int)npw, Hd, ld, nullptr, 0, st);
    if (axis == 1) return launch_pw<true, false, false, false, 1>(c, (int)npw, Hd, ld, nullptr, 0, st);
    return launch_pw<true, false, false, false, 2>(c, (int)npw, Hd, ld, nullptr, 0, st);
}

// Both copies in one pass: complex128 into H64 and complex64 into H32 (same ld).
extern "C" int qd_assemble_dual_launch(const void *d_coef, const double *d_Gx, const double *d_Gy,
                                       const double *d_Gz, const int N[3], const double K[3], void *H64,
                                       void *H32, int64_t ld, int mode, void *stream) {
    if (upload_block_map() != QD_OK) return qd_set_error(QD_ERR_CUDA, "block map upload failed");
    Ctx c;
    c.coef = (const double2 *)d_coef;
    c.G[0] = d_Gx; c.G[1] = d_Gy; c.G[2] = d_Gz;
    for (int a = 0; a < 3; a++) {
        c.N[a] = N[a];
        c.NT[a] = 2 * N[a] - 1;
        c.off[a] = c.NT[a] / 2 - N[a] / 2;
        c.K[a] = K[a];
    }
    c.nT = (int64_t)c.NT[0] * c.NT[1] * c.NT[2];
    int64_t npw = (int64_t)N[0] * N[1] * N[2], nh = 8 * npw;
    (void)nh;
    // complex128 lower triangle (the reference's layout) and the full Hermitian complex64 copy
    return mode == 1 ? launch_pw<true, true, true, true>(c, (int)npw, (double2 *)H64, ld, (float2 *)H32, ld,
                                                         (cudaStream_t)stream)
                     : launch_pw<true, false, true, true>(c, (int)npw, (double2 *)H64, ld, (float2 *)H32, ld,
                                                          (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Hellmann-Feynman contraction: g_s = psi_s^H dH psi_s for the states of a
// window, where dH is the Hamiltonian built from a derivative coefficient
// table.  H is linear in the coefficient table (every element is a sum of
// table entries times polynomials in G, G' and K), so dH/dp is the same
// polynomial evaluated on d(coef)/dp; its elements are generated on the fly
// and contracted at once with all states, never stored.  Lower-triangle
// elements count twice (dH is Hermitian): g = sum_{r>c} 2 Re(conj(psi_r) dH_rc
// psi_c) + sum_r dH_rr |psi_r|^2.
// ---------------------------------------------------------------------------
namespace {
constexpr int GRAD_MB = 16;  // states per pass (held in registers per row)

__global__ void __launch_bounds__(128) grad_contract_kernel(Ctx c, int64_t npw, int64_t nh, const double2 *psi,
                                                            int64_t ldz, int m, int cols_per, double *partial) {
    __shared__ double red[GRAD_MB][4];
    const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t col0 = (int64_t)blockIdx.y * cols_per;
    const int64_t block = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    double acc[GRAD_MB];
#pragma unroll
    for (int s = 0; s < GRAD_MB; s++) acc[s] = 0.0;
    const int64_t row_first = blockIdx.x * (int64_t)blockDim.x;
    const bool skip = row_first + blockDim.x - 1 < col0;  // tile entirely above the diagonal
    if (!skip && row < nh) {
        zc pr[GRAD_MB];
#pragma unroll
        for (int s = 0; s < GRAD_MB; s++)
            pr[s] = s < m ? conj(zc(psi[row + s * ldz])) : zc(0.0);
        const int rb = (int)(row / npw);
        const int i = (int)(row - rb * npw);
        const int r[3] = {i / (c.N[1] * c.N[2]), (i / c.N[2]) % c.N[1], i % c.N[2]};
        const int64_t col_end = col0 + cols_per < nh ? col0 + cols_per : nh;
        for (int64_t col = col0; col < col_end && col <= row; col++) {
            const int cb = (int)(col / npw);
            const int j = (int)(col - cb * npw);
            const int q[3] = {j / (c.N[1] * c.N[2]), (j / c.N[2]) % c.N[1], j % c.N[2]};
            zc v = band_element(c, rb, cb, r, q);
            if (col < row) v = 2.0 * v;
#pragma unroll
            for (int s = 0; s < GRAD_MB; s++) {
                if (s < m) {
                    zc t = pr[s] * v * zc(psi[col + s * ldz]);
                    acc[s] += t.re;
                }
            }
        }
    }
    // block reduction per state
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < GRAD_MB; s++) {
        double x = acc[s];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[s][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < GRAD_MB)
        partial[block * GRAD_MB + threadIdx.x] =
            red[threadIdx.x][0] + red[threadIdx.x][1] + red[threadIdx.x][2] + red[threadIdx.x][3];
}

__global__ void grad_sum_kernel(const double *partial, int64_t nblocks, double *out) {
    __shared__ double red[32];
    const int s = blockIdx.x;
    double x = 0.0;
    for (int64_t b = threadIdx.x; b < nblocks; b += blockDim.x) x += partial[b * GRAD_MB + s];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += red[k];
        out[s] = t;
    }
}

// d = (plus - minus) * scale, element-wise over n complex values
__global__ void coef_diff_kernel(const double2 *plus, const double2 *minus, int64_t n, double scale, double2 *d) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        d[t] = make_double2((plus[t].x - minus[t].x) * scale, (plus[t].y - minus[t].y) * scale);
}
}  // namespace

// d = scale (8 (p1 - m1) - (p2 - m2)): the four-point central difference
__global__ void coef_diff4_kernel(const double2 *p1, const double2 *m1, const double2 *p2, const double2 *m2, int64_t n,
                                  double scale, double2 *d) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        d[t] = make_double2(scale * (8.0 * (p1[t].x - m1[t].x) - (p2[t].x - m2[t].x)),
                            scale * (8.0 * (p1[t].y - m1[t].y) - (p2[t].y - m2[t].y)));
}
extern "C" int qd_coef_diff4(const void *p1, const void *m1, const void *p2, const void *m2, int64_t n, double scale,
                             void *d, void *stream) {
    qd_count_launch(1);
    coef_diff4_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>((const double2 *)p1, (const double2 *)m1,
                                                              (const double2 *)p2, (const double2 *)m2, n, scale,
                                                              (double2 *)d);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "coef diff4: %s", cudaGetErrorString(e));
    return QD_OK;
}

extern "C" int qd_coef_diff(const void *plus, const void *minus, int64_t n, double scale, void *d, void *stream) {
    qd_count_launch(1);
    coef_diff_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>((const double2 *)plus, (const double2 *)minus, n, scale,
                                                             (double2 *)d);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "coef diff: %s", cudaGetErrorString(e));
    return QD_OK;
}

// out[s] = psi_s^H dH psi_s for s < m (device pointers; psi column-major N_H x m, ld ldz).
extern "C" int qd_grad_contract(const void *d_dcoef, const double *d_Gx, const double *d_Gy, const double *d_Gz,
                                const int N[3], const double K[3], const void *psi, int64_t ldz, int m,
                                double *out_dev, void *stream) {
    if (upload_block_map() != QD_OK) return qd_set_error(QD_ERR_CUDA, "block map upload failed");
    Ctx c;
    c.coef = (const double2 *)d_dcoef;
    c.G[0] = d_Gx; c.G[1] = d_Gy; c.G[2] = d_Gz;
    for (int a = 0; a < 3; a++) {
        c.N[a] = N[a];
        c.NT[a] = 2 * N[a] - 1;
        c.off[a] = c.NT[a] / 2 - N[a] / 2;
        c.K[a] = K[a];
    }
    c.nT = (int64_t)c.NT[0] * c.NT[1] * c.NT[2];
    const int64_t npw = (int64_t)N[0] * N[1] * N[2], nh = 8 * npw;
    const int cols_per = 64;
    dim3 grid((unsigned)((nh + 127) / 128), (unsigned)((nh + cols_per - 1) / cols_per));
    const int64_t nblocks = (int64_t)grid.x * grid.y;
    cudaStream_t st = (cudaStream_t)stream;
    double *partial = nullptr;
    if (qd_pool_alloc((void **)&partial, sizeof(double) * (size_t)nblocks * GRAD_MB, st))
        return qd_set_error(QD_ERR_NOMEM, "gradient partial sums");
    for (int s0 = 0; s0 < m; s0 += GRAD_MB) {
        int mb = m - s0 < GRAD_MB ? m - s0 : GRAD_MB;
        qd_count_launch(2);
        grad_contract_kernel<<<grid, 128, 0, st>>>(c, npw, nh, (const double2 *)psi + s0 * ldz, ldz, mb, cols_per,
                                                   partial);
        grad_sum_kernel<<<mb, 256, 0, st>>>(partial, nblocks, out_dev + s0);
    }
    cudaError_t e = cudaGetLastError();
    qd_pool_free(partial, st);
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "gradient contraction: %s", cudaGetErrorString(e));
    return QD_OK;
}

// ---------------------------------------------------------------------------
// Hellmann-Feynman contraction as reciprocal-space correlations (the product
// path of eigen_gradients_8_band).
//
// Every band function is a bilinear form in k1 = G1 + K and k2 = G2 + K whose
// coefficients are fused-table entries at the difference G1 - G2:
//   L_{rb,cb}(G1, G2) = sum_f coef_f(G1 - G2) sum_{a,b=0..3} M_{rb cb f a b} k1_a k2_b
// (k_0 = 1).  With u_{b,a}(G) = k_a(G) psi_b(G) the expectation value is
//   <psi|dH|psi> = Re sum_f sum_D dcoef_f(D) C_f(D),
//   C_f(D) = sum_terms w c conj(u_A) (*) u_B (D) = sum_{G1 - G2 = D} ...,
// w = 2 for the strictly lower band blocks (their upper mirror is the complex
// conjugate) and 1 on the band diagonal.  Each correlation is an FFT product:
// with U = FFT(u) on a grid of P >= 2N - 1 points per axis (no wrap-around of
// D), sum_{G1 - G2 = D} conj(u_A(G1)) u_B(G2) = FFT[conj(U_A) U_B](D) / P^3, and
// by linearity every field needs one transform of the summed spectral
// products.  Per state: 32 forward transforms of the weighted envelopes, 28 of
// the field spectra; then each parameter costs one dot product of its
// derivative table with C.  dH is never formed.
//
// The coefficients M are read off the band functions themselves on the device
// (unit coefficient tables, k1, k2 in {0, e_x, e_y, e_z}), so the bilinear
// forms cannot drift from the assembly.
// ---------------------------------------------------------------------------
namespace {
constexpr int GT_MAX = 1024;
struct GradTerm {
    int f, A, B, pad;
    double cr, ci;
};
__constant__ GradTerm c_gterms[GT_MAX];
__constant__ int c_gterm_off[QD_N_COEF + 1];

// out[((f 4 + i1) 4 + i2) 13 + F]: band function F with coefficient table e_f,
// k1 = e_{i1}, k2 = e_{i2} (index 0: the zero vector), K = 0.
__global__ void grad_poly_kernel(const double2 *ident, double2 *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= QD_N_COEF * 16) return;
    const int f = t / 16, i1 = (t / 4) % 4, i2 = t % 4;
    Ctx c;
    c.coef = ident;
    c.nT = QD_N_COEF;
    for (int a = 0; a < 3; a++) {
        c.G[a] = nullptr;
        c.N[a] = c.NT[a] = 1;
        c.off[a] = 0;
        c.K[a] = 0.0;
    }
    double g1[3] = {0.0, 0.0, 0.0}, g2[3] = {0.0, 0.0, 0.0};
    if (i1) g1[i1 - 1] = 1.0;
    if (i2) g2[i2 - 1] = 1.0;
    zc v[13];
    band_values(c, f, g1, g2, v);
    for (int F = 0; F < 13; F++) out[t * 13 + F] = v[F].d2();
}

// U[(s 32 + b 4 + a) P^3 + g] = k_a(G) psi_s[b, G] at grid point g = G's
// plane-wave index (ix, iy, iz) inside the P0 x P1 x P2 grid, zero elsewhere.
__global__ void grad_weight_kernel(const double2 *psi, int64_t ldz, int m, int npw, int n0, int n1, int n2,
                                   int p0, int p1, int p2, const double *Gx, const double *Gy, const double *Gz,
                                   int o0, int o1, int o2, double K0, double K1, double K2, double2 *U) {
    const int64_t P3 = (int64_t)p0 * p1 * p2;
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (g >= P3 || s >= m) return;
    const int ix = (int)(g / ((int64_t)p1 * p2)), iy = (int)((g / p2) % p1), iz = (int)(g % p2);
    double2 *u = U + (int64_t)s * 32 * P3 + g;
    if (ix >= n0 || iy >= n1 || iz >= n2) {
        for (int A = 0; A < 32; A++) u[A * P3] = make_double2(0.0, 0.0);
        return;
    }
    const int pw = (ix * n1 + iy) * n2 + iz;
    const double k[4] = {1.0, Gx[o0 + ix] + K0, Gy[o1 + iy] + K1, Gz[o2 + iz] + K2};
    for (int b = 0; b < 8; b++) {
        const double2 v = psi[(int64_t)s * ldz + (int64_t)b * npw + pw];
        for (int a = 0; a < 4; a++) u[(b * 4 + a) * P3] = make_double2(k[a] * v.x, k[a] * v.y);
    }
}

// S[(s 28 + f) P^3 + g] = sum over the terms of field f of c conj(U_A(g)) U_B(g).
constexpr int GS_PTS = 64;
__global__ void __launch_bounds__(GS_PTS) grad_spectral_kernel(const double2 *U, int64_t P3, int m, double2 *S) {
    __shared__ double2 u[32][GS_PTS];
    const int s = blockIdx.y;
    const int64_t g = blockIdx.x * (int64_t)GS_PTS + threadIdx.x;
    const bool ok = g < P3 && s < m;
    for (int A = 0; A < 32; A++)
        u[A][threadIdx.x] = ok ? U[((int64_t)s * 32 + A) * P3 + g] : make_double2(0.0, 0.0);
    // each thread reads only its own column: no barrier needed
    if (!ok) return;
    for (int f = 0; f < QD_N_COEF; f++) {
        double re = 0.0, im = 0.0;
        for (int t = c_gterm_off[f]; t < c_gterm_off[f + 1]; t++) {
            const GradTerm T = c_gterms[t];
            const double2 a = u[T.A][threadIdx.x], b = u[T.B][threadIdx.x];
            // conj(a) b
            const double pr = a.x * b.x + a.y * b.y, pi = a.x * b.y - a.y * b.x;
            re += T.cr * pr - T.ci * pi;
            im += T.cr * pi + T.ci * pr;
        }
        S[((int64_t)s * QD_N_COEF + f) * P3 + g] = make_double2(re, im);
    }
}

// partial[s][c] = Re sum over slice c of (f, t) of dcoef[f][t] C[s][f][D(t) mod P];
// grid (GD_CHUNKS, states).  grad_dot_sum_kernel adds the slices of each state
// in a fixed order, so the result does not depend on scheduling.
constexpr int GD_CHUNKS = 64;
__global__ void __launch_bounds__(256) grad_dot_kernel(const double2 *dcoef, int nt0, int nt1, int nt2,
                                                       const double2 *C, int p0, int p1, int p2, double *partial) {
    __shared__ double red[8];
    const int s = blockIdx.y, c = blockIdx.x;
    const int64_t nT = (int64_t)nt0 * nt1 * nt2, P3 = (int64_t)p0 * p1 * p2, tot = QD_N_COEF * nT;
    const int64_t i0 = tot * c / GD_CHUNKS, i1 = tot * (c + 1) / GD_CHUNKS;
    double acc = 0.0;
    for (int64_t idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        const int f = (int)(idx / nT);
        const int64_t t = idx - f * nT;
        const int ix = (int)(t / ((int64_t)nt1 * nt2)), iy = (int)((t / nt2) % nt1), iz = (int)(t % nt2);
        int dx = ix - nt0 / 2, dy = iy - nt1 / 2, dz = iz - nt2 / 2;
        dx += dx < 0 ? p0 : 0;
        dy += dy < 0 ? p1 : 0;
        dz += dz < 0 ? p2 : 0;
        const double2 a = dcoef[idx], b = C[((int64_t)s * QD_N_COEF + f) * P3 + ((int64_t)dx * p1 + dy) * p2 + dz];
        acc += a.x * b.x - a.y * b.y;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        partial[(int64_t)s * GD_CHUNKS + c] = t;
    }
}

// out[s] = sum_c partial[s][c] / P^3, one warp per state
__global__ void grad_dot_sum_kernel(const double *partial, int m, double inv_p3, double *out) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (s >= m) return;
    double x = partial[(int64_t)s * GD_CHUNKS + lane] + partial[(int64_t)s * GD_CHUNKS + 32 + lane];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) out[s] = x * inv_p3;
}

// Smallest P >= n whose prime factors are 2, 3, 5 and 7.
int fft_size(int n) {
    for (int p = n > 1 ? n : 1;; p++) {
        int m = p;
        for (int f : {2, 3, 5, 7})
            while (m % f == 0) m /= f;
        if (m == 1) return p;
    }
}

int g_nterms = -1;

// Term table (field, weighted envelope A, weighted envelope B, w c), once per process.
int upload_grad_terms() {
    if (g_nterms >= 0) return QD_OK;
    double2 *ident = nullptr, *poly = nullptr;
    const size_t npoly = (size_t)QD_N_COEF * 16 * 13;
    if (cudaMalloc(&ident, sizeof(double2) * QD_N_COEF * QD_N_COEF) != cudaSuccess ||
        cudaMalloc(&poly, sizeof(double2) * npoly) != cudaSuccess) {
        cudaFree(ident);
        return qd_set_error(QD_ERR_NOMEM, "gradient term extraction");
    }
    double2 id_h[QD_N_COEF * QD_N_COEF];
    for (int i = 0; i < QD_N_COEF * QD_N_COEF; i++) id_h[i] = make_double2(i % (QD_N_COEF + 1) == 0 ? 1.0 : 0.0, 0.0);
    std::vector<double2> L(npoly);
    int rc = QD_OK;
    if (cudaMemcpy(ident, id_h, sizeof(id_h), cudaMemcpyHostToDevice) != cudaSuccess) rc = QD_ERR_CUDA;
    if (rc == QD_OK) {
        qd_count_launch(1);
        grad_poly_kernel<<<(QD_N_COEF * 16 + 127) / 128, 128>>>(ident, poly);
        if (cudaMemcpy(L.data(), poly, sizeof(double2) * npoly, cudaMemcpyDeviceToHost) != cudaSuccess) rc = QD_ERR_CUDA;
    }
    cudaFree(ident);
    cudaFree(poly);
    if (rc) return qd_set_error(QD_ERR_CUDA, "gradient term extraction failed");
    std::vector<GradTerm> terms;
    int off[QD_N_COEF + 1];
    for (int f = 0; f < QD_N_COEF; f++) {
        off[f] = (int)terms.size();
        for (int rb = 0; rb < 8; rb++)
            for (int cb = 0; cb <= rb; cb++) {
                const int F = bfunc(rb, cb);
                if (F == F_ZERO) continue;
                const double w = (rb > cb ? 2.0 : 1.0) * bfac(rb, cb);
                auto val = [&](int i1, int i2) {
                    const double2 v = L[((size_t)(f * 4 + i1) * 4 + i2) * 13 + F];
                    return zc(v.x, v.y);
                };
                const zc c00 = val(0, 0);
                for (int a = 0; a < 4; a++)
                    for (int b = 0; b < 4; b++) {
                        zc cab;
                        if (a == 0 && b == 0) cab = c00;
                        else if (b == 0) cab = val(a, 0) - c00;
                        else if (a == 0) cab = val(0, b) - c00;
                        else cab = val(a, b) - val(a, 0) - val(0, b) + c00;
                        if (fabs(cab.re) + fabs(cab.im) < 1e-12) continue;
                        GradTerm T;
                        T.f = f;
                        T.A = rb * 4 + a;
                        T.B = cb * 4 + b;
                        T.pad = 0;
                        T.cr = w * cab.re;
                        T.ci = w * cab.im;
                        terms.push_back(T);
                    }
            }
    }
    off[QD_N_COEF] = (int)terms.size();
    if ((int)terms.size() > GT_MAX) return qd_set_error(QD_ERR_UNSUPPORTED, "gradient term table: %zu terms", terms.size());
    if (cudaMemcpyToSymbol(c_gterms, terms.data(), sizeof(GradTerm) * terms.size()) != cudaSuccess ||
        cudaMemcpyToSymbol(c_gterm_off, off, sizeof(off)) != cudaSuccess)
        return qd_set_error(QD_ERR_CUDA, "gradient term upload");
    g_nterms = (int)terms.size();
    return QD_OK;
}
}  // namespace

extern "C" int qd_dft3_batched(double2 *d, int64_t stride_b, int nb, const int n[3], int sign, void *stream);

// Correlation tables of m states (device psi, N_H x m, ld ldz): allocates
// *C_out = m x 28 x P^3 complex values (P from qd_grad_corr_size) on the
// device's pool; release with qd_pool_free.
extern "C" int qd_grad_corr_tables(const double *d_Gx, const double *d_Gy, const double *d_Gz, const int N[3],
                                   const double K[3], const void *psi, int64_t ldz, int m, void **C_out, int P_out[3],
                                   void *stream) {
    if (upload_block_map() != QD_OK) return qd_set_error(QD_ERR_CUDA, "block map upload failed");
    int rc = upload_grad_terms();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int P[3], off[3];
    for (int a = 0; a < 3; a++) {
        P[a] = fft_size(2 * N[a] - 1);
        off[a] = (2 * N[a] - 1) / 2 - N[a] / 2;
        P_out[a] = P[a];
    }
    const int64_t P3 = (int64_t)P[0] * P[1] * P[2], npw = (int64_t)N[0] * N[1] * N[2];
    double2 *U = nullptr, *S = nullptr;
    if (qd_pool_alloc((void **)&U, sizeof(double2) * (size_t)P3 * 32 * m, st) ||
        qd_pool_alloc((void **)&S, sizeof(double2) * (size_t)P3 * QD_N_COEF * m, st)) {
        if (U) qd_pool_free(U, st);
        return qd_set_error(QD_ERR_NOMEM, "gradient correlation buffers (%d states, P = %d %d %d)", m, P[0], P[1], P[2]);
    }
    qd_count_launch(1);
    grad_weight_kernel<<<dim3((unsigned)((P3 + 127) / 128), (unsigned)m), 128, 0, st>>>(
        (const double2 *)psi, ldz, m, (int)npw, N[0], N[1], N[2], P[0], P[1], P[2], d_Gx, d_Gy, d_Gz, off[0], off[1],
        off[2], K[0], K[1], K[2], U);
    if ((rc = qd_dft3_batched(U, P3, 32 * m, P, -1, st)) == QD_OK) {
        qd_count_launch(1);
        grad_spectral_kernel<<<dim3((unsigned)((P3 + GS_PTS - 1) / GS_PTS), (unsigned)m), GS_PTS, 0, st>>>(U, P3, m, S);
        rc = qd_dft3_batched(S, P3, QD_N_COEF * m, P, -1, st);
    }
    cudaError_t e = cudaGetLastError();
    qd_pool_free(U, st);
    if (rc == QD_OK && e != cudaSuccess) rc = qd_set_error(QD_ERR_CUDA, "gradient correlations: %s", cudaGetErrorString(e));
    if (rc) {
        qd_pool_free(S, st);
        return rc;
    }
    *C_out = S;
    return QD_OK;
}

// out[s] = <psi_s| dH |psi_s> for the derivative table d_dcoef, from the
// correlation tables of qd_grad_corr_tables (device pointers).
extern "C" int qd_grad_corr_dot(const void *d_dcoef, const int N[3], const void *C, const int P[3], int m,
                                double *out_dev, void *stream) {
    static_assert(GD_CHUNKS == 64, "grad_dot_sum_kernel adds two slices per lane");
    cudaStream_t st = (cudaStream_t)stream;
    double *partial = nullptr;
    if (qd_pool_alloc((void **)&partial, sizeof(double) * GD_CHUNKS * (size_t)m, st))
        return qd_set_error(QD_ERR_NOMEM, "gradient dot partial sums");
    qd_count_launch(2);
    grad_dot_kernel<<<dim3(GD_CHUNKS, (unsigned)m), 256, 0, st>>>((const double2 *)d_dcoef, 2 * N[0] - 1,
                                                                  2 * N[1] - 1, 2 * N[2] - 1, (const double2 *)C,
                                                                  P[0], P[1], P[2], partial);
    const double inv_p3 = 1.0 / ((double)P[0] * P[1] * P[2]);
    grad_dot_sum_kernel<<<(m + 7) / 8, 256, 0, st>>>(partial, m, inv_p3, out_dev);
    qd_pool_free(partial, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return qd_set_error(QD_ERR_CUDA, "gradient dot: %s", cudaGetErrorString(e));
    return QD_OK;
}

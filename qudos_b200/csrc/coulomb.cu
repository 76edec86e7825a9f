// Coulomb matrix elements on the GPU (code/source/8_band/coulomb_matrix_elements.c:24-627
// and the routines it calls, for free and commensurate Coulomb cells, CME = 1..4).
//
//   1. padded envelopes a_sb and conjugate-reversed copies per state and band
//      on the (2Nx-1)(2Ny-1)(2Nz-1) grid (state_redistribution.c:45-66);
//   2. batched 3-D FFTs of all of them (the library's mixed-radix kernels; the
//      (2N - 1) sizes are odd, prime factors above 7 are one DFT stage each);
//   3. for every pair p = (i <= j) the band-summed pointwise product
//      sum_b conj-rev(a_ib)^ . (a_jb)^ (operands staged by TMA bulk copies up
//      to 32 states), and ONE inverse FFT per pair (the
//      reference transforms back per band and then adds; the transform is
//      linear, so summing first is the same B_ij, B_convolutions.c:332-390);
//   4. B on the Coulomb-cell grid: a scaled copy when the cells agree, else
//      separable sinc weights per axis (B_coulomb_supercell.c:23-139).  For
//      commensurate cells (CL = RCL L) the reference upsamples B onto every
//      RCL-th point and convolves it by FFTs with the electronic cell's cuboid
//      on the Coulomb grid (B_coulomb_supercell_fft.c:23-100); that linear
//      convolution is the same separable sum with the cut-off |GC - G| <=
//      max GC, times the cuboid's softening factor when softening is on;
//      tests check it against the FFT form;
//   5. w(G) times the reversed B (coulomb_matrix_elements.c:370-401, 498-503);
//   6. every pair-pair contraction at once as two reductions over the grid
//      (sum Brw_q B_p and sum conj(Brw_q) B_p), and the dipole/quadrupole
//      moments as two more, in the library's FP64 Gram kernel
//      (eig_refine.cu: row slices, 64 x 64 output tiles);
//   7. on the host: the Madelung constant and the reference's symmetry-reduced
//      index loops (coulomb_integrals.c:23-356), which pick entries of those
//      matrices and add the CME >= 2 corrections.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <complex>
#include <vector>

#include "qd_internal.h"

extern "C" int qd_dft3_batched(double2 *d, int64_t stride_b, int nb, const int n[3], int sign, void *stream);
extern "C" int qd_gram_ex_dev(int64_t n, const void *A, int64_t lda, int ka, const void *B, int64_t ldb, int kb,
                              void *C, int ldc, int conj_a, void *stream);

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)
typedef std::complex<double> cd;

namespace {

const double ESQEPS = QD_ESQEPS;

inline int pair_index(int i, int j) { return j * (j + 1) / 2 + i; }

__global__ void coulomb_pad_kernel(const double2 *Z, int64_t ldz, int nx, int ny, int nz, double2 *Fa,
                                   double2 *Fc) {
    const int sb = blockIdx.y, s = sb / QD_N_BAND, b = sb % QD_N_BAND;
    const int sy = 2 * ny - 1, sz = 2 * nz - 1;
    const int64_t S = (int64_t)(2 * nx - 1) * sy * sz, npw = (int64_t)nx * ny * nz;
    const double2 *a = Z + (int64_t)s * ldz + b * npw;
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < S; m += (int64_t)gridDim.x * blockDim.x) {
        int x = (int)(m / ((int64_t)sy * sz)), y = (int)((m / sz) % sy), z = (int)(m % sz);
        double2 v = make_double2(0.0, 0.0), c = v;
        if (x < nx && y < ny && z < nz) {
            v = a[((int64_t)x * ny + y) * nz + z];
            double2 t = a[((int64_t)(nx - 1 - x) * ny + (ny - 1 - y)) * nz + (nz - 1 - z)];
            c = make_double2(t.x, -t.y);
        }
        Fa[(int64_t)sb * S + m] = v;
        Fc[(int64_t)sb * S + m] = c;
    }
}

// Bp[p] = sum_b Fc[i, b] * Fa[j, b] for p = (i, j), i <= j
__global__ void coulomb_pair_kernel(const double2 *Fa, const double2 *Fc, int64_t S, const int2 *pairs,
                                    double2 *Bp) {
    const int2 ij = pairs[blockIdx.y];
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < S; m += (int64_t)gridDim.x * blockDim.x) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int b = 0; b < QD_N_BAND; b++) {
            double2 u = Fc[((int64_t)ij.x * QD_N_BAND + b) * S + m], v = Fa[((int64_t)ij.y * QD_N_BAND + b) * S + m];
            re += u.x * v.x - u.y * v.y;
            im += u.x * v.y + u.y * v.x;
        }
        Bp[(int64_t)blockIdx.y * S + m] = make_double2(re, im);
    }
}

// The same products with the operands staged by the TMA engine: one block takes
// a tile of tm grid points (tm divides 256) of every state's eight band arrays of Fa
// and Fc, brought into shared memory by bulk copies (cp.async.bulk, completion
// counted on one mbarrier), and forms every pair from there, so each array is
// read from memory once instead of once per pair containing its state
// ((M + 1) / 2 times less traffic).  Threads: tm points x 256 / tm pair groups.  The
// wait for the copies is bounded (2 s of %globaltimer); on expiry the block
// records QD_ERR_TIMEOUT in *err, waits (bounded) for its copies and returns.
__device__ __forceinline__ uint32_t cp_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool cp_bar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(cp_smem(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long cp_now() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool cp_bar_wait(uint64_t *bar, uint32_t parity, unsigned long long limit_ns) {
    const unsigned long long t0 = cp_now();
    for (uint32_t it = 0;; it++) {
        if (cp_bar_try(bar, parity)) return true;
        if ((it & 63) == 63 && cp_now() - t0 > limit_ns) return false;
    }
}

__global__ void __launch_bounds__(256) coulomb_pair_tma_kernel(const double2 *Fa, const double2 *Fc, int64_t S, int M,
                                                               int tm, const int2 *pairs, int P, double2 *Bp,
                                                               int *err) {
    extern __shared__ __align__(128) double2 stile[];  // [2][M * 8][tm]: Fa tiles, then Fc tiles
    __shared__ __align__(8) uint64_t bar;
    const int nk = M * QD_N_BAND;
    double2 *sa = stile, *sc = stile + (size_t)nk * tm;
    const int64_t m0 = (int64_t)blockIdx.x * tm;
    const int cnt = (int)(S - m0 < tm ? S - m0 : tm);
    const uint32_t bytes = (uint32_t)cnt * 16u;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 32;" ::"r"(cp_smem(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // warp 0 issues the copies, each lane arriving once with its own byte count
        const int k0 = threadIdx.x;
        const uint32_t mine = (uint32_t)((nk - k0 + 31) / 32) * 2u * bytes;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(cp_smem(&bar)), "r"(mine)
                     : "memory");
        for (int k = k0; k < nk; k += 32) {
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    cp_smem(sa + (size_t)k * tm)),
                "l"(Fa + (int64_t)k * S + m0), "r"(bytes), "r"(cp_smem(&bar))
                : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    cp_smem(sc + (size_t)k * tm)),
                "l"(Fc + (int64_t)k * S + m0), "r"(bytes), "r"(cp_smem(&bar))
                : "memory");
        }
    }
    if (!cp_bar_wait(&bar, 0, 2000000000ull)) {
        if (threadIdx.x == 0) atomicExch(err, QD_ERR_TIMEOUT);
        cp_bar_wait(&bar, 0, 2000000000ull);  // the copies land before the block leaves
        return;
    }
    const int t = threadIdx.x % tm, g = threadIdx.x / tm, ng = blockDim.x / tm;
    if (t >= cnt) return;
    for (int p = g; p < P; p += ng) {
        const int2 ij = pairs[p];
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int b = 0; b < QD_N_BAND; b++) {
            const double2 u = sc[(size_t)(ij.x * QD_N_BAND + b) * tm + t], v = sa[(size_t)(ij.y * QD_N_BAND + b) * tm + t];
            re += u.x * v.x - u.y * v.y;
            im += u.x * v.y + u.y * v.x;
        }
        Bp[(int64_t)p * S + m0 + t] = make_double2(re, im);
    }
}

// Same cells: B_C = (((inv_vol * B / S) * L1) * L2) * L3, the reference's order of operations.
__global__ void coulomb_copy_kernel(const double2 *Bp, int64_t S, int P, double inv_S, double inv_vol, double L1,
                                    double L2, double L3, double2 *BC) {
    const int64_t total = S * P;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        double2 v = Bp[t];
        double re = v.x * inv_S, im = v.y * inv_S;
        re = ((inv_vol * re) * L1) * L2 * L3;
        im = ((inv_vol * im) * L1) * L2 * L3;
        BC[t] = make_double2(re, im);
    }
}

// One axis of the separable Coulomb-cell weights: out has n_out points along
// `axis` (in has n_in), out[.., c, ..] = scale * sum_g W[c * n_in + g] in[.., g, ..].
__global__ void coulomb_axis_kernel(const double2 *in, int i0, int i1, int i2, int axis, int n_out, const double *W,
                                    double scale, int P, double2 *out) {
    int o[3] = {i0, i1, i2};
    o[axis] = n_out;
    const int64_t Sin = (int64_t)i0 * i1 * i2, Sout = (int64_t)o[0] * o[1] * o[2];
    const int n_in = axis == 0 ? i0 : axis == 1 ? i1 : i2;
    const int64_t total = Sout * P;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = t / Sout, m = t % Sout;
        int c[3] = {(int)(m / ((int64_t)o[1] * o[2])), (int)((m / o[2]) % o[1]), (int)(m % o[2])};
        int cc = c[axis];
        double re = 0.0, im = 0.0;
        for (int g = 0; g < n_in; g++) {
            double w = W[(int64_t)cc * n_in + g];
            if (w == 0.0) continue;
            c[axis] = g;
            double2 v = in[p * Sin + ((int64_t)c[0] * i1 + c[1]) * i2 + c[2]];
            re += w * v.x;
            im += w * v.y;
        }
        out[t] = make_double2(scale * re, scale * im);
    }
}

// Brw[p][m] = B[p][S - 1 - m] * w[m]
__global__ void coulomb_reverse_kernel(const double2 *BC, int64_t S, int P, const double *w, double2 *Brw) {
    const int64_t total = S * P;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = t / S, m = t % S;
        double2 v = BC[p * S + (S - 1 - m)];
        Brw[t] = make_double2(v.x * w[m], v.y * w[m]);
    }
}

inline unsigned blocks_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (unsigned)(b > 4096 ? 4096 : (b < 1 ? 1 : b));
}

}  // namespace

// Geometry and options of one Coulomb evaluation.
struct QdCoulombSpec {
    int N[3];      // electronic plane waves per axis
    int NC[3];     // Coulomb-cell plane waves per axis
    double L[3];   // electronic cell lengths (Angstrom)
    double CL[3];  // Coulomb cell lengths (Angstrom)
    double nr;     // refractive index of the matrix material
    int cme;       // include_CME (1..4)
    int ranks;     // ranks whose blocks the real-space Madelung sum covers
    int commensurate;  // Coulomb_supercell_type 1: CL = RCL L
    double soft_sigma; // Gaussian softening of the cell's cuboid (commensurate cells; 0 = none)
};

namespace {

// Coulomb-grid vectors (host): w, the dipole vectors and the quadrupole vector.
void coulomb_vectors(const QdCoulombSpec &sp, std::vector<double> &w, std::vector<cd> &Ix, std::vector<cd> &Iy,
                     std::vector<cd> &Iz, std::vector<cd> &J) {
    int NT[3];
    std::vector<double> G[3];
    for (int a = 0; a < 3; a++) {
        NT[a] = 2 * sp.NC[a] - 1;
        G[a].resize(NT[a]);
        qd_basis_grid(NT[a], sp.CL[a], G[a].data());
    }
    const int64_t S = (int64_t)NT[0] * NT[1] * NT[2];
    w.assign(S, 0.0);
    Ix.assign(S, cd(0, 0));
    Iy.assign(S, cd(0, 0));
    Iz.assign(S, cd(0, 0));
    J.assign(S, cd(0, 0));
    const double V = sp.CL[0] * sp.CL[1] * sp.CL[2];
    const int cx = NT[0] / 2, cy = NT[1] / 2, cz = NT[2] / 2;
    const cd I(0.0, 1.0);
    for (int64_t m = 0; m < S; m++) {
        int ix = (int)(m / ((int64_t)NT[1] * NT[2])), iy = (int)((m % ((int64_t)NT[1] * NT[2])) / NT[2]),
            iz = (int)(m % NT[2]);
        double gx = G[0][ix], gy = G[1][iy], gz = G[2][iz];
        double g = sqrt(gx * gx + gy * gy + gz * gz);
        bool centre = ix == cx && iy == cy && iz == cz;
        if (!centre) w[m] = ESQEPS / (V * g * g * pow(sp.nr, 2.0));  // coulomb_matrix_elements.c:391-401
        // dipole and quadrupole vectors on the three axes (coulomb_matrix_elements.c:403-478)
        const bool on[3] = {ix != cx && iy == cy && iz == cz, ix == cx && iy != cy && iz == cz,
                            ix == cx && iy == cy && iz != cz};
        const double ga[3] = {gx, gy, gz};
        for (int a = 0; a < 3; a++) {
            const int o0 = a == 0 ? 1 : 0, o1 = a == 2 ? 1 : 2;
            const double La = sp.CL[a], Lp = sp.CL[o0] * sp.CL[o1];
            if (on[a]) {
                double q = ga[a];
                cd dip = Lp * ((La / (I * q)) * cos(0.5 * q * La) + (2.0 * I / (q * q)) * sin(0.5 * q * La));
                if (a == 0) Ix[m] = dip;
                if (a == 1) Iy[m] = dip;
                if (a == 2) Iz[m] = dip;
                J[m] += Lp * ((0.5 * La * La / q) * sin(0.5 * La * q) +
                              (2.0 * I / q) * ((La / (I * q)) * cos(0.5 * q * La) + (2.0 * I / (q * q)) * sin(0.5 * q * La)));
            } else if (centre) {
                J[m] += (1 / 12.0) * pow(La, 3) * Lp;
            }
        }
    }
}

// Madelung constant, summed over the ranks of the reference's distribution
// (coulomb_matrix_elements.c:252-331): rank 0 adds the constant terms, every
// rank its block of the reciprocal sum, and rank r the real-space terms of the
// index block of rank r - 1.
double madelung(const QdCoulombSpec &sp) {
    int NT[3];
    std::vector<double> G[3];
    for (int a = 0; a < 3; a++) {
        NT[a] = 2 * sp.NC[a] - 1;
        G[a].resize(NT[a]);
        qd_basis_grid(NT[a], sp.CL[a], G[a].data());
    }
    const double V = sp.CL[0] * sp.CL[1] * sp.CL[2];
    const double ewald = sqrt(M_PI / (sp.CL[0] * sp.CL[1]));
    double a = -2 * ewald / sqrt(M_PI) - M_PI / (ewald * ewald * V);
    const int64_t S = (int64_t)NT[0] * NT[1] * NT[2];
    const int cx = NT[0] / 2, cy = NT[1] / 2, cz = NT[2] / 2;
    double recip = 0.0;
    for (int64_t m = 0; m < S; m++) {
        int ix = (int)(m / ((int64_t)NT[1] * NT[2])), iy = (int)((m % ((int64_t)NT[1] * NT[2])) / NT[2]),
            iz = (int)(m % NT[2]);
        if (ix == cx && iy == cy && iz == cz) continue;
        double g2 = G[0][ix] * G[0][ix] + G[1][iy] * G[1][iy] + G[2][iz] * G[2][iz];
        recip += (4 * M_PI / V) * exp(-g2 / (4 * ewald * ewald)) / g2;
    }
    const int hy = NT[1] / 2, hz = NT[2] / 2;
    double real = 0.0;
    for (int r = 0; r < sp.ranks; r++) {
        int64_t disp = 0, size = 0;
        for (int q = 0; q < r; q++) {
            disp += size;
            size = S / sp.ranks + ((q < S % sp.ranks) ? 1 : 0);
        }
        for (int64_t t = disp; t < disp + size; t++) {
            int64_t mx = t / ((int64_t)hy * hz), my = (t % ((int64_t)hy * hz)) / hz, mz = (t % ((int64_t)hy * hz)) % hz;
            if (mx == 0 && my == 0 && mz == 0) continue;
            double R = sqrt(pow(mx * sp.CL[0], 2) + pow(my * sp.CL[1], 2) + pow(mz * sp.CL[2], 2));
            real += erfc(R * ewald) / R;
        }
    }
    return a + recip + real;
}

inline int l_start_same(int i, int j, int k) { return j == i ? k : (k == i ? j : (k < j ? i + 1 : i)); }

}  // namespace

// B functions, contractions and the four CME arrays for nv + nc states held
// on the device (Z: N_H x (nv + nc), leading dimension ldz, VB states first).
extern "C" int qd_coulomb_dev(const QdCoulombSpec *sp, const void *Zv, int64_t ldz, int nv, int nc,
                              qd_complex128 *hh, qd_complex128 *ee, qd_complex128 *eh_direct,
                              qd_complex128 *eh_exchange, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    const double2 *Z = (const double2 *)Zv;
    if (nv < 0 || nc < 0 || nv + nc < 1) return qd_set_error(QD_ERR_ARG, "qd_coulomb: no states");
    if (sp->cme < 1 || sp->cme > 4) return qd_set_error(QD_ERR_ARG, "qd_coulomb: CME must be 1..4");
    if (sp->ranks < 1) return qd_set_error(QD_ERR_ARG, "qd_coulomb: ranks must be >= 1");
    const int M = nv + nc, P = M * (M + 1) / 2;
    const int sz3[3] = {2 * sp->N[0] - 1, 2 * sp->N[1] - 1, 2 * sp->N[2] - 1};
    const int szC[3] = {2 * sp->NC[0] - 1, 2 * sp->NC[1] - 1, 2 * sp->NC[2] - 1};
    const int64_t S = (int64_t)sz3[0] * sz3[1] * sz3[2], SC = (int64_t)szC[0] * szC[1] * szC[2];
    if ((int64_t)M * QD_N_BAND > 65535 || P > 65535) return qd_set_error(QD_ERR_ARG, "qd_coulomb: too many states");
    bool same = true;
    for (int a = 0; a < 3; a++) same = same && sp->NC[a] == sp->N[a] && sp->L[a] == sp->CL[a];

    double2 *Fa = nullptr, *Fc = nullptr, *Bp = nullptr, *BC = nullptr, *Brw = nullptr, *tmp = nullptr;
    double2 *V4 = nullptr, *U = nullptr, *Cc = nullptr, *Dm = nullptr, *Dc = nullptr;
    double *wd = nullptr, *Wd = nullptr;
    int2 *pairs_d = nullptr;
    int *errd = nullptr;
    // intermediate grids of the separable Coulomb-cell transform stay within this many points
    const int64_t Smax = (int64_t)(sz3[0] > szC[0] ? sz3[0] : szC[0]) * (sz3[1] > szC[1] ? sz3[1] : szC[1]) *
                         (sz3[2] > szC[2] ? sz3[2] : szC[2]);
    std::vector<void *> owned;
    auto alloc = [&](void **p, size_t bytes) -> int {
        int e = qd_pool_alloc(p, bytes, st);
        if (e) return qd_set_error(QD_ERR_NOMEM, "qd_coulomb: %zu bytes", bytes);
        owned.push_back(*p);
        return QD_OK;
    };
    auto release = [&]() {
        for (void *p : owned) qd_pool_free(p, st);
        owned.clear();
    };
    int rc = QD_OK;
    const size_t zsz = sizeof(double2);
    if ((rc = alloc((void **)&Fa, zsz * M * QD_N_BAND * S)) || (rc = alloc((void **)&Fc, zsz * M * QD_N_BAND * S)) ||
        (rc = alloc((void **)&Bp, zsz * P * S)) || (rc = alloc((void **)&BC, zsz * P * SC)) ||
        (rc = alloc((void **)&Brw, zsz * P * SC)) || (rc = alloc((void **)&tmp, zsz * P * Smax * 2)) ||
        (rc = alloc((void **)&V4, zsz * SC * 4)) || (rc = alloc((void **)&U, zsz * P * P)) ||
        (rc = alloc((void **)&Cc, zsz * P * P)) || (rc = alloc((void **)&Dm, zsz * P * 4)) ||
        (rc = alloc((void **)&Dc, zsz * P * 4)) || (rc = alloc((void **)&wd, sizeof(double) * SC)) ||
        (rc = alloc((void **)&Wd, sizeof(double) * 3 * 128 * 128)) || (rc = alloc((void **)&pairs_d, sizeof(int2) * P)) ||
        (rc = alloc((void **)&errd, sizeof(int)))) {
        release();
        return rc;
    }
    // host-side vectors on the Coulomb grid
    std::vector<double> w;
    std::vector<cd> Ix, Iy, Iz, J;
    coulomb_vectors(*sp, w, Ix, Iy, Iz, J);
    std::vector<cd> v4((size_t)SC * 4);
    for (int64_t m = 0; m < SC; m++) {
        v4[m] = Ix[m];
        v4[SC + m] = Iy[m];
        v4[2 * SC + m] = Iz[m];
        v4[3 * SC + m] = J[m];
    }
    std::vector<int2> pairs(P);
    for (int j = 0; j < M; j++)
        for (int i = 0; i <= j; i++) pairs[pair_index(i, j)] = make_int2(i, j);
#define RCK(x)                        \
    do {                              \
        cudaError_t rck_ = (x);       \
        if (rck_ != cudaSuccess) {    \
            release();                \
            CUDA_OK(rck_);            \
        }                             \
    } while (0)
    RCK(cudaMemcpyAsync(wd, w.data(), sizeof(double) * SC, cudaMemcpyHostToDevice, st));
    RCK(cudaMemcpyAsync(V4, v4.data(), zsz * SC * 4, cudaMemcpyHostToDevice, st));
    RCK(cudaMemcpyAsync(pairs_d, pairs.data(), sizeof(int2) * P, cudaMemcpyHostToDevice, st));

    // 1-3: padded states, forward DFTs, band-summed pair products, inverse DFT per pair
    qd_count_launch(2);
    coulomb_pad_kernel<<<dim3(blocks_for(S), M * QD_N_BAND), 256, 0, st>>>(Z, ldz, sp->N[0], sp->N[1], sp->N[2], Fa,
                                                                          Fc);
    RCK(cudaGetLastError());
    if ((rc = qd_dft3_batched(Fa, S, M * QD_N_BAND, sz3, -1, st)) ||
        (rc = qd_dft3_batched(Fc, S, M * QD_N_BAND, sz3, -1, st))) {
        release();
        return rc;
    }
    qd_count_launch(1);
    if (M <= 32) {
        // tiles of 16 points up to 16 states, 8 points up to 32 (at most 64 KB of shared memory, three
        // blocks per SM); the 256 threads are tm points x 256 / tm pair groups
        const int tm = M <= 16 ? 16 : 8;
        const size_t smem = (size_t)2 * M * QD_N_BAND * tm * sizeof(double2);
        static bool configured = false;
        if (!configured) {
            RCK(cudaFuncSetAttribute(coulomb_pair_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 140 * 1024));
            configured = true;
        }
        RCK(cudaMemsetAsync(errd, 0, sizeof(int), st));
        coulomb_pair_tma_kernel<<<(unsigned)((S + tm - 1) / tm), 256, smem, st>>>(Fa, Fc, S, M, tm, pairs_d, P, Bp,
                                                                                   errd);
        RCK(cudaGetLastError());
        int herr = 0;
        RCK(cudaMemcpyAsync(&herr, errd, sizeof(int), cudaMemcpyDeviceToHost, st));
        RCK(cudaStreamSynchronize(st));
        if (herr) {
            release();
            return qd_set_error(QD_ERR_TIMEOUT, "qd_coulomb: staged pair products: wait for the bulk copies ran out");
        }
    } else {
        coulomb_pair_kernel<<<dim3(blocks_for(S), P), 256, 0, st>>>(Fa, Fc, S, pairs_d, Bp);
        RCK(cudaGetLastError());
    }
    if ((rc = qd_dft3_batched(Bp, S, P, sz3, +1, st))) {
        release();
        return rc;
    }
    // 4: Coulomb-cell grid
    const double inv_vol = 1.0 / (sp->L[0] * sp->L[1] * sp->L[2]);
    if (same) {
        qd_count_launch(1);
        coulomb_copy_kernel<<<blocks_for(S * P), 256, 0, st>>>(Bp, S, P, 1.0 / (double)S, inv_vol, sp->L[0], sp->L[1],
                                                              sp->L[2], BC);
        RCK(cudaGetLastError());
    } else {
        // weights W_a[c, g] = I0(GC_c - G_g) (B_coulomb_supercell.c:50-118)
        std::vector<double> Wh(3 * 128 * 128, 0.0);
        for (int a = 0; a < 3; a++) {
            if (szC[a] > 128 || sz3[a] > 128) {
                release();
                return qd_set_error(QD_ERR_UNSUPPORTED, "qd_coulomb: Coulomb grid above 128 points per axis");
            }
            std::vector<double> Gc(szC[a]), Ge(sz3[a]);
            qd_basis_grid(szC[a], sp->CL[a], Gc.data());
            qd_basis_grid(sz3[a], sp->L[a], Ge.data());
            bool same_a = sp->NC[a] == sp->N[a] && sp->L[a] == sp->CL[a];
            for (int c = 0; c < szC[a]; c++)
                for (int g = 0; g < sz3[a]; g++) {
                    if (same_a && g != c) continue;
                    double d = Gc[c] - Ge[g], v;
                    if (fabs(d) < QD_EPS) v = sp->L[a];
                    else if (fabs(d) > Gc[szC[a] - 1] + QD_EPS) v = 0.0;
                    else v = 2 * sin(d * sp->L[a] / 2) / d;
                    if (sp->soft_sigma != 0.0) v *= exp(-0.5 * sp->soft_sigma * sp->soft_sigma * d * d);
                    Wh[a * 128 * 128 + c * sz3[a] + g] = v;
                }
        }
        RCK(cudaMemcpyAsync(Wd, Wh.data(), sizeof(double) * Wh.size(), cudaMemcpyHostToDevice, st));
        // z, then y, then x; the 1/S of the inverse DFT and 1/V_L in the last pass
        int d0[3] = {sz3[0], sz3[1], sz3[2]};
        double2 *t0 = tmp, *t1 = tmp + P * Smax;
        qd_count_launch(3);
        coulomb_axis_kernel<<<blocks_for((int64_t)d0[0] * d0[1] * szC[2] * P), 256, 0, st>>>(
            Bp, d0[0], d0[1], d0[2], 2, szC[2], Wd + 2 * 128 * 128, 1.0, P, t0);
        d0[2] = szC[2];
        coulomb_axis_kernel<<<blocks_for((int64_t)d0[0] * szC[1] * d0[2] * P), 256, 0, st>>>(
            t0, d0[0], d0[1], d0[2], 1, szC[1], Wd + 1 * 128 * 128, 1.0, P, t1);
        d0[1] = szC[1];
        coulomb_axis_kernel<<<blocks_for(SC * P), 256, 0, st>>>(t1, d0[0], d0[1], d0[2], 0, szC[0], Wd, inv_vol / (double)S,
                                                               P, BC);
        RCK(cudaGetLastError());
    }
    // 5: reversed, weighted
    qd_count_launch(1);
    coulomb_reverse_kernel<<<blocks_for(SC * P), 256, 0, st>>>(BC, SC, P, wd, Brw);
    RCK(cudaGetLastError());
    // 6: contractions over the Coulomb grid (coulomb_integrals.c:62-142 as four products):
    //    U = Brw^T BC, Cc = Brw^H BC, Dm = BC^T V4, Dc = BC^H V4
    {
        int rc = qd_gram_ex_dev(SC, Brw, SC, P, BC, SC, P, U, P, 0, st);
        if (rc == QD_OK) rc = qd_gram_ex_dev(SC, Brw, SC, P, BC, SC, P, Cc, P, 1, st);
        if (rc == QD_OK) rc = qd_gram_ex_dev(SC, BC, SC, P, V4, SC, 4, Dm, P, 0, st);
        if (rc == QD_OK) rc = qd_gram_ex_dev(SC, BC, SC, P, V4, SC, 4, Dc, P, 1, st);
        if (rc != QD_OK) {
            release();
            return rc;
        }
    }
    std::vector<cd> Uh((size_t)P * P), Ch((size_t)P * P), Dmh((size_t)P * 4), Dch((size_t)P * 4);
    RCK(cudaMemcpyAsync(Uh.data(), U, zsz * P * P, cudaMemcpyDeviceToHost, st));
    RCK(cudaMemcpyAsync(Ch.data(), Cc, zsz * P * P, cudaMemcpyDeviceToHost, st));
    RCK(cudaMemcpyAsync(Dmh.data(), Dm, zsz * P * 4, cudaMemcpyDeviceToHost, st));
    RCK(cudaMemcpyAsync(Dch.data(), Dc, zsz * P * 4, cudaMemcpyDeviceToHost, st));
    RCK(cudaStreamSynchronize(st));
    release();
#undef RCK

    // 7: corrections and the index loops
    const double V = sp->CL[0] * sp->CL[1] * sp->CL[2];
    const double c_mono = -ESQEPS / (4 * M_PI * pow(sp->nr, 2.0));
    const double c_dip = (ESQEPS / (4 * M_PI * pow(sp->nr, 2.0))) * (4 * M_PI / (3 * pow(V, 3)));
    const double c_quad = (-ESQEPS / (4 * M_PI * pow(sp->nr, 2.0))) * (2 * M_PI / (3 * pow(V, 2)));
    const double a_mad = sp->cme >= 2 ? madelung(*sp) : 0.0;
    auto Uq = [&](int q, int p) { return Uh[(size_t)p * P + q]; };
    auto Cq = [&](int q, int p) { return Ch[(size_t)p * P + q]; };
    auto pair_term = [&](int i, int j, int k, int l) {
        int p = pair_index(i, j);
        return l >= k ? Uq(pair_index(k, l), p) : Cq(pair_index(l, k), p);
    };
    // d[a][l*M + k] (coulomb_matrix_elements.c:504-520), Q[pair] (:521-524)
    auto dmom = [&](int a, int idx) {
        int l = idx / M, k = idx % M;
        return l >= k ? Dmh[(size_t)a * P + pair_index(k, l)] : Dch[(size_t)a * P + pair_index(l, k)];
    };
    auto dip = [&](int x, int y) {
        return c_dip * (dmom(0, x) * dmom(0, y) + dmom(1, x) * dmom(1, y) + dmom(2, x) * dmom(2, y));
    };
    auto Qp = [&](int p) { return Dmh[(size_t)3 * P + p]; };
    const int cme = sp->cme;
    auto put = [](qd_complex128 *o, size_t idx, cd v) {
        double *d = (double *)o;
        d[2 * idx] = v.real();
        d[2 * idx + 1] = v.imag();
    };
    memset(hh, 0, sizeof(qd_complex128) * (size_t)nv * nv * nv * nv);
    memset(ee, 0, sizeof(qd_complex128) * (size_t)nc * nc * nc * nc);
    memset(eh_direct, 0, sizeof(qd_complex128) * (size_t)nv * nv * nc * nc);
    memset(eh_exchange, 0, sizeof(qd_complex128) * (size_t)nv * nv * nc * nc);
    for (int blk = 0; blk < 2; blk++) {  // hh, then ee (coulomb_integrals.c types 0 and 1)
        const int n = blk ? nc : nv, off = blk ? nv : 0;
        qd_complex128 *out = blk ? ee : hh;
        for (int i = 0; i < n; i++)
            for (int j = i; j < n; j++)
                for (int k = i; k < n; k++)
                    for (int l = l_start_same(i, j, k); l < n; l++) {
                        int I_ = i + off, J_ = j + off, K_ = k + off, L_ = l + off;
                        cd v = pair_term(I_, J_, K_, L_);
                        if (cme >= 2 && i == j && k == l) v += c_mono * a_mad;
                        if (cme >= 3) v += dip(J_ * M + I_, L_ * M + K_);
                        if (cme >= 4) {
                            if (i == j && l >= k) v += c_quad * Qp(pair_index(K_, L_));
                            else if (i == j && l < k) v += c_quad * std::conj(Qp(pair_index(L_, K_)));
                            if (k == l) v += c_quad * Qp(pair_index(I_, J_));
                        }
                        put(out, (((size_t)i * n + j) * n + k) * n + l, v);
                    }
    }
    for (int i = 0; i < nv; i++)  // type 2: direct electron-hole
        for (int j = i; j < nv; j++)
            for (int k = 0; k < nc; k++)
                for (int l = (j == i ? k : 0); l < nc; l++) {
                    int K_ = nv + k, L_ = nv + l;
                    cd v = pair_term(i, j, K_, L_);
                    if (cme >= 2 && i == j && k == l) v += c_mono * a_mad;
                    if (cme >= 3) v += dip(j * M + i, L_ * M + K_);
                    if (cme >= 4) {
                        if (i == j && l >= k) v += c_quad * Qp(pair_index(K_, L_));
                        else if (i == j && l < k) v += c_quad * std::conj(Qp(pair_index(L_, K_)));
                        if (k == l) v += c_quad * Qp(pair_index(i, j));
                    }
                    put(eh_direct, (((size_t)i * nv + j) * nc + k) * nc + l, v);
                }
    for (int i = 0; i < nv; i++)  // type 3: exchange electron-hole
        for (int j = 0; j < nc; j++)
            for (int k = j; k < nc; k++)
                for (int l = (k == j ? i : 0); l < nv; l++) {
                    cd v = Cq(pair_index(l, nv + k), pair_index(i, nv + j));
                    if (cme >= 3) v += dip((nv + j) * M + i, l * M + nv + k);
                    put(eh_exchange, (((size_t)i * nc + j) * nc + k) * nv + l, v);
                }
    return QD_OK;
}

static int spec_from_problem(const qd_problem *pr, int ranks, QdCoulombSpec *sp) {
    const struct supercell_geometry *g = &pr->geo[0];
    if (pr->p.coulomb_type == 1 && (g->RCL1 < 1 || g->RCL2 < 1 || g->RCL3 < 1))
        return qd_set_error(QD_ERR_INPUT, "relative Coulomb lengths must be >= 1");
    sp->commensurate = pr->p.coulomb_type == 1;
    sp->soft_sigma = (sp->commensurate && pr->p.softening != 0) ? pr->p.sigma : 0.0;
    for (int a = 0; a < 3; a++) {
        sp->N[a] = pr->p.N[a];
        sp->NC[a] = pr->p.NC[a];
    }
    sp->L[0] = g->L1;
    sp->L[1] = g->L2;
    sp->L[2] = g->L3;
    sp->CL[0] = g->CL1;
    sp->CL[1] = g->CL2;
    sp->CL[2] = g->CL3;
    sp->nr = pr->mat[0].nr;
    sp->cme = pr->p.cme < 1 ? 1 : pr->p.cme;
    sp->ranks = ranks;
    return QD_OK;
}

extern "C" int qd_coulomb(qd_problem *pr, int n_vb_states, int n_cb_states, const qd_complex128 *eigvec_host,
                          int madelung_ranks, qd_complex128 *hh, qd_complex128 *ee, qd_complex128 *eh_direct,
                          qd_complex128 *eh_exchange) {
    if (!pr || !eigvec_host) return qd_set_error(QD_ERR_ARG, "qd_coulomb: null argument");
    QdCoulombSpec sp;
    int rc = spec_from_problem(pr, madelung_ranks, &sp);
    if (rc) return rc;
    const int M = n_vb_states + n_cb_states;
    void *Z = nullptr;
    if (qd_pool_alloc(&Z, sizeof(qd_complex128) * (size_t)pr->n_h * M, nullptr))
        return qd_set_error(QD_ERR_NOMEM, "qd_coulomb: eigenvectors");
    cudaError_t e = cudaMemcpy(Z, eigvec_host, sizeof(qd_complex128) * (size_t)pr->n_h * M, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        qd_pool_free(Z, nullptr);
        return qd_set_error(QD_ERR_CUDA, "qd_coulomb: %s", cudaGetErrorString(e));
    }
    rc = qd_coulomb_dev(&sp, Z, pr->n_h, n_vb_states, n_cb_states, hh, ee, eh_direct, eh_exchange, nullptr);
    qd_pool_free(Z, nullptr);
    return rc;
}

extern "C" void coulomb_matrix_elements(struct wave_vectors basis, struct wave_vectors coulomb_basis,
                                        struct supercell_geometry *supercell, struct material_params *parameters,
                                        int *N_states, struct eigenstate *eigenstate_vb,
                                        struct eigenstate *eigenstate_cb, struct coulomb_matrix_element CME,
                                        int coulomb_region_type) {
    int rc = QD_OK;
    QdCoulombSpec sp;
    sp.commensurate = coulomb_region_type == 1;
    sp.soft_sigma = (sp.commensurate && softening != 0) ? sigma_softening : 0.0;
    sp.N[0] = basis.N_Gx;
    sp.N[1] = basis.N_Gy;
    sp.N[2] = basis.N_Gz;
    sp.NC[0] = coulomb_basis.N_Gx;
    sp.NC[1] = coulomb_basis.N_Gy;
    sp.NC[2] = coulomb_basis.N_Gz;
    sp.L[0] = supercell[0].L1;
    sp.L[1] = supercell[0].L2;
    sp.L[2] = supercell[0].L3;
    sp.CL[0] = supercell[0].CL1;
    sp.CL[1] = supercell[0].CL2;
    sp.CL[2] = supercell[0].CL3;
    sp.nr = parameters[0].nr;
    sp.cme = include_CME;
    sp.ranks = nprocs > 0 ? nprocs : 1;
    const int nv = 2 * N_states[0], nc = 2 * N_states[1], M = nv + nc;
    const int64_t nh = (int64_t)QD_N_BAND * basis.N_Gx * basis.N_Gy * basis.N_Gz;
    void *Z = nullptr;
    if (rc == QD_OK && qd_pool_alloc(&Z, sizeof(qd_complex128) * (size_t)nh * M, nullptr))
        rc = qd_set_error(QD_ERR_NOMEM, "coulomb_matrix_elements: eigenvectors");
    for (int s = 0; rc == QD_OK && s < M; s++) {
        const qd_complex128 *src = s < nv ? eigenstate_vb[s].fourier : eigenstate_cb[s - nv].fourier;
        if (cudaMemcpy((qd_complex128 *)Z + (size_t)s * nh, src, sizeof(qd_complex128) * nh, cudaMemcpyHostToDevice) !=
            cudaSuccess)
            rc = qd_set_error(QD_ERR_CUDA, "coulomb_matrix_elements: copy of state %d", s);
    }
    if (rc == QD_OK) rc = qd_coulomb_dev(&sp, Z, nh, nv, nc, CME.hh, CME.ee, CME.eh_direct, CME.eh_exchange, nullptr);
    if (Z) qd_pool_free(Z, nullptr);
    if (rc != QD_OK) {
        printf("coulomb_matrix_elements failed: %s\n", qd_last_error_message());
        exit(1);
    }
}

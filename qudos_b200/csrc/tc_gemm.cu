// Complex64 GEMMs of the mixed-precision dense->band reduction on the 5th-
// generation tensor cores (tcgen05.mma kind::tf32, accumulators in TMEM,
// operands staged by TMA with 128-byte swizzle).
//
// FP32 accuracy from TF32 inputs: every operand x is split into
// hi = rna_tf32(x) and lo = rna_tf32(x - hi), and a*b is accumulated as
// hi*hi + hi*lo + lo*hi in FP32 (the "3xTF32" split of Ootomo & Yokota 2022);
// the neglected lo*lo term is ~2^-22 relative.
//
// Complex products as real GEMMs with every operand K-major:
//   output D[i, 2j+c] (one TMEM lane per complex output row i, re/im of
//   column j in adjacent TMEM columns), A'[i, 2k+c] = (Re, Im) of the left
//   factor's row i, and the right factor expanded to two real rows per
//   output column j that carry the 2x2 real form of the complex multiply.
//
// Two products use it:
//   qd_tc_xprod  X = A22 * VT (A22 Hermitian, full storage, complex64): A22's
//                columns are read as K-major rows of conj(A22) = A22^T, so the
//                big operand needs no transform; it is split hi/lo in shared
//                memory by a converter warpgroup.  Split-K partials + reduce.
//   qd_tc_flush  A22 -= [V W] [W V]^H (the aggregated rank-2K update); both
//                factors are small and are laid out and split once per call.
//
// Kernel roles (one CTA per SM, persistent over output tiles):
//   warp 0   TMA producer          warp 1   TMEM owner + MMA issuer
//   warps 2-5 epilogue (TMEM -> registers -> global)
//   warps 6-9 (xprod only) hi/lo converter of the streamed A tile
// Every mbarrier wait is bounded (about 2 s of %globaltimer); on a timeout
// the kernel records an error code, stops issuing work, waits (bounded) for
// its copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "qd_internal.h"

#define CUDA_OK(x)                                                                                    \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            return qd_set_error(QD_ERR_CUDA, "%s:%d %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr int BKF = 32;  // floats per k-block row: 128 bytes = one SWIZZLE_128B atom
constexpr int TILE_M = 128;
constexpr unsigned long long WAIT_NS = 2000000000ull;

enum { MODE_XPROD = 0, MODE_FLUSH = 1 };

template <int MODE> struct Cfg;
template <> struct Cfg<MODE_XPROD> {
    static constexpr int N = 64;  // 32 complex output columns
    static constexpr int STAGES = 4;
    static constexpr int A_BYTES = TILE_M * BKF * 4;
    static constexpr int B_BYTES = N * BKF * 4;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int TX_BYTES = A_BYTES + 2 * B_BYTES;  // A_lo is written by the converter
    static constexpr int EPI_WARPS = 4;                     // + 4 converter warps
    static constexpr int EPI_COLS = 64;                     // TMEM columns per epilogue thread
    static constexpr int CHUNK = 2;                         // k-blocks per TMEM accumulation chain
    static constexpr int WARPS = 2 + EPI_WARPS + 4;
    static constexpr int TMEM_COLS = 128;  // two accumulator buffers of N columns
};
template <> struct Cfg<MODE_FLUSH> {
    static constexpr int N = 256;  // 128 complex output columns
    static constexpr int STAGES = 2;
    static constexpr int A_BYTES = TILE_M * BKF * 4;
    static constexpr int B_BYTES = N * BKF * 4;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int TX_BYTES = STAGE_BYTES;
    static constexpr int EPI_WARPS = 8;  // two warps per TMEM lane quarter, one per column half
    static constexpr int EPI_COLS = 128;
    static constexpr int CHUNK = 1;
    static constexpr int WARPS = 2 + EPI_WARPS;
    static constexpr int TMEM_COLS = 512;
};

struct TcArgs {
    int n_items, tiles_m, tiles_n, splits, kblocks;
    int rows;        // valid output rows (complex)
    int cols;        // valid output columns (complex)
    int a_x0, a_y0;  // coordinate offsets into the A tensor map
    float2 *C;       // flush: C tile origin; xprod: split-K partials
    int64_t ldc;     // flush: ld of C; xprod: ld of one partial block
    int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on one phase.  Gives up after WAIT_NS or when another role
// has raised the CTA's abort flag; returns false then.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
    if (mbar_try(bar, parity)) return true;
    unsigned long long t0 = now_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (*abort_flag) return false;
        if (now_ns() - t0 > WAIT_NS) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap *tm, uint64_t *bar, void *dst, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"((uint64_t)tm), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major operand, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major), 16 B
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;             // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

// kind::tf32 instruction descriptor: D f32, A/B tf32, both K-major, M x N.
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
          "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
__device__ __forceinline__ void split3(float x, float &hi, float &lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - hi);
}

// item -> (tm, tn / split)
__device__ __forceinline__ void item_coords(int MODEv, const TcArgs &a, int item, int &tm, int &tn, int &kb0,
                                            int &kb1) {
    if (MODEv == MODE_XPROD) {
        tm = item % a.tiles_m;
        tn = item / a.tiles_m;  // split index
        kb0 = (int)((int64_t)tn * a.kblocks / a.splits);
        kb1 = (int)((int64_t)(tn + 1) * a.kblocks / a.splits);
    } else {
        // bands of 16 row tiles, column tiles outermost within a band (L2 reuse)
        const int G = 16;
        int band = item / (G * a.tiles_n);
        int local = item - band * G * a.tiles_n;
        int gsz = min(G, a.tiles_m - band * G);
        tm = band * G + local % gsz;
        tn = local / gsz;
        kb0 = 0;
        kb1 = a.kblocks;
    }
}

template <int MODE>
__global__ void __launch_bounds__(Cfg<MODE>::WARPS * 32, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmAlo,
                   const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmBlo, TcArgs args) {
    typedef Cfg<MODE> K;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + K::STAGES * K::STAGE_BYTES);
    uint64_t *conv = full + K::STAGES;
    uint64_t *empty = conv + K::STAGES;
    uint64_t *tfull = empty + K::STAGES;  // [2]
    uint64_t *tempty = tfull + 2;         // [2]
    uint64_t *done = tempty + 2;          // [1]
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < K::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&conv[s], 128);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], K::EPI_WARPS * 32);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)K::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    auto fail = [&](int code) {
        atomicCAS(args.err, 0, code);
        *abort_flag = 1;
    };

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            long issued = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                int tm, tn, kb0, kb1;
                item_coords(MODE, args, item, tm, tn, kb0, kb1);
                for (int kb = kb0; kb < kb1; kb++) {
                    if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag)) {
                        fail(1);
                        ok = false;
                        break;
                    }
                    uint8_t *sA = smem + stage * K::STAGE_BYTES;
                    uint8_t *sAlo = sA + K::A_BYTES;
                    uint8_t *sB = sAlo + K::A_BYTES;
                    uint8_t *sBlo = sB + K::B_BYTES;
                    mbar_expect_tx(&full[stage], K::TX_BYTES);
                    int x = kb * BKF;
                    if (MODE == MODE_XPROD) {
                        tma_load_2d(&tmA, &full[stage], sA, args.a_x0 + x, args.a_y0 + tm * TILE_M);
                        tma_load_2d(&tmB, &full[stage], sB, x, 0);
                        tma_load_2d(&tmBlo, &full[stage], sBlo, x, 0);
                    } else {
                        tma_load_2d(&tmA, &full[stage], sA, x, tm * TILE_M);
                        tma_load_2d(&tmAlo, &full[stage], sAlo, x, tm * TILE_M);
                        tma_load_2d(&tmB, &full[stage], sB, x, tn * K::N);
                        tma_load_2d(&tmBlo, &full[stage], sBlo, x, tn * K::N);
                    }
                    issued++;
                    if (++stage == K::STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            // wait for the copies still in flight (all consumed already on the normal path)
            long outstanding = issued < K::STAGES ? issued : K::STAGES;
            for (long q = 0; q < outstanding; q++) {
                if (--stage < 0) {
                    stage = K::STAGES - 1;
                    phase ^= 1;
                }
                unsigned long long t0 = now_ns();
                while (!mbar_try(&full[stage], phase) && now_ns() - t0 < WAIT_NS) {
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        // The accumulator is restarted every CHUNK k-blocks and drained by the
        // epilogue into FP32 registers: the tensor core's own accumulation
        // then only spans 12*CHUNK MMAs, which keeps its rounding error near
        // that of an FP32 dot product.
        if (lane == 0) {
            const uint32_t idesc = tf32_idesc(TILE_M, K::N);
            int stage = 0;
            uint32_t phase = 0;
            int ab = 0;
            uint32_t aphase = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                int tm, tn, kb0, kb1;
                item_coords(MODE, args, item, tm, tn, kb0, kb1);
                for (int kb = kb0; kb < kb1; kb++) {
                    const int cpos = (kb - kb0) % K::CHUNK;
                    if (cpos == 0) {
                        if (!mbar_wait(&tempty[ab], aphase ^ 1, abort_flag)) {
                            fail(2);
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    if (!mbar_wait(&full[stage], phase, abort_flag) ||
                        (MODE == MODE_XPROD && !mbar_wait(&conv[stage], phase, abort_flag))) {
                        fail(3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)(ab * K::N);
                    uint32_t a_hi = smem_u32(smem + stage * K::STAGE_BYTES);
                    uint32_t a_lo = a_hi + K::A_BYTES;
                    uint32_t b_hi = a_lo + K::A_BYTES;
                    uint32_t b_lo = b_hi + K::B_BYTES;
#pragma unroll
                    for (int kk = 0; kk < BKF / 8; kk++) {  // 8 tf32 = 32 bytes per MMA
                        uint32_t o = kk * 32;
                        uint32_t acc = (cpos > 0 || kk > 0) ? 1u : 0u;
                        umma_tf32(d, sw128_desc(a_hi + o), sw128_desc(b_hi + o), idesc, acc);
                        umma_tf32(d, sw128_desc(a_hi + o), sw128_desc(b_lo + o), idesc, 1u);
                        umma_tf32(d, sw128_desc(a_lo + o), sw128_desc(b_hi + o), idesc, 1u);
                    }
                    umma_commit(&empty[stage]);
                    if (++stage == K::STAGES) {
                        stage = 0;
                        phase ^= 1;
                    }
                    if (cpos == K::CHUNK - 1 || kb == kb1 - 1) {
                        umma_commit(&tfull[ab]);
                        if (++ab == 2) {
                            ab = 0;
                            aphase ^= 1;
                        }
                    }
                }
            }
            // all MMAs issued by this thread complete before TMEM is released
            umma_commit(done);
            unsigned long long t0 = now_ns();
            while (!mbar_try(done, 0) && now_ns() - t0 < WAIT_NS) {
            }
        }
    } else if (warp < 2 + K::EPI_WARPS) {
        // ---------------- epilogue: drain each chunk, sum in FP32 registers ----------------
        const int q = warp & 3;                                 // TMEM lane quarter this warp may access
        const int cbase = ((warp - 2) >> 2) * K::EPI_COLS;    // TMEM column range of this warp
        const int r = q * 32 + lane;
        int ab = 0;
        uint32_t aphase = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
            int tm, tn, kb0, kb1;
            item_coords(MODE, args, item, tm, tn, kb0, kb1);
            float acc[K::EPI_COLS];
#pragma unroll
            for (int c = 0; c < K::EPI_COLS; c++) acc[c] = 0.f;
            const int nch = (kb1 - kb0 + K::CHUNK - 1) / K::CHUNK;
            for (int ch = 0; ch < nch; ch++) {
                if (!mbar_wait(&tfull[ab], aphase, abort_flag)) {
                    fail(4);
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int g = 0; g < K::EPI_COLS / 32; g++) {
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * K::N + cbase + g * 32), v);
#pragma unroll
                    for (int c = 0; c < 32; c++) acc[g * 32 + c] += __uint_as_float(v[c]);
                }
                tc_fence_before();
                mbar_arrive(&tempty[ab]);
                if (++ab == 2) {
                    ab = 0;
                    aphase ^= 1;
                }
            }
            if (!ok) break;
            const int row = tm * TILE_M + r;
            if (row < args.rows) {
                if (MODE == MODE_XPROD) {
                    float2 *Xp = args.C + (int64_t)tn * args.ldc * 32;
#pragma unroll
                    for (int l = 0; l < 32; l++)
                        Xp[row + (int64_t)l * args.ldc] = make_float2(acc[2 * l], acc[2 * l + 1]);
                } else {
#pragma unroll
                    for (int jj = 0; jj < K::EPI_COLS / 2; jj++) {
                        int col = tn * (K::N / 2) + cbase / 2 + jj;
                        if (col < args.cols) {
                            float2 *p = args.C + row + (int64_t)col * args.ldc;
                            float2 c = *p;
                            c.x -= acc[2 * jj];
                            c.y -= acc[2 * jj + 1];
                            *p = c;
                        }
                    }
                }
            }
        }
    } else if (MODE == MODE_XPROD) {
        // ---------------- hi/lo converter of the streamed A tile ----------------
        const int t = threadIdx.x - (2 + K::EPI_WARPS) * 32;  // 0..127
        int stage = 0;
        uint32_t phase = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
            int tm, tn, kb0, kb1;
            item_coords(MODE, args, item, tm, tn, kb0, kb1);
            for (int kb = kb0; kb < kb1; kb++) {
                if (!mbar_wait(&full[stage], phase, abort_flag)) {
                    fail(5);
                    ok = false;
                    break;
                }
                float4 *a = (float4 *)(smem + stage * K::STAGE_BYTES);
                float4 *alo = (float4 *)(smem + stage * K::STAGE_BYTES + K::A_BYTES);
#pragma unroll
                for (int u = 0; u < K::A_BYTES / 16 / 128; u++) {
                    int idx = u * 128 + t;
                    float4 x = a[idx], h, l;
                    split3(x.x, h.x, l.x);
                    split3(x.y, h.y, l.y);
                    split3(x.z, h.z, l.z);
                    split3(x.w, h.w, l.w);
                    a[idx] = h;
                    alo[idx] = l;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                mbar_arrive(&conv[stage]);
                if (++stage == K::STAGES) {
                    stage = 0;
                    phase ^= 1;
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"((uint32_t)K::TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// operand preparation
// ---------------------------------------------------------------------------
// X = A22 VT: right factor rows (2l, 2l+1) over K = (2j, 2j+1):
//   row 2l:   ( Re v_jl,  Im v_jl)      row 2l+1: ( Im v_jl, -Re v_jl)
// so that D[i, 2l] = Re(conj(A_ji) v_jl) summed, D[i, 2l+1] = Im(...).
__global__ void prep_xprod_b_kernel(const float2 *VT, int64_t ldvt, int m, int nb, float *Bhi, float *Blo,
                                    int64_t pitch) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y;
    if (2 * (int64_t)j >= pitch) return;
    float2 v = (j < m && l < nb) ? VT[j + (int64_t)l * ldvt] : make_float2(0.f, 0.f);
    float h0, l0, h1, l1, h2, l2;
    split3(v.x, h0, l0);
    split3(v.y, h1, l1);
    split3(-v.x, h2, l2);
    int64_t r0 = (int64_t)(2 * l) * pitch + 2 * j, r1 = r0 + pitch;
    *(float2 *)(Bhi + r0) = make_float2(h0, h1);
    *(float2 *)(Blo + r0) = make_float2(l0, l1);
    *(float2 *)(Bhi + r1) = make_float2(h1, h2);
    *(float2 *)(Blo + r1) = make_float2(l1, l2);
}

// Flush factors: P = [V | W], Q = [W | V] (rows voff.., K columns each).
//   A'[i, 2k+c] = (Re, Im) P_ik                       (mt rows x 4K floats)
//   B'[2j, 2k..] = ( Re Q_jk, Im Q_jk),  B'[2j+1, 2k..] = (-Im Q_jk, Re Q_jk)
// so that D[i, 2j] + i D[i, 2j+1] = sum_k P_ik conj(Q_jk).
// Tiles of 32 rows x 32 complex k through shared memory (column-major in,
// row-major out).
__global__ void prep_flush_kernel(const float2 *V, const float2 *W, int64_t ldv, int64_t voff, int mt, int K,
                                  float *Ahi, float *Alo, float *Bhi, float *Blo) {
    __shared__ float2 tp[32][33], tq[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const int64_t pitch = 4 * (int64_t)K;
    for (int yy = ty; yy < 32; yy += 8) {
        int k = k0 + yy, i = i0 + tx;
        float2 p = make_float2(0.f, 0.f), qv = p;
        if (i < mt && k < 2 * K) {
            const float2 *Pc = k < K ? V + (int64_t)k * ldv : W + (int64_t)(k - K) * ldv;
            const float2 *Qc = k < K ? W + (int64_t)k * ldv : V + (int64_t)(k - K) * ldv;
            p = Pc[voff + i];
            qv = Qc[voff + i];
        }
        tp[yy][tx] = p;
        tq[yy][tx] = qv;
    }
    __syncthreads();
    for (int yy = ty; yy < 32; yy += 8) {
        int i = i0 + yy, k = k0 + tx;
        if (i >= mt || k >= 2 * K) continue;
        float2 p = tp[tx][yy], qv = tq[tx][yy];
        float h0, l0, h1, l1, h2, l2;
        split3(p.x, h0, l0);
        split3(p.y, h1, l1);
        int64_t a = (int64_t)i * pitch + 2 * k;
        *(float2 *)(Ahi + a) = make_float2(h0, h1);
        *(float2 *)(Alo + a) = make_float2(l0, l1);
        split3(qv.x, h0, l0);
        split3(qv.y, h1, l1);
        split3(-qv.y, h2, l2);
        int64_t b0 = (int64_t)(2 * i) * pitch + 2 * k, b1 = b0 + pitch;
        *(float2 *)(Bhi + b0) = make_float2(h0, h1);
        *(float2 *)(Blo + b0) = make_float2(l0, l1);
        *(float2 *)(Bhi + b1) = make_float2(h2, h0);
        *(float2 *)(Blo + b1) = make_float2(l2, l0);
    }
}

__global__ void reduce_splits_kernel(const float2 *Xp, int64_t ldp, int splits, int m, int nb, float2 *X,
                                     int64_t ldx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int l = blockIdx.y;
    if (i >= m || l >= nb) return;
    float2 s = make_float2(0.f, 0.f);
    for (int q = 0; q < splits; q++) {
        float2 v = Xp[(int64_t)q * ldp * 32 + i + (int64_t)l * ldp];
        s.x += v.x;
        s.y += v.y;
    }
    X[i + (int64_t)l * ldx] = s;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder() {
    if (g_encode) return QD_OK;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CUDA_OK(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn)
        return qd_set_error(QD_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return QD_OK;
}

// 2-D fp32 tensor (inner extent `inner` floats, `outer` rows, row pitch in
// bytes), box of 32 floats x box_rows rows, 128-byte swizzle, zero fill.
int make_map(CUtensorMap *m, const void *base, uint64_t inner, uint64_t outer, uint64_t pitch_bytes, int box_rows) {
    if (((uintptr_t)base & 15) || (pitch_bytes & 15))
        return qd_set_error(QD_ERR_ARG, "tensor map: base or pitch not 16-byte aligned");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {pitch_bytes};
    cuuint32_t box[2] = {(cuuint32_t)BKF, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return qd_set_error(QD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return QD_OK;
}

int g_nsm = 0;
int sm_count() {
    if (!g_nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
        if (g_nsm <= 0) g_nsm = 148;
    }
    return g_nsm;
}

template <int MODE>
int smem_bytes() {
    return Cfg<MODE>::STAGES * Cfg<MODE>::STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
}

template <int MODE>
int launch(const CUtensorMap &a, const CUtensorMap &alo, const CUtensorMap &b, const CUtensorMap &blo,
           const TcArgs &args, cudaStream_t st) {
    static bool configured = false;
    int smem = smem_bytes<MODE>();
    if (!configured) {
        CUDA_OK(cudaFuncSetAttribute(tc_gemm_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        configured = true;
    }
    int grid = args.n_items < sm_count() ? args.n_items : sm_count();
    if (grid < 1) return QD_OK;
    qd_count_launch(1);
    tc_gemm_kernel<MODE><<<grid, Cfg<MODE>::WARPS * 32, smem, st>>>(a, alo, b, blo, args);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

}  // namespace

// Work buffers of the tensor-core path (device), sized for an n x n matrix
// and rank-2K updates with K <= kmax.
struct QdTcWork {
    float *bx_hi, *bx_lo;  // 64 x pitch_x
    int64_t pitch_x;
    float2 *xp;  // split-K partials: splits x (ldp x 32)
    int64_t ldp;
    int max_splits;
    float *fa_hi, *fa_lo, *fb_hi, *fb_lo;  // flush factors
    int64_t n;
    int kmax;
    int *err;
};

extern "C" int qd_tc_work_alloc(int64_t n, int kmax, QdTcWork **out) {
    QdTcWork *w = (QdTcWork *)calloc(1, sizeof(QdTcWork));
    if (!w) return qd_set_error(QD_ERR_NOMEM, "qd_tc_work_alloc");
    w->n = n;
    w->kmax = kmax;
    w->pitch_x = ((2 * n + 31) / 32) * 32;
    w->ldp = ((n + 31) / 32) * 32;
    w->max_splits = 16;
    size_t bx = sizeof(float) * 64 * (size_t)w->pitch_x;
    size_t xp = sizeof(float2) * 32 * (size_t)w->ldp * w->max_splits;
    size_t fa = sizeof(float) * (size_t)n * 4 * kmax;
    size_t fb = 2 * fa;
    void *p[7] = {nullptr};
    size_t sz[7] = {bx, bx, xp, fa, fa, fb, fb};
    for (int i = 0; i < 7; i++) {
        if (cudaMalloc(&p[i], sz[i]) != cudaSuccess) {
            for (int k = 0; k < i; k++) cudaFree(p[k]);
            free(w);
            cudaGetLastError();
            return qd_set_error(QD_ERR_NOMEM, "qd_tc_work_alloc: %zu bytes", sz[i]);
        }
    }
    w->bx_hi = (float *)p[0];
    w->bx_lo = (float *)p[1];
    w->xp = (float2 *)p[2];
    w->fa_hi = (float *)p[3];
    w->fa_lo = (float *)p[4];
    w->fb_hi = (float *)p[5];
    w->fb_lo = (float *)p[6];
    if (cudaMalloc(&w->err, sizeof(int)) != cudaSuccess) {
        for (int k = 0; k < 7; k++) cudaFree(p[k]);
        free(w);
        return qd_set_error(QD_ERR_NOMEM, "qd_tc_work_alloc");
    }
    cudaMemset(w->err, 0, sizeof(int));
    *out = w;
    return QD_OK;
}

extern "C" void qd_tc_work_free(QdTcWork *w) {
    if (!w) return;
    void *p[8] = {w->bx_hi, w->bx_lo, w->xp, w->fa_hi, w->fa_lo, w->fb_hi, w->fb_lo, w->err};
    for (int i = 0; i < 8; i++)
        if (p[i]) cudaFree(p[i]);
    free(w);
}

// Error code left by the tensor-core kernels (0 = none); clears it.
extern "C" int qd_tc_work_check(QdTcWork *w) {
    int e = 0;
    CUDA_OK(cudaMemcpy(&e, w->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(w->err, 0, sizeof(int));
        return qd_set_error(QD_ERR_TIMEOUT, "tensor-core GEMM: wait timed out (role %d)", e);
    }
    return QD_OK;
}

// X[0:m, 0:nb] = A22 * VT, A22 = A[off:off+m, off:off+m] of the full
// Hermitian complex64 matrix A (n x n, lda); VT is m x nb (ldvt), nb <= 32.
extern "C" int qd_tc_xprod(const void *A, int64_t lda, int64_t n, int64_t off, int m, const void *VT, int64_t ldvt,
                           int nb, void *X, int64_t ldx, QdTcWork *w, void *stream) {
    if (m <= 0 || nb <= 0) return QD_OK;
    if (nb > 32 || off + m > n || n > w->n) return qd_set_error(QD_ERR_ARG, "qd_tc_xprod: bad sizes");
    if (off & 1) return qd_set_error(QD_ERR_ARG, "qd_tc_xprod: trailing offset must be even");
    int rc = get_encoder();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t pitch = ((2 * (int64_t)m + 31) / 32) * 32;
    qd_count_launch(1);
    prep_xprod_b_kernel<<<dim3((unsigned)((pitch / 2 + 127) / 128), 32), 128, 0, st>>>(
        (const float2 *)VT, ldvt, m, nb, w->bx_hi, w->bx_lo, pitch);
    CUDA_OK(cudaGetLastError());
    CUtensorMap ta, tb, tblo;
    if ((rc = make_map(&ta, A, 2 * (uint64_t)n, (uint64_t)n, (uint64_t)lda * 8, TILE_M))) return rc;
    if ((rc = make_map(&tb, w->bx_hi, (uint64_t)pitch, 64, (uint64_t)pitch * 4, 64))) return rc;
    if ((rc = make_map(&tblo, w->bx_lo, (uint64_t)pitch, 64, (uint64_t)pitch * 4, 64))) return rc;
    TcArgs a;
    a.tiles_m = (m + TILE_M - 1) / TILE_M;
    a.tiles_n = 1;
    a.kblocks = (int)((2 * (int64_t)m + BKF - 1) / BKF);
    int nsm = sm_count();
    int splits = (2 * nsm + a.tiles_m - 1) / a.tiles_m;  // about two items per SM
    if (splits > w->max_splits) splits = w->max_splits;
    if (splits > a.kblocks) splits = a.kblocks;
    if (splits < 1) splits = 1;
    a.splits = splits;
    a.n_items = a.tiles_m * splits;
    a.rows = m;
    a.cols = nb;
    a.a_x0 = (int)(2 * off);
    a.a_y0 = (int)off;
    a.C = w->xp;
    a.ldc = w->ldp;
    a.err = w->err;
    if (m > w->ldp) return qd_set_error(QD_ERR_ARG, "qd_tc_xprod: m exceeds the work buffers");
    if ((rc = launch<MODE_XPROD>(ta, ta, tb, tblo, a, st))) return rc;
    qd_count_launch(1);
    reduce_splits_kernel<<<dim3((unsigned)((m + 127) / 128), nb), 128, 0, st>>>(w->xp, w->ldp, splits, m, nb,
                                                                                  (float2 *)X, ldx);
    CUDA_OK(cudaGetLastError());
    return QD_OK;
}

// A[off:off+mt, off:off+mt] -= P Q^H with P = [V W], Q = [W V] taken from
// rows voff..voff+mt-1 and the first K columns of V and W (ldv).
extern "C" int qd_tc_flush(void *A, int64_t lda, int64_t off, int mt, const void *V, const void *W, int64_t ldv,
                           int64_t voff, int K, QdTcWork *w, void *stream) {
    if (mt <= 0 || K <= 0) return QD_OK;
    if (K > w->kmax || mt > w->n) return qd_set_error(QD_ERR_ARG, "qd_tc_flush: bad sizes");
    int rc = get_encoder();
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t pitch = 4 * (int64_t)K;
    qd_count_launch(1);
    prep_flush_kernel<<<dim3((unsigned)((mt + 31) / 32), (unsigned)((2 * K + 31) / 32)), dim3(32, 8), 0, st>>>(
        (const float2 *)V, (const float2 *)W, ldv, voff, mt, K, w->fa_hi, w->fa_lo, w->fb_hi, w->fb_lo);
    CUDA_OK(cudaGetLastError());
    CUtensorMap ta, talo, tb, tblo;
    if ((rc = make_map(&ta, w->fa_hi, (uint64_t)pitch, (uint64_t)mt, (uint64_t)pitch * 4, TILE_M))) return rc;
    if ((rc = make_map(&talo, w->fa_lo, (uint64_t)pitch, (uint64_t)mt, (uint64_t)pitch * 4, TILE_M))) return rc;
    if ((rc = make_map(&tb, w->fb_hi, (uint64_t)pitch, 2 * (uint64_t)mt, (uint64_t)pitch * 4, 256))) return rc;
    if ((rc = make_map(&tblo, w->fb_lo, (uint64_t)pitch, 2 * (uint64_t)mt, (uint64_t)pitch * 4, 256))) return rc;
    TcArgs a;
    a.tiles_m = (mt + TILE_M - 1) / TILE_M;
    a.tiles_n = (mt + 127) / 128;
    a.splits = 1;
    a.kblocks = (int)((pitch + BKF - 1) / BKF);
    a.n_items = a.tiles_m * a.tiles_n;
    a.rows = mt;
    a.cols = mt;
    a.a_x0 = 0;
    a.a_y0 = 0;
    a.C = (float2 *)A + off + off * lda;
    a.ldc = lda;
    a.err = w->err;
    return launch<MODE_FLUSH>(ta, talo, tb, tblo, a, st);
}

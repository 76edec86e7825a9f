// Complex64 GEMMs of the mixed-precision dense->band reduction on the 5th-
// generation tensor cores (tcgen05.mma kind::tf32, accumulators in TMEM,
// operands staged by TMA with 128-byte swizzle).
//
// FP32 accuracy from TF32 inputs: every operand x is split into
// hi = tf32(x) and lo = tf32(x - hi) (round to nearest), and a*b is accumulated as
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
//                big operand needs no transform; a converter warpgroup splits
//                it hi/lo into tensor memory, where the MMAs read it.  Split-K
//                partials + reduce.
//   qd_tc_flush  A22 -= [V W] [W V]^H (the aggregated rank-2K update) on the
//                lower-triangle tiles, mirrored into the upper triangle; both
//                factors are small and are laid out and split once per call.
//
// Both kernels are persistent (one CTA per SM) and warp-specialised: TMA
// producer(s), MMA-issuing thread(s) (one owns TMEM), epilogue warps
// that drain TMEM, and (xprod) a converter warpgroup.  The accumulator is
// restarted every one or two k-blocks and summed in FP32 registers by the
// epilogue, which keeps the tensor core's internal accumulation short.
// Every mbarrier wait is bounded (about 2 s of %globaltimer); on a timeout
// the kernel records an error code, stops issuing work, waits (bounded) for
// its copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

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
// A pipeline wait gives up after g_wait_ns of %globaltimer (set at run time by
// qd_set_wait_limits, default 2 s).  The waits that drain a CTA's own copies
// and MMAs in flight before it exits keep the fixed DRAIN_NS, so that an
// aborted CTA never leaves with work still landing in its shared memory.
constexpr unsigned long long WAIT_NS_DEFAULT = 2000000000ull;
constexpr unsigned long long DRAIN_NS = 2000000000ull;
__device__ unsigned long long g_wait_ns = WAIT_NS_DEFAULT;

struct TcArgs {
    int n_items, tiles_m, tiles_n, splits, kblocks;
    int rows;        // valid output rows (complex)
    int cols;        // valid output columns (complex)
    int a_x0, a_y0;  // coordinate offsets into the A tensor map
    float2 *C;       // flush: C tile origin; xprod: split-K partials
    int64_t ldc;     // flush: ld of C; xprod: ld of one partial block
    int kdim;        // flush: rank of the update (K)
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
// Bounded wait on one phase.  Gives up after g_wait_ns or when another role
// has raised the CTA's abort flag; returns false then.
// The clock and the abort flag are read every 64 polls only: the waiting warps
// of a CTA would otherwise keep the SM's conversion/special-register pipe busy.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns(), limit = g_wait_ns;
    for (uint32_t it = 1;; it++) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 0) {
            if (*abort_flag) return false;
            if (now_ns() - t0 > limit) return false;
        }
    }
}

// Warp-wide bounded wait: lane 0 polls, the warp then synchronises (which
// orders lane 0's acquire before the other lanes' reads).  All 32 lanes call.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort_flag) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
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
// A operand from tensor memory (K-major: row i in lane i, element k in column k).
__device__ __forceinline__ void umma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32_issue(uint32_t taddr, uint32_t *v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
          "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// Each lane of the warp writes 32 consecutive 32-bit columns of its own lane.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]), "f"(v[16]),
        "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]), "f"(v[24]),
        "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Round to the nearest TF32 value (10 stored mantissa bits, ties away from
// zero) with integer operations: add half an ulp of TF32 to the magnitude
// bits and clear the 13 bits below.  Finite inputs far from FLT_MAX only.
__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xffffe000u);
}
// x = hi + lo with hi, lo TF32 values: hi carries 11 significant bits, the
// exact remainder x - hi (|x - hi| <= 2^-11 |x|) is rounded again, so
// |x - hi - lo| <= 2^-22 |x|.
__device__ __forceinline__ void split3(float x, float &hi, float &lo) {
    hi = tf32_round(x);
    lo = tf32_round(x - hi);
}

// Lower-triangle tile (tm >= tn) of item `item` among T(T+1)/2, in bands of
// 16 row tiles (column tiles outermost within a band) for L2 reuse of the
// factor tiles.
__device__ __forceinline__ void lower_tile(int item, int T, int &tm, int &tn) {
    // items before band g (all bands before are full): 128 g^2 + 8 g
    int g = (int)((-8.0 + sqrt(64.0 + 512.0 * (double)item)) / 256.0);
    while (g > 0 && 128LL * g * g + 8LL * g > item) g--;
    while (128LL * (g + 1) * (g + 1) + 8LL * (g + 1) <= item) g++;
    int local = item - (128 * g * g + 8 * g);
    int gs = min(16, T - 16 * g);
    if (local < 16 * g * gs) {
        tn = local / gs;
        tm = 16 * g + local % gs;
    } else {
        int t = local - 16 * g * gs, c = 0;
        while (t >= gs - c) {
            t -= gs - c;
            c++;
        }
        tn = 16 * g + c;
        tm = tn + t;
    }
}

__device__ __forceinline__ void xprod_item(const TcArgs &a, int item, int &tm, int &s, int &kb0, int &kb1) {
    tm = item % a.tiles_m;
    s = item / a.tiles_m;
    kb0 = (int)((int64_t)s * a.kblocks / a.splits);
    kb1 = (int)((int64_t)(s + 1) * a.kblocks / a.splits);
}

// Epilogue chunk loop shared by both kernels: drains every accumulation chunk
// of one item from TMEM into FP32 registers.  Returns false on abort.
template <int NCOLS, int ACC_COLS>
__device__ __forceinline__ bool drain_item(float (&acc)[ACC_COLS], int nch, uint32_t tmem_base, int q, int cbase,
                                           int &ab, uint32_t &aphase, uint64_t *tfull, uint64_t *tempty,
                                           volatile int *abort_flag) {
#pragma unroll
    for (int c = 0; c < ACC_COLS; c++) acc[c] = 0.f;
    for (int ch = 0; ch < nch; ch++) {
        if (!mbar_wait_warp(&tfull[ab], aphase, abort_flag)) return false;
        tc_fence_after();
#pragma unroll
        for (int g = 0; g < ACC_COLS / 64; g++) {  // two loads in flight per wait
            uint32_t v[64];
            const uint32_t ta = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * NCOLS + cbase + g * 64);
            tmem_ld32_issue(ta, v);
            tmem_ld32_issue(ta + 32, v + 32);
            tmem_ld_wait();
#pragma unroll
            for (int c = 0; c < 64; c++) acc[g * 64 + c] += __uint_as_float(v[c]);
        }
        tc_fence_before();
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&tempty[ab]);  // one arrival per warp
        if (++ab == 2) {
            ab = 0;
            aphase ^= 1;
        }
    }
    return true;
}

__device__ __forceinline__ void ring_next(int &s, uint32_t &ph, int n) {
    if (++s == n) {
        s = 0;
        ph ^= 1;
    }
}
__device__ __forceinline__ void ring_prev(int &s, uint32_t &ph, int n) {
    if (--s < 0) {
        s = n - 1;
        ph ^= 1;
    }
}
__device__ __forceinline__ void wait_bounded(uint64_t *bar, uint32_t parity) {
    unsigned long long t0 = now_ns();
    for (uint32_t it = 1; !mbar_try(bar, parity); it++)
        if ((it & 63) == 0 && now_ns() - t0 >= DRAIN_NS) break;
}

// ---------------------------------------------------------------------------
// X = A22 VT.  Three rings, each advanced once per k-block:
//   A  (XA_STAGES x 16 KB smem): TMA fp32 tiles of A22, released as soon as
//      the converter has read them, so that the ring turns over at DRAM latency;
//   B  (XB_STAGES x 16 KB smem): TMA tiles of the right factor, hi and lo;
//   L  (XL_STAGES x 64 TMEM columns): hi (columns 0-31) and lo (32-63) of the
//      A tile, written by the converter with tcgen05.st (thread = row = TMEM
//      lane) and read by the MMAs as their A operand, so the split tile never
//      passes through shared memory: per k-block shared memory carries 16 KB
//      in and out of the A ring and the B tiles, which keeps its bandwidth
//      below the DRAM stream's.
// The B tiles come from L2 and have their own producer so that their latency
// is not serialised behind the converter.
// One thread issues at most about one MMA per 45 cycles, and a k-block takes
// 12 MMAs (3 products x 4 steps of K = 8), so two threads issue them: warp 1
// the steps 0-1, warp 11 the steps 2-3, each into its own accumulator; the
// epilogue adds the two.  The B ring and the L ring have the same depth and
// advance together, so one barrier per stage (emptyL) frees both the B tile and
// the TMEM stage: each issuer commits once per k-block.  The barriers the MMAs
// release (emptyL, tfull, done) expect one commit from each issuer.
//   warp 0 A producer, warps 1 and 11 MMA, warps 2-5 epilogue, warps 6-9
//   converter, warp 10 B producer.
// TMEM: columns [0, 256) the two issuers' double-buffered accumulators of 64
// (issuer h, buffer ab at 128 h + 64 ab), [256, 256 + 64 XL_STAGES) L.
// ---------------------------------------------------------------------------
constexpr int XA_STAGES = 8, XB_STAGES = 4, XL_STAGES = 4;
static_assert(XB_STAGES == XL_STAGES, "the B and L rings share their release barrier");
constexpr int X_N = 64;
constexpr int X_A_BYTES = TILE_M * BKF * 4;  // 16 KB
constexpr int X_B_BYTES = X_N * BKF * 4;     // 8 KB (hi or lo)
constexpr int X_SMEM = XA_STAGES * X_A_BYTES + XB_STAGES * 2 * X_B_BYTES;
constexpr int X_CHUNK = 2;
constexpr int X_WARPS = 12;
constexpr int X_ISSUERS = 2;
constexpr int X_L_COL0 = 2 * X_ISSUERS * X_N;
constexpr int X_TMEM_COLS = 512;
static_assert(X_L_COL0 + 2 * BKF * XL_STAGES <= X_TMEM_COLS, "TMEM columns");

// Epilogue of the X product: every accumulation chunk is the sum of the two
// issuers' accumulators (columns 64 (2 h + ab) of this warp's lane quarter).
__device__ __forceinline__ bool drain_pair(float (&acc)[X_N], int nch, uint32_t tmem_base, int q, int &ab,
                                           uint32_t &aphase, uint64_t *tfull, uint64_t *tempty,
                                           volatile int *abort_flag) {
#pragma unroll
    for (int c = 0; c < X_N; c++) acc[c] = 0.f;
    for (int ch = 0; ch < nch; ch++) {
        if (!mbar_wait_warp(&tfull[ab], aphase, abort_flag)) return false;
        tc_fence_after();
#pragma unroll
        for (int h = 0; h < 2; h++) {
            uint32_t v[X_N];
            const uint32_t ta = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)((h * 2 + ab) * X_N);
            tmem_ld32_issue(ta, v);
            tmem_ld32_issue(ta + 32, v + 32);
            tmem_ld_wait();
#pragma unroll
            for (int c = 0; c < X_N; c++) acc[c] += __uint_as_float(v[c]);
        }
        tc_fence_before();
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&tempty[ab]);  // one arrival per warp
        if (++ab == 2) {
            ab = 0;
            aphase ^= 1;
        }
    }
    return true;
}

__global__ void __launch_bounds__(X_WARPS * 32, 1)
    xprod_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 const __grid_constant__ CUtensorMap tmBlo, TcArgs args) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *ringA = smem, *ringB = smem + XA_STAGES * X_A_BYTES;
    uint64_t *fullA = (uint64_t *)(smem + X_SMEM);
    uint64_t *emptyA = fullA + XA_STAGES;
    uint64_t *fullB = emptyA + XA_STAGES;
    uint64_t *conv = fullB + XB_STAGES;
    uint64_t *emptyL = conv + XL_STAGES;
    uint64_t *tfull = emptyL + XL_STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *done = tempty + 2;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < XA_STAGES; s++) {
            mbar_init(&fullA[s], 1);
            mbar_init(&emptyA[s], 4);  // released by the four converter warps
        }
        for (int s = 0; s < XB_STAGES; s++) mbar_init(&fullB[s], 1);
        for (int s = 0; s < XL_STAGES; s++) {
            mbar_init(&conv[s], 4);  // one arrival per converter warp
            mbar_init(&emptyL[s], X_ISSUERS);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], X_ISSUERS);
            mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
        }
        mbar_init(done, X_ISSUERS);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)X_TMEM_COLS)
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

    if (warp == 0 || warp == 10) {
        // ---------------- producers: A ring (warp 0), B ring (warp 10) ----------------
        if (lane == 0) {
            const bool isA = warp == 0;
            const int nst = isA ? XA_STAGES : XB_STAGES;
            uint64_t *full = isA ? fullA : fullB, *empty = isA ? emptyA : emptyL;
            int s = 0;
            uint32_t ph = 0;
            long issued = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                int tm, sp, kb0, kb1;
                xprod_item(args, item, tm, sp, kb0, kb1);
                for (int kb = kb0; kb < kb1; kb++) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) {
                        fail(isA ? 1 : 6);
                        ok = false;
                        break;
                    }
                    if (isA) {
                        mbar_expect_tx(&full[s], X_A_BYTES);
                        tma_load_2d(&tmA, &full[s], ringA + s * X_A_BYTES, args.a_x0 + kb * BKF,
                                    args.a_y0 + tm * TILE_M);
                    } else {
                        uint8_t *b = ringB + s * 2 * X_B_BYTES;
                        mbar_expect_tx(&full[s], 2 * X_B_BYTES);
                        tma_load_2d(&tmB, &full[s], b, kb * BKF, 0);
                        tma_load_2d(&tmBlo, &full[s], b + X_B_BYTES, kb * BKF, 0);
                    }
                    issued++;
                    ring_next(s, ph, nst);
                }
            }
            long outstanding = issued < nst ? issued : nst;
            for (long q = 0; q < outstanding; q++) {
                ring_prev(s, ph, nst);
                wait_bounded(&full[s], ph);
            }
        }
    } else if (warp == 1 || warp == 11) {
        // ---------------- MMA issuers (accumulation restarted every X_CHUNK k-blocks) ----------------
        if (lane == 0) {
            const int h = warp == 11;  // K steps 2h, 2h + 1 of every k-block
            const uint32_t idesc = tf32_idesc(TILE_M, X_N);
            const uint64_t bdesc0 = sw128_desc(smem_u32(ringB));
            int sb = 0, sl = 0, ab = 0;
            uint32_t pb = 0, pl = 0, aphase = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                int tm, sp, kb0, kb1;
                xprod_item(args, item, tm, sp, kb0, kb1);
                for (int kb = kb0; kb < kb1; kb++) {
                    const int cpos = (kb - kb0) % X_CHUNK;
                    if (cpos == 0) {
                        if (!mbar_wait(&tempty[ab], aphase ^ 1, abort_flag)) {
                            fail(2);
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    if (!mbar_wait(&fullB[sb], pb, abort_flag) || !mbar_wait(&conv[sl], pl, abort_flag)) {
                        fail(3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)((h * 2 + ab) * X_N);
                    const uint32_t a_hi = tmem_base + (uint32_t)(X_L_COL0 + sl * 2 * BKF + h * 16);
                    const uint32_t a_lo = a_hi + BKF;
                    // +32 bytes along K in the B tile = +2 in the descriptor's address field
                    const uint64_t bh = bdesc0 + (uint64_t)((sb * 2 * X_B_BYTES + h * 64) >> 4);
                    const uint64_t bl = bh + (X_B_BYTES >> 4);
#pragma unroll
                    for (int kk = 0; kk < 2; kk++) {
                        uint32_t acc = (cpos > 0 || kk > 0) ? 1u : 0u;
                        umma_tf32_ts(d, a_hi + kk * 8, bh + 2 * kk, idesc, acc);
                        umma_tf32_ts(d, a_hi + kk * 8, bl + 2 * kk, idesc, 1u);
                        umma_tf32_ts(d, a_lo + kk * 8, bh + 2 * kk, idesc, 1u);
                    }
                    umma_commit(&emptyL[sl]);  // frees B stage sb == sl and TMEM stage sl
                    ring_next(sb, pb, XB_STAGES);
                    ring_next(sl, pl, XL_STAGES);
                    if (cpos == X_CHUNK - 1 || kb == kb1 - 1) {
                        umma_commit(&tfull[ab]);
                        if (++ab == 2) {
                            ab = 0;
                            aphase ^= 1;
                        }
                    }
                }
            }
            umma_commit(done);
            wait_bounded(done, 0);
        }
    } else if (warp < 6) {
        // ---------------- epilogue: split-K partials ----------------
        const int q = warp & 3, r = q * 32 + lane;
        int ab = 0;
        uint32_t aphase = 0;
        for (int item = blockIdx.x; item < args.n_items; item += gridDim.x) {
            int tm, sp, kb0, kb1;
            xprod_item(args, item, tm, sp, kb0, kb1);
            float acc[X_N];
            if (!drain_pair(acc, (kb1 - kb0 + X_CHUNK - 1) / X_CHUNK, tmem_base, q, ab, aphase, tfull, tempty,
                                 abort_flag)) {
                fail(4);
                break;
            }
            const int row = tm * TILE_M + r;
            if (row < args.rows) {
                float2 *Xp = args.C + (int64_t)sp * args.ldc * 32;
#pragma unroll
                for (int l = 0; l < 32; l++) Xp[row + (int64_t)l * args.ldc] = make_float2(acc[2 * l], acc[2 * l + 1]);
            }
        }
    } else {
        // ---------------- converter: A fp32 -> hi and lo in TMEM (L ring); releases the A slot ----------------
        // Thread = row of the A tile = TMEM lane (warp w reaches lanes 32 (w % 4) ..).
        const int q = warp & 3, row = q * 32 + lane;
        const uint32_t lane_base = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)X_L_COL0;
        int sa = 0, sl = 0;
        uint32_t pa = 0, pl = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
            int tm, sp, kb0, kb1;
            xprod_item(args, item, tm, sp, kb0, kb1);
            for (int kb = kb0; kb < kb1; kb++) {
                if (!mbar_wait_warp(&fullA[sa], pa, abort_flag) || !mbar_wait_warp(&emptyL[sl], pl ^ 1, abort_flag)) {
                    fail(5);
                    ok = false;
                    break;
                }
                tc_fence_after();
                // row `row` of the 128-byte-swizzled tile: 16-byte chunk c sits at c ^ (row % 8)
                const float4 *a = (const float4 *)(ringA + sa * X_A_BYTES) + row * 8;
                float hi[BKF], lo[BKF];
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    float4 x = a[c ^ (row & 7)];
                    split3(x.x, hi[4 * c], lo[4 * c]);
                    split3(x.y, hi[4 * c + 1], lo[4 * c + 1]);
                    split3(x.z, hi[4 * c + 2], lo[4 * c + 2]);
                    split3(x.w, hi[4 * c + 3], lo[4 * c + 3]);
                }
                const uint32_t t = lane_base + (uint32_t)(sl * 2 * BKF);
                tmem_st32(t, hi);
                tmem_st32(t + BKF, lo);
                tmem_st_wait();
                tc_fence_before();
                __syncwarp();
                // The A slot is released only now: the completed TMEM stores
                // consumed every value read from it.  Released right after the
                // loads, the next TMA tile (an async-proxy write) could land
                // before loads delayed by other CTAs on the SM had read the slot.
                if (lane == 0) {  // one arrival per warp
                    mbar_arrive(&emptyA[sa]);
                    mbar_arrive(&conv[sl]);
                }
                ring_next(sa, pa, XA_STAGES);
                ring_next(sl, pl, XL_STAGES);
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"((uint32_t)X_TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// C -= P Q^H on the lower-triangle tiles of the Hermitian trailing matrix;
// the strictly upper part is written as the conjugate transpose (so the
// stored matrix stays exactly Hermitian) and diagonal entries stay real.
//   warp 0 producer, warp 1 MMA, warps 2-9 epilogue (two per lane quarter).
// ---------------------------------------------------------------------------
constexpr int F_STAGES = 2;
constexpr int F_N = 256;
constexpr int F_A_BYTES = TILE_M * BKF * 4;  // 16 KB
constexpr int F_B_BYTES = F_N * BKF * 4;     // 32 KB
constexpr int F_STAGE_BYTES = 2 * F_A_BYTES + 2 * F_B_BYTES;
constexpr int F_SMEM = F_STAGES * F_STAGE_BYTES;
// Epilogue staging for the mirrored (upper-triangle) stores: per epilogue
// warp 8 columns x 32 rows of complex64 (one batch of F_LD columns).
constexpr int F_MIRROR_BYTES = 8 * 8 * 33 * 8;
constexpr int F_EPI_COLS = 128;
#ifndef F_CHUNK
#define F_CHUNK 2  // k-blocks per accumulation chunk
#endif
constexpr int F_WARPS = 10;
constexpr int F_TMEM_COLS = 512;

__global__ void __launch_bounds__(F_WARPS * 32, 1)
    flush_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmAlo,
                 const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmBlo, TcArgs args) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + F_SMEM);
    uint64_t *empty = full + F_STAGES;
    uint64_t *tfull = empty + F_STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *done = tempty + 2;
    uint32_t *tmem_slot = (uint32_t *)(done + 1);
    volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int T = args.tiles_m;
    if (threadIdx.x == 0) {
        for (int s = 0; s < F_STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 8);  // one arrival per epilogue warp
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)F_TMEM_COLS)
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
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            long issued = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                int tm, tn;
                lower_tile(item, T, tm, tn);
                for (int kb = 0; kb < args.kblocks; kb++) {
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) {
                        fail(1);
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + s * F_STAGE_BYTES;
                    mbar_expect_tx(&full[s], F_STAGE_BYTES);
                    int x = kb * BKF;
                    tma_load_2d(&tmA, &full[s], st, x, tm * TILE_M);
                    tma_load_2d(&tmAlo, &full[s], st + F_A_BYTES, x, tm * TILE_M);
                    tma_load_2d(&tmB, &full[s], st + 2 * F_A_BYTES, x, tn * F_N);
                    tma_load_2d(&tmBlo, &full[s], st + 2 * F_A_BYTES + F_B_BYTES, x, tn * F_N);
                    issued++;
                    ring_next(s, ph, F_STAGES);
                }
            }
            long outstanding = issued < F_STAGES ? issued : F_STAGES;
            for (long q = 0; q < outstanding; q++) {
                ring_prev(s, ph, F_STAGES);
                wait_bounded(&full[s], ph);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = tf32_idesc(TILE_M, F_N);
            int s = 0, ab = 0;
            uint32_t ph = 0, aphase = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < args.n_items && ok; item += gridDim.x) {
                for (int kb = 0; kb < args.kblocks; kb++) {  // F_CHUNK k-blocks per accumulation chunk
                    const int cpos = kb % F_CHUNK;
                    if (cpos == 0 && !mbar_wait(&tempty[ab], aphase ^ 1, abort_flag)) {
                        fail(2);
                        ok = false;
                        break;
                    }
                    if (!mbar_wait(&full[s], ph, abort_flag)) {
                        fail(3);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)(ab * F_N);
                    const uint32_t a_hi = smem_u32(smem + s * F_STAGE_BYTES);
                    const uint32_t a_lo = a_hi + F_A_BYTES, b_hi = a_lo + F_A_BYTES, b_lo = b_hi + F_B_BYTES;
#pragma unroll
                    for (int kk = 0; kk < BKF / 8; kk++) {
                        uint32_t o = kk * 32;
                        umma_tf32(d, sw128_desc(a_hi + o), sw128_desc(b_hi + o), idesc, (cpos > 0 || kk > 0) ? 1u : 0u);
                        umma_tf32(d, sw128_desc(a_hi + o), sw128_desc(b_lo + o), idesc, 1u);
                        umma_tf32(d, sw128_desc(a_lo + o), sw128_desc(b_hi + o), idesc, 1u);
                    }
                    umma_commit(&empty[s]);
                    ring_next(s, ph, F_STAGES);
                    if (cpos == F_CHUNK - 1 || kb == args.kblocks - 1) {
                        umma_commit(&tfull[ab]);
                        if (++ab == 2) {
                            ab = 0;
                            aphase ^= 1;
                        }
                    }
                }
            }
            umma_commit(done);
            wait_bounded(done, 0);
        }
    } else {
        const int q = warp & 3, r = q * 32 + lane;
        const int cbase = ((warp - 2) >> 2) * F_EPI_COLS;
        int ab = 0;
        uint32_t aphase = 0;
        for (int item = blockIdx.x; item < args.n_items; item += gridDim.x) {
            int tm, tn;
            lower_tile(item, T, tm, tn);
            float acc[F_EPI_COLS];
            if (!drain_item<F_N, F_EPI_COLS>(acc, (args.kblocks + F_CHUNK - 1) / F_CHUNK, tmem_base, q, cbase, ab, aphase, tfull, tempty,
                                             abort_flag)) {
                fail(4);
                break;
            }
            const int row = tm * TILE_M + r;
            const int row0 = tm * TILE_M + q * 32;  // first row of this warp
            float2 *Crow = args.C + row;             // C[row, :]
            const int col0 = tn * (F_N / 2) + cbase / 2;
            // this warp's staging area: stage[j][rr] = updated C[row0 + rr, col0 + j0 + j]
            // (after the 512 bytes of barriers that follow the operand stages)
            float2(*stage)[33] = (float2(*)[33])(smem + F_SMEM + 512 + (warp - 2) * (8 * 33 * 8));
            // Batches of F_LD columns: all loads of a batch are issued before its
            // stores (a store may alias a later load, so the compiler would
            // otherwise keep every load behind the previous store).  The lower
            // element goes back in place (32 consecutive rows of one column per
            // store); its conjugate, the upper element (col, row), is staged in
            // shared memory and stored transposed, so that lanes write runs of 8
            // consecutive rows of a column of C instead of 32 separate columns.
            constexpr int F_LD = 8;
#pragma unroll
            for (int j0 = 0; j0 < F_EPI_COLS / 2; j0 += F_LD) {
                float2 cv[F_LD];
#pragma unroll
                for (int j = 0; j < F_LD; j++) {
                    const int col = col0 + j0 + j;
                    cv[j] = (row < args.rows && col < args.cols && col <= row) ? __ldcg(Crow + (int64_t)col * args.ldc)
                                                                              : make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int j = 0; j < F_LD; j++) {
                    const int col = col0 + j0 + j;
                    float2 c = cv[j];
                    c.x -= acc[2 * (j0 + j)];
                    c.y -= acc[2 * (j0 + j) + 1];
                    if (col == row) c.y = 0.f;
                    if (row < args.rows && col < args.cols && col <= row) Crow[(int64_t)col * args.ldc] = c;
                    stage[j][lane] = c;
                }
                __syncwarp();
                // mirror: lane (rr, cc) stores rows row0 + rr + 4 it of column col0 + j0 + cc of the
                // tile's transpose, i.e. C[col0 + j0 + cc, row0 + rr + 4 it] = conj(stage[cc][rr + 4 it])
                {
                    const int cc = lane & 7, rr = lane >> 3;
                    const int mcol = col0 + j0 + cc;  // row index of the upper element
#pragma unroll
                    for (int it = 0; it < 8; it++) {
                        const int rl = rr + 4 * it;
                        const int mrow = row0 + rl;  // column index of the upper element
                        if (mrow < args.rows && mcol < args.cols && mcol < mrow) {
                            const float2 v = stage[cc][rl];
                            args.C[mcol + (int64_t)mrow * args.ldc] = make_float2(v.x, -v.y);
                        }
                    }
                }
                __syncwarp();
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"((uint32_t)F_TMEM_COLS)
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
    return qd_sm_budget(g_nsm);
}

constexpr int SMEM_EXTRA = 1024 /*alignment*/ + 512 /*barriers*/;

// Device time of every launch of the two kernels, bracketed by CUDA events on
// the launching stream; read (and reset) by qd_tc_kernel_stats.  Also the
// algorithmic work of each launch: bytes of the trailing matrix read by the
// X product (8 m^2), flops of the Hermitian rank-2K update (8 mt (mt+1) K).
struct KernelTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<double> launch_work;  // algorithmic work of each timed launch
    int used = 0;
    double work = 0.0;
};
thread_local KernelTimer g_timer[2];
void timer_mark(int which, cudaStream_t st) {
    KernelTimer &t = g_timer[which];
    if (t.used == (int)t.ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        t.ev.push_back(e);
    }
    cudaEventRecord(t.ev[t.used++], st);
}

int launch_xprod(const CUtensorMap &a, const CUtensorMap &b, const CUtensorMap &blo, const TcArgs &args,
                 cudaStream_t st) {
    static bool configured = false;
    const int smem = X_SMEM + SMEM_EXTRA;
    if (!configured) {
        CUDA_OK(cudaFuncSetAttribute(xprod_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        configured = true;
    }
    int grid = args.n_items < sm_count() ? args.n_items : sm_count();
    if (grid < 1) return QD_OK;
    qd_count_launch(1);
    timer_mark(0, st);
    xprod_kernel<<<grid, X_WARPS * 32, smem, st>>>(a, b, blo, args);
    CUDA_OK(cudaGetLastError());
    timer_mark(0, st);
    g_timer[0].work += 8.0 * (double)args.rows * (double)args.rows;
    g_timer[0].launch_work.push_back(8.0 * (double)args.rows * (double)args.rows);
    return QD_OK;
}

int launch_flush(const CUtensorMap &a, const CUtensorMap &alo, const CUtensorMap &b, const CUtensorMap &blo,
                 const TcArgs &args, cudaStream_t st) {
    static bool configured = false;
    const int smem = F_SMEM + F_MIRROR_BYTES + SMEM_EXTRA;
    if (!configured) {
        CUDA_OK(cudaFuncSetAttribute(flush_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        configured = true;
    }
    int grid = args.n_items < sm_count() ? args.n_items : sm_count();
    if (grid < 1) return QD_OK;
    qd_count_launch(1);
    timer_mark(1, st);
    flush_kernel<<<grid, F_WARPS * 32, smem, st>>>(a, alo, b, blo, args);
    CUDA_OK(cudaGetLastError());
    timer_mark(1, st);
    g_timer[1].work += 8.0 * (double)args.rows * (double)(args.rows + 1) * (double)args.kdim;
    g_timer[1].launch_work.push_back(8.0 * (double)args.rows * (double)(args.rows + 1) * (double)args.kdim);
    return QD_OK;
}

}  // namespace

// Limit of the pipeline waits for the current device (ns; negative: default).
extern "C" int qd_tc_set_wait_limit(long long ns) {
    const unsigned long long v = ns < 0 ? WAIT_NS_DEFAULT : (unsigned long long)ns;
    CUDA_OK(cudaMemcpyToSymbol(g_wait_ns, &v, sizeof(v)));
    return QD_OK;
}

extern "C" void qd_tc_work_free_on(struct QdTcWork *w, cudaStream_t st);

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

extern "C" int qd_tc_work_alloc_on(int64_t n, int kmax, QdTcWork **out, cudaStream_t st) {
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
    void **dst[8] = {(void **)&w->bx_hi, (void **)&w->bx_lo, (void **)&w->xp, (void **)&w->fa_hi,
                     (void **)&w->fa_lo, (void **)&w->fb_hi, (void **)&w->fb_lo, (void **)&w->err};
    size_t sz[8] = {bx, bx, xp, fa, fa, fb, fb, sizeof(int)};
    for (int i = 0; i < 8; i++) {
        if (qd_pool_alloc(dst[i], sz[i], st) != 0) {
            qd_tc_work_free_on(w, st);
            return qd_set_error(QD_ERR_NOMEM, "tensor-core work buffers: %zu bytes", sz[i]);
        }
    }
    CUDA_OK(cudaMemsetAsync(w->err, 0, sizeof(int), st));
    *out = w;
    return QD_OK;
}

extern "C" void qd_tc_work_free_on(QdTcWork *w, cudaStream_t st) {
    if (!w) return;
    void *p[8] = {w->bx_hi, w->bx_lo, w->xp, w->fa_hi, w->fa_lo, w->fb_hi, w->fb_lo, w->err};
    for (int i = 0; i < 8; i++)
        if (p[i]) qd_pool_free(p[i], st);
    free(w);
}

extern "C" int qd_tc_work_alloc(int64_t n, int kmax, QdTcWork **out) {
    int rc = qd_tc_work_alloc_on(n, kmax, out, 0);
    if (rc == QD_OK) CUDA_OK(cudaStreamSynchronize(0));
    return rc;
}

extern "C" void qd_tc_work_free(QdTcWork *w) { qd_tc_work_free_on(w, 0); }

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
    // Split-K count: the items (row tile, k range) are equal, so the grid of
    // one CTA per SM finishes together when their count is just below a
    // multiple of the SM count.  Pick the split with the best fill of the last
    // wave (ties: fewer splits, fewer partials to reduce).
    const int nsm = sm_count();
    int splits = 1;
    double best = -1.0;
    for (int sp = 1; sp <= w->max_splits && sp <= a.kblocks; sp++) {
        const long items = (long)a.tiles_m * sp;
        const long waves = (items + nsm - 1) / nsm;
        const double fill = (double)items / (double)(waves * nsm);
        if (fill > best + 1e-3) {
            best = fill;
            splits = sp;
        }
    }
    a.splits = splits;
    a.n_items = a.tiles_m * splits;
    a.kdim = 0;
    a.rows = m;
    a.cols = nb;
    a.a_x0 = (int)(2 * off);
    a.a_y0 = (int)off;
    a.C = w->xp;
    a.ldc = w->ldp;
    a.err = w->err;
    if (m > w->ldp) return qd_set_error(QD_ERR_ARG, "qd_tc_xprod: m exceeds the work buffers");
    if ((rc = launch_xprod(ta, tb, tblo, a, st))) return rc;
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
    a.tiles_n = a.tiles_m;
    a.splits = 1;
    a.kblocks = (int)((pitch + BKF - 1) / BKF);
    a.n_items = a.tiles_m * (a.tiles_m + 1) / 2;  // lower-triangle tiles
    a.kdim = K;
    a.rows = mt;
    a.cols = mt;
    a.a_x0 = 0;
    a.a_y0 = 0;
    a.C = (float2 *)A + off + off * lda;
    a.ldc = lda;
    a.err = w->err;
    return launch_flush(ta, talo, tb, tblo, a, st);
}

// Per-launch device times (ms) and algorithmic work of the X-product (which =
// 0) or trailing-update kernel (which = 1) since the previous reset, without
// resetting: up to `cap` launches into ms[] and work[]; returns the number
// of launches recorded (or a negative QD_ERR_*).  Synchronises the device.
extern "C" int qd_tc_kernel_launches(int which, int cap, double *ms, double *work) {
    if (which < 0 || which > 1 || cap < 0) return -qd_set_error(QD_ERR_ARG, "qd_tc_kernel_launches: bad arguments");
    if (cudaDeviceSynchronize() != cudaSuccess) return -qd_set_error(QD_ERR_CUDA, "qd_tc_kernel_launches: sync");
    KernelTimer &t = g_timer[which];
    const int n = t.used / 2;
    for (int i = 0; i < n && i < cap; i++) {
        float x = 0.f;
        if (cudaEventElapsedTime(&x, t.ev[2 * i], t.ev[2 * i + 1]) != cudaSuccess)
            return -qd_set_error(QD_ERR_CUDA, "qd_tc_kernel_launches: event");
        ms[i] = x;
        work[i] = i < (int)t.launch_work.size() ? t.launch_work[i] : 0.0;
    }
    return n;
}

// Launches, summed device time (ms) and algorithmic work of the X-product
// (which = 0; work in bytes) or trailing-update kernel (which = 1; work in
// flops) since the previous call; synchronises the device.
extern "C" int qd_tc_kernel_stats(int which, long long *launches, double *ms, double *work) {
    if (which < 0 || which > 1) return qd_set_error(QD_ERR_ARG, "qd_tc_kernel_stats: which must be 0 or 1");
    CUDA_OK(cudaDeviceSynchronize());
    KernelTimer &t = g_timer[which];
    double total = 0.0;
    for (int i = 0; i + 1 < t.used; i += 2) {
        float x = 0.f;
        CUDA_OK(cudaEventElapsedTime(&x, t.ev[i], t.ev[i + 1]));
        total += x;
    }
    *launches = t.used / 2;
    *ms = total;
    *work = t.work;
    t.used = 0;
    t.work = 0.0;
    t.launch_work.clear();
    return QD_OK;
}

// Shared pieces of the eigensolver kernels: complex scalar templates, block
// reductions and the stage-1 workspace.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

template <typename R>
struct cpx {
    R re, im;
};

// Workspace of the dense -> band reduction (eig_stage1.cu).
struct Stage1Work {
    void *VT, *X, *M, *Y, *Tall, *Rall, *Vacc, *Wacc, *S1, *S2, *gram, *tau;
    void *part;  // partial sums of the tall A^H B reductions (panel_ops.cu)
    size_t part_bytes;
    struct QdTcWork *tc;  // tensor-core GEMM work buffers (mixed path), or null
    double2 *red, *rowbuf;
    unsigned *bar;
    int *err;
    int npanels, agg;
    int64_t ldv;
};

template <typename R>
__device__ __forceinline__ cpx<R> mk(R a, R b) {
    cpx<R> z;
    z.re = a;
    z.im = b;
    return z;
}
template <typename R>
__device__ __forceinline__ cpx<R> cadd(cpx<R> a, cpx<R> b) { return mk<R>(a.re + b.re, a.im + b.im); }
template <typename R>
__device__ __forceinline__ cpx<R> csub(cpx<R> a, cpx<R> b) { return mk<R>(a.re - b.re, a.im - b.im); }
template <typename R>
__device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
    return mk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ cpx<R> cmulc(cpx<R> a, cpx<R> b) {
    return mk<R>(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
}
template <typename R>
__device__ __forceinline__ cpx<R> cconj(cpx<R> a) { return mk<R>(a.re, -a.im); }
template <typename R>
__device__ __forceinline__ R cabs2(cpx<R> a) { return a.re * a.re + a.im * a.im; }

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block of one double; every thread gets the result.  `scratch`
// holds >= 33 doubles in shared memory.
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = lane < nw ? scratch[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) scratch[32] = t;
    }
    __syncthreads();
    return scratch[32];
}

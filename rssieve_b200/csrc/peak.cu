// peak.cu -- the roofline denominators of the BSGS kernel, measured on the
// device: the Montgomery-product throughput (every thread runs eight
// independent dependency chains of the same mmul() the kernels use, so the
// 32-bit IMAD pipe, not latency, is the limit, on a 62-bit prime) and the raw
// 32x32->64 multiply throughput, from which the multiplier-bound product rate
// is the wide-multiply rate / 11, and the FP64 modular-product throughput of
// the steps below 2^51.  Rates are operations / kernel time (CUDA events on
// the stream).
#include "mont.cuh"
#include "rs_internal.h"

namespace rs {

__global__ void __launch_bounds__(256) k_mulmod_peak(u64 *out, u64 p, u64 q, u64 b, int iters)
{
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    u64 a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = (t * 8ull + j + 1) % p;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = mmul(a[j], b, p, q);
    }
    u64 x = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) x ^= a[j];
    out[t] = x;
}

// Wide-multiply throughput: sixteen independent chains per thread of one
// 32x32->64 multiply-add each step, c = lo32(c) * m + c (mad.wide.u32, whose
// low operand is the previous result, so nothing can be hoisted or folded).
// A 64-bit Montgomery product needs 11 such products (a*b: 4, lo*q mod 2^64:
// 3, hi(m*p): 4), so rate / 11 is the product rate the multiplier allows.
__global__ void __launch_bounds__(256) k_widemul_peak(u64 *out, u32 m, int iters)
{
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    u64 c[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) c[j] = t * 16ull + j + 1;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) c[j] = (u64)(u32)c[j] * m + c[j];
    }
    u64 x = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) x ^= c[j];
    out[t] = x;
}

// FP64 modular-product throughput: eight independent chains per thread of the
// kernels' fp_mulfix by a fixed multiplier, on a prime just above 2^50 (the
// 100-sequence benchmark's p-range), where the BSGS steps use it.
__global__ void __launch_bounds__(256) k_fpmul_peak(u64 *out, double p, double w, double wq, int iters)
{
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = (double)(t * 8ull + j + 1);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fp_mulfix(a[j], w, wq, p);
    }
    u64 x = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) x ^= (u64)a[j];
    out[t] = x;
}

cudaError_t launch_fpmul_peak(u64 *out, int blocks, int iters, cudaStream_t st)
{
    const u64 p = 1125899906842679ull;       // prime just above 2^50
    const u64 w = 0x123456789ABCull % p;
    k_fpmul_peak<<<blocks, 256, 0, st>>>(out, (double)p, (double)w, (double)w / (double)p, iters);
    return cudaGetLastError();
}

cudaError_t launch_widemul_peak(u64 *out, int blocks, int iters, cudaStream_t st)
{
    k_widemul_peak<<<blocks, 256, 0, st>>>(out, 0x9E3779B1u, iters);
    return cudaGetLastError();
}

cudaError_t launch_mulmod_peak(u64 *out, int blocks, int iters, cudaStream_t st)
{
    const u64 p = 4611686018427387847ull;    // prime below 2^62
    u64 q = p;
    for (int i = 0; i < 5; ++i) q *= 2 - p * q;
    k_mulmod_peak<<<blocks, 256, 0, st>>>(out, p, q, 0x123456789ABCDEFull % p, iters);
    return cudaGetLastError();
}

}  // namespace rs

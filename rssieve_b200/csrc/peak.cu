// peak.cu -- the chip's Montgomery-product throughput, the roofline
// denominator for the BSGS kernel.  Every thread runs eight independent
// dependency chains of the same mmul() the kernels use (so the 32-bit IMAD
// pipe, not latency, is the limit), on a 62-bit prime, for a fixed number of
// steps; the rate is products / kernel time (CUDA events on the stream).
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

cudaError_t launch_mulmod_peak(u64 *out, int blocks, int iters, cudaStream_t st)
{
    const u64 p = 4611686018427387847ull;    // prime below 2^62
    u64 q = p;
    for (int i = 0; i < 5; ++i) q *= 2 - p * q;
    k_mulmod_peak<<<blocks, 256, 0, st>>>(out, p, q, 0x123456789ABCDEFull % p, iters);
    return cudaGetLastError();
}

}  // namespace rs

// noalloc.cu -- prime generation into caller-owned device memory, with no
// device allocation on any call.
//
// The generator behind rs_primes_generate (k_sieve, then the Baillie-PSW test
// of sieve.cu) needs scratch: the table of odd sieving primes below 2^16, the
// buffer of sieve survivors that the test reads, and counters.
// rs_primes_generate keeps these in its context, allocated with cudaMalloc.
// This variant keeps them in one file-scope device array of fixed size,
// g_na_scratch below, so a call allocates nothing; the caller passes the
// output array and the count word.  It runs the one-pass form of the test
// (k_mr), which needs no second list of base-2 probable primes; the primes it
// returns are the same.
//
// Limit: a call covers at most RS_NOALLOC_MAX_WIDTH = 2^22 integers, i.e. at
// most 2^21 odd values, which is exactly the survivor capacity, so the
// survivor buffer can never overflow.  Wider ranges are rejected with RS_EARG.
//
// Set-up: the first call in a CUDA context (the primary context of the device
// current on the calling thread, or the driver-API context made current)
// looks up the scratch address with cudaGetSymbolAddress, fills the
// sieving-prime table with a one-CTA kernel on the caller's stream and waits
// for that stream.  Later calls in that context only enqueue work and return;
// they still query the symbol address and the context's unique ID, so a
// context created anew (after cudaDeviceReset, whose new context holds a
// zeroed copy of the array) is set up again rather than trusted.  The first
// call in a context should therefore come before any stream capture.
//
// What starts at zero: every call resets the survivor counter, the error word
// and the caller's count word with cudaMemsetAsync on the caller's stream
// before its kernels; the output array needs no clearing.
//
// There is one scratch per device: two calls whose work overlaps on the
// device (different streams, no ordering between them) race on it and give
// wrong results.  Order them on one stream or with events.
#include <cstdio>
#include <mutex>

#include "rs_host.h"
#include "rs_internal.h"

using namespace rs;

namespace {

constexpr u32 NA_CAND_CAP = 1u << 21;        // survivor slots (u64 each): 16 MiB
constexpr u32 NA_SP_SLOTS = 6656;            // u32 slots for the 6541 odd primes < 2^16
constexpr u32 NA_NSP = 6541;                 // pi(2^16) - 1
constexpr u32 NA_CTR_SLOTS = 64;             // u32: [0] survivors [1] error flags [2] set-up count
constexpr size_t NA_WORDS = NA_CAND_CAP + NA_SP_SLOTS / 2 + NA_CTR_SLOTS / 2;
static_assert(RS_NOALLOC_MAX_WIDTH / 2 == NA_CAND_CAP, "survivor capacity must cover every odd value of a call");

// The scratch: survivors, then sieving primes, then counters (all offsets
// are multiples of 256 bytes).
static __device__ __align__(256) u64 g_na_scratch[NA_WORDS];

// Contexts set up so far, by the driver's unique context ID (never reused in
// a process).  A context beyond the table's capacity replaces the oldest entry.
constexpr int NA_MAX_CTX = 64;
struct CtxState {
    unsigned long long ctx_id = 0;    // 0: unused
    u64 *scratch = nullptr;
    int sms = 0;
};
std::mutex g_na_mu;
CtxState g_na_ctx[NA_MAX_CTX];
int g_na_next = 0;

// The unique ID of the calling thread's current context, through the driver
// entry points the runtime exposes (no link against the driver library).
typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);
int current_ctx_id(unsigned long long *id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
            rs_set_error("the CUDA driver does not provide cuCtxGetCurrent/cuCtxGetId");
            return RS_ECUDA;
        }
        get_current = (CtxGetCurrentFn)f1;
        get_id = (CtxGetIdFn)f2;
    }
    void *ctx = nullptr;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
        rs_set_error("no current CUDA context");
        return RS_ECUDA;
    }
    return RS_OK;
}

// Odd primes below 2^16 in ascending order: one CTA sieves the 2^15 odd
// values 2i+1 in shared memory and compacts them with a block-wide scan.
__global__ void __launch_bounds__(1024) k_na_small_primes(u32 *__restrict__ sp, u32 *__restrict__ count)
{
    __shared__ u32 comp[1024];                // bit i of word w: value 2(32w+i)+1 is composite
    __shared__ u32 warp_sum[32];
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    comp[tid] = (tid == 0) ? 1u : 0u;         // 1 is not prime
    __syncthreads();
    for (u32 r = 3; r < 256; r += 2) {
        // multiples r*r, r*r+2r, ... as odd indices (v-1)/2
        for (u32 i = (r * r - 1) / 2 + tid * r; i < 32768; i += 1024 * r) atomicOr(&comp[i >> 5], 1u << (i & 31));
    }
    __syncthreads();
    const u32 live = ~comp[tid];
    const u32 cnt = __popc(live);
    u32 incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (u32)o) incl += v;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        u32 s = warp_sum[lane], t = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 v = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= (u32)o) t += v;
        }
        warp_sum[lane] = t - s;               // exclusive prefix of the warp totals
        if (lane == 31) *count = t;
    }
    __syncthreads();
    u32 pos = warp_sum[warp] + incl - cnt;
    u32 bits = live;
    while (bits) {
        u32 b = __ffs(bits) - 1;
        bits &= bits - 1;
        sp[pos++] = 2 * (tid * 32 + b) + 1;
    }
}

#define NA_CU(call)                                                                           \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            rs_set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return RS_ECUDA;                                                                  \
        }                                                                                     \
    } while (0)

// Once per context, with it current: SM count and the sieving-prime table in
// the scratch at ptr.  Waits for the caller's stream.
int na_setup(int dev, void *ptr, cudaStream_t st, CtxState *out)
{
    int sms = 0;
    NA_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    u64 *scr = (u64 *)ptr;
    u32 *sp = (u32 *)(scr + NA_CAND_CAP);
    u32 *ctrs = sp + NA_SP_SLOTS;
    k_na_small_primes<<<1, 1024, 0, st>>>(sp, ctrs + 2);
    NA_CU(cudaGetLastError());
    u32 n = 0;
    NA_CU(cudaMemcpyAsync(&n, ctrs + 2, 4, cudaMemcpyDeviceToHost, st));
    NA_CU(cudaStreamSynchronize(st));
    if (n != NA_NSP) {
        rs_set_error("static scratch set-up found %u sieving primes, expected %u", n, NA_NSP);
        return RS_EDEVICE;
    }
    out->scratch = scr;
    out->sms = sms;
    return RS_OK;
}

}  // namespace

extern "C" int rs_primes_generate_noalloc(uint64_t p0, uint64_t p1, uint64_t *d_primes, uint32_t cap,
                                          uint32_t *d_count, void *stream)
{
    if (!d_count || (!d_primes && cap)) {
        rs_set_error("rs_primes_generate_noalloc: d_count is NULL, or d_primes is NULL with cap > 0");
        return RS_EARG;
    }
    if (p0 >= p1) {
        rs_set_error("rs_primes_generate_noalloc: empty range [%llu, %llu)", (unsigned long long)p0,
                     (unsigned long long)p1);
        return RS_EARG;
    }
    if (p1 - p0 > RS_NOALLOC_MAX_WIDTH) {
        rs_set_error("rs_primes_generate_noalloc: range width %llu exceeds the static scratch limit of %llu "
                     "integers per call",
                     (unsigned long long)(p1 - p0), (unsigned long long)RS_NOALLOC_MAX_WIDTH);
        return RS_EARG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        rs_set_error("no CUDA device available");
        return RS_ENODEV;
    }
    int dev = -1;
    NA_CU(cudaGetDevice(&dev));
    // the address in this context (this also makes the runtime's context current)
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_na_scratch);
    if (e != cudaSuccess || !ptr) {
        rs_set_error("cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                     cudaGetErrorString(e));
        return RS_ECUDA;
    }
    unsigned long long cid = 0;
    int rc = current_ctx_id(&cid);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    CtxState ds;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        int slot = -1;
        for (int i = 0; i < NA_MAX_CTX; ++i)
            if (g_na_ctx[i].ctx_id == cid) slot = i;
        if (slot < 0 || g_na_ctx[slot].scratch != (u64 *)ptr) {
            if (slot < 0) {
                slot = g_na_next;
                g_na_next = (g_na_next + 1) % NA_MAX_CTX;
            }
            g_na_ctx[slot] = CtxState();
            CtxState fresh;
            rc = na_setup(dev, ptr, st, &fresh);
            if (rc) return rc;
            fresh.ctx_id = cid;
            g_na_ctx[slot] = fresh;
        }
        ds = g_na_ctx[slot];
    }
    u64 *cands = ds.scratch;
    u32 *sp = (u32 *)(ds.scratch + NA_CAND_CAP);
    u32 *ctrs = sp + NA_SP_SLOTS;
    if (p0 < 3) p0 = 3;
    u64 base = p0 | 1ull;
    u64 nodd = (base < p1) ? (p1 - base + 1) / 2 : 0;
    NA_CU(cudaMemsetAsync(ctrs, 0, 2 * sizeof(u32), st));
    NA_CU(cudaMemsetAsync(d_count, 0, sizeof(u32), st));
    if (nodd == 0) return RS_OK;
    NA_CU(launch_sieve(base, nodd, p1, sp, NA_NSP, cands, NA_CAND_CAP, ctrs, ctrs + 1, st));
    NA_CU(launch_mr(cands, ctrs, NA_CAND_CAP, (u64 *)d_primes, cap, d_count, ctrs + 1, ds.sms, st));
    return RS_OK;
}

// sieve.cu -- sieve-prime generation over a segment [lo, hi) of the p-range.
//
// Replaces the reference's getsegprimes/addsmallprimes kernels
// (kernels/getsegprimes.cl:128-182, kernels/addsmallprimes.cl:8-27, driven by
// cl_sieve.cpp:1303-1320).  The reference emits base-2 strong probable primes
// after removing multiples of 2..113; here each CTA runs a segmented
// Eratosthenes sieve over 2^17 odd numbers in shared memory with every odd
// prime below 2^16, compacts the survivors with warp ballots/popc, and a
// second kernel proves the survivors at or above 65537^2 prime with the
// Baillie-PSW test (a base-2 strong probable-prime test, then a strong Lucas
// test; deterministic below 2^64, see is_prime_bpsw).  Survivors below
// 65537^2 are prime already.  The result is the exact set of odd primes in
// [lo, hi).
#include "mont.cuh"
#include "rs_internal.h"

namespace rs {

// x mod r for a 64-bit x and a 32-bit r, from three 32-bit remainders.
__device__ __forceinline__ u32 mod64_32(u64 x, u32 r)
{
    u32 hi = (u32)(x >> 32), lo = (u32)x;
    u32 t = (u32)(0u - r) % r;            // 2^32 mod r
    u64 a = (u64)(hi % r) * t + (lo % r); // < r^2 + r < 2^33
    return (u32)(a % r);
}

// One CTA sieves odd values base_odd + 2*i for i in [blk*BITS, blk*BITS+nbits).
// ctrs[0] counts survivors written to cands.  The caller's exit test is
// uniform over the CTA.
__device__ __forceinline__ void sieve_block(u64 base_odd, u64 nodd, u32 blk, const u32 *__restrict__ sp, u32 nsp,
                                            u64 *__restrict__ cands, u32 cand_cap, u32 *ctrs, u32 *err)
{
    constexpr u32 BITS = SIEVE_WORDS * 32;
    __shared__ u32 bits[SIEVE_WORDS];
    __shared__ u32 starts[7000];
    const u32 tid = threadIdx.x;
    const u64 i0 = (u64)blk * BITS;
    if (i0 >= nodd) return;
    // the table must start with 3: an empty or zeroed table would make the
    // one-prime-per-thread marking loop below step by 0 forever
    if (nsp == 0 || sp[0] != 3u) {
        if (tid == 0) atomicOr(err, ERR_SIEVE_TABLE);
        return;
    }
    const u32 nbits = (u32)min((u64)BITS, nodd - i0);
    const u64 bb = base_odd + 2 * i0;                   // value of bit 0 (odd)
    const u64 vlast = bb + 2 * (u64)(nbits - 1);
    for (u32 w = tid; w < SIEVE_WORDS; w += SIEVE_TPB) bits[w] = 0;

    // first index to mark for each sieving prime r with r^2 <= vlast
    u32 np_used = 0;
    for (u32 k = tid; k < nsp; k += SIEVE_TPB) {
        u32 r = sp[k];
        u64 rr = (u64)r * r;
        u32 s = 0xFFFFFFFFu;
        if (rr <= vlast) {
            u32 m = mod64_32(bb, r);
            u32 j = (u32)(((u64)((r - m) % r) * ((r + 1) >> 1)) % r);   // bb + 2j == 0 (mod r)
            u64 v = bb + 2 * (u64)j;
            if (v < rr) j = (u32)((rr - bb) >> 1);                     // start at r^2, never at r
            if ((u64)j < nbits) s = j;
        }
        starts[k] = s;
    }
    // number of primes with r^2 <= vlast (sp is ascending)
    {
        u32 lo = 0, hi2 = nsp;
        while (lo < hi2) {
            u32 mid = (lo + hi2) >> 1;
            if ((u64)sp[mid] * sp[mid] <= vlast) lo = mid + 1; else hi2 = mid;
        }
        np_used = lo;
    }
    __syncthreads();

    // small primes: all threads stride over the multiples of one prime
    u32 k = 0;
    for (; k < np_used && sp[k] < 2 * SIEVE_TPB; ++k) {
        u32 r = sp[k], s = starts[k];
        if (s == 0xFFFFFFFFu) continue;
        for (u32 i = s + tid * r; i < nbits; i += SIEVE_TPB * r) atomicOr(&bits[i >> 5], 1u << (i & 31));
    }
    // large primes: one prime per thread
    for (u32 kk = k + tid; kk < np_used; kk += SIEVE_TPB) {
        u32 r = sp[kk], s = starts[kk];
        for (u32 i = s; i < nbits; i += r) atomicOr(&bits[i >> 5], 1u << (i & 31));
    }
    __syncthreads();

    // warp-ballot / popc compaction of the unmarked (prime or MR-candidate) values
    const u32 lane = tid & 31;
    const u32 nw = (nbits + 31) >> 5;
    for (u32 w0 = 0; w0 < SIEVE_WORDS; w0 += SIEVE_TPB) {
        u32 w = w0 + tid;
        u32 live = 0;
        if (w < nw) {
            live = ~bits[w];
            u32 rem = nbits - w * 32;
            if (rem < 32) live &= (1u << rem) - 1;
        }
        u32 cnt = __popc(live);
        u32 incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (u32)o) incl += v;
        }
        u32 total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        u32 basepos = 0;
        if (lane == 31 && total) basepos = atomicAdd(&ctrs[0], total);
        basepos = __shfl_sync(0xFFFFFFFFu, basepos, 31);
        if (total == 0) continue;
        u32 pos = basepos + incl - cnt;
        if (basepos + total > cand_cap) {
            if (lane == 0) atomicOr(err, ERR_CAND_OVERFLOW);
            continue;
        }
        while (live) {
            u32 b = __ffs(live) - 1;
            live &= live - 1;
            cands[pos++] = bb + 2 * (u64)(w * 32 + b);
        }
    }
}

__global__ void __launch_bounds__(SIEVE_TPB) k_sieve(u64 base_odd, u64 nodd, const u32 *__restrict__ sp, u32 nsp,
                                                     u64 *__restrict__ cands, u32 cand_cap, u32 *ctrs, u32 *err)
{
    sieve_block(base_odd, nodd, blockIdx.x, sp, nsp, cands, cand_cap, ctrs, err);
}

// Batch round: blockIdx.y is the range; its window and buffers come from the
// range's slots.
__global__ void __launch_bounds__(SIEVE_TPB) k_sieve_batch(const BatchWin *__restrict__ wins, const u32 *__restrict__ sp,
                                                           u32 nsp, u64 *__restrict__ cands, u32 ccap, u32 *ctrs,
                                                           u32 *err)
{
    const u32 r = blockIdx.y;
    const BatchWin w = wins[r];
    sieve_block(w.base_odd, w.nodd, blockIdx.x, sp, nsp, cands + (size_t)r * ccap, ccap, ctrs + r * BR_CTRS, err);
}

// Strong probable prime to base a (a < n), n - 1 = d * 2^t with d odd.
__device__ __forceinline__ bool sprp_base(u64 n, const Mont &M, u64 d, int t, u64 a)
{
    const u64 mone = n - M.one;           // Montgomery form of -1
    u64 x = mpow(to_mont(a, M), d, M);
    if (x == M.one || x == mone) return true;
    for (int s = 1; s < t; ++s) {
        x = mmul(x, x, n, M.q);
        if (x == mone) return true;
    }
    return false;
}

// Deterministic primality below 2^64: the seven strong-probable-prime bases
// of verify_factor.c:102.
__device__ bool is_prime_mr(u64 n)
{
    if (n < MR_BOUND) return true;        // sieve survivor below 65537^2
    const u32 bases[7] = {2u, 325u, 9375u, 28178u, 450775u, 9780504u, 1795265022u};
    const Mont M = mont_init(n);
    const u64 nm1 = n - 1;
    const int t = __ffsll((long long)nm1) - 1;
    const u64 d = nm1 >> t;
    for (int i = 0; i < 7; ++i)           // every base is below n >= 65537^2
        if (!sprp_base(n, M, d, t, bases[i])) return false;
    return true;
}

// floor(sqrt(n))^2 == n, by the bitwise integer square root.
__device__ bool is_square(u64 n)
{
    u64 r = 0, bit = 1ull << 62, x = n;
    while (bit > x) bit >>= 2;
    while (bit) {
        if (x >= r + bit) { x -= r + bit; r = (r >> 1) + bit; }
        else r >>= 1;
        bit >>= 2;
    }
    return r * r == n;
}

// x / 2 mod n for odd n and x in [0, n); also halves a Montgomery residue.
__device__ __forceinline__ u64 mhalf(u64 x, u64 n)
{
    return (x & 1) ? (x >> 1) + (n >> 1) + 1 : x >> 1;
}

// Selfridge's D for n (odd, not 1): the first of 5, -7, 9, -11, ... with
// Jacobi (D/n) = -1.  Returns 0 when the search shows n composite (a common
// factor, or n a square, which has no such D) and 1 when no D turned up
// within 64 candidates; neither is a possible D.
__device__ int selfridge_d(u64 n)
{
    int D = 5;
    for (int tries = 0;; ++tries) {
        if (tries == 64) return 1;
        const u32 a = (u32)(D < 0 ? -D : D);
        int j = jacobi32((u32)(n % a), a);                 // (n/a), then reciprocity
        if ((a & 3) == 3 && (n & 3) == 3) j = -j;
        if (D < 0 && (n & 3) == 3) j = -j;                 // (-1/n)
        if (j == -1) return D;
        if (j == 0) return 0;                              // gcd(a, n) > 1 with a < n
        if (tries == 8 && is_square(n)) return 0;          // a square has no such D
        D = (D > 0) ? -(D + 2) : (-D + 2);
    }
}

// Strong Lucas probable-prime test with Selfridge's parameters: D is the first
// of 5, -7, 9, -11, ... with Jacobi (D/n) = -1, P = 1, Q = (1 - D)/4; with
// n + 1 = d * 2^s (d odd), n passes if U_d = 0 or V_(d*2^r) = 0 for some r < s.
// Only V is carried: the ladder keeps the pair (V_k, V_(k+1)) and Q^k in
// Montgomery form and per bit b of d forms
//   V_(2k+1) = V_k V_(k+1) - P Q^k,   V_(2(k+b)) = V_(k+b)^2 - 2 Q^(k+b),
//   Q^(2k+b) = Q^k Q^(k+b),
// four products whatever b is, so the lanes of a warp never diverge on the
// bits of their own d.  U_d follows from D U_k = 2 V_(k+1) - P V_k (with
// alpha, beta the roots of x^2 - P x + Q: 2(alpha^(k+1) + beta^(k+1)) -
// (alpha + beta)(alpha^k + beta^k) = (alpha - beta)(alpha^k - beta^k)), and
// gcd(D, n) = 1, so U_d = 0 exactly when 2 V_(d+1) = V_d.  Returns 1 (probable
// prime), 0 (composite), or -1 when no D turned up within 64 candidates (the
// caller then decides otherwise).  n is odd, above 65537^2 and below 2^64 - 1.
__device__ int lucas_strong(u64 n, const Mont &M)
{
    const int D = selfridge_d(n);
    if (D == 0) return 0;
    if (D == 1) return -1;
    const int Qi = (1 - D) / 4;
    const u64 Qm = to_mont(Qi >= 0 ? (u64)Qi : n - (u64)(-Qi), M);
    const int s = __ffsll((long long)(n + 1)) - 1;
    const u64 d = (n + 1) >> s;
    // k = 1: V_1 = P = 1, V_2 = P^2 - 2Q
    u64 Vk = M.one, Vk1 = msub(M.one, madd(Qm, Qm, n), n), Qk = Qm;
    for (int bit = 62 - __clzll(d); bit >= 0; --bit) {
        const bool one = (d >> bit) & 1;
        const u64 t = mmul(Qk, one ? Qm : M.one, n, M.q);            // Q^(k+b)
        const u64 mid = msub(mmul(Vk, Vk1, n, M.q), Qk, n);          // V_(2k+1)
        const u64 vs = one ? Vk1 : Vk;
        const u64 sq = msub(mmul(vs, vs, n, M.q), madd(t, t, n), n);  // V_(2(k+b))
        Qk = mmul(Qk, t, n, M.q);
        Vk = one ? mid : sq;
        Vk1 = one ? sq : mid;
    }
    if (madd(Vk1, Vk1, n) == Vk) return 1;                 // U_d = 0
    u64 V = Vk;
    for (int r = 0; r < s; ++r) {
        if (V == 0) return 1;
        if (r + 1 < s) {
            V = msub(mmul(V, V, n, M.q), madd(Qk, Qk, n), n);
            Qk = mmul(Qk, Qk, n, M.q);
        }
    }
    return 0;
}

// lucas_strong for n < 2^51 on the FP64 pipe: the same ladder on plain
// residues held exactly in doubles, products by fp_mul (1/n correctly
// rounded), sums and differences exact in doubles with one correction each.
__device__ int lucas_strong_fp(u64 n)
{
    const int D = selfridge_d(n);
    if (D == 0) return 0;
    if (D == 1) return -1;
    const double nd = fp_exact(n), ninv = 1.0 / nd;
    auto add = [&](double a, double b) { const double t = a + b; return (t >= nd) ? t - nd : t; };
    auto sub = [&](double a, double b) { const double t = a - b; return (t < 0.0) ? t + nd : t; };
    const int Qi = (1 - D) / 4;
    const double Qd = fp_exact(Qi >= 0 ? (u64)Qi : n - (u64)(-Qi));
    const int s = __ffsll((long long)(n + 1)) - 1;
    const u64 d = (n + 1) >> s;
    // k = 1: V_1 = P = 1, V_2 = P^2 - 2Q
    double Vk = 1.0, Vk1 = sub(1.0, add(Qd, Qd)), Qk = Qd;
    for (int bit = 62 - __clzll(d); bit >= 0; --bit) {
        const bool one = (d >> bit) & 1;
        const double t = fp_mul(Qk, one ? Qd : 1.0, nd, ninv);          // Q^(k+b)
        const double mid = sub(fp_mul(Vk, Vk1, nd, ninv), Qk);          // V_(2k+1)
        const double vs = one ? Vk1 : Vk;
        const double sq = sub(fp_mul(vs, vs, nd, ninv), add(t, t));     // V_(2(k+b))
        Qk = fp_mul(Qk, t, nd, ninv);
        Vk = one ? mid : sq;
        Vk1 = one ? sq : mid;
    }
    if (add(Vk1, Vk1) == Vk) return 1;                     // U_d = 0
    double V = Vk;
    for (int r = 0; r < s; ++r) {
        if (V == 0.0) return 1;
        if (r + 1 < s) {
            V = sub(fp_mul(V, V, nd, ninv), add(Qk, Qk));
            Qk = fp_mul(Qk, Qk, nd, ninv);
        }
    }
    return 0;
}

// The strong Lucas test on the pipe that suits n.
__device__ __forceinline__ int lucas_test(u64 n)
{
    return (n < FP_BOUND) ? lucas_strong_fp(n) : lucas_strong(n, mont_init(n));
}

// Strong probable prime to base 2: 2^d by squarings with a doubling (an
// addition) for every set bit of d below the top one, chosen by select so the
// lanes of a warp stay converged.
__device__ __forceinline__ bool sprp2(u64 n, const Mont &M, u64 d, int t)
{
    const u64 mone = n - M.one;
    u64 x = madd(M.one, M.one, n);                         // 2 in Montgomery form
    for (int bit = 62 - __clzll(d); bit >= 0; --bit) {
        x = mmul(x, x, n, M.q);
        const u64 x2 = madd(x, x, n);
        x = ((d >> bit) & 1) ? x2 : x;
    }
    if (x == M.one || x == mone) return true;
    for (int i = 1; i < t; ++i) {
        x = mmul(x, x, n, M.q);
        if (x == mone) return true;
    }
    return false;
}

// Deterministic primality of a sieve survivor below 2^64 (Baillie-PSW): a
// strong probable prime to base 2 that also passes the strong Lucas test with
// Selfridge's parameters.  No composite below 2^64 passes both: J. Feitsma and
// W. Galway enumerated every base-2 Fermat pseudoprime below 2^64 (published
// 2009-2010, about 118.9 million numbers), and J. Gilchrist checked that none of
// them is a strong Lucas probable prime with these parameters, i.e. there is no
// Baillie-PSW pseudoprime below 2^64 (reported 2009, on Feitsma's list; it is
// the verification that makes BPSW a deterministic test in that range).  About
// 3.5 Miller-Rabin rounds of work per prime instead of the seven bases of
// is_prime_mr, which remains the answer when no Lucas parameter is found.
__device__ bool is_prime_bpsw(u64 n)
{
    if (n < MR_BOUND) return true;        // sieve survivor below 65537^2
    if (n == ~0ull) return false;         // 2^64 - 1 = 3 * 5 * 17 * 257 * 641 * 65537 * 6700417
    const Mont M = mont_init(n);
    const u64 nm1 = n - 1;
    const int t = __ffsll((long long)nm1) - 1;
    if (!sprp2(n, M, nm1 >> t, t)) return false;
    const int l = lucas_strong(n, M);
    return (l >= 0) ? (l == 1) : is_prime_mr(n);
}

// Appends v of the lanes with keep set to list[*ctr ...] with one atomic per
// warp (ballot compaction); flags err and drops the warp's values when the
// list is full.  All 32 lanes call it.
__device__ __forceinline__ void warp_push(bool keep, u64 v, u64 *__restrict__ list, u32 cap, u32 *ctr, u32 *err,
                                          u32 flag)
{
    const u32 lane = threadIdx.x & 31;
    const u32 mask = __ballot_sync(0xFFFFFFFFu, keep);
    if (!mask) return;
    u32 basepos = 0;
    if (lane == 0) basepos = atomicAdd(ctr, __popc(mask));
    basepos = __shfl_sync(0xFFFFFFFFu, basepos, 0);
    if (basepos + __popc(mask) > cap) {
        if (lane == 0) atomicOr(err, flag);
        return;
    }
    if (keep) list[basepos + __popc(mask & ((1u << lane) - 1))] = v;
}

// Warp-stride Baillie-PSW over cands[0, min(*cand_ctr, cand_cap)) with ballot compaction into primes.
__device__ __forceinline__ void mr_list(const u64 *__restrict__ cands, const u32 *cand_ctr, u32 cand_cap,
                                        u64 *__restrict__ primes, u32 prime_cap, u32 *prime_ctr, u32 *err)
{
    const u32 n = min(*cand_ctr, cand_cap);
    const u32 lane = threadIdx.x & 31;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 b0 = warp * 32; b0 < n; b0 += nwarps * 32) {
        const u32 idx = b0 + lane;
        u64 v = 0;
        bool pr = false;
        if (idx < n) {
            v = cands[idx];
            pr = is_prime_bpsw(v);
        }
        warp_push(pr, v, primes, prime_cap, prime_ctr, err, ERR_PRIME_OVERFLOW);
    }
}

__global__ void __launch_bounds__(256) k_mr(const u64 *__restrict__ cands, const u32 *__restrict__ ctrs,
                                            u32 cand_cap, u64 *__restrict__ primes, u32 prime_cap, u32 *prime_ctr,
                                            u32 *err)
{
    mr_list(cands, ctrs, cand_cap, primes, prime_cap, prime_ctr, err);
}

// The same test in two passes, so that the Lucas ladder runs on full warps.
// About 57% of the survivors of a sieve by the primes below 2^16 are prime at
// p near 2^50 (Mertens: 1/ln p over e^-gamma/ln 2^16), and the base-2 test
// rejects almost every composite; in one pass a warp runs the Lucas ladder
// (four products per bit, against about one for the base-2 test) as soon as
// one lane passed base 2, so 40% of its lanes idle through it.  Pass 1 sends
// survivors below 65537^2 (proven by the sieve) to primes and base-2 strong
// probable primes to mid; pass 2 runs the Lucas test over mid.
__global__ void __launch_bounds__(256) k_mr_sprp(const u64 *__restrict__ cands, const u32 *__restrict__ ctrs,
                                                 u32 cand_cap, u64 *__restrict__ primes, u32 prime_cap,
                                                 u32 *prime_ctr, u64 *__restrict__ mid, u32 *mid_ctr, u32 *err)
{
    const u32 n = min(ctrs[0], cand_cap);
    const u32 lane = threadIdx.x & 31;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 b0 = warp * 32; b0 < n; b0 += nwarps * 32) {
        const u32 idx = b0 + lane;
        u64 v = 0;
        bool small = false, pass = false;
        if (idx < n) {
            v = cands[idx];
            if (v < MR_BOUND) {
                small = true;
            } else if (v != ~0ull) {       // 2^64 - 1 = 3 * 5 * 17 * 257 * 641 * 65537 * 6700417
                const Mont M = mont_init(v);
                const int t = __ffsll((long long)(v - 1)) - 1;
                pass = sprp2(v, M, (v - 1) >> t, t);
            }
        }
        warp_push(small, v, primes, prime_cap, prime_ctr, err, ERR_PRIME_OVERFLOW);
        warp_push(pass, v, mid, cand_cap, mid_ctr, err, ERR_CAND_OVERFLOW);
    }
}

__global__ void __launch_bounds__(256) k_mr_lucas(const u64 *__restrict__ mid, const u32 *__restrict__ mid_ctr,
                                                  u32 mid_cap, u64 *__restrict__ primes, u32 prime_cap,
                                                  u32 *prime_ctr, u32 *err)
{
    const u32 n = min(*mid_ctr, mid_cap);
    const u32 lane = threadIdx.x & 31;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 b0 = warp * 32; b0 < n; b0 += nwarps * 32) {
        const u32 idx = b0 + lane;
        u64 v = 0;
        bool pr = false;
        if (idx < n) {
            v = mid[idx];
            const int l = lucas_test(v);
            pr = (l >= 0) ? (l == 1) : is_prime_mr(v);
        }
        warp_push(pr, v, primes, prime_cap, prime_ctr, err, ERR_PRIME_OVERFLOW);
    }
}

// Batch round in two passes, as k_mr_sprp/k_mr_lucas: pass 1 over the
// survivors of every range (one index space, prefix_c) sends the base-2 strong
// probable primes, with their range, to one mid list; pass 2 runs the Lucas
// test over it.  Survivors below 65537^2 go straight to their range's slots.
__global__ void __launch_bounds__(256) k_mr_batch_sprp(const u64 *__restrict__ cands, u32 ccap,
                                                       u64 *__restrict__ primes, u32 rcap, u32 *ctrs,
                                                       const u32 *__restrict__ prefix_c, u32 nr,
                                                       u64 *__restrict__ mid, u32 *__restrict__ mid_r, u32 mid_cap,
                                                       u32 *mid_ctr, u32 *err)
{
    const u32 total = prefix_c[nr];
    const u32 lane = threadIdx.x & 31;
    const u32 warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u32 nwarps = (gridDim.x * blockDim.x) >> 5;
    for (u32 b0 = warp * 32; b0 < total; b0 += nwarps * 32) {
        const u32 i = b0 + lane;
        u64 v = 0;
        u32 r = 0;
        bool pass = false;
        if (i < total) {
            r = prefix_find(prefix_c, nr, i);
            v = cands[(size_t)r * ccap + (i - prefix_c[r])];
            if (v < MR_BOUND) {
                const u32 pos = atomicAdd(&ctrs[r * BR_CTRS + 1], 1u);
                if (pos < rcap) primes[(size_t)r * rcap + pos] = v;
                else atomicOr(err, ERR_PRIME_OVERFLOW);
            } else if (v != ~0ull) {
                const Mont M = mont_init(v);
                const int t = __ffsll((long long)(v - 1)) - 1;
                pass = sprp2(v, M, (v - 1) >> t, t);
            }
        }
        const u32 mask = __ballot_sync(0xFFFFFFFFu, pass);
        if (!mask) continue;
        u32 basepos = 0;
        if (lane == 0) basepos = atomicAdd(mid_ctr, __popc(mask));
        basepos = __shfl_sync(0xFFFFFFFFu, basepos, 0);
        if (basepos + __popc(mask) > mid_cap) {
            if (lane == 0) atomicOr(err, ERR_CAND_OVERFLOW);
            continue;
        }
        if (pass) {
            const u32 pos = basepos + __popc(mask & ((1u << lane) - 1));
            mid[pos] = v;
            mid_r[pos] = r;
        }
    }
}

__global__ void __launch_bounds__(256) k_mr_batch_lucas(const u64 *__restrict__ mid, const u32 *__restrict__ mid_r,
                                                        u32 mid_cap, const u32 *__restrict__ mid_ctr,
                                                        u64 *__restrict__ primes, u32 rcap, u32 *ctrs, u32 *err)
{
    const u32 n = min(*mid_ctr, mid_cap);
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const u64 v = mid[i];
        const int l = lucas_test(v);
        if (!((l >= 0) ? (l == 1) : is_prime_mr(v))) continue;
        const u32 r = mid_r[i];
        const u32 pos = atomicAdd(&ctrs[r * BR_CTRS + 1], 1u);
        if (pos < rcap) primes[(size_t)r * rcap + pos] = v;
        else atomicOr(err, ERR_PRIME_OVERFLOW);
    }
}

// Next window of every range, sized for win[r] primes (width win*ln p, at
// most 0.6*rcap primes: the slot's capacity with a wide margin) and clamped to
// the range's end (a range lies entirely on one side of 2^63).  Also clears
// the range's counters.
__global__ void k_batch_windows(BatchRange *ranges, BatchWin *wins, const u32 *win, u32 nranges, u32 rcap, u32 *ctrs)
{
    const u32 r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    BatchRange R = ranges[r];
    BatchWin w;
    w.lo = R.p_cur;
    w.hi = R.p_cur;
    const double target = min((double)win[r], 0.6 * (double)rcap);
    if (R.active && R.p_cur < R.p_end && target > 0) {
        const double lnp = log((double)(R.p_cur < 3 ? 3 : R.p_cur));
        u64 width = (u64)(target * lnp);
        if (width < 4096) width = 4096;
        w.hi = (R.p_end - R.p_cur > width) ? R.p_cur + width : R.p_end;
    }
    u64 lo = w.lo < 3 ? 3 : w.lo;
    w.base_odd = lo | 1ull;
    w.nodd = (w.hi > w.base_odd) ? (w.hi - w.base_odd + 1) / 2 : 0;
    wins[r] = w;
    ranges[r].p_cur = w.hi;
    for (int i = 0; i < BR_CTRS; ++i) ctrs[r * BR_CTRS + i] = 0;
}

cudaError_t launch_sieve(u64 base_odd, u64 nodd, u64 hi, const u32 *sp, u32 nsp, u64 *cands, u32 cand_cap, u32 *ctrs,
                         u32 *err, cudaStream_t st)
{
    (void)hi;
    if (nodd == 0) return cudaSuccess;
    constexpr u64 BITS = (u64)SIEVE_WORDS * 32;
    u64 blocks = (nodd + BITS - 1) / BITS;
    k_sieve<<<(unsigned)blocks, SIEVE_TPB, 0, st>>>(base_odd, nodd, sp, nsp, cands, cand_cap, ctrs, err);
    return cudaGetLastError();
}

cudaError_t launch_batch_windows(BatchRange *ranges, BatchWin *wins, const u32 *win, u32 nranges, u32 rcap, u32 *ctrs,
                                 cudaStream_t st)
{
    k_batch_windows<<<(nranges + 127) / 128, 128, 0, st>>>(ranges, wins, win, nranges, rcap, ctrs);
    return cudaGetLastError();
}

cudaError_t launch_sieve_batch(const BatchWin *wins, u32 nranges, u32 max_blocks, const u32 *sp, u32 nsp, u64 *cands,
                               u32 ccap, u32 *ctrs, u32 *err, cudaStream_t st)
{
    k_sieve_batch<<<dim3(max_blocks, nranges), SIEVE_TPB, 0, st>>>(wins, sp, nsp, cands, ccap, ctrs, err);
    return cudaGetLastError();
}

cudaError_t launch_mr_batch2(const u64 *cands, u32 ccap, u64 *primes, u32 rcap, u32 *ctrs, u32 nranges,
                             const u32 *prefix_c, u64 *mid, u32 *mid_r, u32 mid_cap, u32 *mid_ctr, u32 *err, int sms,
                             cudaStream_t st)
{
    k_mr_batch_sprp<<<sms * 8, 256, 0, st>>>(cands, ccap, primes, rcap, ctrs, prefix_c, nranges, mid, mid_r, mid_cap,
                                              mid_ctr, err);
    k_mr_batch_lucas<<<sms * 8, 256, 0, st>>>(mid, mid_r, mid_cap, mid_ctr, primes, rcap, ctrs, err);
    return cudaGetLastError();
}

cudaError_t launch_mr(const u64 *cands, const u32 *ctrs, u32 cand_cap, u64 *primes, u32 prime_cap, u32 *prime_ctr,
                      u32 *err, int sms, cudaStream_t st)
{
    k_mr<<<sms * 8, 256, 0, st>>>(cands, ctrs, cand_cap, primes, prime_cap, prime_ctr, err);
    return cudaGetLastError();
}

cudaError_t launch_mr2(const u64 *cands, const u32 *ctrs, u32 cand_cap, u64 *primes, u32 prime_cap, u32 *prime_ctr,
                       u64 *mid, u32 *mid_ctr, u32 *err, int sms, cudaStream_t st)
{
    k_mr_sprp<<<sms * 8, 256, 0, st>>>(cands, ctrs, cand_cap, primes, prime_cap, prime_ctr, mid, mid_ctr, err);
    k_mr_lucas<<<sms * 8, 256, 0, st>>>(mid, mid_ctr, cand_cap, primes, prime_cap, prime_ctr, err);
    return cudaGetLastError();
}

}  // namespace rs

// setup.cu -- per-prime set-up for the BSGS search.
//
// Replaces the reference's setup and sort kernels (kernels/setup.cl:89-209,
// kernels/sort.cl:11-104).  The arithmetic is re-derived rather than ported.
//
// Term k*b^n + c (c = +-1) is divisible by p iff k*b^n == -c (mod p).  Write
// n = nmin + off + e*u with a split modulus e (one table of powers of s = b^e
// serves every sequence) and u = (q+1)*Q - 1 - j with baby index j in [0,Q)
// and giant index q.  Then
//      s^j == T * S^q,   T = -c * k * b^(nmin + off + e*(Q-1)),   S = s^Q,
// so the baby table holds s^j and no modular inverse is needed (the reference
// batch-inverts every k and b^Q, setup.cl:133-166).
//
// Residue classes of n.  The reference splits n by parity when b is a
// quadratic non-residue mod p (e = 2) and filters with d-th power residues
// (setup.cl:22-87).  Here both come from one character of larger order.  Let D
// be the part of p-1 made of the primes up to 61, and chi(x) = x^((p-1)/D),
// which maps onto the D-th roots of unity.  If k*b^n == -c then
//      chi(b)^n = chi(-c) / chi(k),
// so (1) a target is impossible unless chi(-c)/chi(k) lies in the subgroup
// generated by chi(b), of order eo (the reference's filters are the cases
// d | D of this), and (2) n mod e is fixed, for every divisor e of eo, by the
// discrete logarithm of h = chi(b)^(eo/e) -- a table of e values.  e is the
// largest divisor of eo up to 64.  Every n the reference finds satisfies both,
// so the eliminated terms are the same, while each sequence's giant steps
// shrink from L/Q to L/(e*Q) (e = 2 is the reference's parity case; at the
// 2^50 p-range of the 100-sequence job e averages well above 2).
// Primes dividing b or any k, and primes where no k survives, are skipped for
// every sequence as setup.cl:156-162,205-208 do.
//
// Kernel 1 (one thread per prime) does the per-prime scalars; kernel 2 (one
// warp per prime, lanes over k) classifies the sequences, chooses the prime's
// baby-step count Q' (the launch's Q, Q/2 or Q/4: fewer baby steps when the
// split modulus leaves few giant steps) and writes the compacted targets;
// kernel 3 (one thread per prime) writes the giant-step split and the baby-
// and giant-step start tables.  Per-prime work that is the same for every
// sequence runs one prime per thread, where it costs 1/32 of the issue slots
// it would take in the warp-per-prime kernel.
#include "mont.cuh"
#include "rs_internal.h"

namespace rs {

constexpr u32 SPLIT_MAX = 64;        // largest split modulus e (6 bits of offset per target)

// mpow out of line, for the per-prime powers off the kernels' main path: one
// copy of the loop keeps the kernels small enough for the instruction cache.
__device__ __noinline__ u64 mpow_call(u64 x, u64 e, Mont M) { return mpow(x, e, M); }

constexpr int NCP = 3;            // baby steps per thread: C, C/2 or C/4 (index k: C >> k)

struct PrimeAux {        // kernel 1 -> kernel 2 scalars
    u64 r2;              // R^2 mod p
    u64 bm;              // Montgomery b
    u64 xD;              // (p-1)/D: chi(x) = x^xD
    u64 xe;              // eo/e
    u64 hm1;             // Montgomery h^-1, h = chi(b)^xe of order e
    u64 wr0[NCP];        // per baby-step count Q'_k = tpb*(C >> k): b^(nmin + e(Q'_k - 1)) * R^2 (mod p)
    u64 S[NCP];          //   and Montgomery s^Q'_k
    u32 e;               // split modulus
    u32 flags;           // AUX_* below
};
constexpr u32 AUX_NEG_EO = 1u;   // chi(-1)^eo = -1: for c = +1 the membership test wants z^eo == -1
constexpr u32 AUX_NEG_XE = 2u;   // chi(-1)^xe = -1: for c = +1 the class search wants z1*h^r == -1

// Moves every factor L of x into D (L a compile-time prime): applied for each
// prime up to 61, it leaves D = the 61-smooth part of p-1 and x = (p-1)/D.
template <u32 L>
__device__ __forceinline__ void strip(u64 &x, u64 &D)
{
    while (x % L == 0) { x /= L; D *= L; }
}

// Order of g in the group of D-th roots of unity (D 61-smooth): remove the
// prime factor L from eo while g^(eo/L) is still 1.
template <u32 L>
__device__ __forceinline__ void order_step(u64 &eo, u64 g, const Mont &M)
{
    while (eo % L == 0 && mpow_call(g, eo / L, M) == M.one) eo /= L;
}

// x^e mod p on the FP64 pipe (p < FP_BOUND), plain residues held exactly in
// doubles, pinv = 1/p; e may be 0.  Out of line like mpow_call.
__device__ __noinline__ double fpow_call(double x, u64 e, double p, double pinv)
{
    if (e == 0) return 1.0;
    double a = x;
    for (int bit = 62 - __clzll(e); bit >= 0; --bit) {
        a = fp_mul(a, a, p, pinv);
        if ((e >> bit) & 1) a = fp_mul(a, x, p, pinv);
    }
    return a;
}

// order_step for a plain g below FP_BOUND, by FP64 powers.
template <u32 L>
__device__ __forceinline__ void order_step_fp(u64 &eo, double g, double p, double pinv)
{
    while (eo % L == 0 && fpow_call(g, eo / L, p, pinv) == 1.0) eo /= L;
}

// Largest divisor of eo that is at most SPLIT_MAX (by 32-bit remainders when
// eo fits in 32 bits, the usual case, and from the largest candidate down).
__device__ __forceinline__ u32 split_modulus(u64 eo)
{
    if (eo >> 32) {
        for (u32 d = SPLIT_MAX; d > 1; --d)
            if (eo % d == 0) return d;
        return 1;
    }
    const u32 e32 = (u32)eo;
#pragma unroll
    for (u32 d = SPLIT_MAX; d > 1; --d)
        if (e32 % d == 0) return d;
    return 1;
}

// b^e as an integer when it is at most 16 (baby steps by additions), else 0.
__device__ __forceinline__ u32 small_power(u32 b, u32 e)
{
    u64 v = 1;
    for (u32 i = 0; i < e; ++i) {
        v *= b;
        if (v > 16) return 0;
    }
    return (u32)v;
}

// Per-prime constants of prime p into record t, with the powers that depend
// on the baby-step count for each of the counts kernel 2 chooses from.
__device__ __forceinline__ void setup_prime_one(const JobDev *__restrict__ job, u64 p, u32 t, u32 jb,
                                                PrimeHdr *__restrict__ hdr, PrimeAux *__restrict__ aux,
                                                const JobGeom &gm)
{
    PrimeHdr H;
    H.p = 0; H.q = 0; H.one = 0; H.s = 0; H.S = 0; H.numk = 0; H.e = 0; H.G = 0; H.Lc = 0; H.smul = 0; H.job = jb;
    H.Mg = 0; H.cp = 0; H.Sh = 0; H.Sw = 0; H.ssw = 0; H.sp = 0; H.Sp = 0; H.u2 = 0; H.Sq = 0;
    const Mont M = mont_init(p);
    const u32 b = job->base;
    const u64 bm = to_mont(b, M);
    if (bm == 0) { hdr[t] = H; return; }                 // p | b: no term is divisible by p
    // D = 61-smooth part of p-1, xD = (p-1)/D
    u64 xD = p - 1, D = 1;
    strip<2>(xD, D);  strip<3>(xD, D);  strip<5>(xD, D);  strip<7>(xD, D);  strip<11>(xD, D);
    strip<13>(xD, D); strip<17>(xD, D); strip<19>(xD, D); strip<23>(xD, D); strip<29>(xD, D);
    strip<31>(xD, D); strip<37>(xD, D); strip<41>(xD, D); strip<43>(xD, D); strip<47>(xD, D);
    strip<53>(xD, D); strip<59>(xD, D); strip<61>(xD, D);
    u64 gb, eo = D;                                       // chi(b), of order eo | D
    if (p < FP_BOUND) {                                   // the power and the order on the FP64 pipe
        const double pd = fp_exact(p), pinv = 1.0 / pd;
        const double g = fpow_call(fp_exact(b % p), xD, pd, pinv);
        order_step_fp<2>(eo, g, pd, pinv);  order_step_fp<3>(eo, g, pd, pinv);  order_step_fp<5>(eo, g, pd, pinv);
        order_step_fp<7>(eo, g, pd, pinv);  order_step_fp<11>(eo, g, pd, pinv); order_step_fp<13>(eo, g, pd, pinv);
        order_step_fp<17>(eo, g, pd, pinv); order_step_fp<19>(eo, g, pd, pinv); order_step_fp<23>(eo, g, pd, pinv);
        order_step_fp<29>(eo, g, pd, pinv); order_step_fp<31>(eo, g, pd, pinv); order_step_fp<37>(eo, g, pd, pinv);
        order_step_fp<41>(eo, g, pd, pinv); order_step_fp<43>(eo, g, pd, pinv); order_step_fp<47>(eo, g, pd, pinv);
        order_step_fp<53>(eo, g, pd, pinv); order_step_fp<59>(eo, g, pd, pinv); order_step_fp<61>(eo, g, pd, pinv);
        gb = to_mont(fp_int(g), M);
    } else {
        gb = mpow(bm, xD, M);
        order_step<2>(eo, gb, M);  order_step<3>(eo, gb, M);  order_step<5>(eo, gb, M);  order_step<7>(eo, gb, M);
        order_step<11>(eo, gb, M); order_step<13>(eo, gb, M); order_step<17>(eo, gb, M); order_step<19>(eo, gb, M);
        order_step<23>(eo, gb, M); order_step<29>(eo, gb, M); order_step<31>(eo, gb, M); order_step<37>(eo, gb, M);
        order_step<41>(eo, gb, M); order_step<43>(eo, gb, M); order_step<47>(eo, gb, M); order_step<53>(eo, gb, M);
        order_step<59>(eo, gb, M); order_step<61>(eo, gb, M);
    }
    const u32 e = split_modulus(eo);
    const u64 xe = eo / e;
    const u64 s = mpow_call(bm, e, M);
    PrimeAux X;
    X.r2 = M.r2;
    X.bm = bm;
    X.xD = xD;
    X.xe = xe;
    X.hm1 = mpow_call(mpow_call(gb, xe, M), (u64)(e - 1), M);
    X.e = e;
    const bool chi_m1 = (xD & 1) != 0;                    // chi(-1) = (-1)^xD
    X.flags = ((chi_m1 && (eo & 1)) ? AUX_NEG_EO : 0u) | ((chi_m1 && (xe & 1)) ? AUX_NEG_XE : 0u);
    // Q'_k = 2^(m+2-k), m = log2(Q/4): s^(Q'-1) by t <- t^2 * s from s^(2^m - 1).
    // Below FP_BOUND the powers are FP64 products of plain residues, moved
    // into Montgomery form (and R^2 form for wr0) at the end.
    const int m = __ffs((int)(gm.q >> 2)) - 1;
    if (p < FP_BOUND) {
        const double pd = fp_exact(p), pinv = 1.0 / pd;
        const double sd = fp_exact(from_mont(s, M));
        const double bn = fpow_call(fp_exact(b % p), (u64)job->nmin, pd, pinv);
        double tq = 1.0;
        for (int i = 0; i < m; ++i) tq = fp_mul(fp_mul(tq, tq, pd, pinv), sd, pd, pinv);
#pragma unroll
        for (int k = NCP - 1; k >= 0; --k) {              // k = NCP-1: Q/4, then Q/2, Q
            if (k != NCP - 1) tq = fp_mul(fp_mul(tq, tq, pd, pinv), sd, pd, pinv);
            X.wr0[k] = mmul(to_mont(fp_int(fp_mul(bn, tq, pd, pinv)), M), M.r2, p, M.q);
            X.S[k] = to_mont(fp_int(fp_mul(tq, sd, pd, pinv)), M);
        }
    } else {
        const u64 bn = mpow_call(bm, (u64)job->nmin, M);
        u64 tq = M.one;
        for (int i = 0; i < m; ++i) tq = mmul(mmul(tq, tq, p, M.q), s, p, M.q);
#pragma unroll
        for (int k = NCP - 1; k >= 0; --k) {              // k = NCP-1: Q/4, then Q/2, Q
            if (k != NCP - 1) tq = mmul(mmul(tq, tq, p, M.q), s, p, M.q);
            X.wr0[k] = mmul(mmul(bn, tq, p, M.q), M.r2, p, M.q);
            X.S[k] = mmul(tq, s, p, M.q);
        }
    }
    H.p = p; H.q = M.q; H.one = M.one; H.s = s; H.e = e;
    if (!(p >> 63)) {                                     // Shoup multiplier of the baby steps below 2^63
        H.sp = from_mont(s, M);
        H.ssw = shoup_of_mont(s, M.q);
    }
    H.smul = small_power(b, e);
    hdr[t] = H;
    aux[t] = X;
}


// Kernel 1.  Single job: primes[first, first+count) into records [0, count).
// Batch (BATCH): the primes of every range as one index space (prefix: prefix
// sums of the ranges' prime counts); prime i of range r is record r*rcap + i,
// with its job's sequences.  rec_of[i] keeps that record index, so kernels 2
// and 3 need no search over the prefix sums.
template <bool BATCH>
__global__ void __launch_bounds__(256) k_setup_prime(const JobDev *__restrict__ jobs, const u64 *__restrict__ primes,
                                                     u32 first, u32 count, PrimeHdr *__restrict__ hdr,
                                                     PrimeAux *__restrict__ aux, JobGeom gm,
                                                     const JobGeom *__restrict__ geoms,
                                                     const BatchRange *__restrict__ ranges,
                                                     const u32 *__restrict__ prefix, u32 nr, u32 rcap,
                                                     u32 *__restrict__ rec_of)
{
    const u32 stride = gridDim.x * blockDim.x;
    if constexpr (BATCH) {
        const u32 total = prefix[nr];
        for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
            const u32 r = prefix_find(prefix, nr, i);
            const u32 rec = r * rcap + (i - prefix[r]);
            const u32 jb = ranges[r].job;
            rec_of[i] = rec;
            setup_prime_one(jobs + jb, primes[rec], rec, jb, hdr, aux, geoms[jb]);
        }
    } else {
        for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
            setup_prime_one(jobs, primes[first + t], t, 0, hdr, aux, gm);
    }
}

// Baby steps per thread for a prime with nk targets of Le giant-step units
// each: the index k of the per-thread count C >> k in {C, C/2, C/4} (Q' =
// tpb*(C >> k) baby steps) that minimises Q' + GIANT_COST * (nk * ceil(Le/Q')
// giant steps + 2 start products per giant thread).  A prime with a large
// split modulus has few giant steps per target and takes fewer baby steps.
// tpb and C are powers of two, so every division is a shift.
constexpr float GIANT_COST = 0.8f;
__device__ __forceinline__ u32 choose_cp(const JobGeom &gm, u32 nk, u64 Le)
{
    u32 best_k = 0;
    float best = 3.0e38f;
    const int lq = 31 - __clz(gm.tpb * gm.c);
    const u32 g0 = gm.tpb / nk;
    for (u32 k = 0; k < NCP; ++k) {
        const u64 qp = 1ull << (lq - k);
        const u64 mg = (Le + qp - 1) >> (lq - k);
        u64 g = g0 < 1 ? 1 : g0;
        if (g > mg) g = mg;
        const float cost = (float)qp + GIANT_COST * ((float)nk * (float)mg + 2.0f * (float)(nk * g));
        if (cost < best) { best = cost; best_k = k; }
    }
    return best_k;
}

// a[r] = x[r]^ex for r < R, the R chains interleaved (the exponent is the same
// for every lane and chain, so the loop is uniform over the warp); ex >= 1.
// LAZY (p < 2^62): the chains stay in [0, 2p) without per-product corrections.
template <int R, bool LAZY>
__device__ __forceinline__ void mpow_multi(u64 (&a)[4], const u64 (&x)[4], u64 ex, const Mont &M)
{
    auto mul = [&](u64 u, u64 v) { return LAZY ? mmul_lazy(u, v, M.p, M.q) : mmul(u, v, M.p, M.q); };
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = x[r];
    for (int bit = 62 - __clzll(ex); bit >= 0; --bit) {
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = LAZY ? msqr_lazy(a[r], M.p, M.q) : mmul(a[r], a[r], M.p, M.q);
        if ((ex >> bit) & 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) a[r] = mul(a[r], x[r]);
        }
    }
    if (LAZY) {
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = mred(a[r], M.p);
    }
}

template <bool LAZY>
__device__ __forceinline__ void mpow_lanes(u32 R, u64 (&a)[4], const u64 (&x)[4], u64 ex, const Mont &M)
{
    if (R == 1) mpow_multi<1, LAZY>(a, x, ex, M);
    else if (R == 2) mpow_multi<2, LAZY>(a, x, ex, M);
    else if (R == 3) mpow_multi<3, LAZY>(a, x, ex, M);
    else mpow_multi<4, LAZY>(a, x, ex, M);
}

// The chains of mpow_multi on the FP64 pipe (p < FP_BOUND): plain residues
// held exactly in doubles, products by fp_mul_signed, so the chains run in
// signed residues in (-p, p) and are made canonical once at the end.
template <int R>
__device__ __forceinline__ void fpow_multi(double (&a)[4], const double (&x)[4], u64 ex, double pd, double pinv)
{
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = x[r];
    for (int bit = 62 - __clzll(ex); bit >= 0; --bit) {
#pragma unroll
        for (int r = 0; r < R; ++r) a[r] = fp_mul_signed(a[r], a[r], pd, pinv);
        if ((ex >> bit) & 1) {
#pragma unroll
            for (int r = 0; r < R; ++r) a[r] = fp_mul_signed(a[r], x[r], pd, pinv);
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = (a[r] < 0.0) ? a[r] + pd : a[r];
}

// z = chi(k_i) = k_i^xD in Montgomery form for the lane's sequences
// i = lane + 32r < K, into zs[i].  (Out of line, with the caller's state
// saved once per prime instead of spilled, it measured 3-6% slower.)
// Below FP_BOUND the chains run on the FP64 pipe two at a time (four
// interleaved chains would not fit the kernel's 64 registers), as a rolled
// loop over pairs of rounds so that one copy of the chain code serves them.
__device__ __forceinline__ void chi_of_ks(const JobDev *__restrict__ job, u32 lane, u32 K, const Mont M, u64 xD,
                                          u64 *zs)
{
    const u64 p = M.p;
    const u32 R = (K + 31) / 32;
    if (p < FP_BOUND) {
        const double pd = fp_exact(p), pinv = 1.0 / pd;
#pragma unroll 1
        for (u32 r0 = 0; r0 < R; r0 += 2) {
            double x[4], zd[4];
#pragma unroll
            for (u32 h = 0; h < 2; ++h) {
                const u32 i = lane + 32 * (r0 + h);
                const u64 kv = (i < K) ? job->k[i] : 1;
                x[h] = fp_exact((kv < p) ? kv : kv % p);
            }
            if (r0 + 1 < R) fpow_multi<2>(zd, x, xD, pd, pinv);
            else fpow_multi<1>(zd, x, xD, pd, pinv);
#pragma unroll
            for (u32 h = 0; h < 2; ++h)
                if (r0 + h < R) zs[lane + 32 * (r0 + h)] = to_mont(fp_int(zd[h]), M);
        }
    } else {
        u64 x[4], z[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const u32 i = lane + 32 * r;
            const u64 kv = (i < K) ? job->k[i] : 1;
            x[r] = to_mont((kv < p) ? kv : kv % p, M);
        }
        if (p >> 62) mpow_lanes<false>(R, z, x, xD, M);
        else mpow_lanes<true>(R, z, x, xD, M);
#pragma unroll
        for (u32 r = 0; r < 4; ++r)
            if (r < R) zs[lane + 32 * r] = z[r];
    }
}

// Class lookup: the e values h^(-r) (r < e <= SPLIT_MAX, all distinct and
// nonzero) in an open-addressed table of CLS_SLOTS 64-bit keys with their r
// beside them, so a sequence's class costs one or two probes instead of a
// walk over up to e entries (e averages about 28 at 2^50).
constexpr u32 CLS_SLOTS = 2 * SPLIT_MAX;
static_assert((CLS_SLOTS & (CLS_SLOTS - 1)) == 0, "slot index wraps by a mask");

__device__ __forceinline__ u32 cls_hash(u64 v) { return (((u32)v ^ (u32)(v >> 32)) * 0x9E3779B1u) >> 25; }
static_assert(CLS_SLOTS == 128, "cls_hash yields 7 bits");

// Inserts key v (nonzero, not yet present) with index r; lanes insert
// concurrently, a slot going to the lane whose compare-and-swap finds it empty.
// At most SPLIT_MAX keys share CLS_SLOTS slots, so the walk always ends.
__device__ __forceinline__ void cls_insert(u64 *ck, unsigned char *cr, u64 v, u32 r)
{
    u32 s = cls_hash(v);
    for (u32 n = 0; n < CLS_SLOTS; ++n) {
        if (atomicCAS(reinterpret_cast<unsigned long long *>(&ck[s]), 0ull, (unsigned long long)v) == 0ull) {
            cr[s] = (unsigned char)r;
            return;
        }
        s = (s + 1) & (CLS_SLOTS - 1);
    }
}

// r with ck[.] == v, or none when v is absent (an empty slot ends the walk).
__device__ __forceinline__ u32 cls_find(const u64 *ck, const unsigned char *cr, u64 v, u32 none)
{
    u32 s = cls_hash(v);
    for (u32 n = 0; n < CLS_SLOTS; ++n) {
        const u64 k = ck[s];
        if (k == v) return cr[s];
        if (k == 0) break;
        s = (s + 1) & (CLS_SLOTS - 1);
    }
    return none;
}

// Sequence classes, targets, baby-step count and the start tables of record w
// (one warp).  tw: this warp's table of SPLIT_MAX powers of b, the CLS_SLOTS
// keys of its class lookup and chi(k) of up to 128 sequences; cr: the
// lookup's indices.
__device__ __forceinline__ void setup_k_one(const JobDev *__restrict__ job, u32 w, u32 lane, PrimeHdr *__restrict__ hdr,
                                            const PrimeAux *__restrict__ aux, u64 *__restrict__ tabs,
                                            u64 *__restrict__ tgt, unsigned short *__restrict__ meta,
                                            u64 *__restrict__ stats, u32 *__restrict__ err, const JobGeom &gm,
                                            u64 *tw, unsigned char *cr)
{
    PrimeHdr H = hdr[w];
    if (H.p == 0) {
        if (lane == 0) atomicAdd(&stats[ST_SKIPPED], 1ull);
        return;
    }
    const PrimeAux &X = aux[w];
    Mont M;
    M.p = H.p; M.q = H.q; M.one = H.one; M.r2 = X.r2;
    const u64 p = H.p;
    const u32 K = job->kcount;
    const u32 e = X.e;
    const u64 mone = p - M.one;
    u64 *tg = tgt + (size_t)w * KSTRIDE;
    unsigned short *mg_ = meta + (size_t)w * KSTRIDE;
    // the class lookup gets h^(-r) and, for now, wt[r] = b^r, for r < e: lane
    // l forms h^(-l) and b^l by a multiplicative scan over the warp (five
    // products each); entries 32..63 take one more product by h^(-32) and b^32
    static_assert(SPLIT_MAX <= 64, "two rounds of 32 table entries");
    u64 *wt = tw, *ck = tw + SPLIT_MAX, *zs = ck + CLS_SLOTS;
    __syncwarp();                                          // the previous prime's readers are done
#pragma unroll
    for (u32 i = 0; i < CLS_SLOTS; i += 32) ck[i + lane] = 0;
    __syncwarp();
    {
        const u64 hm1 = X.hm1, bm = X.bm;
        u64 hv = (lane == 0) ? M.one : hm1, bv = (lane == 0) ? M.one : bm;
#pragma unroll 1
        for (int o = 1; o < 32; o <<= 1) {
            const u64 hu = __shfl_up_sync(0xFFFFFFFFu, hv, o), bu = __shfl_up_sync(0xFFFFFFFFu, bv, o);
            if (lane >= (u32)o) {
                hv = mmul(hv, hu, p, M.q);
                bv = mmul(bv, bu, p, M.q);
            }
        }
        if (lane < e) {
            cls_insert(ck, cr, hv, lane);
            wt[lane] = bv;
        }
        if (e > 32) {
            const u64 h32 = mmul(__shfl_sync(0xFFFFFFFFu, hv, 31), hm1, p, M.q);
            const u64 b32 = mmul(__shfl_sync(0xFFFFFFFFu, bv, 31), bm, p, M.q);
            if (lane + 32 < e) {
                cls_insert(ck, cr, mmul(hv, h32, p, M.q), lane + 32);
                wt[lane + 32] = mmul(bv, b32, p, M.q);
            }
        }
    }
    // z = chi(k) = k^xD for the lane's sequences i = lane + 32r, r < R: one
    // exponent for the whole warp, R independent chains per lane
    const u32 R = (K + 31) / 32;
    chi_of_ks(job, lane, K, M, X.xD, zs);
    __syncwarp();
    // pass 1: the class of every sequence; the kept ones' k mod p and class
    // offset go to the record (compacted), the target itself once Q' is known.
    // The rounds read chi(k) back from shared memory, so the loop is not
    // unrolled: one copy of its code keeps the kernel's hot path short.
    const u32 nmod = job->nmin % e;
    u32 nk = 0;
    bool divk = false, lost = false;
#pragma unroll 1
    for (u32 rd = 0; rd < R; ++rd) {
        const u32 i = lane + 32 * rd;
        const u64 zr = zs[i];
        bool keep = false;
        u64 kr = 0;
        unsigned short mt = 0;
        if (i < K) {
            const u64 kv = job->k[i];
            kr = (kv < p) ? kv : kv % p;
            if (kr == 0) {
                divk = true;
            } else {
                const int ci = job->c[i];
                // the target is possible iff (chi(-c)/z)^eo == 1, i.e.
                // z1^e == chi(-c)^eo with z1 = z^xe; chi(-c) is 1 for c = -1.
                // When xe = 1 (eo = e, the usual case) that is exactly "the class
                // search below finds r", so the power is skipped.
                const u64 z1 = (X.xe == 1) ? zr : mpow_call(zr, X.xe, M);
                const u64 want = (ci == 1 && (X.flags & AUX_NEG_EO)) ? mone : M.one;
                const bool pass = (X.xe == 1) || mpow_call(z1, (u64)e, M) == want;
                if (pass) {
                    // n == r (mod e) where z1 * h^r == chi(-c)^xe, i.e.
                    // h^(-r) == z1 or, when chi(-c)^xe == -1, == p - z1
                    // (z1 is a unit, so both lie in (0, p))
                    const bool neg = (ci == 1) && (X.flags & AUX_NEG_XE);
                    const u32 r = cls_find(ck, cr, neg ? p - z1 : z1, e);
                    if (r < e) {
                        const u32 off = (r + e - nmod) % e;
                        mt = (unsigned short)(i | (off << 7));
                        keep = true;
                    } else if (X.xe != 1) {
                        lost = true;                      // cannot happen: the class exists when the test passes
                    }
                }
            }
        }
        const u32 km_ = __ballot_sync(0xFFFFFFFFu, keep);
        if (keep) {
            const u32 pos = nk + __popc(km_ & ((1u << lane) - 1));
            tg[pos] = kr;
            mg_[pos] = mt;
        }
        nk += __popc(km_);
    }
    if (lost) atomicOr(err, ERR_SETUP_CLASS);
    divk = __any_sync(0xFFFFFFFFu, divk);
    if (divk || nk == 0) {
        if (lane == 0) {
            hdr[w].p = 0;
            atomicAdd(&stats[ST_SKIPPED], 1ull);
        }
        return;
    }
    // baby steps for this prime (the giant-step tables follow in kernel 3)
    const u64 Le = ((u64)job->L + e - 1) / e;
    const u32 kc = choose_cp(gm, nk, Le);
    // targets T = -c * k * b^(nmin + off + e(Q'-1)): wt[r] = b^(nmin + e(Q'-1) + r) * R^2
    const u64 wr0 = X.wr0[kc];
    for (u32 r = lane; r < e; r += 32) wt[r] = mmul(wr0, wt[r], p, M.q);
    __syncwarp();                                          // also orders pass 1's record writes
    for (u32 j = lane; j < nk; j += 32) {
        const u32 m = mg_[j];
        u64 T = mmul(tg[j], wt[m >> 7], p, M.q);
        if (job->c[m & 0x7Fu] == 1) T = mneg(T, p);
        tg[j] = T;
    }
    if (lane == 0) {
        hdr[w].numk = nk;
        hdr[w].cp = gm.c >> kc;
    }
}

// Baby- and giant-step tables of record t (one thread): giant steps per target
// Mg = ceil(ceil(L/e)/Q'), G chunks of Lc steps per target (numk*G <= tpb),
// A[l] = s^(cp*l), B[l] = s^(32*cp*l) (baby starts), Z1[l] = S^(Lc*l),
// Z2[l] = S^(32*Lc*l) (giant starts) with S = s^Q', and the Shoup quotient of S.
// Adds the prime's targets and its search kind to the thread's tallies.
__device__ __forceinline__ void setup_tabs_one(const JobDev *__restrict__ job, u32 t, PrimeHdr *__restrict__ hdr,
                                               const PrimeAux *__restrict__ aux, u64 *__restrict__ tabs,
                                               const JobGeom &gm, u32 &n_targets, u32 &n_full, u32 &n_split)
{
    PrimeHdr H = hdr[t];
    if (H.p == 0) return;
    const u64 p = H.p, q = H.q;
    Mont M;
    M.p = p; M.q = q; M.one = H.one; M.r2 = 0;
    const u32 e = H.e, cp = H.cp, nk = H.numk;
    const u32 kc = 31 - __clz(gm.c / cp);
    const u32 qp = gm.tpb * cp;
    const u64 Le = ((u64)job->L + e - 1) / e;
    const u32 Mg = (u32)((Le + qp - 1) / qp);
    u32 G = gm.tpb / nk;
    if (G < 1) G = 1;
    if (G > Mg) G = Mg;
    const u32 Lc = (Mg + G - 1) / G;
    G = (Mg + Lc - 1) / Lc;
    const u64 S = aux[t].S[kc];
    const u64 Sh = mpow(S, (u64)(Lc >> 1), M);            // start of a thread's second giant chain
    const u64 z = (Lc & 1) ? mmul(mmul(Sh, Sh, p, q), S, p, q) : mmul(Sh, Sh, p, q);   // S^Lc
    u64 u2 = H.s;                                          // s^(cp/2) and s^cp, cp a power of two >= 2
    for (u32 c = cp >> 1; c > 1; c >>= 1) u2 = mmul(u2, u2, p, q);
    const u64 u = mmul(u2, u2, p, q);
    u64 *tb = tabs + (size_t)t * TABS;
    // four power tables, two chains at a time, each only as long as the BSGS
    // kernel reads it: A[t % 32] and B[t / 32] for its threads t < tpb, Z1[g % 32]
    // and Z2[g / 32] for the giant chunks g < G (the rest of the record's table
    // space is left as it is).  Below FP_BOUND the BSGS kernel forms its start
    // values with FP64 products of plain residues, x*y mod p instead of x*y/R:
    // there Z2, s^(cp/2) and S^(Lc/2) are stored plain, so baby and giant values
    // alike carry R^2 instead of R; and the tables' own chains run on the FP64
    // pipe with plain multipliers (an R-form start times plain powers stays in
    // R-form).  z^32 is needed only when G > 32, and then the Z1 chain has run
    // all 32 steps.
    const u32 nb = gm.tpb >> 5, nz1 = min(G, 32u), nz2 = (G + 31) >> 5;
    const bool fp = (p < FP_BOUND);
    if (fp) {
        const double pd = (double)p, pinv = 1.0 / pd;
        const double up = fp_exact(from_mont(u, M)), zp = fp_exact(from_mont(z, M));
        double a = fp_exact(M.one), b = a;
        for (u32 l = 0; l < 32; ++l) {
            tb[l] = fp_int(a);
            a = fp_mul(a, up, pd, pinv);
            if (l < nz1) {
                tb[64 + l] = fp_int(b);
                b = fp_mul(b, zp, pd, pinv);
            }
        }
        const double u32p = fp_exact(from_mont(fp_int(a), M));                  // plain u^32
        const double z32 = (nz2 > 1) ? fp_exact(from_mont(fp_int(b), M)) : 0.0;  // plain z^32
        a = fp_exact(M.one);
        b = 1.0;
        for (u32 l = 0; l < nb; ++l) {
            tb[32 + l] = fp_int(a);
            a = fp_mul(a, u32p, pd, pinv);
            if (l < nz2) {
                tb[96 + l] = fp_int(b);
                b = fp_mul(b, z32, pd, pinv);
            }
        }
    } else {
        u64 a = M.one, b = M.one;
        for (u32 l = 0; l < 32; ++l) {
            tb[l] = a;
            a = mmul(a, u, p, q);
            if (l < nz1) {
                tb[64 + l] = b;
                b = mmul(b, z, p, q);
            }
        }
        const u64 u32p = a, z32 = b;                       // u^32, and z^32 when G > 32
        a = M.one;
        b = M.one;
        for (u32 l = 0; l < nb; ++l) {
            tb[32 + l] = a;
            a = mmul(a, u32p, p, q);
            if (l < nz2) {
                tb[96 + l] = b;
                b = mmul(b, z32, p, q);
            }
        }
    }
    PrimeHdr &h = hdr[t];
    h.G = G;
    h.Lc = Lc;
    h.Mg = Mg;
    h.S = S;
    h.Sh = Sh;
    h.u2 = u2;
    if (!(p >> 63)) {                                      // Shoup multiplier of the giant steps below 2^63
        h.Sp = from_mont(S, M);
        h.Sw = shoup_of_mont(S, q);
    }
    if (fp) {                                              // FP64 quotients of the baby and giant multipliers
        const double pd = (double)p;
        h.S = (u64)__double_as_longlong((double)H.sp / pd);
        h.Sq = (u64)__double_as_longlong((double)h.Sp / pd);
        // the FP64 start values: plain s^(cp/2) and S^(Lc/2), 1/p in the Shoup
        // quotients' place and R^2 mod p (the value of s^0) in the other
        h.u2 = from_mont(u2, M);
        h.Sh = from_mont(Sh, M);
        h.Sw = (u64)__double_as_longlong(1.0 / pd);
        h.ssw = aux[t].r2;
    }
    n_targets += nk;
    if (e >= 2) ++n_split; else ++n_full;
}

// Kernel 3: one thread per prime (indexing as kernel 1).
template <bool BATCH>
__global__ void __launch_bounds__(256) k_setup_tabs(const JobDev *__restrict__ jobs, PrimeHdr *__restrict__ hdr,
                                                    const PrimeAux *__restrict__ aux, u32 count,
                                                    u64 *__restrict__ tabs, u64 *__restrict__ stats, JobGeom gm,
                                                    const JobGeom *__restrict__ geoms,
                                                    const u32 *__restrict__ prefix, u32 nr,
                                                    const u32 *__restrict__ rec_of)
{
    const u32 stride = gridDim.x * blockDim.x;
    u32 nt = 0, nf = 0, ns = 0;
    if constexpr (BATCH) {
        const u32 total = prefix[nr];
        for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
            const u32 rec = rec_of[i];
            const u32 jb = hdr[rec].job;
            setup_tabs_one(jobs + jb, rec, hdr, aux, tabs, geoms[jb], nt, nf, ns);
        }
    } else {
        for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
            setup_tabs_one(jobs, t, hdr, aux, tabs, gm, nt, nf, ns);
    }
    // one atomic per warp and counter
    nt = __reduce_add_sync(0xFFFFFFFFu, nt);
    nf = __reduce_add_sync(0xFFFFFFFFu, nf);
    ns = __reduce_add_sync(0xFFFFFFFFu, ns);
    if ((threadIdx.x & 31) == 0) {
        if (nt) atomicAdd(&stats[ST_TARGETS], (u64)nt);
        if (nf) atomicAdd(&stats[ST_FULL], (u64)nf);
        if (ns) atomicAdd(&stats[ST_PARITY], (u64)ns);
    }
}


// Kernel 2: one warp per prime; lanes walk the sequences.  BATCH as kernel 1.
template <bool BATCH>
__global__ void __launch_bounds__(SETUP_TPB, 4) k_setup_k(const JobDev *__restrict__ jobs, PrimeHdr *__restrict__ hdr,
                                                       const PrimeAux *__restrict__ aux, u32 count,
                                                       u64 *__restrict__ tabs, u64 *__restrict__ tgt,
                                                       unsigned short *__restrict__ meta, u64 *__restrict__ stats,
                                                       u32 *__restrict__ err, JobGeom gm,
                                                       const JobGeom *__restrict__ geoms,
                                                       const u32 *__restrict__ prefix, u32 nr,
                                                       const u32 *__restrict__ rec_of)
{
    __shared__ u64 s_tw[SETUP_TPB / 32][SPLIT_MAX + CLS_SLOTS + 4 * 32];   // per warp: powers of b, class lookup keys, chi(k)
    __shared__ unsigned char s_cr[SETUP_TPB / 32][CLS_SLOTS];     //   and the lookup's class indices
    const u32 lane = threadIdx.x & 31;
    const u32 nwarps = gridDim.x * (SETUP_TPB / 32);
    u64 *tw = s_tw[threadIdx.x >> 5];
    unsigned char *cr = s_cr[threadIdx.x >> 5];
    // w is uniform over the warp, so the warp-wide ballots of a prime stay whole
    if constexpr (BATCH) {
        const u32 total = prefix[nr];
        for (u32 i = (blockIdx.x * SETUP_TPB + threadIdx.x) >> 5; i < total; i += nwarps) {
            const u32 rec = rec_of[i];
            const u32 jb = hdr[rec].job;
            setup_k_one(jobs + jb, rec, lane, hdr, aux, tabs, tgt, meta, stats, err, geoms[jb], tw, cr);
        }
    } else {
        for (u32 w = (blockIdx.x * SETUP_TPB + threadIdx.x) >> 5; w < count; w += nwarps)
            setup_k_one(jobs, w, lane, hdr, aux, tabs, tgt, meta, stats, err, gm, tw, cr);
    }
}

cudaError_t launch_setup(const JobDev *job, const u64 *primes, u32 first, u32 count, PrimeHdr *hdr, void *aux, u64 *tabs,
                         u64 *tgt, unsigned short *meta, u64 *stats, u32 *err, int geom, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    const JobGeom gm = job_geom(geom);
    k_setup_prime<false><<<(count + 255) / 256, 256, 0, st>>>(job, primes, first, count, hdr, (PrimeAux *)aux, gm,
                                                              nullptr, nullptr, nullptr, 0, 0, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const u32 wpb = SETUP_TPB / 32;
    k_setup_k<false><<<(count + wpb - 1) / wpb, SETUP_TPB, 0, st>>>(job, hdr, (const PrimeAux *)aux, count, tabs, tgt,
                                                                   meta, stats, err, gm, nullptr, nullptr, 0, nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_setup_tabs<false><<<(count + 255) / 256, 256, 0, st>>>(job, hdr, (const PrimeAux *)aux, count, tabs, stats, gm,
                                                             nullptr, nullptr, 0, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_setup_batch(const JobDev *jobs, const JobGeom *geoms, const BatchRange *ranges, const u64 *primes,
                               u32 rcap, const u32 *prefix_p, u32 nranges, PrimeHdr *hdr, void *aux, u64 *tabs,
                               u64 *tgt, unsigned short *meta, u64 *stats, u32 *err, u32 *rec_of, int sms,
                               cudaStream_t st)
{
    JobGeom gm{};
    // full-device grids; the kernels stride over the primes of every range
    k_setup_prime<true><<<sms * 4, 256, 0, st>>>(jobs, primes, 0, 0, hdr, (PrimeAux *)aux, gm, geoms, ranges,
                                                 prefix_p, nranges, rcap, rec_of);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_setup_k<true><<<sms * 4, SETUP_TPB, 0, st>>>(jobs, hdr, (const PrimeAux *)aux, 0, tabs, tgt, meta, stats, err,
                                                   gm, geoms, prefix_p, nranges, rec_of);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_setup_tabs<true><<<sms * 4, 256, 0, st>>>(jobs, hdr, (const PrimeAux *)aux, 0, tabs, stats, gm, geoms,
                                                prefix_p, nranges, rec_of);
    return cudaGetLastError();
}

size_t setup_aux_bytes() { return sizeof(PrimeAux); }

}  // namespace rs

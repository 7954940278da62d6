// setup.cu -- per-prime set-up for the BSGS search.
//
// Replaces the reference's setup and sort kernels (kernels/setup.cl:89-209,
// kernels/sort.cl:11-104).  The arithmetic is re-derived rather than ported:
//
// Term k*b^n + c (c = +-1) is divisible by p iff k*b^n == -c (mod p).  Write
// n = nmin + off + e*u with e = 1 (b a quadratic residue mod p: one table for
// every n) or e = 2 (b a non-residue: even n, off = 0, and odd n, off = 1,
// share one table of powers of s = b^2), and u = (q+1)*Q - 1 - j with baby
// index j in [0,Q) and giant index q.  Then
//      s^j == T * S^q,   T = -c * k * b^(nmin + off + e*(Q-1)),   S = s^Q,
// so the baby table holds s^j and no modular inverse is needed (the reference
// batch-inverts every k and b^Q, setup.cl:133-166).
//
// The prefilter is the reference's (setup.cl:22-87), restated on k itself:
// the target b^n == -c*k^-1 must be a d-th power whenever b is one (d | p-1,
// d in {3,4,5,7,8,9,11,13,17,19,23,29}), i.e. k^((p-1)/d) == (-c)^((p-1)/d);
// and its quadratic character (-c/p)(k/p), computed with Jacobi symbols instead
// of an Euler power, decides impossible / full range / even n / odd n.
// Primes dividing b or any k, and primes where no k survives, are skipped for
// every sequence exactly as setup.cl:156-162,205-208 do.
//
// Kernel 1 (one thread per prime) does the per-prime scalars; kernel 2 (one
// warp per prime, lanes over k) classifies the sequences and writes the
// compacted targets and the giant-step start tables.
#include "mont.cuh"
#include "rs_internal.h"

namespace rs {

__device__ __constant__ u32 c_DS[NDS] = {3, 4, 5, 7, 8, 9, 11, 13, 17, 19, 23, 29};

// Legendre symbol (x/p) for x = 2^v2 * xodd, p an odd prime not dividing x,
// by quadratic reciprocity: (xodd/p) = (p mod xodd / xodd) * (-1)^((xodd-1)/2*(p-1)/2).
__device__ __forceinline__ int legendre_of(u64 xodd, u32 v2, u64 xrd, u64 p)
{
    int t = 1;
    const u32 r8 = (u32)p & 7;
    if ((v2 & 1) && (r8 == 3 || r8 == 5)) t = -t;      // (2/p)
    if (xodd == 1) return t;
    u64 a = mod_barrett(p, xodd, xrd);
    if (a == 0) return 0;
    if ((xodd & 3) == 3 && (p & 3) == 3) t = -t;
    int j = (xodd >> 32) ? jacobi64(a, xodd) : jacobi32((u32)a, (u32)xodd);
    return t * j;
}

// (p-1)/DS[j] for a compile-time j (division by a constant)
__device__ __forceinline__ u64 pm1_div(u64 pm1, int j)
{
    switch (j) {
    case 0: return pm1 / 3;   case 1: return pm1 >> 2;  case 2: return pm1 / 5;   case 3: return pm1 / 7;
    case 4: return pm1 >> 3;  case 5: return pm1 / 9;   case 6: return pm1 / 11;  case 7: return pm1 / 13;
    case 8: return pm1 / 17;  case 9: return pm1 / 19;  case 10: return pm1 / 23; default: return pm1 / 29;
    }
}

struct PrimeAux {        // kernel 1 -> kernel 2 scalars
    u64 r2;              // R^2 mod p
    u64 wr0, wr1;        // b^(nmin+e(Q-1)) * R^2 and b^(nmin+1+e(Q-1)) * R^2 (mod p)
    u32 amask;           // active power-residue degrees (bit j <=> DS[j])
    u32 pad_;
};

// Per-prime constants of prime p into record t.
__device__ __forceinline__ void setup_prime_one(const JobDev *__restrict__ job, u64 p, u32 t, u32 jb,
                                                PrimeHdr *__restrict__ hdr, PrimeAux *__restrict__ aux,
                                                u64 *__restrict__ tabs, const JobGeom &gm)
{
    PrimeHdr H;
    H.p = 0; H.q = 0; H.one = 0; H.s = 0; H.S = 0; H.numk = 0; H.e = 0; H.G = 0; H.Lc = 0; H.smul = 0; H.job = jb;
    H.Sh = 0; H.Sw = 0;
    const Mont M = mont_init(p);
    const u32 b = job->base;
    const u64 bm = to_mont(b, M);
    if (bm == 0) { hdr[t] = H; return; }                 // p | b: no term is divisible by p
    const int rg = legendre_of(job->bodd, job->bv2, job->brd, p);
    const u32 e = (rg == -1) ? 2u : 1u;
    const u64 s = (e == 2) ? mmul(bm, bm, p, M.q) : bm;
    const u64 S = mpow(s, (u64)gm.q, M);
    const u64 W0 = mpow(bm, (u64)job->nmin + (u64)e * (gm.q - 1), M);
    PrimeAux X;
    X.r2 = M.r2;
    X.wr0 = mmul(W0, M.r2, p, M.q);
    X.wr1 = mul_base(X.wr0, b, bm, M);
    // d-th power residuosity of b (good_pr, setup.cl:11-48)
    u32 am = 0;
    const u64 pm1 = p - 1;
#pragma unroll
    for (int j = 0; j < NDS; ++j) {
        u64 ex = pm1_div(pm1, j);
        if (ex * c_DS[j] == pm1 && ex > 0 && mpow(bm, ex, M) == M.one) am |= 1u << j;
    }
    X.amask = am;
    X.pad_ = 0;
    // baby-step start tables: A[l] = s^(C*l), B[w] = s^(32*C*w)
    u64 *tb = tabs + (size_t)t * TABS;
    const u64 u = mpow(s, (u64)gm.c, M);
    u64 a = M.one;
    for (int l = 0; l < 32; ++l) { tb[l] = a; a = mmul(a, u, p, M.q); }
    const u64 v = a;                                      // u^32
    a = M.one;
    for (int w = 0; w < 32; ++w) { tb[32 + w] = a; a = mmul(a, v, p, M.q); }
    const u64 bb = (e == 2) ? (u64)b * b : (u64)b;
    H.p = p; H.q = M.q; H.one = M.one; H.s = s; H.S = S; H.e = e;
    H.Sw = (p >> 63) ? 0 : shoup_const(from_mont(S, M), p);   // nonzero: from_mont(S) = s^Q != 0 mod p
    H.smul = (bb <= 16) ? (u32)bb : 0u;
    hdr[t] = H;
    aux[t] = X;
}


// Kernel 1.  Single job: primes[first, first+count) into records [0, count)
// with the launch's geometry gm.  Batch (BATCH): the primes of every range as
// one index space (prefix: prefix sums of the ranges' prime counts); prime i
// of range r is record r*rcap + i, with its job's sequences and geometry.
template <bool BATCH>
__global__ void __launch_bounds__(256) k_setup_prime(const JobDev *__restrict__ jobs, const u64 *__restrict__ primes,
                                                     u32 first, u32 count, PrimeHdr *__restrict__ hdr,
                                                     PrimeAux *__restrict__ aux, u64 *__restrict__ tabs, JobGeom gm,
                                                     const JobGeom *__restrict__ geoms,
                                                     const BatchRange *__restrict__ ranges,
                                                     const u32 *__restrict__ prefix, u32 nr, u32 rcap)
{
    const u32 stride = gridDim.x * blockDim.x;
    if (BATCH) {
        const u32 total = prefix[nr];
        for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
            const u32 r = prefix_find(prefix, nr, i);
            const u32 rec = r * rcap + (i - prefix[r]);
            const u32 jb = ranges[r].job;
            setup_prime_one(jobs + jb, primes[rec], rec, jb, hdr, aux, tabs, geoms[jb]);
        }
        return;
    }
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += stride)
        setup_prime_one(jobs, primes[first + t], t, 0, hdr, aux, tabs, gm);
}

// Sequence classes, targets and giant-step tables of record w (one warp).
__device__ __forceinline__ void setup_k_one(const JobDev *__restrict__ job, u32 w, u32 lane, PrimeHdr *__restrict__ hdr,
                                            const PrimeAux *__restrict__ aux, u64 *__restrict__ tabs,
                                            u64 *__restrict__ tgt, unsigned char *__restrict__ meta,
                                            u64 *__restrict__ stats, const JobGeom &gm)
{
    PrimeHdr H = hdr[w];
    if (H.p == 0) {
        if (lane == 0) atomicAdd(&stats[ST_SKIPPED], 1ull);
        return;
    }
    const PrimeAux X = aux[w];
    Mont M;
    M.p = H.p; M.q = H.q; M.one = H.one; M.r2 = X.r2;
    const u64 p = H.p;
    const u32 K = job->kcount;
    const bool m1qr = ((p & 3) == 1);                     // (-1/p) = +1
    const u64 mone = p - M.one;
    u32 nk = 0;
    bool divk = false;
    for (u32 i0 = 0; i0 < K; i0 += 32) {
        const u32 i = i0 + lane;
        bool keep = false;
        u64 T = 0;
        unsigned char mt = 0;
        if (i < K) {
            const u64 kv = job->k[i];
            const u64 kr = (kv < p) ? kv : kv % p;
            if (kr == 0) {
                divk = true;
            } else {
                const int ci = job->c[i];
                int ra = legendre_of(job->kodd[i], job->kv2[i], job->krd[i], p);
                if (ci == 1 && !m1qr) ra = -ra;           // (-c/p)(k/p) is the character of -c*k^-1
                u32 off = 0;
                bool ok;
                if (H.e == 1) ok = (ra == 1);
                else { ok = true; off = ((ra == 1) ? 0u : 1u) ^ (job->nmin & 1u); }   // n even <=> off == nmin mod 2
                if (ok && X.amask) {
                    const u64 km = to_mont(kr, M);
#pragma unroll 1
                    for (int j = 0; j < NDS; ++j) {
                        if (!((X.amask >> j) & 1)) continue;
                        const u64 ex = pm1_div(p - 1, j);
                        const u64 want = (ci == 1 && (ex & 1)) ? mone : M.one;
                        if (mpow(km, ex, M) != want) { ok = false; break; }
                    }
                }
                if (ok) {
                    T = mmul(kr, off ? X.wr1 : X.wr0, p, M.q);
                    if (ci == 1) T = mneg(T, p);
                    mt = (unsigned char)(i | (off << 7));
                    keep = true;
                }
            }
        }
        const u32 km_ = __ballot_sync(0xFFFFFFFFu, keep);
        if (keep) {
            const u32 pos = nk + __popc(km_ & ((1u << lane) - 1));
            tgt[(size_t)w * KSTRIDE + pos] = T;
            meta[(size_t)w * KSTRIDE + pos] = mt;
        }
        nk += __popc(km_);
    }
    divk = __any_sync(0xFFFFFFFFu, divk);
    if (divk || nk == 0) {
        if (lane == 0) {
            hdr[w].p = 0;
            atomicAdd(&stats[ST_SKIPPED], 1ull);
        }
        return;
    }
    // giant-phase split: G chunks of Lc giant steps per target, numk*G <= tpb
    const u32 Mg = (H.e == 2) ? gm.m2 : gm.m1;
    u32 G = gm.tpb / nk;
    if (G < 1) G = 1;
    if (G > Mg) G = Mg;
    const u32 Lc = (Mg + G - 1) / G;
    G = (Mg + Lc - 1) / Lc;
    // Z1[l] = S^(Lc*l), Z2[w] = S^(32*Lc*w), lane l computes entry l of both
    const u64 z = mpow(H.S, (u64)Lc, M);
    u64 acc = M.one, pw = z, acc2 = M.one;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit) {
        if ((lane >> bit) & 1) acc = mmul(acc, pw, p, M.q);
        pw = mmul(pw, pw, p, M.q);
    }
    // pw = z^32
#pragma unroll
    for (int bit = 0; bit < 5; ++bit) {
        if ((lane >> bit) & 1) acc2 = mmul(acc2, pw, p, M.q);
        pw = mmul(pw, pw, p, M.q);
    }
    u64 *tb = tabs + (size_t)w * TABS;
    tb[64 + lane] = acc;
    tb[96 + lane] = acc2;
    const u64 sh = mpow(H.S, (u64)(Lc >> 1), M);
    if (lane == 0) {
        hdr[w].numk = nk;
        hdr[w].G = G;
        hdr[w].Lc = Lc;
        hdr[w].Sh = sh;
        atomicAdd(&stats[ST_TARGETS], (u64)nk);
        atomicAdd(&stats[H.e == 2 ? ST_PARITY : ST_FULL], 1ull);
    }
}


// Kernel 2: one warp per prime; lanes walk the sequences.  BATCH as kernel 1.
template <bool BATCH>
__global__ void __launch_bounds__(SETUP_TPB, 6) k_setup_k(const JobDev *__restrict__ jobs, PrimeHdr *__restrict__ hdr,
                                                       const PrimeAux *__restrict__ aux, u32 count,
                                                       u64 *__restrict__ tabs, u64 *__restrict__ tgt,
                                                       unsigned char *__restrict__ meta, u64 *__restrict__ stats,
                                                       JobGeom gm, const JobGeom *__restrict__ geoms,
                                                       const BatchRange *__restrict__ ranges,
                                                       const u32 *__restrict__ prefix, u32 nr, u32 rcap)
{
    const u32 lane = threadIdx.x & 31;
    const u32 nwarps = gridDim.x * (SETUP_TPB / 32);
    // w is uniform over the warp, so the warp-wide ballots of a prime stay whole
    if (BATCH) {
        const u32 total = prefix[nr];
        for (u32 i = (blockIdx.x * SETUP_TPB + threadIdx.x) >> 5; i < total; i += nwarps) {
            const u32 r = prefix_find(prefix, nr, i);
            const u32 rec = r * rcap + (i - prefix[r]);
            const u32 jb = ranges[r].job;
            setup_k_one(jobs + jb, rec, lane, hdr, aux, tabs, tgt, meta, stats, geoms[jb]);
        }
        return;
    }
    for (u32 w = (blockIdx.x * SETUP_TPB + threadIdx.x) >> 5; w < count; w += nwarps)
        setup_k_one(jobs, w, lane, hdr, aux, tabs, tgt, meta, stats, gm);
}

cudaError_t launch_setup(const JobDev *job, const u64 *primes, u32 first, u32 count, PrimeHdr *hdr, void *aux, u64 *tabs,
                         u64 *tgt, unsigned char *meta, u64 *stats, int geom, u32 L, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    const BsgsGeom &g = BSGS_GEOMS[geom];
    JobGeom gm;
    gm.q = g.q; gm.c = g.c; gm.tpb = g.tpb; gm.pad_ = 0;
    gm.m1 = (u32)(((u64)L + g.q - 1) / g.q);
    gm.m2 = (u32)(((u64)L + 2ull * g.q - 1) / (2ull * g.q));
    k_setup_prime<false><<<(count + 255) / 256, 256, 0, st>>>(job, primes, first, count, hdr, (PrimeAux *)aux, tabs, gm,
                                                              nullptr, nullptr, nullptr, 0, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const u32 wpb = SETUP_TPB / 32;
    k_setup_k<false><<<(count + wpb - 1) / wpb, SETUP_TPB, 0, st>>>(job, hdr, (const PrimeAux *)aux, count, tabs, tgt,
                                                                   meta, stats, gm, nullptr, nullptr, nullptr, 0, 0);
    return cudaGetLastError();
}

cudaError_t launch_setup_batch(const JobDev *jobs, const JobGeom *geoms, const BatchRange *ranges, const u64 *primes,
                               u32 rcap, const u32 *prefix_p, u32 nranges, PrimeHdr *hdr, void *aux, u64 *tabs,
                               u64 *tgt, unsigned char *meta, u64 *stats, int sms, cudaStream_t st)
{
    JobGeom gm{};
    // full-device grids; the kernels stride over the primes of every range
    k_setup_prime<true><<<sms * 4, 256, 0, st>>>(jobs, primes, 0, 0, hdr, (PrimeAux *)aux, tabs, gm, geoms, ranges,
                                                 prefix_p, nranges, rcap);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_setup_k<true><<<sms * 6, SETUP_TPB, 0, st>>>(jobs, hdr, (const PrimeAux *)aux, 0, tabs, tgt, meta, stats, gm,
                                                   geoms, ranges, prefix_p, nranges, rcap);
    return cudaGetLastError();
}

size_t setup_aux_bytes() { return sizeof(PrimeAux); }

}  // namespace rs

// bsgs.cu -- baby-step giant-step search, one prime per CTA at a time.
//
// Replaces the reference's giantfull/giantparity kernels (kernels/giant.cl:77-323).
// For one prime p with per-prime record (see setup.cu):
//   baby phase   y_j = s^j for j in [0,Q'), Q' = TPB*cp with cp = C, C/2 or
//                C/4 chosen per prime by the set-up: thread t computes
//                y_{t*cp..t*cp+cp-1} from its start A[t%32]*B[t/32] with cheap
//                steps (doublings when b^e is 2 or 4, else one modular
//                product), checks y_j == 1 to detect ord(s) < Q'
//                (giant.cl:123-134), then inserts j < ord into a shared-memory
//                hash table.
//   giant phase  gamma = T_i * S^q for q in [0,Mg): thread (i,g) walks q in
//                [g*Lc, (g+1)*Lc) from T_i * S^(g*Lc) as two interleaved
//                chains, one modular product (Shoup's for p < 2^63, else
//                Montgomery) and one table probe per step (giant.cl:170-192).  A match
//                s^j == gamma gives n = nmin + off_i + e*((q+1)*Q' - 1 - j),
//                where s = b^e and off_i is target i's class of n mod e
//                (setup.cu; e = 2 is the reference's parity split).
//   small order  ord(s) < Q': each target is looked up once and every n in
//                range with the same residue mod e*ord is claimed (giant.cl:146-168).
//   claims       atomicAnd on the term's bitmap bit; the first claimer appends
//                {p, n, seq} to the factor buffer (giant.cl:21-39,158-162).
//
// Hash table: NB buckets in shared memory.  Bucket b is 16 bytes of
// fingerprints -- seven 16-bit slots and an eighth halfword that is 0x8000
// when the bucket overflowed, i.e. later values continued into the next bucket
// (linear probing) -- plus seven 16-bit baby indices j in a separate array and
// a 16-bit fill count in a third (two per word, so that the counts' atomics
// spread over all shared-memory banks).  Every halfword has one writer or
// writers of one value, so all table writes are plain 16-bit stores.
// A fingerprint match is verified exactly by recomputing y_j from its
// thread's start value, so the search is exact for every 64-bit value (the
// reference's split lo32/hi32 table cannot find values whose low 32 bits are
// zero, giant.cl:46,63).
#include "mont.cuh"
#include "rs_internal.h"

#include <type_traits>

namespace rs {

constexpr u32 HMUL = 0x9E3779B1u;

// Table hash of a 64-bit residue: h = (lo32 ^ hi32) * 0x9E3779B1.  The bucket
// is floor(h * NB / 2^32), i.e. the top bits of h; the fingerprint comes from
// the low 16 bits of h with bit 14 cleared and bit 10 set, which makes it the
// bit pattern of a normal (finite, nonzero) fp16 number.  Both words of the
// residue are folded in because the baby chain for small bases is a run of
// doublings whose low bits alone repeat shifted patterns.
template <u32 NB>
__device__ __forceinline__ void tab_hash(u64 val, u32 &bucket, u32 &fp)
{
    const u32 h = ((u32)val ^ (u32)(val >> 32)) * HMUL;
    bucket = __umulhi(h, NB);
    fp = (h & 0xBFFFu) | 0x0400u;
}

// Lane-wise fp16 equality of two packed pairs: 0xFFFF per equal half.  For
// normal fp16 patterns equality of values is equality of bits, and an empty
// slot (+0) never equals a fingerprint, so this is an exact 16-bit compare
// that covers two slots per instruction.
__device__ __forceinline__ u32 heq2(u32 a, u32 b)
{
    u32 d;
    asm("set.eq.u32.f16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

struct Table {
    uint4 *fpb;                // NB buckets of fingerprints + overflow flag
    unsigned short *jt;        // j of slot k of bucket b at jt[8*b + k]
    u32 *cnt;                  // fill count of bucket b in half (b & 1) of cnt[b >> 1]
};

constexpr u32 OVF_FLAG = 0x80000000u;   // bit 31 of a bucket's last word: halfword 7 = 0x8000

// Slot claim in bucket b: the count's atomicAdd hands out the slot.
__device__ __forceinline__ u32 tab_claim(const Table &T, u32 b)
{
    const u32 sh = (b & 1u) << 4;
    return (atomicAdd(&T.cnt[b >> 1], 1u << sh) >> sh) & 0xFFFFu;
}

// Fills slot `slot` of bucket b, or flags b as overflowed when slot > 6.
// Returns whether the value was placed.
__device__ __forceinline__ bool tab_fill(const Table &T, u32 b, u32 slot, u32 fp, u32 j)
{
    unsigned short *h = reinterpret_cast<unsigned short *>(&T.fpb[b]);
    if (slot < 7) {
        h[slot] = (unsigned short)fp;
        T.jt[8 * b + slot] = (unsigned short)j;
        return true;
    }
    h[7] = 0x8000u;
    return false;
}

// One insertion attempt into bucket b; on a full bucket, b advances and false
// is returned.
template <u32 NB>
__device__ __forceinline__ bool tab_try(const Table &T, u32 &b, u32 fp, u32 j)
{
    if (tab_fill(T, b, tab_claim(T, b), fp, j)) return true;
    b = (b + 1 == NB) ? 0u : b + 1;
    return false;
}

// halfword k (0..6) of a bucket
__device__ __forceinline__ u32 slot_fp(const uint4 &bv, int k)
{
    const u32 w = (k < 2) ? bv.x : (k < 4) ? bv.y : (k < 6) ? bv.z : bv.w;
    return (k & 1) ? (w >> 16) : (w & 0xFFFFu);
}

// y -> y*s: doubling/quadrupling for b = 2 (the common case), additions for
// b^e <= 16, a Montgomery product otherwise (smul is uniform per prime)
// 2x mod p for p < 2^63 (2x cannot wrap): one compare, one predicated subtract
__device__ __forceinline__ u64 dbl63(u64 x, u64 p)
{
    x += x;
    return (x >= p) ? x - p : x;
}

__device__ __forceinline__ u64 baby_step(u64 x, u32 smul, u64 s, u64 p, u64 q)
{
    if (smul == 2) return madd(x, x, p);
    if (smul == 4) { x = madd(x, x, p); return madd(x, x, p); }
    return smul ? mul_small(x, smul, p) : mmul(x, s, p, q);
}

// ---- TMA 1D bulk copies and mbarriers (record prefetch) ----
__device__ __forceinline__ u32 smem_u32(const void *p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u64 *bar, u32 count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(u64 *bar, u32 bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// global -> this CTA's shared memory, completion counted on bar (no multicast)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, u32 bytes, u64 *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(u64 *bar, u32 parity)
{
    u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// One prime's record as the setup kernels lay it out, staged in shared memory.
struct RecBuf {
    PrimeHdr hdr;
    u64 tabs[TABS];                 // A[32] B[32] Z1[32] Z2[32]
    u64 tgt[KSTRIDE];
    unsigned short meta[KSTRIDE];   // sequence | offset << 7
};
static_assert(sizeof(RecBuf) % 16 == 0, "bulk copies move 16-byte units");

constexpr u32 WAIT_BOUND = 1u << 24;   // default try_wait rounds before a copy is declared lost

// ---- per-CTA state in shared memory, read by the out-of-line rare paths ----
// The hot loops stay small (and in the instruction cache) because matches,
// overflowed buckets, small orders and claims run in __noinline__ functions
// that take a few scalars and find everything else here.
struct PrimeCtx {
    u64 p, q, s;         // the prime, p^-1 mod 2^64, Montgomery b^e
    u32 smul, e;         // baby-step multiplier when additions suffice; split modulus
    u32 cp, qp;          // baby steps per thread and per prime (qp = TPB * cp)
    u32 fp;              // FP64 steps (MODE 2): table and giant values are the bits of doubles
};
extern __shared__ __align__(128) unsigned char smem_raw[];
__shared__ BsgsArgs s_args;
__shared__ BsgsArgs s_args_next;                         // batch launches: the job arguments of the next prime
__shared__ PrimeCtx s_ctx;
__shared__ unsigned long long s_cands, s_dups, s_facs;   // per-CTA totals
__shared__ unsigned long long s_baby, s_giant, s_small;  // per-CTA totals kept by thread 0
__shared__ u32 s_nsol, s_sol_i[KMAX], s_sol_u0[KMAX];   // small-order solutions

// A residue's table value: the residue itself, or with FP64 steps (MODE 2) the
// bit pattern of the double that holds it exactly (every step of that mode
// yields canonical residues, so equal residues have equal bits).
__device__ __forceinline__ u64 fp_val(u64 v) { return (u64)__double_as_longlong(fp_exact(v)); }
__device__ __forceinline__ u64 fp_res(u64 bits) { return (u64)__longlong_as_double((long long)bits); }
__device__ __forceinline__ u64 to_val(u64 v) { return s_ctx.fp ? fp_val(v) : v; }
__device__ __forceinline__ u64 to_res(u64 val) { return s_ctx.fp ? fp_res(val) : val; }

// Dynamic shared memory: fingerprints | indices | counts | start values | giant
// start powers | two record staging buffers.
template <int TPB, int NB>
struct Smem {
    static __device__ __forceinline__ Table table()
    {
        Table T;
        T.fpb = reinterpret_cast<uint4 *>(smem_raw);
        T.jt = reinterpret_cast<unsigned short *>(T.fpb + NB);
        T.cnt = reinterpret_cast<u32 *>(T.jt + 8 * NB);
        return T;
    }
    static __device__ __forceinline__ u64 *start() { return reinterpret_cast<u64 *>(table().cnt + NB / 2); }
    static __device__ __forceinline__ u64 *zs() { return start() + TPB; }
    static __device__ __forceinline__ RecBuf *rec() { return reinterpret_cast<RecBuf *>(zs() + TPB); }
    static constexpr size_t bytes() { return (size_t)NB * 16 + (size_t)NB * 16 + (size_t)NB * 2 + (size_t)TPB * 16 + 2 * sizeof(RecBuf); }
};

// First claimer of term (seq, n) clears its bitmap bit and appends the factor.
__device__ __forceinline__ void claim(u64 p, u32 seq, u32 n)
{
    const BsgsArgs &a = s_args;
    const u32 o = n - a.nmin;
    u32 *w = a.bitmap + (size_t)seq * a.words + (o >> 5);
    const u32 mask = 1u << (o & 31);
    const u32 old = atomicAnd(w, ~mask);
    if (old & mask) {
        const u32 f = atomicAdd(a.factor_ctr, 1u);
        atomicAdd(&s_facs, 1ull);
        if (f < a.factor_cap) {
            FactorRec r;
            r.p = p; r.n = n; r.seq = seq;
            a.factors[f] = r;
        } else {
            atomicOr(a.err, ERR_FACTOR_OVERFLOW);
        }
    } else {
        atomicAdd(&s_dups, 1ull);
    }
}

// exact check of a fingerprint match: y_j == val ?  (y_j from its thread's
// start, by integer steps on the residues whatever the launch's step kind)
__device__ __forceinline__ bool verify(const u64 *s_start, u32 j, u64 val)
{
    const PrimeCtx c = s_ctx;
    if (j >= c.qp) return false;
    u64 y = to_res(s_start[j / c.cp]);
    for (u32 r = j % c.cp; r; --r) y = baby_step(y, c.smul, c.s, c.p, c.q);
    return y == to_res(val);
}

// Giant-step match or overflowed bucket: check every matching slot of the
// chain starting at bucket b exactly and claim n = nmin + off + e*((q+1)Q'-1-j).
template <int TPB, int C, int NB>
__device__ __noinline__ void giant_slow(u64 gamma, u32 b, u32 fp, u32 qq, u32 meta)
{
    const u32 Q = s_ctx.qp;
    const Table T = Smem<TPB, NB>::table();
    const u64 *st = Smem<TPB, NB>::start();
    for (int pr = 0; pr < BSGS_MAXPROBE; ++pr) {
        const uint4 bv = T.fpb[b];
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            if (slot_fp(bv, k) != fp) continue;
            atomicAdd(&s_cands, 1ull);
            const u32 j = T.jt[8 * b + k];
            if (!verify(st, j, gamma)) continue;
            const u64 u = (u64)(qq + 1) * Q - 1 - j;
            const u64 n = (u64)s_args.nmin + (meta >> 7) + (u64)s_ctx.e * u;
            if (n <= s_args.nmax) claim(s_ctx.p, meta & 0x7Fu, (u32)n);
        }
        if (!(bv.w & OVF_FLAG)) break;
        b = (b + 1 == NB) ? 0u : b + 1;
    }
}

// The giant step's table probe: one 128-bit load, four paired fp16 compares
// and one branch in the common case.  The flag half of the last word (0 or
// 0x8000, i.e. +-0 as fp16) never equals a fingerprint, so all eight halves
// are compared without masking.
template <int TPB, int C, int NB>
__device__ __forceinline__ void giant_probe(const Table &T, u64 g, u32 qq, u32 meta)
{
    u32 b, fp;
    tab_hash<NB>(g, b, fp);
    const u32 kk = fp * 0x10001u;
    const uint4 bv = T.fpb[b];
    const u32 m = heq2(bv.x, kk) | heq2(bv.y, kk) | heq2(bv.z, kk) | heq2(bv.w, kk);
    if (__builtin_expect((m | (bv.w & OVF_FLAG)) != 0, 0)) {
        // about 1% of buckets overflowed: with no match here, the next bucket
        // is checked inline, and only matches or longer chains go out of line
        bool slow = (m != 0);
        if (!slow) {
            const uint4 bn = T.fpb[(b + 1 == NB) ? 0u : b + 1];
            slow = ((heq2(bn.x, kk) | heq2(bn.y, kk) | heq2(bn.z, kk) | heq2(bn.w, kk)) | (bn.w & OVF_FLAG)) != 0;
        }
        if (slow) giant_slow<TPB, C, NB>(g, b, fp, qq, meta);
    }
}

// Continues an insertion whose home bucket was full; returns 1 if the walk
// gave up after maxprobe buckets.
template <int NB>
__device__ __noinline__ u32 insert_walk(u32 b, u32 fp, u32 j, int maxprobe)
{
    const Table T = Smem<0, NB>::table();
    b = (b + 1 == NB) ? 0u : b + 1;
    for (int pr = 1; pr < maxprobe; ++pr)
        if (tab_try<NB>(T, b, fp, j)) return 0;
    return 1;
}

__device__ __forceinline__ void clear_table(const Table &T, u32 nb)
{
    for (u32 i = threadIdx.x; i < nb; i += blockDim.x) T.fpb[i] = make_uint4(0u, 0u, 0u, 0u);
    for (u32 i = threadIdx.x; i < nb / 8; i += blockDim.x) reinterpret_cast<uint4 *>(T.cnt)[i] = make_uint4(0u, 0u, 0u, 0u);
}

// ord(s) < Q': rebuild the table from the distinct values j < ord (the
// speculative one may hold repeats).  Called by the whole CTA.
template <int TPB, int C, int NB>
__device__ __noinline__ void rebuild_table(u32 order)
{
    const Table T = Smem<TPB, NB>::table();
    const u64 *st = Smem<TPB, NB>::start();
    const PrimeCtx c = s_ctx;
    clear_table(T, NB);
    __syncthreads();
    u64 y = to_res(st[threadIdx.x]);
    u32 pend = 0;
    for (u32 i = 0; i < c.cp; ++i) {
        const u32 j = threadIdx.x * c.cp + i;
        if (j < order) {
            u32 b, fpv;
            tab_hash<NB>(to_val(y), b, fpv);
            int pr = 0;
            while (pr < BSGS_MAXPROBE && !tab_try<NB>(T, b, fpv, j)) ++pr;
            if (pr >= BSGS_MAXPROBE) pend = 1;
        }
        y = baby_step(y, c.smul, c.s, c.p, c.q);
    }
    if (pend) atomicOr(s_args.err, ERR_HASH_OVERFLOW);
    __syncthreads();
}

// ord(s) < Q': each target is looked up once; every n in range with the same
// residue mod e*ord is claimed (giant.cl:146-168).  Called by the whole CTA.
template <int TPB, int C, int NB>
__device__ __noinline__ void small_order_search(const RecBuf *R, u32 order)
{
    const u32 Q = s_ctx.qp;
    const Table T = Smem<TPB, NB>::table();
    const u64 *st = Smem<TPB, NB>::start();
    const u32 tid = threadIdx.x;
    if (tid < R->hdr.numk) {
        // FP64 launches' tables carry R^2: the target T*R times R^2 mod p
        // (the header's ssw there) by one Montgomery product
        const u64 Tv = to_val(s_ctx.fp ? mmul(R->tgt[tid], R->hdr.ssw, s_ctx.p, s_ctx.q) : R->tgt[tid]);
        u32 b, fp;
        tab_hash<NB>(Tv, b, fp);
        for (int pr = 0; pr < BSGS_MAXPROBE; ++pr) {
            const uint4 bv = T.fpb[b];
            for (int k = 0; k < 7; ++k) {
                if (slot_fp(bv, k) != fp) continue;
                atomicAdd(&s_cands, 1ull);
                const u32 j = T.jt[8 * b + k];
                if (j >= order || !verify(st, j, Tv)) continue;
                const u32 ks = atomicAdd(&s_nsol, 1u);
                s_sol_i[ks] = tid;
                s_sol_u0[ks] = (Q - 1 - j) % order;
            }
            if (!(bv.w & OVF_FLAG)) break;
            b = (b + 1 == NB) ? 0u : b + 1;
        }
    }
    __syncthreads();
    const u32 nsol = s_nsol;
    const u32 e = s_ctx.e;
    for (u32 k = 0; k < nsol; ++k) {
        const u32 m = R->meta[s_sol_i[k]];
        const u32 seq = m & 0x7Fu, off = m >> 7;
        for (u64 u = s_sol_u0[k] + (u64)tid * order;; u += (u64)TPB * order) {
            const u64 n = (u64)s_args.nmin + off + (u64)e * u;
            if (n > s_args.nmax) break;
            claim(s_ctx.p, seq, (u32)n);
        }
    }
}

// Work item i of a batch launch: range slot k contributes prefix[k+1]-prefix[k]
// primes (0 when it is not in the launch's group), in record slots
// k*rcap + (0, 1, ...).
__device__ __forceinline__ u32 batch_slot(u32 i, u32 nr, const u32 *prefix, u32 rcap)
{
    const u32 k = prefix_find(prefix, nr, i);
    return k * rcap + (i - prefix[k]);
}

// MODE: 2 = every prime below FP_BOUND = 2^51 (FP64 baby and giant steps,
// fp_mulfix), 1 = every prime below 2^63 (Shoup steps), 0 = every prime at or
// above 2^63 (Montgomery giant steps).  1024 / TPB CTAs share an SM, so the
// bound keeps each thread at 64 registers.  BATCH: the primes of several
// ranges (jobs) in one launch -- work item i maps to a record slot through the
// group's prefix sums, and each prime's job arguments come from job_args.
template <int TPB, int C, int NB, int MODE, bool BATCH>
__global__ void __launch_bounds__(TPB, 1024 / TPB) k_bsgs(BsgsArgs a, const PrimeHdr *__restrict__ hdr,
                                                 const u64 *__restrict__ tabs, const u64 *__restrict__ tgt,
                                                 const unsigned short *__restrict__ meta, u32 count, u32 *work_ctr,
                                                 const BsgsArgs *__restrict__ job_args, u32 nr,
                                                 const u32 *__restrict__ prefix, u32 rcap)
{
    constexpr u32 NONE = 0xFFFFFFFFu;
    if (BATCH) count = prefix[nr];
    auto slot_of = [&](u32 i) -> u32 {
        if (i >= count) return NONE;
        return BATCH ? batch_slot(i, nr, prefix, rcap) : i;
    };
    constexpr u32 Q = TPB * C;
    static_assert(Q <= 65536, "baby indices are stored in 16 bits");
    static_assert(NB <= 65536, "bucket indices are packed into 16 bits");
    constexpr int IBMAX = 8;                                      // values inserted per round (two chains)
    static_assert(C >= IBMAX, "cp in {C, C/2, C/4} splits into rounds of IBMAX/2, IBMAX/4 or IBMAX/8 per chain");
    const Table T = Smem<TPB, NB>::table();
    u64 *s_start = Smem<TPB, NB>::start();
    u64 *s_Z = Smem<TPB, NB>::zs();
    RecBuf *rec = Smem<TPB, NB>::rec();                           // two staging buffers
    __shared__ __align__(8) u64 s_bar[3];                        // [2]: never completed (failure test)
    __shared__ u32 s_idx[2], s_order, s_spill, s_abort, s_claim;
    const u32 wait_bound = a.wait_bound ? a.wait_bound : WAIT_BOUND;
    u32 pend_buf = 0, pend_par = 0;                               // the copy waited for when aborting

    const u32 tid = threadIdx.x;
    auto fetch = [&](u32 buf, u32 idx) {                          // thread 0 only
        RecBuf *r = &rec[buf];
        mbar_expect_tx(&s_bar[buf], (u32)sizeof(RecBuf));
        bulk_load(&r->hdr, hdr + idx, (u32)sizeof(PrimeHdr), &s_bar[buf]);
        bulk_load(r->tabs, tabs + (size_t)idx * TABS, TABS * 8, &s_bar[buf]);
        bulk_load(r->tgt, tgt + (size_t)idx * KSTRIDE, KSTRIDE * 8, &s_bar[buf]);
        bulk_load(r->meta, meta + (size_t)idx * KSTRIDE, KSTRIDE * 2, &s_bar[buf]);
    };
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init(&s_bar[2], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_args = a;
        s_abort = 0;
        s_cands = 0;
        s_dups = 0;
        s_facs = 0;
        s_baby = 0;
        s_giant = 0;
        s_small = 0;
        const u32 i0 = slot_of(atomicAdd(work_ctr, 1u));
        s_idx[0] = i0;
        if (i0 != NONE) fetch(0, i0);
        s_claim = slot_of(atomicAdd(work_ctr, 1u));              // the prime after it, resolved ahead
        if (BATCH && i0 != NONE) s_args_next = job_args[hdr[i0].job];
    }
    __syncthreads();

    for (u32 it = 0;; ++it) {
        const u32 buf = it & 1;
        const u32 idx = s_idx[buf];
        if (idx == NONE) break;
        // this prime's record was fetched one prime ago; the wait is bounded.
        // A failure test sends the first wait to s_bar[2], which no copy or
        // arrival ever completes, so the bound runs out.
        pend_buf = buf;
        pend_par = (it >> 1) & 1;
        {
            const bool dead = (a.test_stall != 0) && (it == 0);
            u64 *bar = dead ? &s_bar[2] : &s_bar[buf];
            const u32 par = dead ? 0u : pend_par;
            u32 n = 0;
            while (!mbar_try_wait(bar, par)) {
                if (++n > wait_bound) { atomicOr(&s_abort, 1u); break; }
            }
        }
        const RecBuf &R = rec[buf];
        const bool live = (R.hdr.p != 0);
        const u64 p = R.hdr.p, q = R.hdr.q, s = R.hdr.s;
        const u32 e = R.hdr.e, smul = R.hdr.smul;
        const u32 cp = R.hdr.cp;                                  // baby steps per thread for this prime
        // The next prime's index (and, for a batch, its job's arguments) were
        // claimed and resolved during the previous prime, off the barriers'
        // critical path: thread 0 only copies them here.
        if (tid == 0) {
            s_order = 0xFFFFFFFFu;
            s_nsol = 0;
            s_spill = 0;
            s_ctx.p = p; s_ctx.q = q; s_ctx.s = s; s_ctx.smul = smul; s_ctx.e = e;
            s_ctx.cp = cp; s_ctx.qp = TPB * cp; s_ctx.fp = (MODE == 2);
            if (BATCH) s_args = s_args_next;
        }
        if (live) clear_table(T, NB);
        __syncthreads();
        if (s_abort) break;
        if (tid == 0) {
            const u32 nxt = s_claim;
            s_idx[buf ^ 1] = nxt;
            if (nxt != NONE) {                                    // rec[buf^1] was last read before the previous barrier
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                fetch(buf ^ 1, nxt);
            }
        }
        // MODE 2: start values by FP64 products x*y mod p (1/p in the header's
        // Sw), the set-up having stored Z2, s^(cp/2) and S^(Lc/2) plain: baby and
        // giant values carry R^2 (the header's ssw) where the integer modes'
        // Montgomery products leave R
        const double pd = fp_exact(p), pinv = __longlong_as_double((long long)R.hdr.Sw);
        if (live) {
            if (tid < R.hdr.G) {
                const u64 z1 = R.tabs[64 + (tid & 31)], z2 = R.tabs[96 + (tid >> 5)];
                s_Z[tid] = (MODE == 2) ? (u64)__double_as_longlong(fp_mul(fp_exact(z1), fp_exact(z2), pd, pinv))
                                       : mmul(z1, z2, p, q);
            }
            // ---- baby steps y_j = s^j, j < Q' = TPB*cp, inserted as they are produced ----
            // Speculative: ord(s) < Q' is only known after the barrier; then the
            // table (which may hold repeats) is rebuilt from j < ord.
            const u64 ta = R.tabs[tid & 31], tb = R.tabs[32 + (tid >> 5)];
            // s^(cp*tid); MODE 2: table values are the bits of the doubles holding the residues
            const u64 x0 = (MODE == 2) ? (u64)__double_as_longlong(fp_mul(fp_exact(ta), fp_exact(tb), pd, pinv))
                                       : mmul(ta, tb, p, q);
            const u64 one = (MODE == 2) ? fp_val(R.hdr.ssw) : R.hdr.one;
            s_start[tid] = x0;
            u32 spill = 0;
            // Two chains per thread, j in [tid*cp, tid*cp + cp/2) and the next
            // cp/2 (started from s^(cp/2) further), so the two products of a step
            // are independent.  The step kind is uniform per prime (b^e = 2, 4 or
            // other) and is chosen once, so the loop body carries no dispatch;
            // the least j > 0 with y_j = 1 is kept per thread and merged with one
            // atomicMin.  Other multipliers take Shoup's product by the plain s
            // below 2^63 (the same residues as the Montgomery product verify()
            // uses).
            u32 minj = 0xFFFFFFFFu;
            const u64 ssw = R.hdr.ssw;
            const u64 sp = R.hdr.sp;
            const u32 half = cp >> 1;
            u64 xa = x0, xb;
            if (MODE == 2)
                xb = (u64)__double_as_longlong(fp_mul(__longlong_as_double((long long)x0), fp_exact(R.hdr.u2), pd, pinv));
            else
                xb = mmul(x0, R.hdr.u2, p, q);
            const double sd = fp_exact(sp), sq = __longlong_as_double((long long)R.hdr.S);
            // IB2 values of each chain are hashed and stepped, then inserted, per
            // round (IB2 = IBMAX/2, or cp/2 when it is smaller)
            auto babies = [&](auto kind, auto ibc) {
                constexpr int K = decltype(kind)::value;          // 2, 4: doublings; 1: Shoup; 0: baby_step
                constexpr int IB2 = decltype(ibc)::value;
                auto step = [&](u64 v) -> u64 {
                    if (MODE == 2) {
                        double x = __longlong_as_double((long long)v);
                        if (K == 1) x = fp_mulfix(x, sd, sq, pd);
                        else { x = fp_dbl(x, pd); if (K == 4) x = fp_dbl(x, pd); }
                        return (u64)__double_as_longlong(x);
                    }
                    if (K == 0) return baby_step(v, smul, s, p, q);
                    if (K == 1) return shoup_mul(v, sp, ssw, p);
                    if (MODE == 1) { v = dbl63(v, p); return (K == 4) ? dbl63(v, p) : v; }
                    v = madd(v, v, p);
                    return (K == 4) ? madd(v, v, p) : v;
                };
#pragma unroll 1
                for (u32 h0 = 0; h0 < half; h0 += IB2) {
                    u32 bf[2 * IB2], old[2 * IB2];                // bucket << 16 | fingerprint; claimed slot
#pragma unroll
                    for (int i = 0; i < IB2; ++i) {
                        const u32 ja = tid * cp + h0 + i, jb = ja + half;
                        if (ja != 0 && xa == one) minj = min(minj, ja);
                        if (xb == one) minj = min(minj, jb);
                        u32 bk, fp;
                        tab_hash<NB>(xa, bk, fp);
                        bf[2 * i] = (bk << 16) | fp;
                        tab_hash<NB>(xb, bk, fp);
                        bf[2 * i + 1] = (bk << 16) | fp;
                        xa = step(xa);
                        xb = step(xb);
                    }
#pragma unroll
                    for (int i = 0; i < 2 * IB2; ++i) old[i] = tab_claim(T, bf[i] >> 16);
#pragma unroll
                    for (int i = 0; i < 2 * IB2; ++i) {
                        const u32 j = tid * cp + h0 + (i >> 1) + ((i & 1) ? half : 0u);
                        const u32 bk = bf[i] >> 16, fp = bf[i] & 0xFFFFu;
                        if (!tab_fill(T, bk, old[i], fp, j)) spill |= insert_walk<NB>(bk, fp, j, BSGS_SPEC_PROBE);
                    }
                }
            };
            // (FP64 steps keep three double constants live: rounds of two
            // values per chain keep the loop within 64 registers)
            auto babies_cp = [&](auto kind) {
                if (MODE != 2 && half >= IBMAX / 2) babies(kind, std::integral_constant<int, IBMAX / 2>{});
                else if (half >= IBMAX / 4) babies(kind, std::integral_constant<int, IBMAX / 4>{});
                else babies(kind, std::integral_constant<int, IBMAX / 8>{});
            };
            if (smul == 2) babies_cp(std::integral_constant<int, 2>{});
            else if (smul == 4) babies_cp(std::integral_constant<int, 4>{});
            else if constexpr (MODE >= 1) babies_cp(std::integral_constant<int, 1>{});
            else babies_cp(std::integral_constant<int, 0>{});
            if (minj != 0xFFFFFFFFu) atomicMin(&s_order, minj);
            if (spill) s_spill = 1;
        }
        __syncthreads();
        // the last thread (idle in the giant phase unless every thread has a
        // chunk) claims the prime after next and loads the next prime's job
        // arguments; both are read after this prime's last barrier
        if (tid == TPB - 1) {
            s_claim = slot_of(atomicAdd(work_ctr, 1u));
            const u32 nx = s_idx[buf ^ 1];
            if (BATCH && nx != NONE) s_args_next = job_args[hdr[nx].job];
        }
        const u32 order = s_order;
        const u32 Mg = R.hdr.Mg;
        if (live) {
            if (order != 0xFFFFFFFFu) rebuild_table<TPB, C, NB>(order);
            else if (tid == 0 && s_spill) atomicOr(a.err, ERR_HASH_OVERFLOW);

            if (order == 0xFFFFFFFFu) {
                // ---- giant steps: two independent chains per thread ----
                // chain A walks q in [q0, q0+h), chain B q in [q0+h, q1), h = Lc/2;
                // B starts from A's start times S^h (Sh), so the two products of
                // a step are independent and overlap in the pipeline.  Below
                // 2^63 the step is Shoup's product by the fixed s^Q' (Sw is its
                // quotient constant), else the Montgomery product by S.
                const u32 numk = R.hdr.numk, G = R.hdr.G, Lc = R.hdr.Lc;
                const u64 S = R.hdr.S, Sw = R.hdr.Sw, Sp = R.hdr.Sp;
                const double Sd = fp_exact(Sp), Sqd = __longlong_as_double((long long)R.hdr.Sq);
                if (tid < numk * G) {
                    // i = tid / G by a float reciprocal: (tid + 1/2) / G lies at
                    // least 1/(2G) from an integer, and the two roundings err by
                    // under 2^-22 relative (below 2^-12 * (1024/G) absolute)
                    const u32 i = (u32)(((float)tid + 0.5f) * __frcp_rn((float)G)), g = tid - i * G;
                    const u32 q0 = g * Lc;
                    const u32 q1 = min(q0 + Lc, Mg);
                    const u32 h = Lc >> 1;
                    const u32 nA = min(h, q1 - q0), nB = (q1 - q0) - nA;
                    const u32 m = R.meta[i];
                    u64 gA, gB;
                    if (MODE == 2) {
                        const double a0 = fp_mul(fp_exact(R.tgt[i]), __longlong_as_double((long long)s_Z[g]), pd, pinv);
                        gA = (u64)__double_as_longlong(a0);
                        gB = (u64)__double_as_longlong(fp_mul(a0, fp_exact(R.hdr.Sh), pd, pinv));
                    } else {
                        gA = mmul(R.tgt[i], s_Z[g], p, q);
                        gB = mmul(gA, R.hdr.Sh, p, q);
                    }
                    auto gstep = [&](u64 v) -> u64 {
                        if (MODE == 2)
                            return (u64)__double_as_longlong(fp_mulfix(__longlong_as_double((long long)v), Sd, Sqd, pd));
                        if (MODE == 1) return shoup_mul(v, Sp, Sw, p);
                        return mmul(v, S, p, q);
                    };
                    // chain B has nA or nA+1 steps, except in a target's last,
                    // shorter chunk, where it may have fewer or none
                    const u32 nt = max(nA, nB);
                    for (u32 t = 0; t < nt; ++t) {
                        if (t < nA) {
                            giant_probe<TPB, C, NB>(T, gA, q0 + t, m);
                            gA = gstep(gA);
                        }
                        if (t < nB) {
                            giant_probe<TPB, C, NB>(T, gB, q0 + h + t, m);
                            gB = gstep(gB);
                        }
                    }
                }
            } else {
                small_order_search<TPB, C, NB>(&R, order);
            }
            if (tid == 0) {
                s_baby += min(order, TPB * cp);
                if (order == 0xFFFFFFFFu) s_giant += (u64)R.hdr.numk * Mg;
                else s_small += 1;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        atomicAdd(&a.stats[ST_BABY], s_baby);
        atomicAdd(&a.stats[ST_GIANT], s_giant);
        atomicAdd(&a.stats[ST_SMALLORDER], s_small);
        atomicAdd(&a.stats[ST_CANDIDATES], s_cands);
        atomicAdd(&a.stats[ST_DUPS], s_dups);
        atomicAdd(&a.stats[ST_FACTORS], s_facs);
        atomicAdd(&a.stats[ST_HITS], s_dups + s_facs);
    }
    if (s_abort && tid == 0) {
        // A record wait gave up.  The CTA stopped before fetching another record,
        // so the only copy that can still be in flight is the one waited for:
        // report, then let it land (bounded by the default) before the CTA's
        // shared memory is released.
        atomicOr(a.err, ERR_TMA_TIMEOUT);
        u32 n = 0;
        while (n < WAIT_BOUND && !mbar_try_wait(&s_bar[pend_buf], pend_par)) ++n;
    }
}

template <int G, int MODE, bool BATCH = false>
static cudaError_t launch_geom(const BsgsArgs &a, const PrimeHdr *hdr, const u64 *tabs, const u64 *tgt,
                              const unsigned short *meta, u32 count, u32 *work_ctr, int sms, cudaStream_t st,
                              const BsgsArgs *job_args = nullptr, u32 nr = 0, const u32 *prefix = nullptr,
                              u32 rcap = 0)
{
    constexpr BsgsGeom g = BSGS_GEOMS[G];
    auto kern = k_bsgs<g.tpb, g.c, g.nb, MODE, BATCH>;
    const size_t smem = Smem<g.tpb, g.nb>::bytes();
    static thread_local int per_sm[32] = {0};            // resident CTAs per SM, per device
    int dev = 0;
    cudaGetDevice(&dev);
    int &occ = per_sm[dev & 31];
    if (occ == 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, g.tpb, smem);
        if (e != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
    }
    const u64 want = (u64)sms * (u64)occ;
    const unsigned grid = (unsigned)((BATCH || want < count) ? want : count);
    kern<<<grid, g.tpb, smem, st>>>(a, hdr, tabs, tgt, meta, count, work_ctr, job_args, nr, prefix, rcap);
    return cudaGetLastError();
}

template <int G, int MODE>
static cudaError_t set_smem()
{
    constexpr BsgsGeom g = BSGS_GEOMS[G];
    cudaError_t e = cudaFuncSetAttribute(k_bsgs<g.tpb, g.c, g.nb, MODE, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Smem<g.tpb, g.nb>::bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bsgs<g.tpb, g.c, g.nb, MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Smem<g.tpb, g.nb>::bytes());
}

template <int G>
static size_t smem_of() { return Smem<BSGS_GEOMS[G].tpb, BSGS_GEOMS[G].nb>::bytes(); }

size_t bsgs_smem_bytes(int geom)
{
    switch (geom) {
    case 0: return smem_of<0>();
    case 1: return smem_of<1>();
    case 2: return smem_of<2>();
    case 3: return smem_of<3>();
    default: return smem_of<4>();
    }
}

cudaError_t bsgs_prepare()
{
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    chk(set_smem<0, 0>()); chk(set_smem<0, 1>()); chk(set_smem<0, 2>());
    chk(set_smem<1, 0>()); chk(set_smem<1, 1>()); chk(set_smem<1, 2>());
    chk(set_smem<2, 0>()); chk(set_smem<2, 1>()); chk(set_smem<2, 2>());
    chk(set_smem<3, 0>()); chk(set_smem<3, 1>()); chk(set_smem<3, 2>());
    chk(set_smem<4, 0>()); chk(set_smem<4, 1>()); chk(set_smem<4, 2>());
    return e;
}

cudaError_t launch_bsgs(const BsgsArgs &a, const PrimeHdr *hdr, const u64 *tabs, const u64 *tgt,
                        const unsigned short *meta, u32 count, u32 *work_ctr, u64 pmin, u64 pmax, int geom, int sms,
                        cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    const u64 TOP = 1ull << 63;
    if (pmin < TOP && pmax > TOP) return cudaErrorInvalidValue;   // the caller splits launches at 2^63
    if (pmin < FP_BOUND && pmax > FP_BOUND) return cudaErrorInvalidValue;   // and at FP_BOUND
    const int mode = (pmax <= FP_BOUND) ? 2 : (pmax <= TOP) ? 1 : 0;
#define RS_BSGS_CASE(G)                                                                                  \
    case G:                                                                                              \
        return mode == 2 ? launch_geom<G, 2>(a, hdr, tabs, tgt, meta, count, work_ctr, sms, st)          \
             : mode == 1 ? launch_geom<G, 1>(a, hdr, tabs, tgt, meta, count, work_ctr, sms, st)          \
                         : launch_geom<G, 0>(a, hdr, tabs, tgt, meta, count, work_ctr, sms, st);
    switch (geom) {
        RS_BSGS_CASE(0)
        RS_BSGS_CASE(1)
        RS_BSGS_CASE(2)
        RS_BSGS_CASE(3)
        RS_BSGS_CASE(4)
    default: return cudaErrorInvalidValue;
    }
#undef RS_BSGS_CASE
}

// prefix[0] = 0, prefix[k+1] = prefix[k] + counter `which` of range slot k
// (capped at rcap) when it is active and in the (geom, shoup) group -- or, for
// geom < 0, when it is active -- else + 0.  One block of 256 threads: each
// sums a contiguous run of slots, a block scan offsets the runs.
__global__ void __launch_bounds__(256) k_batch_prefix(const BatchRange *ranges, u32 nr, int geom, int mode,
                                                      const u32 *ctrs, u32 rcap, u32 *prefix, int which)
{
    __shared__ u32 part[256];
    const u32 t = threadIdx.x;
    const u32 per = (nr + 255) / 256;
    const u32 k0 = t * per, k1 = min(k0 + per, nr);
    auto cnt = [&](u32 k) -> u32 {
        const BatchRange R = ranges[k];
        const bool in = R.active && (geom < 0 || (R.geom == geom && R.mode == mode));
        return in ? min(ctrs[k * BR_CTRS + which], rcap) : 0u;
    };
    u32 sum = 0;
    for (u32 k = k0; k < k1; ++k) sum += cnt(k);
    part[t] = sum;
    __syncthreads();
    for (u32 o = 1; o < 256; o <<= 1) {           // inclusive Hillis-Steele scan
        const u32 v = (t >= o) ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    u32 acc = part[t] - sum;                      // exclusive prefix of this run
    if (t == 0) prefix[0] = 0;
    for (u32 k = k0; k < k1; ++k) {
        acc += cnt(k);
        prefix[k + 1] = acc;
    }
}

// Every BSGS group's prefix sums in one launch: block g computes those of
// group g = 3*geometry + step kind (BatchRange::mode) into prefix + g*(nr+1) and
// clears the group's work counter.
__global__ void __launch_bounds__(256) k_batch_group_prefix(const BatchRange *ranges, u32 nr, const u32 *ctrs,
                                                            u32 rcap, u32 *prefix, u32 *work)
{
    __shared__ u32 part[256];
    const u32 g = blockIdx.x;
    const int geom = (int)(g / 3), mode = (int)(g % 3);
    u32 *pf = prefix + (size_t)g * (nr + 1);
    const u32 t = threadIdx.x;
    if (t == 0) work[g] = 0;
    const u32 per = (nr + 255) / 256;
    const u32 k0 = t * per, k1 = min(k0 + per, nr);
    auto cnt = [&](u32 k) -> u32 {
        const BatchRange R = ranges[k];
        const bool in = R.active && R.geom == geom && R.mode == mode;
        return in ? min(ctrs[k * BR_CTRS + 1], rcap) : 0u;
    };
    u32 sum = 0;
    for (u32 k = k0; k < k1; ++k) sum += cnt(k);
    part[t] = sum;
    __syncthreads();
    for (u32 o = 1; o < 256; o <<= 1) {
        const u32 v = (t >= o) ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    u32 acc = part[t] - sum;
    if (t == 0) pf[0] = 0;
    for (u32 k = k0; k < k1; ++k) {
        acc += cnt(k);
        pf[k + 1] = acc;
    }
}

cudaError_t launch_batch_group_prefix(const BatchRange *ranges, u32 nr, const u32 *ctrs, u32 rcap, u32 *prefix,
                                      u32 *work, cudaStream_t st)
{
    k_batch_group_prefix<<<3 * NGEOM, 256, 0, st>>>(ranges, nr, ctrs, rcap, prefix, work);
    return cudaGetLastError();
}

cudaError_t launch_batch_prefix_all(const BatchRange *ranges, u32 nr, int which, u32 cap, const u32 *ctrs,
                                    u32 *prefix, cudaStream_t st)
{
    k_batch_prefix<<<1, 256, 0, st>>>(ranges, nr, -1, 0, ctrs, cap, prefix, which);
    return cudaGetLastError();
}

cudaError_t launch_bsgs_batch(const BsgsArgs &a, const BsgsArgs *job_args, const PrimeHdr *hdr, const u64 *tabs,
                              const u64 *tgt, const unsigned short *meta, u32 nr, const u32 *prefix, u32 rcap,
                              u32 *work_ctr, int mode, int geom, int sms, cudaStream_t st)
{
#define RS_BSGS_BCASE(G)                                                                                           \
    case G:                                                                                                        \
        return mode == 2 ? launch_geom<G, 2, true>(a, hdr, tabs, tgt, meta, 0, work_ctr, sms, st, job_args, nr, prefix, \
                                                   rcap)                                                           \
             : mode == 1 ? launch_geom<G, 1, true>(a, hdr, tabs, tgt, meta, 0, work_ctr, sms, st, job_args, nr, prefix, \
                                                   rcap)                                                           \
                         : launch_geom<G, 0, true>(a, hdr, tabs, tgt, meta, 0, work_ctr, sms, st, job_args, nr, prefix, \
                                                   rcap);
    switch (geom) {
        RS_BSGS_BCASE(0)
        RS_BSGS_BCASE(1)
        RS_BSGS_BCASE(2)
        RS_BSGS_BCASE(3)
        RS_BSGS_BCASE(4)
    default: return cudaErrorInvalidValue;
    }
#undef RS_BSGS_BCASE
}

}  // namespace rs

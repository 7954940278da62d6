// bsgs.cu -- baby-step giant-step search, one prime per CTA at a time.
//
// Replaces the reference's giantfull/giantparity kernels (kernels/giant.cl:77-323).
// For one prime p with per-prime record (see setup.cu):
//   baby phase   y_j = s^j for j in [0,Q), Q = TPB*C: thread t computes
//                y_{tC..tC+C-1} from its start A[t%32]*B[t/32] with C-1 cheap
//                steps (additions when b^e <= 16), checks y_j == 1 to detect
//                ord(s) < Q (giant.cl:123-134), then inserts j < ord into a
//                shared-memory hash table.
//   giant phase  gamma = T_i * S^q for q in [0,M): thread (i,g) walks q in
//                [g*Lc, (g+1)*Lc) from T_i * S^(g*Lc) as two interleaved
//                chains, one Montgomery product and one table probe per step
//                (giant.cl:170-192).  A match
//                s^j == gamma gives n = nmin + off_i + e*((q+1)*Q - 1 - j).
//   small order  ord(s) < Q: each target is looked up once and every n in
//                range with the same residue mod e*ord is claimed (giant.cl:146-168).
//   claims       atomicAnd on the term's bitmap bit; the first claimer appends
//                {p, n, seq} to the factor buffer (giant.cl:21-39,158-162).
//
// Hash table: NB buckets of four 32-bit slots in shared memory (load 1/2),
// filled through per-bucket slot counters (see tab_try).
// A slot holds a 16-bit fingerprint of y, j+1 in bits 1..15 and, in slot 3, an
// overflow flag in bit 0 that tells a probe to continue into the next bucket
// (see tab_hash for the bucket and fingerprint).  A fingerprint
// match is verified exactly by recomputing y_j from its thread's start value,
// so the search is exact for every 64-bit value (the reference's split
// lo32/hi32 table cannot find values whose low 32 bits are zero, giant.cl:46,63).
#include "mont.cuh"
#include "rs_internal.h"

namespace rs {

constexpr u32 HMUL = 0x9E3779B1u;

// Table hash of a 64-bit residue: h = (lo32 ^ hi32) * 0x9E3779B1.  The bucket
// is the top NBLOG bits of h and the 16-bit fingerprint the bits below them.
// Both words are folded in because the baby chain for small bases is a run of
// doublings (x -> 2x mod p): the low bits alone repeat shifted patterns and
// crowd a few buckets.
template <u32 NBLOG>
__device__ __forceinline__ void tab_hash(u64 val, u32 &bucket, u32 &key)
{
    const u32 h = ((u32)val ^ (u32)(val >> 32)) * HMUL;
    bucket = h >> (32 - NBLOG);
    key = (h << NBLOG) & 0xFFFF0000u;
}

// Slot claim: a 16-bit counter per bucket (two per word) hands out slots with
// one atomicAdd and no read-before-write.  Slots 0..2 take a plain store; slot
// 3 takes an atomicOr so a concurrent overflow flag (bit 0) survives.  A value
// that finds its bucket full flags it and moves to the next bucket.  Returns
// true when placed; on false, b is the next bucket to try.
template <u32 NBLOG>
__device__ __forceinline__ bool tab_try(u32 *tab32, u32 *cnt, u32 &b, u32 ent)
{
    constexpr u32 NB = 1u << NBLOG;
    const u32 sh = (b & 1u) << 4;
    const u32 slot = (atomicAdd(&cnt[b >> 1], 1u << sh) >> sh) & 0xFFFFu;
    if (slot < 3) { tab32[b * 4 + slot] = ent; return true; }
    if (slot == 3) { atomicOr(&tab32[b * 4 + 3], ent); return true; }
    atomicOr(&tab32[b * 4 + 3], 1u);       // bucket full: mark overflow
    b = (b + 1) & (NB - 1);
    return false;
}

// bit k set when slot k of bucket bv holds an entry whose fingerprint is key
__device__ __forceinline__ u32 bucket_match(const uint4 &bv, u32 key)
{
    u32 m = 0;
    m |= (((bv.x ^ key) < 0x10000u) & ((bv.x & 0xFFFEu) != 0)) ? 1u : 0u;
    m |= (((bv.y ^ key) < 0x10000u) & ((bv.y & 0xFFFEu) != 0)) ? 2u : 0u;
    m |= (((bv.z ^ key) < 0x10000u) & ((bv.z & 0xFFFEu) != 0)) ? 4u : 0u;
    m |= (((bv.w ^ key) < 0x10000u) & ((bv.w & 0xFFFEu) != 0)) ? 8u : 0u;
    return m;
}

__device__ __forceinline__ u32 slot_j(const uint4 &bv, int k)
{
    const u32 w = (k == 0) ? bv.x : (k == 1) ? bv.y : (k == 2) ? bv.z : bv.w;
    return ((w >> 1) & 0x7FFFu) - 1;
}

// Calls f(j) for every slot whose fingerprint matches val.  The common case
// (no match, bucket not flagged) is one 128-bit load, compares and one branch;
// matches and overflow chains take the out-of-line path.
template <u32 NBLOG, class F>
__device__ __forceinline__ void tab_probe(const uint4 *table, u64 val, F &&f)
{
    constexpr u32 NB = 1u << NBLOG;
    u32 b, key;
    tab_hash<NBLOG>(val, b, key);
    uint4 bv = table[b];
    u32 m = bucket_match(bv, key);
    if (__builtin_expect((m | (bv.w & 1u)) != 0, 0)) {
        for (int pr = 0; pr < BSGS_MAXPROBE; ++pr) {
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                f(slot_j(bv, k));
            }
            if (!(bv.w & 1u)) break;
            b = (b + 1) & (NB - 1);
            bv = table[b];
            m = bucket_match(bv, key);
        }
    }
}

// y -> y*s: doubling/quadrupling for b = 2 (the common case), additions for
// b^e <= 16, a Montgomery product otherwise (smul is uniform per prime)
__device__ __forceinline__ u64 baby_step(u64 x, u32 smul, u64 s, u64 p, u64 q)
{
    if (smul == 2) return madd(x, x, p);
    if (smul == 4) { x = madd(x, x, p); return madd(x, x, p); }
    return smul ? mul_small(x, smul, p) : mmul(x, s, p, q);
}

__device__ __forceinline__ void claim(const BsgsArgs &a, u64 p, u32 seq, u32 n, unsigned long long *s_dups,
                                      unsigned long long *s_facs)
{
    const u32 o = n - a.nmin;
    u32 *w = a.bitmap + (size_t)seq * a.words + (o >> 5);
    const u32 mask = 1u << (o & 31);
    const u32 old = atomicAnd(w, ~mask);
    if (old & mask) {
        const u32 f = atomicAdd(a.factor_ctr, 1u);
        atomicAdd(s_facs, 1ull);
        if (f < a.factor_cap) {
            FactorRec r;
            r.p = p; r.n = n; r.seq = seq;
            a.factors[f] = r;
        } else {
            atomicOr(a.err, ERR_FACTOR_OVERFLOW);
        }
    } else {
        atomicAdd(s_dups, 1ull);
    }
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
    unsigned char meta[KSTRIDE];
};
static_assert(sizeof(RecBuf) % 16 == 0, "bulk copies move 16-byte units");

constexpr u32 WAIT_BOUND = 1u << 24;   // try_wait rounds before a copy is declared lost

template <int TPB, int C, int NBLOG>
__global__ void __launch_bounds__(TPB, 1) k_bsgs(BsgsArgs a, const PrimeHdr *__restrict__ hdr,
                                                 const u64 *__restrict__ tabs, const u64 *__restrict__ tgt,
                                                 const unsigned char *__restrict__ meta, u32 count, u32 *work_ctr)
{
    constexpr u32 Q = TPB * C;
    constexpr u32 NB = 1u << NBLOG;
    constexpr int IB = 8;                                         // values inserted per batch
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint4 *table = reinterpret_cast<uint4 *>(smem_raw);
    u32 *tab32 = reinterpret_cast<u32 *>(table);
    u32 *s_cnt = reinterpret_cast<u32 *>(table + NB);             // NB 16-bit slot counters
    u64 *s_start = reinterpret_cast<u64 *>(s_cnt + NB / 2);
    u64 *s_Z = s_start + TPB;
    RecBuf *rec = reinterpret_cast<RecBuf *>(s_Z + TPB);          // two staging buffers
    __shared__ __align__(8) u64 s_bar[2];
    __shared__ unsigned long long s_cands, s_dups, s_facs;        // per-kernel totals
    __shared__ u32 s_idx[2], s_order, s_nsol, s_spill, s_abort;
    __shared__ u32 s_sol_i[KMAX], s_sol_u0[KMAX];

    const u32 tid = threadIdx.x;
    auto fetch = [&](u32 buf, u32 idx) {                          // thread 0 only
        RecBuf *r = &rec[buf];
        mbar_expect_tx(&s_bar[buf], (u32)sizeof(RecBuf));
        bulk_load(&r->hdr, hdr + idx, (u32)sizeof(PrimeHdr), &s_bar[buf]);
        bulk_load(r->tabs, tabs + (size_t)idx * TABS, TABS * 8, &s_bar[buf]);
        bulk_load(r->tgt, tgt + (size_t)idx * KSTRIDE, KSTRIDE * 8, &s_bar[buf]);
        bulk_load(r->meta, meta + (size_t)idx * KSTRIDE, KSTRIDE, &s_bar[buf]);
    };
    u64 st_baby = 0, st_giant = 0, st_small = 0;                  // thread 0's tallies
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_cands = 0;
        s_dups = 0;
        s_facs = 0;
        const u32 i0 = atomicAdd(work_ctr, 1u);
        s_idx[0] = i0;
        if (i0 < count) fetch(0, i0);
    }
    __syncthreads();

    for (u32 it = 0;; ++it) {
        const u32 buf = it & 1;
        const u32 idx = s_idx[buf];
        if (idx >= count) break;
        // this prime's record was fetched one prime ago; the wait is bounded
        {
            u32 n = 0;
            while (!mbar_try_wait(&s_bar[buf], (it >> 1) & 1)) {
                if (++n > WAIT_BOUND) { atomicOr(&s_abort, 1u); break; }
            }
        }
        // claim the next prime; the result is consumed after the table clear,
        // so this warp keeps issuing while the atomic is in flight
        u32 nxt = 0;
        if (tid == 0) {
            s_order = 0xFFFFFFFFu;
            s_nsol = 0;
            s_spill = 0;
            nxt = atomicAdd(work_ctr, 1u);
        }
        const RecBuf &R = rec[buf];
        const bool live = (R.hdr.p != 0);
        const u64 p = R.hdr.p, q = R.hdr.q, s = R.hdr.s;
        const u32 e = R.hdr.e, smul = R.hdr.smul;
        if (live)
            for (u32 i = tid; i < NB + NB / 8; i += TPB) table[i] = make_uint4(0u, 0u, 0u, 0u);   // table + counters
        __syncthreads();
        if (s_abort) break;
        if (tid == 0) {
            s_idx[buf ^ 1] = nxt;
            if (nxt < count) {                                    // rec[buf^1] was last read before the previous barrier
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                fetch(buf ^ 1, nxt);
            }
        }
        if (live) {
            if (tid < R.hdr.G) s_Z[tid] = mmul(R.tabs[64 + (tid & 31)], R.tabs[96 + (tid >> 5)], p, q);
            // ---- baby steps y_j = s^j, inserted as they are produced ----
            // Speculative: ord(s) < Q is only known after the barrier; then the
            // table (which may hold repeats) is rebuilt from j < ord below.
            const u64 one = R.hdr.one;
            u64 x = mmul(R.tabs[tid & 31], R.tabs[32 + (tid >> 5)], p, q);   // s^(C*tid)
            s_start[tid] = x;
            u32 spill = 0;
#pragma unroll
            for (int h0 = 0; h0 < C; h0 += IB) {
                u32 bk[IB], en[IB], old[IB];
#pragma unroll
                for (int i = 0; i < IB; ++i) {
                    const u32 j = tid * C + h0 + i;
                    if (j != 0 && x == one) atomicMin(&s_order, j);
                    u32 key;
                    tab_hash<NBLOG>(x, bk[i], key);
                    en[i] = key | ((j + 1) << 1);
                    x = baby_step(x, smul, s, p, q);
                }
#pragma unroll
                for (int i = 0; i < IB; ++i) old[i] = atomicAdd(&s_cnt[bk[i] >> 1], 1u << ((bk[i] & 1u) << 4));
#pragma unroll
                for (int i = 0; i < IB; ++i) {
                    const u32 slot = (old[i] >> ((bk[i] & 1u) << 4)) & 0xFFFFu;
                    if (slot < 3) tab32[bk[i] * 4 + slot] = en[i];
                    else if (slot == 3) atomicOr(&tab32[bk[i] * 4 + 3], en[i]);
                    else {
                        atomicOr(&tab32[bk[i] * 4 + 3], 1u);      // full: flag and try the next buckets
                        u32 b = (bk[i] + 1) & (NB - 1);
                        int pr = 1;
                        while (pr < BSGS_SPEC_PROBE && !tab_try<NBLOG>(tab32, s_cnt, b, en[i])) ++pr;
                        if (pr >= BSGS_SPEC_PROBE) spill = 1;
                    }
                }
            }
            if (spill) s_spill = 1;
        }
        __syncthreads();
        const u32 order = s_order;
        const u32 Mg = (e == 2) ? a.M2 : a.M1;
        if (live) {
            if (order < Q) {
                // ord(s) < Q: rebuild the table from the distinct values j < ord
                for (u32 i = tid; i < NB + NB / 8; i += TPB) table[i] = make_uint4(0u, 0u, 0u, 0u);
                __syncthreads();
                u64 y = s_start[tid];
                u32 pend = 0;
                for (int i = 0; i < C; ++i) {
                    const u32 j = tid * C + i;
                    if (j < order) {
                        u32 b, key;
                        tab_hash<NBLOG>(y, b, key);
                        int pr = 0;
                        while (pr < BSGS_MAXPROBE && !tab_try<NBLOG>(tab32, s_cnt, b, key | ((j + 1) << 1))) ++pr;
                        if (pr >= BSGS_MAXPROBE) pend = 1;
                    }
                    y = baby_step(y, smul, s, p, q);
                }
                if (pend) atomicOr(a.err, ERR_HASH_OVERFLOW);
                __syncthreads();
            } else if (tid == 0 && s_spill) {
                atomicOr(a.err, ERR_HASH_OVERFLOW);
            }

            // exact check of a fingerprint match: y_j == val ?
            auto verify = [&](u32 j, u64 val) -> bool {
                if (j >= Q) return false;
                u64 y = s_start[j / C];
                for (u32 r = j % C; r; --r) y = baby_step(y, smul, s, p, q);
                return y == val;
            };

            if (order == 0xFFFFFFFFu) {
                // ---- giant steps: two independent chains per thread ----
                // chain A walks q in [q0, q0+h), chain B q in [q0+h, q1), h = Lc/2;
                // B starts from A's start times S^h (Sh), so the two Montgomery
                // products of a step are independent and overlap in the pipeline.
                const u32 numk = R.hdr.numk, G = R.hdr.G, Lc = R.hdr.Lc;
                const u64 S = R.hdr.S;
                if (tid < numk * G) {
                    const u32 i = tid / G, g = tid - i * G;
                    const u32 q0 = g * Lc;
                    const u32 q1 = min(q0 + Lc, Mg);
                    const u32 h = Lc >> 1;
                    const u32 nA = min(h, q1 - q0), nB = (q1 - q0) - nA;
                    const u32 m = R.meta[i];
                    const u32 seq = m & 0x7Fu, off = m >> 7;
                    u64 gA = mmul(R.tgt[i], s_Z[g], p, q);
                    u64 gB = mmul(gA, R.hdr.Sh, p, q);
                    auto hit = [&](u32 qq, u32 j, u64 gamma) {
                        atomicAdd(&s_cands, 1ull);
                        if (!verify(j, gamma)) return;
                        const u64 u = (u64)(qq + 1) * Q - 1 - j;
                        const u64 n = (u64)a.nmin + off + (u64)e * u;
                        if (n <= a.nmax) claim(a, p, seq, (u32)n, &s_dups, &s_facs);
                    };
                    for (u32 t = 0; t < nB; ++t) {
                        if (t < nA) {
                            const u32 qa = q0 + t;
                            const u64 ga = gA;
                            tab_probe<NBLOG>(table, ga, [&](u32 j) { hit(qa, j, ga); });
                            gA = mmul(gA, S, p, q);
                        }
                        const u32 qb = q0 + h + t;
                        const u64 gb = gB;
                        tab_probe<NBLOG>(table, gb, [&](u32 j) { hit(qb, j, gb); });
                        gB = mmul(gB, S, p, q);
                    }
                }
            } else {
                // ---- ord(s) < Q: one lookup per target ----
                if (tid < R.hdr.numk) {
                    const u64 T = R.tgt[tid];
                    tab_probe<NBLOG>(table, T, [&](u32 j) {
                        atomicAdd(&s_cands, 1ull);
                        if (j >= order || !verify(j, T)) return;
                        const u32 k = atomicAdd(&s_nsol, 1u);
                        s_sol_i[k] = tid;
                        s_sol_u0[k] = (Q - 1 - j) % order;
                    });
                }
                __syncthreads();
                const u32 nsol = s_nsol;
                for (u32 k = 0; k < nsol; ++k) {
                    const u32 i = s_sol_i[k];
                    const u32 m = R.meta[i];
                    const u32 seq = m & 0x7Fu, off = m >> 7;
                    for (u64 u = s_sol_u0[k] + (u64)tid * order;; u += (u64)TPB * order) {
                        const u64 n = (u64)a.nmin + off + (u64)e * u;
                        if (n > a.nmax) break;
                        claim(a, p, seq, (u32)n, &s_dups, &s_facs);
                    }
                }
            }
            if (tid == 0) {
                st_baby += min(order, Q);
                if (order == 0xFFFFFFFFu) st_giant += (u64)R.hdr.numk * Mg;
                else st_small += 1;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        atomicAdd(&a.stats[ST_BABY], st_baby);
        atomicAdd(&a.stats[ST_GIANT], st_giant);
        atomicAdd(&a.stats[ST_SMALLORDER], st_small);
        atomicAdd(&a.stats[ST_CANDIDATES], s_cands);
        atomicAdd(&a.stats[ST_DUPS], s_dups);
        atomicAdd(&a.stats[ST_FACTORS], s_facs);
        atomicAdd(&a.stats[ST_HITS], s_dups + s_facs);
    }
    if (s_abort) {
        // a record copy never completed: report, then give copies in flight a bounded chance to land
        if (tid == 0) atomicOr(a.err, ERR_TMA_TIMEOUT);
        for (int b = 0; b < 2; ++b) {
            u32 n = 0;
            while (n < WAIT_BOUND && !mbar_try_wait(&s_bar[b], 0) && !mbar_try_wait(&s_bar[b], 1)) ++n;
        }
    }
}

size_t bsgs_smem_bytes()
{
    constexpr size_t NB = 1u << BSGS_NBLOG;
    return NB * 16 + NB * 2 + BSGS_TPB * 8 * 2 + 2 * sizeof(RecBuf);
}

cudaError_t bsgs_prepare()
{
    return cudaFuncSetAttribute(k_bsgs<BSGS_TPB, BSGS_C, BSGS_NBLOG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bsgs_smem_bytes());
}

cudaError_t launch_bsgs(const BsgsArgs &a, const PrimeHdr *hdr, const u64 *tabs, const u64 *tgt,
                        const unsigned char *meta, u32 count, u32 *work_ctr, int sms, cudaStream_t st)
{
    if (count == 0) return cudaSuccess;
    auto kern = k_bsgs<BSGS_TPB, BSGS_C, BSGS_NBLOG>;
    const size_t smem = bsgs_smem_bytes();
    unsigned grid = ((u32)sms < count) ? (unsigned)sms : (unsigned)count;
    kern<<<grid, BSGS_TPB, smem, st>>>(a, hdr, tabs, tgt, meta, count, work_ctr);
    return cudaGetLastError();
}

}  // namespace rs

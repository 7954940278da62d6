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
// Hash table: NB buckets of four 32-bit slots in shared memory (load 1/2).
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

template <u32 NBLOG>
__device__ __forceinline__ void tab_insert(uint4 *table, u64 val, u32 j, u32 *err)
{
    constexpr u32 NB = 1u << NBLOG;
    u32 b, key;
    tab_hash<NBLOG>(val, b, key);
    const u32 ent = key | ((j + 1) << 1);
    for (int pr = 0; pr < BSGS_MAXPROBE;) {
        u32 *sl = reinterpret_cast<u32 *>(&table[b]);
        u32 cur[4];
        asm volatile("ld.volatile.shared.v4.u32 {%0,%1,%2,%3}, [%4];"
                     : "=r"(cur[0]), "=r"(cur[1]), "=r"(cur[2]), "=r"(cur[3])
                     : "r"((u32)__cvta_generic_to_shared(sl)));
        int k = 0;
        while (k < 4 && (cur[k] >> 1) != 0) ++k;
        if (k < 4) {
            // slots only ever fill, so a stale 'empty' just fails the CAS; re-read then
            if (atomicCAS(&sl[k], cur[k], cur[k] | ent) == cur[k]) return;
            continue;
        }
        atomicOr(&sl[3], 1u);                // bucket full: mark overflow, go on
        b = (b + 1) & (NB - 1);
        ++pr;
    }
    atomicOr(err, ERR_HASH_OVERFLOW);
}

// Calls f(j) for every slot whose fingerprint matches val.
template <u32 NBLOG, class F>
__device__ __forceinline__ void tab_probe(const uint4 *table, u64 val, F &&f)
{
    constexpr u32 NB = 1u << NBLOG;
    u32 b, key;
    tab_hash<NBLOG>(val, b, key);
    for (int pr = 0; pr < BSGS_MAXPROBE; ++pr) {
        const uint4 bv = table[b];
        if (((bv.x ^ key) < 0x10000u) && (bv.x & 0xFFFEu)) f(((bv.x >> 1) & 0x7FFFu) - 1);
        if (((bv.y ^ key) < 0x10000u) && (bv.y & 0xFFFEu)) f(((bv.y >> 1) & 0x7FFFu) - 1);
        if (((bv.z ^ key) < 0x10000u) && (bv.z & 0xFFFEu)) f(((bv.z >> 1) & 0x7FFFu) - 1);
        if (((bv.w ^ key) < 0x10000u) && (bv.w & 0xFFFEu)) f(((bv.w >> 1) & 0x7FFFu) - 1);
        if (!(bv.w & 1u)) break;
        b = (b + 1) & (NB - 1);
    }
}

__device__ __forceinline__ u64 baby_step(u64 x, u32 smul, u64 s, u64 p, u64 q)
{
    return smul ? mul_small(x, smul, p) : mmul(x, s, p, q);
}

__device__ __forceinline__ void claim(const BsgsArgs &a, u64 p, u32 seq, u32 n, u32 *s_dups, u32 *s_facs)
{
    const u32 o = n - a.nmin;
    u32 *w = a.bitmap + (size_t)seq * a.words + (o >> 5);
    const u32 mask = 1u << (o & 31);
    const u32 old = atomicAnd(w, ~mask);
    if (old & mask) {
        const u32 f = atomicAdd(a.factor_ctr, 1u);
        atomicAdd(s_facs, 1u);
        if (f < a.factor_cap) {
            FactorRec r;
            r.p = p; r.n = n; r.seq = seq;
            a.factors[f] = r;
        } else {
            atomicOr(a.err, ERR_FACTOR_OVERFLOW);
        }
    } else {
        atomicAdd(s_dups, 1u);
    }
}

template <int TPB, int C, int NBLOG>
__global__ void __launch_bounds__(TPB, 1) k_bsgs(BsgsArgs a, const PrimeHdr *__restrict__ hdr,
                                                 const u64 *__restrict__ tabs, const u64 *__restrict__ tgt,
                                                 const unsigned char *__restrict__ meta, u32 count, u32 *work_ctr)
{
    constexpr u32 Q = TPB * C;
    constexpr u32 NB = 1u << NBLOG;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *table = reinterpret_cast<uint4 *>(smem_raw);
    u64 *s_start = reinterpret_cast<u64 *>(table + NB);
    u64 *s_T = s_start + TPB;
    u64 *s_Z = s_T + KSTRIDE;
    unsigned char *s_meta = reinterpret_cast<unsigned char *>(s_Z + TPB);
    __shared__ u32 s_idx, s_order, s_dups, s_cands, s_nsol, s_facs;
    __shared__ u32 s_sol_i[KMAX], s_sol_u0[KMAX];

    const u32 tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            s_idx = atomicAdd(work_ctr, 1u);
            s_order = 0xFFFFFFFFu;
            s_dups = 0;
            s_cands = 0;
            s_nsol = 0;
            s_facs = 0;
        }
        __syncthreads();
        const u32 idx = s_idx;
        if (idx >= count) break;
        const PrimeHdr H = hdr[idx];
        if (H.p == 0) {
            __syncthreads();
            continue;
        }
        const u64 p = H.p, q = H.q, one = H.one, s = H.s, S = H.S;
        const u32 numk = H.numk, e = H.e, smul = H.smul;
        const u64 *tb = tabs + (size_t)idx * TABS;

        for (u32 i = tid; i < NB; i += TPB) table[i] = make_uint4(0u, 0u, 0u, 0u);
        for (u32 i = tid; i < numk; i += TPB) {
            s_T[i] = tgt[(size_t)idx * KSTRIDE + i];
            s_meta[i] = meta[(size_t)idx * KSTRIDE + i];
        }
        if (tid < H.G) s_Z[tid] = mmul(tb[64 + (tid & 31)], tb[96 + (tid >> 5)], p, q);

        // ---- baby steps ----
        u64 v[C];
        v[0] = mmul(tb[tid & 31], tb[32 + (tid >> 5)], p, q);   // s^(C*tid)
        s_start[tid] = v[0];
#pragma unroll
        for (int i = 1; i < C; ++i) v[i] = baby_step(v[i - 1], smul, s, p, q);
#pragma unroll
        for (int i = 0; i < C; ++i) {
            const u32 j = tid * C + i;
            if (j != 0 && v[i] == one) atomicMin(&s_order, j);
        }
        __syncthreads();
        const u32 order = s_order;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            const u32 j = tid * C + i;
            if (j < order) tab_insert<NBLOG>(table, v[i], j, a.err);
        }
        __syncthreads();

        // exact check of a fingerprint match: y_j == val ?
        auto verify = [&](u32 j, u64 val) -> bool {
            if (j >= Q) return false;
            u64 y = s_start[j / C];
            for (u32 r = j % C; r; --r) y = baby_step(y, smul, s, p, q);
            return y == val;
        };

        const u32 Mg = (e == 2) ? a.M2 : a.M1;
        if (order == 0xFFFFFFFFu) {
            // ---- giant steps: two independent chains per thread ----
            // chain A walks q in [q0, q0+h), chain B q in [q0+h, q1), h = Lc/2;
            // B starts from A's start times S^h (H.Sh), so the two Montgomery
            // products of a step are independent and overlap in the pipeline.
            const u32 G = H.G, Lc = H.Lc;
            if (tid < numk * G) {
                const u32 i = tid / G, g = tid - i * G;
                const u32 q0 = g * Lc;
                const u32 q1 = min(q0 + Lc, Mg);
                const u32 h = Lc >> 1;
                const u32 nA = min(h, q1 - q0), nB = (q1 - q0) - nA;
                const u32 m = s_meta[i];
                const u32 seq = m & 0x7Fu, off = m >> 7;
                u64 gA = mmul(s_T[i], s_Z[g], p, q);
                u64 gB = mmul(gA, H.Sh, p, q);
                auto hit = [&](u32 qq, u32 j, u64 gamma) {
                    atomicAdd(&s_cands, 1u);
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
            if (tid < numk) {
                const u64 T = s_T[tid];
                tab_probe<NBLOG>(table, T, [&](u32 j) {
                    atomicAdd(&s_cands, 1u);
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
                const u32 m = s_meta[i];
                const u32 seq = m & 0x7Fu, off = m >> 7;
                for (u64 u = s_sol_u0[k] + (u64)tid * order;; u += (u64)TPB * order) {
                    const u64 n = (u64)a.nmin + off + (u64)e * u;
                    if (n > a.nmax) break;
                    claim(a, p, seq, (u32)n, &s_dups, &s_facs);
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            atomicAdd(&a.stats[ST_BABY], (u64)min(order, Q));
            if (order == 0xFFFFFFFFu) atomicAdd(&a.stats[ST_GIANT], (u64)numk * Mg);
            else atomicAdd(&a.stats[ST_SMALLORDER], 1ull);
            if (s_cands) atomicAdd(&a.stats[ST_CANDIDATES], (u64)s_cands);
            if (s_dups) atomicAdd(&a.stats[ST_DUPS], (u64)s_dups);
            if (s_facs) atomicAdd(&a.stats[ST_FACTORS], (u64)s_facs);
            if (s_dups + s_facs) atomicAdd(&a.stats[ST_HITS], (u64)(s_dups + s_facs));
        }
    }
}

size_t bsgs_smem_bytes()
{
    constexpr size_t NB = 1u << BSGS_NBLOG;
    return NB * 16 + BSGS_TPB * 8 + KSTRIDE * 8 + BSGS_TPB * 8 + KSTRIDE;
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

// rs_internal.h -- device data layout shared by the kernels and the engine.
//
// Per job (a set of <= 100 sequences k_i*b^n+c_i sharing b, and an n-range)
// the device holds a JobDev descriptor, the candidate bitmap and a factor
// buffer.  Per segment of the p-range the device holds the generated primes;
// per chunk of primes the setup kernel writes one record per prime (header,
// power tables, BSGS targets) that the BSGS kernel consumes.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace rs {

typedef unsigned long long u64;
typedef unsigned int u32;
typedef unsigned char u8;

constexpr int KMAX = 100;            // sequences per job (inputfile.cpp:356-361)
constexpr int KSTRIDE = 112;         // padded per-prime target stride (16-byte multiple for bulk copies)
constexpr int TABS = 128;            // u64 power-table entries per prime

// BSGS kernel geometries: Q = tpb * c baby steps per prime, nb buckets of
// seven slots (load about 0.4), 1024 / tpb CTAs per SM sharing its 228 KB of
// shared memory.  The giant phase needs tpb >= KMAX (one thread per target).
struct BsgsGeom {
    u32 q, tpb, c, nb;
};
constexpr int NGEOM = 5;
constexpr BsgsGeom BSGS_GEOMS[NGEOM] = {
    {16384, 1024, 16, 6144},   // 1 CTA per SM
    {8192, 512, 16, 2944},     // 2
    {4096, 256, 16, 1376},     // 4 (with the 2.2 KB record buffers, 1408 buckets would leave room for 3)
    {2048, 256, 8, 704},       // 4
    {1024, 128, 8, 352},       // 8
};
constexpr int geom_index(u32 q)
{
    return q == 16384 ? 0 : q == 8192 ? 1 : q == 4096 ? 2 : q == 2048 ? 3 : q == 1024 ? 4 : -1;
}

// Model cost of one prime for a geometry, in baby-step units: Q baby steps plus
// the giant steps of the targets that survive the prefilter (about 0.6 of the
// sequences), each over one class of n modulo the prime's split modulus e
// (ceil(L/(eQ)) steps, about 0.15 L/Q on average over primes, and at least
// one), a giant step costing about 1.2 baby steps, and the per-prime fixed
// work (table clear, barriers) of about 0.15 Q.
inline double geom_model_cost(int g, u32 kcount, u32 L)
{
    const double q = BSGS_GEOMS[g].q;
    const double m = 0.15 * (double)L / q + 0.5;
    return 1.15 * q + 1.2 * 0.6 * kcount * (m < 1.0 ? 1.0 : m);
}
inline int geom_model_best(u32 kcount, u32 L)
{
    int best = 0;
    for (int g = 1; g < NGEOM; ++g)
        if (geom_model_cost(g, kcount, L) < geom_model_cost(best, kcount, L)) best = g;
    return best;
}
// Measured geometries per device and job shape (base, kcount, L), shared by the
// single-job contexts and the batches of the process; -1 when none is recorded.
inline u64 job_shape_key(u32 base, u32 kcount, u32 L)
{
    return ((u64)base << 40) ^ ((u64)kcount << 32) ^ (u64)L;
}
int tuned_geom_get(int device, u64 shape);
void tuned_geom_put(int device, u64 shape, int geom);
constexpr int BSGS_MAXPROBE = 64;
constexpr int BSGS_SPEC_PROBE = 64;         // bucket walk bound while ord(s) is still unknown

constexpr int SETUP_TPB = 256;              // 8 primes (warps) per block
constexpr int SIEVE_TPB = 512;
constexpr int SIEVE_WORDS = 4096;           // 2^17 odd numbers per sieve block
constexpr u64 MR_BOUND = 4295098369ULL;     // 65537^2: below it the sieve by all primes < 2^16 is exact

// error bits (JobDev-independent, one word per context)
constexpr u32 ERR_PRIME_OVERFLOW = 1u;      // segment produced more primes than the buffer holds
constexpr u32 ERR_CAND_OVERFLOW = 2u;
constexpr u32 ERR_HASH_OVERFLOW = 4u;       // a bucket chain exceeded BSGS_MAXPROBE
constexpr u32 ERR_FACTOR_OVERFLOW = 8u;     // factor buffer full (cannot happen: sized to the bitmap)
constexpr u32 ERR_TMA_TIMEOUT = 16u;        // a bulk copy did not complete within the wait bound
constexpr u32 ERR_SIEVE_TABLE = 32u;        // the sieving-prime table is missing (does not start with 3)
constexpr u32 ERR_SETUP_CLASS = 64u;        // a target passed the residue test but no class of n matched (cannot happen)

// statistics counters (u64)
enum Stat {
    ST_PRIMES = 0,        // primes generated (and tested)
    ST_SKIPPED,           // primes dividing b or some k, or with no solvable k (setup.cl:156-162,205-208)
    ST_FULL,              // primes searched over every n (split modulus e = 1)
    ST_PARITY,            // primes searched over one class of n mod e per sequence (e >= 2; e = 2: parity)
    ST_TARGETS,           // sum over primes of surviving k
    ST_BABY,              // baby steps executed
    ST_GIANT,             // giant steps executed (one Montgomery product and one lookup each)
    ST_SMALLORDER,        // primes with ord(b^e) < Q
    ST_CANDIDATES,        // fingerprint matches verified
    ST_HITS,              // verified solutions p | k*b^n+c with n in range
    ST_FACTORS,           // bitmap claims won
    ST_DUPS,              // solutions whose bitmap bit was already clear
    ST_SIEVE_CANDS,       // sieve survivors given to Miller-Rabin
    ST_COUNT
};

struct JobDev {
    u32 base, kcount, nmin, nmax;
    u32 L;               // nmax - nmin + 1
    u32 words;           // bitmap words per sequence
    u64 k[KMAX];
    int c[KMAX];
    u32 *bitmap;         // kcount * words
};

// Below FP_BOUND = 2^51 the BSGS steps run on the FP64 pipe (fp_mulfix in
// mont.cuh): residues are exact integers in doubles, and a product by a fixed
// multiplier w takes its quotient from the double w/p.
constexpr u64 FP_BOUND = 1ull << 51;
// The set-up's chi chains (products of two variable factors, fp_mul) run on
// the FP64 pipe below FP_BOUND as well.

struct PrimeHdr {        // 128 bytes (a 16-byte multiple: copied by TMA bulk copies)
    u64 p;               // 0 = skipped
    u64 q;               // p^-1 mod 2^64
    u64 one;             // 2^64 mod p
    u64 s;               // Montgomery b^e, e = the split modulus (n runs over one class mod e per target)
    u64 S;               // Montgomery s^Q' (Q' = this prime's baby-step count), for p >= 2^63; below
                         // FP_BOUND the bits of the double sp/p (FP64 baby steps)
    u32 numk;            // surviving targets
    u32 e;               // split modulus, 1..64
    u32 G, Lc;           // giant phase: G chunks of Lc giant steps
    u32 smul;            // b^e as an integer when the baby step uses additions, else 0
    u32 job;             // job index within a batch (0 for a single job)
    u32 Mg;              // giant steps per target: ceil(ceil(L/e)/Q'), Q' = TPB*cp
    u32 cp;              // baby steps per thread for this prime (C, C/2 or C/4 of the launch's geometry)
    u64 Sh;              // Montgomery S^(Lc/2): start of a thread's second giant chain
    u64 Sw;              // floor(Sp*2^64/p), Sp = s^Q' mod p (plain), for Shoup giant steps; 0 when p >= 2^63
    u64 ssw;             // floor(sp*2^64/p), sp = s mod p (plain), for Shoup baby steps; 0 when p >= 2^63
    u64 sp, Sp;          // s and s^Q' as plain residues, the Shoup multipliers (0 when p >= 2^63)
    u64 u2;              // Montgomery s^(cp/2): start offset of a thread's second baby chain
    u64 Sq;              // below FP_BOUND: the bits of the double Sp/p (FP64 giant steps); else 0
};
static_assert(sizeof(PrimeHdr) == 128, "PrimeHdr is copied in 16-byte units");

struct FactorRec {       // one claimed term: p | k[seq]*b^n + c[seq]
    u64 p;
    u32 n;
    u32 seq;
};

struct BsgsArgs {
    u32 base, nmin, nmax, words;
    u32 *bitmap;
    FactorRec *factors;
    u32 *factor_ctr;
    u32 factor_cap;
    u64 *stats;
    u32 *err;
    u32 wait_bound;      // try_wait rounds before a record copy counts as lost (0: WAIT_BOUND)
    u32 test_stall;      // 1: each CTA's first record wait is on a barrier that nothing completes
};

// ---- batches: many jobs, each with one or more p-ranges, advanced in rounds ----
// A range's window of one round, written on the device by k_batch_windows.
struct BatchWin {
    u64 lo, hi;          // this round's [lo, hi) (lo == hi: the range is done)
    u64 base_odd, nodd;  // odd values base_odd + 2i, i < nodd, covering [lo, hi)
};
struct BatchRange {      // device state of one range slot
    u64 p_cur, p_end;    // next window start, end of the range
    u32 job;             // job slot it belongs to
    u8 active;           // slot in use
    u8 mode;             // BSGS step kind: 2 p_end <= 2^51 (FP64), 1 p_end <= 2^63 (Shoup), 0 p >= 2^63
    u8 geom;             // BSGS geometry index of its job
    u8 pad_;
};
// per-range counters of a round: [0] sieve survivors, [1] primes, [2] pad, [3] pad
constexpr int BR_CTRS = 4;
// per-job BSGS geometry as the set-up kernels need it
struct JobGeom {
    u32 q, c, tpb, pad_;
};
inline JobGeom job_geom(int g)
{
    JobGeom G;
    G.q = BSGS_GEOMS[g].q;
    G.c = BSGS_GEOMS[g].c;
    G.tpb = BSGS_GEOMS[g].tpb;
    G.pad_ = 0;
    return G;
}

// Index i of work spread over nr ranges with prefix sums prefix[0..nr]:
// the range k with prefix[k] <= i < prefix[k+1] (i < prefix[nr]).
__device__ __forceinline__ u32 prefix_find(const u32 *prefix, u32 nr, u32 i)
{
    u32 lo = 0, hi = nr;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (prefix[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// launch wrappers (sieve.cu, setup.cu, bsgs.cu)
cudaError_t launch_sieve(u64 base_odd, u64 nodd, u64 hi, const u32 *sp, u32 nsp, u64 *cands, u32 cand_cap,
                         u32 *ctrs, u32 *err, cudaStream_t st);
cudaError_t launch_mr(const u64 *cands, const u32 *ctrs, u32 cand_cap, u64 *primes, u32 prime_cap, u32 *prime_ctr,
                      u32 *err, int sms, cudaStream_t st);
// the same test in two passes (base 2 into mid, then Lucas over mid); mid
// holds cand_cap values and *mid_ctr starts at zero
cudaError_t launch_mr2(const u64 *cands, const u32 *ctrs, u32 cand_cap, u64 *primes, u32 prime_cap, u32 *prime_ctr,
                       u64 *mid, u32 *mid_ctr, u32 *err, int sms, cudaStream_t st);
cudaError_t launch_setup(const JobDev *job, const u64 *primes, u32 first, u32 count, PrimeHdr *hdr, void *aux, u64 *tabs,
                         u64 *tgt, unsigned short *meta, u64 *stats, u32 *err, int geom, cudaStream_t st);
size_t setup_aux_bytes();
// every prime of the launch lies in [pmin, pmax), entirely below or entirely at or above 2^63
cudaError_t launch_bsgs(const BsgsArgs &a, const PrimeHdr *hdr, const u64 *tabs, const u64 *tgt,
                        const unsigned short *meta, u32 count, u32 *work_ctr, u64 pmin, u64 pmax, int geom, int sms,
                        cudaStream_t st);
size_t bsgs_smem_bytes(int geom);
cudaError_t bsgs_prepare();   // per device, before the first launch
cudaError_t launch_mulmod_peak(u64 *out, int blocks, int iters, cudaStream_t st);
cudaError_t launch_widemul_peak(u64 *out, int blocks, int iters, cudaStream_t st);
cudaError_t launch_fpmul_peak(u64 *out, int blocks, int iters, cudaStream_t st);

// batch rounds (sieve.cu, setup.cu, bsgs.cu)
// win[r]: primes range slot r should cover this round (0: none); capped at 0.6*rcap
cudaError_t launch_batch_windows(BatchRange *ranges, BatchWin *wins, const u32 *win, u32 nranges, u32 rcap, u32 *ctrs,
                                 cudaStream_t st);
cudaError_t launch_sieve_batch(const BatchWin *wins, u32 nranges, u32 max_blocks, const u32 *sp, u32 nsp, u64 *cands,
                               u32 ccap, u32 *ctrs, u32 *err, cudaStream_t st);
// Baillie-PSW over the survivors of all ranges (prefix_c: their counts'
// prefix sums) in two passes: base-2 strong probable primes of every range
// (value and range) into mid, then the Lucas test over it; primes go to their
// range's slots; *mid_ctr starts at zero
cudaError_t launch_mr_batch2(const u64 *cands, u32 ccap, u64 *primes, u32 rcap, u32 *ctrs, u32 nranges,
                             const u32 *prefix_c, u64 *mid, u32 *mid_r, u32 mid_cap, u32 *mid_ctr, u32 *err, int sms,
                             cudaStream_t st);
// set-up of the primes of all ranges (prefix_p: prefix sums of their counts;
// rec_of: room for one record index per prime, nranges * rcap)
cudaError_t launch_setup_batch(const JobDev *jobs, const JobGeom *geoms, const BatchRange *ranges, const u64 *primes,
                               u32 rcap, const u32 *prefix_p, u32 nranges, PrimeHdr *hdr, void *aux, u64 *tabs,
                               u64 *tgt, unsigned short *meta, u64 *stats, u32 *err, u32 *rec_of, int sms,
                               cudaStream_t st);
// one BSGS launch per (geometry, mode) group g = 3*geometry + mode over range
// slots [0, nr): prefix + g*(nr+1) (nr+1 entries) counts the primes of the
// active slots of that group only; work[g] is cleared
cudaError_t launch_batch_group_prefix(const BatchRange *ranges, u32 nr, const u32 *ctrs, u32 rcap, u32 *prefix,
                                      u32 *work, cudaStream_t st);
// prefix over every active range of counter `which` (0: survivors, 1: primes), each capped at cap
cudaError_t launch_batch_prefix_all(const BatchRange *ranges, u32 nr, int which, u32 cap, const u32 *ctrs,
                                    u32 *prefix, cudaStream_t st);
cudaError_t launch_bsgs_batch(const BsgsArgs &a, const BsgsArgs *job_args, const PrimeHdr *hdr, const u64 *tabs,
                              const u64 *tgt, const unsigned short *meta, u32 nr, const u32 *prefix, u32 rcap,
                              u32 *work_ctr, int mode, int geom, int sms, cudaStream_t st);

}  // namespace rs

// host helpers shared by engine.cu and batch.cu
struct rs_seqs;
std::vector<rs::u32> rs_small_primes();                       // odd primes below 2^16, ascending
void jobdev_from_seqs(const rs_seqs *s, rs::JobDev *out);    // JobDev of a job (bitmap pointer null)

/*
 * rsoracle.h -- CPU oracle for the RSSieve BSGS sieve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is loaded by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by
 * nothing else.  The product (rssieve_b200/) never links or calls it.
 *
 * It restates, in plain C, the algorithm of the reference (mfl0p/RSSieve):
 *   - 64-bit Montgomery arithmetic           kernels/common.cl:24-176
 *   - the 2-PRP prime generator              kernels/getsegprimes.cl:37-182,
 *                                            kernels/addsmallprimes.cl:8-27,
 *                                            cl_sieve.cpp:453-512 (wheel offset)
 *   - per-prime setup + prefilter            kernels/setup.cl:11-209
 *   - parity sort / BSGS constants           kernels/sort.cl:11-104
 *   - BSGS giant kernels + bitmap claims     kernels/giant.cl:21-323
 *   - Q/HSIZE/M/QQ/MM parameter rule         cl_sieve.cpp:885-938
 *   - CPU factor verification                verify_factor.c:14-181
 * plus two independent checkers that share no code path with the BSGS port:
 *   - a segmented sieve + 7-base Miller-Rabin true-prime generator, and
 *   - a brute-force term oracle that steps b^n mod p over every n.
 *
 * k is widened from the reference's int (k < 2^31, inputfile.cpp:366) to u64.
 */
#ifndef RSORACLE_H
#define RSORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAX_SEQ 100

typedef struct {
    uint32_t base;              /* b, one base for all sequences            */
    uint32_t kcount;            /* number of sequences (<= 100)             */
    uint32_t nmin, nmax;        /* global n range, nmin even                */
    uint32_t words_per_seq;     /* ceil((nmax-nmin+1)/32)                    */
    uint64_t k[OR_MAX_SEQ];     /* k_i > 0                                   */
    int32_t  c[OR_MAX_SEQ];     /* c_i = +1 or -1                            */
    uint32_t *bitmap;           /* kcount*words_per_seq, 1 = live candidate  */
} or_job;

typedef struct {
    uint64_t p;
    uint32_t n;
    uint32_t seq;               /* index into k[]/c[]                        */
} or_factor;

/* ---- arithmetic (common.cl) ---- */
uint64_t or_invert(uint64_t p);
uint64_t or_m_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t q);
uint64_t or_add(uint64_t a, uint64_t b, uint64_t p);
uint64_t or_powmod(uint64_t mbase, uint64_t exp, uint64_t p, uint64_t q, uint64_t one);

/* ---- primes ---- */
int    or_is_prime(uint64_t n);     /* 7-base SPRP test of verify_factor.c:100-128 */
int    or_sprp2(uint64_t n);        /* strong base-2 PRP test, getsegprimes.cl:37-66 */
size_t or_primes(uint64_t lo, uint64_t hi, uint64_t *out, size_t cap);  /* true odd primes in [lo,hi) */
size_t or_prp2(uint64_t lo, uint64_t hi, uint64_t *out, size_t cap);    /* reference prime set in [lo,hi) */

/* ---- verify (verify_factor.c:131-181): 1 = factor, 0 = not a factor, -1 = p composite ---- */
int or_verify_factor(uint64_t p, uint64_t k, uint32_t n, int32_t c, uint32_t base);

/* ---- brute-force term oracle ----
 * For every prime (run in parallel) and every n in [nmin,nmax] it
 * evaluates b^n mod p and claims the bitmap bit of every term p | k*b^n+c.
 * ref_skip != 0 applies the reference's rule that a prime dividing b or any k
 * is skipped for all sequences (setup.cl:156-162).
 * Returns the number of factors written (claims); *dups counts hits on
 * in-range terms whose bit was already clear. */
size_t or_brute(or_job *job, const uint64_t *primes, size_t np, int ref_skip,
                or_factor *out, size_t cap, uint64_t *dups);

/* ---- reference parameter rule (cl_sieve.cpp:893-938, NVIDIA 48 KB local memory) ---- */
typedef struct { uint32_t Q, hsize, m, QQ, mm; } or_params;
or_params or_ref_params(uint32_t nmin, uint32_t nmax);

/* ---- reference setup+sort restated, for comparison with the compiled reference ----
 * For each prime: row[8] after setup (row[0]==0 => skipped) and per-k
 * (hadj, parity, kidx) packed in the order setup.cl writes them (kidx descending),
 * terminated by parity==0 when fewer than kcount survive. */
typedef struct { uint64_t hadj; int32_t parity; int32_t kidx; } or_kdata;
void or_setup(const or_job *job, uint32_t Q, const uint64_t *primes, size_t np,
              uint64_t *rows /* np*8 */, or_kdata *kd /* np*kcount */);

/* ---- CPU port of the reference BSGS pipeline (setup -> sort -> giantfull/giantparity) ----
 * primes: any order.  Claims follow giant.cl (first claimer wins on the bitmap).
 * nthreads <= 1 runs the primes in the given order on one thread (deterministic).
 * dup_ref counts duplicates exactly as giant.cl:163,187,195-196 does (including hits
 * above nmax that fall inside the reference's M*Q coverage); dup_inrange only
 * counts hits with n in [nmin,nmax].  Returns the number of factors written. */
typedef struct { uint64_t mulmods; uint64_t lookups; uint64_t dup_ref; uint64_t dup_inrange; uint64_t skipped; } or_stats;
size_t or_bsgs(or_job *job, const uint64_t *primes, size_t np, int nthreads,
               or_factor *out, size_t cap, or_stats *stats);

/* ---- host result handling restated from cl_sieve.cpp:515-643 ----
 * Sorts factors by (p,n), verifies each, drops composite p, and returns the
 * number kept (compacted in place).  *false_factor set if any verify failed. */
size_t or_verify_and_sort(const or_job *job, or_factor *f, size_t nf, int *false_factor, uint64_t *checksum);

/* ---- test-input helper (not a restatement) ----
 * First n in [n_lo, n_hi) whose k = -c*b^-n mod p is below kmax with parity
 * par (0 even, 1 odd, -1 any): then p | k*b^n+c.  Returns 1 and fills
 * *k_out, *n_out, or 0 when there is none. */
int or_plant(uint64_t p, uint32_t b, int32_t c, uint32_t n_lo, uint32_t n_hi, uint64_t kmax, int par,
             uint64_t *k_out, uint32_t *n_out);

#ifdef __cplusplus
}
#endif
#endif

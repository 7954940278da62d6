/*
 * rssieve_b200.h -- C ABI of the B200 RSSieve sieve library.
 *
 * The reference (mfl0p/RSSieve) has no plugin or FFI API: it is a process
 * (main.cpp) whose hot path lives in cl_sieve.cpp + simpleCL.c and a set of
 * OpenCL kernels.  This header is the seam that replaces that internal layer:
 * plain C types, caller-owned host buffers, library-owned device memory, one
 * CUDA device per context, every entry point returns an error code (never
 * exits).  A context is not reentrant; use one per host thread.
 *
 * Terms are k*b^n + c with c = +1 or -1; "seq" indexes the sequences of a job.
 * k is 64-bit here (the reference stores it as int, inputfile.cpp:366).
 */
#ifndef RSSIEVE_B200_H
#define RSSIEVE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RS_MAX_SEQ 100          /* MAX_SEQUENCES, cl_sieve.h:2 */

/* error codes */
#define RS_OK 0
#define RS_EARG (-1)            /* invalid argument or state */
#define RS_ECUDA (-2)           /* CUDA runtime error (message in rs_last_error) */
#define RS_ENOMEM (-3)
#define RS_EDEVICE (-4)         /* a kernel raised an internal error flag */
#define RS_EIO (-5)             /* file open/read/write failure */
#define RS_EPARSE (-6)          /* malformed input file */
#define RS_ESTATE (-7)          /* checkpoint missing, corrupt or for another job */
#define RS_EVERIFY (-8)         /* a device factor failed host verification */
#define RS_ENODEV (-9)          /* no CUDA device / library built without one */
#define RS_EBUSY (-10)          /* no free batch slot: run rounds and release finished jobs */

/* One job: up to 100 sequences sharing a base and an n-range.  Mirrors the
 * job fields of workStatus (cl_sieve.h:21-26) plus the candidate bitmap of
 * searchData (cl_sieve.h:30-36, inputfile.cpp:15-21): word seq*words_per_seq
 * + (n-nmin)/32, bit (n-nmin)%32, 1 = term still a candidate. */
typedef struct rs_seqs {
    uint32_t base;
    uint32_t kcount;
    uint32_t nmin;
    uint32_t nmax;
    uint64_t k[RS_MAX_SEQ];
    int32_t c[RS_MAX_SEQ];
    uint64_t words_per_seq;
    uint32_t *bitmap;           /* owned by the rs_seqs object */
} rs_seqs;

/* A found factor p | k[seq]*b^n + c[seq]; replaces struct factor (cl_sieve.h:4-8),
 * which carried the signed int k instead of the sequence index. */
typedef struct rs_factor {
    uint64_t p;
    uint32_t n;
    uint32_t seq;
} rs_factor;

/* Device counters.  primes = primes tested (the reference's g_sum/primecount,
 * setup.cl:99-101, which counts 2-PRPs); dups = solutions whose term was
 * already eliminated or is not a candidate (g_primecount[6], giant.cl:195-196,
 * counted here for n in [nmin,nmax] only). */
typedef struct rs_counters {
    uint64_t primes;
    uint64_t skipped;           /* p | b, p | some k, or no solvable k */
    uint64_t full;              /* primes searched over every n */
    uint64_t parity;            /* primes searched over one class of n mod e per sequence, e >= 2
                                   (e = 2 is the reference's parity split; larger e come from
                                   power-residue characters of higher order) */
    uint64_t targets;           /* sum of surviving k over searched primes */
    uint64_t baby;              /* baby steps */
    uint64_t giant;             /* giant steps = Montgomery products + probes */
    uint64_t small_order;       /* primes where ord(b^e) < Q */
    uint64_t candidates;        /* fingerprint matches verified */
    uint64_t hits;              /* verified solutions with n in [nmin,nmax] (factors + dups) */
    uint64_t factors;           /* terms eliminated */
    uint64_t dups;
    uint64_t sieve_cands;       /* reserved */
} rs_counters;

/* checkpoint scalars of workStatus (cl_sieve.h:21-26) */
typedef struct rs_state {
    uint64_t pmin, pmax, p, checksum, primecount, factorcount, last_trickle, dupcount;
} rs_state;

/* ---------------- host services (no GPU needed) ---------------- */

const char *rs_version(void);
const char *rs_strerror(int code);
/* detail of the last error on the calling thread */
const char *rs_last_error(void);

/* ABCD input (sr2sieve/sr5sieve format); replaces read_input, inputfile.cpp:251-465.
 * Same rules: one base, c = +-1, <= 100 sequences, k > 0, n0 > 0, delta lines,
 * '#' comments; nmin is rounded down to even.  k may be up to 2^64-1. */
int rs_abcd_parse(const char *text, size_t len, rs_seqs **out);
int rs_abcd_read(const char *path, rs_seqs **out);
/* Build a job directly; bitmap may be NULL (all n in [nmin,nmax] are candidates). */
int rs_seqs_create(uint32_t base, uint32_t kcount, const uint64_t *k, const int32_t *c, uint32_t nmin,
                   uint32_t nmax, const uint32_t *bitmap, rs_seqs **out);
void rs_seqs_free(rs_seqs *s);
/* number of candidate terms (set bits) */
uint64_t rs_seqs_count(const rs_seqs *s);

/* verify_factor.c:131-181: 1 if p is prime and p | k*b^n+c, 0 if not a factor,
 * -1 if p is composite. */
int rs_verify_factor(uint64_t p, uint64_t k, uint32_t n, int32_t c, uint32_t base);
/* deterministic primality below 2^64 (verify_factor.c:100-128) */
int rs_is_prime(uint64_t n);

/* "p | k*b^n+c\n" exactly as cl_sieve.cpp:624 prints it */
int rs_format_factor(const rs_seqs *s, const rs_factor *f, char *buf, size_t len);
/* read_factors_file_update_bitmap, cl_sieve.cpp:797-863: clear the bitmap bit
 * of every term listed in a factor file; *lines = number of lines read. */
int rs_factors_file_apply(const char *path, rs_seqs *s, uint64_t *lines);
/* getResults' host half, cl_sieve.cpp:590-631: sort by (p,n), verify each
 * factor, drop composite p, append the lines to path, update state checksum
 * and factorcount.  Returns RS_EVERIFY (and writes nothing) on a false factor. */
int rs_factors_commit(const char *path, const rs_seqs *s, rs_factor *f, size_t n, rs_state *st);
/* finalizeResults, cl_sieve.cpp:738-795 */
int rs_factors_finalize(const char *path, const rs_state *st);

/* Checkpoint files; replace write_state/read_state, cl_sieve.cpp:185-319.
 * When every k < 2^31 the file is the reference's 488-byte workStatus layout
 * with its additive state_sum; otherwise a versioned layout with 64-bit k.
 * rs_state_read validates the job fields, the p-range and the checksum and
 * fails with RS_ESTATE otherwise: st is in/out, and on entry st->pmin and
 * st->pmax must hold the run's p-range (read_state compares them first,
 * cl_sieve.cpp:236-242). */
int rs_state_write(const char *path, const rs_state *st, const rs_seqs *s);
int rs_state_read(const char *path, rs_state *st, const rs_seqs *s);
/* Both A/B files: newest valid one wins (cl_sieve.cpp:288-318).  A file for
 * another p-range is invalid before the two are compared, so a stale file of
 * a different run never shadows a good one.  st->pmin/st->pmax are the run's
 * range on entry.  Returns 1 and fills st and which (0 = A, 1 = B) when a
 * valid state exists, 0 when none. */
int rs_state_resume(const char *path_a, const char *path_b, rs_state *st, const rs_seqs *s, int *which);

/* ---------------- device ---------------- */

typedef struct rs_ctx rs_ctx;

/* Context on one CUDA device (replaces sclHard/progData, cl_sieve.h:39-49 and
 * the device set-up of main.cpp:260-303). */
int rs_ctx_create(int device, rs_ctx **out);
void rs_ctx_destroy(rs_ctx *ctx);
/* Launch on a caller stream (cudaStream_t as void*); NULL = the context's own. */
int rs_ctx_set_stream(rs_ctx *ctx, void *stream);
int rs_device_count(void);

/* Baby steps per prime Q for the BSGS search of this context's jobs: 1024,
 * 2048, 4096, 8192 or 16384, or 0 (the default) to choose per job.  Replaces
 * the reference's Q/M rule, which fixes Q from the n-range when the kernels
 * are built (cl_sieve.cpp:893-938).  In automatic mode a model of the per-prime
 * cost keeps the candidates within 2x of its best, the first full chunks of
 * the job run with each in turn (their results count, as every Q is exact),
 * and the fastest measured one is kept; later jobs of the same shape (base,
 * sequence count, n-range length) on the context reuse it.  Takes effect at
 * once. */
int rs_set_baby_steps(rs_ctx *ctx, uint32_t q);
/* The Q in use; *tuning (may be NULL) is 1 while candidates are being timed. */
int rs_get_baby_steps(rs_ctx *ctx, uint32_t *q, int *tuning);
/* Bounded device waits.  Each CTA of the BSGS kernel waits for the next prime's
 * record copy for at most `tries` rounds of mbarrier try_wait (0: the default,
 * 2^24 rounds); when a wait runs out, the CTA lets the copy land, stops, and
 * rs_run_range returns RS_EDEVICE with error flag 0x10, leaving the context
 * usable.  test_stall = 1 sends each CTA's first wait to a barrier that
 * nothing completes, so the bound always runs out: it exists to test that path
 * (the reference's host polls its queue without bound, cl_sieve.cpp:331-379;
 * there is no counterpart).  Takes effect at the next rs_run_range. */
int rs_set_wait_limit(rs_ctx *ctx, uint32_t tries, int test_stall);
/* Upload a job: sequences, n-range and bitmap (cl_sieve.cpp:1115-1120,1266). */
int rs_job_load(rs_ctx *ctx, const rs_seqs *s);
/* Sieve every prime in [p0,p1) (3 <= p0 < p1 <= 2^64-1): one pass of the
 * segment loop cl_sieve.cpp:1292-1403.  Found factors accumulate on the
 * device; *delta (may be NULL) receives this call's counters. */
int rs_run_range(rs_ctx *ctx, uint64_t p0, uint64_t p1, rs_counters *delta);
/* Copy out and clear the accumulated factors (the device half of getResults,
 * cl_sieve.cpp:537-590).  With cap too small, returns RS_EARG and *n = count. */
int rs_factors_fetch(rs_ctx *ctx, rs_factor *buf, size_t cap, size_t *n);
/* Download the device bitmap (for checkpoints and tests). */
int rs_bitmap_download(rs_ctx *ctx, uint32_t *dst, size_t words);
/* cumulative counters since rs_job_load */
int rs_counters_get(rs_ctx *ctx, rs_counters *out);
/* The prime generator alone: odd primes in [p0,p1), unordered, for tests. */
int rs_primes_generate(rs_ctx *ctx, uint64_t p0, uint64_t p1, uint64_t *dst, size_t cap, size_t *n);
/* average duration (ms) of the BSGS kernel launches of the last rs_run_range,
 * measured with CUDA events on the launching stream, and the launch count */
int rs_last_timing(rs_ctx *ctx, double *bsgs_ms, double *total_kernel_ms, uint32_t *bsgs_launches,
                   uint32_t *kernel_launches);

/* ---------------- batches: many jobs on one device ----------------
 * The reference sieves one job per process (cl_sieve.cpp:975-1451).  A batch
 * holds many independent jobs -- own sequences, n-range, bitmap and p-range
 * each -- and advances all of them in rounds of device-resident work: every
 * unfinished job sieves its next window (about 39 000 primes) per round, the
 * BSGS work of all jobs that share a geometry runs in one persistent launch,
 * and the host waits once per round.  After the first round a round is
 * replayed from a captured CUDA graph.  Jobs may be added between rounds and
 * released when done, so a batch also serves a stream of work units.  Each
 * job's eliminated terms equal what rs_run_range gives for the same job and
 * p-range. */
typedef struct rs_batch rs_batch;
/* max_jobs job slots and range_slots range slots (0: 64 each).  Each range slot
 * holds one round's buffers (about 136 MB); a job takes one range slot, or two
 * when its p-range straddles 2^63. */
int rs_batch_create(int device, uint32_t max_jobs, uint32_t range_slots, rs_batch **out);
void rs_batch_destroy(rs_batch *b);
/* A caller stream (cudaStream_t as void*, not the legacy NULL stream); only
 * before the first rs_batch_run. */
int rs_batch_set_stream(rs_batch *b, void *stream);
/* Adds a job with its p-range [p0, p1) (3 <= p0 < p1, or p0 == p1 for a
 * template, see rs_batch_add_clone); q fixes its baby-step
 * count (as rs_set_baby_steps).  With q = 0 the job takes the count that a
 * context (rs_run_range) on the same device measured for a job of the same
 * shape (base, sequence count, n-range), else the cost model's choice.  The job's
 * bitmap is copied to the device.  *job (may be NULL) receives its slot.
 * RS_EBUSY when no job or range slot is free. */
int rs_batch_add(rs_batch *b, const rs_seqs *s, uint64_t p0, uint64_t p1, uint32_t q, uint32_t *job);
/* A new job with job src's sequences, geometry and current bitmap, copied on
 * the device (no host transfer), over [p0, p1) cut into nsplit equal parts
 * (one range slot each, sharing the bitmap), so that a unit can spread over
 * the device.  A job added with p0 == p1 is a resident template: it takes no
 * range slot and never runs, and serves as the source of clones -- e.g. one
 * template per input file, one clone per work unit, each unit with its own
 * bitmap. */
int rs_batch_add_clone(rs_batch *b, uint32_t src, uint64_t p0, uint64_t p1, uint32_t nsplit, uint32_t *job);
/* Primes a job should cover in each following round, spread over its
 * unfinished ranges (each range at most about 39 000 per round); 0 pauses it.
 * Jobs start with full windows.  A serving loop sets these per round to order
 * work (e.g. earliest deadline or shortest remaining first). */
int rs_batch_set_budget(rs_batch *b, uint32_t job, uint64_t primes);
/* Every job slot's state in one read: done (job finished; 0 for free slots),
 * primes tested and p-range left to sieve -- arrays of max_jobs entries, each
 * may be NULL. */
int rs_batch_poll(rs_batch *b, uint8_t *done, uint64_t *primes, uint64_t *remaining);
/* Free job slots and range slots. */
int rs_batch_free_slots(rs_batch *b, uint32_t *jobs, uint32_t *ranges);
/* Device memory a job, or a clone of it, holds while admitted: its bitmap and
 * a factor list with room for every candidate term. */
int rs_batch_job_bytes(rs_batch *b, uint32_t job, uint64_t *bytes);
/* Maps `bytes` of device memory into the batch's job pool ahead of time, so that
 * later admissions up to that total reuse it instead of mapping new memory
 * (which can take hundreds of milliseconds).  RS_ENOMEM when the device cannot
 * provide it.  Serving loops admit units by footprint within this reserve. */
int rs_batch_reserve(rs_batch *b, uint64_t bytes);
/* Frees a job's slots (fetch its factors and bitmap first). */
int rs_batch_release(rs_batch *b, uint32_t job);
/* Runs up to max_rounds rounds (0: until every job is done, or every
 * unfinished job is paused by a zero budget); *done = 1 once every job's
 * p-range is finished. */
int rs_batch_run(rs_batch *b, uint32_t max_rounds, int *done);
/* Per job, as rs_factors_fetch / rs_bitmap_download. */
int rs_batch_factors_fetch(rs_batch *b, uint32_t job, rs_factor *buf, size_t cap, size_t *n);
int rs_batch_bitmap_download(rs_batch *b, uint32_t job, uint32_t *dst, size_t words);
/* A job's baby-step count, primes tested so far and whether its range is done
 * (each pointer may be NULL). */
int rs_batch_job_info(rs_batch *b, uint32_t job, uint32_t *q, uint64_t *primes, int *done);
/* Counters summed over every job the batch has run. */
int rs_batch_counters(rs_batch *b, rs_counters *out);

/* Throughput of independent 64-bit Montgomery products (the kernels' mmul)
 * on this device, in 10^9 products/s: the roofline denominator of the
 * integer-multiply-bound BSGS kernel. */
int rs_mulmod_peak(rs_ctx *ctx, double *gmulmods_per_s, double *ms);
/* Measured 32x32->64 multiply throughput of the device (10^9 wide products/s,
 * sixteen independent mad.wide.u32 chains per thread).  A 64-bit Montgomery
 * product takes 11 of them, so *gwide_per_s / 11 is the product rate the
 * multiplier itself allows.  A measurement aid with no reference counterpart
 * (the reference reports no roofline). */
int rs_widemul_peak(rs_ctx *ctx, double *gwide_per_s, double *ms);
/* Throughput of independent FP64 modular products by a fixed multiplier (the
 * product the BSGS steps use below 2^51: an exact two-product, a quotient from
 * the double w/p, one correction), in 10^9 products/s, on a prime just above
 * 2^50.  A measurement aid with no reference counterpart. */
int rs_fpmul_peak(rs_ctx *ctx, double *gfpmul_per_s, double *ms);

/* Largest range width (p1 - p0) that rs_primes_generate_noalloc accepts. */
#define RS_NOALLOC_MAX_WIDTH (1ull << 22)

/* The prime generator of rs_primes_generate, for callers that must not
 * allocate device memory: no cudaMalloc or cudaFree, no allocating library
 * routine, no context.  No counterpart in the reference (its getsegprimes
 * writes into buffers that cl_sieve.cpp allocates up front).
 *
 * Writes the odd primes of [p0,p1), unordered, to d_primes (caller-owned
 * device memory, room for cap values) and their total number to *d_count
 * (caller-owned device word), both on `stream` (a cudaStream_t; NULL is the
 * legacy default stream).  The call enqueues work and returns; read *d_count
 * after the stream is done.  If *d_count > cap the output is incomplete:
 * repeat with more room or a narrower range.  p0 < 3 is raised to 3.
 *
 * Scratch is one fixed device array in the library (about 16 MiB per device,
 * reserved when its module loads).  Hence: p1 - p0 must not exceed
 * RS_NOALLOC_MAX_WIDTH (RS_EARG otherwise, with the limit in rs_last_error);
 * the first call on a device does a one-time set-up that waits for `stream`,
 * so make it before any stream capture; and calls whose work overlaps on one
 * device (different streams, unordered) race on the shared scratch.  Each call
 * resets its scratch counters and *d_count itself; nothing needs zeroing. */
int rs_primes_generate_noalloc(uint64_t p0, uint64_t p1, uint64_t *d_primes, uint32_t cap, uint32_t *d_count,
                               void *stream);

#ifdef __cplusplus
}
#endif
#endif

/*
 * rsoracle.c -- CPU oracle for the RSSieve BSGS sieve path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  See rsoracle.h for what each part
 * restates; every function names the reference file:line it follows.
 * Parity pins: rsoracle's setup restatement is compared value-for-value with
 * the reference's own kernels/setup.cl compiled under oracle/ref_shim.hpp,
 * its verify restatement with the reference's own verify_factor.c, and its
 * BSGS port with the independent brute-force term oracle below.
 */
#include "rsoracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------ */
/* Montgomery arithmetic, kernels/common.cl:24-47                            */
/* ------------------------------------------------------------------------ */

/* Newton iteration for p^-1 mod 2^64 -- common.cl:24-28 */
uint64_t or_invert(uint64_t p)
{
    uint64_t p_inv = 1, prev = 0;
    while (p_inv != prev) { prev = p_inv; p_inv *= 2 - p * p_inv; }
    return p_inv;
}

/* Montgomery product a*b*2^-64 mod p, q = p^-1 mod 2^64 -- common.cl:33-40 */
uint64_t or_m_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t q)
{
    u128 ab = (u128)a * b;
    uint64_t lo = (uint64_t)ab, hi = (uint64_t)(ab >> 64);
    uint64_t m = lo * q;
    uint64_t mp = (uint64_t)(((u128)m * p) >> 64);
    uint64_t r = hi - mp;
    return (hi < mp) ? r + p : r;
}

/* a+b mod p for a,b < p -- common.cl:42-47 */
uint64_t or_add(uint64_t a, uint64_t b, uint64_t p)
{
    uint64_t c = (a >= p - b) ? p : 0;
    return a + b - c;
}

/* plain left-to-right powmod of a Montgomery base (exact for every exponent) */
uint64_t or_powmod(uint64_t mbase, uint64_t exp, uint64_t p, uint64_t q, uint64_t one)
{
    if (exp == 0) return one;
    if (exp == 1) return mbase;
    uint64_t cur = 0x8000000000000000ULL >> (__builtin_clzll(exp) + 1);
    uint64_t a = mbase;
    while (cur) {
        a = or_m_mul(a, a, p, q);
        if (exp & cur) a = or_m_mul(a, mbase, p, q);
        cur >>= 1;
    }
    return a;
}

/* powmodlg / basepowmodlg with the reference's OpenCL shift semantics:
 * common.cl:51-63 and 67-90 compute curBit >>= clz(exp)+1 with a 64-bit
 * shift count that OpenCL masks to 6 bits, so exp == 1 walks 64 squarings.
 * The value mbase^(2^64+1) is what the reference kernel produces there. */
static uint64_t ref_powlg(uint64_t mbase, uint64_t exp, uint64_t p, uint64_t q)
{
    uint64_t cur = 0x8000000000000000ULL >> ((__builtin_clzll(exp) + 1) & 63);
    uint64_t a = mbase;
    while (cur) {
        a = or_m_mul(a, a, p, q);
        if (exp & cur) a = or_m_mul(a, mbase, p, q);
        cur >>= 1;
    }
    return a;
}

/* powmodsm / basepowmodsm, 32-bit exponent -- common.cl:93-135 */
static uint64_t ref_powsm(uint64_t mbase, uint32_t exp, uint64_t p, uint64_t q, uint64_t one)
{
    if (!exp) return one;
    if (exp == 1) return mbase;
    uint32_t cur = 0x80000000u >> (__builtin_clz(exp) + 1);
    uint64_t a = mbase;
    while (cur) {
        a = or_m_mul(a, a, p, q);
        if (exp & cur) a = or_m_mul(a, mbase, p, q);
        cur >>= 1;
    }
    return a;
}

/* the per-prime row getsegprimes.cl:173-179 / addsmallprimes.cl:18-23 build */
typedef struct { uint64_t s[8]; } row8;
static row8 make_row(uint64_t p)
{
    row8 r;
    memset(&r, 0, sizeof r);
    r.s[0] = p;
    r.s[1] = or_invert(p);
    r.s[2] = (0 - p) % p;               /* one = 2^64 mod p */
    r.s[4] = p - r.s[2];                /* nmo = p - one    */
    r.s[3] = or_add(r.s[2], r.s[2], p); /* two              */
    return r;
}

/* ------------------------------------------------------------------------ */
/* Primality                                                                 */
/* ------------------------------------------------------------------------ */

/* strong base-2 PRP test -- getsegprimes.cl:37-66, with its masked shift */
int or_sprp2(uint64_t N)
{
    if (N < 3 || !(N & 1)) return 0;
    uint64_t q = or_invert(N), one = (0 - N) % N, nmo = N - one, two = or_add(one, one, N);
    int t = __builtin_ctzll(N - 1);
    uint64_t exp = N >> t;
    uint64_t cur = 0x8000000000000000ULL >> ((__builtin_clzll(exp) + 1) & 63);
    uint64_t a = two;
    while (cur) {
        a = or_m_mul(a, a, N, q);
        if (exp & cur) a = or_add(a, a, N);
        cur >>= 1;
    }
    if (a == one || a == nmo) return 1;
    for (int s = 1; s < t; ++s) {
        a = or_m_mul(a, a, N, q);
        if (a == nmo) return 1;
    }
    return 0;
}

/* strong PRP to one base -- verify_factor.c:57-95 */
static int sprp_base(uint32_t base, uint64_t p, uint64_t q, uint64_t one, uint64_t pmo,
                     uint64_t r2, int t, uint64_t exp)
{
    uint64_t a = or_m_mul(base, r2, p, q);
    const uint64_t mbase = a;
    uint64_t cur = 0x8000000000000000ULL >> ((__builtin_clzll(exp) + 1) & 63);
    while (cur) {
        a = or_m_mul(a, a, p, q);
        if (exp & cur) a = or_m_mul(a, mbase, p, q);
        cur >>= 1;
    }
    if (a == one || a == pmo) return 1;
    for (int s = 1; s < t; ++s) {
        a = or_m_mul(a, a, p, q);
        if (a == pmo) return 1;
    }
    return 0;
}

static uint64_t r2_of(uint64_t p, uint64_t q, uint64_t one)
{
    /* verify_factor.c:137-141 / setup.cl:112-119: (4R)^(2^5) -> R^2 */
    uint64_t two = or_add(one, one, p);
    uint64_t t = or_add(two, two, p);
    for (int i = 0; i < 5; ++i) t = or_m_mul(t, t, p, q);
    return t;
}

/* deterministic below 2^64 -- verify_factor.c:100-128 */
int or_is_prime(uint64_t p)
{
    static const uint32_t bases[7] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    if (p < 2) return 0;
    if (p % 2 == 0) return p == 2;
    if (p == 3) return 1;
    uint64_t q = or_invert(p), one = (0 - p) % p, pmo = p - one;
    uint64_t r2 = r2_of(p, q, one);
    int t = __builtin_ctzll(p - 1);
    uint64_t exp = p >> t;
    for (int i = 0; i < 7; ++i) {
        uint32_t base = bases[i];
        if (base >= p) {
            base %= p;
            if (base == 0) continue;
        }
        if (!sprp_base(base, p, q, one, pmo, r2, t, exp)) return 0;
    }
    return 1;
}

/* sieving primes below 2^16 for the independent true-prime generator */
static uint32_t g_small_primes[7000];
static int g_nsmall = 0;
static void init_small_primes(void)
{
    if (g_nsmall) return;
    static unsigned char comp[65537];
    int n = 0;
    for (uint32_t i = 2; i <= 65536; ++i) {
        if (comp[i]) continue;
        g_small_primes[n++] = i;
        for (uint64_t j = (uint64_t)i * i; j <= 65536; j += i) comp[j] = 1;
    }
    __atomic_store_n(&g_nsmall, n, __ATOMIC_RELEASE);
}

/* Segmented Eratosthenes with all odd primes < 2^16, then 7-base SPRP for the
 * survivors at or above 65537^2 (below that the sieve alone is exact).
 * Writes the odd primes of [lo,hi) in ascending order. */
size_t or_primes(uint64_t lo, uint64_t hi, uint64_t *out, size_t cap)
{
    init_small_primes();
    if (lo < 3) lo = 3;
    if (hi <= lo) return 0;
    size_t cnt = 0;
    const uint64_t CH = (uint64_t)1 << 22;          /* odd numbers per chunk */
    unsigned char *mark = (unsigned char *)malloc(CH);
    uint64_t a = lo | 1;                            /* first odd >= lo */
    while (a < hi) {
        uint64_t nodd = (hi - a + 1) / 2;           /* odd numbers in [a,hi) */
        if (nodd > CH) nodd = CH;
        memset(mark, 0, nodd);
        uint64_t last = a + 2 * (nodd - 1);
        for (int i = 1; i < g_nsmall; ++i) {        /* skip 2 */
            uint64_t r = g_small_primes[i];
            if (r * r > last) break;
            u128 s = ((u128)a + r - 1) / r * r;     /* first multiple >= a */
            if (!(s & 1)) s += r;                   /* odd multiple */
            if (s < (u128)r * r) s = (u128)r * r;
            for (u128 x = s; x <= last; x += 2 * r) mark[(uint64_t)(x - a) / 2] = 1;
        }
        for (uint64_t i = 0; i < nodd; ++i) {
            if (mark[i]) continue;
            uint64_t v = a + 2 * i;
            if (v >= 4295098369ULL && !or_is_prime(v)) continue;
            if (cnt < cap) out[cnt] = v;
            ++cnt;
        }
        if (nodd < CH) break;
        a += 2 * nodd;
    }
    free(mark);
    return cnt;
}

/* The reference's sieve-prime set: primes <= 113 from addsmallprimes.cl:8-27
 * (run for [p, min(stop,114)), cl_sieve.cpp:1304-1310) plus every number in
 * [max(lo,114),hi) coprime to 2..113 that passes strong_prp_two
 * (getsegprimes.cl:141-181; the mod-30 wheel + bit tables of 7..113 select
 * exactly the integers coprime to all primes <= 113).  Ascending order. */
size_t or_prp2(uint64_t lo, uint64_t hi, uint64_t *out, size_t cap)
{
    static const uint32_t sp[30] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61,
                                    67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113};
    size_t cnt = 0;
    for (int i = 0; i < 30; ++i)
        if (sp[i] >= lo && sp[i] < hi && sp[i] < 114) { if (cnt < cap) out[cnt] = sp[i]; ++cnt; }
    uint64_t a = lo < 114 ? 114 : lo;
    if (a >= hi) return cnt;
    a |= 1;
    const uint64_t CH = (uint64_t)1 << 22;
    unsigned char *mark = (unsigned char *)malloc(CH);
    while (a < hi) {
        uint64_t nodd = (hi - a + 1) / 2;
        if (nodd > CH) nodd = CH;
        memset(mark, 0, nodd);
        uint64_t last = a + 2 * (nodd - 1);
        for (int i = 1; i < 30; ++i) {
            uint64_t r = sp[i];
            u128 s = ((u128)a + r - 1) / r * r;
            if (!(s & 1)) s += r;
            for (u128 x = s; x <= last; x += 2 * r) mark[(uint64_t)(x - a) / 2] = 1;
        }
        for (uint64_t i = 0; i < nodd; ++i) {
            if (mark[i]) continue;
            uint64_t v = a + 2 * i;
            if (!or_sprp2(v)) continue;
            if (cnt < cap) out[cnt] = v;
            ++cnt;
        }
        if (nodd < CH) break;
        a += 2 * nodd;
    }
    free(mark);
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* verify_factor.c:131-181 (n exponentiation written exactly for every n)    */
/* ------------------------------------------------------------------------ */
int or_verify_factor(uint64_t p, uint64_t k, uint32_t n, int32_t c, uint32_t base)
{
    if (p < 3 || !(p & 1)) return -1;
    uint64_t q = or_invert(p), one = (0 - p) % p;
    uint64_t two = or_add(one, one, p);
    uint64_t r2 = r2_of(p, q, one);
    uint64_t mbase = (base == 2) ? two : or_m_mul(base, r2, p, q);
    if (!or_is_prime(p)) return -1;
    uint64_t a = or_powmod(mbase, n, p, q, one);
    a = or_m_mul(a, k, p, q);                 /* k*b^n mod p, standard form */
    if (a == 1 && c == -1) return 1;
    if (a == p - 1 && c == 1) return 1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Bitmap claim -- giant.cl:21-39                                            */
/* ------------------------------------------------------------------------ */
static int claim(or_job *job, uint32_t seq, uint64_t n)
{
    if (n < job->nmin || n > job->nmax) return 0;
    uint64_t off = n - job->nmin;
    uint32_t *w = &job->bitmap[(size_t)seq * job->words_per_seq + (off >> 5)];
    uint32_t mask = 1u << (off & 31u);
    uint32_t old = __atomic_fetch_and(w, ~mask, __ATOMIC_RELAXED);
    return (old & mask) != 0;
}

static void emit(or_factor *out, size_t cap, size_t *cnt, uint64_t p, uint32_t n, uint32_t seq)
{
    size_t i = __atomic_fetch_add(cnt, 1, __ATOMIC_RELAXED);
    if (i < cap) { out[i].p = p; out[i].n = n; out[i].seq = seq; }
}

/* ------------------------------------------------------------------------ */
/* Brute-force term oracle (independent of the BSGS logic)                   */
/* ------------------------------------------------------------------------ */

/* modular inverse by the extended Euclidean algorithm, a in [1,p) */
static uint64_t inv_euclid(uint64_t a, uint64_t p)
{
    __int128 t = 0, nt = 1, r = p, nr = a;
    while (nr) {
        __int128 qq = r / nr, tmp;
        tmp = t - qq * nt; t = nt; nt = tmp;
        tmp = r - qq * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += p;
    return (uint64_t)t;
}

static uint64_t mulmod_plain(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }

size_t or_brute(or_job *job, const uint64_t *primes, size_t np, int ref_skip,
                or_factor *out, size_t cap, uint64_t *dups)
{
    size_t cnt = 0;
    uint64_t dup = 0;
    const uint32_t K = job->kcount;
    /* primes run in parallel: claims are atomic, so the eliminated-term set,
     * the final bitmap and the duplicate count do not depend on the order */
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : dup) if (np > 64)
#endif
    for (long long ip = 0; ip < (long long)np; ++ip) {
        uint64_t p = primes[ip];
        if (p < 3 || !(p & 1)) continue;
        uint64_t bm = job->base % p;
        if (bm == 0) continue;                       /* b^n = 0: no term is divisible */
        /* targets b^n == -c_i * k_i^-1 (mod p), as Montgomery residues */
        uint64_t q = or_invert(p), one = (0 - p) % p, r2 = r2_of(p, q, one);
        uint64_t tv[256]; int16_t ts[256]; uint8_t used[256];
        memset(used, 0, sizeof used);
        int skip = 0;
        for (uint32_t i = 0; i < K; ++i) {
            uint64_t km = job->k[i] % p;
            if (km == 0) { if (ref_skip) { skip = 1; break; } continue; }
            uint64_t inv = inv_euclid(km, p);
            uint64_t t = (job->c[i] == 1) ? (p - inv) % p : inv;
            uint64_t tm = or_m_mul(t, r2, p, q);
            uint32_t h = (uint32_t)(tm * 0x9E3779B97F4A7C15ULL >> 56);
            while (used[h]) h = (h + 1) & 255;
            used[h] = 1; tv[h] = tm; ts[h] = (int16_t)i;
        }
        if (skip) continue;
        /* x = b^nmin, stepped by b for every n */
        uint64_t x = 1 % p, e = job->nmin, bb = bm;
        while (e) { if (e & 1) x = mulmod_plain(x, bb, p); bb = mulmod_plain(bb, bb, p); e >>= 1; }
        uint64_t xm = or_m_mul(x, r2, p, q), mb = or_m_mul(bm, r2, p, q);
        for (uint64_t n = job->nmin; n <= job->nmax; ++n) {
            uint32_t h = (uint32_t)(xm * 0x9E3779B97F4A7C15ULL >> 56);
            while (used[h]) {
                if (tv[h] == xm) {
                    if (claim(job, (uint32_t)ts[h], n)) emit(out, cap, &cnt, p, (uint32_t)n, (uint32_t)ts[h]);
                    else ++dup;
                }
                h = (h + 1) & 255;
            }
            xm = or_m_mul(xm, mb, p, q);
        }
    }
    if (dups) *dups = dup;
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* Reference parameter rule -- cl_sieve.cpp:893-938                          */
/* ------------------------------------------------------------------------ */
or_params or_ref_params(uint32_t nmin, uint32_t nmax)
{
    or_params r;
    uint32_t L = nmax - nmin + 1;
    uint32_t targetQ = (uint32_t)ceil(sqrt((double)L));
    r.Q = 1024; r.hsize = 2048;
    while (r.Q < 4096 && r.Q < targetQ) { r.Q <<= 1; r.hsize <<= 1; }
    /* NVIDIA exposes 49152 B of local memory: 8192*4+4+16 always fits (:904-920) */
    r.m = (uint32_t)ceil((double)L / r.Q);
    r.QQ = r.Q << 1;
    r.mm = (uint32_t)ceil((double)L / r.QQ);
    return r;
}

/* ------------------------------------------------------------------------ */
/* setup.cl:11-209 restated                                                  */
/* ------------------------------------------------------------------------ */

/* setup_pr -- setup.cl:22-56 */
static int setup_pr(const row8 *pr, uint64_t pmo, uint64_t *expo, int *resg)
{
    static const uint32_t ds[12] = {3, 4, 5, 7, 8, 9, 11, 13, 17, 19, 23, 29};
    const uint64_t pm = pr->s[0] - 1;
    int r = 0;
    for (int i = 0; i < 12; ++i) {
        uint64_t d = ds[i];
        expo[r] = pm / d;
        /* good_pr, setup.cl:11-17 */
        if (pm == expo[r] * d && ref_powlg(pr->s[3], expo[r], pr->s[0], pr->s[1]) == pr->s[2]) r++;
    }
    expo[12] = pm >> 1;
    uint64_t rg = ref_powlg(pr->s[3], expo[12], pr->s[0], pr->s[1]);
    *resg = (rg == pr->s[2]) - (rg == pmo);
    return r;
}

/* prefilter -- setup.cl:59-87 */
static int prefilter(uint64_t hk_inv, uint64_t p, uint64_t q, uint64_t one, uint64_t pmo,
                     const uint64_t *power, int powcnt, int rg)
{
    uint64_t ra;
    for (int i = 0; i < powcnt; ++i) {
        ra = ref_powlg(hk_inv, power[i], p, q);
        if (ra != one) return 0;
    }
    ra = ref_powlg(hk_inv, power[12], p, q);
    if (rg == -1) {
        if (ra == one) return 2;
        else if (ra == pmo) return 3;
        else return 0;
    }
    if (rg == 1 && ra == pmo) return 0;
    return 1;
}

/* Montgomery form of the base -- setup.cl:121-128 */
static uint64_t mont_base(uint32_t base, uint64_t p, uint64_t q, uint64_t one, uint64_t two, uint64_t r2)
{
    uint64_t four = or_add(two, two, p);
    if (base == 2) return two;
    if (base == 3) return or_add(one, two, p);
    if (base == 5) return or_add(four, one, p);
    return or_m_mul(base, r2, p, q);
}

/* one prime through setup.cl:89-209: updates row (s0=0 skip, s3=mbase,
 * s5=gQ_inv) and writes kd[0..] in the kernel's order; returns #k kept or -1 */
static int setup_one(const or_job *job, uint32_t Q, row8 *pr, or_kdata *kd)
{
    const int K = (int)job->kcount;
    const uint64_t p = pr->s[0], q = pr->s[1];
    uint64_t four = or_add(pr->s[3], pr->s[3], p);
    uint64_t r2 = four;
    for (int i = 0; i < 5; ++i) r2 = or_m_mul(r2, r2, p, q);
    pr->s[3] = mont_base(job->base, p, q, pr->s[2], pr->s[3], r2);
    uint64_t mk[OR_MAX_SEQ + 1], prefix[OR_MAX_SEQ + 1];
    uint64_t gQ = ref_powsm(pr->s[3], Q, p, q, pr->s[2]);
    mk[K] = gQ;
    for (int i = 0; i < K; ++i) mk[i] = or_m_mul(job->k[i], r2, p, q);
    prefix[0] = mk[0];
    for (int i = 1; i < K + 1; ++i) prefix[i] = or_m_mul(prefix[i - 1], mk[i], p, q);
    uint64_t inv_total = ref_powlg(prefix[K], p - 2, p, q);
    uint64_t one = or_m_mul(prefix[K], inv_total, p, q);
    if (one != pr->s[2]) { pr->s[0] = 0; return -1; }
    uint64_t prev = prefix[K - 1];
    pr->s[5] = or_m_mul(inv_total, prev, p, q);          /* gQ_inv */
    inv_total = or_m_mul(inv_total, mk[K], p, q);
    int resg;
    uint64_t expo[13];
    int tests = setup_pr(pr, pr->s[4], expo, &resg);
    int count[4] = {0, 0, 0, 0};
    int pos = 0;
    for (int i = K - 1; i >= 0; --i) {
        prev = (i == 0) ? pr->s[2] : prefix[i - 1];
        uint64_t k_inv = or_m_mul(inv_total, prev, p, q);
        inv_total = or_m_mul(inv_total, mk[i], p, q);
        uint64_t hk_inv = (job->c[i] > 0) ? or_m_mul(pr->s[4], k_inv, p, q) : k_inv;
        int parity = prefilter(hk_inv, p, q, pr->s[2], pr->s[4], expo, tests, resg);
        count[parity]++;
        if (parity) { kd[pos].hadj = hk_inv; kd[pos].parity = parity; kd[pos].kidx = i; pos++; }
    }
    if (pos < K) { kd[pos].hadj = 0; kd[pos].parity = 0; kd[pos].kidx = 0; }
    if (count[0] == K) { pr->s[0] = 0; return -1; }
    return pos;
}

void or_setup(const or_job *job, uint32_t Q, const uint64_t *primes, size_t np,
              uint64_t *rows, or_kdata *kd)
{
    for (size_t i = 0; i < np; ++i) {
        row8 r = make_row(primes[i]);
        setup_one(job, Q, &r, kd + i * job->kcount);
        memcpy(rows + i * 8, r.s, sizeof r.s);
    }
}

/* ------------------------------------------------------------------------ */
/* giant.cl restated: lo32 table + hi32/idx arrays, giant.cl:41-75           */
/* ------------------------------------------------------------------------ */
typedef struct { uint32_t *lt, *ht; int16_t *hi; uint32_t mask; } htab;

static void h_insert(htab *t, uint64_t val, int idx)
{
    uint32_t lo = (uint32_t)val, hi = (uint32_t)(val >> 32);
    uint32_t pos = lo & t->mask;
    for (;;) {
        if (t->lt[pos] == 0) {          /* atomic_cmpxchg(&lt[pos],0,lo)==0 */
            t->lt[pos] = lo;
            t->ht[pos] = hi;
            t->hi[pos] = (int16_t)idx;
            return;
        }
        pos = (pos + 1) & t->mask;
    }
}

static int h_lookup(const htab *t, uint64_t val, int *out)
{
    uint32_t lo = (uint32_t)val, hi = (uint32_t)(val >> 32);
    uint32_t pos = lo & t->mask, start = pos;
    for (uint32_t e = t->lt[pos]; e; e = t->lt[pos]) {
        if (e == lo && t->ht[pos] == hi) { *out = (int)t->hi[pos]; return 1; }
        pos = (pos + 1) & t->mask;
        if (pos == start) break;
    }
    return 0;
}

typedef struct { uint64_t hadj; int32_t kidx; } kpar;

/* giantfull (parity 1, step 1, span Q, M giant steps) and giantparity
 * (parity 2/3, step 2, span QQ, MM giant steps) -- giant.cl:77-323 */
static void giant_one(or_job *job, const or_params *pp, htab *t, uint64_t p, uint64_t q, uint64_t one,
                      uint64_t mbase, uint64_t gQ_inv, int parity, const kpar *ks, int numk,
                      or_factor *out, size_t cap, size_t *cnt, or_stats *st)
{
    const uint32_t span = (parity == 1) ? pp->Q : pp->QQ;
    const uint32_t nsteps = (parity == 1) ? pp->m : pp->mm;
    const uint32_t jstep = (parity == 1) ? 1 : 2;
    const uint64_t nstart = job->nmin + (parity == 3 ? 1 : 0);
    memset(t->lt, 0, sizeof(uint32_t) * pp->hsize);
    /* baby steps: gj = b^(nstart + j); order detection against b^nstart (:123-134, :247-258) */
    uint64_t g0 = ref_powsm(mbase, (uint32_t)nstart, p, q, one);
    uint64_t g = g0, bstep = (jstep == 1) ? mbase : or_m_mul(mbase, mbase, p, q);
    uint32_t order = 0;
    uint64_t mm = 0;
    for (uint32_t j = 0; j < span; j += jstep) {
        if (j && g == g0) { order = j; break; }
        h_insert(t, g, (int)j);
        g = or_m_mul(g, bstep, p, q);
        ++mm;
    }
    uint64_t lk = 0, dref = 0, din = 0;
    if (order) {
        /* :146-168 / :270-292 */
        for (int i = 0; i < numk; ++i) {
            int r;
            ++lk;
            if (!h_lookup(t, ks[i].hadj, &r)) continue;
            for (uint64_t n = nstart + (uint64_t)r; n <= job->nmax; n += order) {
                if (claim(job, (uint32_t)ks[i].kidx, n)) emit(out, cap, cnt, p, (uint32_t)n, (uint32_t)ks[i].kidx);
                else { ++dref; ++din; }
            }
        }
    } else {
        /* :170-192 / :294-318: gamma = hadj * gQ_inv^(q*jstep) */
        uint64_t gstep = (jstep == 1) ? gQ_inv : or_m_mul(gQ_inv, gQ_inv, p, q);
        uint64_t z = one;
        for (uint32_t qq = 0; qq < nsteps; ++qq) {
            for (int i = 0; i < numk; ++i) {
                uint64_t gamma = or_m_mul(ks[i].hadj, z, p, q);
                int r;
                ++mm; ++lk;
                if (!h_lookup(t, gamma, &r)) continue;
                uint64_t n = nstart + (uint64_t)qq * span + (uint64_t)r;
                if (claim(job, (uint32_t)ks[i].kidx, n)) emit(out, cap, cnt, p, (uint32_t)n, (uint32_t)ks[i].kidx);
                else { ++dref; if (n <= job->nmax) ++din; }
            }
            z = or_m_mul(z, gstep, p, q);
            ++mm;
        }
    }
    __atomic_fetch_add(&st->mulmods, mm, __ATOMIC_RELAXED);
    __atomic_fetch_add(&st->lookups, lk, __ATOMIC_RELAXED);
    __atomic_fetch_add(&st->dup_ref, dref, __ATOMIC_RELAXED);
    __atomic_fetch_add(&st->dup_inrange, din, __ATOMIC_RELAXED);
}

size_t or_bsgs(or_job *job, const uint64_t *primes, size_t np, int nthreads,
               or_factor *out, size_t cap, or_stats *stats)
{
    or_stats st;
    memset(&st, 0, sizeof st);
    or_params pp = or_ref_params(job->nmin, job->nmax);
    size_t cnt = 0;
    const int K = (int)job->kcount;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
#endif
    {
        htab t;
        t.mask = pp.hsize - 1;
        t.lt = (uint32_t *)malloc(sizeof(uint32_t) * pp.hsize);
        t.ht = (uint32_t *)malloc(sizeof(uint32_t) * pp.hsize);
        t.hi = (int16_t *)malloc(sizeof(int16_t) * pp.hsize);
        or_kdata kd[OR_MAX_SEQ];
        kpar kf[OR_MAX_SEQ], ke[OR_MAX_SEQ], ko[OR_MAX_SEQ];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 16)
#endif
        for (long long ip = 0; ip < (long long)np; ++ip) {
            row8 r = make_row(primes[ip]);
            int nk = setup_one(job, pp.Q, &r, kd);
            if (nk < 0) { __atomic_fetch_add(&st.skipped, 1, __ATOMIC_RELAXED); continue; }
            /* sort.cl:251-282: bin by parity class, in setup's write order */
            int nf = 0, ne = 0, no = 0;
            for (int i = 0; i < K; ++i) {
                if (!kd[i].parity) break;
                kpar kp = {kd[i].hadj, kd[i].kidx};
                if (kd[i].parity == 1) kf[nf++] = kp;
                else if (kd[i].parity == 2) ke[ne++] = kp;
                else ko[no++] = kp;
            }
            const uint64_t p = r.s[0], q = r.s[1], one = r.s[2], mbase = r.s[3], gQ_inv = r.s[5];
            if (nf) giant_one(job, &pp, &t, p, q, one, mbase, gQ_inv, 1, kf, nf, out, cap, &cnt, &st);
            if (ne) giant_one(job, &pp, &t, p, q, one, mbase, gQ_inv, 2, ke, ne, out, cap, &cnt, &st);
            if (no) giant_one(job, &pp, &t, p, q, one, mbase, gQ_inv, 3, ko, no, out, cap, &cnt, &st);
        }
        free(t.lt); free(t.ht); free(t.hi);
    }
    if (stats) *stats = st;
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* getResults restated -- cl_sieve.cpp:515-529 (order), :594-631 (verify)    */
/* ------------------------------------------------------------------------ */
static int fcmp(const void *a, const void *b)
{
    const or_factor *x = (const or_factor *)a, *y = (const or_factor *)b;
    if (x->p != y->p) return x->p < y->p ? -1 : 1;
    if (x->n != y->n) return x->n < y->n ? -1 : 1;
    return 0;
}

size_t or_verify_and_sort(const or_job *job, or_factor *f, size_t nf, int *false_factor, uint64_t *checksum)
{
    qsort(f, nf, sizeof *f, fcmp);
    size_t kept = 0;
    int bad = 0;
    uint64_t cs = 0;
    for (size_t i = 0; i < nf; ++i) {
        int v = or_verify_factor(f[i].p, job->k[f[i].seq], f[i].n, job->c[f[i].seq], job->base);
        if (v == 0) { bad = 1; continue; }
        if (v < 0) continue;                     /* composite 2-PRP: dropped (:612-613) */
        cs += f[i].p + job->k[f[i].seq] + f[i].n + (uint64_t)(int64_t)job->c[f[i].seq];
        f[kept++] = f[i];
    }
    if (false_factor) *false_factor = bad;
    if (checksum) *checksum = cs;
    return kept;
}

/* ------------------------------------------------------------------------ */
/* Test-input helper (not a restatement): planted factors                   */
/* ------------------------------------------------------------------------ */

/* Finds a term k*b^n+c that the prime p divides, with n in [n_lo, n_hi) and
 * k < kmax of the wanted parity (par: 0 even, 1 odd, -1 either).  Walks n up
 * from n_lo with t_n = -c*b^-n mod p, so k = t_n is the only k < p with
 * p | k*b^n+c; returns 1 with the first hit, 0 when none exists in the range.
 * Lets parity tests place known factors in the p-windows of the benchmark
 * configurations, where random jobs have almost none. */
int or_plant(uint64_t p, uint32_t b, int32_t c, uint32_t n_lo, uint32_t n_hi, uint64_t kmax, int par,
             uint64_t *k_out, uint32_t *n_out)
{
    if (p < 3 || !(p & 1) || b % p == 0 || n_lo >= n_hi) return 0;
    const uint64_t q = or_invert(p), one = (0 - p) % p, r2 = r2_of(p, q, one);
    const uint64_t binv = inv_euclid(b % p, p);
    const uint64_t mbinv = or_m_mul(binv, r2, p, q);
    /* t = -c * binv^n_lo, in Montgomery form */
    uint64_t t = or_powmod(mbinv, n_lo, p, q, one);
    if (c == 1) t = t ? p - t : 0;
    for (uint64_t n = n_lo; n < n_hi; ++n) {
        const uint64_t k = or_m_mul(t, 1, p, q);
        if (k && k < kmax && (par < 0 || (int)(k & 1) == par)) {
            *k_out = k;
            *n_out = (uint32_t)n;
            return 1;
        }
        t = or_m_mul(t, mbinv, p, q);
    }
    return 0;
}

// host.cpp -- host services of the C ABI: ABCD input, factor verification,
// factor file and checkpoint files.  No GPU is touched here, so everything in
// this file is testable on a CPU-only machine.
//
// Formats are the reference's (they are the drop-in interface): the ABCD
// reader follows inputfile.cpp:188-465, the factor line cl_sieve.cpp:624, the
// factor-file re-read cl_sieve.cpp:797-863, the checkpoint workStatus
// cl_sieve.h:21-26 with write_state/read_state cl_sieve.cpp:185-319.  k is
// widened to 64 bits; checkpoints keep the reference's 488-byte layout when
// every k fits its int.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cinttypes>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rs_host.h"

typedef unsigned __int128 u128;

static thread_local char g_err[512];

extern "C" void rs_set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

extern "C" const char *rs_last_error(void) { return g_err; }

extern "C" const char *rs_version(void) { return "rssieve_b200 1.0 (sm_100a)"; }

extern "C" const char *rs_strerror(int code)
{
    switch (code) {
    case RS_OK: return "ok";
    case RS_EARG: return "invalid argument";
    case RS_ECUDA: return "CUDA error";
    case RS_ENOMEM: return "out of memory";
    case RS_EDEVICE: return "device error flag";
    case RS_EIO: return "I/O error";
    case RS_EPARSE: return "parse error";
    case RS_ESTATE: return "invalid checkpoint";
    case RS_EVERIFY: return "factor verification failed";
    case RS_ENODEV: return "no CUDA device";
    case RS_EBUSY: return "no free batch slot";
    default: return "unknown error";
    }
}

// ---------------------------------------------------------------------------
// jobs
// ---------------------------------------------------------------------------

static rs_seqs *seqs_alloc(uint32_t base, uint32_t kcount, uint32_t nmin, uint32_t nmax)
{
    rs_seqs *s = (rs_seqs *)calloc(1, sizeof(rs_seqs));
    if (!s) return nullptr;
    s->base = base;
    s->kcount = kcount;
    s->nmin = nmin;
    s->nmax = nmax;
    s->words_per_seq = ((uint64_t)nmax - nmin + 1 + 31) / 32;
    s->bitmap = (uint32_t *)calloc((size_t)kcount * s->words_per_seq, 4);
    if (!s->bitmap) { free(s); return nullptr; }
    return s;
}

extern "C" void rs_seqs_free(rs_seqs *s)
{
    if (!s) return;
    free(s->bitmap);
    free(s);
}

extern "C" int rs_seqs_validate(const rs_seqs *s)
{
    if (!s) return RS_EARG;
    if (s->base < 2) { rs_set_error("base must be >= 2"); return RS_EARG; }
    if (s->kcount < 1 || s->kcount > RS_MAX_SEQ) { rs_set_error("kcount must be in [1,100]"); return RS_EARG; }
    if (s->nmin > s->nmax) { rs_set_error("nmin > nmax"); return RS_EARG; }
    if (s->words_per_seq != ((uint64_t)s->nmax - s->nmin + 1 + 31) / 32) { rs_set_error("bad words_per_seq"); return RS_EARG; }
    if (!s->bitmap) { rs_set_error("no bitmap"); return RS_EARG; }
    for (uint32_t i = 0; i < s->kcount; ++i) {
        if (s->k[i] == 0) { rs_set_error("k must be > 0 (seq %u)", i); return RS_EARG; }
        if (s->c[i] != 1 && s->c[i] != -1) { rs_set_error("c must be +1 or -1 (seq %u)", i); return RS_EARG; }
    }
    return RS_OK;
}

extern "C" int rs_seqs_create(uint32_t base, uint32_t kcount, const uint64_t *k, const int32_t *c, uint32_t nmin,
                              uint32_t nmax, const uint32_t *bitmap, rs_seqs **out)
{
    if (!out || !k || !c || kcount < 1 || kcount > RS_MAX_SEQ || nmin > nmax) return RS_EARG;
    rs_seqs *s = seqs_alloc(base, kcount, nmin, nmax);
    if (!s) return RS_ENOMEM;
    for (uint32_t i = 0; i < kcount; ++i) { s->k[i] = k[i]; s->c[i] = c[i]; }
    const size_t words = (size_t)kcount * s->words_per_seq;
    if (bitmap) {
        memcpy(s->bitmap, bitmap, words * 4);
    } else {
        const uint64_t bits = (uint64_t)nmax - nmin + 1;
        for (uint32_t i = 0; i < kcount; ++i)
            for (uint64_t b = 0; b < bits; ++b) s->bitmap[i * s->words_per_seq + (b >> 5)] |= 1u << (b & 31);
    }
    int rc = rs_seqs_validate(s);
    if (rc) { rs_seqs_free(s); return rc; }
    *out = s;
    return RS_OK;
}

// Set bits of words[0, n), 64 at a time.  The POPCNT form is chosen at run
// time: without it the compiler's portable popcount made counting a 75 MB
// bitmap take about 35 ms, which rs_job_load pays on every load.
// (inlined into its caller, so that the caller's target decides the instruction)
template <bool HW>
static inline __attribute__((always_inline)) uint64_t count_bits(const uint32_t *words, size_t n)
{
    uint64_t c = 0;
    size_t i = 0;
    for (; i + 2 <= n; i += 2) {
        uint64_t w;
        memcpy(&w, words + i, 8);
        c += (uint64_t)__builtin_popcountll(w);
    }
    for (; i < n; ++i) c += (uint64_t)__builtin_popcount(words[i]);
    return c;
}
__attribute__((target("popcnt"))) static uint64_t count_bits_hw(const uint32_t *words, size_t n)
{
    return count_bits<true>(words, n);
}

extern "C" uint64_t rs_seqs_count(const rs_seqs *s)
{
    if (!s || !s->bitmap) return 0;
    const size_t words = (size_t)s->kcount * s->words_per_seq;
    static const bool hw = __builtin_cpu_supports("popcnt");
    return hw ? count_bits_hw(s->bitmap, words) : count_bits<false>(s->bitmap, words);
}

// ---------------------------------------------------------------------------
// ABCD input -- inputfile.cpp:188-465
// ---------------------------------------------------------------------------

static int parse_header(const char *line, uint64_t *k, uint32_t *b, int32_t *c, uint32_t *n)
{
    // "ABCD k*b^$a+c [n0] // Sieved to p", the tail optional (inputfile.cpp:188-227)
    uint64_t kk = 0, pd = 0;
    uint32_t bb = 0, nn = 0;
    int32_t cc = 0;
    int got = sscanf(line, "ABCD %" SCNu64 "*%" SCNu32 "^$a%" SCNd32 " [%" SCNu32 "] // Sieved to %" SCNu64, &kk, &bb,
                     &cc, &nn, &pd);
    if (got == 5 || got == 4) {
        *k = kk; *b = bb; *c = cc; *n = nn;
        return 1;
    }
    return 0;
}

extern "C" int rs_abcd_parse(const char *text, size_t len, rs_seqs **out)
{
    if (!text || !out) return RS_EARG;
    *out = nullptr;
    std::vector<std::vector<uint32_t>> ns;
    std::vector<uint64_t> ks;
    std::vector<int32_t> cs;
    std::vector<uint32_t> firstN, lastN;
    int64_t gbase = -1;
    int cur = -1;
    uint32_t running = 0;
    uint64_t line_no = 0;
    size_t pos = 0;
    std::string line;
    while (pos < len) {
        size_t e = pos;
        while (e < len && text[e] != '\n') ++e;
        line.assign(text + pos, e - pos);
        if (e < len) line.push_back('\n');
        pos = e + 1;
        ++line_no;
        const char *s = line.c_str();
        while (*s && isspace((unsigned char)*s)) ++s;
        if (*s == '\0' || *s == '#') continue;
        uint32_t delta = 0;
        if (sscanf(line.c_str(), "%" SCNu32, &delta) == 1) {
            if (cur < 0) { rs_set_error("line %" PRIu64 ": delta line before first ABCD header", line_no); return RS_EPARSE; }
            uint32_t r = running + delta;
            if (r < running) { rs_set_error("line %" PRIu64 ": overflow while accumulating n += delta", line_no); return RS_EPARSE; }
            running = r;
            lastN[cur] = running;
            ns[cur].push_back(running);
            continue;
        }
        uint64_t hk;
        uint32_t hb, hn;
        int32_t hc;
        if (!parse_header(line.c_str(), &hk, &hb, &hc, &hn)) { rs_set_error("line %" PRIu64 ": invalid or unrecognised line", line_no); return RS_EPARSE; }
        if (hk == 0) { rs_set_error("line %" PRIu64 ": invalid K (must be > 0)", line_no); return RS_EPARSE; }
        if (hn == 0) { rs_set_error("line %" PRIu64 ": invalid N0 (must be > 0)", line_no); return RS_EPARSE; }
        if (hb < 2) { rs_set_error("line %" PRIu64 ": invalid base in ABCD header (B must be >= 2)", line_no); return RS_EPARSE; }
        if (gbase < 0) gbase = hb;
        else if ((uint32_t)gbase != hb) { rs_set_error("line %" PRIu64 ": mismatched base (B must match all sequences)", line_no); return RS_EPARSE; }
        if (hc != 1 && hc != -1) { rs_set_error("line %" PRIu64 ": not standard form k*b^n+/-1 (c must be +1 or -1)", line_no); return RS_EPARSE; }
        if (ks.size() >= RS_MAX_SEQ) { rs_set_error("line %" PRIu64 ": too many sequences (MAX_SEQUENCES=%d)", line_no, RS_MAX_SEQ); return RS_EPARSE; }
        cur = (int)ks.size();
        ks.push_back(hk);
        cs.push_back(hc);
        firstN.push_back(hn);
        lastN.push_back(hn);
        ns.emplace_back();
        running = hn;
        ns[cur].push_back(hn);
    }
    if (ks.empty()) { rs_set_error("no sequences found in input"); return RS_EPARSE; }
    uint32_t nmin = UINT32_MAX, nmax = 0;
    for (size_t i = 0; i < ks.size(); ++i) {
        nmin = std::min(nmin, firstN[i]);
        nmax = std::max(nmax, lastN[i]);
    }
    if (nmin & 1u) nmin--;                        // bitmap NMIN must be even (inputfile.cpp:405-407)
    rs_seqs *s = seqs_alloc((uint32_t)gbase, (uint32_t)ks.size(), nmin, nmax);
    if (!s) return RS_ENOMEM;
    for (size_t i = 0; i < ks.size(); ++i) {
        s->k[i] = ks[i];
        s->c[i] = cs[i];
        for (uint32_t n : ns[i]) {
            uint64_t off = (uint64_t)n - nmin;
            s->bitmap[i * s->words_per_seq + (off >> 5)] |= 1u << (off & 31);
        }
    }
    *out = s;
    return RS_OK;
}

static int read_file(const char *path, std::string &out)
{
    FILE *f = fopen(path, "rb");
    if (!f) { rs_set_error("unable to open %s: %s", path, strerror(errno)); return RS_EIO; }
    char buf[1 << 16];
    size_t n;
    out.clear();
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
    int bad = ferror(f);
    fclose(f);
    if (bad) { rs_set_error("read error on %s", path); return RS_EIO; }
    return RS_OK;
}

extern "C" int rs_abcd_read(const char *path, rs_seqs **out)
{
    std::string text;
    int rc = read_file(path, text);
    if (rc) return rc;
    rc = rs_abcd_parse(text.data(), text.size(), out);
    if (rc == RS_EPARSE) {
        std::string m = std::string(path) + ":" + g_err;
        rs_set_error("%s", m.c_str());
    }
    return rc;
}

// ---------------------------------------------------------------------------
// verification -- verify_factor.c:100-181, arithmetic restated
// ---------------------------------------------------------------------------

static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)(((u128)a * b) % p); }

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p)
{
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

static bool sprp(uint64_t n, uint64_t a)
{
    uint64_t d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; ++s; }
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) return true;
    for (int i = 1; i < s; ++i) {
        x = mulmod(x, x, n);
        if (x == n - 1) return true;
    }
    return false;
}

extern "C" int rs_is_prime(uint64_t n)
{
    static const uint64_t bases[7] = {2, 325, 9375, 28178, 450775, 9780504, 1795265022};
    if (n < 2) return 0;
    if (n % 2 == 0) return n == 2;
    if (n < 9) return n > 1;
    for (uint64_t b : bases) {
        uint64_t a = b % n;
        if (a == 0) continue;
        if (!sprp(n, a)) return 0;
    }
    return 1;
}

extern "C" int rs_verify_factor(uint64_t p, uint64_t k, uint32_t n, int32_t c, uint32_t base)
{
    if (!rs_is_prime(p) || p < 3) return -1;
    uint64_t a = mulmod(k % p, powmod(base, n, p), p);     // k*b^n mod p
    if (a == 1 && c == -1) return 1;
    if (a == p - 1 && c == 1) return 1;
    return 0;
}

// ---------------------------------------------------------------------------
// factor file -- cl_sieve.cpp:515-643, 738-863
// ---------------------------------------------------------------------------

extern "C" int rs_format_factor(const rs_seqs *s, const rs_factor *f, char *buf, size_t len)
{
    if (!s || !f || !buf || f->seq >= s->kcount) return RS_EARG;
    int w = snprintf(buf, len, "%" PRIu64 " | %" PRIu64 "*%u^%u%+d\n", f->p, s->k[f->seq], s->base, f->n, s->c[f->seq]);
    return (w > 0 && (size_t)w < len) ? RS_OK : RS_EARG;
}

extern "C" int rs_factors_file_apply(const char *path, rs_seqs *s, uint64_t *lines)
{
    if (!path || !s) return RS_EARG;
    FILE *fp = fopen(path, "r");
    if (!fp) { rs_set_error("Cannot open %s", path); return RS_EIO; }
    char line[512];
    uint64_t ln = 0;
    while (fgets(line, sizeof line, fp)) {
        ++ln;
        uint64_t p, k;
        uint32_t b, n, cchk;
        char bar, sign, extra;
        int fields = sscanf(line, " %" SCNu64 " %c %" SCNu64 " * %" SCNu32 " ^ %" SCNu32 " %c %" SCNu32 " %c", &p, &bar,
                            &k, &b, &n, &sign, &cchk, &extra);
        if (fields != 7 || bar != '|' || (sign != '+' && sign != '-') || cchk != 1 || b != s->base) {
            fclose(fp);
            rs_set_error("Invalid line read in factors file %" PRIu64 ": %s", ln, line);
            return RS_EPARSE;
        }
        // mark_factor_used, inputfile.cpp:89-107
        const int32_t c = (sign == '+') ? 1 : -1;
        for (uint32_t i = 0; i < s->kcount; ++i) {
            if (s->k[i] == k && s->c[i] == c) {
                if (n >= s->nmin && n <= s->nmax) {
                    uint64_t off = (uint64_t)n - s->nmin;
                    s->bitmap[i * s->words_per_seq + (off >> 5)] &= ~(1u << (off & 31));
                }
                break;
            }
        }
    }
    fclose(fp);
    if (lines) *lines = ln;
    return RS_OK;
}

extern "C" int rs_factors_commit(const char *path, const rs_seqs *s, rs_factor *f, size_t n, rs_state *st)
{
    if (!s || (n && !f) || !st) return RS_EARG;
    // factorcompare, cl_sieve.cpp:515-527: ascending p, then n
    std::sort(f, f + n, [](const rs_factor &a, const rs_factor &b) {
        return a.p != b.p ? a.p < b.p : a.n < b.n;
    });
    std::vector<int> res(n);
    for (size_t i = 0; i < n; ++i) {
        if (f[i].seq >= s->kcount) { rs_set_error("factor with bad sequence index"); return RS_EARG; }
        res[i] = rs_verify_factor(f[i].p, s->k[f[i].seq], f[i].n, s->c[f[i].seq], s->base);
        if (res[i] == 0) {
            rs_set_error("CPU factor verification failed!  %" PRIu64 " is not a factor of %" PRIu64 "*%u^%u%+d", f[i].p,
                         s->k[f[i].seq], s->base, f[i].n, s->c[f[i].seq]);
            return RS_EVERIFY;
        }
    }
    FILE *out = nullptr;
    for (size_t i = 0; i < n; ++i) {
        if (res[i] < 0) continue;                  // composite p (cannot come from this library's prime generator)
        if (!out) {
            out = fopen(path, "a");
            if (!out) { rs_set_error("Cannot open %s", path); return RS_EIO; }
        }
        char line[128];
        rs_format_factor(s, &f[i], line, sizeof line);
        if (fputs(line, out) < 0) { fclose(out); rs_set_error("Cannot write to %s", path); return RS_EIO; }
        st->factorcount++;
        st->checksum += f[i].p + s->k[f[i].seq] + f[i].n + (uint64_t)(int64_t)s->c[f[i].seq];
    }
    if (out && fclose(out) != 0) { rs_set_error("Cannot write to %s", path); return RS_EIO; }
    return RS_OK;
}

extern "C" int rs_factors_finalize(const char *path, const rs_state *st)
{
    if (!path || !st) return RS_EARG;
    if (st->factorcount) {
        FILE *f = fopen(path, "r");
        if (!f) { rs_set_error("Cannot open %s", path); return RS_EIO; }
        char line[256];
        uint64_t lc = 0;
        while (fgets(line, sizeof line, f)) ++lc;
        fclose(f);
        if (lc < st->factorcount) { rs_set_error("ERROR: Missing factors in %s", path); return RS_EIO; }
    }
    FILE *f = fopen(path, "a");
    if (!f) { rs_set_error("Cannot open %s", path); return RS_EIO; }
    if (!st->factorcount && fputs("no factors\n", f) < 0) { fclose(f); return RS_EIO; }
    fclose(f);
    return RS_OK;
}

// ---------------------------------------------------------------------------
// checkpoints -- cl_sieve.h:21-26, cl_sieve.cpp:185-319
// ---------------------------------------------------------------------------

// the reference's 488-byte workStatus
struct WorkStatusV1 {
    uint64_t pmin, pmax, p, checksum, primecount, factorcount, last_trickle, state_sum, dupcount;
    uint32_t nmin, nmax, base;
    int32_t kcount;
    int32_t klist[RS_MAX_SEQ];
};
static_assert(sizeof(WorkStatusV1) == 488, "workStatus layout");

// versioned layout for k >= 2^31
struct WorkStatusV2 {
    char magic[8];                  // "RSB200\0\2"
    uint64_t pmin, pmax, p, checksum, primecount, factorcount, last_trickle, state_sum, dupcount;
    uint32_t nmin, nmax, base;
    int32_t kcount;
    uint64_t k[RS_MAX_SEQ];
    int8_t c[RS_MAX_SEQ];
    uint8_t pad[4];
};
static const char kMagicV2[8] = {'R', 'S', 'B', '2', '0', '0', 0, 2};

static bool fits_v1(const rs_seqs *s)
{
    for (uint32_t i = 0; i < s->kcount; ++i)
        if (s->k[i] > 0x7FFFFFFFull) return false;
    return true;
}

template <class W>
static uint64_t scalar_sum(const W &w)
{
    return w.base + w.pmin + w.pmax + w.p + w.checksum + w.primecount + w.factorcount + w.last_trickle + w.nmin +
           w.nmax + (uint64_t)(int64_t)w.kcount + w.dupcount;
}

extern "C" int rs_state_write(const char *path, const rs_state *st, const rs_seqs *s)
{
    if (!path || !st || !s) return RS_EARG;
    FILE *out = fopen(path, "wb");
    if (!out) { rs_set_error("Cannot open %s", path); return RS_EIO; }
    size_t ok;
    if (fits_v1(s)) {
        WorkStatusV1 w;
        memset(&w, 0, sizeof w);
        w.pmin = st->pmin; w.pmax = st->pmax; w.p = st->p; w.checksum = st->checksum;
        w.primecount = st->primecount; w.factorcount = st->factorcount; w.last_trickle = st->last_trickle;
        w.dupcount = st->dupcount; w.nmin = s->nmin; w.nmax = s->nmax; w.base = s->base; w.kcount = (int32_t)s->kcount;
        w.state_sum = scalar_sum(w);
        for (uint32_t i = 0; i < s->kcount; ++i) {
            w.klist[i] = s->c[i] > 0 ? (int32_t)s->k[i] : -(int32_t)s->k[i];
            w.state_sum += (uint64_t)(int64_t)w.klist[i];
        }
        ok = fwrite(&w, sizeof w, 1, out);
    } else {
        WorkStatusV2 w;
        memset(&w, 0, sizeof w);
        memcpy(w.magic, kMagicV2, 8);
        w.pmin = st->pmin; w.pmax = st->pmax; w.p = st->p; w.checksum = st->checksum;
        w.primecount = st->primecount; w.factorcount = st->factorcount; w.last_trickle = st->last_trickle;
        w.dupcount = st->dupcount; w.nmin = s->nmin; w.nmax = s->nmax; w.base = s->base; w.kcount = (int32_t)s->kcount;
        w.state_sum = scalar_sum(w);
        for (uint32_t i = 0; i < s->kcount; ++i) {
            w.k[i] = s->k[i];
            w.c[i] = (int8_t)s->c[i];
            w.state_sum += w.k[i] + (uint64_t)(int64_t)w.c[i];
        }
        ok = fwrite(&w, sizeof w, 1, out);
    }
    if (ok != 1) { fclose(out); rs_set_error("Cannot write checkpoint to %s", path); return RS_EIO; }
    if (fclose(out) != 0) { rs_set_error("Cannot write checkpoint to %s", path); return RS_EIO; }
    return RS_OK;
}

// st is in/out: on entry st->pmin and st->pmax are the run's p-range, and a
// file written for another range is rejected like one for another job (the
// reference's read_state compares base, pmin, pmax, nmin, nmax and kcount
// before it looks at the checksum, cl_sieve.cpp:236-242,266-272).
extern "C" int rs_state_read(const char *path, rs_state *st, const rs_seqs *s)
{
    if (!path || !st || !s) return RS_EARG;
    const uint64_t want_pmin = st->pmin, want_pmax = st->pmax;
    std::string data;
    FILE *f = fopen(path, "rb");
    if (!f) { rs_set_error("no checkpoint %s", path); return RS_EIO; }
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) data.append(buf, n);
    fclose(f);
    auto fill = [&](const auto &w) {
        st->pmin = w.pmin; st->pmax = w.pmax; st->p = w.p; st->checksum = w.checksum; st->primecount = w.primecount;
        st->factorcount = w.factorcount; st->last_trickle = w.last_trickle; st->dupcount = w.dupcount;
    };
    if (data.size() >= sizeof(WorkStatusV2) && memcmp(data.data(), kMagicV2, 8) == 0) {
        WorkStatusV2 w;
        memcpy(&w, data.data(), sizeof w);
        if (w.base != s->base || w.pmin != want_pmin || w.pmax != want_pmax || w.nmin != s->nmin ||
            w.nmax != s->nmax || w.kcount != (int32_t)s->kcount) {
            rs_set_error("Invalid checkpoint file %s", path);
            return RS_ESTATE;
        }
        uint64_t sum = scalar_sum(w);
        for (int32_t i = 0; i < w.kcount; ++i) {
            sum += w.k[i] + (uint64_t)(int64_t)w.c[i];
            if (w.k[i] != s->k[i] || w.c[i] != s->c[i]) { rs_set_error("Invalid checkpoint file %s", path); return RS_ESTATE; }
        }
        if (sum != w.state_sum) { rs_set_error("Checksum error in %s", path); return RS_ESTATE; }
        fill(w);
        return RS_OK;
    }
    if (data.size() < sizeof(WorkStatusV1)) { rs_set_error("Cannot parse %s", path); return RS_ESTATE; }
    WorkStatusV1 w;
    memcpy(&w, data.data(), sizeof w);
    if (w.base != s->base || w.pmin != want_pmin || w.pmax != want_pmax || w.nmin != s->nmin || w.nmax != s->nmax ||
        w.kcount != (int32_t)s->kcount) {
        rs_set_error("Invalid checkpoint file %s", path);
        return RS_ESTATE;
    }
    uint64_t sum = scalar_sum(w);
    for (int32_t i = 0; i < w.kcount; ++i) {
        sum += (uint64_t)(int64_t)w.klist[i];
        const int64_t want = s->c[i] > 0 ? (int64_t)s->k[i] : -(int64_t)s->k[i];
        if ((int64_t)w.klist[i] != want) { rs_set_error("Invalid checkpoint file %s", path); return RS_ESTATE; }
    }
    if (sum != w.state_sum) { rs_set_error("Checksum error in %s", path); return RS_ESTATE; }
    fill(w);
    return RS_OK;
}

extern "C" int rs_state_resume(const char *path_a, const char *path_b, rs_state *st, const rs_seqs *s, int *which)
{
    if (!st || !s) return RS_EARG;
    rs_state a = *st, b = *st;             // both carry the run's pmin/pmax into rs_state_read
    bool ga = rs_state_read(path_a, &a, s) == RS_OK;
    bool gb = rs_state_read(path_b, &b, s) == RS_OK;
    if (ga && gb) {
        if (a.p > b.p) gb = false;            // newest wins; a tie goes to B (cl_sieve.cpp:289-295)
        else ga = false;
    }
    if (ga) { *st = a; if (which) *which = 0; return 1; }
    if (gb) { *st = b; if (which) *which = 1; return 1; }
    return 0;
}

// cli.cpp -- the rssieve command line, a drop-in for the reference binary.
//
// Same interface as main.cpp:25-134 and cl_sieve.cpp:975-1451: -p P0 -P P1
// (3 <= p < P < 2^64, [p,P) half-open, 'e' exponents accepted), -i ABCD file,
// -f factor file (default psp_sr2sieve.out), -h help; unknown tokens are
// ignored; -s reports that the self test is not implemented.  The device is
// gpu_device_num from init_data.xml when present, else 0 (README.md:45-58).
// Checkpoints alternate stateA.ckp / stateB.ckp every 60 s; on resume the
// factor file is re-read to clear already reported terms.  Without BOINC the
// fraction-done / trickle calls of the reference are not needed.
#include <cerrno>
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "rssieve_b200.h"

#define STATE_A "stateA.ckp"
#define STATE_B "stateB.ckp"

static void die(const char *what, int rc)
{
    fprintf(stderr, "%s: %s (%s)\n", what, rs_strerror(rc), rs_last_error());
    printf("%s: %s (%s)\n", what, rs_strerror(rc), rs_last_error());
    exit(EXIT_FAILURE);
}

static void help()
{
    printf("rssieve_b200: a B200 Riesel Sierpinski sieve for multiple sequences k*b^n+-1 using the BSGS algorithm.\n");
    printf("Program usage:\n");
    printf("-p #\t\t\tStarting prime factor p\n");
    printf("-P #\t\t\tEnd prime factor P\n");
    printf("\t\t\tP range is 3 <= -p < -P < 2^64, [-p, -P) exclusive\n");
    printf("-i inputfile\t\tUse specified sr2sieve ABCD input file with a maximum of 100 sequences\n");
    printf("-f factorfile\t\tOverride default factor file name (psp_sr2sieve.out) with specified file name.\n");
    printf("-h\t\t\tPrint this help\n");
    exit(EXIT_FAILURE);
}

// parse_uint64 of main.cpp:40-70: decimal with an optional e exponent
static int parse_u64(uint64_t *res, const char *str, uint64_t lo, uint64_t hi)
{
    if (!str || !*str) return -1;
    char *tail;
    errno = 0;
    uint64_t num = strtoull(str, &tail, 10);
    if (errno) return -2;
    if (*tail == 'e' || *tail == 'E') {
        ++tail;
        errno = 0;
        uint64_t ex = strtoul(tail, &tail, 10);
        if (errno) return -2;
        if (*tail) return -1;
        while (ex-- > 0) {
            if (num > hi / 10) return -2;
            num *= 10;
        }
    } else if (*tail) {
        return -1;
    }
    if (num < lo || num > hi) return -2;
    *res = num;
    return 0;
}

static bool is_perfect_power(uint64_t b, uint32_t *root)
{
    // cl_sieve.cpp:646-658
    for (uint64_t a = 2; a * a <= b; ++a) {
        uint64_t p = a * a;
        while (p < b) p *= a;
        if (p == b) { *root = (uint32_t)a; return true; }
    }
    return false;
}

static int device_from_init_data()
{
    FILE *f = fopen("init_data.xml", "r");
    if (!f) return 0;
    char buf[4096];
    size_t n = fread(buf, 1, sizeof buf - 1, f);
    fclose(f);
    buf[n] = 0;
    const char *t = strstr(buf, "<gpu_device_num>");
    if (!t) return 0;
    return atoi(t + strlen("<gpu_device_num>"));
}

int main(int argc, char **argv)
{
    uint64_t pmin = 0, pmax = 0;
    const char *input = nullptr, *factor_file = "psp_sr2sieve.out";
    bool test = false;
    fprintf(stderr, "\n%s\n", rs_version());
    fprintf(stderr, "Command line: ");
    for (int i = 0; i < argc; ++i) fprintf(stderr, "%s ", argv[i]);
    fprintf(stderr, "\n");
    for (int i = 1; i < argc; ++i) {
        const char *t = argv[i];
        if (!strcmp(t, "-p") && i + 1 < argc) {
            if (parse_u64(&pmin, argv[++i], 3, UINT64_MAX)) { fprintf(stderr, "Invalid value for -p: %s\n", argv[i]); printf("Invalid value for -p: %s\n", argv[i]); }
        } else if (!strcmp(t, "-P") && i + 1 < argc) {
            if (parse_u64(&pmax, argv[++i], 4, UINT64_MAX)) { fprintf(stderr, "Invalid value for -P: %s\n", argv[i]); printf("Invalid value for -P: %s\n", argv[i]); }
        } else if (!strcmp(t, "-i") && i + 1 < argc) {
            input = argv[++i];
        } else if (!strcmp(t, "-f") && i + 1 < argc) {
            factor_file = argv[++i];
        } else if (!strcmp(t, "-s")) {
            test = true;
        } else if (!strcmp(t, "-h")) {
            help();
        }
        // unknown flags are ignored (main.cpp:131)
    }
    if (test) {
        fprintf(stderr, "self test not implemented yet!\n");
        printf("self test not implemented yet!\n");
        return EXIT_FAILURE;
    }
    if (!input) {
        printf("ERROR: no input file specified!\n");
        fprintf(stderr, "ERROR: no input file specified!\n");
        return EXIT_FAILURE;
    }
    rs_seqs *seqs = nullptr;
    int rc = rs_abcd_read(input, &seqs);
    if (rc) die("reading input", rc);
    printf("Sequences read: %u\nBase = %u\n", seqs->kcount, seqs->base);
    fprintf(stderr, "Sequences read: %u\nBase = %u\n", seqs->kcount, seqs->base);
    uint32_t root;
    if (is_perfect_power(seqs->base, &root)) {
        printf("\nerror: selected base %u is a perfect power of base %u!\n", seqs->base, root);
        fprintf(stderr, "error: selected base %u is a perfect power of base %u!\n", seqs->base, root);
        return EXIT_FAILURE;
    }
    if (!pmin || !pmax) {
        printf("\n-p and -P arguments are required\nuse -h for help\n");
        fprintf(stderr, "-p and -P arguments are required\n");
        return EXIT_FAILURE;
    }
    if (pmin > pmax) {
        printf("pmin <= pmax is required\nuse -h for help\n");
        fprintf(stderr, "pmin <= pmax is required\n");
        return EXIT_FAILURE;
    }
    rs_state st;
    memset(&st, 0, sizeof st);
    st.pmin = pmin;
    st.pmax = pmax;
    st.p = pmin;
    printf("Starting sieve at p: %" PRIu64 " n: %u\nStopping sieve at P: %" PRIu64 " N: %u\n", pmin, seqs->nmin, pmax,
           seqs->nmax);
    bool write_a_next = true;
    int which = 0;
    if (rs_state_resume(STATE_A, STATE_B, &st, seqs, &which) == 1) {
        write_a_next = (which == 1);
        printf("Resuming from checkpoint in %s\nCurrent p: %" PRIu64 "\n", which ? STATE_B : STATE_A, st.p);
        fprintf(stderr, "Resuming from checkpoint, current p: %" PRIu64 "\n", st.p);
        if (st.p == st.pmax) {
            printf("Workunit complete.\n");
            fprintf(stderr, "Workunit complete.\n");
            return EXIT_SUCCESS;
        }
        uint64_t lines = 0;
        rc = rs_factors_file_apply(factor_file, seqs, &lines);
        if (rc) die("reading factor file", rc);
        if (lines < st.factorcount) {
            fprintf(stderr, "ERROR: Missing factors in %s !!!\n", factor_file);
            printf("ERROR: Missing factors in %s !!!\n", factor_file);
            return EXIT_FAILURE;
        }
        printf("Updated bitmap with %" PRIu64 " factors from %s\n", lines, factor_file);
    } else {
        memset(&st, 0, sizeof st);
        st.pmin = pmin;
        st.pmax = pmax;
        st.p = pmin;
        FILE *f = fopen(factor_file, "w");
        if (!f) { fprintf(stderr, "Cannot open %s !!!\n", factor_file); return EXIT_FAILURE; }
        fclose(f);
        st.last_trickle = (uint64_t)time(nullptr);
    }
    rs_ctx *ctx = nullptr;
    rc = rs_ctx_create(device_from_init_data(), &ctx);
    if (rc) die("device set-up", rc);
    rc = rs_job_load(ctx, seqs);
    if (rc) die("job upload", rc);
    std::vector<rs_factor> fbuf;
    auto flush = [&]() {
        size_t n = 0;
        int r = rs_factors_fetch(ctx, nullptr, 0, &n);
        if (r && r != RS_EARG) die("fetching factors", r);
        fbuf.resize(n ? n : 1);
        r = rs_factors_fetch(ctx, fbuf.data(), fbuf.size(), &n);
        if (r) die("fetching factors", r);
        if (n) printf("Verifying %zu factors on CPU...\n", n);
        r = rs_factors_commit(factor_file, seqs, fbuf.data(), n, &st);
        if (r) die("verifying factors", r);
        // checkpoint, alternating A/B (write_state, cl_sieve.cpp:185-217)
        r = rs_state_write(write_a_next ? STATE_A : STATE_B, &st, seqs);
        if (r == RS_OK) write_a_next = !write_a_next;
        else fprintf(stderr, "Cannot write checkpoint. Continuing...\n");
        printf("Checkpoint, current p: %" PRIu64 "\n", st.p);
    };
    printf("Starting Sieve...\n");
    fprintf(stderr, "Starting Sieve...\n");
    auto t0 = std::chrono::steady_clock::now();
    auto last_ckpt = t0;
    uint64_t width = 1ull << 28;
    while (st.p < st.pmax) {
        uint64_t stop = (st.pmax - st.p > width) ? st.p + width : st.pmax;
        auto c0 = std::chrono::steady_clock::now();
        rs_counters d;
        rc = rs_run_range(ctx, st.p, stop, &d);
        if (rc) die("sieve", rc);
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        st.primecount += d.primes;
        st.dupcount += d.dups;
        st.p = stop;
        // aim for a few seconds per device call
        if (secs < 1.0 && width < (1ull << 40)) width *= 2;
        else if (secs > 8.0 && width > (1ull << 24)) width /= 2;
        auto now = std::chrono::steady_clock::now();
        if (std::chrono::duration<double>(now - last_ckpt).count() > 60.0) {
            flush();
            last_ckpt = now;
        }
    }
    st.p = st.pmax;
    flush();
    rc = rs_factors_finalize(factor_file, &st);
    if (rc) die("finalizing factor file", rc);
    double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fprintf(stderr, "Sieve complete.\nfactors %" PRIu64 ", prime count %" PRIu64 ", duplicate factors %" PRIu64 "\n",
            st.factorcount, st.primecount, st.dupcount);
    printf("Sieve finished in %d sec.\n", (int)total);
    printf("factors %" PRIu64 ", prime count %" PRIu64 ", checksum %016" PRIX64 ", duplicate factors %" PRIu64 "\n",
           st.factorcount, st.primecount, st.checksum, st.dupcount);
    rs_ctx_destroy(ctx);
    rs_seqs_free(seqs);
    return EXIT_SUCCESS;
}

// engine.cu -- device context, job upload and the segment loop behind the C ABI.
//
// Replaces the host orchestration of cl_sieve.cpp:975-1451 (buffer set-up,
// profileGPU's segment sizing, the main loop clearn -> addsmallprimes ->
// getsegprimes -> setup -> sort -> giantfull/giantparity) and the OpenCL
// plumbing of simpleCL.c.  One CUDA stream per context; the host waits once
// per segment for the prime count, then launches set-up and BSGS over chunks
// of primes.  Device counters and the factor buffer accumulate across calls.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "rs_internal.h"
#include "rs_host.h"

using namespace rs;

struct rs_ctx {
    int device = -1;
    int sms = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    // sieving primes (odd primes < 2^16)
    u32 *d_sp = nullptr;
    u32 nsp = 0;
    // segment buffers
    u64 *d_cands = nullptr;
    u64 *d_mid = nullptr;       // base-2 strong probable primes awaiting the Lucas pass (cand_cap)
    u32 cand_cap = 0;
    u64 *d_primes = nullptr;
    u32 prime_cap = 0;
    u32 *d_ctrs = nullptr;      // [0] sieve survivors, [1] primes, [2] BSGS work counter, [3] factor count, [4] mid list
    u32 *d_err = nullptr;
    u64 *d_stats = nullptr;
    u32 *h_pin = nullptr;       // pinned: ctrs[4], err
    // per-chunk prime records
    u32 chunk_cap = 0;
    PrimeHdr *d_hdr = nullptr;
    void *d_aux = nullptr;
    u64 *d_tabs = nullptr;
    u64 *d_tgt = nullptr;
    unsigned short *d_meta = nullptr;
    // job
    bool job_loaded = false;
    JobDev h_job;
    JobDev *d_job = nullptr;
    u32 *d_bitmap = nullptr;
    size_t bitmap_words = 0;
    FactorRec *d_factors = nullptr;
    u32 factor_cap = 0;
    size_t bitmap_alloc = 0, factor_alloc = 0;   // capacities (words, records): buffers only grow
    u64 primes_total = 0;
    // BSGS geometry: forced (index into BSGS_GEOMS) or chosen per job by the tuner
    int geom_forced = -1;
    int geom = 0;
    bool tuning = false;
    int tune_cand[NGEOM];
    int tune_ncand = 0, tune_next = 0;
    double tune_ms[NGEOM];
    u64 tune_primes[NGEOM];
    std::vector<int> chunk_geom;
    // bounded device waits (rs_set_wait_limit)
    u32 wait_bound = 0;
    u32 test_stall = 0;
    // timing of the last rs_run_range
    std::vector<cudaEvent_t> ev;
    double last_bsgs_ms = 0, last_total_ms = 0;
    u32 last_bsgs_launches = 0, last_kernel_launches = 0;
};

#define CU(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) {                                                  \
            rs_set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return RS_ECUDA;                                                      \
        }                                                                         \
    } while (0)

static void free_job(rs_ctx *c)
{
    cudaFree(c->d_bitmap);
    cudaFree(c->d_factors);
    c->d_bitmap = nullptr;
    c->d_factors = nullptr;
    c->bitmap_alloc = c->factor_alloc = 0;
    c->job_loaded = false;
}

std::vector<u32> rs_small_primes()
{
    std::vector<u32> v;
    std::vector<char> comp(65536, 0);
    for (u32 i = 2; i < 65536; ++i) {
        if (comp[i]) continue;
        if (i > 2) v.push_back(i);
        for (u64 j = (u64)i * i; j < 65536; j += i) comp[j] = 1;
    }
    return v;
}

extern "C" int rs_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" void rs_ctx_destroy(rs_ctx *c)
{
    if (!c) return;
    if (c->device >= 0) cudaSetDevice(c->device);
    free_job(c);
    cudaFree(c->d_sp);
    cudaFree(c->d_cands);
    cudaFree(c->d_mid);
    cudaFree(c->d_primes);
    cudaFree(c->d_ctrs);
    cudaFree(c->d_err);
    cudaFree(c->d_stats);
    cudaFree(c->d_hdr);
    cudaFree(c->d_aux);
    cudaFree(c->d_tabs);
    cudaFree(c->d_tgt);
    cudaFree(c->d_meta);
    cudaFree(c->d_job);
    if (c->h_pin) cudaFreeHost(c->h_pin);
    for (auto e : c->ev) cudaEventDestroy(e);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

extern "C" int rs_ctx_create(int device, rs_ctx **out)
{
    if (!out) return RS_EARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        rs_set_error("no CUDA device available");
        return RS_ENODEV;
    }
    if (device < 0 || device >= ndev) {
        rs_set_error("device %d out of range (%d devices)", device, ndev);
        return RS_EARG;
    }
    rs_ctx *c = new rs_ctx();
    c->device = device;
    auto fail = [&](int r) { rs_ctx_destroy(c); return r; };
    if (cudaSetDevice(device) != cudaSuccess) return fail((rs_set_error("cudaSetDevice failed"), RS_ECUDA));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(RS_ECUDA);
    c->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) return fail(RS_ECUDA);
    c->stream = c->own;
    std::vector<u32> sp = rs_small_primes();
    c->nsp = (u32)sp.size();
    c->cand_cap = 1u << 24;
    c->prime_cap = 1u << 24;
    c->chunk_cap = 1u << 17;
    if (cudaMalloc(&c->d_sp, sp.size() * 4) != cudaSuccess ||
        cudaMalloc(&c->d_cands, (size_t)c->cand_cap * 8) != cudaSuccess ||
        cudaMalloc(&c->d_mid, (size_t)c->cand_cap * 8) != cudaSuccess ||
        cudaMalloc(&c->d_primes, (size_t)c->prime_cap * 8) != cudaSuccess ||
        cudaMalloc(&c->d_ctrs, 16 * 4) != cudaSuccess || cudaMalloc(&c->d_err, 4) != cudaSuccess ||
        cudaMalloc(&c->d_stats, ST_COUNT * 8) != cudaSuccess ||
        cudaMalloc(&c->d_hdr, (size_t)c->chunk_cap * sizeof(PrimeHdr)) != cudaSuccess ||
        cudaMalloc(&c->d_aux, (size_t)c->chunk_cap * setup_aux_bytes()) != cudaSuccess ||
        cudaMalloc(&c->d_tabs, (size_t)c->chunk_cap * TABS * 8) != cudaSuccess ||
        cudaMalloc(&c->d_tgt, (size_t)c->chunk_cap * KSTRIDE * 8) != cudaSuccess ||
        cudaMalloc(&c->d_meta, (size_t)c->chunk_cap * KSTRIDE * 2) != cudaSuccess ||
        cudaMalloc(&c->d_job, sizeof(JobDev)) != cudaSuccess ||
        cudaMallocHost(&c->h_pin, 64) != cudaSuccess) {
        rs_set_error("device allocation failed");
        return fail(RS_ENOMEM);
    }
    if (cudaMemcpy(c->d_sp, sp.data(), sp.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(c->d_ctrs, 0, 64) != cudaSuccess || cudaMemset(c->d_err, 0, 4) != cudaSuccess ||
        cudaMemset(c->d_stats, 0, ST_COUNT * 8) != cudaSuccess)
        return fail(RS_ECUDA);
    if (bsgs_prepare() != cudaSuccess) {
        rs_set_error("BSGS kernel needs %zu B of shared memory", bsgs_smem_bytes(0));
        return fail(RS_ECUDA);
    }
    *out = c;
    return RS_OK;
}

extern "C" int rs_ctx_set_stream(rs_ctx *c, void *stream)
{
    if (!c) return RS_EARG;
    c->stream = stream ? (cudaStream_t)stream : c->own;
    return RS_OK;
}

// Jobs of one shape share a tuned geometry (a reloaded or resumed job skips
// tuning), across every context and batch on the device.
static std::mutex g_tuned_mu;
static std::map<std::pair<int, u64>, int> g_tuned;

int rs::tuned_geom_get(int device, u64 shape)
{
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    auto it = g_tuned.find({device, shape});
    return it == g_tuned.end() ? -1 : it->second;
}

void rs::tuned_geom_put(int device, u64 shape, int geom)
{
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_tuned[{device, shape}] = geom;
}

static u64 job_shape(const rs_ctx *c)
{
    return job_shape_key(c->h_job.base, c->h_job.kcount, c->h_job.L);
}

// Starts the per-job tuner: the candidates are the geometries whose model cost
// is within 2x of the model's best; the first chunks cycle through them.
static void tune_start(rs_ctx *c)
{
    c->tune_ncand = 0;
    c->tune_next = 0;
    for (int g = 0; g < NGEOM; ++g) { c->tune_ms[g] = 0; c->tune_primes[g] = 0; }
    if (c->geom_forced >= 0) {
        c->geom = c->geom_forced;
        c->tuning = false;
        return;
    }
    double best = 1e300;
    int gb = 0;
    for (int g = 0; g < NGEOM; ++g) {
        double v = geom_model_cost(g, c->h_job.kcount, c->h_job.L);
        if (v < best) { best = v; gb = g; }
    }
    for (int g = 0; g < NGEOM; ++g)
        if (geom_model_cost(g, c->h_job.kcount, c->h_job.L) <= 2.0 * best) c->tune_cand[c->tune_ncand++] = g;
    c->geom = gb;
    c->tuning = (c->tune_ncand > 1);
    const int known = tuned_geom_get(c->device, job_shape(c));
    if (known >= 0) {
        c->geom = known;
        c->tuning = false;
    }
}

// Records one chunk's BSGS time; ends tuning once every candidate has timed at
// least 2^18 primes, keeping the fastest per prime.
static void tune_record(rs_ctx *c, int g, u32 primes, float ms)
{
    if (!c->tuning || primes < 32768) return;
    c->tune_ms[g] += ms;
    c->tune_primes[g] += primes;
    for (int i = 0; i < c->tune_ncand; ++i)
        if (c->tune_primes[c->tune_cand[i]] < (1u << 18)) return;
    double best = 1e300;
    for (int i = 0; i < c->tune_ncand; ++i) {
        const int gi = c->tune_cand[i];
        const double v = c->tune_ms[gi] / (double)c->tune_primes[gi];
        if (v < best) { best = v; c->geom = gi; }
    }
    c->tuning = false;
    tuned_geom_put(c->device, job_shape(c), c->geom);
}

extern "C" int rs_set_baby_steps(rs_ctx *c, uint32_t q)
{
    if (!c) return RS_EARG;
    if (q != 0 && geom_index(q) < 0) {
        rs_set_error("baby-step count %u is not one of 1024, 2048, 4096, 8192, 16384 (or 0 for automatic)", q);
        return RS_EARG;
    }
    c->geom_forced = q ? geom_index(q) : -1;
    if (c->job_loaded) tune_start(c);
    return RS_OK;
}

extern "C" int rs_set_wait_limit(rs_ctx *c, uint32_t tries, int test_stall)
{
    if (!c || test_stall < 0 || test_stall > 1) return RS_EARG;
    c->wait_bound = tries;
    c->test_stall = (u32)test_stall;
    return RS_OK;
}

extern "C" int rs_get_baby_steps(rs_ctx *c, uint32_t *q, int *tuning)
{
    if (!c || !q) return RS_EARG;
    *q = BSGS_GEOMS[c->geom].q;
    if (tuning) *tuning = c->tuning ? 1 : 0;
    return RS_OK;
}

// Device record of a job: sequences and n-range (bitmap pointer left null).
void jobdev_from_seqs(const rs_seqs *s, JobDev *out)
{
    memset(out, 0, sizeof *out);
    out->base = s->base;
    out->kcount = s->kcount;
    out->nmin = s->nmin;
    out->nmax = s->nmax;
    out->L = s->nmax - s->nmin + 1;
    out->words = (u32)s->words_per_seq;
    for (u32 i = 0; i < s->kcount; ++i) {
        out->k[i] = s->k[i];
        out->c[i] = s->c[i];
    }
}

extern "C" int rs_job_load(rs_ctx *c, const rs_seqs *s)
{
    if (!c || !s) return RS_EARG;
    int rc = rs_seqs_validate(s);
    if (rc) return rc;
    CU(cudaSetDevice(c->device));
    c->job_loaded = false;
    JobDev J;
    jobdev_from_seqs(s, &J);
    c->bitmap_words = (size_t)s->kcount * s->words_per_seq;
    uint64_t cand = rs_seqs_count(s);
    c->factor_cap = (u32)std::min<uint64_t>(cand + 1, 0xFFFFFFF0ull);
    // the buffers of an earlier job are reused when large enough: a fresh
    // allocation synchronises the device and maps new memory, which costs more
    // than the upload itself when jobs are loaded one after another
    if (c->bitmap_words > c->bitmap_alloc || c->factor_cap > c->factor_alloc) {
        const size_t bw = std::max(c->bitmap_words, c->bitmap_alloc);
        const size_t fr = std::max((size_t)c->factor_cap, c->factor_alloc);
        free_job(c);
        if (cudaMalloc(&c->d_bitmap, bw * 4) != cudaSuccess ||
            cudaMalloc(&c->d_factors, fr * sizeof(FactorRec)) != cudaSuccess) {
            free_job(c);
            rs_set_error("cannot allocate the bitmap (%zu words) and factor buffer", c->bitmap_words);
            return RS_ENOMEM;
        }
        c->bitmap_alloc = bw;
        c->factor_alloc = fr;
    }
    J.bitmap = c->d_bitmap;
    c->h_job = J;
    CU(cudaMemcpyAsync(c->d_bitmap, s->bitmap, c->bitmap_words * 4, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->d_job, &c->h_job, sizeof(JobDev), cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemsetAsync(c->d_ctrs, 0, 64, c->stream));
    CU(cudaMemsetAsync(c->d_err, 0, 4, c->stream));
    CU(cudaMemsetAsync(c->d_stats, 0, ST_COUNT * 8, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->primes_total = 0;
    c->job_loaded = true;
    tune_start(c);
    return RS_OK;
}

// segment width: about 60% of the prime buffer by the prime density 1/ln p,
// and few enough sieve survivors (density < 0.07 above 65537^2) for the
// candidate buffer; the kernels flag an overflow and the segment is redone
// at half the width if the estimate was short.
static u64 segment_width(const rs_ctx *c, u64 p)
{
    double lnp = std::log((double)(p < 3 ? 3 : p));
    double w = 0.6 * c->prime_cap * lnp;
    double wc = c->cand_cap / 0.07;
    if (p >= MR_BOUND && w > wc) w = wc;
    if (w > 4.0e9) w = 4.0e9;
    if (w < 1048576.0) w = 1048576.0;
    return (u64)w;
}

static int ensure_events(rs_ctx *c, size_t n)
{
    while (c->ev.size() < n) {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        c->ev.push_back(e);
    }
    return RS_OK;
}

// Generates the primes of [lo,hi) into d_primes; returns RS_OK and *np, or
// RS_EARG-free retry signal via *overflow.
static int gen_segment(rs_ctx *c, u64 lo, u64 hi, u32 *np, bool *overflow)
{
    *overflow = false;
    *np = 0;
    u64 base = lo | 1ull;
    if (base >= hi) return RS_OK;
    u64 nodd = (hi - base + 1) / 2;
    CU(cudaMemsetAsync(c->d_ctrs, 0, 2 * 4, c->stream));
    CU(cudaMemsetAsync(c->d_ctrs + 4, 0, 4, c->stream));
    CU(cudaMemsetAsync(c->d_err, 0, 4, c->stream));
    CU(launch_sieve(base, nodd, hi, c->d_sp, c->nsp, c->d_cands, c->cand_cap, c->d_ctrs, c->d_err, c->stream));
    CU(launch_mr2(c->d_cands, c->d_ctrs, c->cand_cap, c->d_primes, c->prime_cap, c->d_ctrs + 1, c->d_mid,
                  c->d_ctrs + 4, c->d_err, c->sms, c->stream));
    CU(cudaMemcpyAsync(c->h_pin, c->d_ctrs, 2 * 4, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemcpyAsync(c->h_pin + 4, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    u32 err = c->h_pin[4];
    if (err & (ERR_CAND_OVERFLOW | ERR_PRIME_OVERFLOW)) {
        *overflow = true;
        return RS_OK;
    }
    if (err) {
        rs_set_error("prime generator raised error flags 0x%x", err);
        return RS_EDEVICE;
    }
    *np = c->h_pin[1];
    return RS_OK;
}

extern "C" int rs_primes_generate(rs_ctx *c, uint64_t p0, uint64_t p1, uint64_t *dst, size_t cap, size_t *n)
{
    if (!c || !n || p0 >= p1) return RS_EARG;
    if (p0 < 3) p0 = 3;
    CU(cudaSetDevice(c->device));
    size_t total = 0;
    u64 p = p0;
    while (p < p1) {
        u64 w = segment_width(c, p);
        u64 hi = (p1 - p > w) ? p + w : p1;
        u32 np;
        bool ov;
        int rc = gen_segment(c, p, hi, &np, &ov);
        if (rc) return rc;
        if (ov) {
            rs_set_error("prime buffer overflow");
            return RS_EDEVICE;
        }
        if (dst && total < cap) {
            size_t take = std::min<size_t>(np, cap - total);
            CU(cudaMemcpy(dst + total, c->d_primes, take * 8, cudaMemcpyDeviceToHost));
        }
        total += np;
        p = hi;
    }
    *n = total;
    return (dst && total > cap) ? RS_EARG : RS_OK;
}

static int read_stats(rs_ctx *c, u64 *out)
{
    CU(cudaMemcpyAsync(out, c->d_stats, ST_COUNT * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return RS_OK;
}

extern "C" int rs_run_range(rs_ctx *c, uint64_t p0, uint64_t p1, rs_counters *delta)
{
    if (!c || !c->job_loaded) {
        rs_set_error("rs_run_range: no job loaded");
        return RS_EARG;
    }
    if (p0 < 3) p0 = 3;
    if (p1 <= p0) {
        if (delta) memset(delta, 0, sizeof *delta);
        return RS_OK;
    }
    CU(cudaSetDevice(c->device));
    u64 before[ST_COUNT];
    int rc = read_stats(c, before);
    if (rc) return rc;
    c->last_bsgs_ms = 0;
    c->last_total_ms = 0;
    c->last_bsgs_launches = 0;
    c->last_kernel_launches = 0;
    BsgsArgs a;
    a.base = c->h_job.base;
    a.nmin = c->h_job.nmin;
    a.nmax = c->h_job.nmax;
    a.words = c->h_job.words;
    a.bitmap = c->d_bitmap;
    a.factors = c->d_factors;
    a.factor_ctr = c->d_ctrs + 3;
    a.factor_cap = c->factor_cap;
    a.stats = c->d_stats;
    a.err = c->d_err;
    a.wait_bound = c->wait_bound;
    a.test_stall = c->test_stall;
    u64 p = p0;
    u64 width = segment_width(c, p);
    u64 seg_primes = 0;
    const u64 TOP = 1ull << 63;
    while (p < p1) {
        u64 hi = (p1 - p > width) ? p + width : p1;
        if (p < TOP && hi > TOP) hi = TOP;          // a launch is either all Shoup or all Montgomery
        if (p < FP_BOUND && hi > FP_BOUND) hi = FP_BOUND;   // and either all FP64 or all integer steps
        rc = ensure_events(c, 2);
        if (rc) return rc;
        CU(cudaEventRecord(c->ev[0], c->stream));
        u32 np;
        bool ov;
        rc = gen_segment(c, p, hi, &np, &ov);
        if (rc) return rc;
        if (ov) {
            width = (hi - p) / 2;
            if (width < 65536) {
                rs_set_error("prime buffer overflow at p=%llu", (unsigned long long)p);
                return RS_EDEVICE;
            }
            continue;
        }
        c->last_kernel_launches += 2;
        u32 nchunks = (np + c->chunk_cap - 1) / c->chunk_cap;
        rc = ensure_events(c, 2 + 2 * (size_t)nchunks);
        if (rc) return rc;
        CU(cudaMemsetAsync(c->d_err, 0, 4, c->stream));
        c->chunk_geom.assign(nchunks, c->geom);
        for (u32 ci = 0; ci < nchunks; ++ci) {
            u32 first = ci * c->chunk_cap;
            u32 cnt = std::min(c->chunk_cap, np - first);
            // while tuning, full chunks cycle through the candidate geometries
            const int g = (c->tuning && cnt >= 32768) ? c->tune_cand[c->tune_next++ % c->tune_ncand] : c->geom;
            c->chunk_geom[ci] = g;
            CU(launch_setup(c->d_job, c->d_primes, first, cnt, c->d_hdr, c->d_aux, c->d_tabs, c->d_tgt, c->d_meta,
                            c->d_stats, c->d_err, g, c->stream));
            CU(cudaMemsetAsync(c->d_ctrs + 2, 0, 4, c->stream));
            CU(cudaEventRecord(c->ev[2 + 2 * ci], c->stream));
            CU(launch_bsgs(a, c->d_hdr, c->d_tabs, c->d_tgt, c->d_meta, cnt, c->d_ctrs + 2, p, hi, g, c->sms,
                           c->stream));
            CU(cudaEventRecord(c->ev[3 + 2 * ci], c->stream));
            c->last_kernel_launches += 3;
            c->last_bsgs_launches += 1;
        }
        CU(cudaEventRecord(c->ev[1], c->stream));
        CU(cudaMemcpyAsync(c->h_pin + 4, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream));
        CU(cudaStreamSynchronize(c->stream));
        if (c->h_pin[4]) {
            rs_set_error("BSGS raised error flags 0x%x at p in [%llu,%llu)", c->h_pin[4], (unsigned long long)p,
                         (unsigned long long)hi);
            return RS_EDEVICE;
        }
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
        c->last_total_ms += ms;
        for (u32 ci = 0; ci < nchunks; ++ci) {
            CU(cudaEventElapsedTime(&ms, c->ev[2 + 2 * ci], c->ev[3 + 2 * ci]));
            c->last_bsgs_ms += ms;
            tune_record(c, c->chunk_geom[ci], std::min(c->chunk_cap, np - ci * c->chunk_cap), ms);
        }
        seg_primes += np;
        p = hi;
        width = segment_width(c, p);
    }
    u64 after[ST_COUNT];
    rc = read_stats(c, after);
    if (rc) return rc;
    c->primes_total += seg_primes;
    if (delta) {
        u64 *d = reinterpret_cast<u64 *>(delta);
        for (int i = 0; i < ST_COUNT; ++i) d[i] = after[i] - before[i];
        delta->primes = seg_primes;     // counted on the host: the device only sees segment totals
    }
    return RS_OK;
}

extern "C" int rs_factors_fetch(rs_ctx *c, rs_factor *buf, size_t cap, size_t *n)
{
    if (!c || !n || !c->job_loaded) return RS_EARG;
    CU(cudaSetDevice(c->device));
    CU(cudaMemcpyAsync(c->h_pin + 8, c->d_ctrs + 3, 4, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    u32 cnt = c->h_pin[8];
    *n = cnt;
    if (cnt > c->factor_cap) {
        rs_set_error("factor buffer overflowed (%u > %u)", cnt, c->factor_cap);
        return RS_EDEVICE;
    }
    if (cnt > cap || (cnt && !buf)) return RS_EARG;
    static_assert(sizeof(rs_factor) == sizeof(FactorRec), "factor layout");
    if (cnt) CU(cudaMemcpyAsync(buf, c->d_factors, (size_t)cnt * sizeof(FactorRec), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaMemsetAsync(c->d_ctrs + 3, 0, 4, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return RS_OK;
}

extern "C" int rs_bitmap_download(rs_ctx *c, uint32_t *dst, size_t words)
{
    if (!c || !dst || !c->job_loaded || words < c->bitmap_words) return RS_EARG;
    CU(cudaSetDevice(c->device));
    CU(cudaMemcpyAsync(dst, c->d_bitmap, c->bitmap_words * 4, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return RS_OK;
}

extern "C" int rs_counters_get(rs_ctx *c, rs_counters *out)
{
    if (!c || !out) return RS_EARG;
    CU(cudaSetDevice(c->device));
    int rc = read_stats(c, reinterpret_cast<u64 *>(out));
    out->primes = c->primes_total;
    return rc;
}

extern "C" int rs_last_timing(rs_ctx *c, double *bsgs_ms, double *total_ms, uint32_t *bl, uint32_t *kl)
{
    if (!c) return RS_EARG;
    if (bsgs_ms) *bsgs_ms = c->last_bsgs_launches ? c->last_bsgs_ms / c->last_bsgs_launches : 0.0;
    if (total_ms) *total_ms = c->last_total_ms;
    if (bl) *bl = c->last_bsgs_launches;
    if (kl) *kl = c->last_kernel_launches;
    return RS_OK;
}

extern "C" int rs_widemul_peak(rs_ctx *c, double *gwide_per_s, double *ms_out)
{
    if (!c || !gwide_per_s) return RS_EARG;
    CU(cudaSetDevice(c->device));
    const int blocks = c->sms * 8, iters = 8192;
    u64 *out = nullptr;
    CU(cudaMalloc(&out, (size_t)blocks * 256 * 8));
    int rc = ensure_events(c, 2);
    if (rc) { cudaFree(out); return rc; }
    CU(launch_widemul_peak(out, blocks, 64, c->stream));          // warm-up
    CU(cudaEventRecord(c->ev[0], c->stream));
    CU(launch_widemul_peak(out, blocks, iters, c->stream));
    CU(cudaEventRecord(c->ev[1], c->stream));
    CU(cudaEventSynchronize(c->ev[1]));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    cudaFree(out);
    *gwide_per_s = (double)blocks * 256 * 16 * iters / (ms * 1e-3) / 1e9;
    if (ms_out) *ms_out = ms;
    return RS_OK;
}

extern "C" int rs_fpmul_peak(rs_ctx *c, double *gfpmul_per_s, double *ms_out)
{
    if (!c || !gfpmul_per_s) return RS_EARG;
    CU(cudaSetDevice(c->device));
    const int blocks = c->sms * 8, iters = 4096;
    u64 *out = nullptr;
    CU(cudaMalloc(&out, (size_t)blocks * 256 * 8));
    int rc = ensure_events(c, 2);
    if (rc) { cudaFree(out); return rc; }
    CU(launch_fpmul_peak(out, blocks, 64, c->stream));          // warm-up
    CU(cudaEventRecord(c->ev[0], c->stream));
    CU(launch_fpmul_peak(out, blocks, iters, c->stream));
    CU(cudaEventRecord(c->ev[1], c->stream));
    CU(cudaEventSynchronize(c->ev[1]));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    cudaFree(out);
    *gfpmul_per_s = (double)blocks * 256 * 8 * iters / (ms * 1e-3) / 1e9;
    if (ms_out) *ms_out = ms;
    return RS_OK;
}

extern "C" int rs_mulmod_peak(rs_ctx *c, double *gmulmods_per_s, double *ms_out)
{
    if (!c || !gmulmods_per_s) return RS_EARG;
    CU(cudaSetDevice(c->device));
    const int blocks = c->sms * 8, iters = 4096;
    u64 *out = nullptr;
    CU(cudaMalloc(&out, (size_t)blocks * 256 * 8));
    int rc = ensure_events(c, 2);
    if (rc) { cudaFree(out); return rc; }
    CU(launch_mulmod_peak(out, blocks, 64, c->stream));          // warm-up
    CU(cudaEventRecord(c->ev[0], c->stream));
    CU(launch_mulmod_peak(out, blocks, iters, c->stream));
    CU(cudaEventRecord(c->ev[1], c->stream));
    CU(cudaEventSynchronize(c->ev[1]));
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    cudaFree(out);
    *gmulmods_per_s = (double)blocks * 256 * 8 * iters / (ms * 1e-3) / 1e9;
    if (ms_out) *ms_out = ms;
    return RS_OK;
}

// batch.cu -- many independent jobs sieved together (the batched form).
//
// The reference sieves one job per process: its host loop runs clearn ->
// getsegprimes -> setup -> sort -> giant per segment and waits on the device
// between kernels (cl_sieve.cpp:1292-1403).  A batch holds up to thousands of
// jobs (own sequences, n-range, bitmap and p-range each) on one device and
// advances all of them in rounds.  A round is a fixed sequence of launches
// whose window bounds, prime counts and work lists live in device memory:
//
//   k_batch_windows  next window of every range (sized for ~0.6*RCAP primes)
//   k_sieve_batch    segmented sieve, blockIdx.y = range
//   k_mr_batch       Miller-Rabin, blockIdx.y = range
//   k_setup_*<true>  per-prime set-up, blockIdx.y = range
//   per (geometry, product) group: prefix of the group's prime counts, then one
//   persistent k_bsgs<..., true> over all primes of the group's ranges (each
//   prime carries its job index and loads that job's arguments)
//   k_batch_account  primes tested per range, unfinished-range count
//
// so the host only waits once per round, to read the error word and whether
// any range is unfinished.  The first round runs eagerly (it also sizes the
// persistent grids); it is then captured as a CUDA graph and replayed.
//
// A job's p-range is split at 2^63 into two ranges (Shoup giant steps below,
// Montgomery above) that share its bitmap and factor list.  Each job's BSGS
// geometry comes from the per-prime cost model (geom_model_best) unless the
// caller fixes Q.
#include <algorithm>
#include <cstring>
#include <vector>

#include "rs_host.h"
#include "rs_internal.h"

using namespace rs;

namespace {

constexpr u32 RCAP = 1u << 16;     // primes per range per round
constexpr u32 CCAP = 2 * RCAP;     // sieve survivors per range per round (at most ~1.3 RCAP)

struct BJob {
    JobDev jd;
    int geom;
    u32 *d_bitmap = nullptr;
    size_t bitmap_words = 0;
    FactorRec *d_factors = nullptr;
    u32 factor_cap = 0;
    std::vector<u32> ranges;
};

struct Group {
    int geom;
    bool shoup;
    std::vector<u32> ranges;
    u32 *d_ranges = nullptr;   // the group's range indices
    u32 *d_prefix = nullptr;   // nr + 1 prefix sums of their prime counts
    u32 *d_work = nullptr;     // work counter of the group's BSGS launch
};

__global__ void k_batch_account(const BatchRange *ranges, const u32 *ctrs, u32 rcap, u32 nranges, u64 *range_primes,
                                u64 *stats, u32 *unfinished)
{
    const u32 r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    const u32 n = min(ctrs[r * BR_CTRS + 1], rcap);
    range_primes[r] += n;
    if (n) atomicAdd((unsigned long long *)&stats[ST_PRIMES], (unsigned long long)n);
    if (ranges[r].p_cur < ranges[r].p_end) atomicAdd(unfinished, 1u);
}

}  // namespace

struct rs_batch {
    int device = -1;
    int sms = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::vector<BJob> jobs;
    std::vector<BatchRange> h_ranges;
    std::vector<Group> groups;
    bool built = false;
    // device tables
    u32 *d_sp = nullptr;
    u32 nsp = 0;
    JobDev *d_jobs = nullptr;
    JobGeom *d_geoms = nullptr;
    BsgsArgs *d_args = nullptr;
    u32 *d_fctrs = nullptr;
    BatchRange *d_ranges = nullptr;
    BatchWin *d_wins = nullptr;
    u32 *d_ctrs = nullptr;
    u64 *d_range_primes = nullptr;
    // per-range round buffers
    u64 *d_cands = nullptr, *d_primes = nullptr;
    PrimeHdr *d_hdr = nullptr;
    void *d_aux = nullptr;
    u64 *d_tabs = nullptr, *d_tgt = nullptr;
    unsigned char *d_meta = nullptr;
    u32 *d_err = nullptr;
    u64 *d_stats = nullptr;
    u32 *d_unfinished = nullptr;
    u32 *h_pin = nullptr;       // [0] error word, [1] unfinished ranges
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    u64 rounds = 0;
    bool done = false;
};

#define BCU(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            rs_set_error("%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);    \
            return RS_ECUDA;                                                                      \
        }                                                                                         \
    } while (0)

extern "C" void rs_batch_destroy(rs_batch *b)
{
    if (!b) return;
    if (b->device >= 0) cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto &j : b->jobs) {
        cudaFree(j.d_bitmap);
        cudaFree(j.d_factors);
    }
    for (auto &g : b->groups) {
        cudaFree(g.d_ranges);
        cudaFree(g.d_prefix);
        cudaFree(g.d_work);
    }
    void *ptrs[] = {b->d_sp, b->d_jobs, b->d_geoms, b->d_args, b->d_fctrs, b->d_ranges, b->d_wins, b->d_ctrs,
                    b->d_range_primes, b->d_cands, b->d_primes, b->d_hdr, b->d_aux, b->d_tabs, b->d_tgt, b->d_meta,
                    b->d_err, b->d_stats, b->d_unfinished};
    for (void *p : ptrs) cudaFree(p);
    if (b->h_pin) cudaFreeHost(b->h_pin);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
}

extern "C" int rs_batch_create(int device, rs_batch **out)
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
    rs_batch *b = new rs_batch();
    b->device = device;
    auto fail = [&](int rc) { rs_batch_destroy(b); return rc; };
    if (cudaSetDevice(device) != cudaSuccess) return fail(RS_ECUDA);
    if (cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return fail(RS_ECUDA);
    if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) return fail(RS_ECUDA);
    b->stream = b->own;
    std::vector<u32> sp = rs_small_primes();
    b->nsp = (u32)sp.size();
    if (cudaMalloc(&b->d_sp, sp.size() * 4) != cudaSuccess || cudaMalloc(&b->d_err, 4) != cudaSuccess ||
        cudaMalloc(&b->d_stats, ST_COUNT * 8) != cudaSuccess || cudaMalloc(&b->d_unfinished, 4) != cudaSuccess ||
        cudaMallocHost(&b->h_pin, 16) != cudaSuccess) {
        rs_set_error("device allocation failed");
        return fail(RS_ENOMEM);
    }
    if (cudaMemcpy(b->d_sp, sp.data(), sp.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->d_err, 0, 4) != cudaSuccess || cudaMemset(b->d_stats, 0, ST_COUNT * 8) != cudaSuccess)
        return fail(RS_ECUDA);
    if (bsgs_prepare() != cudaSuccess) {
        rs_set_error("cannot configure the BSGS kernels' shared memory");
        return fail(RS_ECUDA);
    }
    *out = b;
    return RS_OK;
}

extern "C" int rs_batch_set_stream(rs_batch *b, void *stream)
{
    if (!b || b->built) return RS_EARG;      // the captured round is bound to one stream
    b->stream = stream ? (cudaStream_t)stream : b->own;
    return RS_OK;
}

extern "C" int rs_batch_add(rs_batch *b, const rs_seqs *s, uint64_t p0, uint64_t p1, uint32_t q, uint32_t *job)
{
    if (!b || !s) return RS_EARG;
    if (b->built) {
        rs_set_error("rs_batch_add: the batch has already run; create a new batch for more jobs");
        return RS_EARG;
    }
    if (q != 0 && geom_index(q) < 0) {
        rs_set_error("baby-step count %u is not one of 1024, 2048, 4096, 8192, 16384 (or 0 for the model)", q);
        return RS_EARG;
    }
    int rc = rs_seqs_validate(s);
    if (rc) return rc;
    if (p0 < 3) p0 = 3;
    if (p1 <= p0) {
        rs_set_error("rs_batch_add: empty p-range");
        return RS_EARG;
    }
    BCU(cudaSetDevice(b->device));
    BJob J;
    jobdev_from_seqs(s, &J.jd);
    J.geom = q ? geom_index(q) : geom_model_best(J.jd.kcount, J.jd.L);
    J.bitmap_words = (size_t)s->kcount * s->words_per_seq;
    const uint64_t cand = rs_seqs_count(s);
    J.factor_cap = (u32)std::min<uint64_t>(cand + 1, 0xFFFFFFF0ull);
    if (cudaMalloc(&J.d_bitmap, J.bitmap_words * 4) != cudaSuccess ||
        cudaMalloc(&J.d_factors, (size_t)J.factor_cap * sizeof(FactorRec)) != cudaSuccess) {
        cudaFree(J.d_bitmap);
        cudaFree(J.d_factors);
        rs_set_error("cannot allocate the bitmap and factor buffer of batch job %zu", b->jobs.size());
        return RS_ENOMEM;
    }
    J.jd.bitmap = J.d_bitmap;
    BCU(cudaMemcpy(J.d_bitmap, s->bitmap, J.bitmap_words * 4, cudaMemcpyHostToDevice));
    const u32 jid = (u32)b->jobs.size();
    const u64 TOP = 1ull << 63;
    auto add_range = [&](u64 lo, u64 hi) {
        BatchRange R;
        R.p_cur = lo;
        R.p_end = hi;
        R.job = jid;
        R.pad_ = 0;
        J.ranges.push_back((u32)b->h_ranges.size());
        b->h_ranges.push_back(R);
    };
    if (p0 < TOP && p1 > TOP) {
        add_range(p0, TOP);
        add_range(TOP, p1);
    } else {
        add_range(p0, p1);
    }
    b->jobs.push_back(J);
    if (job) *job = jid;
    return RS_OK;
}

// Allocates the round buffers and device tables and forms the BSGS groups.
static int batch_build(rs_batch *b)
{
    const u32 J = (u32)b->jobs.size(), R = (u32)b->h_ranges.size();
    if (J == 0) {
        rs_set_error("rs_batch_run: no jobs");
        return RS_EARG;
    }
    auto alloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
    if (!alloc((void **)&b->d_jobs, J * sizeof(JobDev)) || !alloc((void **)&b->d_geoms, J * sizeof(JobGeom)) ||
        !alloc((void **)&b->d_args, J * sizeof(BsgsArgs)) || !alloc((void **)&b->d_fctrs, J * 4) ||
        !alloc((void **)&b->d_ranges, R * sizeof(BatchRange)) || !alloc((void **)&b->d_wins, R * sizeof(BatchWin)) ||
        !alloc((void **)&b->d_ctrs, (size_t)R * BR_CTRS * 4) || !alloc((void **)&b->d_range_primes, R * 8) ||
        !alloc((void **)&b->d_cands, (size_t)R * CCAP * 8) || !alloc((void **)&b->d_primes, (size_t)R * RCAP * 8) ||
        !alloc((void **)&b->d_hdr, (size_t)R * RCAP * sizeof(PrimeHdr)) ||
        !alloc(&b->d_aux, (size_t)R * RCAP * setup_aux_bytes()) ||
        !alloc((void **)&b->d_tabs, (size_t)R * RCAP * TABS * 8) ||
        !alloc((void **)&b->d_tgt, (size_t)R * RCAP * KSTRIDE * 8) ||
        !alloc((void **)&b->d_meta, (size_t)R * RCAP * KSTRIDE)) {
        rs_set_error("cannot allocate the round buffers of %u ranges", R);
        return RS_ENOMEM;
    }
    std::vector<JobDev> jd(J);
    std::vector<JobGeom> jg(J);
    std::vector<BsgsArgs> ja(J);
    for (u32 j = 0; j < J; ++j) {
        const BJob &B = b->jobs[j];
        const BsgsGeom &g = BSGS_GEOMS[B.geom];
        jd[j] = B.jd;
        JobGeom &G = jg[j];
        G.q = g.q; G.c = g.c; G.tpb = g.tpb; G.pad_ = 0;
        G.m1 = (u32)(((u64)B.jd.L + g.q - 1) / g.q);
        G.m2 = (u32)(((u64)B.jd.L + 2ull * g.q - 1) / (2ull * g.q));
        BsgsArgs &A = ja[j];
        A.base = B.jd.base; A.nmin = B.jd.nmin; A.nmax = B.jd.nmax; A.words = B.jd.words;
        A.M1 = G.m1; A.M2 = G.m2;
        A.bitmap = B.d_bitmap;
        A.factors = B.d_factors;
        A.factor_ctr = b->d_fctrs + j;
        A.factor_cap = B.factor_cap;
        A.stats = b->d_stats;
        A.err = b->d_err;
    }
    BCU(cudaMemcpy(b->d_jobs, jd.data(), J * sizeof(JobDev), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_geoms, jg.data(), J * sizeof(JobGeom), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_args, ja.data(), J * sizeof(BsgsArgs), cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_ranges, b->h_ranges.data(), R * sizeof(BatchRange), cudaMemcpyHostToDevice));
    BCU(cudaMemset(b->d_fctrs, 0, J * 4));
    BCU(cudaMemset(b->d_range_primes, 0, R * 8));
    BCU(cudaMemset(b->d_ctrs, 0, (size_t)R * BR_CTRS * 4));
    // groups: ranges with the same geometry and the same side of 2^63
    for (u32 r = 0; r < R; ++r) {
        const int g = b->jobs[b->h_ranges[r].job].geom;
        const bool shoup = b->h_ranges[r].p_end <= (1ull << 63);
        auto it = std::find_if(b->groups.begin(), b->groups.end(),
                               [&](const Group &x) { return x.geom == g && x.shoup == shoup; });
        if (it == b->groups.end()) {
            b->groups.push_back(Group{g, shoup, {}, nullptr, nullptr, nullptr});
            it = b->groups.end() - 1;
        }
        it->ranges.push_back(r);
    }
    for (auto &g : b->groups) {
        const u32 nr = (u32)g.ranges.size();
        if (!alloc((void **)&g.d_ranges, nr * 4) || !alloc((void **)&g.d_prefix, (nr + 1) * 4) ||
            !alloc((void **)&g.d_work, 4)) {
            rs_set_error("cannot allocate the BSGS group tables");
            return RS_ENOMEM;
        }
        BCU(cudaMemcpy(g.d_ranges, g.ranges.data(), nr * 4, cudaMemcpyHostToDevice));
    }
    b->built = true;
    return RS_OK;
}

// Enqueues one round on b->stream (also what the graph captures).
static int batch_round(rs_batch *b)
{
    const u32 R = (u32)b->h_ranges.size();
    cudaStream_t st = b->stream;
    // widest window: 0.6*RCAP*ln(2^64) values, i.e. 0.3*RCAP*44.4 odd values
    const u32 max_blocks = (u32)((0.3 * RCAP * 44.4) / (SIEVE_WORDS * 32.0)) + 2;
    BCU(cudaMemsetAsync(b->d_unfinished, 0, 4, st));
    BCU(launch_batch_windows(b->d_ranges, b->d_wins, R, RCAP, b->d_ctrs, st));
    BCU(launch_sieve_batch(b->d_wins, R, max_blocks, b->d_sp, b->nsp, b->d_cands, CCAP, b->d_ctrs, b->d_err, st));
    BCU(launch_mr_batch(b->d_cands, CCAP, b->d_primes, RCAP, b->d_ctrs, R, b->d_err, b->sms, st));
    BCU(launch_setup_batch(b->d_jobs, b->d_geoms, b->d_ranges, b->d_primes, RCAP, b->d_ctrs, R, b->d_hdr, b->d_aux,
                           b->d_tabs, b->d_tgt, b->d_meta, b->d_stats, st));
    BsgsArgs a;
    memset(&a, 0, sizeof a);
    a.stats = b->d_stats;
    a.err = b->d_err;
    for (auto &g : b->groups) {
        const u32 nr = (u32)g.ranges.size();
        BCU(launch_batch_prefix(g.d_ranges, nr, b->d_ctrs, RCAP, g.d_prefix, st));
        BCU(cudaMemsetAsync(g.d_work, 0, 4, st));
        BCU(launch_bsgs_batch(a, b->d_args, b->d_hdr, b->d_tabs, b->d_tgt, b->d_meta, g.d_ranges, nr, g.d_prefix, RCAP,
                              g.d_work, g.shoup, g.geom, b->sms, st));
    }
    k_batch_account<<<(R + 127) / 128, 128, 0, st>>>(b->d_ranges, b->d_ctrs, RCAP, R, b->d_range_primes, b->d_stats,
                                                     b->d_unfinished);
    BCU(cudaGetLastError());
    return RS_OK;
}

extern "C" int rs_batch_run(rs_batch *b, uint32_t max_rounds, int *done)
{
    if (!b) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    if (!b->built) {
        int rc = batch_build(b);
        if (rc) return rc;
    }
    for (uint32_t i = 0; (max_rounds == 0 || i < max_rounds) && !b->done; ++i) {
        if (b->rounds == 0) {
            int rc = batch_round(b);                 // eager: sizes the persistent grids
            if (rc) return rc;
        } else {
            if (!b->exec) {
                BCU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                int rc = batch_round(b);
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(b->stream, &g);
                if (rc) {
                    if (g) cudaGraphDestroy(g);
                    return rc;
                }
                BCU(e);
                b->graph = g;
                BCU(cudaGraphInstantiate(&b->exec, b->graph, 0));
            }
            BCU(cudaGraphLaunch(b->exec, b->stream));
        }
        BCU(cudaMemcpyAsync(b->h_pin, b->d_err, 4, cudaMemcpyDeviceToHost, b->stream));
        BCU(cudaMemcpyAsync(b->h_pin + 1, b->d_unfinished, 4, cudaMemcpyDeviceToHost, b->stream));
        BCU(cudaStreamSynchronize(b->stream));
        ++b->rounds;
        if (b->h_pin[0]) {
            rs_set_error("batch round %llu raised error flags 0x%x", (unsigned long long)b->rounds, b->h_pin[0]);
            return RS_EDEVICE;
        }
        b->done = (b->h_pin[1] == 0);
    }
    if (done) *done = b->done ? 1 : 0;
    return RS_OK;
}

extern "C" int rs_batch_factors_fetch(rs_batch *b, uint32_t job, rs_factor *buf, size_t cap, size_t *n)
{
    if (!b || !n || job >= b->jobs.size() || !b->built) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    BCU(cudaMemcpyAsync(b->h_pin + 2, b->d_fctrs + job, 4, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    const u32 cnt = b->h_pin[2];
    *n = cnt;
    const BJob &J = b->jobs[job];
    if (cnt > J.factor_cap) {
        rs_set_error("factor buffer of batch job %u overflowed", job);
        return RS_EDEVICE;
    }
    if (cnt > cap || (cnt && !buf)) return RS_EARG;
    static_assert(sizeof(rs_factor) == sizeof(FactorRec), "factor layout");
    if (cnt) BCU(cudaMemcpyAsync(buf, J.d_factors, (size_t)cnt * sizeof(FactorRec), cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaMemsetAsync(b->d_fctrs + job, 0, 4, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return RS_OK;
}

extern "C" int rs_batch_bitmap_download(rs_batch *b, uint32_t job, uint32_t *dst, size_t words)
{
    if (!b || !dst || job >= b->jobs.size() || words < b->jobs[job].bitmap_words) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    BCU(cudaMemcpyAsync(dst, b->jobs[job].d_bitmap, b->jobs[job].bitmap_words * 4, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return RS_OK;
}

extern "C" int rs_batch_job_info(rs_batch *b, uint32_t job, uint32_t *q, uint64_t *primes, int *done)
{
    if (!b || job >= b->jobs.size()) return RS_EARG;
    const BJob &J = b->jobs[job];
    if (q) *q = BSGS_GEOMS[J.geom].q;
    if (!primes && !done) return RS_OK;
    if (!b->built) {
        if (primes) *primes = 0;
        if (done) *done = 0;
        return RS_OK;
    }
    BCU(cudaSetDevice(b->device));
    std::vector<u64> rp(b->h_ranges.size());
    std::vector<BatchRange> rr(b->h_ranges.size());
    BCU(cudaMemcpyAsync(rp.data(), b->d_range_primes, rp.size() * 8, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaMemcpyAsync(rr.data(), b->d_ranges, rr.size() * sizeof(BatchRange), cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    u64 n = 0;
    bool all = true;
    for (u32 r : J.ranges) {
        n += rp[r];
        all = all && rr[r].p_cur >= rr[r].p_end;
    }
    if (primes) *primes = n;
    if (done) *done = all ? 1 : 0;
    return RS_OK;
}

extern "C" int rs_batch_counters(rs_batch *b, rs_counters *out)
{
    if (!b || !out) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    static_assert(sizeof(rs_counters) == ST_COUNT * 8, "counter layout");
    BCU(cudaMemcpyAsync(out, b->d_stats, ST_COUNT * 8, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return RS_OK;
}

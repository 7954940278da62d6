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
//   k_mr_batch_sprp, k_mr_batch_lucas  Baillie-PSW over the survivors of every
//                    range at once (base 2, then Lucas over the passers)
//   k_setup_*<true>  per-prime set-up over the primes of every range at once
//   k_batch_group_prefix  every (geometry, product) group's prefix sums of its
//                    ranges' prime counts, in one launch
//   per group, on its own branch (fork/join through events): one persistent
//   k_bsgs<..., true> over all primes of the group's ranges (each prime carries
//   its job index and loads that job's arguments); the branches overlap, so one
//   group's last wave does not idle the device
//   k_batch_account  primes tested per range, unfinished-range count
//
// so the host only waits once per round, to read the error word and whether
// any range is unfinished.  The first round runs eagerly (it also sizes the
// persistent grids); it is then captured as a CUDA graph and replayed.
//
// A job's p-range is split at 2^63 into two ranges (Shoup giant steps below,
// Montgomery above) that share its bitmap and factor list.  Each job's BSGS
// geometry is the one a single-job run on the device measured for the job's
// shape (base, sequence count, n-range), else the per-prime cost model's
// (geom_model_best), unless the caller fixes Q.
//
// Capacity is fixed when the batch is created: job slots and range slots (each
// range slot owns one round's buffers, about 136 MB).  Jobs can be added
// between rounds -- their tables are written to device memory that the
// captured round reads -- and a finished job's slots are released for the
// next one, so the batch also serves a stream of arriving work units.  The
// ten BSGS groups (geometry x product) cover every range slot and count only
// the slots currently in them, so the captured round never changes.  A job's
// bitmap and factor list come from the batch's own stream-ordered memory pool,
// which keeps freed blocks mapped and can be grown ahead of time
// (rs_batch_reserve): admitting or releasing a job neither
// synchronises the device nor maps new pages.
#include <algorithm>
#include <cstring>
#include <vector>

#include "rs_host.h"
#include "rs_internal.h"

using namespace rs;

namespace {

constexpr u32 RCAP = 1u << 16;     // primes per range per round
constexpr u32 CCAP = 2 * RCAP;     // sieve survivors per range per round (at most ~1.3 RCAP)
constexpr u32 DEF_JOBS = 64, DEF_RANGES = 64;

struct BJob {
    bool used = false;
    JobDev jd;
    int geom = 0;
    u32 *d_bitmap = nullptr;
    size_t bitmap_words = 0;
    FactorRec *d_factors = nullptr;
    u32 factor_cap = 0;
    std::vector<u32> ranges;
};

constexpr int NGROUP = 3 * NGEOM;  // BSGS groups: g = 3*geometry + step kind (2 FP64, 1 Shoup, 0 Montgomery)

__global__ void k_batch_account(const BatchRange *ranges, const u32 *ctrs, u32 rcap, u32 nranges, u64 *range_primes,
                                u64 *stats, u32 *unfinished)
{
    const u32 r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nranges) return;
    const BatchRange R = ranges[r];
    if (!R.active) return;
    const u32 n = min(ctrs[r * BR_CTRS + 1], rcap);
    range_primes[r] += n;
    if (n) atomicAdd((unsigned long long *)&stats[ST_PRIMES], (unsigned long long)n);
    if (R.p_cur < R.p_end) atomicAdd(unfinished, 1u);
}

}  // namespace

struct rs_batch {
    int device = -1;
    int sms = 0;
    u32 max_jobs = 0, nranges = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    std::vector<BJob> jobs;
    std::vector<BatchRange> h_ranges;      // host copy of the range slots' fixed fields
    std::vector<char> range_used;
    std::vector<u32> h_win;                // primes per round per range slot (0: paused)
    std::vector<char> range_done;          // from the last rs_batch_poll
    bool win_dirty = false;
    u32 *d_win = nullptr;
    u32 *d_prefix_c = nullptr, *d_prefix_p = nullptr;   // prefix sums over all ranges: survivors, primes
    u32 *h_win_pin = nullptr;
    u32 *d_gprefix = nullptr;              // NGROUP x (nranges + 1) prefix sums of the groups' prime counts
    u32 *d_gwork = nullptr;                // NGROUP work counters of the groups' BSGS launches
    cudaStream_t side[NGROUP] = {};        // one branch per group: the groups' launches overlap
    cudaEvent_t fork = nullptr, join[NGROUP] = {};
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
    u64 *d_mid = nullptr;                  // base-2 probable primes of all ranges awaiting the Lucas pass
    u32 *d_mid_r = nullptr;                //   and their ranges (R * CCAP entries)
    u32 *d_mid_ctr = nullptr;
    u32 *d_rec_of = nullptr;               // record index of each prime of a round (R * RCAP)
    PrimeHdr *d_hdr = nullptr;
    void *d_aux = nullptr;
    u64 *d_tabs = nullptr, *d_tgt = nullptr;
    unsigned short *d_meta = nullptr;
    u32 *d_err = nullptr;
    u64 *d_stats = nullptr;
    u32 *d_unfinished = nullptr;
    u32 *h_pin = nullptr;       // [0] error word, [1] unfinished ranges, [2] factor count
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaMemPool_t pool = nullptr;          // jobs' bitmaps and factor lists; keeps freed memory mapped
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
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto &j : b->jobs) {
        if (j.d_bitmap) cudaFreeAsync(j.d_bitmap, b->stream);
        if (j.d_factors) cudaFreeAsync(j.d_factors, b->stream);
    }
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->pool) cudaMemPoolDestroy(b->pool);
    for (int g = 0; g < NGROUP; ++g) {
        if (b->side[g]) cudaStreamDestroy(b->side[g]);
        if (b->join[g]) cudaEventDestroy(b->join[g]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    void *ptrs[] = {b->d_sp, b->d_jobs, b->d_geoms, b->d_args, b->d_fctrs, b->d_ranges, b->d_wins, b->d_ctrs,
                    b->d_range_primes, b->d_cands, b->d_primes, b->d_hdr, b->d_aux, b->d_tabs, b->d_tgt, b->d_meta,
                    b->d_err, b->d_stats, b->d_unfinished, b->d_win, b->d_prefix_c, b->d_prefix_p,
                    b->d_gprefix, b->d_gwork, b->d_mid, b->d_mid_r, b->d_mid_ctr, b->d_rec_of};
    for (void *p : ptrs) cudaFree(p);
    if (b->h_pin) cudaFreeHost(b->h_pin);
    if (b->h_win_pin) cudaFreeHost(b->h_win_pin);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
}

extern "C" int rs_batch_create(int device, uint32_t max_jobs, uint32_t range_slots, rs_batch **out)
{
    if (!out) return RS_EARG;
    *out = nullptr;
    if (max_jobs == 0) max_jobs = DEF_JOBS;
    if (range_slots == 0) range_slots = DEF_RANGES;
    if (max_jobs > 65536 || range_slots > 4096) {
        rs_set_error("rs_batch_create: at most 65536 jobs and 4096 range slots");
        return RS_EARG;
    }
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
    b->max_jobs = max_jobs;
    b->nranges = range_slots;
    auto fail = [&](int rc) { rs_batch_destroy(b); return rc; };
    if (cudaSetDevice(device) != cudaSuccess) return fail(RS_ECUDA);
    if (cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return fail(RS_ECUDA);
    if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess) return fail(RS_ECUDA);
    b->stream = b->own;
    b->jobs.resize(max_jobs);
    b->h_ranges.assign(range_slots, BatchRange{});
    b->range_used.assign(range_slots, 0);
    b->h_win.assign(range_slots, 0);
    b->range_done.assign(range_slots, 0);
    const u32 J = max_jobs, R = range_slots;
    std::vector<u32> sp = rs_small_primes();
    b->nsp = (u32)sp.size();
    auto alloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
    if (!alloc((void **)&b->d_sp, sp.size() * 4) || !alloc((void **)&b->d_err, 4) ||
        !alloc((void **)&b->d_stats, ST_COUNT * 8) || !alloc((void **)&b->d_unfinished, 4) ||
        !alloc((void **)&b->d_jobs, (size_t)J * sizeof(JobDev)) || !alloc((void **)&b->d_geoms, J * sizeof(JobGeom)) ||
        !alloc((void **)&b->d_args, J * sizeof(BsgsArgs)) || !alloc((void **)&b->d_fctrs, J * 4) ||
        !alloc((void **)&b->d_ranges, R * sizeof(BatchRange)) || !alloc((void **)&b->d_wins, R * sizeof(BatchWin)) ||
        !alloc((void **)&b->d_ctrs, (size_t)R * BR_CTRS * 4) || !alloc((void **)&b->d_range_primes, R * 8) ||
        !alloc((void **)&b->d_cands, (size_t)R * CCAP * 8) || !alloc((void **)&b->d_primes, (size_t)R * RCAP * 8) ||
        !alloc((void **)&b->d_mid, (size_t)R * CCAP * 8) || !alloc((void **)&b->d_mid_r, (size_t)R * CCAP * 4) ||
        !alloc((void **)&b->d_mid_ctr, 4) || !alloc((void **)&b->d_rec_of, (size_t)R * RCAP * 4) ||
        !alloc((void **)&b->d_hdr, (size_t)R * RCAP * sizeof(PrimeHdr)) ||
        !alloc(&b->d_aux, (size_t)R * RCAP * setup_aux_bytes()) ||
        !alloc((void **)&b->d_tabs, (size_t)R * RCAP * TABS * 8) ||
        !alloc((void **)&b->d_tgt, (size_t)R * RCAP * KSTRIDE * 8) ||
        !alloc((void **)&b->d_meta, (size_t)R * RCAP * KSTRIDE * 2) || !alloc((void **)&b->d_win, R * 4) ||
        !alloc((void **)&b->d_prefix_c, (R + 1) * 4) || !alloc((void **)&b->d_prefix_p, (R + 1) * 4) ||
        cudaMallocHost(&b->h_pin, 16) != cudaSuccess || cudaMallocHost(&b->h_win_pin, R * 4) != cudaSuccess) {
        rs_set_error("cannot allocate a batch of %u range slots (about %zu MB)", R,
                     (size_t)R * RCAP * (sizeof(PrimeHdr) + TABS * 8 + KSTRIDE * 10 + 24 + 8 + 16 + 24 + 4) >> 20);
        return fail(RS_ENOMEM);
    }
    if (cudaMemcpy(b->d_sp, sp.data(), sp.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->d_err, 0, 4) != cudaSuccess || cudaMemset(b->d_stats, 0, ST_COUNT * 8) != cudaSuccess ||
        cudaMemset(b->d_jobs, 0, (size_t)J * sizeof(JobDev)) != cudaSuccess ||
        cudaMemset(b->d_geoms, 0, J * sizeof(JobGeom)) != cudaSuccess ||
        cudaMemset(b->d_args, 0, J * sizeof(BsgsArgs)) != cudaSuccess || cudaMemset(b->d_fctrs, 0, J * 4) != cudaSuccess ||
        cudaMemset(b->d_ranges, 0, R * sizeof(BatchRange)) != cudaSuccess ||
        cudaMemset(b->d_ctrs, 0, (size_t)R * BR_CTRS * 4) != cudaSuccess ||
        cudaMemset(b->d_range_primes, 0, R * 8) != cudaSuccess || cudaMemset(b->d_win, 0, R * 4) != cudaSuccess)
        return fail(RS_ECUDA);
    if (bsgs_prepare() != cudaSuccess) {
        rs_set_error("cannot configure the BSGS kernels' shared memory");
        return fail(RS_ECUDA);
    }
    {
        // a pool of our own whose freed blocks stay mapped: admitting a job after
        // releasing one reuses memory instead of mapping new pages at every sync
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&b->pool, &props) != cudaSuccess) return fail(RS_ECUDA);
        uint64_t keep = ~0ull;
        if (cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
            return fail(RS_ECUDA);
    }
    if (!alloc((void **)&b->d_gprefix, (size_t)NGROUP * (R + 1) * 4) || !alloc((void **)&b->d_gwork, NGROUP * 4)) {
        rs_set_error("cannot allocate the BSGS group tables");
        return fail(RS_ENOMEM);
    }
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return fail(RS_ECUDA);
    for (int g = 0; g < NGROUP; ++g)
        if (cudaStreamCreateWithFlags(&b->side[g], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[g], cudaEventDisableTiming) != cudaSuccess)
            return fail(RS_ECUDA);
    *out = b;
    return RS_OK;
}

extern "C" int rs_batch_set_stream(rs_batch *b, void *stream)
{
    if (!b || b->rounds) return RS_EARG;     // the captured round is bound to one stream
    if (!stream) {
        rs_set_error("rs_batch_set_stream: a batch captures its rounds, which the legacy NULL stream cannot");
        return RS_EARG;
    }
    b->stream = (cudaStream_t)stream;
    return RS_OK;
}

static int batch_add_job(rs_batch *b, const rs_seqs *s, const BJob *src, uint64_t p0, uint64_t p1, uint32_t q,
                         uint32_t nsplit, uint32_t *job);

extern "C" int rs_batch_add(rs_batch *b, const rs_seqs *s, uint64_t p0, uint64_t p1, uint32_t q, uint32_t *job)
{
    if (!b || !s) return RS_EARG;
    if (q != 0 && geom_index(q) < 0) {
        rs_set_error("baby-step count %u is not one of 1024, 2048, 4096, 8192, 16384 (or 0 for the model)", q);
        return RS_EARG;
    }
    int rc = rs_seqs_validate(s);
    if (rc) return rc;
    if (p1 < p0) {
        rs_set_error("rs_batch_add: p1 < p0");
        return RS_EARG;
    }
    return batch_add_job(b, s, nullptr, p0, p1, q, 1, job);
}

// Adds a job from host sequences s, or (s == nullptr) as a copy of job slot src
// made on the device.  p0 == p1: a resident template that takes no range slot.
// The p-range is cut into nsplit equal parts, and at 2^51 and 2^63 (where the
// BSGS step kind changes), one range slot each.
static int batch_add_job(rs_batch *b, const rs_seqs *s, const BJob *src, uint64_t p0, uint64_t p1, uint32_t q,
                         uint32_t nsplit, uint32_t *job)
{
    const bool tmpl = (p0 == p1);
    if (p0 < 3) p0 = 3;
    if (!tmpl && p1 <= p0) {
        rs_set_error("rs_batch_add: empty p-range");
        return RS_EARG;
    }
    const u64 TOP = 1ull << 63;
    std::vector<u64> cuts;                   // range boundaries p0 = c0 < c1 < ... < p1
    if (!tmpl) {
        if (nsplit < 1) nsplit = 1;
        if (nsplit > p1 - p0) nsplit = (u32)(p1 - p0);
        const u64 w = (p1 - p0) / nsplit;
        cuts.push_back(p0);
        for (u32 i = 1; i < nsplit; ++i) cuts.push_back(p0 + i * w);
        if (p0 < TOP && p1 > TOP) cuts.push_back(TOP);
        if (p0 < FP_BOUND && p1 > FP_BOUND) cuts.push_back(FP_BOUND);
        cuts.push_back(p1);
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
    }
    const u32 need = tmpl ? 0 : (u32)cuts.size() - 1;
    u32 jid = 0;
    while (jid < b->max_jobs && b->jobs[jid].used) ++jid;
    std::vector<u32> slots;
    for (u32 r = 0; r < b->nranges && slots.size() < need; ++r)
        if (!b->range_used[r]) slots.push_back(r);
    if (jid == b->max_jobs || slots.size() < need) {
        rs_set_error("rs_batch_add: no free job or range slot (%u jobs, %u range slots)", b->max_jobs, b->nranges);
        return RS_EBUSY;
    }
    BCU(cudaSetDevice(b->device));
    BJob &J = b->jobs[jid];
    J = BJob();
    if (s) {
        jobdev_from_seqs(s, &J.jd);
        if (q) {
            J.geom = geom_index(q);
        } else {        // measured by a single-job run of this shape on the device, else the model
            const int known = tuned_geom_get(b->device, job_shape_key(J.jd.base, J.jd.kcount, J.jd.L));
            J.geom = known >= 0 ? known : geom_model_best(J.jd.kcount, J.jd.L);
        }
        J.bitmap_words = (size_t)s->kcount * s->words_per_seq;
        const uint64_t cand = rs_seqs_count(s);
        J.factor_cap = (u32)std::min<uint64_t>(cand + 1, 0xFFFFFFF0ull);
    } else {
        J.jd = src->jd;
        J.geom = src->geom;
        J.bitmap_words = src->bitmap_words;
        J.factor_cap = src->factor_cap;
    }
    const u32 fcap = tmpl ? 1u : J.factor_cap;       // a template never claims; its clones get factor_cap
    if (cudaMallocFromPoolAsync((void **)&J.d_bitmap, J.bitmap_words * 4, b->pool, b->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void **)&J.d_factors, (size_t)fcap * sizeof(FactorRec), b->pool, b->stream) !=
            cudaSuccess) {
        cudaGetLastError();              // the failed pool allocation must not surface at the next round
        if (J.d_bitmap) cudaFreeAsync(J.d_bitmap, b->stream);
        if (J.d_factors) cudaFreeAsync(J.d_factors, b->stream);
        J = BJob();
        rs_set_error("cannot allocate the bitmap and factor buffer of a batch job");
        return RS_ENOMEM;
    }
    J.jd.bitmap = J.d_bitmap;
    J.used = true;
    const JobGeom G = job_geom(J.geom);
    BsgsArgs A;
    memset(&A, 0, sizeof A);
    A.base = J.jd.base; A.nmin = J.jd.nmin; A.nmax = J.jd.nmax; A.words = J.jd.words;
    A.bitmap = J.d_bitmap;
    A.factors = J.d_factors;
    A.factor_ctr = b->d_fctrs + jid;
    A.factor_cap = fcap;
    A.stats = b->d_stats;
    A.err = b->d_err;
    if (s)    // pageable source: the copy completes before the call returns
        BCU(cudaMemcpyAsync(J.d_bitmap, s->bitmap, J.bitmap_words * 4, cudaMemcpyHostToDevice, b->stream));
    else
        BCU(cudaMemcpyAsync(J.d_bitmap, src->d_bitmap, J.bitmap_words * 4, cudaMemcpyDeviceToDevice, b->stream));
    BCU(cudaMemcpyAsync(b->d_jobs + jid, &J.jd, sizeof(JobDev), cudaMemcpyHostToDevice, b->stream));
    BCU(cudaMemcpyAsync(b->d_geoms + jid, &G, sizeof G, cudaMemcpyHostToDevice, b->stream));
    BCU(cudaMemcpyAsync(b->d_args + jid, &A, sizeof A, cudaMemcpyHostToDevice, b->stream));
    BCU(cudaMemsetAsync(b->d_fctrs + jid, 0, 4, b->stream));
    for (u32 i = 0; i < need; ++i) {
        const u32 r = slots[i];
        const u64 lo = cuts[i], hi = cuts[i + 1];
        BatchRange R;
        memset(&R, 0, sizeof R);
        R.p_cur = lo;
        R.p_end = hi;
        R.job = jid;
        R.active = 1;
        R.mode = (hi <= FP_BOUND) ? 2 : (hi <= TOP) ? 1 : 0;
        R.geom = (u8)J.geom;
        b->h_ranges[r] = R;
        b->range_used[r] = 1;
        b->range_done[r] = 0;
        b->h_win[r] = (u32)(0.6 * RCAP);       // full windows until a budget is set
        b->win_dirty = true;
        J.ranges.push_back(r);
        BCU(cudaMemcpyAsync(b->d_ranges + r, &b->h_ranges[r], sizeof R, cudaMemcpyHostToDevice, b->stream));
        BCU(cudaMemsetAsync(b->d_range_primes + r, 0, 8, b->stream));
    }
    BCU(cudaStreamSynchronize(b->stream));     // the host structs above go out of scope
    b->done = false;
    if (job) *job = jid;
    return RS_OK;
}

extern "C" int rs_batch_reserve(rs_batch *b, uint64_t bytes)
{
    if (!b) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    void *p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, b->pool, b->stream) != cudaSuccess) {
        cudaGetLastError();
        rs_set_error("rs_batch_reserve: cannot map %llu bytes of device memory", (unsigned long long)bytes);
        return RS_ENOMEM;
    }
    BCU(cudaFreeAsync(p, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return RS_OK;
}

extern "C" int rs_batch_job_bytes(rs_batch *b, uint32_t job, uint64_t *bytes)
{
    if (!b || !bytes || job >= b->max_jobs || !b->jobs[job].used) return RS_EARG;
    const BJob &J = b->jobs[job];
    *bytes = (uint64_t)J.bitmap_words * 4 + (uint64_t)J.factor_cap * sizeof(FactorRec);
    return RS_OK;
}

extern "C" int rs_batch_free_slots(rs_batch *b, uint32_t *jobs, uint32_t *ranges)
{
    if (!b) return RS_EARG;
    u32 fj = 0, fr = 0;
    for (const auto &j : b->jobs) fj += j.used ? 0 : 1;
    for (char u : b->range_used) fr += u ? 0 : 1;
    if (jobs) *jobs = fj;
    if (ranges) *ranges = fr;
    return RS_OK;
}

extern "C" int rs_batch_release(rs_batch *b, uint32_t job)
{
    if (!b || job >= b->max_jobs || !b->jobs[job].used) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    BJob &J = b->jobs[job];
    for (u32 r : J.ranges) {
        BatchRange R;
        memset(&R, 0, sizeof R);
        b->h_ranges[r] = R;
        b->range_used[r] = 0;
        b->h_win[r] = 0;
        b->win_dirty = true;
        BCU(cudaMemcpyAsync(b->d_ranges + r, &b->h_ranges[r], sizeof R, cudaMemcpyHostToDevice, b->stream));
    }
    BCU(cudaFreeAsync(J.d_bitmap, b->stream));
    BCU(cudaFreeAsync(J.d_factors, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    J = BJob();
    return RS_OK;
}

extern "C" int rs_batch_add_clone(rs_batch *b, uint32_t src, uint64_t p0, uint64_t p1, uint32_t nsplit, uint32_t *job)
{
    if (!b || src >= b->max_jobs || !b->jobs[src].used) return RS_EARG;
    if (p1 <= p0 || p1 <= 3) {
        rs_set_error("rs_batch_add_clone: empty p-range");
        return RS_EARG;
    }
    const BJob copy = b->jobs[src];          // the slot vector is not resized, but keep a stable copy
    return batch_add_job(b, nullptr, &copy, p0, p1, 0, nsplit, job);
}

// Enqueues one round on b->stream (also what the graph captures).
static int batch_round(rs_batch *b)
{
    const u32 R = b->nranges;
    cudaStream_t st = b->stream;
    // widest window: 0.6*RCAP*ln(2^64) values, i.e. 0.3*RCAP*44.4 odd values
    const u32 max_blocks = (u32)((0.3 * RCAP * 44.4) / (SIEVE_WORDS * 32.0)) + 2;
    BCU(cudaMemsetAsync(b->d_unfinished, 0, 4, st));
    BCU(launch_batch_windows(b->d_ranges, b->d_wins, b->d_win, R, RCAP, b->d_ctrs, st));
    BCU(launch_sieve_batch(b->d_wins, R, max_blocks, b->d_sp, b->nsp, b->d_cands, CCAP, b->d_ctrs, b->d_err, st));
    BCU(launch_batch_prefix_all(b->d_ranges, R, 0, CCAP, b->d_ctrs, b->d_prefix_c, st));
    BCU(cudaMemsetAsync(b->d_mid_ctr, 0, 4, st));
    BCU(launch_mr_batch2(b->d_cands, CCAP, b->d_primes, RCAP, b->d_ctrs, R, b->d_prefix_c, b->d_mid, b->d_mid_r,
                         R * CCAP, b->d_mid_ctr, b->d_err, b->sms, st));
    BCU(launch_batch_prefix_all(b->d_ranges, R, 1, RCAP, b->d_ctrs, b->d_prefix_p, st));
    BCU(launch_setup_batch(b->d_jobs, b->d_geoms, b->d_ranges, b->d_primes, RCAP, b->d_prefix_p, R, b->d_hdr,
                           b->d_aux, b->d_tabs, b->d_tgt, b->d_meta, b->d_stats, b->d_err, b->d_rec_of, b->sms,
                           st));
    BsgsArgs a;
    memset(&a, 0, sizeof a);
    a.stats = b->d_stats;
    a.err = b->d_err;
    // the groups' prefix sums in one launch, then one persistent BSGS launch per
    // group on its own branch (fork/join through events, so a captured round is
    // a graph with parallel branches): one group's last wave overlaps the others
    BCU(launch_batch_group_prefix(b->d_ranges, R, b->d_ctrs, RCAP, b->d_gprefix, b->d_gwork, st));
    BCU(cudaEventRecord(b->fork, st));
    for (int g = 0; g < NGROUP; ++g) {
        BCU(cudaStreamWaitEvent(b->side[g], b->fork, 0));
        BCU(launch_bsgs_batch(a, b->d_args, b->d_hdr, b->d_tabs, b->d_tgt, b->d_meta, R,
                              b->d_gprefix + (size_t)g * (R + 1), RCAP, b->d_gwork + g, g % 3, g / 3, b->sms,
                              b->side[g]));
        BCU(cudaEventRecord(b->join[g], b->side[g]));
        BCU(cudaStreamWaitEvent(st, b->join[g], 0));
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
    bool any = false;
    for (char u : b->range_used) any = any || u;
    if (!any) b->done = true;
    for (uint32_t i = 0; (max_rounds == 0 || i < max_rounds) && !b->done; ++i) {
        if (b->win_dirty) {                          // per-slot round targets, read by the round's first kernel
            memcpy(b->h_win_pin, b->h_win.data(), b->nranges * 4);
            BCU(cudaMemcpyAsync(b->d_win, b->h_win_pin, b->nranges * 4, cudaMemcpyHostToDevice, b->stream));
            b->win_dirty = false;
        }
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
        bool any_win = false;
        for (u32 r = 0; r < b->nranges; ++r) any_win = any_win || (b->range_used[r] && b->h_win[r]);
        if (!any_win) break;                         // every unfinished range is paused: nothing to run
    }
    if (done) *done = b->done ? 1 : 0;
    return RS_OK;
}

extern "C" int rs_batch_set_budget(rs_batch *b, uint32_t job, uint64_t primes)
{
    if (!b || job >= b->max_jobs || !b->jobs[job].used) return RS_EARG;
    const BJob &J = b->jobs[job];
    u32 live = 0;
    for (u32 r : J.ranges) live += b->range_done[r] ? 0 : 1;
    const u64 cap = (u64)(0.6 * RCAP);
    for (u32 r : J.ranges) {
        u64 w = 0;
        if (!b->range_done[r] && live) w = (primes + live - 1) / live;
        if (w > cap) w = cap;
        if (b->h_win[r] != (u32)w) {
            b->h_win[r] = (u32)w;
            b->win_dirty = true;
        }
    }
    return RS_OK;
}

extern "C" int rs_batch_poll(rs_batch *b, uint8_t *done, uint64_t *primes, uint64_t *remaining)
{
    if (!b) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    const u32 R = b->nranges;
    std::vector<BatchRange> rr(R);
    std::vector<u64> rp(R);
    BCU(cudaMemcpyAsync(rr.data(), b->d_ranges, R * sizeof(BatchRange), cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaMemcpyAsync(rp.data(), b->d_range_primes, R * 8, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    for (u32 j = 0; j < b->max_jobs; ++j) {
        const BJob &J = b->jobs[j];
        u64 n = 0, rem = 0;
        bool all = true;
        for (u32 r : J.ranges) {
            const bool fin = rr[r].p_cur >= rr[r].p_end;
            b->range_done[r] = fin ? 1 : 0;
            n += rp[r];
            rem += fin ? 0 : rr[r].p_end - rr[r].p_cur;
            all = all && fin;
        }
        if (done) done[j] = (J.used && all) ? 1 : 0;
        if (primes) primes[j] = n;
        if (remaining) remaining[j] = rem;
    }
    return RS_OK;
}

extern "C" int rs_batch_factors_fetch(rs_batch *b, uint32_t job, rs_factor *buf, size_t cap, size_t *n)
{
    if (!b || !n || job >= b->max_jobs || !b->jobs[job].used) return RS_EARG;
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
    if (!b || !dst || job >= b->max_jobs || !b->jobs[job].used || words < b->jobs[job].bitmap_words) return RS_EARG;
    BCU(cudaSetDevice(b->device));
    BCU(cudaMemcpyAsync(dst, b->jobs[job].d_bitmap, b->jobs[job].bitmap_words * 4, cudaMemcpyDeviceToHost, b->stream));
    BCU(cudaStreamSynchronize(b->stream));
    return RS_OK;
}

extern "C" int rs_batch_job_info(rs_batch *b, uint32_t job, uint32_t *q, uint64_t *primes, int *done)
{
    if (!b || job >= b->max_jobs || !b->jobs[job].used) return RS_EARG;
    const BJob &J = b->jobs[job];
    if (q) *q = BSGS_GEOMS[J.geom].q;
    if (!primes && !done) return RS_OK;
    BCU(cudaSetDevice(b->device));
    u64 n = 0;
    bool all = true;
    for (u32 r : J.ranges) {
        u64 rp = 0;
        BatchRange rr;
        BCU(cudaMemcpyAsync(&rp, b->d_range_primes + r, 8, cudaMemcpyDeviceToHost, b->stream));
        BCU(cudaMemcpyAsync(&rr, b->d_ranges + r, sizeof rr, cudaMemcpyDeviceToHost, b->stream));
        BCU(cudaStreamSynchronize(b->stream));
        n += rp;
        all = all && rr.p_cur >= rr.p_end;
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

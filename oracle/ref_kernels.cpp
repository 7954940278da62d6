/*
 * ref_kernels.cpp -- builds the reference's own kernels/common.cl, setup.cl and
 * sort.cl (from where they lie in the reference tree; REFDIR is passed by the
 * Makefile) and its verify_factor.c into oracle/_ref/librsref.so, with a small
 * C driver that runs them one work-item at a time, like cl_sieve.cpp:1322-1326
 * launches setup and sort over a segment.  TEST INFRASTRUCTURE ONLY.
 */
#include "ref_shim.hpp"
#include <cstring>
#include <vector>

#define RS_STR2(x) #x
#define RS_STR(x) RS_STR2(x)

namespace refshim {
thread_local size_t g_gid;
int *g_klist;
int g_kcount;
uint32_t g_Q, g_NMIN, g_LS;
}  // namespace refshim

#define __kernel
#define __global
#define KCOUNT ::refshim::g_kcount
#define Q ::refshim::g_Q
#define NMIN ::refshim::g_NMIN
#define LS ::refshim::g_LS
#define klist ::refshim::g_klist
#define ulong uint64_t
#define uint uint32_t

/* one namespace per base literal (common.cl:74-85, setup.cl:122-131 test BASE with #if) */
#define BASE 2
namespace ref_b2 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#define BASE 3
namespace ref_b3 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#define BASE 5
namespace ref_b5 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#define BASE 6
namespace ref_b6 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#define BASE 7
namespace ref_b7 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#define BASE 10
namespace ref_b10 {
using namespace ::refshim;
#include RS_STR(REFDIR/kernels/common.cl)
#include RS_STR(REFDIR/kernels/setup.cl)
#include RS_STR(REFDIR/kernels/sort.cl)
}
#undef BASE
#undef ulong
#undef uint
#undef klist

namespace refv {
#include RS_STR(REFDIR/verify_factor.c)
}

using refshim::ulong8;

template <class NSKD, class NSKP, class SetupF, class SortF>
static int run(SetupF setupf, SortF sortf, uint32_t kcount, const int32_t *kl, uint32_t nmin, uint32_t Qv,
               uint32_t LSv, const uint64_t *primes, uint32_t np, uint64_t *rows_setup, uint64_t *kd_hadj,
               int32_t *kd_parity, int32_t *kd_kidx, uint32_t *counts, uint64_t *rows_cls, uint64_t *kp_hadj,
               int32_t *kp_kidx, int32_t *kcounts)
{
    std::vector<int> klv(kl, kl + kcount);
    refshim::g_klist = klv.data();
    refshim::g_kcount = (int)kcount;
    refshim::g_Q = Qv;
    refshim::g_NMIN = nmin;
    refshim::g_LS = LSv;
    std::vector<ulong8> gp(np), gf(np), ge(np), go(np);
    for (uint32_t i = 0; i < np; ++i) {
        /* the row getsegprimes.cl:173-179 writes */
        uint64_t p = primes[i];
        uint64_t q = ::ref_b2::invert(p), one = (0 - p) % p, nmo = p - one, two = ::ref_b2::add(one, one, p);
        gp[i].s0 = p; gp[i].s1 = q; gp[i].s2 = one; gp[i].s3 = two; gp[i].s4 = nmo;
        gp[i].s5 = 0; gp[i].s6 = 0; gp[i].s7 = 0;
    }
    std::vector<NSKD> gk((size_t)np * kcount);
    std::vector<NSKP> kf((size_t)np * kcount), ke((size_t)np * kcount), ko((size_t)np * kcount);
    std::vector<int> cf(np), ce(np), co(np);
    uint32_t pc[7] = {np, 0, 0, 0, 0, 0, 0};
    uint64_t sum = 0;
    for (uint32_t g = 0; g < np; ++g) { refshim::g_gid = g; setupf(gp.data(), pc, gk.data(), &sum); }
    for (uint32_t i = 0; i < np; ++i) {
        uint64_t *r = rows_setup + (size_t)i * 8;
        r[0] = gp[i].s0; r[1] = gp[i].s1; r[2] = gp[i].s2; r[3] = gp[i].s3;
        r[4] = gp[i].s4; r[5] = gp[i].s5; r[6] = gp[i].s6; r[7] = gp[i].s7;
        for (uint32_t j = 0; j < kcount; ++j) {
            const NSKD &d = gk[(size_t)i * kcount + j];
            kd_hadj[(size_t)i * kcount + j] = d.hadj;
            kd_parity[(size_t)i * kcount + j] = d.parity;
            kd_kidx[(size_t)i * kcount + j] = d.kidx;
        }
    }
    for (uint32_t g = 0; g < np; ++g) {
        refshim::g_gid = g;
        sortf(pc, gp.data(), gf.data(), ge.data(), go.data(), gk.data(), kf.data(), ke.data(), ko.data(), cf.data(),
              ce.data(), co.data());
    }
    counts[0] = pc[3]; counts[1] = pc[4]; counts[2] = pc[5];
    const std::vector<ulong8> *cls[3] = {&gf, &ge, &go};
    const std::vector<NSKP> *kls[3] = {&kf, &ke, &ko};
    const std::vector<int> *kcs[3] = {&cf, &ce, &co};
    for (int c = 0; c < 3; ++c) {
        for (uint32_t i = 0; i < counts[c]; ++i) {
            const ulong8 &u = (*cls[c])[i];
            uint64_t *r = rows_cls + ((size_t)c * np + i) * 8;
            r[0] = u.s0; r[1] = u.s1; r[2] = u.s2; r[3] = u.s3; r[4] = u.s4; r[5] = u.s5; r[6] = u.s6; r[7] = u.s7;
            int nk = (*kcs[c])[i];
            kcounts[(size_t)c * np + i] = nk;
            for (int j = 0; j < nk; ++j) {
                const NSKP &kp = (*kls[c])[(size_t)i * kcount + j];
                kp_hadj[((size_t)c * np + i) * kcount + j] = kp.hadj;
                kp_kidx[((size_t)c * np + i) * kcount + j] = kp.kidx;
            }
        }
    }
    return 0;
}

#define DISPATCH(NS)                                                                                   \
    return run<NS::kdata, NS::kparity>(NS::setup, NS::sort, kcount, klist_in, nmin, Qv, LSv, primes, np, \
                                       rows_setup, kd_hadj, kd_parity, kd_kidx, counts, rows_cls, kp_hadj,    \
                                       kp_kidx, kcounts)

extern "C" {
/* Runs the reference's setup kernel then its sort kernel over np primes.
 * Outputs (caller-allocated):
 *   rows_setup[np*8]          g_prime after setup (s0==0: skipped)
 *   kd_*[np*kcount]           g_k kdata after setup
 *   counts[3]                 g_primecount[3..5] after sort (#full, #even, #odd rows)
 *   rows_cls[3*np*8]          g_prime_full / _even / _odd rows
 *   kp_*[3*np*kcount]         g_k_full / _even / _odd kparity
 *   kcounts[3*np]             g_kcount_full / _even / _odd
 * Returns -1 for a base that has no compiled namespace. */
int rsref_setup_sort(uint32_t base, uint32_t kcount, const int32_t *klist_in, uint32_t nmin, uint32_t Qv, uint32_t LSv,
                     const uint64_t *primes, uint32_t np, uint64_t *rows_setup, uint64_t *kd_hadj, int32_t *kd_parity,
                     int32_t *kd_kidx, uint32_t *counts, uint64_t *rows_cls, uint64_t *kp_hadj, int32_t *kp_kidx,
                     int32_t *kcounts)
{
    switch (base) {
    case 2: DISPATCH(ref_b2);
    case 3: DISPATCH(ref_b3);
    case 5: DISPATCH(ref_b5);
    case 6: DISPATCH(ref_b6);
    case 7: DISPATCH(ref_b7);
    case 10: DISPATCH(ref_b10);
    default: return -1;
    }
}

/* the reference's verify_factor.c:131-181, unmodified */
int rsref_verify_factor(uint64_t p, uint64_t k, uint32_t n, int32_t c, uint32_t base)
{
    return refv::verify_factor(p, k, n, c, base);
}

/* the reference's isPrime (verify_factor.c:100-128), with the set-up
 * verify_factor.c:134-141 performs before calling it */
int rsref_is_prime(uint64_t p)
{
    uint64_t q = refv::invert(p), one = (0 - p) % p, pmo = p - one, two = refv::add(one, one, p);
    uint64_t t = refv::add(two, two, p);
    for (int i = 0; i < 5; ++i) t = refv::m_mul(t, t, p, q);
    return refv::isPrime(p, q, one, pmo, two, t) ? 1 : 0;
}

/* strong_prp_two of getsegprimes.cl is not C++; the same base-2 strong PRP
 * test is verify_factor.c's strong_prp (verify_factor.c:57-95) with base 2 */
int rsref_sprp2(uint64_t n)
{
    if (n < 3 || !(n & 1)) return 0;
    uint64_t q = refv::invert(n), one = (0 - n) % n, pmo = n - one, two = refv::add(one, one, n);
    uint64_t t = refv::add(two, two, n);
    for (int i = 0; i < 5; ++i) t = refv::m_mul(t, t, n, q);
    int tz = __builtin_ctzll(n - 1);
    uint64_t exp = n >> tz;
    uint64_t cur = 0x8000000000000000ULL >> ((__builtin_clzll(exp) + 1) & 63);
    return refv::strong_prp(2, n, q, one, pmo, t, tz, exp, cur) ? 1 : 0;
}

uint64_t rsref_m_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t q) { return ref_b2::m_mul(a, b, p, q); }
uint64_t rsref_invert(uint64_t p) { return ref_b2::invert(p); }
uint64_t rsref_powmodlg(uint64_t mbase, uint64_t exp, uint64_t p, uint64_t q) { return ref_b2::powmodlg(mbase, exp, p, q); }
}

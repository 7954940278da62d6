/*
 * ref_shim.hpp -- lets the reference's OpenCL C kernels kernels/common.cl,
 * kernels/setup.cl and kernels/sort.cl compile unmodified as C++ so that the
 * oracle can run the reference's own per-prime setup, prefilter and parity
 * sort on the CPU.  TEST INFRASTRUCTURE ONLY (see rsoracle.h).
 *
 * What it maps:
 *   ulong/uint            -> uint64_t/uint32_t
 *   mul_hi, clz           -> __int128 / __builtin_clz*
 *   atomic_inc            -> __atomic_fetch_add (kernels run one work-item at a time)
 *   get_global_id(0)      -> a thread_local set by the driver loop
 *   ulong8 (.s0-.s7)      -> a struct of lane_t; the OpenCL vector literal
 *                            (ulong8)(a,b,...,h) is built by an overloaded comma
 *                            on lane_t, since in C++ it is a cast of a comma
 *                            expression (its first operand is always a .sN lane
 *                            in sort.cl:300-312)
 *   -D constants          -> runtime globals (KCOUNT, Q, NMIN, LS, klist); BASE
 *                            stays a literal because common.cl/setup.cl test it
 *                            with #if, so one namespace is built per base.
 * kernels/giant.cl and kernels/getsegprimes.cl are not valid C++ (OpenCL __local
 * pointers in parameter lists, unmarked vector literals) and are restated in
 * rsoracle.c instead.
 */
#pragma once
#include <cstdint>
#include <cstddef>
#include <cinttypes>
#include <cstdio>
#include <sys/types.h>

namespace refshim {
struct lane_t {
    uint64_t v;
    lane_t() = default;
    explicit lane_t(uint64_t x) : v(x) {}
    operator uint64_t() const { return v; }
    lane_t &operator=(uint64_t x) { v = x; return *this; }
};
struct u8b { uint64_t v[8]; int n; };
inline u8b operator,(lane_t a, uint64_t b) { u8b r{}; r.v[0] = a.v; r.v[1] = b; r.n = 2; return r; }
inline u8b operator,(u8b a, uint64_t b) { if (a.n < 8) a.v[a.n] = b; a.n++; return a; }
struct ulong8 {
    lane_t s0, s1, s2, s3, s4, s5, s6, s7;
    ulong8() = default;
    explicit ulong8(u8b b) : s0(b.v[0]), s1(b.v[1]), s2(b.v[2]), s3(b.v[3]),
                             s4(b.v[4]), s5(b.v[5]), s6(b.v[6]), s7(b.v[7]) {}
};
inline uint64_t mul_hi(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) >> 64); }
inline uint64_t clz(uint64_t x) { return x ? (uint64_t)__builtin_clzll(x) : 64; }
inline uint32_t clz(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32; }
inline uint32_t atomic_inc(uint32_t *p) { return __atomic_fetch_add(p, 1u, __ATOMIC_RELAXED); }

extern thread_local size_t g_gid;
inline size_t get_global_id(int) { return g_gid; }

/* runtime values of the reference's -D constants (cl_sieve.cpp:1010-1011) */
extern int *g_klist;
extern int g_kcount;
extern uint32_t g_Q, g_NMIN, g_LS;
}  // namespace refshim

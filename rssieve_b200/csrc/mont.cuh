// mont.cuh -- exact 64-bit modular arithmetic for sm_100a.
//
// Montgomery representation with R = 2^64: x is held as x*R mod p.  The
// product is REDC(a*b) = a*b*R^-1 mod p with q = p^-1 mod 2^64, the same
// reduction the reference uses (kernels/common.cl:33-40): because m*p agrees
// with a*b in the low 64 bits, the result is hi(a*b) - hi(m*p), corrected by
// +p when negative.  Valid for every odd p < 2^64 when a*b < p*2^64.
//
#pragma once
#include <cstdint>

typedef unsigned long long u64;
typedef unsigned int u32;

#define RS_DEV __device__ __forceinline__

// Montgomery product: a*b*2^-64 mod p, result in [0,p).  Written with plain
// 64-bit products: nvcc lowers a*b and __umul64hi to IMAD.WIDE sequences that
// measured 20% faster than hand-written 32-bit carry chains on sm_100a.
RS_DEV u64 mmul(u64 a, u64 b, u64 p, u64 q)
{
    const u64 lo = a * b;
    const u64 hi = __umul64hi(a, b);
    const u64 m = lo * q;
    const u64 mp = __umul64hi(m, p);
    const u64 r = hi - mp;
    return (hi < mp) ? r + p : r;
}

// x*w mod p for a fixed multiplier w < p with its precomputed quotient
// wp = floor(w*2^64/p) (Shoup's method; for p < 2^63).  For any x < 2^64,
// x*w - floor(x*wp/2^64)*p lies in [0, 2p): one conditional subtraction.
// Ten 32x32 products against the Montgomery product's eleven, with shorter
// carry chains.  The representation of x is preserved (x*R times w stays
// x*w*R), so it mixes freely with Montgomery-form values.
RS_DEV u64 shoup_mul(u64 x, u64 w, u64 wp, u64 p)
{
    const u64 qh = __umul64hi(x, wp);
    const u64 r = x * w - qh * p;
    return (r >= p) ? r - p : r;
}

// Montgomery product without the final correction, for p < 2^62: for a, b in
// [0, 2p), (a*b - m*p)/2^64 lies in (-p, p), so adding p gives a result in
// (0, 2p) congruent to a*b*2^-64.  Chains of products stay in [0, 2p); one
// conditional subtraction (mred) makes the end result canonical.
RS_DEV u64 mmul_lazy(u64 a, u64 b, u64 p, u64 q)
{
    const u64 lo = a * b;
    const u64 hi = __umul64hi(a, b);
    const u64 m = lo * q;
    return hi + p - __umul64hi(m, p);
}
RS_DEV u64 mred(u64 x, u64 p) { return (x >= p) ? x - p : x; }

// mmul_lazy(a, a) with the square formed from three 32x32 products instead of
// a general 64x64 product: a = a1*2^32 + a0 < 2^63 gives a^2 = a1^2*2^64 +
// (2*a0*a1)*2^32 + a0^2, where 2*a0*a1 < 2^64 since a1 < 2^31.
RS_DEV u64 msqr_lazy(u64 a, u64 p, u64 q)
{
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32);
    const u64 l = (u64)a0 * a0;
    const u64 m = (u64)a0 * a1;
    const u64 lo = l + (m << 33);
    const u64 hi = (u64)a1 * a1 + (m >> 31) + (lo < l ? 1u : 0u);
    const u64 t = lo * q;
    return hi + p - __umul64hi(t, p);
}

// round(a*b + c) - c for the exact product a*b, with c = 1.5*2^52: the fma
// rounds once into [2^52, 2^53), where the doubles are the integers, so this
// is a*b rounded to the nearest integer (ties to even) for |a*b| < 2^51, on
// the FP64 pipe (rint would run on the slower conversion unit).
RS_DEV double fp_round_prod(double a, double b)
{
    const double c = 6755399441055744.0;
    return fma(a, b, c) - c;
}

// x*w mod p on the FP64 pipe, for p < 2^51 and x, w in [0, p) held exactly in
// doubles, with wq = w/p (correctly rounded).  h = x*w rounded and the exact
// error l = fma(x, w, -h) (the two-product of Dekker and Kahan's FMA form) give
// x*w = h + l.  q, the exact product x*wq rounded to an integer, is within 1 of
// t = x*w/p: wq carries one rounding, a relative error below 2^-53, i.e. below
// 1/4 since t < p < 2^51, and the rounding adds at most 1/2.  So r = x*w - q*p
// lies in (-p, p); it is formed exactly, since h - q*p is an integer below
// 2^53 in magnitude (one fma) and adding l stays below 2^53.  One correction
// makes it canonical.  About eight FP64 operations, against eighteen integer
// ones for Shoup's product.
RS_DEV double fp_mulfix(double x, double w, double wq, double p)
{
    const double h = x * w;
    const double l = fma(x, w, -h);
    const double q = fp_round_prod(x, wq);
    const double r = fma(-q, p, h) + l;
    return (r < 0.0) ? r + p : r;
}

// x*y mod p on the FP64 pipe for two variable factors, p < 2^51, with pinv =
// 1/p: as fp_mulfix, with the quotient from the exact product h*pinv rounded
// to an integer.  h and pinv carry one rounding each, a relative error below
// 2^-52, i.e. below 1/2 for t = x*y/p < 2^51, so again q is within 1 of t and
// r lies in (-p, p).
RS_DEV double fp_mul(double x, double y, double p, double pinv)
{
    const double h = x * y;
    const double l = fma(x, y, -h);
    const double q = fp_round_prod(h, pinv);
    const double r = fma(-q, p, h) + l;
    return (r < 0.0) ? r + p : r;
}

// fp_mul without its correction, for chains of products: for x, y in (-p, p)
// the bounds above hold unchanged (|x*y| < p^2, so |t| < p and q is within 1
// of t), hence r = x*y - q*p is exact and lies in (-p, p) again.  A chain
// stays in signed residues and is made canonical once at its end.
RS_DEV double fp_mul_signed(double x, double y, double p, double pinv)
{
    const double h = x * y;
    const double l = fma(x, y, -h);
    const double q = fp_round_prod(h, pinv);
    return fma(-q, p, h) + l;
}

// The double equal to v < 2^52, without a conversion instruction: v in the
// mantissa of 2^52 + v (exponent field 0x433), then 2^52 subtracted exactly.
RS_DEV double fp_exact(u64 v)
{
    return __longlong_as_double((long long)(0x4330000000000000ull | v)) - 4503599627370496.0;
}

// The integer held by a double d in [0, 2^52), without a conversion
// instruction: d + 2^52 puts it in the mantissa (exactly), which is masked out.
RS_DEV u64 fp_int(double d)
{
    return (u64)__double_as_longlong(d + 4503599627370496.0) & ((1ull << 52) - 1);
}

// 2x mod p for x in [0, p), p < 2^52: exact in FP64.
RS_DEV double fp_dbl(double x, double p)
{
    const double d = x + x;
    return (d >= p) ? d - p : d;
}

// Shoup's quotient floor(w * 2^64 / p) of the plain value w < p < 2^63, from
// its Montgomery form wm = w * 2^64 mod p: w * 2^64 = wp * p + wm, so
// wp * p == -wm (mod 2^64) and wp = -wm * p^-1 mod 2^64 (q = p^-1 mod 2^64).
RS_DEV u64 shoup_of_mont(u64 wm, u64 q) { return (0 - wm) * q; }

// a + b mod p for a, b in [0,p); correct for p up to 2^64-1 (wrapping add).
RS_DEV u64 madd(u64 a, u64 b, u64 p)
{
    u64 c = (a >= p - b) ? p : 0;
    return a + b - c;
}

RS_DEV u64 msub(u64 a, u64 b, u64 p) { return (a >= b) ? a - b : a - b + p; }
RS_DEV u64 mneg(u64 a, u64 p) { return a ? p - a : 0; }

// p^-1 mod 2^64 by Newton iteration: p*p == 1 mod 8 gives 3 correct bits,
// each step doubles them (3, 6, 12, 24, 48, 96).
RS_DEV u64 inv64(u64 p)
{
    u64 x = p;
#pragma unroll
    for (int i = 0; i < 5; ++i) x *= 2 - p * x;
    return x;
}

// 2^64 mod p for odd p >= 3 without a 64-bit division: reduce 2^64 - p' by
// binary long division, where p' = p << s has its top bit set.
RS_DEV u64 r_mod(u64 p)
{
    int s = __clzll(p);
    u64 ps = p << s;              // ps in [2^63, 2^64)
    u64 r = 0 - ps;               // 2^64 - ps < ps, and 2^64 == r (mod ps)
    // r == 2^64 (mod ps) hence (mod p); now reduce r from < p*2^s to < p
    for (int i = s - 1; i >= 0; --i) {
        u64 t = p << i;
        if (r >= t) r -= t;
    }
    return r;
}

// Montgomery constants of one prime.
struct Mont {
    u64 p, q, one, r2;
};

RS_DEV Mont mont_init(u64 p)
{
    Mont M;
    M.p = p;
    M.q = inv64(p);
    M.one = r_mod(p);
    // R^2 = (4R)^(2^5) in Montgomery form (4^32 = 2^64), as setup.cl:112-119
    u64 two = madd(M.one, M.one, p);
    u64 t = madd(two, two, p);
#pragma unroll
    for (int i = 0; i < 5; ++i) t = mmul(t, t, p, M.q);
    M.r2 = t;
    return M;
}

RS_DEV u64 to_mont(u64 x, const Mont &M) { return mmul(x, M.r2, M.p, M.q); }   // any x < 2^64
RS_DEV u64 from_mont(u64 x, const Mont &M) { return mmul(x, 1, M.p, M.q); }

// x^e for a Montgomery x, left-to-right binary; e may be 0 or 1.
RS_DEV u64 mpow(u64 x, u64 e, const Mont &M)
{
    if (e == 0) return M.one;
    u64 a = x;
    for (int bit = 62 - __clzll(e); bit >= 0; --bit) {
        a = mmul(a, a, M.p, M.q);
        if ((e >> bit) & 1) a = mmul(a, x, M.p, M.q);
    }
    return a;
}

// x * b mod p for a small integer multiplier b in [1, 16] by doubling and
// adding (no multiply); the reference does the same for b = 2, 3, 5
// (common.cl:74-85).  Larger b use mmul with the Montgomery form of b.
RS_DEV u64 mul_small(u64 x, u32 b, u64 p)
{
    u64 acc = x;
    int top = 31 - __clz(b);
    for (int i = top - 1; i >= 0; --i) {
        acc = madd(acc, acc, p);
        if ((b >> i) & 1) acc = madd(acc, x, p);
    }
    return acc;
}

// Multiplication by the base: mul_small when b <= 16, else Montgomery.
RS_DEV u64 mul_base(u64 x, u32 b, u64 bm, const Mont &M)
{
    return (b <= 16) ? mul_small(x, b, M.p) : mmul(x, bm, M.p, M.q);
}

// Jacobi symbol (a/n) for odd n > 0 and 0 <= a < n: binary algorithm
// (strip factors of two with the (2/n) rule, swap with quadratic
// reciprocity, subtract).  Returns -1, 0 or 1.
RS_DEV int jacobi32(u32 a, u32 n)
{
    int t = 1;
    while (a) {
        int z = __ffs((int)a) - 1;
        a >>= z;
        u32 r8 = n & 7;
        if ((z & 1) && (r8 == 3 || r8 == 5)) t = -t;
        if (a < n) {
            u32 tmp = a; a = n; n = tmp;
            if ((a & 3) == 3 && (n & 3) == 3) t = -t;
        }
        a -= n;
    }
    return (n == 1) ? t : 0;
}

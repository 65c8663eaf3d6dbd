// elementary.cuh -- deterministic FP64 elementary functions for the D-Claw step.
//
// exp, expm1, tanh, pow, atan, tan and log, written with only IEEE +,
// -, *, /, fused multiply-add, rint and bit operations, so that a host build
// (g++ -ffp-contract=off) and the sm_100a build (--fmad=false; the fused
// multiply-adds are explicit fma() calls) return the same bits for the same
// argument. The CUDA step uses these in place of the toolkit's libm; the
// oracle can use them too ("portable libm" mode), which makes GPU-vs-oracle
// parity exact to the bit.
//
// Two families:
//  * exp, expm1, tanh and pow (h^(7/3), 10^y, x^(1/3)) restate the
//    published algorithms glibc runs
//    on x86-64 (ARM optimized-routines' exp and pow; fdlibm's expm1 and
//    tanh), with their constants and their fused multiply-adds, so they
//    return glibc's bits: the libm of the reference's gfortran build on
//    x86-64 Linux.
//  * atan and tan are correctly rounded (glibc's, from IBM's Accurate
//    Mathematical Library, rest on tables of Gal's accurate-table points
//    that are not derivable from a definition; they are correctly rounded
//    in all but about 0.2 % of arguments).
//  * log (src2method 2 only) is this project's own, within 2 ulp: glibc's
//    rests on a searched table.
//
// log's method (published): x = 2^k f with f in [sqrt(1/2), sqrt(2));
// log f = 2 atanh(s), s = (f - 1)/(f + 1) (f - 1 exact), by the Taylor
// series of atanh on |s| <= 0.1716; log x = k ln2_hi + (k ln2_lo + log f).
// The methods of atan and tan are given where they are defined.
// Constants of the project's own functions were produced with 80-digit
// decimal arithmetic; the tables with 300-bit arithmetic (gen_libm_tables.py).
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

#include "libm_tables.cuh"

#ifndef DC_HD
#if defined(__CUDACC__)
#define DC_HD __host__ __device__ __forceinline__
#else
#define DC_HD inline
#endif
#endif

namespace dclaw {
namespace em {

DC_HD double bits2d(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
#endif
}

DC_HD uint64_t d2bits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t b;
    memcpy(&b, &d, sizeof b);
    return b;
#endif
}

// 2^k for -1022 <= k <= 1023
DC_HD double pow2i(int k) { return bits2d((uint64_t)(k + 1023) << 52); }

constexpr double LN2_HI = 0.6931471803691238;        // 0x3fe62e42fee00000 (32-bit head)
constexpr double LN2_LO = 1.9082149292705877e-10;    // tail
constexpr double PIO2_1 = 1.5707963267341256;        // pi/2 in three 33-bit pieces
constexpr double PIO2_2 = 6.077100506303966e-11;
constexpr double PIO2_3 = 2.0222662487959506e-21;
constexpr double TWO_OVER_PI = 0.6366197723675814;   // 0x3fe45f306dc9c883
constexpr double PIO2_HI = 1.5707963267948966;       // pi/2 head + tail
constexpr double PIO2_LO = 6.123233995736766e-17;

// 1/n!
constexpr double IF2 = 0.5, IF3 = 0.16666666666666666, IF4 = 0.041666666666666664,
                 IF5 = 0.008333333333333333, IF6 = 0.001388888888888889, IF7 = 0.0001984126984126984,
                 IF8 = 2.48015873015873e-05, IF9 = 2.7557319223985893e-06, IF10 = 2.755731922398589e-07,
                 IF11 = 2.505210838544172e-08, IF12 = 2.08767569878681e-09, IF13 = 1.6059043836821613e-10,
                 IF14 = 1.1470745597729725e-11, IF15 = 7.647163731819816e-13, IF16 = 4.779477332387385e-14,
                 IF17 = 2.8114572543455206e-15, IF18 = 1.5619206968586225e-16, IF19 = 8.22063524662433e-18,
                 IF20 = 4.110317623312165e-19;

// ---- exp: the table-driven method of ARM's optimized-routines -------------
// exp(x) = 2^(k/128) e^r with x = k ln2/128 + r, |r| <= ln2/256; 2^(k/128) =
// H (1 + T) from a 128-entry table (libm_tables.cuh, generated from that
// definition); e^r - 1 by a degree-5 polynomial. This is the published
// algorithm (optimized-routines math/exp.c, Szabolcs Nagy 2018) that glibc
// uses from 2.28 on (sysdeps/ieee754/dbl-64/e_exp.c), with its constants,
// and with the fused multiply-adds that glibc's x86-64 FMA build of it
// executes (GCC contracts a*b + c where the product has one use in the same
// basic block): the results are glibc's to the bit on an x86-64 host with
// FMA, the libm the reference's gfortran build calls (measured: no
// difference in 6e7 random arguments over the whole range, subnormal
// results included). Within 0.51 ulp.
#if defined(__CUDACC__)
static __device__ const uint64_t EXP_TAB_DEV[256] = {DCLAW_EXP_TABLE_DATA};
#endif
static const uint64_t EXP_TAB_HOST[256] = {DCLAW_EXP_TABLE_DATA};

DC_HD uint64_t exp_tab(unsigned i) {
#if defined(__CUDA_ARCH__)
    return __ldg(reinterpret_cast<const unsigned long long*>(EXP_TAB_DEV) + i);
#else
    return EXP_TAB_HOST[i];
#endif
}

constexpr double EXP_INVLN2N = 0x1.71547652b82fep0 * 128.0, EXP_SHIFT = 0x1.8p52,
                 EXP_NEGLN2HIN = -0x1.62e42fefa0000p-8, EXP_NEGLN2LON = -0x1.cf79abc9e3b3ap-47,
                 EXP_C2 = 0x1.ffffffffffdbdp-2, EXP_C3 = 0x1.555555555543cp-3, EXP_C4 = 0x1.55555cf172b91p-5,
                 EXP_C5 = 0x1.1111167a4d017p-7;

DC_HD unsigned top12(double x) { return (unsigned)(d2bits(x) >> 52); }

// |x| >= 512: the scale 2^(k/128) is outside the normal range and is applied
// in two steps; below 2^-1022 the sum is rounded once before scaling
DC_HD double exp_special(double tmp, uint64_t sbits, uint64_t ki) {
    if ((ki & 0x80000000ull) == 0) {
        sbits -= 1009ull << 52;
        const double scale = bits2d(sbits);
        return 0x1p1009 * fma(scale, tmp, scale);
    }
    sbits += 1022ull << 52;
    const double scale = bits2d(sbits);
    // the product feeds two sums in different blocks: not fused
    const double st = scale * tmp;
    double y = scale + st;
    if (y < 1.0) {
        double lo = scale - y + st;
        const double hi = 1.0 + y;
        lo = 1.0 - hi + y + lo;
        y = (hi + lo) - 1.0;
        if (y == 0.0) y = 0.0;
    }
    return 0x1p-1022 * y;
}

// e^(x + xtail) for finite x, |xtail| < 2^-15 |x| (0 for exp itself: adding
// it changes no bit); pow calls it with the low part of y log x
DC_HD double exp_core(double x, double xtail) {
    unsigned abstop = top12(x) & 0x7ffu;
    if (abstop - top12(0x1p-54) >= top12(512.0) - top12(0x1p-54)) {
        if ((int)(abstop - top12(0x1p-54)) < 0) return 1.0 + x;  // |x| < 2^-54
        if (abstop >= top12(1024.0)) return (d2bits(x) >> 63) ? 0.0 : bits2d(0x7ff0000000000000ull);
        abstop = 0;  // 512 <= |x| < 1024
    }
    double kd = fma(EXP_INVLN2N, x, EXP_SHIFT);
    const uint64_t ki = d2bits(kd);
    kd -= EXP_SHIFT;
    double r = fma(kd, EXP_NEGLN2LON, fma(kd, EXP_NEGLN2HIN, x));
    r += xtail;
    const unsigned idx = 2u * (unsigned)(ki % 128u);
    const uint64_t top = ki << 45;
    const double tail = bits2d(exp_tab(idx));
    const uint64_t sbits = exp_tab(idx + 1) + top;
    const double r2 = r * r;
    const double tmp = fma(r2 * r2, fma(r, EXP_C5, EXP_C4), fma(r2, fma(r, EXP_C3, EXP_C2), tail + r));
    if (abstop == 0) return exp_special(tmp, sbits, ki);
    const double scale = bits2d(sbits);
    return fma(scale, tmp, scale);
}

DC_HD double d_exp(double x) {
    const unsigned abstop = top12(x) & 0x7ffu;
    if (abstop >= top12(1024.0) && abstop - top12(0x1p-54) < 0x80000000u) {
        if (d2bits(x) == 0xfff0000000000000ull) return 0.0;
        if (abstop >= top12(bits2d(0x7ff0000000000000ull))) return 1.0 + x;  // inf, nan
    }
    return exp_core(x, 0.0);
}

// ---- pow: the published method of ARM's optimized-routines ------------------
// x^y = e^(y log x), log x in a double and a tail worth about 15 more bits:
// x = 2^k z, z in [0x1.69555p-1, 0x1.69555p0), log x = k ln2 + log c +
// log1p(z/c - 1) with c from a 128-entry table (libm_tables.cuh, generated
// from its definition) and a degree-8 polynomial; the product y log x in
// double-double; e^ by exp_core with the tail. The published algorithm
// (optimized-routines math/pow.c, Szabolcs Nagy 2018) that glibc runs from
// 2.28 on (sysdeps/ieee754/dbl-64/e_pow.c), with its constants and the fused
// multiply-adds of its x86-64 FMA build: glibc's bits on such a host
// (measured: no difference in 1.8e7 random arguments, x^(7/3), x^(1/3) and
// 10^y). Within 0.52 ulp. The step raises only positive bases (h^(7/3),
// tanh^(1/3), 10^y); a negative finite base returns NaN here.
#if defined(__CUDACC__)
static __device__ const double POW_LOG_TAB_DEV[384] = {DCLAW_POW_LOG_TABLE_DATA};
#endif
static const double POW_LOG_TAB_HOST[384] = {DCLAW_POW_LOG_TABLE_DATA};

DC_HD double pow_log_tab(unsigned k) {
#if defined(__CUDA_ARCH__)
    return __ldg(POW_LOG_TAB_DEV + k);
#else
    return POW_LOG_TAB_HOST[k];
#endif
}

constexpr double POW_LN2HI = 0x1.62e42fefa3800p-1, POW_LN2LO = 0x1.ef35793c76730p-45;
constexpr double POW_A0 = -0x1p-1, POW_A1 = 0x1.555555555556p-2 * -2, POW_A2 = -0x1.0000000000006p-2 * -2,
                 POW_A3 = 0x1.999999959554ep-3 * 4, POW_A4 = -0x1.555555529a47ap-3 * 4,
                 POW_A5 = 0x1.2495b9b4845e9p-3 * -8, POW_A6 = -0x1.0002b8b263fc3p-3 * -8;

// log of the positive normal number with bits ix, as hi + *tail
DC_HD double pow_log(uint64_t ix, double* tail) {
    const uint64_t tmp = ix - 0x3fe6955500000000ull;
    const unsigned i = (unsigned)((tmp >> 45) % 128u);
    const int k = (int)((int64_t)tmp >> 52);
    const double z = bits2d(ix - (tmp & (0xfffull << 52)));
    const double kd = (double)k;
    const double invc = pow_log_tab(3 * i), logc = pow_log_tab(3 * i + 1), logctail = pow_log_tab(3 * i + 2);
    const double r = fma(z, invc, -1.0);  // exact: 1/c has few bits
    const double t1 = fma(kd, POW_LN2HI, logc);
    const double t2 = t1 + r;
    const double lo1 = fma(kd, POW_LN2LO, logctail);
    const double lo2 = t1 - t2 + r;
    const double ar = POW_A0 * r;
    const double ar2 = r * ar;
    const double ar3 = r * ar2;
    const double hi = t2 + ar2;
    const double lo3 = fma(ar, r, -ar2);
    const double lo4 = t2 - hi + ar2;
    const double p = ar3 * fma(ar2, fma(ar2, fma(r, POW_A6, POW_A5), fma(r, POW_A4, POW_A3)), fma(r, POW_A2, POW_A1));
    const double lo = lo1 + lo2 + lo3 + lo4 + p;
    const double y = hi + lo;
    *tail = hi - y + lo;
    return y;
}

DC_HD bool zeroinfnan(uint64_t i) { return 2 * i - 1 >= 2 * 0x7ff0000000000000ull - 1; }

DC_HD double d_pow(double x, double y) {
    uint64_t ix = d2bits(x);
    const uint64_t iy = d2bits(y);
    const unsigned topx = top12(x), topy = top12(y);
    if (topx - 0x001u >= 0x7ffu - 0x001u || (topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {
        if (zeroinfnan(iy)) {
            if (2 * iy == 0) return 1.0;
            if (ix == 0x3ff0000000000000ull) return 1.0;
            if (2 * ix > 2 * 0x7ff0000000000000ull || 2 * iy > 2 * 0x7ff0000000000000ull) return x + y;
            if (2 * ix == 2 * 0x3ff0000000000000ull) return 1.0;
            if ((2 * ix < 2 * 0x3ff0000000000000ull) == !(iy >> 63)) return 0.0;
            return y * y;
        }
        if (zeroinfnan(ix)) {
            const double x2 = x * x;  // +0 or +inf (negative bases are not handled)
            return (iy >> 63) ? 1.0 / x2 : x2;
        }
        if (ix >> 63) return bits2d(0x7ff8000000000000ull);
        if ((topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {
            if (ix == 0x3ff0000000000000ull) return 1.0;
            if ((topy & 0x7ffu) < 0x3beu) return ix > 0x3ff0000000000000ull ? 1.0 + y : 1.0 - y;
            return (ix > 0x3ff0000000000000ull) == (topy < 0x800u) ? bits2d(0x7ff0000000000000ull) : 0.0;
        }
        if (topx == 0) {  // subnormal x: normalise, the exponent goes negative
            ix = d2bits(x * 0x1p52);
            ix &= 0x7fffffffffffffffull;
            ix -= 52ull << 52;
        }
    }
    if (ix >> 63) return bits2d(0x7ff8000000000000ull);
    double lo;
    const double hi = pow_log(ix, &lo);
    const double ehi = y * hi;
    const double elo = fma(y, lo, fma(y, hi, -ehi));
    return exp_core(ehi, elo);
}

// ---- expm1 and tanh: Sun's fdlibm method ------------------------------------
// expm1: x = k ln2 + r (ln2 in a 32-bit head and a tail), e^r - 1 by the
// rational form r - r^2/2 (... ) with the five scaled coefficients Q1..Q5
// and the correction c of the reduction, then 2^k (e^r - 1 + 1) - 1 by
// ranges of k. tanh x = 1 - 2/(expm1(2|x|) + 2) for |x| >= 1, -t/(t + 2)
// with t = expm1(-2|x|) below, +-1 beyond 22. These are fdlibm's s_expm1.c
// and s_tanh.c as glibc carries them (dbl-64/s_expm1.c with the polynomial
// in the split form R1 + h2 R2 + h4 R3), with the fused multiply-adds of
// glibc's x86-64 FMA build: glibc's bits on such a host (measured: no
// difference in 7e7 random arguments).
constexpr double EM1_LN2_HI = 6.93147180369123816490e-01, EM1_LN2_LO = 1.90821492927058770002e-10,
                 EM1_INVLN2 = 1.44269504088896338700e+00, EM1_O_THRESHOLD = 7.09782712893383973096e+02,
                 EM1_Q1 = -3.33333333333331316428e-02, EM1_Q2 = 1.58730158725481460165e-03,
                 EM1_Q3 = -7.93650757867487942473e-05, EM1_Q4 = 4.00821782732936239552e-06,
                 EM1_Q5 = -2.01099218183624371326e-07;

DC_HD uint32_t hi_word(double d) { return (uint32_t)(d2bits(d) >> 32); }
DC_HD double with_hi_word(double d, uint32_t h) {
    return bits2d(((uint64_t)h << 32) | (d2bits(d) & 0xffffffffull));
}

DC_HD double d_expm1(double x) {
    uint32_t hx = hi_word(x);
    const uint32_t xsb = hx & 0x80000000u;
    hx &= 0x7fffffffu;
    if (hx >= 0x4043687Au) {  // |x| >= 56 ln2
        if (hx >= 0x40862E42u) {
            if (hx >= 0x7ff00000u) {
                if (((hx & 0xfffffu) | (uint32_t)d2bits(x)) != 0) return x + x;
                return xsb == 0 ? x : -1.0;
            }
            if (x > EM1_O_THRESHOLD) return bits2d(0x7ff0000000000000ull);
        }
        if (xsb != 0) return -1.0;
    }
    double hi, lo, c = 0.0, t;
    int k;
    if (hx > 0x3fd62e42u) {  // |x| > ln2/2
        if (hx < 0x3FF0A2B2u) {  // and < 3 ln2/2
            if (xsb == 0) {
                hi = x - EM1_LN2_HI;
                lo = EM1_LN2_LO;
                k = 1;
            } else {
                hi = x + EM1_LN2_HI;
                lo = -EM1_LN2_LO;
                k = -1;
            }
        } else {
            k = (int)fma(EM1_INVLN2, x, xsb == 0 ? 0.5 : -0.5);
            t = (double)k;
            hi = fma(-t, EM1_LN2_HI, x);  // exact
            lo = t * EM1_LN2_LO;
        }
        x = hi - lo;
        c = (hi - x) - lo;
    } else if (hx < 0x3c900000u) {  // |x| < 2^-54
        return x;
    } else {
        k = 0;
    }
    const double hfx = 0.5 * x;
    const double hxs = x * hfx;
    const double R1 = fma(hxs, EM1_Q1, 1.0), h2 = hxs * hxs;
    const double R2 = fma(hxs, EM1_Q3, EM1_Q2), h4 = h2 * h2;
    const double R3 = fma(hxs, EM1_Q5, EM1_Q4);
    const double r1 = fma(h4, R3, fma(h2, R2, R1));
    t = fma(-r1, hfx, 3.0);
    double e = hxs * ((r1 - t) / fma(-x, t, 6.0));
    if (k == 0) return x - fma(x, e, -hxs);
    e = fma(x, e - c, -c);
    e -= hxs;
    if (k == -1) return fma(0.5, x - e, -0.5);
    if (k == 1) {
        if (x < -0.25) return -2.0 * (e - (x + 0.5));
        return fma(2.0, x - e, 1.0);
    }
    double y;
    if (k <= -2 || k > 56) {
        y = 1.0 - (e - x);
        if (k == 1024) y = y * 2.0 * 0x1p1023;
        else y = with_hi_word(y, hi_word(y) + ((uint32_t)k << 20));
        return y - 1.0;
    }
    if (k < 20) {
        t = with_hi_word(1.0, 0x3ff00000u - (0x200000u >> k));  // 1 - 2^-k
        y = t - (e - x);
    } else {
        t = with_hi_word(1.0, (uint32_t)(0x3ff - k) << 20);  // 2^-k
        y = x - (e + t);
        y += 1.0;
    }
    return with_hi_word(y, hi_word(y) + ((uint32_t)k << 20));
}

DC_HD double d_tanh(double x) {
    const uint64_t u = d2bits(x);
    const int32_t jx = (int32_t)(u >> 32), ix = jx & 0x7fffffff;
    const uint32_t lx = (uint32_t)u;
    if (ix >= 0x7ff00000) return jx >= 0 ? 1.0 / x + 1.0 : 1.0 / x - 1.0;
    double z;
    if (ix < 0x40360000) {  // |x| < 22
        if ((ix | (int32_t)lx) == 0) return x;
        if (ix < 0x3c800000) return x * (1.0 + x);  // |x| < 2^-55
        if (ix >= 0x3ff00000) {
            const double t = d_expm1(2.0 * fabs(x));
            z = 1.0 - 2.0 / (t + 2.0);
        } else {
            const double t = d_expm1(-2.0 * fabs(x));
            z = -t / (t + 2.0);
        }
    } else {
        z = 1.0;  // 1 - 1e-300 rounds to 1
    }
    return jx >= 0 ? z : -z;
}

// ---- atan and tan, correctly rounded --------------------------------------
// glibc's atan and tan (IBM's Accurate Mathematical Library, s_atan.c and
// s_tan.c) are correctly rounded except in about 0.2 % of arguments, where
// they return the other neighbour; their tables of accurate-table points
// cannot be rebuilt from a definition. These two are correctly rounded
// instead, which matches glibc everywhere else: both evaluate the function
// in double-double arithmetic (a value as an unevaluated sum hi + lo,
// Dekker 1971; the error-free sum and product of Knuth and of the fused
// multiply-add) to about 2^-83 relative, then round once.
//
//   atan  |x| > 1: atan x = pi/2 - atan(1/x). a in [0, 1]: c = k/64 nearest
//         to a, atan a = atan c + atan t with t = (a - c)/(1 + a c) (|t| <=
//         2^-7), atan c from a table (hi + lo), atan t by its Taylor series
//         to t^13.
//   tan   x = n pi/2 + r (pi/2 in three parts, Cody & Waite), |r| <= pi/4;
//         c = k/64 nearest to |r|, tan(c + t) = (tan c + tan t)/(1 - tan c
//         tan t), tan c from a table, tan t by its Taylor series to t^11;
//         odd n: -1/tan r, the same quotient inverted.

struct dd {
    double hi, lo;
};

// error-free sum (Knuth) and product (fused multiply-add)
DC_HD dd two_sum(double a, double b) {
    const double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
DC_HD dd fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
    const double s = a + b;
    return {s, b - (s - a)};
}
DC_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return {p, fma(a, b, -p)};
}
DC_HD dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    s = fast_two_sum(s.hi, s.lo + t.hi);
    return fast_two_sum(s.hi, s.lo + t.lo);
}
DC_HD dd dd_mul(dd a, dd b) {
    const dd p = two_prod(a.hi, b.hi);
    return fast_two_sum(p.hi, fma(a.hi, b.lo, fma(a.lo, b.hi, p.lo)));
}
// a / b in double-double (no overflow or underflow in 1/b.hi and a.hi/b.hi)
DC_HD dd dd_div(dd a, dd b) {
    const double rb = 1.0 / b.hi;
    const double q1 = a.hi * rb;
    // exact residual of the first quotient, then the rest of the dividend
    double r = fma(-q1, b.hi, a.hi);
    r = r + (a.lo - q1 * b.lo);
    return fast_two_sum(q1, r * rb);
}

constexpr double THIRD_HI = 0x1.5555555555555p-2, THIRD_LO = 0x1.5555555555555p-56;

#if defined(__CUDACC__)
static __device__ const double ATAN_TAB_DEV[130] = {DCLAW_ATAN_TABLE_DATA};
static __device__ const double TAN_TAB_DEV[104] = {DCLAW_TAN_TABLE_DATA};
#endif
static const double ATAN_TAB_HOST[130] = {DCLAW_ATAN_TABLE_DATA};
static const double TAN_TAB_HOST[104] = {DCLAW_TAN_TABLE_DATA};

DC_HD dd atan_tab(int k) {
#if defined(__CUDA_ARCH__)
    return {__ldg(ATAN_TAB_DEV + 2 * k), __ldg(ATAN_TAB_DEV + 2 * k + 1)};
#else
    return {ATAN_TAB_HOST[2 * k], ATAN_TAB_HOST[2 * k + 1]};
#endif
}
DC_HD dd tan_tab(int k) {
#if defined(__CUDA_ARCH__)
    return {__ldg(TAN_TAB_DEV + 2 * k), __ldg(TAN_TAB_DEV + 2 * k + 1)};
#else
    return {TAN_TAB_HOST[2 * k], TAN_TAB_HOST[2 * k + 1]};
#endif
}

// t * (1 + u) - t with u = -t^2/3 + t^4 P(t^2) (atan) or +t^2/3 + ... (tan):
// the series' tail beyond its first term, for |t| <= 2^-7, in double-double
DC_HD dd series_tail(dd t, double sgn3, double p) {
    dd s = two_prod(t.hi, t.hi);
    s.lo = fma(2.0 * t.hi, t.lo, s.lo);
    // s/3 in double-double
    dd m = two_prod(s.hi, THIRD_HI);
    m.lo = fma(s.hi, THIRD_LO, fma(s.lo, THIRD_HI, m.lo));
    // u = sgn3 s/3 + s^2 p
    const dd u = fast_two_sum(sgn3 * m.hi, fma(s.hi * s.hi, p, sgn3 * m.lo));
    const dd v = two_prod(t.hi, u.hi);
    return {v.hi, fma(t.hi, u.lo, fma(t.lo, u.hi, v.lo))};
}

DC_HD double d_atan(double x) {
    if (!(x == x)) return x + x;
    const double a = fabs(x);
    if (a < 0x1p-27) return x;                               // |atan x - x| < ulp/4
    if (a > 0x1p53) return copysign(PIO2_HI, x);             // within ulp/4 of pi/2
    const bool inv = a > 1.0;
    dd r;
    if (inv) {
        const double h = 1.0 / a;
        r = {h, fma(-h, a, 1.0) * h};
    } else {
        r = {a, 0.0};
    }
    const int k = (int)(r.hi * 64.0 + 0.5);
    const double c = (double)k * 0.015625;
    // a - c is exact (Sterbenz for k >= 1); 1 + a c in double-double
    const dd num = inv ? two_sum(r.hi - c, r.lo) : dd{r.hi - c, 0.0};
    const dd pc = two_prod(r.hi, c);
    dd den = fast_two_sum(1.0, pc.hi);
    den = fast_two_sum(den.hi, den.lo + fma(r.lo, c, pc.lo));
    const dd t = dd_div(num, den);
    // atan t = t - t^3/3 + t^5/5 - ... - t^11/11 + t^13/13
    const double s = t.hi * t.hi;
    double p = 0.07692307692307693;                          // 1/13
    p = p * s - 0.09090909090909091;                         // -1/11
    p = p * s + 0.1111111111111111;                          // 1/9
    p = p * s - 0.14285714285714285;                         // -1/7
    p = p * s + 0.2;                                         // 1/5
    const dd tail = series_tail(t, -1.0, p);
    dd at = dd_add(t, tail);
    at = dd_add(atan_tab(k), at);
    if (inv) at = dd_add(dd{PIO2_HI, PIO2_LO}, dd{-at.hi, -at.lo});
    return copysign(at.hi, x);
}

DC_HD double d_tan(double x) {
    if (!(x == x)) return x + x;
    const double ax = fabs(x);
    if (ax < 0x1p-27) return x;                              // |tan x - x| < ulp/4
    if (ax > 1.0e300) return bits2d(0x7ff8000000000000ull);
    const double kd = rint(x * TWO_OVER_PI);
    dd r;
    if (kd == 0.0) {
        r = {x, 0.0};
    } else {
        // x - kd pi/2: the first product is exact for |kd| < 2^20 (33-bit
        // head), the rest in double-double. Beyond that (|x| > 1.6e6; the
        // step's argument is phi + psi, |psi| < pi/2) the reduction is not
        // exact and the result not correctly rounded.
        const double r1 = x - kd * PIO2_1;
        const dd p2 = two_prod(kd, PIO2_2);
        r = two_sum(r1, -p2.hi);
        r = fast_two_sum(r.hi, r.lo - (p2.lo + kd * PIO2_3));
    }
    const double sg = r.hi < 0.0 ? -1.0 : 1.0;
    r = {sg * r.hi, sg * r.lo};
    int k = (int)(r.hi * 64.0 + 0.5);
    if (k > 51) k = 51;  // only reached by an inexact reduction (|x| > 1.6e6)
    const double c = (double)k * 0.015625;
    const dd t = two_sum(r.hi - c, r.lo);
    // tan t = t + t^3/3 + 2t^5/15 + 17t^7/315 + 62t^9/2835 + 1382t^11/155925
    const double s = t.hi * t.hi;
    double p = 0.008863235529902197;                         // 1382/155925
    p = p * s + 0.021869488536155203;                        // 62/2835
    p = p * s + 0.05396825396825397;                         // 17/315
    p = p * s + 0.13333333333333333;                         // 2/15
    const dd tail = series_tail(t, 1.0, p);
    const dd tt = dd_add(t, tail);
    const dd tc = tan_tab(k);
    const dd num = dd_add(tc, tt);
    const dd pr = dd_mul(tc, tt);
    const dd den = dd_add(dd{1.0, 0.0}, dd{-pr.hi, -pr.lo});
    const long long n = (long long)kd;
    double res;
    if (n & 1) {
        const dd q = dd_div(den, num);  // cot r = 1 / tan r
        res = -q.hi;
    } else {
        const dd q = dd_div(num, den);
        res = q.hi;
    }
    return sg * res;
}

// natural logarithm (src2method 2's substep bounds)
DC_HD double d_log(double x) {
    if (!(x == x)) return x + x;
    if (x < 0.0) return bits2d(0x7ff8000000000000ull);
    if (x == 0.0) return bits2d(0xfff0000000000000ull);
    if (x > 1.7976931348623157e308) return x;
    uint64_t b = d2bits(x);
    int e = (int)((b >> 52) & 0x7ff);
    int k = 0;
    if (e == 0) {  // subnormal: scale into the normal range
        b = d2bits(x * 18014398509481984.0);  // 2^54
        e = (int)((b >> 52) & 0x7ff);
        k = -54;
    }
    k += e - 1023;
    double f = bits2d((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
    if (f > 1.4142135623730951) {
        f = f * 0.5;
        k += 1;
    }
    double s = (f - 1.0) / (f + 1.0);
    double z = s * s;
    double q = 0.07407407407407407;  // 2/27, then 2/(2n+1) down to 2/3
    q = q * z + 0.08;
    q = q * z + 0.08695652173913043;
    q = q * z + 0.09523809523809523;
    q = q * z + 0.10526315789473684;
    q = q * z + 0.11764705882352941;
    q = q * z + 0.13333333333333333;
    q = q * z + 0.15384615384615385;
    q = q * z + 0.18181818181818182;
    q = q * z + 0.2222222222222222;
    q = q * z + 0.2857142857142857;
    q = q * z + 0.4;
    q = q * z + 0.6666666666666666;
    double lf = 2.0 * s + s * (z * q);
    double kd = (double)k;
    return kd * LN2_HI + (kd * LN2_LO + lf);
}

// h^(7/3) for h > 0 (Manning friction): the reference's h**(7.d0/3.d0),
// glibc's pow at the double nearest 7/3
DC_HD double d_pow_7_3(double h) { return d_pow(h, 7.0 / 3.0); }

}  // namespace em
}  // namespace dclaw

// elementary.cuh -- deterministic FP64 elementary functions for the D-Claw step.
//
// exp, expm1 (small arguments), tanh, atan, tan and h^(7/3), written from
// the mathematics with only IEEE +, -, *, /, rint and bit operations, so that
// a host build (g++ -ffp-contract=off) and the sm_100a build (--fmad=false)
// return the same bits for the same argument. The CUDA step uses these in
// place of the toolkit's libm; the oracle can use them too ("portable libm"
// mode), which makes GPU-vs-oracle parity exact to the bit. Accuracy is
// within about 2 ulp of the true value (see tests/test_elementary.py).
//
// Methods (published):
//   exp   Cody & Waite argument reduction x = k ln2 + r with ln2 split into a
//         32-bit head and a tail (Cody & Waite, "Software Manual for the
//         Elementary Functions", 1980), Taylor series of e^r on |r| <= ln2/2
//         with the leading 1 + r added last.
//   tanh  tanh x = (e^2x - 1) / (e^2x + 1) on |x|, with the Taylor series of
//         expm1 for 2|x| <= 1; exactly +-1 for |x| >= 22, x for |x| < 2^-28.
//   atan  atan(1/a) = pi/2 - atan(a) for a > 1, then the table reduction
//         atan a = atan c + atan((a - c)/(1 + a c)), c = k/8, with atan(k/8)
//         as head + tail doubles, and the Taylor series of atan on |t| <= 1/16.
//   tan   Cody & Waite reduction by pi/2 (three-part split), Taylor series of
//         sin and cos on |r| <= pi/4, tan = s/c or -c/s by quadrant.
//   h^(7/3) = h^2 * cbrt(h), cbrt by Newton iteration from an exponent guess.
//   log   x = 2^k f with f in [sqrt(1/2), sqrt(2)); log f = 2 atanh(s),
//         s = (f - 1)/(f + 1) (f - 1 exact), by the Taylor series of atanh
//         on |s| <= 0.1716; log x = k ln2_hi + (k ln2_lo + log f).
// The constants were produced with 80-digit decimal arithmetic.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

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

// y * 2^k for -1100 < k < 1100 (two steps outside the normal exponent range)
DC_HD double scale2(double y, int k) {
    if (k > 1023) {
        y = y * pow2i(1023);
        k -= 1023;
        if (k > 1023) k = 1023;
    } else if (k < -1021) {
        y = y * pow2i(-1021);
        k += 1021;
        if (k < -1021) k = -1021;
    }
    return y * pow2i(k);
}

constexpr double LN2_HI = 0.6931471803691238;        // 0x3fe62e42fee00000 (32-bit head)
constexpr double LN2_LO = 1.9082149292705877e-10;    // tail
constexpr double INV_LN2 = 1.4426950408889634;       // 0x3ff71547652b82fe
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
                 IF20 = 4.110317623312165e-19, IF21 = 1.9572941063391263e-20, IF22 = 8.896791392450574e-22;

DC_HD double d_exp(double x) {
    if (!(x == x)) return x + x;
    if (x > 709.782712893384) return bits2d(0x7ff0000000000000ull);
    if (x < -745.1332191019412) return 0.0;
    double kd = rint(x * INV_LN2);
    int k = (int)kd;
    double r = (x - kd * LN2_HI) - kd * LN2_LO;
    double q = IF13;
    q = q * r + IF12;
    q = q * r + IF11;
    q = q * r + IF10;
    q = q * r + IF9;
    q = q * r + IF8;
    q = q * r + IF7;
    q = q * r + IF6;
    q = q * r + IF5;
    q = q * r + IF4;
    q = q * r + IF3;
    q = q * r + IF2;
    double s = r + (r * r) * q;
    return scale2(1.0 + s, k);
}

// expm1 for |y| <= 1.2
DC_HD double d_expm1_small(double y) {
    double q = IF22;
    q = q * y + IF21;
    q = q * y + IF20;
    q = q * y + IF19;
    q = q * y + IF18;
    q = q * y + IF17;
    q = q * y + IF16;
    q = q * y + IF15;
    q = q * y + IF14;
    q = q * y + IF13;
    q = q * y + IF12;
    q = q * y + IF11;
    q = q * y + IF10;
    q = q * y + IF9;
    q = q * y + IF8;
    q = q * y + IF7;
    q = q * y + IF6;
    q = q * y + IF5;
    q = q * y + IF4;
    q = q * y + IF3;
    q = q * y + IF2;
    return y + (y * y) * q;
}

DC_HD double d_tanh(double x) {
    if (!(x == x)) return x + x;
    double a = fabs(x);
    double t;
    if (a >= 22.0) {
        t = 1.0;
    } else if (a < 3.725290298461914e-09) {  // 2^-28
        t = a;
    } else {
        double y = 2.0 * a;
        double e = y <= 1.0 ? d_expm1_small(y) : d_exp(y) - 1.0;
        t = e / (e + 2.0);
    }
    return copysign(t, x);
}

// atan(k/8), head + tail
DC_HD double atan_tab_hi(int k) {
    switch (k) {
        case 1: return 0.12435499454676144;
        case 2: return 0.24497866312686414;
        case 3: return 0.35877067027057225;
        case 4: return 0.4636476090008061;
        case 5: return 0.5585993153435624;
        case 6: return 0.6435011087932844;
        case 7: return 0.7188299996216245;
        case 8: return 0.7853981633974483;
        default: return 0.0;
    }
}
DC_HD double atan_tab_lo(int k) {
    switch (k) {
        case 1: return -3.1253241424539383e-18;
        case 2: return 1.0698755618734451e-17;
        case 3: return -2.4623815582638635e-17;
        case 4: return 2.2698777452961687e-17;
        case 5: return -5.4556305485916264e-18;
        case 6: return 1.5834785051444286e-17;
        case 7: return -2.1478388444456983e-17;
        case 8: return 3.061616997868383e-17;
        default: return 0.0;
    }
}

DC_HD double d_atan(double x) {
    if (!(x == x)) return x + x;
    double a = fabs(x);
    bool inv = a > 1.0;
    if (inv) a = 1.0 / a;
    int k = (int)(a * 8.0 + 0.5);
    double c = (double)k * 0.125;
    double t = (a - c) / (1.0 + a * c);
    double t2 = t * t;
    double p = 0.058823529411764705;     // 1/17
    p = p * t2 - 0.06666666666666667;    // -1/15
    p = p * t2 + 0.07692307692307693;    // 1/13
    p = p * t2 - 0.09090909090909091;    // -1/11
    p = p * t2 + 0.1111111111111111;     // 1/9
    p = p * t2 - 0.14285714285714285;    // -1/7
    p = p * t2 + 0.2;                    // 1/5
    p = p * t2 - 0.3333333333333333;     // -1/3
    double at = t + (t * t2) * p;
    double r = atan_tab_hi(k) + (atan_tab_lo(k) + at);
    if (inv) r = (PIO2_HI - r) + PIO2_LO;
    return copysign(r, x);
}

DC_HD double d_tan(double x) {
    if (!(x == x)) return x + x;
    if (x == 0.0) return x;
    if (fabs(x) > 1.0e300) return bits2d(0x7ff8000000000000ull);
    double kd = rint(x * TWO_OVER_PI);
    double r = ((x - kd * PIO2_1) - kd * PIO2_2) - kd * PIO2_3;
    long long k = (long long)kd;
    double r2 = r * r;
    double sp = -IF19;
    sp = sp * r2 + IF17;
    sp = sp * r2 - IF15;
    sp = sp * r2 + IF13;
    sp = sp * r2 - IF11;
    sp = sp * r2 + IF9;
    sp = sp * r2 - IF7;
    sp = sp * r2 + IF5;
    sp = sp * r2 - IF3;
    double s = r + (r * r2) * sp;
    double cp = IF20;
    cp = cp * r2 - IF18;
    cp = cp * r2 + IF16;
    cp = cp * r2 - IF14;
    cp = cp * r2 + IF12;
    cp = cp * r2 - IF10;
    cp = cp * r2 + IF8;
    cp = cp * r2 - IF6;
    cp = cp * r2 + IF4;
    double c = 1.0 + r2 * (-0.5 + r2 * cp);
    return (k & 1) ? -c / s : s / c;
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

// h^(7/3) for h > 0 (Manning friction)
DC_HD double d_pow_7_3(double h) {
    if (!(h > 0.0)) return h == 0.0 ? 0.0 : bits2d(0x7ff8000000000000ull);
    if (h > 1.0e300) return bits2d(0x7ff0000000000000ull);
    uint64_t b = d2bits(h);
    int ex = (int)((b >> 52) & 0x7ff) - 1023;
    if (ex == -1023) return (h * h) * 0.0;  // subnormal: (h^2) underflows anyway
    int e3 = ex >= 0 ? ex / 3 : -((-ex + 2) / 3);
    double y = pow2i(e3);
    for (int it = 0; it < 8; ++it) y = y - (y * y * y - h) / (3.0 * (y * y));
    return (h * h) * y;
}

}  // namespace em
}  // namespace dclaw

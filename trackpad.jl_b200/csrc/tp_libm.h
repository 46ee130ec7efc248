// tp_libm.h -- asin, sin, cos, tan, atan evaluated identically on host and device.
//
// The tracking maps call these functions per particle.  Their results must not
// depend on which processor evaluates them: the exact-bend map of the
// reference computes x' as a difference of O(1) terms, so a one-ulp change in
// a libm result of a previous element becomes a visible difference in x.  Both
// the CUDA kernels and the CPU oracle therefore use this one implementation,
// written with explicitly rounded IEEE operations only (no fused multiply-add,
// no contraction), so both produce the same bits.
//
// Method (exp, expm1, sinh and cosh too, at the end of this file): the published fdlibm algorithms (Sun Microsystems, as distributed in
// FreeBSD msun and used by Julia's Base.Math for Float64): rational minimax
// approximation for asin on |x| < 0.5 and the half-angle identity above it;
// minimax polynomial kernels for sin, cos and tan on [-pi/4, pi/4] with a
// three-stage Cody-Waite reduction by pi/2 for |x| < 2^20 * pi/2; reduction of
// atan to [0, 7/16] through four breakpoints with a minimax polynomial.  The
// constants are the published coefficients of those approximations.  Accuracy
// is checked against the C library (< 1 ulp) in the CPU tests.  Arguments
// beyond the Cody-Waite range (|x| >= 2^20 * pi/2, only reachable by a particle
// that is already lost) use the platform function.
// The coefficient tables and branch structure below follow fdlibm, whose
// routines carry this notice:
//
//   Copyright (C) 1993 by Sun Microsystems, Inc. All rights reserved.
//
//   Developed at SunPro, a Sun Microsystems, Inc. business.
//   Permission to use, copy, modify, and distribute this
//   software is freely granted, provided that this notice
//   is preserved.
//
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define TPM_FN __host__ __device__ __forceinline__
#else
#define TPM_FN inline
#endif

namespace tp {
namespace libm {

// Explicitly rounded operations: never contracted into an FMA on the device.
TPM_FN double add(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
TPM_FN double sub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
TPM_FN double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
TPM_FN double dv(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
TPM_FN double sq(double a) {
#if defined(__CUDA_ARCH__)
    return __dsqrt_rn(a);
#else
    return sqrt(a);
#endif
}

TPM_FN uint64_t bits(double x) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__double_as_longlong(x));
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}
TPM_FN double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(u));
#else
    double x;
    memcpy(&x, &u, 8);
    return x;
#endif
}
// High 32 bits without the sign (biased exponent and top of the mantissa).
TPM_FN uint32_t hix(double x) { return uint32_t(bits(x) >> 32) & 0x7fffffffu; }
TPM_FN double clear_low(double x) { return from_bits(bits(x) & 0xffffffff00000000ull); }
TPM_FN double fabs_(double x) { return from_bits(bits(x) & 0x7fffffffffffffffull); }
TPM_FN double neg(double x) { return from_bits(bits(x) ^ 0x8000000000000000ull); }

// ---------------------------------------------------------------------------
// asin
// ---------------------------------------------------------------------------
constexpr double PIO2_HI = 1.57079632679489655800e+00;
constexpr double PIO2_LO = 6.12323399573676603587e-17;
constexpr double PIO4_HI = 7.85398163397448278999e-01;
constexpr double PS0 = 1.66666666666666657415e-01, PS1 = -3.25565818622400915405e-01,
                 PS2 = 2.01212532134862925881e-01, PS3 = -4.00555345006794114027e-02,
                 PS4 = 7.91534994289814532176e-04, PS5 = 3.47933107596021167570e-05;
constexpr double QS1 = -2.40339491173441421878e+00, QS2 = 2.02094576023350569471e+00,
                 QS3 = -6.88283971605453293030e-01, QS4 = 7.70381505559019352791e-02;

TPM_FN double asin_p(double t) {
    return mul(t, add(PS0, mul(t, add(PS1, mul(t, add(PS2, mul(t, add(PS3, mul(t, add(PS4, mul(t, PS5)))))))))));
}
TPM_FN double asin_q(double t) {
    return add(1.0, mul(t, add(QS1, mul(t, add(QS2, mul(t, add(QS3, mul(t, QS4))))))));
}

TPM_FN double asin(double x) {
    const uint32_t ix = hix(x);
    const double ax = fabs_(x);
    if (ix >= 0x3ff00000u) {                 // |x| >= 1 or NaN
        if (ax == 1.0) return add(mul(x, PIO2_HI), mul(x, PIO2_LO));
        return sub(x, x) / sub(x, x);        // NaN
    }
    if (ix < 0x3fe00000u) {                  // |x| < 0.5
        if (ix < 0x3e500000u) return x;      // |x| < 2^-26: asin(x) rounds to x
        double t = mul(x, x);
        double w = dv(asin_p(t), asin_q(t));
        return add(x, mul(x, w));
    }
    double w = sub(1.0, ax);
    double t = mul(w, 0.5);
    double p = asin_p(t), q = asin_q(t);
    double s = sq(t);
    double r;
    if (ix >= 0x3fef3333u) {                 // |x| >= 0.975
        w = dv(p, q);
        r = sub(PIO2_HI, sub(mul(2.0, add(s, mul(s, w))), PIO2_LO));
    } else {
        double f = clear_low(s);
        double c = dv(sub(t, mul(f, f)), add(s, f));
        double rr = dv(p, q);
        double pp = sub(mul(mul(2.0, s), rr), sub(PIO2_LO, mul(2.0, c)));
        double qq = sub(PIO4_HI, mul(2.0, f));
        r = sub(PIO4_HI, sub(pp, qq));
    }
    return (bits(x) >> 63) ? neg(r) : r;
}

// ---------------------------------------------------------------------------
// sin / cos / tan kernels on [-pi/4, pi/4]; x + y is the reduced argument.
// ---------------------------------------------------------------------------
constexpr double S1 = -1.66666666666666324348e-01, S2 = 8.33333333332248946124e-03,
                 S3 = -1.98412698298579493134e-04, S4 = 2.75573137070700676789e-06,
                 S5 = -2.50507602534068634195e-08, S6 = 1.58969099521155010221e-10;
constexpr double C1 = 4.16666666666666019037e-02, C2 = -1.38888888888741095749e-03,
                 C3 = 2.48015872894767294178e-05, C4 = -2.75573143513906633035e-07,
                 C5 = 2.08757232129817482790e-09, C6 = -1.13596475577881948265e-11;

TPM_FN double k_sin(double x, double y, bool has_tail) {
    double z = mul(x, x);
    double v = mul(z, x);
    double r = add(S2, mul(z, add(S3, mul(z, add(S4, mul(z, add(S5, mul(z, S6))))))));
    if (!has_tail) return add(x, mul(v, add(S1, mul(z, r))));
    return sub(x, sub(sub(mul(z, sub(mul(0.5, y), mul(v, r))), y), mul(v, S1)));
}

TPM_FN double k_cos(double x, double y) {
    double z = mul(x, x);
    double r = mul(z, add(C1, mul(z, add(C2, mul(z, add(C3, mul(z, add(C4, mul(z, add(C5, mul(z, C6)))))))))));
    double hz = mul(0.5, z);
    double w = sub(1.0, hz);
    return add(w, add(sub(sub(1.0, w), hz), sub(mul(z, r), mul(x, y))));
}

constexpr double T0 = 3.33333333333334091986e-01, T1 = 1.33333333333201242699e-01,
                 T2 = 5.39682539762260521377e-02, T3 = 2.18694882948595424599e-02,
                 T4 = 8.86323982359930005737e-03, T5 = 3.59207910759131235356e-03,
                 T6 = 1.45620945432529025516e-03, T7 = 5.88041240820264096874e-04,
                 T8 = 2.46463134818469906812e-04, T9 = 7.81794442939557092300e-05,
                 T10 = 7.14072491382608190305e-05, T11 = -1.85586374855275456654e-05,
                 T12 = 2.59073051863633712884e-05;
constexpr double PIO4 = 7.85398163397448278999e-01, PIO4LO = 3.06161699786838301793e-17;

// tan(x + y) for iy = 1, -1/tan(x + y) for iy = -1.
TPM_FN double k_tan(double x, double y, int iy) {
    const uint32_t hx = uint32_t(bits(x) >> 32);
    const uint32_t ix = hx & 0x7fffffffu;
    const bool big = ix >= 0x3fe59428u;  // |x| >= 0.6744
    if (ix < 0x3e300000u) {              // |x| < 2^-28
        if (iy == 1) return x;
        // -1/x computed accurately from its high part
        double w = add(x, y);
        double z = clear_low(w);
        double v = sub(y, sub(z, x));
        double a = dv(-1.0, w);
        double t = clear_low(a);
        double s = add(1.0, mul(t, z));
        return add(t, mul(a, add(s, mul(t, v))));
    }
    if (big) {
        if (hx >> 31) { x = neg(x); y = neg(y); }
        double z = sub(PIO4, x);
        double w = sub(PIO4LO, y);
        x = add(z, w);
        y = 0.0;
    }
    double z = mul(x, x);
    double w = mul(z, z);
    double r = add(T1, mul(w, add(T3, mul(w, add(T5, mul(w, add(T7, mul(w, add(T9, mul(w, T11))))))))));
    double v = mul(z, add(T2, mul(w, add(T4, mul(w, add(T6, mul(w, add(T8, mul(w, add(T10, mul(w, T12)))))))))));
    double s = mul(z, x);
    r = add(y, mul(z, add(mul(s, add(r, v)), y)));
    r = add(r, mul(T0, s));
    w = add(x, r);
    if (big) {
        double vv = double(iy);
        double res = sub(vv, mul(2.0, sub(x, sub(dv(mul(w, w), add(w, vv)), r))));
        return (hx >> 31) ? neg(res) : res;
    }
    if (iy == 1) return w;
    double zz = clear_low(w);
    double vv = sub(r, sub(zz, x));
    double a = dv(-1.0, w);
    double t = clear_low(a);
    double ss = add(1.0, mul(t, zz));
    return add(t, mul(a, add(ss, mul(t, vv))));
}

// ---------------------------------------------------------------------------
// Reduction by pi/2 (three-stage Cody-Waite) for |x| < 2^20 * pi/2.
// Returns n mod 4 and x - n*pi/2 as y0 + y1.
// ---------------------------------------------------------------------------
constexpr double INVPIO2 = 6.36619772367581382433e-01;
constexpr double PIO2_1 = 1.57079632673412561417e+00, PIO2_1T = 6.07710050650619224932e-11;
constexpr double PIO2_2 = 6.07710050630396597660e-11, PIO2_2T = 2.02226624879595063154e-21;
constexpr double PIO2_3 = 2.02226624871116645580e-21, PIO2_3T = 8.47842766036889956997e-32;

TPM_FN int expo(double x) { return int((bits(x) >> 52) & 0x7ff); }

TPM_FN int rem_pio2(double x, double* y0, double* y1) {
    const double t = fabs_(x);
    const int n = int(add(mul(t, INVPIO2), 0.5));
    const double fn = double(n);
    double r = sub(t, mul(fn, PIO2_1));
    double w = mul(fn, PIO2_1T);
    const int j = expo(t);
    double a = sub(r, w);
    if (j - expo(a) > 16) {  // second stage: cancellation lost > 16 bits
        double tt = r;
        w = mul(fn, PIO2_2);
        r = sub(tt, w);
        w = sub(mul(fn, PIO2_2T), sub(sub(tt, r), w));
        a = sub(r, w);
        if (j - expo(a) > 49) {  // third stage
            tt = r;
            w = mul(fn, PIO2_3);
            r = sub(tt, w);
            w = sub(mul(fn, PIO2_3T), sub(sub(tt, r), w));
            a = sub(r, w);
        }
    }
    double b = sub(sub(r, a), w);
    if (bits(x) >> 63) {
        *y0 = neg(a);
        *y1 = neg(b);
        return (-n) & 3;
    }
    *y0 = a;
    *y1 = b;
    return n & 3;
}

constexpr uint32_t HI_PIO4 = 0x3fe921fbu;       // |x| <= pi/4 (high word)
constexpr uint32_t HI_MEDIUM = 0x413921fbu;     // 2^20 * pi/2

TPM_FN double sin(double x) {
    const uint32_t ix = hix(x);
    if (ix <= HI_PIO4) {
        if (ix < 0x3e500000u) return x;  // |x| < 2^-26
        return k_sin(x, 0.0, false);
    }
    if (ix >= 0x7ff00000u) return sub(x, x);  // inf or NaN
    if (ix >= HI_MEDIUM) return ::sin(x);
    double y0, y1;
    switch (rem_pio2(x, &y0, &y1)) {
        case 0: return k_sin(y0, y1, true);
        case 1: return k_cos(y0, y1);
        case 2: return neg(k_sin(y0, y1, true));
        default: return neg(k_cos(y0, y1));
    }
}

TPM_FN double cos(double x) {
    const uint32_t ix = hix(x);
    if (ix <= HI_PIO4) {
        if (ix < 0x3e46a09eu) return 1.0;  // |x| < 2^-27 * sqrt(2): cos(x) rounds to 1
        return k_cos(x, 0.0);
    }
    if (ix >= 0x7ff00000u) return sub(x, x);
    if (ix >= HI_MEDIUM) return ::cos(x);
    double y0, y1;
    switch (rem_pio2(x, &y0, &y1)) {
        case 0: return k_cos(y0, y1);
        case 1: return neg(k_sin(y0, y1, true));
        case 2: return neg(k_cos(y0, y1));
        default: return k_sin(y0, y1, true);
    }
}

TPM_FN double tan(double x) {
    const uint32_t ix = hix(x);
    if (ix <= HI_PIO4) return k_tan(x, 0.0, 1);
    if (ix >= 0x7ff00000u) return sub(x, x);
    if (ix >= HI_MEDIUM) return ::tan(x);
    double y0, y1;
    int n = rem_pio2(x, &y0, &y1);
    return k_tan(y0, y1, (n & 1) ? -1 : 1);
}

// ---------------------------------------------------------------------------
// atan
// ---------------------------------------------------------------------------
TPM_FN double atanhi(int i) {
    return i == 0 ? 4.63647609000806093515e-01
                  : i == 1 ? 7.85398163397448278999e-01 : i == 2 ? 9.82793723247329054082e-01 : 1.57079632679489655800e+00;
}
TPM_FN double atanlo(int i) {
    return i == 0 ? 2.26987774529616870924e-17
                  : i == 1 ? 3.06161699786838301793e-17 : i == 2 ? 1.39033110312309984516e-17 : 6.12323399573676603587e-17;
}
constexpr double AT0 = 3.33333333333329318027e-01, AT1 = -1.99999999998764832476e-01,
                 AT2 = 1.42857142725034663711e-01, AT3 = -1.11111104054623557880e-01,
                 AT4 = 9.09088713343650656196e-02, AT5 = -7.69187620504482999495e-02,
                 AT6 = 6.66107313738753120669e-02, AT7 = -5.83357013379057348645e-02,
                 AT8 = 4.97687799461593236017e-02, AT9 = -3.65315727442169155270e-02,
                 AT10 = 1.62858201153657823623e-02;

TPM_FN double atan(double x) {
    const uint32_t ix = hix(x);
    const bool negx = bits(x) >> 63;
    if (ix >= 0x44100000u) {  // |x| >= 2^66 (or NaN)
        if (x != x) return add(x, x);
        double r = add(atanhi(3), atanlo(3));
        return negx ? neg(r) : r;
    }
    int id;
    if (ix < 0x3fdc0000u) {  // |x| < 0.4375
        if (ix < 0x3e400000u) return x;  // |x| < 2^-27
        id = -1;
    } else {
        x = fabs_(x);
        if (ix < 0x3ff30000u) {        // |x| < 1.1875
            if (ix < 0x3fe60000u) {    // 7/16 <= |x| < 11/16
                id = 0;
                x = dv(sub(mul(2.0, x), 1.0), add(2.0, x));
            } else {                   // 11/16 <= |x| < 19/16
                id = 1;
                x = dv(sub(x, 1.0), add(x, 1.0));
            }
        } else {
            if (ix < 0x40038000u) {    // |x| < 2.4375
                id = 2;
                x = dv(sub(x, 1.5), add(1.0, mul(1.5, x)));
            } else {                   // 2.4375 <= |x| < 2^66
                id = 3;
                x = dv(-1.0, x);
            }
        }
    }
    double z = mul(x, x);
    double w = mul(z, z);
    double s1 = mul(z, add(AT0, mul(w, add(AT2, mul(w, add(AT4, mul(w, add(AT6, mul(w, add(AT8, mul(w, AT10)))))))))));
    double s2 = mul(w, add(AT1, mul(w, add(AT3, mul(w, add(AT5, mul(w, add(AT7, mul(w, AT9)))))))));
    if (id < 0) return sub(x, mul(x, add(s1, s2)));
    double r = sub(atanhi(id), sub(sub(mul(x, add(s1, s2)), atanlo(id)), x));
    return negx ? neg(r) : r;
}

// ---------------------------------------------------------------------------
// exp, expm1, sinh, cosh (fdlibm methods).  exp: x = k ln2 + r with ln2 split
// in a head and a tail, |r| <= ln2/2, and a minimax polynomial for the
// rational form r*(exp(r)+1)/(exp(r)-1); expm1: the same reduction with a
// correction term c for the rounding of r, and a minimax polynomial for the
// rational form of expm1 on the primary range; sinh and cosh from expm1 for
// small arguments and from exp otherwise.
// ---------------------------------------------------------------------------
constexpr double LN2_HI = 6.93147180369123816490e-01, LN2_LO = 1.90821492927058770002e-10;
constexpr double INV_LN2 = 1.44269504088896338700e+00;
constexpr double EXP_P1 = 1.66666666666666019037e-01, EXP_P2 = -2.77777777770155933842e-03,
                 EXP_P3 = 6.61375632143793436117e-05, EXP_P4 = -1.65339022054652515390e-06,
                 EXP_P5 = 4.13813679705723846039e-08;
constexpr double EXP_OVER = 7.09782712893383973096e+02, EXP_UNDER = -7.45133219101941108420e+02;
constexpr double EM1_Q1 = -3.33333333333331316428e-02, EM1_Q2 = 1.58730158725481460165e-03,
                 EM1_Q3 = -7.93650757867487942473e-05, EM1_Q4 = 4.00821782732936239552e-06,
                 EM1_Q5 = -2.01099218183624371326e-07;
constexpr double TWO_M1000 = 9.33263618503218878990e-302;  // 2^-1000

// y * 2^k by adding k to the biased exponent (y normal, result normal).
TPM_FN double add_expo(double y, int k) { return from_bits(bits(y) + (uint64_t(int64_t(k)) << 52)); }

TPM_FN double exp(double x) {
    const uint32_t hx = hix(x);
    const bool neg_x = (bits(x) >> 63) != 0;
    if (hx >= 0x40862E42u) {                       // |x| >= 709.78 or not finite
        if (hx >= 0x7ff00000u) {
            if (((bits(x) & 0x000fffffffffffffull) != 0)) return add(x, x);  // NaN
            return neg_x ? 0.0 : x;                 // exp(+-inf)
        }
        if (x > EXP_OVER) return from_bits(0x7ff0000000000000ull);  // overflow
        if (x < EXP_UNDER) return 0.0;
    }
    double hi = 0.0, lo = 0.0, r;
    int k = 0;
    if (hx > 0x3fd62e42u) {                        // |x| > ln2/2
        if (hx < 0x3FF0A2B2u) {                    // |x| < 1.5 ln2: k = +-1
            hi = neg_x ? add(x, LN2_HI) : sub(x, LN2_HI);
            lo = neg_x ? -LN2_LO : LN2_LO;
            k = neg_x ? -1 : 1;
        } else {
            k = int(add(mul(INV_LN2, x), neg_x ? -0.5 : 0.5));
            const double t = double(k);
            hi = sub(x, mul(t, LN2_HI));
            lo = mul(t, LN2_LO);
        }
        r = sub(hi, lo);
    } else if (hx < 0x3e300000u) {                 // |x| < 2^-28
        return add(1.0, x);
    } else {
        r = x;
    }
    const double t = mul(r, r);
    const double c =
        sub(r, mul(t, add(EXP_P1, mul(t, add(EXP_P2, mul(t, add(EXP_P3, mul(t, add(EXP_P4, mul(t, EXP_P5))))))))));
    if (k == 0) return sub(1.0, sub(dv(mul(r, c), sub(c, 2.0)), r));
    const double y = sub(1.0, sub(sub(lo, dv(mul(r, c), sub(2.0, c))), hi));
    if (k >= -1021) return add_expo(y, k);
    return mul(add_expo(y, k + 1000), TWO_M1000);
}

TPM_FN double expm1(double x) {
    const uint32_t hx = hix(x);
    const bool neg_x = (bits(x) >> 63) != 0;
    if (hx >= 0x4043687Au) {                       // |x| >= 56 ln2
        if (hx >= 0x40862E42u) {
            if (hx >= 0x7ff00000u) {
                if ((bits(x) & 0x000fffffffffffffull) != 0) return add(x, x);
                return neg_x ? -1.0 : x;
            }
            if (x > EXP_OVER) return from_bits(0x7ff0000000000000ull);  // overflow
        }
        if (neg_x) return -1.0;                     // x < -56 ln2: rounds to -1
    }
    double hi, lo, c = 0.0;
    int k = 0;
    if (hx > 0x3fd62e42u) {                        // |x| > ln2/2
        if (hx < 0x3FF0A2B2u) {
            if (!neg_x) { hi = sub(x, LN2_HI); lo = LN2_LO; k = 1; }
            else { hi = add(x, LN2_HI); lo = -LN2_LO; k = -1; }
        } else {
            k = int(add(mul(INV_LN2, x), neg_x ? -0.5 : 0.5));
            const double t = double(k);
            hi = sub(x, mul(t, LN2_HI));
            lo = mul(t, LN2_LO);
        }
        x = sub(hi, lo);
        c = sub(sub(hi, x), lo);
    } else if (hx < 0x3c900000u) {                 // |x| < 2^-54
        return x;
    }
    const double hfx = mul(0.5, x);
    const double hxs = mul(x, hfx);
    const double r1 = add(1.0, mul(hxs, add(EM1_Q1, mul(hxs, add(EM1_Q2, mul(hxs, add(EM1_Q3,
                                  mul(hxs, add(EM1_Q4, mul(hxs, EM1_Q5))))))))));
    const double t = sub(3.0, mul(r1, hfx));
    double e = mul(hxs, dv(sub(r1, t), sub(6.0, mul(x, t))));
    if (k == 0) return sub(x, sub(mul(x, e), hxs));
    e = sub(mul(x, sub(e, c)), c);
    e = sub(e, hxs);
    if (k == -1) return sub(mul(0.5, sub(x, e)), 0.5);
    if (k == 1) {
        if (x < -0.25) return mul(-2.0, sub(e, add(x, 0.5)));
        return add(1.0, mul(2.0, sub(x, e)));
    }
    if (k <= -2 || k > 56) {
        const double y = sub(1.0, sub(e, x));
        return sub(add_expo(y, k), 1.0);
    }
    if (k < 20) {
        const double t1 = from_bits(uint64_t(0x3ff00000u - (0x200000u >> k)) << 32);  // 1 - 2^-k
        const double y = sub(t1, sub(e, x));
        return add_expo(y, k);
    }
    const double t2 = from_bits(uint64_t(uint32_t(0x3ff - k) << 20) << 32);  // 2^-k
    double y = sub(x, add(e, t2));
    y = add(y, 1.0);
    return add_expo(y, k);
}

TPM_FN double sinh(double x) {
    const uint32_t ix = hix(x);
    if (ix >= 0x7ff00000u) return add(x, x);
    const double h = (bits(x) >> 63) ? -0.5 : 0.5;
    const double ax = fabs_(x);
    if (ix < 0x40360000u) {                        // |x| < 22
        if (ix < 0x3e300000u) return x;            // |x| < 2^-28
        const double t = expm1(ax);
        if (ix < 0x3ff00000u) return mul(h, sub(mul(2.0, t), dv(mul(t, t), add(t, 1.0))));
        return mul(h, add(t, dv(t, add(t, 1.0))));
    }
    if (ix < 0x40862E42u) return mul(h, exp(ax));  // |x| < log(DBL_MAX)
    const double w = exp(mul(0.5, ax));             // up to the overflow threshold
    return mul(mul(h, w), w);
}

TPM_FN double cosh(double x) {
    const uint32_t ix = hix(x);
    if (ix >= 0x7ff00000u) return mul(x, x);
    const double ax = fabs_(x);
    if (ix < 0x3fd62e43u) {                        // |x| < ln2/2
        const double t = expm1(ax);
        const double w = add(1.0, t);
        if (ix < 0x3c800000u) return w;
        return add(1.0, dv(mul(t, t), add(w, w)));
    }
    if (ix < 0x40360000u) {                        // |x| < 22
        const double t = exp(ax);
        return add(mul(0.5, t), dv(0.5, t));
    }
    if (ix < 0x40862E42u) return mul(0.5, exp(ax));
    const double w = exp(mul(0.5, ax));
    return mul(mul(0.5, w), w);
}

}  // namespace libm
}  // namespace tp

// tp_maps.cuh -- per-particle maps of the tracking path, FP64, in registers.
//
// Each function restates one pass! building block of TrackPad.jl
// (src/tracking.jl) with the reference's operation order, so that a build
// without FMA contraction reproduces the oracle bit for bit wherever the
// reference calls no transcendental function.  Element-constant subexpressions
// arrive precomputed in the record (tp_program.h); quantities that depend only
// on delta (which no thick-element sub-step changes) are cached per element:
//   A   = 1 + 2*delta*beti + delta^2   (drift6, tracking.jl:90)
//   bd  = beti + delta                 (drift6 z update; dp1 of the exact bend)
//   opd = 1 + delta
// Multiplication of those cached values reproduces the reference's per-call
// values exactly, because IEEE operations are deterministic.  sin, cos, tan,
// asin, atan, exp, sinh and cosh come from tp_libm.h (the same bits on host and
// device).
#pragma once
#include <math_constants.h>
#include <stdint.h>

#include "tp_libm.h"
#include "tp_program.h"

namespace tp {
namespace dev {

constexpr double C_LIGHT = 2.99792458e8;  // src/elements/rf.jl:28
constexpr double EPSD = 2.220446049250313e-16;

struct P6 {
    double x, px, y, py, z, d;
};

struct DCache {
    double A, bd, opd;
};

__device__ __forceinline__ void make_cache(const P6& s, double beti, DCache& c) {
    c.A = 1.0 + 2.0 * s.d * beti + s.d * s.d;
    c.bd = beti + s.d;
    c.opd = 1.0 + s.d;
}

__device__ __forceinline__ void set_nan(P6& s) {
    const double q = CUDART_NAN;
    s.x = q; s.px = q; s.y = q; s.py = q; s.z = q; s.d = q;
}

// drift6, exact Hamiltonian branch (src/tracking.jl:89-99).
__device__ __forceinline__ void drift_exact(P6& s, double L, double Lbeti, const DCache& c) {
    double pz2 = c.A - s.px * s.px - s.py * s.py;
    if (pz2 <= 0.0) {
        set_nan(s);
        return;
    }
    double NormL = L / sqrt(pz2);
    s.x = s.x + NormL * s.px;
    s.y = s.y + NormL * s.py;
    s.z = s.z + NormL * c.bd - Lbeti;
}

// drift6, linearised branch (src/tracking.jl:100-107).
__device__ __forceinline__ void drift_lin(P6& s, double L, const DCache& c) {
    double NormL = L / c.opd;
    s.x = s.x + NormL * s.px;
    s.y = s.y + NormL * s.py;
    s.z = s.z + NormL * (s.px * s.px + s.py * s.py) / (2.0 * c.opd);
}

template <bool EXACT>
__device__ __forceinline__ void drift(P6& s, double L, double Lbeti, const DCache& c) {
    if (EXACT) drift_exact(s, L, Lbeti, c);
    else drift_lin(s, L, c);
}

// Horner evaluation shared by strthinkick / bndthinkick (src/tracking.jl:252-259, 293-300).
template <int M>
__device__ __forceinline__ void horner(const double* pa, const double* pb, double x, double y, double& re, double& im) {
    re = pb[M];
    im = pa[M];
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        double t = re * x - im * y + pb[i];
        im = im * x + re * y + pa[i];
        re = t;
    }
}

// strthinkick (src/tracking.jl:284-305).
template <int M>
__device__ __forceinline__ void thin_kick(P6& s, const double* pa, const double* pb, double K) {
    double re, im;
    horner<M>(pa, pb, s.x, s.y, re, im);
    s.px = s.px - K * re;
    s.py = s.py + K * im;
}

// bndthinkick (src/tracking.jl:243-270); Kh = K*irho (the reference's L*irho).
template <int M>
__device__ __forceinline__ void bend_kick(P6& s, const double* pa, const double* pb, double K, double Kh, double irho,
                                          double beti) {
    double re, im;
    horner<M>(pa, pb, s.x, s.y, re, im);
    s.px = s.px - K * (re - (s.d - s.x * irho) * irho);
    s.py = s.py + K * im;
    s.z = s.z + Kh * s.x * beti;
}

// symplectic4_pass (src/tracking.jl:317-341) for one multipole record.
template <int M, bool EXACT>
__device__ __forceinline__ void multipole_body(P6& s, const double* w, int nsteps, double beti) {
    const double L1 = w[mp::L1], L2 = w[mp::L2], K1 = w[mp::K1], K2 = w[mp::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[mp::PA + i]; pb[i] = w[mp::PB + i]; }
    const double L1b = L1 * beti, L2b = L2 * beti;
    DCache c;
    make_cache(s, beti, c);
    // D(L1) K(K1) D(L2) K(K2) D(L2) K(K1) D(L1) per step, as one loop (code size).
    // The last D(L1) of a step and the first D(L1) of the next follow each
    // other with no kick between: px, py and delta are unchanged, so the second
    // reuses the first's NormL = L1/sqrt(pz2) (the same bits).  Where pz2 <= 0
    // drift6 returns NaN coordinates; here NormL is NaN, which makes x, y and z
    // NaN (px and py follow in the next kick): x is NaN either way, so
    // check_lost flags the particle at this element and its entrance
    // coordinates are kept, as with drift6's NaN vector.
    double NormL = 0.0;
#pragma unroll 1
    for (int k = 0; k < 4 * nsteps; ++k) {
        const int j = k & 3;
        const bool outer = (j == 0) || (j == 3);
        const double Lk = outer ? L1 : L2;
        if (EXACT) {
            if (j != 0 || k == 0) {
                double pz2 = c.A - s.px * s.px - s.py * s.py;
                NormL = pz2 <= 0.0 ? CUDART_NAN : Lk / sqrt(pz2);
            }
            s.x = s.x + NormL * s.px;
            s.y = s.y + NormL * s.py;
            s.z = s.z + NormL * c.bd - (outer ? L1b : L2b);
        } else {
            drift<EXACT>(s, Lk, outer ? L1b : L2b, c);
        }
        if (j != 3) thin_kick<M>(s, pa, pb, j == 1 ? K2 : K1);
    }
}

// Out of line for the orders lattices use rarely (0: a body with no field, 3:
// octupoles).  Quadrupoles (order 1) and sextupoles (order 2) run inline in the
// element loop: a call there saves and restores the caller's live registers
// through the stack at every magnet, and inlining the two made the DBA step
// 6 % faster, the 256-variant batch 5 % and the gradient's forward sweep 9 %.
template <int M, bool EXACT>
__device__ __noinline__ void multipole(P6& s, const double* w, int nsteps, double beti) {
    multipole_body<M, EXACT>(s, w, nsteps, beti);
}

// true when 0/opd is zero, i.e. `e - 0/(1+delta)` equals e exactly.
__device__ __forceinline__ bool zero_quotient_ok(double opd) { return opd != 0.0 && !isnan(opd); }

// edge_fringe_entrance / edge_fringe_exit (src/tracking.jl:160-221).
__device__ __forceinline__ void edge_fringe(P6& s, double irho, double fx, double e, double fc, int method,
                                            bool fc_zero, bool is_exit) {
    const double opd = 1.0 + s.d;
    double fy;
    if (method == 3) {
        double q = s.px / opd;
        fy = irho * libm::tan(is_exit ? (e - fc - q) : (e - fc + q));
    } else if (method == 2) {
        if (fc_zero) fy = zero_quotient_ok(opd) ? fx / opd : CUDART_NAN;
        else fy = irho * libm::tan(e - fc / opd) / opd;
    } else {
        if (fc_zero) fy = zero_quotient_ok(opd) ? fx : CUDART_NAN;
        else fy = irho * libm::tan(e - fc / opd);
    }
    s.px = s.px + s.x * fx;
    s.py = s.py - s.y * fy;
}

// pass!(::SBend) after the misalignment (src/tracking.jl:661-699).
template <int M, bool EXACT>
__device__ __noinline__ void sbend(P6& s, const double* w, const RecHdr& h, double beti) {
    const double irho = w[sb::IRHO];
    if (h.flags & RF_FRINGE_IN)
        edge_fringe(s, irho, w[sb::FX_IN], w[sb::E_IN], w[sb::FC_IN], h.method_in, h.flags & RF_FC_IN_ZERO, false);
    const double L1 = w[mp::L1], L2 = w[mp::L2], K1 = w[mp::K1], K2 = w[mp::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[mp::PA + i]; pb[i] = w[mp::PB + i]; }
    const double L1b = L1 * beti, L2b = L2 * beti;
    const double K1h = K1 * irho, K2h = K2 * irho;
    DCache c;
    make_cache(s, beti, c);
    for (int st = 0; st < h.nsteps; ++st) {
        drift<EXACT>(s, L1, L1b, c);
        bend_kick<M>(s, pa, pb, K1, K1h, irho, beti);
        drift<EXACT>(s, L2, L2b, c);
        bend_kick<M>(s, pa, pb, K2, K2h, irho, beti);
        drift<EXACT>(s, L2, L2b, c);
        bend_kick<M>(s, pa, pb, K1, K1h, irho, beti);
        drift<EXACT>(s, L1, L1b, c);
    }
    if (h.flags & RF_FRINGE_OUT)
        edge_fringe(s, irho, w[sb::FX_OUT], w[sb::E_OUT], w[sb::FC_OUT], h.method_out, h.flags & RF_FC_OUT_ZERO, true);
}

// ---------------------------------------------------------------------------
// Exact sector bend (src/tracking.jl:717-973).  dp1 = beti + delta = c.bd.
// ---------------------------------------------------------------------------
// One out-of-line copy of asin for the bend maps: a smaller hot loop (the
// kernels are limited by instruction fetch as much as by the FP64 pipe).
static __device__ __noinline__ double asin_ool(double x) { return libm::asin(x); }

// pxyz (:717-720) with dp1^2 precomputed.
__device__ __forceinline__ double pxyz(double dp1sq, double px, double py) {
    double val = dp1sq - px * px - py * py;
    return val > 0.0 ? sqrt(val) : 0.0;
}

// Julia clamp(v, -1, 1): NaN passes through (fmin/fmax would drop it).
__device__ __forceinline__ double jclamp(double v) { return v > 1.0 ? 1.0 : (v < -1.0 ? -1.0 : v); }

// yrot (:727-745) with c = cos(phi), s = sin(phi).
__device__ __forceinline__ void yrot(P6& s6, double c, double s, double dp1) {
    double pz = pxyz(dp1 * dp1, s6.px, s6.py);
    double p = c * pz - s * s6.px;
    double px_new = s * pz + c * s6.px;
    double x_new = s6.x * pz / p;
    double y_new = s6.y + s6.x * s6.py * s / p;
    double z_new = s6.z + dp1 * s6.x * s / p;
    s6.x = x_new; s6.px = px_new; s6.y = y_new; s6.z = z_new;
}

// bend_fringe, Forest 13.13 (:752-815).
static __device__ __noinline__ void bend_fringe(P6& r, double irho, double gK, double dp1) {
    const double b0 = irho;
    double pz = pxyz(dp1 * dp1, r.px, r.py);
    double px = r.px;
    double py = r.py;
    double xp = px / pz;
    double yp = py / pz;
    double term1 = 1.0 + xp * xp * (2.0 + yp * yp);
    double term2 = xp / (1.0 + yp * yp);
    double phi = -b0 * libm::tan(b0 * gK * term1 * pz - libm::atan(term2));
    double px2 = px * px;
    double py2 = py * py;
    double pz2 = pz * pz;
    double pz4 = pz2 * pz2;
    double py2z2 = (py2 + pz2);
    double arg_sec = (b0 * gK * (pz4 + px2 * (py2 + 2.0 * pz2))) / (pz2 * pz) - libm::atan(px * pz / (py2 + pz2));
    double sec = 1.0 / libm::cos(arg_sec);
    double powsec = sec * sec;
    double py4 = py2 * py2;
    double py6 = py4 * py2;
    double pz5 = pz4 * pz;
    double pz6 = pz4 * pz2;
    double py2z2_sq = py2z2 * py2z2;
    double denom = pz5 * (py4 + px2 * pz2 + 2.0 * py2 * pz2 + pz4);
    double dpx_num = -(b0 * (px2 * pz4 * (py2 - pz2) - pz6 * (py2 + pz2) +
                             b0 * gK * px *
                                 (pz2 * py2z2_sq * (2.0 * py2 + 3.0 * pz2) + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4) +
                                  px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 9.0 * py2 * pz4 + 5.0 * pz6)))) *
                     powsec;
    double dpx = dpx_num / denom;
    double dpy_num = -(b0 * py *
                       (px * pz4 * (py2 + pz2) +
                        b0 * gK *
                            (-(pz4 * py2z2_sq) + px2 * px2 * (3.0 * py2 * pz2 + 4.0 * pz4) +
                             px2 * (3.0 * py6 + 10.0 * py4 * pz2 + 11.0 * py2 * pz4 + 3.0 * pz6)))) *
                     powsec;
    double dpy = dpy_num / denom;
    double dd_num = (b0 * dp1 *
                     (px * pz4 * (py2 - pz2) +
                      b0 * gK *
                          (-(pz4 * py2z2_sq) + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4) +
                           px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 7.0 * py2 * pz4 + pz6)))) *
                    powsec;
    double dd = dd_num / denom;
    double yf = (2.0 * r.y) / (1.0 + sqrt(1.0 - 2.0 * dpy * r.y));
    double dxf = 0.5 * dpx * (yf * yf);
    double dct = 0.5 * dd * (yf * yf);
    double dpyf = phi * yf;
    r.x = r.x + dxf;
    r.y = yf;
    r.py = r.py - dpyf;
    r.z = r.z - dct;
}

// bend_edge, Forest 12.41 (:822-851); c, s, s2 = cos, sin, sin(2 theta); thh = theta/rhoinv.
static __device__ __forceinline__ void bend_edge_body(P6& r, double rhoinv, double c, double s, double s2,
                                                      double theta, double thh, double dp1) {
    const double dp1sq = dp1 * dp1;
    double pz = pxyz(dp1sq, r.px, r.py);
    double d2 = pxyz(dp1sq, 0.0, r.py);
    double px_new = r.px * c + (pz - rhoinv * r.x) * s;
    double val1 = jclamp(r.px / d2);
    double val2 = jclamp(px_new / d2);
    double dasin = asin_ool(val1) - asin_ool(val2);
    double num = r.x * (r.px * s2 + s * s * (2.0 * pz - rhoinv * r.x));
    double den = pxyz(dp1sq, px_new, r.py) + pz * c - r.px * s;
    double x_new = r.x * c + num / den;
    double y_new = r.y + r.py * (thh + dasin / rhoinv);
    double z_new = r.z + dp1 / rhoinv * (theta + dasin);
    r.x = x_new; r.px = px_new; r.y = y_new; r.z = z_new;
}

// Out of line in the forward sweeps: inline there (with bend_fringe) it made the
// gradient's forward sweep 14 % slower.  The reverse sweep, whose kernel has
// twice the registers, inlines bend_edge_body for its inverse (3 % faster).
static __device__ __noinline__ void bend_edge(P6& r, double rhoinv, double c, double s, double s2, double theta,
                                       double thh, double dp1) {
    bend_edge_body(r, rhoinv, c, s, s2, theta, thh, dp1);
}

// exact_bend_body, Forest 12.18 (:858-894): one call, no state carried.
__device__ __forceinline__ void body_one(P6& r, double irho, double L, double Lbeti, double cs, double sn, double dp1,
                                         bool straight) {
    const double dp1sq = dp1 * dp1;
    double pz = pxyz(dp1sq, r.px, r.py);
    if (straight) {
        double NormL = L / pz;
        r.x = r.x + r.px * NormL;
        r.y = r.y + r.py * NormL;
        r.z = r.z + NormL * dp1 - Lbeti;
        return;
    }
    double pzmx = pz - (1.0 + r.x * irho);
    double px_new = r.px * cs + pzmx * sn;
    double d2 = pxyz(dp1sq, 0.0, r.py);
    double val1 = jclamp(r.px / d2);
    double val2 = jclamp(px_new / d2);
    double dasin = L + (libm::asin(val1) - libm::asin(val2)) / irho;
    double x_new = (pxyz(dp1sq, px_new, r.py) - pzmx * cs + r.px * sn - 1.0) / irho;
    r.y = r.y + r.py * dasin;
    r.z = r.z + dp1 * dasin - Lbeti;
    r.x = x_new;
    r.px = px_new;
}

// a / b from y = RN(1/b) by Markstein's sequence: q = RN(a*y), r = a - b*q
// (exact with an FMA), RN(q + r*y) is the correctly rounded quotient a/b
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990; Theorem 8.10 of "IA-64 and
// Elementary Functions").  The identity needs b, y and the quotient in the
// normal range; outside it (and for a = 0, inf or NaN) the IEEE division runs.
// Finite normal number (device code must not call std::isnormal).
__device__ __forceinline__ bool is_normal(double v) {
    const double av = fabs(v);
    return av >= 2.2250738585072014e-308 && av <= 1.7976931348623157e308;
}

// The IEEE division of div_rcp's rare out-of-range case, out of line: the
// kernels are limited by instruction fetch, and three inlined divisions in the
// exact-bend body loop cost more there than the call on the rare path.
static __device__ __noinline__ double div_ool(double a, double b) { return a / b; }

__device__ __forceinline__ double div_rcp(double a, double b, double y) {
    double q = __dmul_rn(a, y);
    double r = fma(-q, b, a);
    double q1 = fma(r, y, q);
    double aq = fabs(q);
    if (!(aq > 1e-280 && aq < 1e280)) q1 = div_ool(a, b);
    return q1;
}

// Consecutive exact_bend_body calls with no kick in between.  py and delta are
// unchanged by the body, so d2 = pxyz(dp1, 0, py) is the same for every call,
// the pz of a call is the pxyz(dp1, px_new, py) of the previous one, and its
// asin(clamp(px/d2)) is the previous asin(clamp(px_new/d2)).  Carrying them
// leaves every operation of every call as the reference performs it.
struct BodyCarry {
    double dp1sq, pysq, d2, d2inv, pz, as1;
    bool rcp_d2;
};

__device__ __forceinline__ void body_carry_init(const P6& r, double dp1, BodyCarry& b) {
    b.dp1sq = dp1 * dp1;
    b.pysq = r.py * r.py;
    double v0 = b.dp1sq - 0.0 * 0.0 - b.pysq;
    b.d2 = v0 > 0.0 ? sqrt(v0) : 0.0;
    b.d2inv = 1.0 / b.d2;
    b.rcp_d2 = is_normal(b.d2) && is_normal(b.d2inv);
    double v = b.dp1sq - r.px * r.px - b.pysq;
    b.pz = v > 0.0 ? sqrt(v) : 0.0;
    b.as1 = asin_ool(jclamp(r.px / b.d2));
}

// One exact_bend_body call (:869-893) with the carried values.  The three
// quotients have divisors that are fixed for the whole body (d2, irho), so
// with normal divisors they use the reciprocal sequence (same bits as the
// division).
template <bool RCP_IRHO>
__device__ __forceinline__ void body_carry_step(P6& r, BodyCarry& b, double irho, double irho_inv, double L,
                                                double Lbeti, double cs, double sn, double dp1) {
    double pzmx = b.pz - (1.0 + r.x * irho);
    double px_new = r.px * cs + pzmx * sn;
    double q2 = b.rcp_d2 ? div_rcp(px_new, b.d2, b.d2inv) : px_new / b.d2;
    double as2 = asin_ool(jclamp(q2));
    double das = b.as1 - as2;
    double dasin = L + (RCP_IRHO ? div_rcp(das, irho, irho_inv) : das / irho);
    double v = b.dp1sq - px_new * px_new - b.pysq;
    double pz_new = v > 0.0 ? sqrt(v) : 0.0;
    double num = pz_new - pzmx * cs + r.px * sn - 1.0;
    double x_new = RCP_IRHO ? div_rcp(num, irho, irho_inv) : num / irho;
    r.y = r.y + r.py * dasin;
    r.z = r.z + dp1 * dasin - Lbeti;
    r.x = x_new;
    r.px = px_new;
    b.pz = pz_new;
    b.as1 = as2;
}

template <bool RCP_IRHO>
__device__ __forceinline__ void body_carry_run(P6& r, const double* w, int nsteps, double irho, double dp1,
                                               double beti) {
    const double L1 = w[eb::L1], L2 = w[eb::L2];
    const double L1b = L1 * beti, L2b = L2 * beti;
    const double cs1 = w[eb::CS1], sn1 = w[eb::SN1], cs2 = w[eb::CS2], sn2 = w[eb::SN2];
    const double irho_inv = w[eb::IRHO_INV];
    BodyCarry b;
    body_carry_init(r, dp1, b);
    // Sub-steps L1, L2, L2, L1 of every Yoshida step, as one loop (code size).
#pragma unroll 1
    for (int k = 0; k < 4 * nsteps; ++k) {
        const bool outer = ((k & 3) == 0) || ((k & 3) == 3);
        body_carry_step<RCP_IRHO>(r, b, irho, irho_inv, outer ? L1 : L2, outer ? L1b : L2b, outer ? cs1 : cs2,
                                  outer ? sn1 : sn2, dp1);
    }
}

// Body of pass!(::ExactSBend) between the entrance and exit wedges (:921-953).
template <int M>
__device__ __noinline__ void exact_body(P6& r, const double* w, const RecHdr& h, double beti) {
    const double irho = w[eb::IRHO];
    const double dp1 = beti + r.d;
    const bool straight = h.flags & RF_STRAIGHT;
    if (h.flags & RF_BODY_ONE) {
        body_one(r, irho, w[eb::L1], w[eb::L1] * beti, w[eb::CS1], w[eb::SN1], dp1, straight);
        return;
    }
    const double L1 = w[eb::L1], L2 = w[eb::L2];
    const double L1b = L1 * beti, L2b = L2 * beti;
    const double cs1 = w[eb::CS1], sn1 = w[eb::SN1], cs2 = w[eb::CS2], sn2 = w[eb::SN2];
    if ((h.flags & RF_NOKICK) && !straight) {
        if (h.nsteps <= 0) return;
        if (h.flags & RF_RCP_IRHO) body_carry_run<true>(r, w, h.nsteps, irho, dp1, beti);
        else body_carry_run<false>(r, w, h.nsteps, irho, dp1, beti);
        return;
    }
    const double K1 = w[eb::K1], K2 = w[eb::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[eb::PA + i]; pb[i] = w[eb::PB + i]; }
    for (int st = 0; st < h.nsteps; ++st) {
        body_one(r, irho, L1, L1b, cs1, sn1, dp1, straight);
        thin_kick<M>(r, pa, pb, K1);
        body_one(r, irho, L2, L2b, cs2, sn2, dp1, straight);
        thin_kick<M>(r, pa, pb, K2);
        body_one(r, irho, L2, L2b, cs2, sn2, dp1, straight);
        thin_kick<M>(r, pa, pb, K1);
        body_one(r, irho, L1, L1b, cs1, sn1, dp1, straight);
    }
}

// pass!(::ExactSBend) after the misalignment (src/tracking.jl:909-965).
__device__ __forceinline__ void exact_sbend(P6& r, const double* w, const RecHdr& h, double beti) {
    const double irho = w[eb::IRHO];
    const double gk = w[eb::GK];
    const double dp1 = beti + r.d;  // delta is constant through the element
    if (h.flags & RF_YROT_IN) yrot(r, w[eb::YC_IN], w[eb::YS_IN], dp1);
    if (h.flags & RF_FRINGE_IN) bend_fringe(r, irho, gk, dp1);
    if (h.flags & RF_EDGE)
        bend_edge(r, irho, w[eb::EC_IN], w[eb::ES_IN], w[eb::ES2_IN], w[eb::ETH_IN], w[eb::ETHH_IN], dp1);
    switch (h.order) {
        case 0: exact_body<0>(r, w, h, beti); break;
        case 1: exact_body<1>(r, w, h, beti); break;
        case 2: exact_body<2>(r, w, h, beti); break;
        default: exact_body<3>(r, w, h, beti); break;
    }
    if (h.flags & RF_EDGE)
        bend_edge(r, irho, w[eb::EC_OUT], w[eb::ES_OUT], w[eb::ES2_OUT], w[eb::ETH_OUT], w[eb::ETHH_OUT], dp1);
    if (h.flags & RF_FRINGE_OUT) bend_fringe(r, -irho, gk, dp1);
    if (h.flags & RF_YROT_OUT) yrot(r, w[eb::YC_OUT], w[eb::YS_OUT], dp1);
}

// pass!(::RFCavity) (src/tracking.jl:502-518); beta2 = beta*beta with beta = 1/beti.
template <bool EXACT>
__device__ __forceinline__ void rf_cavity(P6& s, const double* w, const RecHdr& h, double beti, double beta2) {
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        drift<EXACT>(s, w[rf::LH], w[rf::LH] * beti, c);
    }
    if (h.flags & RF_ENERGY) {
        double phase = w[rf::W] * ((s.z - w[rf::LAG]) / C_LIGHT) - w[rf::PHILAG];
        s.d = s.d - w[rf::NV] * libm::sin(phase) / beta2;
    }
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        drift<EXACT>(s, w[rf::LH], w[rf::LH] * beti, c);
    }
}

// pass!(::Solenoid) (src/tracking.jl:537-562).
template <bool EXACT>
__device__ __noinline__ void solenoid(P6& s, const double* w, double beti) {
    const double ks = w[sol::KS];
    const double L = w[sol::L];
    if (ks == 0.0) {
        DCache c;
        make_cache(s, beti, c);
        drift<EXACT>(s, L, L * beti, c);
        return;
    }
    double p_norm = 1.0 / (1.0 + s.d);
    double x = s.x, xpr = s.px * p_norm, y = s.y, ypr = s.py * p_norm;
    double H = ks * p_norm / 2.0;
    double S = libm::sin(L * H);
    double C = libm::cos(L * H);
    double x_new = x * C * C + xpr * C * S / H + y * C * S + ypr * S * S / H;
    double px_new = (-x * H * C * S + xpr * C * C - y * H * S * S + ypr * C * S) / p_norm;
    double y_new = -x * C * S - xpr * S * S / H + y * C * C + ypr * C * S / H;
    double py_new = (x * H * S * S - xpr * C * S - y * C * S * H + ypr * C * C) / p_norm;
    double z_new = s.z + L * (H * H * (x * x + y * y) + 2.0 * H * (xpr * y - ypr * x) + xpr * xpr + ypr * ypr) / 2.0;
    s.x = x_new; s.px = px_new; s.y = y_new; s.py = py_new; s.z = z_new;
}

// pass!(::Corrector) (src/tracking.jl:587-599).
__device__ __forceinline__ void corrector(P6& s, const double* w) {
    const double xk = w[cor::XK], yk = w[cor::YK];
    double p_norm = 1.0 / (1.0 + s.d);
    double NormL = w[cor::L] * p_norm;
    double z_new = s.z + NormL * p_norm *
                             (xk * xk / 3.0 + yk * yk / 3.0 + s.px * s.px + s.py * s.py + s.px * xk + s.py * yk) / 2.0;
    double x_new = s.x + NormL * (s.px + xk / 2.0);
    double px_new = s.px + xk;
    double y_new = s.y + NormL * (s.py + yk / 2.0);
    double py_new = s.py + yk;
    s.x = x_new; s.px = px_new; s.y = y_new; s.py = py_new; s.z = z_new;
}

// pass!(::Translation) (src/tracking.jl:1182-1192).
__device__ __forceinline__ void translation(P6& s, const double* w, double beti) {
    double pz2 = 1.0 + 2.0 * s.d * beti + s.d * s.d - s.px * s.px - s.py * s.py;
    if (pz2 <= 0.0) { set_nan(s); return; }
    double pz = sqrt(pz2);
    double x_new = s.x - (w[trn::DX] + w[trn::DS] * s.px / pz);
    double y_new = s.y - (w[trn::DY] + w[trn::DS] * s.py / pz);
    double z_new = s.z + w[trn::DS] * (beti + s.d) / pz;
    s.x = x_new; s.y = y_new; s.z = z_new;
}

// pass!(::YRotation) (src/tracking.jl:1194-1218).
__device__ __forceinline__ void yrotation(P6& s, const double* w, double beti) {
    const double ca = w[yr::CA], sa = w[yr::SA], ta = w[yr::TA];
    double pz2 = 1.0 + 2.0 * s.d * beti + s.d * s.d - s.px * s.px - s.py * s.py;
    if (pz2 <= 0.0) { set_nan(s); return; }
    double pz = sqrt(pz2);
    double ptt = 1.0 - ta * s.px / pz;
    if (fabs(ptt) < 1.4901161193847656e-08) { set_nan(s); return; }
    double x_new = s.x / (ca * ptt);
    double px_new = ca * s.px + sa * pz;
    double y_new = s.y + ta * s.x * s.py / (pz * ptt);
    double z_new = s.z + ta * s.x * (beti + s.d) / (pz * ptt);
    s.x = x_new; s.px = px_new; s.y = y_new; s.z = z_new;
}

// pass!(::CrabCavity) (src/tracking.jl:1531-1547).
template <bool EXACT>
__device__ __forceinline__ void crab_cavity(P6& s, const double* w, const RecHdr& h, double beti) {
    const double volt = w[crab::VOLT], E = w[crab::E], k = w[crab::K];
    double ang = k * s.z + w[crab::PHI];
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        drift<EXACT>(s, w[crab::LH], w[crab::LH] * beti, c);
    }
    double px_new = s.px + (volt / E) * libm::sin(ang * beti);
    double delta_new = s.d - (k * volt / E * beti) * s.x * libm::cos(ang * beti);
    s.px = px_new;
    s.d = delta_new;
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        drift<EXACT>(s, w[crab::LH], w[crab::LH] * beti, c);
    }
}

// pass!(::AccelCavity) (src/tracking.jl:1549-1559).
__device__ __forceinline__ void accel_cavity(P6& s, const double* w, double beta2) {
    if (beta2 <= EPSD) return;
    double sv = libm::sin(w[acc::K] * s.z + w[acc::PHIS]) - w[acc::SINPHIS];
    s.d = s.d + (w[acc::VOLT] / (beta2 * w[acc::E])) * sv;
}

// pass!(::LongitudinalRFMap) (src/tracking.jl:1575-1585).
__device__ __forceinline__ void long_rf_map(P6& s, const double* w, double beta) {
    double eta = w[lrf::ALPHAC] - (1.0 - beta * beta);
    s.z = s.z - (6.283185307179586 * w[lrf::H] * eta / w[lrf::K]) * s.d;
}

// pass!(::StrongThinGaussianBeam) (src/tracking.jl:1610-1619).
__device__ __forceinline__ void strong_thin_gauss(P6& s, const double* w) {
    double dx = s.x - w[stg::XO];
    double dy = s.y - w[stg::YO];
    double g = w[stg::AMP] * libm::exp(-0.5 * (dx * dx / w[stg::SX2] + dy * dy / w[stg::SY2]));
    s.px = s.px - g * dx / w[stg::SX2];
    s.py = s.py - g * dy / w[stg::SY2];
}

// LBend (src/tracking.jl:1076-1170): method-1 edges around the linear
// combined-function body; G1, G2 depend on delta through p_norm.
static __device__ __noinline__ void lbend(P6& s, const double* w, const RecHdr& h) {
    const double kx = w[lb::KX], L = w[lb::L];
    edge_fringe(s, w[lb::IRHO], w[lb::FX_IN], w[lb::E_IN], w[lb::FC_IN], 1, h.flags & RF_FC_IN_ZERO, false);
    const double p_norm = 1.0 / (1.0 + s.d);
    const double G1 = w[lb::G1C] * p_norm;
    const double G2 = w[lb::NGRD] * p_norm;
    const double tol = 1.4901161193847656e-08;  // sqrt(eps(Float64))
    double MHD = 1.0, M12 = L, M21 = 0.0, MVD = 1.0, M34 = L, M43 = 0.0;
    double arg1 = 0.0, sqrtG1 = 0.0;
    const bool big1 = fabs(G1) >= tol;
    if (big1) {
        if (G1 > 0.0) {
            sqrtG1 = sqrt(G1);
            arg1 = L * sqrtG1;
            MHD = libm::cos(arg1); M12 = libm::sin(arg1) / sqrtG1; M21 = -libm::sin(arg1) * sqrtG1;
        } else {
            sqrtG1 = sqrt(-G1);
            arg1 = L * sqrtG1;
            MHD = libm::cosh(arg1); M12 = libm::sinh(arg1) / sqrtG1; M21 = libm::sinh(arg1) * sqrtG1;
        }
    }
    if (fabs(G2) >= tol) {
        if (G2 > 0.0) {
            const double sq = sqrt(G2), arg2 = L * sq;
            MVD = libm::cos(arg2); M34 = libm::sin(arg2) / sq; M43 = -libm::sin(arg2) * sq;
        } else {
            const double sq = sqrt(-G2), arg2 = L * sq;
            MVD = libm::cosh(arg2); M34 = libm::sinh(arg2) / sq; M43 = libm::sinh(arg2) * sq;
        }
    }
    const double x = s.x, xpr = s.px * p_norm, y = s.y, ypr = s.py * p_norm;
    const double dterm = s.d * p_norm - w[lb::BYERR];
    double x_new = MHD * x + M12 * xpr;
    double px_new = (M21 * x + MHD * xpr) / p_norm;
    if (fabs(G1) < tol) {
        x_new = x_new + dterm * L * L * kx / 2.0;
        px_new = px_new + dterm * L * kx / p_norm;
    } else if (G1 > 0.0) {
        x_new = x_new + dterm * (1.0 - libm::cos(arg1)) * kx / G1;
        px_new = px_new + dterm * libm::sin(arg1) * kx / (sqrtG1 * p_norm);
    } else {
        x_new = x_new + dterm * (1.0 - libm::cosh(arg1)) * kx / G1;
        px_new = px_new + dterm * libm::sinh(arg1) * kx / (sqrtG1 * p_norm);
    }
    const double y_new = MVD * y + M34 * ypr;
    const double py_new = (M43 * y + MVD * ypr) / p_norm;
    double z_new = s.z + xpr * xpr * (L + MHD * M12) / 4.0;
    if (big1) {
        z_new = z_new + (L - MHD * M12) * (x * x * G1 + dterm * dterm * kx * kx / G1 - 2.0 * x * kx * dterm) / 4.0;
        z_new = z_new + M12 * M21 * (x * xpr - xpr * dterm * kx / G1) / 2.0;
        z_new = z_new + (kx * x * M12 + xpr * (1.0 - MHD) * kx / G1 + dterm * (L - M12) * kx * kx / G1);
    }
    z_new = z_new + ((L - MVD * M34) * y * y * G2 + ypr * ypr * (L + MVD * M34)) / 4.0;
    z_new = z_new + M34 * M43 * y * ypr / 2.0;
    s.x = x_new; s.px = px_new; s.y = y_new; s.py = py_new; s.z = z_new;
    edge_fringe(s, w[lb::IRHO], w[lb::FX_OUT], w[lb::E_OUT], w[lb::FC_OUT], 1, h.flags & RF_FC_OUT_ZERO, true);
}

// LorentzBoost / InvLorentzBoost (src/tracking.jl:1587-1606).
__device__ __forceinline__ void lorentz_boost(P6& s, const double* w) {
    const double ic = w[lor::A], ta = w[lor::B];
    double x_new = s.x + ta * s.z;
    double d_new = s.d - ta * s.px;
    s.x = x_new; s.px = s.px * ic; s.py = s.py * ic; s.z = s.z * ic; s.d = d_new;
}

__device__ __forceinline__ void inv_lorentz_boost(P6& s, const double* w) {
    const double ca = w[lor::A], sa = w[lor::B];
    double x_new = s.x - sa * s.z;
    double d_new = s.d + sa * s.px;
    s.x = x_new; s.px = s.px * ca; s.py = s.py * ca; s.z = s.z * ca; s.d = d_new;
}

// StrongGaussianBeam (src/tracking.jl:1621-1641): the slice weights and
// offsets follow the fixed words.
static __device__ __noinline__ void strong_gauss(P6& s, const double* w) {
    const int nz = int(w[sgb::NZ]);
    const double* wt = w + sgb::WORDS;
    const double factor = w[sgb::FACTOR], sx2 = w[sgb::SX2], sy2 = w[sgb::SY2];
    double px = s.px, py = s.py;
    for (int i = 0; i < nz; ++i) {
        const double dx = s.x - wt[nz + i];
        const double dy = s.y - wt[2 * nz + i];
        const double g = wt[i] * libm::exp(-0.5 * (dx * dx / sx2 + dy * dy / sy2));
        px = px - factor * g * dx / sx2;
        py = py - factor * g * dy / sy2;
    }
    s.px = px;
    s.py = py;
}

// LongitudinalRLCWake (src/tracking.jl:1647-1654, wake.jl:27-37).
__device__ __forceinline__ void rlc_wake(P6& s, const double* w) {
    const double zc = s.z / C_LIGHT;
    const double t = isnan(zc) ? zc : (zc > 0.0 ? 0.0 : zc);  // Julia min(z/c, 0)
    double wf = 0.0;
    if (!(t > 0.0))
        wf = w[rlc::A] * (libm::cos(w[rlc::W0P] * t) + libm::sin(w[rlc::W0P] * t) / w[rlc::D2Q0P]) *
             libm::exp(w[rlc::W0] * t / w[rlc::D2Q0]);
    s.d = s.d - w[rlc::SCALE] * wf;
}

// LongitudinalWake (src/tracking.jl:1656-1663, wake.jl:68-91): linear
// interpolation in the table after the fixed words; with sorted times
// (h.order = 1) the segment is found by bisection, which selects the same
// segment as the reference's scan.
static __device__ __noinline__ void tab_wake(P6& s, const double* w, const RecHdr& h) {
    const int n = int(w[tw::N]);
    const double* xs = w + tw::WORDS;
    const double* ys = xs + n;
    const double t = s.z / C_LIGHT;
    double wf = 0.0;
    if (!(t > w[tw::T1F])) {
        const double x = t * w[tw::FLIP];
        if (x <= xs[0]) {
            const double slope = (ys[1] - ys[0]) / (xs[1] - xs[0]);
            wf = ys[0] + slope * (x - xs[0]);
        } else if (x >= xs[n - 1]) {
            const double slope = (ys[n - 1] - ys[n - 2]) / (xs[n - 1] - xs[n - 2]);
            wf = ys[n - 1] + slope * (x - xs[n - 1]);
        } else if (isnan(x)) {
            wf = ys[n - 1];
        } else {
            int i = 1;
            if (h.order == 1) {  // first i with x < xs[i]; x < xs[n-1] here
                int lo = 1, hi = n - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (x < xs[mid]) hi = mid; else lo = mid + 1;
                }
                i = lo;
            } else {
                while (i < n - 1 && !(x < xs[i])) ++i;
            }
            if (x < xs[i]) {
                const double slope = (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1]);
                wf = ys[i - 1] + slope * (x - xs[i - 1]);
            } else {
                wf = ys[n - 1];
            }
        }
    }
    s.d = s.d - w[tw::SCALE] * wf;
}

// Wiggler (src/tracking.jl:1224-1529): 4th-order composition of the
// second-order map _wig_map_2nd, whose kicks are the vector potential of the
// By (horizontal) and Bx (vertical) harmonics; optional radiation kicks.
// Zw, the longitudinal position inside the wiggler, advances by dl/2 twice
// per map (the same sequence for every particle).
__device__ __forceinline__ double sinc_taylor(double x) {
    const double x2 = x * x;
    return 1.0 - x2 / 6.0 * (1.0 - x2 / 20.0 * (1.0 - x2 / 42.0 * (1.0 - x2 / 72.0)));
}

static __device__ __noinline__ void wig_ax_axpy(const double* w, double x, double y, double Zw, double& ax, double& axpy) {
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    ax = 0.0;
    axpy = 0.0;
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double cx = libm::cos(kx * x), chy = libm::cosh(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ax = ax + hp[wg::C_AX] * cx * chy * sz;
        const double shy = libm::sinh(ky * y);
        const double sxkx = hp[wg::SINC] != 0.0 ? libm::sin(kx * x) / kx : x * sinc_taylor(kx * x);
        axpy = axpy + hp[wg::C_AXPY] * sxkx * shy * sz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double shx = libm::sinh(kx * x), sy = libm::sin(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ax = ax + hp[wg::C_AX] * shx * sy * sz;
        const double chx = libm::cosh(kx * x), cy = libm::cos(ky * y);
        axpy = axpy + hp[wg::C_AXPY] * chx * cy * sz;
    }
}

static __device__ __noinline__ void wig_ay_aypx(const double* w, double x, double y, double Zw, double& ay, double& aypx) {
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    ay = 0.0;
    aypx = 0.0;
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double sx = libm::sin(kx * x), shy = libm::sinh(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ay = ay + hp[wg::C_AY] * sx * shy * sz;
        const double cx = libm::cos(kx * x), chy = libm::cosh(ky * y);
        aypx = aypx + hp[wg::C_AYPX] * cx * chy * sz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double chx = libm::cosh(kx * x), cy = libm::cos(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ay = ay + hp[wg::C_AY] * chx * cy * sz;
        const double shx = libm::sinh(kx * x);
        const double syky = hp[wg::SINC] != 0.0 ? libm::sin(ky * y) / ky : y * sinc_taylor(ky * y);
        aypx = aypx + hp[wg::C_AYPX] * shx * syky * sz;
    }
}

__device__ __forceinline__ void wig_map_2nd(P6& s, const double* w, double dl, double dl2, double& Zw) {
    const double inv1pd = 1.0 / (1.0 + s.d);
    const double dld = dl * inv1pd;
    const double dl2d = dl2 * inv1pd;
    Zw = Zw + dl2;
    double a, ap;
    wig_ay_aypx(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.y = s.y + dl2d * s.py;
    s.z = s.z + (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    wig_ay_aypx(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    wig_ax_axpy(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - a;
    s.py = s.py - ap;
    s.x = s.x + dld * s.px;
    s.z = s.z + (dld / 2.0) * (s.px * s.px) * inv1pd;
    wig_ax_axpy(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + a;
    s.py = s.py + ap;
    wig_ay_aypx(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.y = s.y + dl2d * s.py;
    s.z = s.z + (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    wig_ay_aypx(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    Zw = Zw + dl2;
}

// _wig_B (transverse field) and _wig_radiation_kicks, between the removal and
// the restoration of the vector-potential kick (tracking.jl:1400-1463, 1477-1483).
static __device__ __noinline__ void wig_rad_block(P6& s, const double* w, double Zw) {
    double ax, axpy, ay, aypx;
    wig_ax_axpy(w, s.x, s.y, Zw, ax, axpy);
    wig_ay_aypx(w, s.x, s.y, Zw, ay, aypx);
    s.px = s.px - ax;
    s.py = s.py - ay;
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    double Bxv = 0.0, Byv = 0.0;
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double sx = libm::sin(kx * s.x), cx = libm::cos(kx * s.x);
        const double chy = libm::cosh(ky * s.y), shy = libm::sinh(ky * s.y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * sx * shy * cz;
        Byv = Byv - hp[wg::B_Y] * cx * chy * cz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double shx = libm::sinh(kx * s.x), chx = libm::cosh(kx * s.x);
        const double sy = libm::sin(ky * s.y), cy = libm::cos(ky * s.y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * chx * cy * cz;
        Byv = Byv - hp[wg::B_Y] * shx * sy * cz;
    }
    const double B2 = Bxv * Bxv + Byv * Byv;
    if (B2 != 0.0) {
        const double irho2 = B2 / w[wg::HH];
        const double dFactor = (1.0 + s.d) * (1.0 + s.d);
        const double dDelta = -w[wg::SRCOEF] * dFactor * irho2 * w[wg::SL];
        const double scale = 1.0 + dDelta;
        s.px = s.px * scale;
        s.py = s.py * scale;
        s.d = s.d + dDelta;
    }
    s.px = s.px + ax;
    s.py = s.py + ay;
}

static __device__ __noinline__ void wiggler(P6& s, const double* w) {
    const long long nstep = (long long)w[wg::NSTEP];
    const double dl1 = w[wg::DL1], dl0 = w[wg::DL0], dl1h = w[wg::DL1H], dl0h = w[wg::DL0H];
    const bool rad = w[wg::RAD] == 1.0;
    double Zw = 0.0;
    if (rad) wig_rad_block(s, w, Zw);
    for (long long k = 0; k < nstep; ++k) {
        wig_map_2nd(s, w, dl1, dl1h, Zw);
        wig_map_2nd(s, w, dl0, dl0h, Zw);
        wig_map_2nd(s, w, dl1, dl1h, Zw);
        if (rad) wig_rad_block(s, w, Zw);
    }
}

// Misalignment (src/tracking.jl:60-67): r + t, and the column-major 6x6 product.
__device__ __forceinline__ void mat6(const double* R, P6& s) {
    double v[6] = {s.x, s.px, s.y, s.py, s.z, s.d};
    double o[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double acc = R[i] * v[0];
#pragma unroll
        for (int j = 1; j < 6; ++j) acc = acc + R[j * 6 + i] * v[j];
        o[i] = acc;
    }
    s.x = o[0]; s.px = o[1]; s.y = o[2]; s.py = o[3]; s.z = o[4]; s.d = o[5];
}

__device__ __forceinline__ void mis_entrance(const MisalignDev& m, P6& s) {
    s.x = s.x + m.t1[0]; s.px = s.px + m.t1[1]; s.y = s.y + m.t1[2];
    s.py = s.py + m.t1[3]; s.z = s.z + m.t1[4]; s.d = s.d + m.t1[5];
    if (m.r1nz) mat6(m.r1, s);
}

__device__ __forceinline__ void mis_exit(const MisalignDev& m, P6& s) {
    if (m.r2nz) mat6(m.r2, s);
    s.x = s.x + m.t2[0]; s.px = s.px + m.t2[1]; s.y = s.y + m.t2[2];
    s.py = s.py + m.t2[3]; s.z = s.z + m.t2[4]; s.d = s.d + m.t2[5];
}

// The kinds outside the integrator core, out of line behind one call site.
template <bool EXACT>
static __device__ __noinline__ bool apply_rare(P6& s, const double* w, const RecHdr& h, double beti, double beta,
                                               double beta2) {
    switch (h.kind) {
        case DK_SOLENOID: solenoid<EXACT>(s, w, beti); break;
        case DK_CORRECTOR: corrector(s, w); break;
        case DK_TRANSLATION: translation(s, w, beti); break;
        case DK_YROTATION: yrotation(s, w, beti); break;
        case DK_CRAB: crab_cavity<EXACT>(s, w, h, beti); break;
        case DK_ACCEL: accel_cavity(s, w, beta2); break;
        case DK_LONG_RF_MAP: long_rf_map(s, w, beta); break;
        case DK_LORENTZ: lorentz_boost(s, w); break;
        case DK_INV_LORENTZ: inv_lorentz_boost(s, w); break;
        case DK_STRONG_THIN_GAUSS: strong_thin_gauss(s, w); break;
        case DK_LBEND: lbend(s, w, h); break;
        case DK_SGB: strong_gauss(s, w); break;
        case DK_RLC_WAKE: rlc_wake(s, w); break;
        case DK_TAB_WAKE: tab_wake(s, w, h); break;
        case DK_WIGGLER: wiggler(s, w); break;
        case DK_NAN: set_nan(s); break;
        default: return false;
    }
    return true;
}

// One lattice entry.  Returns false for an unknown record kind.  RARE =
// false drops the call of apply_rare (tables of core kinds only): the tracking
// kernel is then the integrator core alone, which measured 2.5% faster on the
// DBA ring than the same loop with the rare kinds' dispatch reachable.
template <bool EXACT, bool RARE = true>
__device__ __forceinline__ bool apply_record(P6& s, const double* rec, const RecHdr& h, const MisalignDev* mis,
                                             double beti, double beta, double beta2) {
    const double* w = rec + HDR_WORDS;
    if (h.flags & RF_MISALIGN) mis_entrance(mis[h.aux], s);
    switch (h.kind) {
        case DK_IDENTITY: break;
        case DK_DRIFT: {
            DCache c;
            make_cache(s, beti, c);
            drift<EXACT>(s, w[drift::L], w[drift::L] * beti, c);
            break;
        }
        case DK_MULTIPOLE:
            switch (h.order) {
                case 0: multipole<0, EXACT>(s, w, h.nsteps, beti); break;
                case 1: multipole_body<1, EXACT>(s, w, h.nsteps, beti); break;
                case 2: multipole_body<2, EXACT>(s, w, h.nsteps, beti); break;
                default: multipole<3, EXACT>(s, w, h.nsteps, beti); break;
            }
            break;
        case DK_THIN:
            switch (h.order) {
                case 0: thin_kick<0>(s, w + thin::PA, w + thin::PB, 1.0); break;
                case 1: thin_kick<1>(s, w + thin::PA, w + thin::PB, 1.0); break;
                case 2: thin_kick<2>(s, w + thin::PA, w + thin::PB, 1.0); break;
                default: thin_kick<3>(s, w + thin::PA, w + thin::PB, 1.0); break;
            }
            break;
        case DK_SBEND:
            switch (h.order) {
                case 0: sbend<0, EXACT>(s, w, h, beti); break;
                case 1: sbend<1, EXACT>(s, w, h, beti); break;
                case 2: sbend<2, EXACT>(s, w, h, beti); break;
                default: sbend<3, EXACT>(s, w, h, beti); break;
            }
            break;
        case DK_EXACT_SBEND: exact_sbend(s, w, h, beti); break;
        case DK_RF: rf_cavity<EXACT>(s, w, h, beti, beta2); break;
        default:
            if (!RARE || !apply_rare<EXACT>(s, w, h, beti, beta, beta2)) return false;
            break;
    }
    if (h.flags & RF_MISALIGN) mis_exit(mis[h.aux], s);
    return true;
}

}  // namespace dev
}  // namespace tp

// tp_reverse.cuh -- reverse (adjoint) maps of the tracking path.
//
// Every function here takes the state AFTER one building block of pass!
// (src/tracking.jl) and the cotangent (adjoint) of that state, and
//   1. rebuilds the state BEFORE the block with the block's exact inverse:
//      the integrators are time-reversible, so drift(L)^-1 = drift(-L),
//      kick(K)^-1 = kick(-K), exact_bend_body(L)^-1 = exact_bend_body(-L),
//      bend_edge(theta)^-1 = bend_edge(-theta), yrot(phi)^-1 = yrot(-phi);
//      bend_fringe, whose py update is implicit, is inverted by fixed-point
//      iteration on py;
//   2. replaces the cotangent by its pull-back through the block at that
//      rebuilt input (the transposed Jacobian times the cotangent).
// The adjoint kernel walks a K-turn segment of the lattice backwards this way,
// starting from a stored particle state, so no per-element tape is kept.
//
// Derivatives are hand-derived from the forward maps of tp_maps.cuh.  Two
// helpers come up throughout: for pz = sqrt(D - px^2 - py^2), with D = dp1^2,
//   dpz = (dp1*ddp1 - px*dpx - py*dpy) / pz,
// and for asin(px/d2) with d2 = sqrt(D - py^2) (so sqrt(d2^2 - px^2) = pz),
//   d asin(px/d2) = (dpx - px*dd2/d2) / pz.
// The bend_fringe coefficients are differentiated in forward mode with a
// three-direction dual number (px, py, dp1), the only inputs they have.
// Inside a K-turn segment the rebuilt states drift from the forward ones by
// the rounding of the inverse maps (about 1e-13 absolute per turn on the DBA
// ring); each segment restarts from its stored state.
#pragma once
#include "tp_maps.cuh"

namespace tp {
namespace dev {

// Cotangent of a P6.
struct L6 {
    double x, px, y, py, z, d;
};

// ---------------------------------------------------------------------------
// Drifts (src/tracking.jl:87-108)
// ---------------------------------------------------------------------------
// Exact branch: x' = x + N px, y' = y + N py, z' = z + N bd - L beti with
// N = L / sqrt(A - px^2 - py^2); px, py, delta unchanged, so pz is the same
// before and after.  dN = -N bd ddelta / pz2 + N (px dpx + py dpy) / pz2.
__device__ __forceinline__ void rev_drift_exact(P6& s, L6& l, double L, double Lbeti, const DCache& c) {
    const double pz2 = c.A - s.px * s.px - s.py * s.py;
    const double N = L / sqrt(pz2);
    s.x = s.x - N * s.px;
    s.y = s.y - N * s.py;
    s.z = s.z - N * c.bd + Lbeti;
    const double g = l.x * s.px + l.y * s.py + l.z * c.bd;
    const double q = g * N / pz2;
    l.px = l.px + l.x * N + q * s.px;
    l.py = l.py + l.y * N + q * s.py;
    l.d = l.d + l.z * N - q * c.bd;
}

// Linearised branch: N = L/opd, z' = z + N (px^2 + py^2) / (2 opd).
__device__ __forceinline__ void rev_drift_lin(P6& s, L6& l, double L, const DCache& c) {
    const double N = L / c.opd;
    const double Q = (s.px * s.px + s.py * s.py) / (2.0 * c.opd);
    s.x = s.x - N * s.px;
    s.y = s.y - N * s.py;
    s.z = s.z - N * Q;
    const double No = N / c.opd;
    const double lx = l.x, ly = l.y, lz = l.z;
    l.px = l.px + lx * N + lz * No * s.px;
    l.py = l.py + ly * N + lz * No * s.py;
    l.d = l.d - No * (lx * s.px + ly * s.py + 2.0 * lz * Q);
}

template <bool EXACT>
__device__ __forceinline__ void rev_drift(P6& s, L6& l, double L, double Lbeti, const DCache& c) {
    if (EXACT) rev_drift_exact(s, l, L, Lbeti, c);
    else rev_drift_lin(s, l, L, c);
}

// ---------------------------------------------------------------------------
// Thin kicks (src/tracking.jl:243-305)
// ---------------------------------------------------------------------------
// f(z) = sum_n (pb_n + i pa_n) z^n and f'(z), z = x + i y.  By Cauchy-Riemann
// d Re f/dx = Re f', d Re f/dy = -Im f', d Im f/dx = Im f', d Im f/dy = Re f'.
template <int M>
__device__ __forceinline__ void horner_d(const double* pa, const double* pb, double x, double y, double& re,
                                         double& im, double& dre, double& dim) {
    re = pb[M];
    im = pa[M];
    dre = 0.0;
    dim = 0.0;
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        // derivative first (uses the previous partial sum)
        double td = dre * x - dim * y + re;
        dim = dim * x + dre * y + im;
        dre = td;
        double t = re * x - im * y + pb[i];
        im = im * x + re * y + pa[i];
        re = t;
    }
}

// strthinkick with length K.  `pm` (1..3) selects the normal coefficient whose
// gradient is accumulated into g (d/d pb_pm of this kick, times the cotangent);
// pm = 0 accumulates nothing.
template <int M>
__device__ __forceinline__ void rev_thin_kick(P6& s, L6& l, const double* pa, const double* pb, double K, int pm,
                                              double& g) {
    double re, im, dre, dim;
    horner_d<M>(pa, pb, s.x, s.y, re, im, dre, dim);
    s.px = s.px + K * re;
    s.py = s.py - K * im;
    const double lpx = l.px, lpy = l.py;
    l.x = l.x - K * (lpx * dre - lpy * dim);
    l.y = l.y + K * (lpx * dim + lpy * dre);
    if (pm > 0 && pm <= M) {
        // z^pm
        double zr = s.x, zi = s.y;
        for (int k = 1; k < pm; ++k) {
            double t = zr * s.x - zi * s.y;
            zi = zr * s.y + zi * s.x;
            zr = t;
        }
        g = g + K * (lpy * zi - lpx * zr);
    }
}

// bndthinkick: px' = px - K (Re f - (delta - x h) h), py' = py + K Im f,
// z' = z + K h x beti.
template <int M>
__device__ __forceinline__ void rev_bend_kick(P6& s, L6& l, const double* pa, const double* pb, double K, double Kh,
                                              double irho, double beti) {
    double re, im, dre, dim;
    horner_d<M>(pa, pb, s.x, s.y, re, im, dre, dim);
    s.px = s.px + K * (re - (s.d - s.x * irho) * irho);
    s.py = s.py - K * im;
    s.z = s.z - Kh * s.x * beti;
    const double lpx = l.px, lpy = l.py;
    l.x = l.x - K * (lpx * (dre + irho * irho) - lpy * dim) + l.z * Kh * beti;
    l.y = l.y + K * (lpx * dim + lpy * dre);
    l.d = l.d + lpx * K * irho;
}

// ---------------------------------------------------------------------------
// Multipole: symplectic4_pass (src/tracking.jl:317-341) run backwards.
// ---------------------------------------------------------------------------
template <int M, bool EXACT>
__device__ __forceinline__ void rev_multipole_body(P6& s, L6& l, const double* w, int nsteps, double beti, int pm,
                                                   double& g) {
    const double L1 = w[mp::L1], L2 = w[mp::L2], K1 = w[mp::K1], K2 = w[mp::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[mp::PA + i]; pb[i] = w[mp::PB + i]; }
    const double L1b = L1 * beti, L2b = L2 * beti;
    DCache c;
    make_cache(s, beti, c);  // delta is unchanged by the element
    // Backwards, the first D(L1) of a step (j = 0) and the last D(L1) of the
    // step before it (j = 3) follow each other with no kick between: px, py and
    // delta are the same, so the second reuses the first's N (the same bits).
    // The pull-back's N / pz2 = L / pz2^(3/2) is N^3 / L^2, with 1/L^2 once per
    // element: no division per drift (a few ulps, which the gradient's
    // tolerance leaves room for).  The sweep runs on survivors only, pz2 > 0.
    // (a zero length has N = 0 and no pull-back term)
    const double iL1sq = L1 * L1 > 0.0 ? 1.0 / (L1 * L1) : 0.0, iL2sq = L2 * L2 > 0.0 ? 1.0 / (L2 * L2) : 0.0;
    double N = 0.0;
#pragma unroll 1
    for (int k = 4 * nsteps - 1; k >= 0; --k) {
        const int j = k & 3;
        const bool outer = (j == 0) || (j == 3);
        if (j != 3) rev_thin_kick<M>(s, l, pa, pb, j == 1 ? K2 : K1, pm, g);
        if (EXACT) {
            if (j != 3 || k == 4 * nsteps - 1) N = (outer ? L1 : L2) / sqrt(c.A - s.px * s.px - s.py * s.py);
            s.x = s.x - N * s.px;
            s.y = s.y - N * s.py;
            s.z = s.z - N * c.bd + (outer ? L1b : L2b);
            const double gq = l.x * s.px + l.y * s.py + l.z * c.bd;
            const double q = gq * (N * N * N) * (outer ? iL1sq : iL2sq);
            l.px = l.px + l.x * N + q * s.px;
            l.py = l.py + l.y * N + q * s.py;
            l.d = l.d + l.z * N - q * c.bd;
        } else {
            rev_drift<EXACT>(s, l, outer ? L1 : L2, outer ? L1b : L2b, c);
        }
    }
}

// Out of line for the orders lattices use rarely (0: a body with no field, 3:
// octupoles).  Quadrupoles (order 1) and sextupoles (order 2) run inline in the
// sweep's element loop: a call there saves and restores the caller's live
// registers through the stack at every magnet, and inlining the two made the
// reverse sweep of the DBA gradient 24-28 % faster.
template <int M, bool EXACT>
__device__ __noinline__ void rev_multipole(P6& s, L6& l, const double* w, int nsteps, double beti, int pm,
                                           double& g) {
    rev_multipole_body<M, EXACT>(s, l, w, nsteps, beti, pm, g);
}

// ---------------------------------------------------------------------------
// SBend: edge_fringe (src/tracking.jl:160-221) and the bend integrator.
// ---------------------------------------------------------------------------
// fy(px, delta) and its partial derivatives, per edge method.
__device__ __forceinline__ void edge_fy(double px, double d, double irho, double fx, double e, double fc, int method,
                                        bool fc_zero, bool is_exit, double& fy, double& dfy_dpx, double& dfy_dd) {
    const double opd = 1.0 + d;
    dfy_dpx = 0.0;
    dfy_dd = 0.0;
    if (method == 3) {
        const double q = px / opd;
        const double sg = is_exit ? -1.0 : 1.0;
        const double t = libm::tan(e - fc + sg * q);
        fy = irho * t;
        const double dt = irho * (1.0 + t * t);
        dfy_dpx = dt * sg / opd;
        dfy_dd = -dt * sg * q / opd;
    } else if (method == 2) {
        if (fc_zero) {
            fy = fx / opd;
            dfy_dd = -fy / opd;
        } else {
            const double t = libm::tan(e - fc / opd);
            fy = irho * t / opd;
            dfy_dd = irho * ((1.0 + t * t) * fc / (opd * opd) - t / opd) / opd;
        }
    } else {
        if (fc_zero) {
            fy = fx;
        } else {
            const double t = libm::tan(e - fc / opd);
            fy = irho * t;
            dfy_dd = irho * (1.0 + t * t) * fc / (opd * opd);
        }
    }
}

// px' = px + x fx, py' = py - y fy(px, delta).
__device__ __forceinline__ void rev_edge_fringe(P6& s, L6& l, double irho, double fx, double e, double fc,
                                                int method, bool fc_zero, bool is_exit) {
    s.px = s.px - s.x * fx;
    double fy, dpx, dd;
    edge_fy(s.px, s.d, irho, fx, e, fc, method, fc_zero, is_exit, fy, dpx, dd);
    s.py = s.py + s.y * fy;
    const double lpy = l.py;
    l.x = l.x + l.px * fx;
    l.y = l.y - lpy * fy;
    l.px = l.px - lpy * s.y * dpx;
    l.d = l.d - lpy * s.y * dd;
}

template <int M, bool EXACT>
__device__ __noinline__ void rev_sbend(P6& s, L6& l, const double* w, const RecHdr& h, double beti) {
    const double irho = w[sb::IRHO];
    if (h.flags & RF_FRINGE_OUT)
        rev_edge_fringe(s, l, irho, w[sb::FX_OUT], w[sb::E_OUT], w[sb::FC_OUT], h.method_out,
                        h.flags & RF_FC_OUT_ZERO, true);
    const double L1 = w[mp::L1], L2 = w[mp::L2], K1 = w[mp::K1], K2 = w[mp::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[mp::PA + i]; pb[i] = w[mp::PB + i]; }
    const double L1b = L1 * beti, L2b = L2 * beti;
    const double K1h = K1 * irho, K2h = K2 * irho;
    DCache c;
    make_cache(s, beti, c);
    // D1 K1 D2 K2 D2 K1 D1 is a palindrome: the reverse visits the same list.
    for (int st = 0; st < h.nsteps; ++st) {
        rev_drift<EXACT>(s, l, L1, L1b, c);
        rev_bend_kick<M>(s, l, pa, pb, K1, K1h, irho, beti);
        rev_drift<EXACT>(s, l, L2, L2b, c);
        rev_bend_kick<M>(s, l, pa, pb, K2, K2h, irho, beti);
        rev_drift<EXACT>(s, l, L2, L2b, c);
        rev_bend_kick<M>(s, l, pa, pb, K1, K1h, irho, beti);
        rev_drift<EXACT>(s, l, L1, L1b, c);
    }
    if (h.flags & RF_FRINGE_IN)
        rev_edge_fringe(s, l, irho, w[sb::FX_IN], w[sb::E_IN], w[sb::FC_IN], h.method_in, h.flags & RF_FC_IN_ZERO,
                        false);
}

// ---------------------------------------------------------------------------
// Exact sector bend (src/tracking.jl:717-973)
// ---------------------------------------------------------------------------
// yrot (:727-745): p = c pz - s px, px' = s pz + c px, x' = x pz / p,
// y' = y + x py s / p, z' = z + dp1 x s / p.
__device__ __forceinline__ void rev_yrot(P6& r, L6& l, double c, double s, double beti) {
    const double dp1 = beti + r.d;
    yrot(r, c, -s, dp1);  // inverse
    const double pz = pxyz(dp1 * dp1, r.px, r.py);
    const double p = c * pz - s * r.px;
    const double ip = 1.0 / p;
    const double xs = r.x * s * ip;
    const double lp = -(l.x * r.x * pz + l.y * r.x * r.py * s + l.z * dp1 * r.x * s) * ip * ip;
    const double lx = l.x * pz * ip + l.y * r.py * s * ip + l.z * dp1 * s * ip;
    const double lpz = l.x * r.x * ip + lp * c + l.px * s;
    const double ipz = 1.0 / pz;
    const double lpx = l.px * c - lp * s - lpz * r.px * ipz;
    const double lpy = l.py + l.y * xs - lpz * r.py * ipz;
    const double ld = l.d + l.z * xs + lpz * dp1 * ipz;
    l.x = lx; l.px = lpx; l.py = lpy; l.d = ld;
}

// bend_edge, Forest 12.41 (:822-851).  Inverse: the same edge with -theta.
__device__ __forceinline__ void rev_bend_edge(P6& r, L6& l, double h, double c, double s, double s2, double theta,
                                              double thh, double beti) {
    const double dp1 = beti + r.d;
    bend_edge_body(r, h, c, -s, -s2, -theta, -thh, dp1);  // inverse, inline
    const double D = dp1 * dp1;
    const double pz = pxyz(D, r.px, r.py);
    const double d2 = pxyz(D, 0.0, r.py);
    const double pxn = r.px * c + (pz - h * r.x) * s;
    const double pzn = pxyz(D, pxn, r.py);
    const double num = r.x * (r.px * s2 + s * s * (2.0 * pz - h * r.x));
    const double den = pzn + pz * c - r.px * s;
    const double dasin = asin_ool(jclamp(r.px / d2)) - asin_ool(jclamp(pxn / d2));
    const double ih = 1.0 / h, ipz = 1.0 / pz, ipzn = 1.0 / pzn, id2 = 1.0 / d2, iden = 1.0 / den;
    const double lds = l.y * r.py * ih + l.z * dp1 * ih;  // cotangent of dasin
    const double lnum = l.x * iden;
    const double lden = -l.x * num * iden * iden;
    double lx = l.x * c + lnum * (r.px * s2 + s * s * (2.0 * pz - 2.0 * h * r.x));
    double lpx = -lden * s + lnum * r.x * s2 + lds * ipz;
    double lpz = lden * c + lnum * r.x * 2.0 * s * s;
    double lpzn = lden;
    double ld2 = -lds * r.px * id2 * ipz + lds * pxn * id2 * ipzn;
    double lpxn = l.px - lds * ipzn - lpzn * pxn * ipzn;
    double lpy = l.py + l.y * (thh + dasin * ih) - lpzn * r.py * ipzn;
    double lD = 0.5 * lpzn * ipzn;
    lpx = lpx + lpxn * c;
    lpz = lpz + lpxn * s;
    lx = lx - lpxn * s * h;
    lpx = lpx - lpz * r.px * ipz;
    lpy = lpy - lpz * r.py * ipz - ld2 * r.py * id2;
    lD = lD + 0.5 * lpz * ipz + 0.5 * ld2 * id2;
    const double ldp1 = l.z * (theta + dasin) * ih + 2.0 * dp1 * lD;
    l.x = lx; l.px = lpx; l.py = lpy; l.d = l.d + ldp1;
}

// Three-direction dual number: value and derivatives along (px, py, dp1).
struct D3 {
    double v, a, b, c;
};
__device__ __forceinline__ D3 d3(double v) { return D3{v, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ D3 operator+(D3 x, D3 y) { return D3{x.v + y.v, x.a + y.a, x.b + y.b, x.c + y.c}; }
__device__ __forceinline__ D3 operator-(D3 x, D3 y) { return D3{x.v - y.v, x.a - y.a, x.b - y.b, x.c - y.c}; }
__device__ __forceinline__ D3 operator-(D3 x) { return D3{-x.v, -x.a, -x.b, -x.c}; }
__device__ __forceinline__ D3 operator*(D3 x, D3 y) {
    return D3{x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b, x.c * y.v + x.v * y.c};
}
__device__ __forceinline__ D3 operator*(double k, D3 y) { return D3{k * y.v, k * y.a, k * y.b, k * y.c}; }
__device__ __forceinline__ D3 operator+(D3 x, double k) { return D3{x.v + k, x.a, x.b, x.c}; }
__device__ __forceinline__ D3 operator+(double k, D3 x) { return D3{x.v + k, x.a, x.b, x.c}; }
__device__ __forceinline__ D3 scale(D3 x, double v, double dv) { return D3{v, dv * x.a, dv * x.b, dv * x.c}; }
__device__ __forceinline__ D3 operator/(D3 x, D3 y) {
    const double q = x.v / y.v;
    const double iy = 1.0 / y.v;
    return D3{q, (x.a - q * y.a) * iy, (x.b - q * y.b) * iy, (x.c - q * y.c) * iy};
}
__device__ __forceinline__ D3 d3_sqrt(D3 x) {
    const double r = sqrt(x.v);
    return scale(x, r, 0.5 / r);
}
__device__ __forceinline__ D3 d3_tan(D3 x) {
    const double t = libm::tan(x.v);
    return scale(x, t, 1.0 + t * t);
}
__device__ __forceinline__ D3 d3_atan(D3 x) { return scale(x, libm::atan(x.v), 1.0 / (1.0 + x.v * x.v)); }
__device__ __forceinline__ D3 d3_cos(D3 x) { return scale(x, libm::cos(x.v), -libm::sin(x.v)); }

// The coefficients of bend_fringe (:752-815) as functions of (px, py, dp1):
// phi (py kick per unit y), dpx, dpy, dd.  Same expressions as the forward map.
__device__ __forceinline__ void fringe_coeffs(D3 px, D3 py, D3 dp1, double b0, double gK, D3& phi, D3& dpx, D3& dpy,
                                              D3& dd) {
    D3 pz = d3_sqrt(dp1 * dp1 - px * px - py * py);
    D3 xp = px / pz;
    D3 yp = py / pz;
    D3 term1 = 1.0 + xp * xp * (2.0 + yp * yp);
    D3 term2 = xp / (1.0 + yp * yp);
    phi = (-b0) * d3_tan((b0 * gK) * term1 * pz - d3_atan(term2));
    D3 px2 = px * px;
    D3 py2 = py * py;
    D3 pz2 = pz * pz;
    D3 pz4 = pz2 * pz2;
    D3 py2z2 = py2 + pz2;
    D3 arg_sec = ((b0 * gK) * (pz4 + px2 * (py2 + 2.0 * pz2))) / (pz2 * pz) - d3_atan(px * pz / (py2 + pz2));
    D3 sec = d3(1.0) / d3_cos(arg_sec);
    D3 powsec = sec * sec;
    D3 py4 = py2 * py2;
    D3 py6 = py4 * py2;
    D3 pz5 = pz4 * pz;
    D3 pz6 = pz4 * pz2;
    D3 py2z2_sq = py2z2 * py2z2;
    D3 denom = pz5 * (py4 + px2 * pz2 + 2.0 * py2 * pz2 + pz4);
    D3 dpx_num = (-b0) * (px2 * pz4 * (py2 - pz2) - pz6 * (py2 + pz2) +
                          (b0 * gK) * px *
                              (pz2 * py2z2_sq * (2.0 * py2 + 3.0 * pz2) + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4) +
                               px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 9.0 * py2 * pz4 + 5.0 * pz6))) *
                 powsec;
    dpx = dpx_num / denom;
    D3 dpy_num = (-b0) * py *
                 (px * pz4 * (py2 + pz2) +
                  (b0 * gK) * (-(pz4 * py2z2_sq) + px2 * px2 * (3.0 * py2 * pz2 + 4.0 * pz4) +
                               px2 * (3.0 * py6 + 10.0 * py4 * pz2 + 11.0 * py2 * pz4 + 3.0 * pz6))) *
                 powsec;
    dpy = dpy_num / denom;
    D3 dd_num = b0 * dp1 *
                (px * pz4 * (py2 - pz2) +
                 (b0 * gK) * (-(pz4 * py2z2_sq) + px2 * px2 * (3.0 * py2 * pz2 + 2.0 * pz4) +
                              px2 * (3.0 * py6 + 8.0 * py4 * pz2 + 7.0 * py2 * pz4 + pz6))) *
                powsec;
    dd = dd_num / denom;
}

// phi alone, in plain doubles (the fixed-point iteration of the inverse).
__device__ __forceinline__ double fringe_phi(double px, double py, double dp1, double b0, double gK) {
    double pz = pxyz(dp1 * dp1, px, py);
    double xp = px / pz;
    double yp = py / pz;
    double term1 = 1.0 + xp * xp * (2.0 + yp * yp);
    double term2 = xp / (1.0 + yp * yp);
    return -b0 * libm::tan(b0 * gK * term1 * pz - libm::atan(term2));
}

// The coefficients with gK = 0 (no fringe-field integral: the case of the
// reference's ERBend defaults).  Then tan(-atan(u)) = -u gives
// phi = b0 xp / (1 + yp^2), and 1/cos^2(atan(u)) = 1 + u^2 with
// u = px pz / (py^2 + pz^2), so no transcendental function is left.
__device__ __forceinline__ void fringe_coeffs_gk0(D3 px, D3 py, D3 dp1, double b0, D3& phi, D3& dpx, D3& dpy,
                                                  D3& dd) {
    D3 px2 = px * px;
    D3 py2 = py * py;
    D3 pz2 = dp1 * dp1 - px2 - py2;
    D3 pz = d3_sqrt(pz2);
    D3 ipz = d3(1.0) / pz;
    D3 xp = px * ipz;
    D3 yp = py * ipz;
    phi = b0 * (xp / (1.0 + yp * yp));
    D3 pz4 = pz2 * pz2;
    D3 py2z2 = py2 + pz2;
    D3 u = px * pz / py2z2;
    D3 powsec = 1.0 + u * u;
    D3 denom = pz4 * pz * (py2 * py2 + px2 * pz2 + 2.0 * py2 * pz2 + pz4);
    D3 w = powsec / denom;
    D3 a = px * pz4;
    dpx = (-b0) * ((px2 * pz4 * (py2 - pz2) - pz4 * pz2 * py2z2) * w);
    dpy = (-b0) * (py * a * py2z2 * w);
    dd = b0 * (dp1 * a * (py2 - pz2) * w);
}

__device__ __forceinline__ double fringe_phi_gk0(double px, double py, double dp1, double b0) {
    double pz = pxyz(dp1 * dp1, px, py);
    double xp = px / pz;
    double yp = py / pz;
    return b0 * (xp / (1.0 + yp * yp));
}

// bend_fringe, Forest 13.13 (:752-815): with yf the new y,
//   x' = x + dpx yf^2/2, y' = yf, py' = py - phi yf, z' = z - dd yf^2/2,
// where yf = 2y / (1 + sqrt(1 - 2 dpy y)) solves y = yf - dpy yf^2 / 2, and
// (phi, dpx, dpy, dd) depend on (px, py, dp1) only.  The inverse solves
// py = py' + phi(px, py, dp1) yf by fixed-point iteration (a contraction:
// |d phi/d py| yf is of order irho * |y|).
__device__ __noinline__ void rev_bend_fringe(P6& r, L6& l, double b0, double gK, double beti) {
    const double dp1v = beti + r.d;
    const double yf = r.y;
    double py = r.py;
    D3 phi, dpx, dpy, dd;
    if (gK == 0.0) {
        for (int it = 0; it < 12; ++it) {
            const double pn = r.py + fringe_phi_gk0(r.px, py, dp1v, b0) * yf;
            if (pn == py) break;
            py = pn;
        }
        fringe_coeffs_gk0(D3{r.px, 1.0, 0.0, 0.0}, D3{py, 0.0, 1.0, 0.0}, D3{dp1v, 0.0, 0.0, 1.0}, b0, phi, dpx, dpy,
                          dd);
    } else {
        for (int it = 0; it < 12; ++it) {
            const double pn = r.py + fringe_phi(r.px, py, dp1v, b0, gK) * yf;
            if (pn == py) break;
            py = pn;
        }
        fringe_coeffs(D3{r.px, 1.0, 0.0, 0.0}, D3{py, 0.0, 1.0, 0.0}, D3{dp1v, 0.0, 0.0, 1.0}, b0, gK, phi, dpx, dpy,
                      dd);
    }
    const double yf2 = yf * yf;
    r.x = r.x - 0.5 * dpx.v * yf2;
    r.y = yf - 0.5 * dpy.v * yf2;
    r.py = py;
    r.z = r.z + 0.5 * dd.v * yf2;
    // cotangents
    const double den = 1.0 - dpy.v * yf;  // d yf / d y = 1/den, d yf / d dpy = yf^2 / (2 den)
    const double lyf = l.y + l.x * dpx.v * yf - l.py * phi.v - l.z * dd.v * yf;
    const double ly = lyf / den;
    const double ldpy = lyf * 0.5 * yf2 / den;
    const double ldpx = 0.5 * l.x * yf2;
    const double ldd = -0.5 * l.z * yf2;
    const double lphi = -l.py * yf;
    const double lpx = lphi * phi.a + ldpx * dpx.a + ldpy * dpy.a + ldd * dd.a;
    const double lpy = lphi * phi.b + ldpx * dpx.b + ldpy * dpy.b + ldd * dd.b;
    const double ldp1 = lphi * phi.c + ldpx * dpx.c + ldpy * dpy.c + ldd * dd.c;
    l.y = ly;
    l.px = l.px + lpx;
    l.py = l.py + lpy;
    l.d = l.d + ldp1;
}

// exact_bend_body, Forest 12.18 (:858-894), backwards.  cs, sn = cos, sin(irho L).
// The inverse is the same body with -L: on the output (px', py, delta) it
// computes pz' = pxyz(px') and the forward's asin(px'/d2), then the input px,
// its pz and asin(px/d2).  py and delta are unchanged by the body, so d2 is
// fixed, and in a run of bodies without kicks between them the input values of
// one reversed call are the output values of the next one reversed: they are
// carried (RevBody), leaving one asin, one sqrt and one division per call.
struct RevBody {
    double D, d2, id2, ih, pzo, ipzo, aso;
};

__device__ __forceinline__ void rev_body_init(const P6& r, double h, double dp1, RevBody& c) {
    c.D = dp1 * dp1;
    c.d2 = pxyz(c.D, 0.0, r.py);
    c.id2 = 1.0 / c.d2;
    c.ih = 1.0 / h;
    c.pzo = pxyz(c.D, r.px, r.py);
    c.ipzo = 1.0 / c.pzo;
    c.aso = asin_ool(jclamp(r.px * c.id2));
}

__device__ __forceinline__ void rev_body_step(P6& r, L6& l, RevBody& c, double h, double L, double Lbeti, double cs,
                                              double sn, double dp1) {
    const double pxo = r.px;  // forward output px'
    const double pzmxo = c.pzo - (1.0 + r.x * h);
    const double px = pxo * cs - pzmxo * sn;
    const double asi = asin_ool(jclamp(px * c.id2));
    const double dasin = L + (asi - c.aso) * c.ih;  // forward dasin
    const double pz = pxyz(c.D, px, r.py);
    const double ipz = 1.0 / pz;
    r.x = (pz - pzmxo * cs - pxo * sn - 1.0) * c.ih;
    r.px = px;
    r.y = r.y - r.py * dasin;
    r.z = r.z - dp1 * dasin + Lbeti;
    // cotangents at the rebuilt input
    const double lds = (l.y * r.py + l.z * dp1) * c.ih;  // cotangent of (as1 - as2)
    const double lpzo = l.x * c.ih;
    const double lpxn = l.px - (lds + lpzo * pxo) * c.ipzo;
    const double lpzmx = -l.x * cs * c.ih + lpxn * sn;
    const double lpx = l.x * sn * c.ih + (lds - lpzmx * px) * ipz + lpxn * cs;
    const double ld2 = lds * c.id2 * (pxo * c.ipzo - px * ipz);
    const double sq = lpzo * c.ipzo + ld2 * c.id2 + lpzmx * ipz;  // 2 x cotangent of D
    const double lpy = l.py + l.y * dasin - sq * r.py;
    const double ld = l.d + l.z * dasin + dp1 * sq;
    l.x = -h * lpzmx; l.px = lpx; l.py = lpy; l.d = ld;
    c.pzo = pz;
    c.ipzo = ipz;
    c.aso = asi;
}

// Straight body (|irho| < 1e-6): an exact drift with pz = sqrt(dp1^2 - px^2 - py^2).
__device__ __forceinline__ void rev_body_straight(P6& r, L6& l, double L, double Lbeti, double dp1) {
    const double pz2 = dp1 * dp1 - r.px * r.px - r.py * r.py;
    const double pz = pz2 > 0.0 ? sqrt(pz2) : 0.0;
    const double N = L / pz;
    r.x = r.x - r.px * N;
    r.y = r.y - r.py * N;
    r.z = r.z - N * dp1 + Lbeti;
    const double g = l.x * r.px + l.y * r.py + l.z * dp1;
    const double q = g * N / pz2;
    l.px = l.px + l.x * N + q * r.px;
    l.py = l.py + l.y * N + q * r.py;
    l.d = l.d + l.z * N - q * dp1;
}

__device__ __forceinline__ void rev_body_one(P6& r, L6& l, double h, double L, double Lbeti, double cs, double sn,
                                             double beti, bool straight) {
    const double dp1 = beti + r.d;
    if (straight) {
        rev_body_straight(r, l, L, Lbeti, dp1);
        return;
    }
    RevBody c;
    rev_body_init(r, h, dp1, c);
    rev_body_step(r, l, c, h, L, Lbeti, cs, sn, dp1);
}

template <int M>
__device__ __forceinline__ void rev_exact_body_in(P6& r, L6& l, const double* w, const RecHdr& h, double beti) {
    const double irho = w[eb::IRHO];
    const bool straight = h.flags & RF_STRAIGHT;
    if (h.flags & RF_BODY_ONE) {
        rev_body_one(r, l, irho, w[eb::L1], w[eb::L1] * beti, w[eb::CS1], w[eb::SN1], beti, straight);
        return;
    }
    const double L1 = w[eb::L1], L2 = w[eb::L2];
    const double L1b = L1 * beti, L2b = L2 * beti;
    const double cs1 = w[eb::CS1], sn1 = w[eb::SN1], cs2 = w[eb::CS2], sn2 = w[eb::SN2];
    if ((h.flags & RF_NOKICK) && !straight) {
        const double dp1 = beti + r.d;
        RevBody c;
        rev_body_init(r, irho, dp1, c);
#pragma unroll 1
        for (int k = 4 * h.nsteps - 1; k >= 0; --k) {
            const bool outer = ((k & 3) == 0) || ((k & 3) == 3);
            rev_body_step(r, l, c, irho, outer ? L1 : L2, outer ? L1b : L2b, outer ? cs1 : cs2, outer ? sn1 : sn2,
                          dp1);
        }
        return;
    }
    const double K1 = w[eb::K1], K2 = w[eb::K2];
    double pa[M + 1], pb[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { pa[i] = w[eb::PA + i]; pb[i] = w[eb::PB + i]; }
    double gdummy = 0.0;
    for (int st = 0; st < h.nsteps; ++st) {
        rev_body_one(r, l, irho, L1, L1b, cs1, sn1, beti, straight);
        rev_thin_kick<M>(r, l, pa, pb, K1, 0, gdummy);
        rev_body_one(r, l, irho, L2, L2b, cs2, sn2, beti, straight);
        rev_thin_kick<M>(r, l, pa, pb, K2, 0, gdummy);
        rev_body_one(r, l, irho, L2, L2b, cs2, sn2, beti, straight);
        rev_thin_kick<M>(r, l, pa, pb, K1, 0, gdummy);
        rev_body_one(r, l, irho, L1, L1b, cs1, sn1, beti, straight);
    }
}

// The exact bend runs inline in the sweep's element loop, with its body inline
// for order 0 (pure dipoles) and out of line for the others: 6 % off the
// reverse sweep of the DBA gradient.  (In the forward sweep, whose kernels have
// half the registers, the same change cost 3 %.)
template <int M>
__device__ __noinline__ void rev_exact_body(P6& r, L6& l, const double* w, const RecHdr& h, double beti) {
    rev_exact_body_in<M>(r, l, w, h, beti);
}

__device__ __forceinline__ void rev_exact_sbend(P6& r, L6& l, const double* w, const RecHdr& h, double beti) {
    const double irho = w[eb::IRHO];
    const double gk = w[eb::GK];
    if (h.flags & RF_YROT_OUT) rev_yrot(r, l, w[eb::YC_OUT], w[eb::YS_OUT], beti);
    if (h.flags & RF_FRINGE_OUT) rev_bend_fringe(r, l, -irho, gk, beti);
    if (h.flags & RF_EDGE)
        rev_bend_edge(r, l, irho, w[eb::EC_OUT], w[eb::ES_OUT], w[eb::ES2_OUT], w[eb::ETH_OUT], w[eb::ETHH_OUT], beti);
    switch (h.order) {
        case 0: rev_exact_body_in<0>(r, l, w, h, beti); break;
        case 1: rev_exact_body<1>(r, l, w, h, beti); break;
        case 2: rev_exact_body<2>(r, l, w, h, beti); break;
        default: rev_exact_body<3>(r, l, w, h, beti); break;
    }
    if (h.flags & RF_EDGE)
        rev_bend_edge(r, l, irho, w[eb::EC_IN], w[eb::ES_IN], w[eb::ES2_IN], w[eb::ETH_IN], w[eb::ETHH_IN], beti);
    if (h.flags & RF_FRINGE_IN) rev_bend_fringe(r, l, irho, gk, beti);
    if (h.flags & RF_YROT_IN) rev_yrot(r, l, w[eb::YC_IN], w[eb::YS_IN], beti);
}

// ---------------------------------------------------------------------------
// RF cavity (src/tracking.jl:502-518): half drift, energy kick on delta that
// depends on z only, half drift.
// ---------------------------------------------------------------------------
template <bool EXACT>
__device__ __forceinline__ void rev_rf(P6& s, L6& l, const double* w, const RecHdr& h, double beti, double beta2) {
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        rev_drift<EXACT>(s, l, w[rf::LH], w[rf::LH] * beti, c);
    }
    if (h.flags & RF_ENERGY) {
        const double phase = w[rf::W] * ((s.z - w[rf::LAG]) / C_LIGHT) - w[rf::PHILAG];
        s.d = s.d + w[rf::NV] * libm::sin(phase) / beta2;
        l.z = l.z - l.d * w[rf::NV] * libm::cos(phase) * (w[rf::W] / C_LIGHT) / beta2;
    }
    if (h.flags & RF_LPOS) {
        DCache c;
        make_cache(s, beti, c);
        rev_drift<EXACT>(s, l, w[rf::LH], w[rf::LH] * beti, c);
    }
}

// The integrator kinds backwards (the body of a record, without its
// misalignment).  pm: normal-coefficient slot of the strength parameter of
// this entry (0 = not a parameter); g accumulates d/d pb_pm.
template <bool EXACT>
__device__ __forceinline__ bool reverse_core(P6& s, L6& l, const double* rec, const RecHdr& h, double beti,
                                               double beta2, int pm, double& g) {
    const double* w = rec + HDR_WORDS;
    switch (h.kind) {
        case DK_IDENTITY: break;
        case DK_DRIFT: {
            DCache c;
            make_cache(s, beti, c);
            rev_drift<EXACT>(s, l, w[drift::L], w[drift::L] * beti, c);
            break;
        }
        case DK_MULTIPOLE:
            switch (h.order) {
                case 0: rev_multipole<0, EXACT>(s, l, w, h.nsteps, beti, pm, g); break;
                case 1: rev_multipole_body<1, EXACT>(s, l, w, h.nsteps, beti, pm, g); break;
                case 2: rev_multipole_body<2, EXACT>(s, l, w, h.nsteps, beti, pm, g); break;
                default: rev_multipole<3, EXACT>(s, l, w, h.nsteps, beti, pm, g); break;
            }
            break;
        case DK_THIN: {
            double gd = 0.0;
            switch (h.order) {
                case 0: rev_thin_kick<0>(s, l, w + thin::PA, w + thin::PB, 1.0, 0, gd); break;
                case 1: rev_thin_kick<1>(s, l, w + thin::PA, w + thin::PB, 1.0, 0, gd); break;
                case 2: rev_thin_kick<2>(s, l, w + thin::PA, w + thin::PB, 1.0, 0, gd); break;
                default: rev_thin_kick<3>(s, l, w + thin::PA, w + thin::PB, 1.0, 0, gd); break;
            }
            break;
        }
        case DK_SBEND:
            switch (h.order) {
                case 0: rev_sbend<0, EXACT>(s, l, w, h, beti); break;
                case 1: rev_sbend<1, EXACT>(s, l, w, h, beti); break;
                case 2: rev_sbend<2, EXACT>(s, l, w, h, beti); break;
                default: rev_sbend<3, EXACT>(s, l, w, h, beti); break;
            }
            break;
        case DK_EXACT_SBEND: rev_exact_sbend(s, l, w, h, beti); break;
        case DK_RF: rev_rf<EXACT>(s, l, w, h, beti, beta2); break;
        default: return false;
    }
    return true;
}

}  // namespace dev
}  // namespace tp

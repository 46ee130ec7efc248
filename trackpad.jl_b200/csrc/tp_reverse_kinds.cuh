// tp_reverse_kinds.cuh -- reverse maps of the element kinds outside the
// integrator core: Solenoid, Corrector, Translation, YRotation, CrabCavity,
// AccelCavity, LongitudinalRFMap, the two Lorentz boosts, the thin and strong
// Gaussian beams, the two longitudinal wakes, LBend and Wiggler, and the
// misalignment rows (src/tracking.jl:60-67).
//
// As in tp_reverse.cuh each function takes the state after the block and its
// cotangent, rebuilds the state before the block with the block's inverse,
// and pulls the cotangent back through the block at that rebuilt state.
//
// Inverses.  Kicks that depend only on coordinates they leave unchanged
// (Gaussian beams, wakes, cavities, correctors, translations) are undone by
// subtracting the same kick; the Lorentz boosts, the longitudinal RF map and
// the misalignment rows are affine and are inverted exactly (the 6x6 rows by
// the host, pivoted Gauss-Jordan in long double); YRotation(a)^-1 =
// YRotation(-a); the solenoid and LBend bodies are linear in the transverse
// coordinates at fixed delta with unit determinant, and their path-length
// term is recomputed from the rebuilt input; the wiggler's second-order map
// is a product of shears, each undone in reverse order, and its radiation
// kick is inverted by solving the quadratic in 1 + delta.  The crab cavity
// evaluates its kick phase at z BEFORE its first half drift, so that z is
// recovered by a bounded fixed-point iteration.
//
// Pull-backs.  Where the derivative is short it is written out; elsewhere the
// Jacobian columns are taken in forward mode with the one-direction dual
// number Dn, from templated copies of the forward maps that follow the
// operations of tp_maps.cuh one for one (six passes for maps of all six
// coordinates, two for kicks that depend on x and y only, one for kicks of z).
#pragma once
#include "tp_reverse.cuh"

namespace tp {
namespace dev {

// ---------------------------------------------------------------------------
// Dual numbers: value and one tangent.
// ---------------------------------------------------------------------------
struct Dn {
    double v, t;
};
__device__ __forceinline__ Dn operator+(Dn a, Dn b) { return {a.v + b.v, a.t + b.t}; }
__device__ __forceinline__ Dn operator+(Dn a, double b) { return {a.v + b, a.t}; }
__device__ __forceinline__ Dn operator+(double a, Dn b) { return {a + b.v, b.t}; }
__device__ __forceinline__ Dn operator-(Dn a, Dn b) { return {a.v - b.v, a.t - b.t}; }
__device__ __forceinline__ Dn operator-(Dn a, double b) { return {a.v - b, a.t}; }
__device__ __forceinline__ Dn operator-(double a, Dn b) { return {a - b.v, -b.t}; }
__device__ __forceinline__ Dn operator-(Dn a) { return {-a.v, -a.t}; }
__device__ __forceinline__ Dn operator*(Dn a, Dn b) { return {a.v * b.v, a.t * b.v + a.v * b.t}; }
__device__ __forceinline__ Dn operator*(Dn a, double b) { return {a.v * b, a.t * b}; }
__device__ __forceinline__ Dn operator*(double a, Dn b) { return {a * b.v, a * b.t}; }
__device__ __forceinline__ Dn operator/(Dn a, Dn b) {
    const double q = a.v / b.v;
    return {q, (a.t - q * b.t) / b.v};
}
__device__ __forceinline__ Dn operator/(Dn a, double b) { return {a.v / b, a.t / b}; }
__device__ __forceinline__ Dn operator/(double a, Dn b) {
    const double q = a / b.v;
    return {q, -q * b.t / b.v};
}

// The math functions on both scalar types.
__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dn a) { return a.v; }
__device__ __forceinline__ double gsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ Dn gsqrt(Dn a) {
    const double r = sqrt(a.v);
    return {r, a.t / (2.0 * r)};
}
__device__ __forceinline__ double gsin(double a) { return libm::sin(a); }
__device__ __forceinline__ Dn gsin(Dn a) { return {libm::sin(a.v), libm::cos(a.v) * a.t}; }
__device__ __forceinline__ double gcos(double a) { return libm::cos(a); }
__device__ __forceinline__ Dn gcos(Dn a) { return {libm::cos(a.v), -libm::sin(a.v) * a.t}; }
__device__ __forceinline__ double gexp(double a) { return libm::exp(a); }
__device__ __forceinline__ Dn gexp(Dn a) {
    const double e = libm::exp(a.v);
    return {e, e * a.t};
}
__device__ __forceinline__ double gsinh(double a) { return libm::sinh(a); }
__device__ __forceinline__ Dn gsinh(Dn a) { return {libm::sinh(a.v), libm::cosh(a.v) * a.t}; }
__device__ __forceinline__ double gcosh(double a) { return libm::cosh(a); }
__device__ __forceinline__ Dn gcosh(Dn a) { return {libm::cosh(a.v), libm::sinh(a.v) * a.t}; }

template <class T>
struct S6T {
    T x, px, y, py, z, d;
};

// l <- J^T l with J the Jacobian of `f` at `in`, one forward-mode pass per
// input coordinate.
template <class F>
__device__ __forceinline__ void pull_back6(const P6& in, L6& l, const F& f) {
    double nl[6];
#pragma unroll 1
    for (int j = 0; j < 6; ++j) {
        S6T<Dn> s;
        s.x = Dn{in.x, j == 0 ? 1.0 : 0.0};
        s.px = Dn{in.px, j == 1 ? 1.0 : 0.0};
        s.y = Dn{in.y, j == 2 ? 1.0 : 0.0};
        s.py = Dn{in.py, j == 3 ? 1.0 : 0.0};
        s.z = Dn{in.z, j == 4 ? 1.0 : 0.0};
        s.d = Dn{in.d, j == 5 ? 1.0 : 0.0};
        f(s);
        nl[j] = l.x * s.x.t + l.px * s.px.t + l.y * s.y.t + l.py * s.py.t + l.z * s.z.t + l.d * s.d.t;
    }
    l.x = nl[0]; l.px = nl[1]; l.y = nl[2]; l.py = nl[3]; l.z = nl[4]; l.d = nl[5];
}

// Drifts on either scalar type (src/tracking.jl:87-108; survivors have pz2 > 0).
template <bool EXACT, class T>
__device__ __forceinline__ void drift_t(S6T<T>& s, double L, double Lbeti, double beti) {
    const T A = 1.0 + 2.0 * s.d * beti + s.d * s.d;
    const T bd = beti + s.d;
    const T opd = 1.0 + s.d;
    if (EXACT) {
        const T NormL = L / gsqrt(A - s.px * s.px - s.py * s.py);
        s.x = s.x + NormL * s.px;
        s.y = s.y + NormL * s.py;
        s.z = s.z + NormL * bd - Lbeti;
    } else {
        const T NormL = L / opd;
        s.x = s.x + NormL * s.px;
        s.y = s.y + NormL * s.py;
        s.z = s.z + NormL * (s.px * s.px + s.py * s.py) / (2.0 * opd);
    }
}

template <bool EXACT>
__device__ __forceinline__ void drift_inv(P6& s, double L, double beti) {
    DCache c;
    make_cache(s, beti, c);
    drift<EXACT>(s, -L, -(L * beti), c);
}

// ---------------------------------------------------------------------------
// Misalignment rows: forward r1 (r + t1) at the entrance, r2 r + t2 at the
// exit.  inv holds r1^-1 and r2^-1 (column-major, 36 words each).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mat6t(const double* R, L6& l) {  // l <- R^T l
    const double v[6] = {l.x, l.px, l.y, l.py, l.z, l.d};
    double o[6];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double acc = R[j * 6] * v[0];
#pragma unroll
        for (int i = 1; i < 6; ++i) acc = acc + R[j * 6 + i] * v[i];
        o[j] = acc;
    }
    l.x = o[0]; l.px = o[1]; l.y = o[2]; l.py = o[3]; l.z = o[4]; l.d = o[5];
}

static __device__ __noinline__ void rev_mis_exit(const MisalignDev& m, const double* inv, P6& s, L6& l) {
    s.x = s.x - m.t2[0]; s.px = s.px - m.t2[1]; s.y = s.y - m.t2[2];
    s.py = s.py - m.t2[3]; s.z = s.z - m.t2[4]; s.d = s.d - m.t2[5];
    if (m.r2nz) {
        mat6(inv + 36, s);
        mat6t(m.r2, l);
    }
}

static __device__ __noinline__ void rev_mis_entrance(const MisalignDev& m, const double* inv, P6& s, L6& l) {
    if (m.r1nz) {
        mat6(inv, s);
        mat6t(m.r1, l);
    }
    s.x = s.x - m.t1[0]; s.px = s.px - m.t1[1]; s.y = s.y - m.t1[2];
    s.py = s.py - m.t1[3]; s.z = s.z - m.t1[4]; s.d = s.d - m.t1[5];
}

// ---------------------------------------------------------------------------
// Corrector (src/tracking.jl:587-599): px, py kicked by xk, yk over length L.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rev_corrector(P6& s, L6& l, const double* w) {
    const double xk = w[cor::XK], yk = w[cor::YK], L = w[cor::L];
    const double pn = 1.0 / (1.0 + s.d);
    const double NormL = L * pn;
    s.px = s.px - xk;
    s.py = s.py - yk;
    s.x = s.x - NormL * (s.px + xk / 2.0);
    s.y = s.y - NormL * (s.py + yk / 2.0);
    const double A = (xk * xk / 3.0 + yk * yk / 3.0 + s.px * s.px + s.py * s.py + s.px * xk + s.py * yk) / 2.0;
    s.z = s.z - NormL * pn * A;
    // z' = z + L pn^2 A, x' = x + L pn (px + xk/2), d pn/d delta = -pn^2
    const double Lp2 = L * pn * pn;
    const double ux = s.px + xk / 2.0, uy = s.py + yk / 2.0;
    const double lx = l.x, ly = l.y, lz = l.z;
    l.px = l.px + lx * NormL + lz * Lp2 * ux;
    l.py = l.py + ly * NormL + lz * Lp2 * uy;
    l.d = l.d - Lp2 * (lx * ux + ly * uy) - lz * 2.0 * Lp2 * pn * A;
}

// ---------------------------------------------------------------------------
// Translation (src/tracking.jl:1182-1192): x -= dx + ds px/pz, y likewise,
// z += ds (beti + delta)/pz; Translation(dx, dy, ds)^-1 = Translation(-dx, -dy, -ds).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rev_translation(P6& s, L6& l, const double* w, double beti) {
    const double ds = w[trn::DS];
    const double pz2 = 1.0 + 2.0 * s.d * beti + s.d * s.d - s.px * s.px - s.py * s.py;
    const double pz = sqrt(pz2);
    const double bd = beti + s.d;
    s.x = s.x + (w[trn::DX] + ds * s.px / pz);
    s.y = s.y + (w[trn::DY] + ds * s.py / pz);
    s.z = s.z - ds * bd / pz;
    // u = px/pz, v = py/pz, q = bd/pz; dpz = (-px dpx - py dpy + bd dd)/pz
    const double ipz3 = 1.0 / (pz2 * pz);
    const double lx = l.x, ly = l.y, lz = l.z;
    const double du_px = (pz2 + s.px * s.px) * ipz3, du_py = s.px * s.py * ipz3, du_d = -s.px * bd * ipz3;
    const double dv_px = s.px * s.py * ipz3, dv_py = (pz2 + s.py * s.py) * ipz3, dv_d = -s.py * bd * ipz3;
    const double dq_px = bd * s.px * ipz3, dq_py = bd * s.py * ipz3, dq_d = 1.0 / pz - bd * bd * ipz3;
    l.px = l.px - ds * (lx * du_px + ly * dv_px) + ds * lz * dq_px;
    l.py = l.py - ds * (lx * du_py + ly * dv_py) + ds * lz * dq_py;
    l.d = l.d - ds * (lx * du_d + ly * dv_d) + ds * lz * dq_d;
}

// ---------------------------------------------------------------------------
// YRotation (src/tracking.jl:1194-1218).
// ---------------------------------------------------------------------------
template <class T>
static __device__ __noinline__ void yrotation_t(S6T<T>& s, double ca, double sa, double ta, double beti) {
    const T pz = gsqrt(1.0 + 2.0 * s.d * beti + s.d * s.d - s.px * s.px - s.py * s.py);
    const T ptt = 1.0 - ta * s.px / pz;
    const T x_new = s.x / (ca * ptt);
    const T px_new = ca * s.px + sa * pz;
    const T y_new = s.y + ta * s.x * s.py / (pz * ptt);
    const T z_new = s.z + ta * s.x * (beti + s.d) / (pz * ptt);
    s.x = x_new; s.px = px_new; s.y = y_new; s.z = z_new;
}

static __device__ __noinline__ void rev_yrotation(P6& s, L6& l, const double* w, double beti) {
    const double ca = w[yr::CA], sa = w[yr::SA], ta = w[yr::TA];
    S6T<double> r{s.x, s.px, s.y, s.py, s.z, s.d};
    yrotation_t(r, ca, -sa, -ta, beti);
    s.x = r.x; s.px = r.px; s.y = r.y; s.z = r.z;
    pull_back6(s, l, [&](S6T<Dn>& q) { yrotation_t(q, ca, sa, ta, beti); });
}

// ---------------------------------------------------------------------------
// Crab cavity (src/tracking.jl:1531-1547).
// ---------------------------------------------------------------------------
template <bool EXACT, class T>
static __device__ __noinline__ void crab_t(S6T<T>& s, const double* w, bool lpos, double beti) {
    const double volt = w[crab::VOLT], E = w[crab::E], k = w[crab::K];
    const T ang = k * s.z + w[crab::PHI];
    if (lpos) drift_t<EXACT>(s, w[crab::LH], w[crab::LH] * beti, beti);
    const T px_new = s.px + (volt / E) * gsin(ang * beti);
    const T delta_new = s.d - (k * volt / E * beti) * s.x * gcos(ang * beti);
    s.px = px_new;
    s.d = delta_new;
    if (lpos) drift_t<EXACT>(s, w[crab::LH], w[crab::LH] * beti, beti);
}

template <bool EXACT>
static __device__ __noinline__ void rev_crab(P6& s, L6& l, const double* w, const RecHdr& h, double beti) {
    const double volt = w[crab::VOLT], E = w[crab::E], k = w[crab::K], LH = w[crab::LH];
    const bool lpos = (h.flags & RF_LPOS) != 0;
    if (lpos) drift_inv<EXACT>(s, LH, beti);
    // s: after the kick.  The kick phase uses z before the first half drift.
    const P6 a = s;
    double z0 = s.z;
    for (int it = 0; it < 64; ++it) {
        const double ang = k * z0 + w[crab::PHI];
        P6 u = a;
        u.px = a.px - (volt / E) * libm::sin(ang * beti);
        u.d = a.d + (k * volt / E * beti) * a.x * libm::cos(ang * beti);
        if (lpos) drift_inv<EXACT>(u, LH, beti);
        s = u;
        if (!lpos || u.z == z0 || isnan(u.z)) break;
        z0 = u.z;
    }
    pull_back6(s, l, [&](S6T<Dn>& q) { crab_t<EXACT>(q, w, lpos, beti); });
}

// ---------------------------------------------------------------------------
// Accelerating cavity (src/tracking.jl:1549-1559): delta += c (sin(k z + phis) - sin phis).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rev_accel(P6& s, L6& l, const double* w, double beta2) {
    if (beta2 <= EPSD) return;
    const double c = w[acc::VOLT] / (beta2 * w[acc::E]);
    const double arg = w[acc::K] * s.z + w[acc::PHIS];
    s.d = s.d - c * (libm::sin(arg) - w[acc::SINPHIS]);
    l.z = l.z + l.d * c * w[acc::K] * libm::cos(arg);
}

// LongitudinalRFMap (src/tracking.jl:1575-1585): z -= c delta.
__device__ __forceinline__ void rev_long_rf_map(P6& s, L6& l, const double* w, double beta) {
    const double eta = w[lrf::ALPHAC] - (1.0 - beta * beta);
    const double c = 6.283185307179586 * w[lrf::H] * eta / w[lrf::K];
    s.z = s.z + c * s.d;
    l.d = l.d - c * l.z;
}

// Lorentz boost: x' = x + ta z, px' = px ic, py' = py ic, z' = z ic, d' = d - ta px.
__device__ __forceinline__ void rev_lorentz(P6& s, L6& l, const double* w) {
    const double ic = w[lor::A], ta = w[lor::B];
    s.px = s.px / ic;
    s.py = s.py / ic;
    s.z = s.z / ic;
    s.x = s.x - ta * s.z;
    s.d = s.d + ta * s.px;
    l.px = l.px * ic - l.d * ta;
    l.py = l.py * ic;
    l.z = l.z * ic + l.x * ta;
}

// Inverse boost: x' = x - sa z, px' = px ca, py' = py ca, z' = z ca, d' = d + sa px.
__device__ __forceinline__ void rev_inv_lorentz(P6& s, L6& l, const double* w) {
    const double ca = w[lor::A], sa = w[lor::B];
    s.px = s.px / ca;
    s.py = s.py / ca;
    s.z = s.z / ca;
    s.x = s.x + sa * s.z;
    s.d = s.d - sa * s.px;
    l.px = l.px * ca + l.d * sa;
    l.py = l.py * ca;
    l.z = l.z * ca - l.x * sa;
}

// ---------------------------------------------------------------------------
// Gaussian beam-beam kicks (src/tracking.jl:1610-1641): px, py kicked by
// functions of x and y.
// ---------------------------------------------------------------------------
template <class T>
static __device__ __noinline__ void stg_kick_t(const double* w, T x, T y, T& kx, T& ky) {
    const T dx = x - w[stg::XO];
    const T dy = y - w[stg::YO];
    const T g = w[stg::AMP] * gexp(-0.5 * (dx * dx / w[stg::SX2] + dy * dy / w[stg::SY2]));
    kx = g * dx / w[stg::SX2];
    ky = g * dy / w[stg::SY2];
}

template <class T>
static __device__ __noinline__ void sgb_kick_t(const double* w, T x, T y, T& kx, T& ky) {
    const int nz = int(w[sgb::NZ]);
    const double* wt = w + sgb::WORDS;
    const double factor = w[sgb::FACTOR], sx2 = w[sgb::SX2], sy2 = w[sgb::SY2];
    kx = T{};
    ky = T{};
    for (int i = 0; i < nz; ++i) {
        const T dx = x - wt[nz + i];
        const T dy = y - wt[2 * nz + i];
        const T g = wt[i] * gexp(-0.5 * (dx * dx / sx2 + dy * dy / sy2));
        kx = kx + factor * g * dx / sx2;
        ky = ky + factor * g * dy / sy2;
    }
}

// px' = px - kx(x, y), py' = py - ky(x, y).
template <bool SGB>
static __device__ __noinline__ void rev_gauss_kick(P6& s, L6& l, const double* w) {
    double kx, ky;
    if (SGB) sgb_kick_t(w, s.x, s.y, kx, ky);
    else stg_kick_t(w, s.x, s.y, kx, ky);
    s.px = s.px + kx;
    s.py = s.py + ky;
    Dn ax, ay, bx, by;
    if (SGB) {
        sgb_kick_t(w, Dn{s.x, 1.0}, Dn{s.y, 0.0}, ax, ay);
        sgb_kick_t(w, Dn{s.x, 0.0}, Dn{s.y, 1.0}, bx, by);
    } else {
        stg_kick_t(w, Dn{s.x, 1.0}, Dn{s.y, 0.0}, ax, ay);
        stg_kick_t(w, Dn{s.x, 0.0}, Dn{s.y, 1.0}, bx, by);
    }
    l.x = l.x - l.px * ax.t - l.py * ay.t;
    l.y = l.y - l.px * bx.t - l.py * by.t;
}

// ---------------------------------------------------------------------------
// Longitudinal wakes (src/tracking.jl:1647-1663): delta -= scale W(z).
// ---------------------------------------------------------------------------
template <class T>
static __device__ __noinline__ T rlc_wf_t(const double* w, T z) {
    const T zc = z / C_LIGHT;
    const T t = isnan(val(zc)) ? zc : (val(zc) > 0.0 ? T{} : zc);
    T wf{};
    if (!(val(t) > 0.0))
        wf = w[rlc::A] * (gcos(w[rlc::W0P] * t) + gsin(w[rlc::W0P] * t) / w[rlc::D2Q0P]) *
             gexp(w[rlc::W0] * t / w[rlc::D2Q0]);
    return wf;
}

template <class T>
static __device__ __noinline__ T tab_wf_t(const double* w, const RecHdr& h, T z) {
    const int n = int(w[tw::N]);
    const double* xs = w + tw::WORDS;
    const double* ys = xs + n;
    const T t = z / C_LIGHT;
    T wf{};
    if (!(val(t) > w[tw::T1F])) {
        const T x = t * w[tw::FLIP];
        const double xv = val(x);
        if (xv <= xs[0]) {
            const double slope = (ys[1] - ys[0]) / (xs[1] - xs[0]);
            wf = ys[0] + slope * (x - xs[0]);
        } else if (xv >= xs[n - 1]) {
            const double slope = (ys[n - 1] - ys[n - 2]) / (xs[n - 1] - xs[n - 2]);
            wf = ys[n - 1] + slope * (x - xs[n - 1]);
        } else if (isnan(xv)) {
            wf = T{} + ys[n - 1];
        } else {
            int i = 1;
            if (h.order == 1) {
                int lo = 1, hi = n - 1;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (xv < xs[mid]) hi = mid; else lo = mid + 1;
                }
                i = lo;
            } else {
                while (i < n - 1 && !(xv < xs[i])) ++i;
            }
            if (xv < xs[i]) {
                const double slope = (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1]);
                wf = ys[i - 1] + slope * (x - xs[i - 1]);
            } else {
                wf = T{} + ys[n - 1];
            }
        }
    }
    return wf;
}

template <bool TAB>
static __device__ __noinline__ void rev_wake(P6& s, L6& l, const double* w, const RecHdr& h) {
    const double scale = TAB ? w[tw::SCALE] : w[rlc::SCALE];
    const Dn wf = TAB ? tab_wf_t(w, h, Dn{s.z, 1.0}) : rlc_wf_t(w, Dn{s.z, 1.0});
    s.d = s.d + scale * wf.v;
    l.z = l.z - l.d * scale * wf.t;
}

// ---------------------------------------------------------------------------
// Solenoid (src/tracking.jl:537-562): a rotation-focusing matrix in
// (x, px/(1+d), y, py/(1+d)) and a path-length term conserved along the body.
// ---------------------------------------------------------------------------
template <bool EXACT, class T>
static __device__ __noinline__ void solenoid_t(S6T<T>& s, const double* w, double beti) {
    const double ks = w[sol::KS];
    const double L = w[sol::L];
    if (ks == 0.0) {
        drift_t<EXACT>(s, L, L * beti, beti);
        return;
    }
    const T p_norm = 1.0 / (1.0 + s.d);
    const T x = s.x, xpr = s.px * p_norm, y = s.y, ypr = s.py * p_norm;
    const T H = ks * p_norm / 2.0;
    const T S = gsin(L * H);
    const T C = gcos(L * H);
    const T x_new = x * C * C + xpr * C * S / H + y * C * S + ypr * S * S / H;
    const T px_new = (-x * H * C * S + xpr * C * C - y * H * S * S + ypr * C * S) / p_norm;
    const T y_new = -x * C * S - xpr * S * S / H + y * C * C + ypr * C * S / H;
    const T py_new = (x * H * S * S - xpr * C * S - y * C * S * H + ypr * C * C) / p_norm;
    const T z_new = s.z + L * (H * H * (x * x + y * y) + 2.0 * H * (xpr * y - ypr * x) + xpr * xpr + ypr * ypr) / 2.0;
    s.x = x_new; s.px = px_new; s.y = y_new; s.py = py_new; s.z = z_new;
}

template <bool EXACT>
static __device__ __noinline__ void rev_solenoid(P6& s, L6& l, const double* w, double beti) {
    const double ks = w[sol::KS];
    const double L = w[sol::L];
    if (ks == 0.0) {
        DCache c;
        make_cache(s, beti, c);
        rev_drift<EXACT>(s, l, L, L * beti, c);
        return;
    }
    // transverse: the same matrix with -L (its inverse); z: the conserved
    // quadratic form at the rebuilt input
    const double p_norm = 1.0 / (1.0 + s.d);
    const double x = s.x, xpr = s.px * p_norm, y = s.y, ypr = s.py * p_norm;
    const double H = ks * p_norm / 2.0;
    const double S = -libm::sin(L * H);
    const double C = libm::cos(L * H);
    const double xi = x * C * C + xpr * C * S / H + y * C * S + ypr * S * S / H;
    const double xpri = -x * H * C * S + xpr * C * C - y * H * S * S + ypr * C * S;
    const double yi = -x * C * S - xpr * S * S / H + y * C * C + ypr * C * S / H;
    const double ypri = x * H * S * S - xpr * C * S - y * C * S * H + ypr * C * C;
    s.x = xi; s.px = xpri / p_norm; s.y = yi; s.py = ypri / p_norm;
    s.z = s.z - L * (H * H * (xi * xi + yi * yi) + 2.0 * H * (xpri * yi - ypri * xi) + xpri * xpri + ypri * ypri) / 2.0;
    pull_back6(s, l, [&](S6T<Dn>& q) { solenoid_t<EXACT>(q, w, beti); });
}

// ---------------------------------------------------------------------------
// LBend (src/tracking.jl:1076-1170): method-1 edges around a linear
// combined-function body.
// ---------------------------------------------------------------------------
// Body coefficients at fixed delta.
template <class T>
struct LbCoefT {
    T MHD, M12, M21, MVD, M34, M43, G1, G2, arg1, sqrtG1, p_norm, dterm;
    bool big1;
};

template <class T>
static __device__ __noinline__ void lb_coef_t(const double* w, T d, LbCoefT<T>& c) {
    const double L = w[lb::L];
    c.p_norm = 1.0 / (1.0 + d);
    c.G1 = w[lb::G1C] * c.p_norm;
    c.G2 = w[lb::NGRD] * c.p_norm;
    const double tol = 1.4901161193847656e-08;
    c.MHD = T{} + 1.0; c.M12 = T{} + L; c.M21 = T{}; c.MVD = T{} + 1.0; c.M34 = T{} + L; c.M43 = T{};
    c.arg1 = T{};
    c.sqrtG1 = T{};
    c.big1 = fabs(val(c.G1)) >= tol;
    if (c.big1) {
        if (val(c.G1) > 0.0) {
            c.sqrtG1 = gsqrt(c.G1);
            c.arg1 = L * c.sqrtG1;
            c.MHD = gcos(c.arg1); c.M12 = gsin(c.arg1) / c.sqrtG1; c.M21 = -gsin(c.arg1) * c.sqrtG1;
        } else {
            c.sqrtG1 = gsqrt(-c.G1);
            c.arg1 = L * c.sqrtG1;
            c.MHD = gcosh(c.arg1); c.M12 = gsinh(c.arg1) / c.sqrtG1; c.M21 = gsinh(c.arg1) * c.sqrtG1;
        }
    }
    if (fabs(val(c.G2)) >= tol) {
        if (val(c.G2) > 0.0) {
            const T sq = gsqrt(c.G2), arg2 = L * sq;
            c.MVD = gcos(arg2); c.M34 = gsin(arg2) / sq; c.M43 = -gsin(arg2) * sq;
        } else {
            const T sq = gsqrt(-c.G2), arg2 = L * sq;
            c.MVD = gcosh(arg2); c.M34 = gsinh(arg2) / sq; c.M43 = gsinh(arg2) * sq;
        }
    }
    c.dterm = d * c.p_norm - w[lb::BYERR];
}

// Dispersion terms of x and px.
template <class T>
static __device__ __noinline__ void lb_disp_t(const double* w, const LbCoefT<T>& c, T& Dx, T& Dpx) {
    const double kx = w[lb::KX], L = w[lb::L];
    const double tol = 1.4901161193847656e-08;
    if (fabs(val(c.G1)) < tol) {
        Dx = c.dterm * L * L * kx / 2.0;
        Dpx = c.dterm * L * kx / c.p_norm;
    } else if (val(c.G1) > 0.0) {
        Dx = c.dterm * (1.0 - gcos(c.arg1)) * kx / c.G1;
        Dpx = c.dterm * gsin(c.arg1) * kx / (c.sqrtG1 * c.p_norm);
    } else {
        Dx = c.dterm * (1.0 - gcosh(c.arg1)) * kx / c.G1;
        Dpx = c.dterm * gsinh(c.arg1) * kx / (c.sqrtG1 * c.p_norm);
    }
}

// Path-length increment at the body input (x, xpr, y, ypr).
template <class T>
static __device__ __noinline__ T lb_dz_t(const double* w, const LbCoefT<T>& c, T x, T xpr, T y, T ypr) {
    const double kx = w[lb::KX], L = w[lb::L];
    T dz = xpr * xpr * (L + c.MHD * c.M12) / 4.0;
    if (c.big1) {
        dz = dz + (L - c.MHD * c.M12) * (x * x * c.G1 + c.dterm * c.dterm * kx * kx / c.G1 - 2.0 * x * kx * c.dterm) / 4.0;
        dz = dz + c.M12 * c.M21 * (x * xpr - xpr * c.dterm * kx / c.G1) / 2.0;
        dz = dz + (kx * x * c.M12 + xpr * (1.0 - c.MHD) * kx / c.G1 + c.dterm * (L - c.M12) * kx * kx / c.G1);
    }
    dz = dz + ((L - c.MVD * c.M34) * y * y * c.G2 + ypr * ypr * (L + c.MVD * c.M34)) / 4.0;
    dz = dz + c.M34 * c.M43 * y * ypr / 2.0;
    return dz;
}

template <class T>
static __device__ __noinline__ void lbend_body_t(S6T<T>& s, const double* w) {
    LbCoefT<T> c;
    lb_coef_t(w, s.d, c);
    const T x = s.x, xpr = s.px * c.p_norm, y = s.y, ypr = s.py * c.p_norm;
    T Dx, Dpx;
    lb_disp_t(w, c, Dx, Dpx);
    const T x_new = c.MHD * x + c.M12 * xpr + Dx;
    const T px_new = (c.M21 * x + c.MHD * xpr) / c.p_norm + Dpx;
    const T y_new = c.MVD * y + c.M34 * ypr;
    const T py_new = (c.M43 * y + c.MVD * ypr) / c.p_norm;
    const T z_new = s.z + lb_dz_t(w, c, x, xpr, y, ypr);
    s.x = x_new; s.px = px_new; s.y = y_new; s.py = py_new; s.z = z_new;
}

static __device__ __noinline__ void rev_lbend(P6& s, L6& l, const double* w, const RecHdr& h) {
    rev_edge_fringe(s, l, w[lb::IRHO], w[lb::FX_OUT], w[lb::E_OUT], w[lb::FC_OUT], 1, h.flags & RF_FC_OUT_ZERO, true);
    {
        LbCoefT<double> c;
        lb_coef_t(w, s.d, c);
        double Dx, Dpx;
        lb_disp_t(w, c, Dx, Dpx);
        // unit-determinant 2x2 blocks: [[a, b], [c, a]]^-1 = [[a, -b], [-c, a]]
        const double X = s.x - Dx, P = (s.px - Dpx) * c.p_norm;
        const double x = c.MHD * X - c.M12 * P, xpr = c.MHD * P - c.M21 * X;
        const double Y = s.y, Q = s.py * c.p_norm;
        const double y = c.MVD * Y - c.M34 * Q, ypr = c.MVD * Q - c.M43 * Y;
        s.z = s.z - lb_dz_t(w, c, x, xpr, y, ypr);
        s.x = x; s.px = xpr / c.p_norm; s.y = y; s.py = ypr / c.p_norm;
    }
    pull_back6(s, l, [&](S6T<Dn>& q) { lbend_body_t(q, w); });
    rev_edge_fringe(s, l, w[lb::IRHO], w[lb::FX_IN], w[lb::E_IN], w[lb::FC_IN], 1, h.flags & RF_FC_IN_ZERO, false);
}

// ---------------------------------------------------------------------------
// Wiggler (src/tracking.jl:1224-1529).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T sinc_taylor_t(T x) {
    const T x2 = x * x;
    return 1.0 - x2 / 6.0 * (1.0 - x2 / 20.0 * (1.0 - x2 / 42.0 * (1.0 - x2 / 72.0)));
}

template <class T>
static __device__ __noinline__ void wig_ax_axpy_t(const double* w, T x, T y, double Zw, T& ax, T& axpy) {
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    ax = T{};
    axpy = T{};
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T cx = gcos(kx * x), chy = gcosh(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ax = ax + hp[wg::C_AX] * cx * chy * sz;
        const T shy = gsinh(ky * y);
        const T sxkx = hp[wg::SINC] != 0.0 ? gsin(kx * x) / kx : x * sinc_taylor_t(kx * x);
        axpy = axpy + hp[wg::C_AXPY] * sxkx * shy * sz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T shx = gsinh(kx * x), sy = gsin(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ax = ax + hp[wg::C_AX] * shx * sy * sz;
        const T chx = gcosh(kx * x), cy = gcos(ky * y);
        axpy = axpy + hp[wg::C_AXPY] * chx * cy * sz;
    }
}

template <class T>
static __device__ __noinline__ void wig_ay_aypx_t(const double* w, T x, T y, double Zw, T& ay, T& aypx) {
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    ay = T{};
    aypx = T{};
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T sx = gsin(kx * x), shy = gsinh(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ay = ay + hp[wg::C_AY] * sx * shy * sz;
        const T cx = gcos(kx * x), chy = gcosh(ky * y);
        aypx = aypx + hp[wg::C_AYPX] * cx * chy * sz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T chx = gcosh(kx * x), cy = gcos(ky * y);
        const double sz = libm::sin(hp[wg::KZ] * Zw + hp[wg::TZ]);
        ay = ay + hp[wg::C_AY] * chx * cy * sz;
        const T shx = gsinh(kx * x);
        const T syky = hp[wg::SINC] != 0.0 ? gsin(ky * y) / ky : y * sinc_taylor_t(ky * y);
        aypx = aypx + hp[wg::C_AYPX] * shx * syky * sz;
    }
}

template <class T>
static __device__ __noinline__ void wig_map_2nd_t(S6T<T>& s, const double* w, double dl, double dl2, double& Zw) {
    const T inv1pd = 1.0 / (1.0 + s.d);
    const T dld = dl * inv1pd;
    const T dl2d = dl2 * inv1pd;
    Zw = Zw + dl2;
    T a, ap;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.y = s.y + dl2d * s.py;
    s.z = s.z + (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    wig_ax_axpy_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - a;
    s.py = s.py - ap;
    s.x = s.x + dld * s.px;
    s.z = s.z + (dld / 2.0) * (s.px * s.px) * inv1pd;
    wig_ax_axpy_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + a;
    s.py = s.py + ap;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.y = s.y + dl2d * s.py;
    s.z = s.z + (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    Zw = Zw + dl2;
}

// Inverse of wig_map_2nd: Zw is the position after the map on entry and
// before it on return.
static __device__ __noinline__ void wig_map_2nd_inv(P6& s, const double* w, double dl, double dl2, double& Zw) {
    const double inv1pd = 1.0 / (1.0 + s.d);
    const double dld = dl * inv1pd;
    const double dl2d = dl2 * inv1pd;
    Zw = Zw - dl2;
    double a, ap;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.z = s.z - (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    s.y = s.y - dl2d * s.py;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    wig_ax_axpy_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - a;
    s.py = s.py - ap;
    s.z = s.z - (dld / 2.0) * (s.px * s.px) * inv1pd;
    s.x = s.x - dld * s.px;
    wig_ax_axpy_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + a;
    s.py = s.py + ap;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px - ap;
    s.py = s.py - a;
    s.z = s.z - (dl2d / 2.0) * (s.py * s.py) * inv1pd;
    s.y = s.y - dl2d * s.py;
    wig_ay_aypx_t(w, s.x, s.y, Zw, a, ap);
    s.px = s.px + ap;
    s.py = s.py + a;
    Zw = Zw - dl2;
}

// Transverse field at (x, y, Zw) (the B part of wig_rad_block).
static __device__ __noinline__ double wig_b2(const double* w, double x, double y, double Zw) {
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    double Bxv = 0.0, Byv = 0.0;
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double sx = libm::sin(kx * x), cx = libm::cos(kx * x);
        const double chy = libm::cosh(ky * y), shy = libm::sinh(ky * y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * sx * shy * cz;
        Byv = Byv - hp[wg::B_Y] * cx * chy * cz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const double shx = libm::sinh(kx * x), chx = libm::cosh(kx * x);
        const double sy = libm::sin(ky * y), cy = libm::cos(ky * y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * chx * cy * cz;
        Byv = Byv - hp[wg::B_Y] * shx * sy * cz;
    }
    return Bxv * Bxv + Byv * Byv;
}

template <class T>
static __device__ __noinline__ void wig_rad_block_t(S6T<T>& s, const double* w, double Zw) {
    T ax, axpy, ay, aypx;
    wig_ax_axpy_t(w, s.x, s.y, Zw, ax, axpy);
    wig_ay_aypx_t(w, s.x, s.y, Zw, ay, aypx);
    s.px = s.px - ax;
    s.py = s.py - ay;
    const int nh = int(w[wg::NH]), nv = int(w[wg::NV]);
    const double* hp = w + wg::WORDS;
    T Bxv{}, Byv{};
    for (int i = 0; i < nh; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T sx = gsin(kx * s.x), cx = gcos(kx * s.x);
        const T chy = gcosh(ky * s.y), shy = gsinh(ky * s.y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * sx * shy * cz;
        Byv = Byv - hp[wg::B_Y] * cx * chy * cz;
    }
    for (int i = 0; i < nv; ++i, hp += wg::HWORDS) {
        const double kx = hp[wg::KX], ky = hp[wg::KY];
        const T shx = gsinh(kx * s.x), chx = gcosh(kx * s.x);
        const T sy = gsin(ky * s.y), cy = gcos(ky * s.y);
        const double cz = libm::cos(hp[wg::KZ] * Zw + hp[wg::TZ]);
        Bxv = Bxv + hp[wg::B_X] * chx * cy * cz;
        Byv = Byv - hp[wg::B_Y] * shx * sy * cz;
    }
    const T B2 = Bxv * Bxv + Byv * Byv;
    if (val(B2) != 0.0) {
        const T irho2 = B2 / w[wg::HH];
        const T dFactor = (1.0 + s.d) * (1.0 + s.d);
        const T dDelta = -w[wg::SRCOEF] * dFactor * irho2 * w[wg::SL];
        const T scale = 1.0 + dDelta;
        s.px = s.px * scale;
        s.py = s.py * scale;
        s.d = s.d + dDelta;
    }
    s.px = s.px + ax;
    s.py = s.py + ay;
}

// Inverse of the radiation block: with u = 1 + delta and c = srcoef irho2 sl,
// the block maps u to u' = u - c u^2; the root near u' is 2u'/(1 + sqrt(1 - 4cu')).
static __device__ __noinline__ void wig_rad_block_inv(P6& s, const double* w, double Zw) {
    double ax, axpy, ay, aypx;
    wig_ax_axpy_t(w, s.x, s.y, Zw, ax, axpy);
    wig_ay_aypx_t(w, s.x, s.y, Zw, ay, aypx);
    s.px = s.px - ax;
    s.py = s.py - ay;
    const double B2 = wig_b2(w, s.x, s.y, Zw);
    if (B2 != 0.0) {
        const double c = w[wg::SRCOEF] * (B2 / w[wg::HH]) * w[wg::SL];
        const double up = 1.0 + s.d;
        const double u = 2.0 * up / (1.0 + sqrt(1.0 - 4.0 * c * up));
        const double dDelta = -c * (u * u);
        const double scale = 1.0 + dDelta;
        s.d = s.d - dDelta;
        s.px = s.px / scale;
        s.py = s.py / scale;
    }
    s.px = s.px + ax;
    s.py = s.py + ay;
}

template <class T>
static __device__ __noinline__ void wiggler_t(S6T<T>& s, const double* w) {
    const long long nstep = (long long)w[wg::NSTEP];
    const double dl1 = w[wg::DL1], dl0 = w[wg::DL0], dl1h = w[wg::DL1H], dl0h = w[wg::DL0H];
    const bool rad = w[wg::RAD] == 1.0;
    double Zw = 0.0;
    if (rad) wig_rad_block_t(s, w, Zw);
    for (long long k = 0; k < nstep; ++k) {
        wig_map_2nd_t(s, w, dl1, dl1h, Zw);
        wig_map_2nd_t(s, w, dl0, dl0h, Zw);
        wig_map_2nd_t(s, w, dl1, dl1h, Zw);
        if (rad) wig_rad_block_t(s, w, Zw);
    }
}

static __device__ __noinline__ void rev_wiggler(P6& s, L6& l, const double* w) {
    const long long nstep = (long long)w[wg::NSTEP];
    const double dl1 = w[wg::DL1], dl0 = w[wg::DL0], dl1h = w[wg::DL1H], dl0h = w[wg::DL0H];
    const bool rad = w[wg::RAD] == 1.0;
    // the forward positions along the wiggler, in the forward's own sums
    double Zend = 0.0;
    for (long long k = 0; k < nstep; ++k) {
        Zend = Zend + dl1h; Zend = Zend + dl1h;
        Zend = Zend + dl0h; Zend = Zend + dl0h;
        Zend = Zend + dl1h; Zend = Zend + dl1h;
    }
    double Zw = Zend;
    for (long long k = nstep - 1; k >= 0; --k) {
        if (rad) wig_rad_block_inv(s, w, Zw);
        wig_map_2nd_inv(s, w, dl1, dl1h, Zw);
        wig_map_2nd_inv(s, w, dl0, dl0h, Zw);
        wig_map_2nd_inv(s, w, dl1, dl1h, Zw);
    }
    if (rad) wig_rad_block_inv(s, w, 0.0);
    pull_back6(s, l, [&](S6T<Dn>& q) { wiggler_t(q, w); });
}

// ---------------------------------------------------------------------------
// One lattice entry backwards, misalignment rows included.  mis/misinv: the
// rows and their inverses (72 words per row: r1^-1, r2^-1).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr bool reverse_supported(int kind) { return kind >= 0 && kind < DK_COUNT; }

// The non-core kinds, out of line: one call site in the reverse sweep's loop.
template <bool EXACT>
static __device__ __noinline__ bool reverse_rare(P6& s, L6& l, const double* w, const RecHdr& h, double beti,
                                                 double beta, double beta2) {
    switch (h.kind) {
        case DK_SOLENOID: rev_solenoid<EXACT>(s, l, w, beti); break;
        case DK_CORRECTOR: rev_corrector(s, l, w); break;
        case DK_TRANSLATION: rev_translation(s, l, w, beti); break;
        case DK_YROTATION: rev_yrotation(s, l, w, beti); break;
        case DK_CRAB: rev_crab<EXACT>(s, l, w, h, beti); break;
        case DK_ACCEL: rev_accel(s, l, w, beta2); break;
        case DK_LONG_RF_MAP: rev_long_rf_map(s, l, w, beta); break;
        case DK_LORENTZ: rev_lorentz(s, l, w); break;
        case DK_INV_LORENTZ: rev_inv_lorentz(s, l, w); break;
        case DK_STRONG_THIN_GAUSS: rev_gauss_kick<false>(s, l, w); break;
        case DK_SGB: rev_gauss_kick<true>(s, l, w); break;
        case DK_RLC_WAKE: rev_wake<false>(s, l, w, h); break;
        case DK_TAB_WAKE: rev_wake<true>(s, l, w, h); break;
        case DK_LBEND: rev_lbend(s, l, w, h); break;
        case DK_WIGGLER: rev_wiggler(s, l, w); break;
        case DK_NAN: set_nan(s); break;  // no particle survives it
        default: return false;
    }
    return true;
}

// RARE = false: tables of core kinds without misalignment rows (the reverse
// sweep is then the integrator core alone).
template <bool EXACT, bool RARE = true>
__device__ __forceinline__ bool reverse_record(P6& s, L6& l, const double* rec, const RecHdr& h,
                                               const MisalignDev* mis, const double* misinv, double beti,
                                               double beta, double beta2, int pm, double& g) {
    if (!RARE) return reverse_core<EXACT>(s, l, rec, h, beti, beta2, pm, g);
    const bool misal = (h.flags & RF_MISALIGN) != 0;
    if (misal) rev_mis_exit(mis[h.aux], misinv + 72 * int64_t(h.aux), s, l);
    const bool ok = h.kind <= DK_RF ? reverse_core<EXACT>(s, l, rec, h, beti, beta2, pm, g)
                                    : reverse_rare<EXACT>(s, l, rec + HDR_WORDS, h, beti, beta, beta2);
    if (misal) rev_mis_entrance(mis[h.aux], misinv + 72 * int64_t(h.aux), s, l);
    return ok;
}

}  // namespace dev
}  // namespace tp

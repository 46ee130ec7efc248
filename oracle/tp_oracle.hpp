// tp_oracle.hpp -- CPU oracle for the TrackPad.jl tracking path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product: only
// the tests, the smoke check and the CPU-baseline leg of the benchmark load it.
// The shipped library does not include, link or call anything in oracle/.
//
// What it is: a line-by-line C++17 restatement of the reference's per-particle
// maps (TrackPad.jl src/tracking.jl) and of its multi-particle drivers
// (src/lattice.jl:260-317), in the reference's own operation order:
//   * x^2 is written x*x (Julia's literal_pow for Float64),
//   * n-ary a+b+c and a*b*c are left folds, as Julia evaluates them,
//   * it is compiled with -ffp-contract=off and no fast-math, so no FMA.
// Every function cites the reference lines it restates.  The scalar type T is a
// template parameter so the same restatement also runs with an op-counting type
// (the algorithmic FLOP table) and with forward-mode dual numbers (Jacobians and
// strength gradients).
//
// Parity status: UNPINNED against reference outputs.  The reference is Julia,
// which is not installed here, and its tests compare live against JuTrack (not
// vendored); it stores no golden vectors.  The restatement is instead checked
// against an independent pure-Python transcription of the same Julia source
// (tests/golden/make_golden.py, bit-exact on the reference's own 10-particle
// parity fixture and test lattices), against analytic limits, symplecticity of
// its Jacobians and time reversibility.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#include "../include/trackpad_b200.h"
#include "../trackpad.jl_b200/csrc/tp_libm.h"

namespace tpo {

// ---------------------------------------------------------------------------
// Constants: src/tracking.jl:25-32, src/elements/rf.jl:28, src/lattice.jl:42
// ---------------------------------------------------------------------------
constexpr double COORD_LIMIT = 1.0;
constexpr double ANGLE_LIMIT = 1.0;
constexpr double DRIFT1 = 0.6756035959798286638;
constexpr double DRIFT2 = -0.1756035959798286639;
constexpr double KICK1 = 1.351207191959657328;
constexpr double KICK2 = -1.702414383919314656;
constexpr double C_LIGHT = 2.99792458e8;
constexpr double M_ELECTRON = 0.51099895069e6;
constexpr double TWO_PI = 6.283185307179586;  // Float64(2pi)
constexpr double EPS = 2.220446049250313e-16; // eps(Float64)

// Scalar helpers.  sin, cos, tan, asin, atan, exp, sinh and cosh of a double come from
// tp_libm.h: the published fdlibm method in explicitly rounded IEEE operations,
// the implementation the CUDA kernels use, so that the oracle and the device
// evaluate the same function (both within 1 ulp of the C library).  Other
// scalar types provide overloads found by argument-dependent lookup.
inline double value_of(double x) { return x; }
inline bool is_nan(double x) { return std::isnan(x); }
inline double sin(double x) { return tp::libm::sin(x); }
inline double cos(double x) { return tp::libm::cos(x); }
inline double tan(double x) { return tp::libm::tan(x); }
inline double asin(double x) { return tp::libm::asin(x); }
inline double atan(double x) { return tp::libm::atan(x); }
inline double exp(double x) { return tp::libm::exp(x); }
inline double expm1(double x) { return tp::libm::expm1(x); }
inline double sinh(double x) { return tp::libm::sinh(x); }
inline double cosh(double x) { return tp::libm::cosh(x); }

// Truncated power series (tp_tpsa_oracle.hpp) specialise this: the TPSA
// extension (ext/TrackPadPolySeriesExt.jl) tracks with the same pass! bodies
// except for an always-exact drift, bend edges whose fy uses the constant
// parts of delta and px, and wakes evaluated at the constant part of z.
template <class T>
struct is_tps : std::false_type {};

template <class T>
struct V6 {
    T v[6];
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
};

template <class T>
inline V6<T> nan6() {
    const double q = std::numeric_limits<double>::quiet_NaN();
    return V6<T>{{T(q), T(q), T(q), T(q), T(q), T(q)}};
}

// Element with the reference struct fields (superset over kinds).
template <class T>
struct Elem {
    int kind = TP_MARKER;
    int max_order = 0, num_int_steps = 0;
    int fbe = 0, fbx = 0;
    int iparam[2] = {0, 0};
    T L = T(0.0), k = T(0.0), angle = T(0.0), e1 = T(0.0), e2 = T(0.0);
    T fint1 = T(0.0), fint2 = T(0.0), gap = T(0.0), gk = T(0.0);
    T pa[4] = {T(0.0), T(0.0), T(0.0), T(0.0)};
    T pb[4] = {T(0.0), T(0.0), T(0.0), T(0.0)};
    T kick[2] = {T(0.0), T(0.0)};
    T volt = T(0.0), freq = T(0.0), h = T(0.0), lag = T(0.0), philag = T(0.0), energy = T(0.0);
    T param[8] = {T(0.0), T(0.0), T(0.0), T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
    bool has_mis = false, r1nz = false, r2nz = false;
    T t1[6], t2[6], r1[36], r2[36];
    const double* aux = nullptr;  // the element's array fields (aux + iparam[0]), iparam[1] words
};

template <class T>
Elem<T> make_elem(const tp_elem& e, const tp_misalign* mis, const double* aux = nullptr) {
    Elem<T> o;
    o.aux = aux ? aux + e.iparam[0] : nullptr;
    o.kind = e.kind;
    o.max_order = e.max_order;
    o.num_int_steps = e.num_int_steps;
    o.fbe = e.fringe_bend_entrance;
    o.fbx = e.fringe_bend_exit;
    o.iparam[0] = e.iparam[0];
    o.iparam[1] = e.iparam[1];
    o.L = T(e.L); o.k = T(e.k); o.angle = T(e.angle); o.e1 = T(e.e1); o.e2 = T(e.e2);
    o.fint1 = T(e.fint1); o.fint2 = T(e.fint2); o.gap = T(e.gap); o.gk = T(e.gk);
    for (int i = 0; i < 4; ++i) { o.pa[i] = T(e.polynom_a[i]); o.pb[i] = T(e.polynom_b[i]); }
    o.kick[0] = T(e.kick_angle[0]); o.kick[1] = T(e.kick_angle[1]);
    o.volt = T(e.volt); o.freq = T(e.freq); o.h = T(e.h); o.lag = T(e.lag);
    o.philag = T(e.philag); o.energy = T(e.energy);
    for (int i = 0; i < 8; ++i) o.param[i] = T(e.param[i]);
    for (int i = 0; i < 6; ++i) { o.t1[i] = T(0.0); o.t2[i] = T(0.0); }
    for (int i = 0; i < 36; ++i) { o.r1[i] = T(0.0); o.r2[i] = T(0.0); }
    if (mis) {
        o.has_mis = true;
        for (int i = 0; i < 6; ++i) { o.t1[i] = T(mis->t1[i]); o.t2[i] = T(mis->t2[i]); }
        for (int i = 0; i < 36; ++i) {
            o.r1[i] = T(mis->r1[i]); o.r2[i] = T(mis->r2[i]);
            if (mis->r1[i] != 0.0) o.r1nz = true;
            if (mis->r2[i] != 0.0) o.r2nz = true;
        }
    }
    return o;
}

// ---------------------------------------------------------------------------
// check_lost: src/tracking.jl:49-52
// ---------------------------------------------------------------------------
template <class T>
inline bool check_lost(const V6<T>& r) {
    using std::abs;
    return is_nan(r[0]) || value_of(abs(r[0])) > COORD_LIMIT || value_of(abs(r[2])) > COORD_LIMIT ||
           value_of(abs(r[1])) > ANGLE_LIMIT || value_of(abs(r[3])) > ANGLE_LIMIT;
}

// apply_misalignment: src/tracking.jl:60-67 (r + t), and `elem.r1 * r` on an
// SMatrix (column-major, summed over columns left to right).
template <class T>
inline V6<T> add_t(const V6<T>& r, const T* t) {
    V6<T> o;
    for (int i = 0; i < 6; ++i) o[i] = r[i] + t[i];
    return o;
}
template <class T>
inline V6<T> mat_mul(const T* R, const V6<T>& r) {
    V6<T> o;
    for (int i = 0; i < 6; ++i) {
        T s = R[i] * r[0];
        for (int j = 1; j < 6; ++j) s = s + R[j * 6 + i] * r[j];
        o[i] = s;
    }
    return o;
}
template <class T>
inline V6<T> entrance(const Elem<T>& e, V6<T> r) {
    r = add_t(r, e.t1);  // t1 is always added (zero vector by default)
    if (e.r1nz) r = mat_mul(e.r1, r);
    return r;
}
template <class T>
inline V6<T> exit_(const Elem<T>& e, V6<T> r) {
    if (e.r2nz) r = mat_mul(e.r2, r);
    r = add_t(r, e.t2);
    return r;
}

// ---------------------------------------------------------------------------
// drift6: src/tracking.jl:87-108
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> drift6(const V6<T>& r, T L, T beti, bool exact) {
    using std::sqrt;
    if constexpr (is_tps<T>::value) {
        // drift6_tpsa (ext/TrackPadPolySeriesExt.jl:57-65): exact, no loss
        // check; L / sqrt(pz2) as L * pz2^(-1/2) (one series)
        T pz2 = T(1.0) + T(2.0) * r[5] * beti + r[5] * r[5] - r[1] * r[1] - r[3] * r[3];
        T NormL = L * rsqrt(pz2);
        T x_new = r[0] + NormL * r[1];
        T y_new = r[2] + NormL * r[3];
        T z_new = r[4] + NormL * (beti + r[5]) - L * beti;
        return V6<T>{{x_new, r[1], y_new, r[3], z_new, r[5]}};
    }
    if (exact) {
        T pz2 = T(1.0) + T(2.0) * r[5] * beti + r[5] * r[5] - r[1] * r[1] - r[3] * r[3];
        if (value_of(pz2) <= 0.0) return nan6<T>();
        T NormL = L / sqrt(pz2);
        T x_new = r[0] + NormL * r[1];
        T y_new = r[2] + NormL * r[3];
        T z_new = r[4] + NormL * (beti + r[5]) - L * beti;
        return V6<T>{{x_new, r[1], y_new, r[3], z_new, r[5]}};
    } else {
        T NormL = L / (T(1.0) + r[5]);
        T x_new = r[0] + NormL * r[1];
        T y_new = r[2] + NormL * r[3];
        T z_new = r[4] + NormL * (r[1] * r[1] + r[3] * r[3]) / (T(2.0) * (T(1.0) + r[5]));
        return V6<T>{{x_new, r[1], y_new, r[3], z_new, r[5]}};
    }
}

// pass!(::Drift): src/tracking.jl:115-132
template <class T>
inline V6<T> pass_drift(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    r = drift6(r, e.L, beti, exact);
    return exit_(e, r);
}

// ---------------------------------------------------------------------------
// Dipole edge focusing: src/tracking.jl:160-189 (entrance), 194-221 (exit)
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> edge_fringe(const V6<T>& r, T inv_rho, T edge_angle, T fint, T gap, int method, bool is_exit) {
    T fringecorr;
    if (value_of(fint) == 0.0 || value_of(gap) == 0.0 || method == 0) {
        fringecorr = T(0.0);
    } else {
        T sedge = sin(edge_angle);
        T cedge = cos(edge_angle);
        fringecorr = inv_rho * gap * fint * (T(1.0) + sedge * sedge) / cedge;
    }
    if constexpr (is_tps<T>::value) {
        // edge_fringe_entrance_tpsa / _exit_tpsa (ext/TrackPadPolySeriesExt.jl:161-215):
        // fx and fy are numbers, fy from the constant parts of delta and px
        const double ir = value_of(inv_rho), ea = value_of(edge_angle), fc = value_of(fringecorr);
        const double d0 = value_of(r[5]), px0 = value_of(r[1]);
        const double fxd = ir * tp::libm::tan(ea);
        double fyd;
        if (method == 2) fyd = ir * tp::libm::tan(ea - fc / (1.0 + d0)) / (1.0 + d0);
        else if (method == 3) fyd = ir * tp::libm::tan(is_exit ? (ea - fc - px0 / (1.0 + d0)) : (ea - fc + px0 / (1.0 + d0)));
        else fyd = ir * tp::libm::tan(ea - fc / (1.0 + d0));
        T px_new = r[1] + r[0] * T(fxd);
        T py_new = r[3] - r[2] * T(fyd);
        return V6<T>{{r[0], px_new, r[2], py_new, r[4], r[5]}};
    }
    T fx = inv_rho * tan(edge_angle);
    T fy;
    if (method == 1) {
        fy = inv_rho * tan(edge_angle - fringecorr / (T(1.0) + r[5]));
    } else if (method == 2) {
        fy = inv_rho * tan(edge_angle - fringecorr / (T(1.0) + r[5])) / (T(1.0) + r[5]);
    } else if (method == 3) {
        if (!is_exit)
            fy = inv_rho * tan(edge_angle - fringecorr + r[1] / (T(1.0) + r[5]));
        else
            fy = inv_rho * tan(edge_angle - fringecorr - r[1] / (T(1.0) + r[5]));
    } else {
        fy = inv_rho * tan(edge_angle - fringecorr / (T(1.0) + r[5]));
    }
    T px_new = r[1] + r[0] * fx;
    T py_new = r[3] - r[2] * fy;
    return V6<T>{{r[0], px_new, r[2], py_new, r[4], r[5]}};
}

// ---------------------------------------------------------------------------
// Thin kicks: bndthinkick src/tracking.jl:243-270, strthinkick :284-305
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> bndthinkick(const V6<T>& r, const T* pa, const T* pb, T L, T irho, int max_order, T beti) {
    T ReSum = pb[max_order];
    T ImSum = pa[max_order];
    for (int i = max_order - 1; i >= 0; --i) {
        T ReSumTemp = ReSum * r[0] - ImSum * r[2] + pb[i];
        ImSum = ImSum * r[0] + ReSum * r[2] + pa[i];
        ReSum = ReSumTemp;
    }
    T px_new = r[1] - L * (ReSum - (r[5] - r[0] * irho) * irho);
    T py_new = r[3] + L * ImSum;
    T z_new = r[4] + L * irho * r[0] * beti;
    return V6<T>{{r[0], px_new, r[2], py_new, z_new, r[5]}};
}

template <class T>
inline V6<T> strthinkick(const V6<T>& r, const T* pa, const T* pb, T L, int max_order) {
    T ReSum = pb[max_order];
    T ImSum = pa[max_order];
    for (int i = max_order - 1; i >= 0; --i) {
        T ReSumTemp = ReSum * r[0] - ImSum * r[2] + pb[i];
        ImSum = ImSum * r[0] + ReSum * r[2] + pa[i];
        ReSum = ReSumTemp;
    }
    T px_new = r[1] - L * ReSum;
    T py_new = r[3] + L * ImSum;
    return V6<T>{{r[0], px_new, r[2], py_new, r[4], r[5]}};
}

// ---------------------------------------------------------------------------
// Yoshida-4 integrators: symplectic4_pass src/tracking.jl:317-341,
// symplectic4_bend_pass :350-375
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> symplectic4_pass(V6<T> r, T L, const T* pa, const T* pb, int max_order, int num_steps,
                              T beti, bool exact) {
    T SL = L / T(double(num_steps));
    T L1 = SL * T(DRIFT1);
    T L2 = SL * T(DRIFT2);
    T K1 = SL * T(KICK1);
    T K2 = SL * T(KICK2);
    for (int s = 0; s < num_steps; ++s) {
        r = drift6(r, L1, beti, exact);
        r = strthinkick(r, pa, pb, K1, max_order);
        r = drift6(r, L2, beti, exact);
        r = strthinkick(r, pa, pb, K2, max_order);
        r = drift6(r, L2, beti, exact);
        r = strthinkick(r, pa, pb, K1, max_order);
        r = drift6(r, L1, beti, exact);
    }
    return r;
}

template <class T>
inline V6<T> symplectic4_bend_pass(V6<T> r, T L, const T* pa, const T* pb, T irho, int max_order,
                                   int num_steps, T beti, bool exact) {
    T SL = L / T(double(num_steps));
    T L1 = SL * T(DRIFT1);
    T L2 = SL * T(DRIFT2);
    T K1 = SL * T(KICK1);
    T K2 = SL * T(KICK2);
    for (int s = 0; s < num_steps; ++s) {
        r = drift6(r, L1, beti, exact);
        r = bndthinkick(r, pa, pb, K1, irho, max_order, beti);
        r = drift6(r, L2, beti, exact);
        r = bndthinkick(r, pa, pb, K2, irho, max_order, beti);
        r = drift6(r, L2, beti, exact);
        r = bndthinkick(r, pa, pb, K1, irho, max_order, beti);
        r = drift6(r, L1, beti, exact);
    }
    return r;
}

// kick_angle folding shared by Quadrupole (:396-411), SBend (:668-682),
// ExactSBend (:931-940), QuadrupoleSC (:1004-1007), SBendSC (:1052-1055).
template <class T>
inline void fold_kick_angle(const Elem<T>& e, T* pa, T* pb) {
    if (value_of(e.L) > 0.0) {
        pb[0] = pb[0] - sin(e.kick[0]) / e.L;
        pa[0] = pa[0] + sin(e.kick[1]) / e.L;
    }
}

// pass!(::Quadrupole): src/tracking.jl:386-427
template <class T>
inline V6<T> pass_quad(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    T pb[4] = {e.pb[0], e.k, e.pb[2], e.pb[3]};
    T pa[4] = {e.pa[0], e.pa[1], e.pa[2], e.pa[3]};
    fold_kick_angle(e, pa, pb);
    r = symplectic4_pass(r, e.L, pa, pb, e.max_order, e.num_int_steps, beti, exact);
    return exit_(e, r);
}

// pass!(::Sextupole): src/tracking.jl:438-459 (no kick_angle folding)
template <class T>
inline V6<T> pass_sext(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    T pb[4] = {e.pb[0], e.pb[1], e.k / T(2.0), e.pb[3]};
    r = symplectic4_pass(r, e.L, e.pa, pb, e.max_order, e.num_int_steps, beti, exact);
    return exit_(e, r);
}

// pass!(::Octupole): src/tracking.jl:470-491
template <class T>
inline V6<T> pass_oct(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    T pb[4] = {e.pb[0], e.pb[1], e.pb[2], e.k / T(6.0)};
    r = symplectic4_pass(r, e.L, e.pa, pb, e.max_order, e.num_int_steps, beti, exact);
    return exit_(e, r);
}

// pass!(::RFCavity): src/tracking.jl:502-518
template <class T>
inline V6<T> pass_rf(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    T beta = T(1.0) / beti;
    if (value_of(e.L) > 0.0) r = drift6(r, e.L / T(2.0), beti, exact);
    if (value_of(e.energy) > 0.0) {
        T nv = e.volt / e.energy;
        T phase = T(TWO_PI) * e.freq * ((r[4] - e.lag) / T(C_LIGHT)) - e.philag;
        T delta_new = r[5] - nv * sin(phase) / (beta * beta);
        r = V6<T>{{r[0], r[1], r[2], r[3], r[4], delta_new}};
    }
    if (value_of(e.L) > 0.0) r = drift6(r, e.L / T(2.0), beti, exact);
    return r;
}

// pass!(::Solenoid): src/tracking.jl:529-570
template <class T>
inline V6<T> pass_solenoid(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    T ks = e.param[0];
    T L = e.L;
    if (value_of(ks) == 0.0) {
        r = drift6(r, L, beti, exact);
    } else {
        T p_norm = T(1.0) / (T(1.0) + r[5]);
        T x = r[0];
        T xpr = r[1] * p_norm;
        T y = r[2];
        T ypr = r[3] * p_norm;
        T H = ks * p_norm / T(2.0);
        T S = sin(L * H);
        T C = cos(L * H);
        T x_new = x * C * C + xpr * C * S / H + y * C * S + ypr * S * S / H;
        T px_new = (-x * H * C * S + xpr * C * C - y * H * S * S + ypr * C * S) / p_norm;
        T y_new = -x * C * S - xpr * S * S / H + y * C * C + ypr * C * S / H;
        T py_new = (x * H * S * S - xpr * C * S - y * C * S * H + ypr * C * C) / p_norm;
        T z_new = r[4] + L * (H * H * (x * x + y * y) + T(2.0) * H * (xpr * y - ypr * x) + xpr * xpr +
                              ypr * ypr) / T(2.0);
        r = V6<T>{{x_new, px_new, y_new, py_new, z_new, r[5]}};
    }
    return exit_(e, r);
}

// pass!(::Corrector): src/tracking.jl:579-607
template <class T>
inline V6<T> pass_corrector(const Elem<T>& e, V6<T> r) {
    r = entrance(e, r);
    T xk = e.param[0], yk = e.param[1];
    T p_norm = T(1.0) / (T(1.0) + r[5]);
    T NormL = e.L * p_norm;
    T z_new = r[4] + NormL * p_norm *
                         (xk * xk / T(3.0) + yk * yk / T(3.0) + r[1] * r[1] + r[3] * r[3] + r[1] * xk +
                          r[3] * yk) / T(2.0);
    T x_new = r[0] + NormL * (r[1] + xk / T(2.0));
    T px_new = r[1] + xk;
    T y_new = r[2] + NormL * (r[3] + yk / T(2.0));
    T py_new = r[3] + yk;
    r = V6<T>{{x_new, px_new, y_new, py_new, z_new, r[5]}};
    return exit_(e, r);
}

// pass!(::ThinMultipole): src/tracking.jl:616-633
template <class T>
inline V6<T> pass_thin_multipole(const Elem<T>& e, V6<T> r) {
    r = entrance(e, r);
    r = strthinkick(r, e.pa, e.pb, T(1.0), e.max_order);
    return exit_(e, r);
}

// pass!(::SBend): src/tracking.jl:657-706.  sbend_core is the part after the
// entrance misalignment and before the exit misalignment; SBendSC
// (src/tracking.jl:1041-1070) runs the same core with clamp(max_order, 0, 3).
template <class T>
inline V6<T> sbend_core(const Elem<T>& e, V6<T> r, T beti, bool exact, int max_order) {
    T irho = e.angle / e.L;
    T pb[4] = {e.pb[0], e.pb[1], e.pb[2], e.pb[3]};
    T pa[4] = {e.pa[0], e.pa[1], e.pa[2], e.pa[3]};
    fold_kick_angle(e, pa, pb);
    if (e.fbe != 0) r = edge_fringe(r, irho, e.e1, e.fint1, e.gap, e.fbe, false);
    r = symplectic4_bend_pass(r, e.L, pa, pb, irho, max_order, e.num_int_steps, beti, exact);
    if (e.fbx != 0) r = edge_fringe(r, irho, e.e2, e.fint2, e.gap, e.fbx, true);
    return r;
}

template <class T>
inline V6<T> pass_sbend(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    r = sbend_core(e, r, beti, exact, e.max_order);
    return exit_(e, r);
}

// ---------------------------------------------------------------------------
// Exact sector bend: pxyz :717-720, yrot :727-745, bend_fringe :752-815,
// bend_edge :822-851, exact_bend_body :858-894, pass!(::ExactSBend) :901-973
// ---------------------------------------------------------------------------
template <class T>
inline T pxyz(T dp1, T px, T py) {
    using std::sqrt;
    T val = dp1 * dp1 - px * px - py * py;
    return value_of(val) > 0.0 ? sqrt(val) : T(0.0);
}

// Julia clamp(x, lo, hi) = ifelse(x > hi, hi, ifelse(x < lo, lo, x)); NaN passes.
template <class T>
inline T clamp1(T x) {
    if (value_of(x) > 1.0) return T(1.0);
    if (value_of(x) < -1.0) return T(-1.0);
    return x;
}

template <class T>
inline V6<T> yrot(const V6<T>& r, T phi, T beti) {
    if (value_of(phi) == 0.0) return r;
    T dp1 = beti + r[5];
    T c = cos(phi);
    T s = sin(phi);
    T pz = pxyz(dp1, r[1], r[3]);
    T p = c * pz - s * r[1];
    T px_new = s * pz + c * r[1];
    T x_new = r[0] * pz / p;
    T y_new = r[2] + r[0] * r[3] * s / p;
    T z_new = r[4] + dp1 * r[0] * s / p;
    return V6<T>{{x_new, px_new, y_new, r[3], z_new, r[5]}};
}

template <class T>
inline V6<T> bend_fringe(const V6<T>& r, T irho, T gK, T beti) {
    using std::sqrt; T b0 = irho;
    T dp1 = beti + r[5];
    T pz = pxyz(dp1, r[1], r[3]);
    T px = r[1];
    T py = r[3];
    T xp = px / pz;
    T yp = py / pz;
    T term1 = T(1.0) + xp * xp * (T(2.0) + yp * yp);
    T term2 = xp / (T(1.0) + yp * yp);
    T phi = -b0 * tan(b0 * gK * term1 * pz - atan(term2));
    T px2 = px * px;
    T py2 = py * py;
    T pz2 = pz * pz;
    T pz4 = pz2 * pz2;
    T py2z2 = (py2 + pz2);
    T arg_sec = (b0 * gK * (pz4 + px2 * (py2 + T(2.0) * pz2))) / (pz2 * pz) - atan(px * pz / (py2 + pz2));
    T sec = T(1.0) / cos(arg_sec);  // Julia sec(x) = inv(cos(x))
    T powsec = sec * sec;
    T py4 = py2 * py2;
    T py6 = py4 * py2;
    T pz5 = pz4 * pz;
    T pz6 = pz4 * pz2;
    T py2z2_sq = py2z2 * py2z2;
    T denom = pz5 * (py4 + px2 * pz2 + T(2.0) * py2 * pz2 + pz4);
    T dpx_num = -(b0 * (px2 * pz4 * (py2 - pz2) - pz6 * (py2 + pz2) +
                        b0 * gK * px *
                            (pz2 * py2z2_sq * (T(2.0) * py2 + T(3.0) * pz2) +
                             px2 * px2 * (T(3.0) * py2 * pz2 + T(2.0) * pz4) +
                             px2 * (T(3.0) * py6 + T(8.0) * py4 * pz2 + T(9.0) * py2 * pz4 + T(5.0) * pz6)))) *
                powsec;
    T dpx = dpx_num / denom;
    T dpy_num = -(b0 * py *
                  (px * pz4 * (py2 + pz2) +
                   b0 * gK *
                       (-(pz4 * py2z2_sq) + px2 * px2 * (T(3.0) * py2 * pz2 + T(4.0) * pz4) +
                        px2 * (T(3.0) * py6 + T(10.0) * py4 * pz2 + T(11.0) * py2 * pz4 + T(3.0) * pz6)))) *
                powsec;
    T dpy = dpy_num / denom;
    T dd_num = (b0 * dp1 *
                (px * pz4 * (py2 - pz2) +
                 b0 * gK *
                     (-(pz4 * py2z2_sq) + px2 * px2 * (T(3.0) * py2 * pz2 + T(2.0) * pz4) +
                      px2 * (T(3.0) * py6 + T(8.0) * py4 * pz2 + T(7.0) * py2 * pz4 + pz6)))) *
               powsec;
    T dd = dd_num / denom;
    T yf = (T(2.0) * r[2]) / (T(1.0) + sqrt(T(1.0) - T(2.0) * dpy * r[2]));
    T dxf = T(0.5) * dpx * (yf * yf);  // 0.5 * dpx * yf^2
    T dct = T(0.5) * dd * (yf * yf);
    T dpyf = phi * yf;
    return V6<T>{{r[0] + dxf, r[1], yf, r[3] - dpyf, r[4] - dct, r[5]}};
}

template <class T>
inline V6<T> bend_edge(const V6<T>& r, T rhoinv, T theta, T beti) {
    using std::abs; if (value_of(abs(rhoinv)) < 1e-6) return r;
    T dp1 = beti + r[5];
    T c = cos(theta);
    T s = sin(theta);
    T pz = pxyz(dp1, r[1], r[3]);
    T d2 = pxyz(dp1, T(0.0), r[3]);
    T px_new = r[1] * c + (pz - rhoinv * r[0]) * s;
    T val1 = clamp1(r[1] / d2);
    T val2 = clamp1(px_new / d2);
    T dasin = asin(val1) - asin(val2);
    T num = r[0] * (r[1] * sin(T(2.0) * theta) + s * s * (T(2.0) * pz - rhoinv * r[0]));
    T den = pxyz(dp1, px_new, r[3]) + pz * c - r[1] * s;
    T x_new = r[0] * c + num / den;
    T y_new = r[2] + r[3] * (theta / rhoinv + dasin / rhoinv);
    T z_new = r[4] + dp1 / rhoinv * (theta + dasin);
    return V6<T>{{x_new, px_new, y_new, r[3], z_new, r[5]}};
}

template <class T>
inline V6<T> exact_bend_body(const V6<T>& r, T irho, T L, T beti) {
    using std::abs; T dp1 = beti + r[5];
    T pz = pxyz(dp1, r[1], r[3]);
    if (value_of(abs(irho)) < 1e-6) {
        T NormL = L / pz;
        return V6<T>{{r[0] + r[1] * NormL, r[1], r[2] + r[3] * NormL, r[3], r[4] + NormL * dp1 - L * beti,
                      r[5]}};
    }
    T pzmx = pz - (T(1.0) + r[0] * irho);
    T cs = cos(irho * L);
    T sn = sin(irho * L);
    T px_new = r[1] * cs + pzmx * sn;
    T d2 = pxyz(dp1, T(0.0), r[3]);
    T val1 = clamp1(r[1] / d2);
    T val2 = clamp1(px_new / d2);
    T dasin = L + (asin(val1) - asin(val2)) / irho;
    T x_new = (pxyz(dp1, px_new, r[3]) - pzmx * cs + r[1] * sn - T(1.0)) / irho;
    T y_new = r[2] + r[3] * dasin;
    T z_new = r[4] + dp1 * dasin - L * beti;
    return V6<T>{{x_new, px_new, y_new, r[3], z_new, r[5]}};
}

template <class T>
inline V6<T> pass_exact_sbend(const Elem<T>& e, V6<T> r, T beti) {
    r = entrance(e, r);
    T irho = e.angle / e.L;
    r = yrot(r, e.e1, beti);
    if (e.fbe != 0) r = bend_fringe(r, irho, e.gk, beti);
    r = bend_edge(r, irho, -e.e1, beti);
    if (e.num_int_steps == 0) {
        r = exact_bend_body(r, irho, e.L, beti);
    } else {
        T SL = e.L / T(double(e.num_int_steps));
        T L1 = SL * T(DRIFT1);
        T L2 = SL * T(DRIFT2);
        T K1 = SL * T(KICK1);
        T K2 = SL * T(KICK2);
        T pb[4] = {e.pb[0], e.pb[1], e.pb[2], e.pb[3]};
        T pa[4] = {e.pa[0], e.pa[1], e.pa[2], e.pa[3]};
        fold_kick_angle(e, pa, pb);
        for (int s = 0; s < e.num_int_steps; ++s) {
            r = exact_bend_body(r, irho, L1, beti);
            r = strthinkick(r, pa, pb, K1, e.max_order);
            r = exact_bend_body(r, irho, L2, beti);
            r = strthinkick(r, pa, pb, K2, e.max_order);
            r = exact_bend_body(r, irho, L2, beti);
            r = strthinkick(r, pa, pb, K1, e.max_order);
            r = exact_bend_body(r, irho, L1, beti);
        }
    }
    r = bend_edge(r, irho, -e.e2, beti);
    if (e.fbx != 0) r = bend_fringe(r, -irho, e.gk, beti);
    r = yrot(r, e.e2, beti);
    return exit_(e, r);
}

// ---------------------------------------------------------------------------
// Space-charge canonical family: src/tracking.jl:981-1070
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> pass_multipole_sc(const Elem<T>& e, V6<T> r, T beti, bool exact, bool fold) {
    r = entrance(e, r);
    T pb[4] = {e.param[0], e.param[1], e.param[2] / T(2.0), e.param[3] / T(6.0)};
    T pa[4] = {e.pa[0], e.pa[1], e.pa[2], e.pa[3]};
    if (fold) fold_kick_angle(e, pa, pb);
    int mo = std::min(std::max(e.max_order, 0), 3);
    r = symplectic4_pass(r, e.L, pa, pb, mo, e.num_int_steps, beti, exact);
    return exit_(e, r);
}

template <class T>
inline V6<T> pass_sbend_sc(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    r = entrance(e, r);
    if (value_of(e.L) == 0.0) return nan6<T>();
    r = sbend_core(e, r, beti, exact, std::min(std::max(e.max_order, 0), 3));
    return exit_(e, r);
}

// Translation: src/tracking.jl:1182-1192
template <class T>
inline V6<T> pass_translation(const Elem<T>& e, const V6<T>& r, T beti) {
    using std::sqrt;
    T pz2 = T(1.0) + T(2.0) * r[5] * beti + r[5] * r[5] - r[1] * r[1] - r[3] * r[3];
    if (value_of(pz2) <= 0.0) return nan6<T>();
    T pz = sqrt(pz2);
    T dx = e.param[0], dy = e.param[1], ds = e.param[2];
    T x_new = r[0] - (dx + ds * r[1] / pz);
    T y_new = r[2] - (dy + ds * r[3] / pz);
    T z_new = r[4] + ds * (beti + r[5]) / pz;
    return V6<T>{{x_new, r[1], y_new, r[3], z_new, r[5]}};
}

// YRotation: src/tracking.jl:1194-1218
template <class T>
inline V6<T> pass_yrotation(const Elem<T>& e, const V6<T>& r, T beti) {
    using std::abs; using std::sqrt; T angle = -e.angle;
    if (value_of(angle) == 0.0) return r;
    T ca = cos(angle);
    T sa = sin(angle);
    T ta = tan(angle);
    T pz2 = T(1.0) + T(2.0) * r[5] * beti + r[5] * r[5] - r[1] * r[1] - r[3] * r[3];
    if (value_of(pz2) <= 0.0) return nan6<T>();
    T pz = sqrt(pz2);
    T ptt = T(1.0) - ta * r[1] / pz;
    if (value_of(abs(ptt)) < 1.4901161193847656e-08) return nan6<T>();  // sqrt(eps(Float64))
    T x_new = r[0] / (ca * ptt);
    T px_new = ca * r[1] + sa * pz;
    T y_new = r[2] + ta * r[0] * r[3] / (pz * ptt);
    T z_new = r[4] + ta * r[0] * (beti + r[5]) / (pz * ptt);
    return V6<T>{{x_new, px_new, y_new, r[3], z_new, r[5]}};
}

// CrabCavity: src/tracking.jl:1531-1547
template <class T>
inline V6<T> pass_crab(const Elem<T>& e, V6<T> r, T beti, bool exact) {
    using std::abs; T volt = e.volt * (T(1.0) + e.param[2]);
    T phi = e.param[1] + e.param[3];
    T E = abs(e.energy);
    if (value_of(E) < EPS || is_nan(E)) E = is_nan(E) ? E : T(EPS);  // max(abs(energy), eps)
    T kk = e.param[0];
    T ang = kk * r[4] + phi;
    if (value_of(e.L) > 0.0) r = drift6(r, e.L / T(2.0), beti, exact);
    T px_new = r[1] + (volt / E) * sin(ang * beti);
    T delta_new = r[5] - (kk * volt / E * beti) * r[0] * cos(ang * beti);
    r = V6<T>{{r[0], px_new, r[2], r[3], r[4], delta_new}};
    if (value_of(e.L) > 0.0) r = drift6(r, e.L / T(2.0), beti, exact);
    return r;
}

// AccelCavity: src/tracking.jl:1549-1559
template <class T>
inline V6<T> pass_accel(const Elem<T>& e, const V6<T>& r, T beti) {
    using std::abs; T beta = T(1.0) / beti;
    T beta2 = beta * beta;
    if (value_of(beta2) <= EPS) return r;
    T E = abs(e.energy);
    if (value_of(E) < EPS || is_nan(E)) E = is_nan(E) ? E : T(EPS);
    T kk = e.param[0], phis = e.param[1];
    T sv = sin(kk * r[4] + phis) - sin(phis);
    T delta_new = r[5] + (e.volt / (beta2 * E)) * sv;
    return V6<T>{{r[0], r[1], r[2], r[3], r[4], delta_new}};
}

// LongitudinalRFMap: src/tracking.jl:1575-1585 (k, h of the linked RF element
// are resolved on the host by _rf_k/_rf_h, :1565-1573)
template <class T>
inline V6<T> pass_long_rf_map(const Elem<T>& e, const V6<T>& r, T beti) {
    using std::abs;
    T kk = e.param[1];
    if (value_of(abs(kk)) <= EPS) return r;
    T hh = e.param[2];
    T beta = T(1.0) / beti;
    T eta = e.param[0] - (T(1.0) - beta * beta);
    T z_new = r[4] - (T(TWO_PI) * hh * eta / kk) * r[5];
    return V6<T>{{r[0], r[1], r[2], r[3], z_new, r[5]}};
}

// LorentzBoost :1587-1595, InvLorentzBoost :1597-1604
template <class T>
inline V6<T> pass_lorentz(const Elem<T>& e, const V6<T>& r, bool inverse) {
    if (e.iparam[0] != 0) return r;
    if (!inverse) {
        T invcos = T(1.0) / e.param[1];
        T tanang = e.param[3];
        T x_new = r[0] + tanang * r[4];
        T delta_new = r[5] - tanang * r[1];
        return V6<T>{{x_new, r[1] * invcos, r[2], r[3] * invcos, r[4] * invcos, delta_new}};
    }
    T sinang = e.param[2], cosang = e.param[1];
    T x_new = r[0] - sinang * r[4];
    T delta_new = r[5] + sinang * r[1];
    return V6<T>{{x_new, r[1] * cosang, r[2], r[3] * cosang, r[4] * cosang, delta_new}};
}

// StrongThinGaussianBeam: src/tracking.jl:1610-1619
template <class T>
inline V6<T> pass_strong_thin_gaussian(const Elem<T>& e, const V6<T>& r) {
    T amp = e.param[0], sx = e.param[1], sy = e.param[2], xo = e.param[3], yo = e.param[4];
    T sx2 = sx * sx;
    if (!(value_of(sx2) >= EPS) && !is_nan(sx2)) sx2 = T(EPS);
    T sy2 = sy * sy;
    if (!(value_of(sy2) >= EPS) && !is_nan(sy2)) sy2 = T(EPS);
    T dx = r[0] - xo;
    T dy = r[2] - yo;
    T g = amp * exp(T(-0.5) * (dx * dx / sx2 + dy * dy / sy2));
    T px_new = r[1] - g * dx / sx2;
    T py_new = r[3] - g * dy / sy2;
    return V6<T>{{r[0], px_new, r[2], py_new, r[4], r[5]}};
}

// ---------------------------------------------------------------------------
// LBend: _lbend_body src/tracking.jl:1076-1150, pass!(::LBend) :1152-1170
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> lbend_body(const V6<T>& r, T L, T grd, T b_angle, T by_error) {
    using std::abs;
    using std::sqrt;
    if (value_of(L) == 0.0) return r;
    T p_norm = T(1.0) / (T(1.0) + r[5]);
    T Kx = b_angle / L;
    T G1 = (Kx * Kx + grd) * p_norm;
    T G2 = -grd * p_norm;
    const double tol = 1.4901161193847656e-08;  // sqrt(eps(Float64))
    T MHD = T(1.0), M12 = L, M21 = T(0.0);
    T MVD = T(1.0), M34 = L, M43 = T(0.0);
    T arg1 = T(0.0), arg2 = T(0.0), sqrtG1 = T(0.0), sqrtG2 = T(0.0);
    if (value_of(abs(G1)) >= tol) {
        if (value_of(G1) > 0.0) {
            sqrtG1 = sqrt(G1);
            arg1 = L * sqrtG1;
            MHD = cos(arg1); M12 = sin(arg1) / sqrtG1; M21 = -sin(arg1) * sqrtG1;
        } else {
            sqrtG1 = sqrt(-G1);
            arg1 = L * sqrtG1;
            MHD = cosh(arg1); M12 = sinh(arg1) / sqrtG1; M21 = sinh(arg1) * sqrtG1;
        }
    }
    if (value_of(abs(G2)) >= tol) {
        if (value_of(G2) > 0.0) {
            sqrtG2 = sqrt(G2);
            arg2 = L * sqrtG2;
            MVD = cos(arg2); M34 = sin(arg2) / sqrtG2; M43 = -sin(arg2) * sqrtG2;
        } else {
            sqrtG2 = sqrt(-G2);
            arg2 = L * sqrtG2;
            MVD = cosh(arg2); M34 = sinh(arg2) / sqrtG2; M43 = sinh(arg2) * sqrtG2;
        }
    }
    T x = r[0], xpr = r[1] * p_norm, y = r[2], ypr = r[3] * p_norm, delta = r[5];
    T dterm = delta * p_norm - by_error;
    T x_new = MHD * x + M12 * xpr;
    T px_new = (M21 * x + MHD * xpr) / p_norm;
    if (value_of(abs(G1)) < tol) {
        x_new = x_new + dterm * L * L * Kx / T(2.0);
        px_new = px_new + dterm * L * Kx / p_norm;
    } else if (value_of(G1) > 0.0) {
        x_new = x_new + dterm * (T(1.0) - cos(arg1)) * Kx / G1;
        px_new = px_new + dterm * sin(arg1) * Kx / (sqrtG1 * p_norm);
    } else {
        x_new = x_new + dterm * (T(1.0) - cosh(arg1)) * Kx / G1;
        px_new = px_new + dterm * sinh(arg1) * Kx / (sqrtG1 * p_norm);
    }
    T y_new = MVD * y + M34 * ypr;
    T py_new = (M43 * y + MVD * ypr) / p_norm;
    T z_new = r[4] + xpr * xpr * (L + MHD * M12) / T(4.0);
    if (value_of(abs(G1)) >= tol) {
        z_new = z_new + (L - MHD * M12) * (x * x * G1 + dterm * dterm * Kx * Kx / G1 - T(2.0) * x * Kx * dterm) / T(4.0);
        z_new = z_new + M12 * M21 * (x * xpr - xpr * dterm * Kx / G1) / T(2.0);
        z_new = z_new + (Kx * x * M12 + xpr * (T(1.0) - MHD) * Kx / G1 + dterm * (L - M12) * Kx * Kx / G1);
    }
    z_new = z_new + ((L - MVD * M34) * y * y * G2 + ypr * ypr * (L + MVD * M34)) / T(4.0);
    z_new = z_new + M34 * M43 * y * ypr / T(2.0);
    return V6<T>{{x_new, px_new, y_new, py_new, z_new, r[5]}};
}

template <class T>
inline V6<T> pass_lbend(const Elem<T>& e, V6<T> r) {
    r = entrance(e, r);
    if (value_of(e.L) == 0.0) return nan6<T>();
    T irho = e.angle / e.L;
    r = edge_fringe(r, irho, e.e1, e.fint1, e.gap, 1, false);
    r = lbend_body(r, e.L, e.param[0], e.angle, e.param[1]);
    r = edge_fringe(r, irho, e.e2, e.fint2, e.gap, 1, true);
    return exit_(e, r);
}

// StrongGaussianBeam: src/tracking.jl:1621-1641 (slice arrays in aux)
template <class T>
inline V6<T> pass_strong_gaussian(const Elem<T>& e, const V6<T>& r) {
    using std::abs;
    const int nz = e.iparam[1] / 3;
    if (nz <= 0) return r;
    T bs0 = e.param[2], bs1 = e.param[3];
    T sx2 = bs0 * bs0;
    if (!(value_of(sx2) >= EPS) && !is_nan(sx2)) sx2 = T(EPS);
    T sy2 = bs1 * bs1;
    if (!(value_of(sy2) >= EPS) && !is_nan(sy2)) sy2 = T(EPS);
    T ae = abs(e.param[1]);
    if (!(value_of(ae) >= EPS) && !is_nan(ae)) ae = T(EPS);
    T factor = e.param[0] / ae;
    T px = r[1], py = r[3];
    for (int i = 0; i < nz; ++i) {
        T w = T(e.aux[i]), xoff = T(e.aux[nz + i]), yoff = T(e.aux[2 * nz + i]);
        T dx = r[0] - xoff;
        T dy = r[2] - yoff;
        T g = w * exp(T(-0.5) * (dx * dx / sx2 + dy * dy / sy2));
        px = px - factor * g * dx / sx2;
        py = py - factor * g * dy / sy2;
    }
    return V6<T>{{r[0], px, r[2], py, r[4], r[5]}};
}

// LongitudinalRLCWake: src/tracking.jl:1647-1654, wakefieldfunc_RLCWake
// src/elements/wake.jl:27-37.  param = freq, Rshunt, Q0, scale.
template <class T>
inline V6<T> pass_rlc_wake(const Elem<T>& e, const V6<T>& r) {
    using std::sqrt;
    if (value_of(e.param[3]) == 0.0) return r;
    if constexpr (is_tps<T>::value) {
        // ext/TrackPadPolySeriesExt.jl:630-639: the wake at the constant part of z
        Elem<double> ed;
        for (int i = 0; i < 4; ++i) ed.param[i] = value_of(e.param[i]);
        V6<double> rd{{0.0, 0.0, 0.0, 0.0, value_of(r[4]), 0.0}};
        const double dd = pass_rlc_wake(ed, rd)[5];  // -scale * W(t)
        return V6<T>{{r[0], r[1], r[2], r[3], r[4], r[5] + T(dd)}};
    }
    T zc = r[4] / T(C_LIGHT);
    T t = is_nan(zc) ? zc : (value_of(zc) > 0.0 ? T(0.0) : zc);  // min(z/c, 0), NaN propagates
    T Q0 = e.param[2];
    T Q0p = sqrt(Q0 * Q0 - T(0.25));
    T w0 = T(TWO_PI) * e.param[0];
    T w0p = w0 / Q0 * Q0p;
    T wf;
    if (value_of(t) > 0.0) {
        wf = T(0.0);
    } else {
        wf = e.param[1] * w0 / Q0 * (cos(w0p * t) + sin(w0p * t) / (T(2.0) * Q0p)) * exp(w0 * t / (T(2.0) * Q0));
    }
    return V6<T>{{r[0], r[1], r[2], r[3], r[4], r[5] - e.param[3] * wf}};
}

// LongitudinalWake: src/tracking.jl:1656-1663, wakefieldfunc and
// _linear_interpolate src/elements/wake.jl:68-91.  aux = times[n], wakefields[n].
template <class T>
inline V6<T> pass_tab_wake(const Elem<T>& e, const V6<T>& r) {
    if (value_of(e.param[1]) == 0.0) return r;
    if constexpr (is_tps<T>::value) {
        // ext/TrackPadPolySeriesExt.jl:641-649: the wake at the constant part of z
        Elem<double> ed;
        ed.aux = e.aux;
        ed.iparam[1] = e.iparam[1];
        for (int i = 0; i < 2; ++i) ed.param[i] = value_of(e.param[i]);
        V6<double> rd{{0.0, 0.0, 0.0, 0.0, value_of(r[4]), 0.0}};
        const double dd = pass_tab_wake(ed, rd)[5];
        return V6<T>{{r[0], r[1], r[2], r[3], r[4], r[5] + T(dd)}};
    }
    const int n = e.iparam[1] / 2;
    const double* xs = e.aux;
    const double* ys = e.aux + n;
    T t = r[4] / T(C_LIGHT);
    T wf;
    if (value_of(t) > xs[0] * value_of(e.param[0])) {
        wf = T(0.0);
    } else {
        T x = t * e.param[0];
        if (value_of(x) <= xs[0]) {
            T slope = (T(ys[1]) - T(ys[0])) / (T(xs[1]) - T(xs[0]));
            wf = T(ys[0]) + slope * (x - T(xs[0]));
        } else if (value_of(x) >= xs[n - 1]) {
            T slope = (T(ys[n - 1]) - T(ys[n - 2])) / (T(xs[n - 1]) - T(xs[n - 2]));
            wf = T(ys[n - 1]) + slope * (x - T(xs[n - 1]));
        } else {
            wf = T(ys[n - 1]);
            for (int i = 1; i < n; ++i) {
                if (value_of(x) < xs[i]) {
                    T slope = (T(ys[i]) - T(ys[i - 1])) / (T(xs[i]) - T(xs[i - 1]));
                    wf = T(ys[i - 1]) + slope * (x - T(xs[i - 1]));
                    break;
                }
            }
        }
    }
    return V6<T>{{r[0], r[1], r[2], r[3], r[4], r[5] - e.param[1] * wf}};
}

// ---------------------------------------------------------------------------
// Wiggler: src/tracking.jl:1224-1529.  aux = NHharm, NVharm, rad, By[6 NH],
// Bx[6 NV]; harmonic i of By is (_, HCw, kx/kw, ky/kw, kz/kw, tz).
// param = lw, Bmax, energy; num_int_steps = Nsteps.
// ---------------------------------------------------------------------------
template <class T>
inline T sinc_taylor(T x) {  // _sinc_taylor :1226-1229
    T x2 = x * x;
    return T(1.0) - x2 / T(6.0) * (T(1.0) - x2 / T(20.0) * (T(1.0) - x2 / T(42.0) * (T(1.0) - x2 / T(72.0))));
}

template <class T>
struct Wig {
    const Elem<T>* e;
    int nh, nv;
    const double* by;
    const double* bx;
    T lw, bmax;
};

template <class T>
inline Wig<T> wig_of(const Elem<T>& e) {
    Wig<T> w;
    w.e = &e;
    w.nh = int(e.aux[0]);
    w.nv = int(e.aux[1]);
    w.by = e.aux + 3;
    w.bx = e.aux + 3 + 6 * w.nh;
    w.lw = e.param[0];
    w.bmax = e.param[1];
    return w;
}

// _wig_ax_axpy :1231-1280
template <class T>
inline void wig_ax_axpy(const Wig<T>& w, T x, T y, T Zw, T Aw, T Po, T& ax, T& axpy) {
    using std::abs;
    T kw = T(TWO_PI) / w.lw;
    ax = T(0.0);
    axpy = T(0.0);
    for (int i = 0; i < w.nh; ++i) {
        const double* b = w.by + 6 * i;
        T HCw = T(b[1]) * Aw / Po;
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T cx = cos(kx * x);
        T chy = cosh(ky * y);
        T sz = sin(kz * Zw + tz);
        ax = ax + HCw * (kw / kz) * cx * chy * sz;
        T shy = sinh(ky * y);
        T sxkx = value_of(abs(kx / kw)) > 1e-6 ? sin(kx * x) / kx : x * sinc_taylor(kx * x);
        axpy = axpy + HCw * (kw / kz) * ky * sxkx * shy * sz;
    }
    for (int i = 0; i < w.nv; ++i) {
        const double* b = w.bx + 6 * i;
        T VCw = T(b[1]) * Aw / Po;
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T shx = sinh(kx * x);
        T sy = sin(ky * y);
        T sz = sin(kz * Zw + tz);
        ax = ax + VCw * (kw / kz) * (ky / kx) * shx * sy * sz;
        T chx = cosh(kx * x);
        T cy = cos(ky * y);
        axpy = axpy + VCw * (kw / kz) * ((ky / kx) * (ky / kx)) * chx * cy * sz;
    }
}

// _wig_ay_aypx :1282-1331
template <class T>
inline void wig_ay_aypx(const Wig<T>& w, T x, T y, T Zw, T Aw, T Po, T& ay, T& aypx) {
    using std::abs;
    T kw = T(TWO_PI) / w.lw;
    ay = T(0.0);
    aypx = T(0.0);
    for (int i = 0; i < w.nh; ++i) {
        const double* b = w.by + 6 * i;
        T HCw = T(b[1]) * Aw / Po;
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T sx = sin(kx * x);
        T shy = sinh(ky * y);
        T sz = sin(kz * Zw + tz);
        ay = ay + HCw * (kw / kz) * (kx / ky) * sx * shy * sz;
        T cx = cos(kx * x);
        T chy = cosh(ky * y);
        aypx = aypx + HCw * (kw / kz) * ((kx / ky) * (kx / ky)) * cx * chy * sz;
    }
    for (int i = 0; i < w.nv; ++i) {
        const double* b = w.bx + 6 * i;
        T VCw = T(b[1]) * Aw / Po;
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T chx = cosh(kx * x);
        T cy = cos(ky * y);
        T sz = sin(kz * Zw + tz);
        ay = ay + VCw * (kw / kz) * chx * cy * sz;
        T shx = sinh(kx * x);
        T syky = value_of(abs(ky / kw)) > 1e-6 ? sin(ky * y) / ky : y * sinc_taylor(ky * y);
        aypx = aypx + VCw * (kw / kz) * kx * shx * syky * sz;
    }
}

// _wig_map_2nd :1333-1378 (Zw is advanced in place)
template <class T>
inline V6<T> wig_map_2nd(const Wig<T>& w, const V6<T>& r, T dl, T& Zw, T Aw, T Po) {
    T delta = r[5];
    T inv1pd = T(1.0) / (T(1.0) + delta);
    T dld = dl * inv1pd;
    T dl2 = dl / T(2.0);
    T dl2d = dl2 * inv1pd;
    Zw = Zw + dl2;
    T x = r[0], px = r[1], y = r[2], py = r[3], z = r[4];
    T a, ap;
    wig_ay_aypx(w, x, y, Zw, Aw, Po, a, ap);
    px = px - ap;
    py = py - a;
    y = y + dl2d * py;
    z = z + (dl2d / T(2.0)) * (py * py) * inv1pd;
    wig_ay_aypx(w, x, y, Zw, Aw, Po, a, ap);
    px = px + ap;
    py = py + a;
    wig_ax_axpy(w, x, y, Zw, Aw, Po, a, ap);
    px = px - a;
    py = py - ap;
    x = x + dld * px;
    z = z + (dld / T(2.0)) * (px * px) * inv1pd;
    wig_ax_axpy(w, x, y, Zw, Aw, Po, a, ap);
    px = px + a;
    py = py + ap;
    wig_ay_aypx(w, x, y, Zw, Aw, Po, a, ap);
    px = px - ap;
    py = py - a;
    y = y + dl2d * py;
    z = z + (dl2d / T(2.0)) * (py * py) * inv1pd;
    wig_ay_aypx(w, x, y, Zw, Aw, Po, a, ap);
    px = px + ap;
    py = py + a;
    Zw = Zw + dl2;
    return V6<T>{{x, px, y, py, z, delta}};
}

// _wig_B :1400-1449 (the longitudinal field is computed and unused, as there)
template <class T>
inline void wig_B(const Wig<T>& w, T x, T y, T Zw, T& Bxv, T& Byv) {
    T kw = T(TWO_PI) / w.lw;
    T PB0 = w.bmax;
    Bxv = T(0.0);
    Byv = T(0.0);
    T Bzv = T(0.0);
    for (int i = 0; i < w.nh; ++i) {
        const double* b = w.by + 6 * i;
        T HCw = T(b[1]);
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T sx = sin(kx * x), cx = cos(kx * x), chy = cosh(ky * y), shy = sinh(ky * y);
        T cz = cos(kz * Zw + tz), sz = sin(kz * Zw + tz);
        Bxv = Bxv + PB0 * HCw * (kx / ky) * sx * shy * cz;
        Byv = Byv - PB0 * HCw * cx * chy * cz;
        Bzv = Bzv + PB0 * HCw * (kz / ky) * cx * shy * sz;
    }
    for (int i = 0; i < w.nv; ++i) {
        const double* b = w.bx + 6 * i;
        T VCw = T(b[1]);
        T kx = T(b[2]) * kw, ky = T(b[3]) * kw, kz = T(b[4]) * kw, tz = T(b[5]);
        T shx = sinh(kx * x), chx = cosh(kx * x), sy = sin(ky * y), cy = cos(ky * y);
        T cz = cos(kz * Zw + tz), sz = sin(kz * Zw + tz);
        Bxv = Bxv + PB0 * VCw * chx * cy * cz;
        Byv = Byv - PB0 * VCw * (ky / kx) * shx * sy * cz;
        Bzv = Bzv - PB0 * VCw * (kz / kx) * cy * shx * sz;
    }
    (void)Bzv;
}

// _wig_radiation_kicks :1451-1463
template <class T>
inline V6<T> wig_rad_kick(const V6<T>& r, T Bxv, T Byv, T Po, T srCoef, T dl) {
    T B2 = Bxv * Bxv + Byv * Byv;
    if (value_of(B2) == 0.0) return r;
    T H = Po * T(M_ELECTRON) / T(C_LIGHT);
    T irho2 = B2 / (H * H);
    T dFactor = (T(1.0) + r[5]) * (T(1.0) + r[5]);
    T dDelta = -srCoef * dFactor * irho2 * dl;
    T scale = T(1.0) + dDelta;
    return V6<T>{{r[0], r[1] * scale, r[2], r[3] * scale, r[4], r[5] + dDelta}};
}

template <class T>
inline V6<T> wig_rad_block(const Wig<T>& w, V6<T> r, T Zw, T Aw, T Po, T srCoef, T SL) {
    T ax, axpy, ay, aypx, Bxv, Byv;
    wig_ax_axpy(w, r[0], r[2], Zw, Aw, Po, ax, axpy);
    wig_ay_aypx(w, r[0], r[2], Zw, Aw, Po, ay, aypx);
    r = V6<T>{{r[0], r[1] - ax, r[2], r[3] - ay, r[4], r[5]}};
    wig_B(w, r[0], r[2], Zw, Bxv, Byv);
    r = wig_rad_kick(r, Bxv, Byv, Po, srCoef, SL);
    return V6<T>{{r[0], r[1] + ax, r[2], r[3] + ay, r[4], r[5]}};
}

// _wig_pass_4th :1380-1398 and _wig_pass_4th_rad :1465-1503; pass!(::Wiggler) :1509-1525
template <class T>
inline V6<T> pass_wiggler(const Elem<T>& e, V6<T> r) {
    using std::sqrt;
    r = entrance(e, r);
    Wig<T> w = wig_of(e);
    const int rad = int(e.aux[2]);
    const int PN = e.num_int_steps;
    const long Nw = long(std::nearbyint(value_of(e.L) / value_of(w.lw)));  // round(Int, L/lw): half to even
    const long Nstep = long(PN) * std::max(1L, Nw);
    T dl = w.lw / T(double(PN));
    T dl1 = dl * T(1.3512071919596573);
    T dl0 = dl * T(-1.7024143839193146);
    T energy = e.param[2];
    T Aw = T(1e-9) * T(C_LIGHT) / (T(M_ELECTRON) * T(1e-9)) / T(TWO_PI) * w.lw * w.bmax;
    T Zw = T(0.0);
    if (rad == 1) {
        T gamma = energy / T(M_ELECTRON);
        T Po = sqrt(gamma * gamma - T(1.0));
        T srCoef = T(2.0 / 3.0) * T(2.8179403205e-15) * (gamma * gamma * gamma);
        r = wig_rad_block(w, r, Zw, Aw, Po, srCoef, dl);
        for (long s = 0; s < Nstep; ++s) {
            r = wig_map_2nd(w, r, dl1, Zw, Aw, Po);
            r = wig_map_2nd(w, r, dl0, Zw, Aw, Po);
            r = wig_map_2nd(w, r, dl1, Zw, Aw, Po);
            r = wig_rad_block(w, r, Zw, Aw, Po, srCoef, dl);
        }
    } else {
        T Po = sqrt((energy / T(M_ELECTRON)) * (energy / T(M_ELECTRON)) - T(1.0));
        for (long s = 0; s < Nstep; ++s) {
            r = wig_map_2nd(w, r, dl1, Zw, Aw, Po);
            r = wig_map_2nd(w, r, dl0, Zw, Aw, Po);
            r = wig_map_2nd(w, r, dl1, Zw, Aw, Po);
        }
    }
    return exit_(e, r);
}

// ---------------------------------------------------------------------------
// pass! dispatch (multiple dispatch in the reference)
// ---------------------------------------------------------------------------
template <class T>
inline V6<T> pass(const Elem<T>& e, const V6<T>& r, T beti, bool exact) {
    switch (e.kind) {
        case TP_MARKER: return r;
        case TP_DRIFT: case TP_DRIFT_SC: return pass_drift(e, r, beti, exact);
        case TP_QUADRUPOLE: return pass_quad(e, r, beti, exact);
        case TP_SEXTUPOLE: return pass_sext(e, r, beti, exact);
        case TP_OCTUPOLE: return pass_oct(e, r, beti, exact);
        case TP_THIN_MULTIPOLE: return pass_thin_multipole(e, r);
        case TP_SBEND: return pass_sbend(e, r, beti, exact);
        case TP_EXACT_SBEND: return pass_exact_sbend(e, r, beti);
        case TP_RFCAVITY: return pass_rf(e, r, beti, exact);
        case TP_SOLENOID: return pass_solenoid(e, r, beti, exact);
        case TP_CORRECTOR: return pass_corrector(e, r);
        case TP_TRANSLATION: return pass_translation(e, r, beti);
        case TP_YROTATION: return pass_yrotation(e, r, beti);
        case TP_CRAB_CAVITY: return pass_crab(e, r, beti, exact);
        case TP_ACCEL_CAVITY: return pass_accel(e, r, beti);
        case TP_LONGITUDINAL_RF_MAP: return pass_long_rf_map(e, r, beti);
        case TP_LORENTZ_BOOST: return pass_lorentz(e, r, false);
        case TP_INV_LORENTZ_BOOST: return pass_lorentz(e, r, true);
        case TP_SPACE_CHARGE: return r;
        case TP_QUADRUPOLE_SC: return pass_multipole_sc(e, r, beti, exact, true);
        case TP_SEXTUPOLE_SC: case TP_OCTUPOLE_SC: return pass_multipole_sc(e, r, beti, exact, false);
        case TP_SBEND_SC: return pass_sbend_sc(e, r, beti, exact);
        case TP_STRONG_THIN_GAUSSIAN_BEAM: return pass_strong_thin_gaussian(e, r);
        case TP_LBEND: return pass_lbend(e, r);
        case TP_STRONG_GAUSSIAN_BEAM: return pass_strong_gaussian(e, r);
        case TP_LONGITUDINAL_RLC_WAKE: return pass_rlc_wake(e, r);
        case TP_LONGITUDINAL_WAKE: return pass_tab_wake(e, r);
        case TP_WIGGLER: return pass_wiggler(e, r);
        default: return nan6<T>();
    }
}

// ---------------------------------------------------------------------------
// Beam: src/lattice.jl:50-61
// ---------------------------------------------------------------------------
inline double beam_beti(double energy, double mass) {
    double gamma = (energy + mass) / mass;
    double beta = std::sqrt(1.0 - 1.0 / (gamma * gamma));
    return 1.0 / beta;
}

// ---------------------------------------------------------------------------
// Time schedule (materialize at each turn): src/time_dependence.jl:163-178
// ---------------------------------------------------------------------------
struct Schedule {
    std::vector<int32_t> fields;  // pairs (element, field)
    int32_t turn0 = 0, nturns = 0;
    std::vector<double> values;   // nturns x nfields
    int nfields() const { return int(fields.size() / 2); }
};

inline void apply_field(tp_elem& e, int field, double v) {
    switch (field) {
        case TP_FIELD_L: e.L = v; break;
        case TP_FIELD_K: e.k = v; break;
        case TP_FIELD_ANGLE: e.angle = v; break;
        case TP_FIELD_E1: e.e1 = v; break;
        case TP_FIELD_E2: e.e2 = v; break;
        case TP_FIELD_VOLT: e.volt = v; break;
        case TP_FIELD_FREQ: e.freq = v; break;
        case TP_FIELD_LAG: e.lag = v; break;
        case TP_FIELD_PHILAG: e.philag = v; break;
        case TP_FIELD_ENERGY: e.energy = v; break;
        case TP_FIELD_NUM_INT_STEPS: e.num_int_steps = int(v); break;
        default:
            if (field >= TP_FIELD_POLYNOM_A0 && field < TP_FIELD_POLYNOM_A0 + 4)
                e.polynom_a[field - TP_FIELD_POLYNOM_A0] = v;
            else if (field >= TP_FIELD_POLYNOM_B0 && field < TP_FIELD_POLYNOM_B0 + 4)
                e.polynom_b[field - TP_FIELD_POLYNOM_B0] = v;
            break;
    }
}

// ---------------------------------------------------------------------------
// Multi-particle drivers
// ---------------------------------------------------------------------------
struct Aperture {
    double ax = 0.0, ay = 0.0;  // <= 0 disables
    bool lost(double x, double y) const {
        return (ax > 0.0 && std::fabs(x) > ax) || (ay > 0.0 && std::fabs(y) > ay);
    }
    // Distance of this check to the nearest loss threshold (reference limits
    // and aperture), used to excuse flips within a tolerance of an edge.
    double edge_distance(const double* r) const {
        double d = std::fabs(std::fabs(r[0]) - COORD_LIMIT);
        d = std::min(d, std::fabs(std::fabs(r[2]) - COORD_LIMIT));
        d = std::min(d, std::fabs(std::fabs(r[1]) - ANGLE_LIMIT));
        d = std::min(d, std::fabs(std::fabs(r[3]) - ANGLE_LIMIT));
        if (ax > 0.0) d = std::min(d, std::fabs(std::fabs(r[0]) - ax));
        if (ay > 0.0) d = std::min(d, std::fabs(std::fabs(r[2]) - ay));
        return d;
    }
};

struct Lattice {
    std::vector<tp_elem> elems;
    std::vector<tp_misalign> mis;
    std::vector<double> aux;  // array fields of the elements
    Schedule sched;

    // Element `i` as materialised at turn `turn`.
    Elem<double> at(int64_t i, int32_t turn) const {
        tp_elem e = elems[size_t(i)];
        int nf = sched.nfields();
        if (nf > 0) {
            int64_t row = int64_t(turn) - sched.turn0;
            if (row >= 0 && row < sched.nturns) {
                for (int j = 0; j < nf; ++j)
                    if (sched.fields[2 * j] == i)
                        apply_field(e, sched.fields[2 * j + 1], sched.values[size_t(row * nf + j)]);
            }
        }
        const tp_misalign* m = (e.misalign_index >= 0) ? &mis[size_t(e.misalign_index)] : nullptr;
        return make_elem<double>(e, m, aux.empty() ? nullptr : aux.data());
    }
};

// One particle through one pass of the lattice, following linepass!'s per
// particle body (src/lattice.jl:266-293).  Returns true when lost; on loss the
// state keeps its value at the entrance of element `*lost_elem`.
inline bool track_one_pass(const Lattice& lat, const std::vector<Elem<double>>& elems, double* r6, double beti,
                           bool exact, const Aperture& ap, int32_t* lost_elem, double* min_edge) {
    V6<double> r{{r6[0], r6[1], r6[2], r6[3], r6[4], r6[5]}};
    for (size_t e = 0; e < elems.size(); ++e) {
        V6<double> rn = pass(elems[e], r, beti, exact);
        if (min_edge) *min_edge = std::min(*min_edge, ap.edge_distance(rn.v));
        if (check_lost(rn) || ap.lost(rn[0], rn[2])) {
            *lost_elem = int32_t(e);
            for (int c = 0; c < 6; ++c) r6[c] = r[c];
            return true;
        }
        r = rn;
    }
    (void)lat;
    for (int c = 0; c < 6; ++c) r6[c] = r[c];
    return false;
}

}  // namespace tpo

// tp_tpsa_oracle.hpp -- CPU oracle for truncated power series (TPSA) tracking.
//
// TEST INFRASTRUCTURE ONLY, like tp_oracle.hpp: loaded by the tests, never by
// the shipped library.
//
// What it restates: the TPSA extension of TrackPad.jl
// (ext/TrackPadPolySeriesExt.jl), which tracks a vector of six CTPS values of
// the third-party PolySeries package (not vendored with the reference) through
// the pass! methods.  The extension's pass! bodies are the particle bodies of
// src/tracking.jl evaluated in CTPS arithmetic, except for three places that
// tp_oracle.hpp special-cases when is_tps<T> holds: the drift is always the
// exact one (drift6_tpsa, :57-65), the bend edges take fy from the constant
// parts of delta and px (:161-215), and the wakes are evaluated at the
// constant part of z (:630-649).  So the oracle's templated pass! bodies run
// unchanged on the Tps type below.
//
// Tps: PolySeries's published algorithm for truncated power series in
// nv = 6 variables (x, px, y, py, z, delta) to total order N, restated:
//   * a series holds the coefficients of the M = C(N+6, 6) monomials of
//     degree <= N, ordered by degree, and within a degree by exponent vector
//     in descending lexicographic order (x^d first, delta^d last);
//   * products are truncated at order N: c_k = sum over the pairs (i, j) with
//     monomial_i * monomial_j = monomial_k, taken in increasing i;
//   * a function f of a series a = a0 + abar (abar without constant term) is
//     its Taylor series sum_k f^(k)(a0)/k! abar^k, evaluated by Horner's rule
//     with N products: inv, sqrt, a^(-1/2), exp, sin, cos;
//   * a / b is a * inv(b); a series divided by a number divides every
//     coefficient.
// A number is kept as a one-coefficient series, so element constants cost no
// more than doubles.
//
// Parity: no PolySeries output is available here; the restatement is pinned
// by series identities (sqrt(a)^2 = a, sin^2 + cos^2 = 1, exp(a) exp(-a) = 1,
// inv(a) a = 1), by its first-order part against the dual-number Jacobian of
// the particle maps, and by its second-order part against finite differences
// of that Jacobian (tests/test_tpsa_oracle.py).
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "tp_oracle.hpp"

namespace tpo {

struct TpsDesc {
    int N = -1;
    int M = 0;
    std::vector<std::array<int, 6>> mono;
    std::vector<int32_t> poff;  // M + 1
    std::vector<int32_t> pi, pj;
};

inline TpsDesc& tps_desc() {
    static TpsDesc d;
    return d;
}

inline uint64_t tps_key(const std::array<int, 6>& e) {
    uint64_t k = 0;
    for (int v = 0; v < 6; ++v) k = k * 64u + uint64_t(e[size_t(v)]);
    return k;
}

// Exponent vectors of total degree `deg` in descending lexicographic order.
inline void tps_enumerate(int deg, int v, std::array<int, 6>& cur, std::vector<std::array<int, 6>>* out) {
    if (v == 5) {
        cur[5] = deg;
        out->push_back(cur);
        return;
    }
    for (int e = deg; e >= 0; --e) {
        cur[size_t(v)] = e;
        tps_enumerate(deg - e, v + 1, cur, out);
    }
}

inline void tps_set_order(int N) {
    TpsDesc& d = tps_desc();
    if (d.N == N) return;
    d = TpsDesc{};
    d.N = N;
    std::array<int, 6> cur{};
    for (int deg = 0; deg <= N; ++deg) tps_enumerate(deg, 0, cur, &d.mono);
    d.M = int(d.mono.size());
    std::unordered_map<uint64_t, int> index;
    for (int k = 0; k < d.M; ++k) index[tps_key(d.mono[size_t(k)])] = k;
    d.poff.assign(size_t(d.M) + 1, 0);
    for (int k = 0; k < d.M; ++k) {
        const auto& mk = d.mono[size_t(k)];
        for (int i = 0; i < d.M; ++i) {
            const auto& mi = d.mono[size_t(i)];
            std::array<int, 6> mj{};
            bool ok = true;
            for (int v = 0; v < 6 && ok; ++v) {
                mj[size_t(v)] = mk[size_t(v)] - mi[size_t(v)];
                ok = mj[size_t(v)] >= 0;
            }
            if (!ok) continue;
            d.pi.push_back(i);
            d.pj.push_back(index.at(tps_key(mj)));
        }
        d.poff[size_t(k) + 1] = int32_t(d.pi.size());
    }
}

struct Tps {
    std::vector<double> c;  // one coefficient: a number; else M coefficients
    Tps() : c(1, 0.0) {}
    Tps(double v) : c(1, v) {}
    bool is_const() const { return c.size() == 1; }
    static Tps full() {
        Tps t;
        t.c.assign(size_t(tps_desc().M), 0.0);
        return t;
    }
    // CTPS(x0, i): the variable i (0-based) about x0
    static Tps var(double x0, int i) {
        Tps t = full();
        t.c[0] = x0;
        t.c[size_t(1 + i)] = 1.0;
        return t;
    }
};

template <>
struct is_tps<Tps> : std::true_type {};

inline double value_of(const Tps& a) { return a.c[0]; }
inline bool is_nan(const Tps& a) { return std::isnan(a.c[0]); }

inline Tps operator+(const Tps& a, const Tps& b) {
    if (a.is_const() && b.is_const()) return Tps(a.c[0] + b.c[0]);
    if (a.is_const()) {
        Tps r = b;
        r.c[0] = a.c[0] + b.c[0];
        return r;
    }
    if (b.is_const()) {
        Tps r = a;
        r.c[0] = a.c[0] + b.c[0];
        return r;
    }
    Tps r = a;
    for (size_t k = 0; k < r.c.size(); ++k) r.c[k] = a.c[k] + b.c[k];
    return r;
}

inline Tps operator-(const Tps& a) {
    Tps r = a;
    for (double& v : r.c) v = -v;
    return r;
}

inline Tps operator-(const Tps& a, const Tps& b) {
    if (a.is_const() && b.is_const()) return Tps(a.c[0] - b.c[0]);
    if (a.is_const()) {
        Tps r = -b;
        r.c[0] = a.c[0] - b.c[0];
        return r;
    }
    if (b.is_const()) {
        Tps r = a;
        r.c[0] = a.c[0] - b.c[0];
        return r;
    }
    Tps r = a;
    for (size_t k = 0; k < r.c.size(); ++k) r.c[k] = a.c[k] - b.c[k];
    return r;
}

inline Tps scale(const Tps& a, double s) {
    Tps r = a;
    for (double& v : r.c) v = v * s;
    return r;
}

inline Tps operator*(const Tps& a, const Tps& b) {
    if (a.is_const()) return scale(b, a.c[0]);
    if (b.is_const()) return scale(a, b.c[0]);
    const TpsDesc& d = tps_desc();
    Tps r = Tps::full();
    for (int k = 0; k < d.M; ++k) {
        int p = d.poff[size_t(k)];
        double s = a.c[size_t(d.pi[size_t(p)])] * b.c[size_t(d.pj[size_t(p)])];
        for (++p; p < d.poff[size_t(k) + 1]; ++p) s = s + a.c[size_t(d.pi[size_t(p)])] * b.c[size_t(d.pj[size_t(p)])];
        r.c[size_t(k)] = s;
    }
    return r;
}

// Taylor coefficients c[0..N] of the supported functions about a0.
enum TpsFn { TF_INV, TF_SQRT, TF_RSQRT, TF_EXP, TF_SIN, TF_COS };

inline void tps_fn_coef(TpsFn f, double a0, int N, double* c) {
    switch (f) {
        case TF_INV:
            c[0] = 1.0 / a0;
            for (int k = 1; k <= N; ++k) c[k] = -c[k - 1] / a0;
            break;
        case TF_SQRT:
            c[0] = std::sqrt(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] * (0.5 - double(k - 1)) / (double(k) * a0);
            break;
        case TF_RSQRT:
            c[0] = 1.0 / std::sqrt(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] * (-0.5 - double(k - 1)) / (double(k) * a0);
            break;
        case TF_EXP:
            c[0] = tp::libm::exp(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] / double(k);
            break;
        case TF_SIN:
        case TF_COS: {
            const double s0 = tp::libm::sin(a0), c0 = tp::libm::cos(a0);
            const double cyc_s[4] = {s0, c0, -s0, -c0};
            const double cyc_c[4] = {c0, -s0, -c0, s0};
            const double* cyc = f == TF_SIN ? cyc_s : cyc_c;
            double fact = 1.0;
            c[0] = cyc[0];
            for (int k = 1; k <= N; ++k) {
                fact = fact * double(k);
                c[k] = cyc[k & 3] / fact;
            }
            break;
        }
    }
}

inline Tps tps_apply(TpsFn f, const Tps& a) {
    const int N = tps_desc().N;
    std::vector<double> c(size_t(N) + 1);
    tps_fn_coef(f, a.c[0], N, c.data());
    if (a.is_const()) return Tps(c[0]);
    Tps abar = a;
    abar.c[0] = 0.0;
    Tps r(c[size_t(N)]);
    for (int k = N - 1; k >= 0; --k) {
        r = r * abar;
        r = r + Tps(c[size_t(k)]);
    }
    return r;
}

inline Tps inv(const Tps& a) { return tps_apply(TF_INV, a); }
inline Tps sqrt(const Tps& a) { return tps_apply(TF_SQRT, a); }
inline Tps rsqrt(const Tps& a) { return tps_apply(TF_RSQRT, a); }
inline Tps exp(const Tps& a) { return tps_apply(TF_EXP, a); }
inline Tps sin(const Tps& a) { return tps_apply(TF_SIN, a); }
inline Tps cos(const Tps& a) { return tps_apply(TF_COS, a); }

inline Tps operator/(const Tps& a, const Tps& b) {
    if (b.is_const()) {
        Tps r = a;
        for (double& v : r.c) v = v / b.c[0];
        return r;
    }
    return a * inv(b);
}

// Functions the particle bodies apply to element constants only.
inline Tps tan(const Tps& a) {
    if (!a.is_const()) throw std::runtime_error("tan of a series is not used by the TPSA pass! methods");
    return Tps(tp::libm::tan(a.c[0]));
}
// |a| by the sign of the constant part (the particle bodies only compare it).
inline Tps abs(const Tps& a) { return a.c[0] < 0.0 ? -a : a; }

// The element kinds the extension defines pass! methods for.
inline bool tpsa_supported(int kind) {
    switch (kind) {
        case TP_EXACT_SBEND: case TP_LBEND: case TP_WIGGLER: return false;
        default: return kind >= 0 && kind < TP_KIND_COUNT;
    }
}

inline V6<Tps> tpsa_pass(const Elem<Tps>& e, const V6<Tps>& r, const Tps& beti) {
    switch (e.kind) {
        case TP_MARKER: case TP_SPACE_CHARGE: return r;
        case TP_DRIFT: case TP_DRIFT_SC: return pass_drift(e, r, beti, true);
        case TP_QUADRUPOLE: return pass_quad(e, r, beti, true);
        case TP_SEXTUPOLE: return pass_sext(e, r, beti, true);
        case TP_OCTUPOLE: return pass_oct(e, r, beti, true);
        case TP_THIN_MULTIPOLE: return pass_thin_multipole(e, r);
        case TP_SBEND: return pass_sbend(e, r, beti, true);
        case TP_RFCAVITY: return pass_rf(e, r, beti, true);
        case TP_SOLENOID: return pass_solenoid(e, r, beti, true);
        case TP_CORRECTOR: return pass_corrector(e, r);
        case TP_TRANSLATION: return pass_translation(e, r, beti);
        case TP_YROTATION: return pass_yrotation(e, r, beti);
        case TP_CRAB_CAVITY: return pass_crab(e, r, beti, true);
        case TP_ACCEL_CAVITY: return pass_accel(e, r, beti);
        case TP_LONGITUDINAL_RF_MAP: return pass_long_rf_map(e, r, beti);
        case TP_LORENTZ_BOOST: return pass_lorentz(e, r, false);
        case TP_INV_LORENTZ_BOOST: return pass_lorentz(e, r, true);
        case TP_QUADRUPOLE_SC: return pass_multipole_sc(e, r, beti, true, true);
        case TP_SEXTUPOLE_SC: case TP_OCTUPOLE_SC: return pass_multipole_sc(e, r, beti, true, false);
        case TP_SBEND_SC: return pass_sbend_sc(e, r, beti, true);
        case TP_STRONG_THIN_GAUSSIAN_BEAM: return pass_strong_thin_gaussian(e, r);
        case TP_STRONG_GAUSSIAN_BEAM: return pass_strong_gaussian(e, r);
        case TP_LONGITUDINAL_RLC_WAKE: return pass_rlc_wake(e, r);
        case TP_LONGITUDINAL_WAKE: return pass_tab_wake(e, r);
        default: throw std::runtime_error("element kind without a TPSA pass! method");
    }
}

}  // namespace tpo

// tp_oracle_capi.cpp -- C entry points of the CPU oracle (ctypes-callable).
//
// TEST INFRASTRUCTURE ONLY: loaded by the tests, the smoke check and the
// benchmark's CPU-baseline leg; never by the shipped library.
//
// Drivers follow src/lattice.jl:260-317 of TrackPad.jl: turns outer, elements
// next, particles innermost, lost particles skipped (`lost_flags[i] == 1`),
// coordinates not written back on loss.  The multi-threaded variant splits the
// particle loop of each element across OpenMP threads; per-particle results
// are identical to the single-threaded loop.
//
// Parity status: unpinned against reference outputs (see tp_oracle.hpp).
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "tp_oracle.hpp"
#include "tp_tpsa_oracle.hpp"

// ---------------------------------------------------------------------------
// Op-counting scalar: the algorithmic FLOP table.  Rules: add/sub/mul/div/sqrt
// count 1, each transcendental call counts TP_FLOPS_PER_TRANSCENDENTAL;
// negation, abs and comparisons count 0.  The oracle never fuses.
// ---------------------------------------------------------------------------
namespace tpo {
struct Cnt {
    double v;
    Cnt() : v(0.0) {}
    Cnt(double x) : v(x) {}
};
static thread_local double g_flops = 0.0;
static thread_local double g_transc = 0.0;
inline double value_of(const Cnt& x) { return x.v; }
inline bool is_nan(const Cnt& x) { return std::isnan(x.v); }
inline Cnt operator+(Cnt a, Cnt b) { g_flops += 1; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { g_flops += 1; return Cnt(a.v - b.v); }
inline Cnt operator*(Cnt a, Cnt b) { g_flops += 1; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { g_flops += 1; return Cnt(a.v / b.v); }
inline Cnt operator-(Cnt a) { return Cnt(-a.v); }
inline Cnt sqrt(Cnt a) { g_flops += 1; return Cnt(std::sqrt(a.v)); }
inline Cnt abs(Cnt a) { return Cnt(std::fabs(a.v)); }
#define TPO_CNT_TRANSC(fn)                                   \
    inline Cnt fn(Cnt a) {                                   \
        g_flops += TP_FLOPS_PER_TRANSCENDENTAL; g_transc += 1; \
        return Cnt(tpo::fn(a.v));                            \
    }
TPO_CNT_TRANSC(sin)
TPO_CNT_TRANSC(cos)
TPO_CNT_TRANSC(tan)
TPO_CNT_TRANSC(asin)
TPO_CNT_TRANSC(atan)
#undef TPO_CNT_TRANSC
inline Cnt exp(Cnt a) { g_flops += TP_FLOPS_PER_TRANSCENDENTAL; g_transc += 1; return Cnt(tpo::exp(a.v)); }
inline Cnt sinh(Cnt a) { g_flops += TP_FLOPS_PER_TRANSCENDENTAL; g_transc += 1; return Cnt(tpo::sinh(a.v)); }
inline Cnt cosh(Cnt a) { g_flops += TP_FLOPS_PER_TRANSCENDENTAL; g_transc += 1; return Cnt(tpo::cosh(a.v)); }

// ---------------------------------------------------------------------------
// Forward-mode dual number with one tangent (independent AD of the oracle).
// ---------------------------------------------------------------------------
struct D1 {
    double v, d;
    D1() : v(0.0), d(0.0) {}
    D1(double x) : v(x), d(0.0) {}
    D1(double x, double dx) : v(x), d(dx) {}
};
inline double value_of(const D1& x) { return x.v; }
inline bool is_nan(const D1& x) { return std::isnan(x.v); }
inline D1 operator+(D1 a, D1 b) { return D1(a.v + b.v, a.d + b.d); }
inline D1 operator-(D1 a, D1 b) { return D1(a.v - b.v, a.d - b.d); }
inline D1 operator*(D1 a, D1 b) { return D1(a.v * b.v, a.d * b.v + a.v * b.d); }
inline D1 operator/(D1 a, D1 b) { double q = a.v / b.v; return D1(q, (a.d - q * b.d) / b.v); }
inline D1 operator-(D1 a) { return D1(-a.v, -a.d); }
inline D1 sqrt(D1 a) { double s = std::sqrt(a.v); return D1(s, a.d / (2.0 * s)); }
inline D1 abs(D1 a) { return a.v < 0.0 ? -a : a; }
inline D1 sin(D1 a) { return D1(tpo::sin(a.v), tpo::cos(a.v) * a.d); }
inline D1 cos(D1 a) { return D1(tpo::cos(a.v), -tpo::sin(a.v) * a.d); }
inline D1 tan(D1 a) { double t = tpo::tan(a.v); return D1(t, (1.0 + t * t) * a.d); }
inline D1 asin(D1 a) { return D1(tpo::asin(a.v), a.d / std::sqrt(1.0 - a.v * a.v)); }
inline D1 atan(D1 a) { return D1(tpo::atan(a.v), a.d / (1.0 + a.v * a.v)); }
inline D1 exp(D1 a) { double e = tpo::exp(a.v); return D1(e, e * a.d); }
inline D1 sinh(D1 a) { return D1(tpo::sinh(a.v), tpo::cosh(a.v) * a.d); }
inline D1 cosh(D1 a) { return D1(tpo::cosh(a.v), tpo::sinh(a.v) * a.d); }
}  // namespace tpo

using namespace tpo;

namespace {

struct Inputs {
    const tp_elem* elems;
    int64_t ne;
    const tp_misalign* mis;
    int64_t nmis;
    const int32_t* sfields;
    int32_t nfields;
    int32_t sturn0;
    int32_t snturns;
    const double* svalues;
};

// Array fields of the elements of the next calls (tp_lattice_create_ex's aux),
// set by orc_set_aux.
std::vector<double> g_aux;
std::string g_tpsa_error;  // message of the last failed TPSA call

Lattice build_lattice(const Inputs& in) {
    Lattice lat;
    lat.aux = g_aux;
    lat.elems.assign(in.elems, in.elems + in.ne);
    if (in.nmis > 0) lat.mis.assign(in.mis, in.mis + in.nmis);
    if (in.nfields > 0) {
        lat.sched.fields.assign(in.sfields, in.sfields + 2 * in.nfields);
        lat.sched.turn0 = in.sturn0;
        lat.sched.nturns = in.snturns;
        lat.sched.values.assign(in.svalues, in.svalues + size_t(in.snturns) * size_t(in.nfields));
    }
    return lat;
}

template <class T>
Elem<T> elem_at(const Lattice& lat, int64_t i, int32_t turn) {
    tp_elem e = lat.elems[size_t(i)];
    int nf = lat.sched.nfields();
    if (nf > 0) {
        int64_t row = int64_t(turn) - lat.sched.turn0;
        if (row >= 0 && row < lat.sched.nturns)
            for (int j = 0; j < nf; ++j)
                if (lat.sched.fields[2 * j] == i)
                    apply_field(e, lat.sched.fields[2 * j + 1], lat.sched.values[size_t(row * nf + j)]);
    }
    const tp_misalign* m = (e.misalign_index >= 0) ? &lat.mis[size_t(e.misalign_index)] : nullptr;
    return make_elem<T>(e, m, lat.aux.empty() ? nullptr : lat.aux.data());
}

}  // namespace

extern "C" {

double orc_beam_beti(double energy, double mass) { return beam_beti(energy, mass); }

int orc_max_threads(void) { return omp_get_max_threads(); }

// The aux array (array fields of StrongGaussianBeam, LongitudinalWake and
// Wiggler elements) used by the following calls; n = 0 clears it.
void orc_set_aux(const double* aux, int64_t n) {
    if (n > 0 && aux) g_aux.assign(aux, aux + n);
    else g_aux.clear();
}

// Markstein's reciprocal division q' = RN(q + r*y), q = RN(a*y), r = a - b*q,
// y = RN(1/b), compared with IEEE a/b on n pairs: returns the number that differ.
int64_t orc_check_rcp_div(const double* a, const double* b, int64_t n) {
    int64_t bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        double y = 1.0 / b[i];
        double q = a[i] * y;
        double r = std::fma(-q, b[i], a[i]);
        double q1 = std::fma(r, y, q);
        double ref = a[i] / b[i];
        if (!(q1 == ref || (std::isnan(q1) && std::isnan(ref)))) ++bad;
    }
    return bad;
}

// The shared transcendental functions (which: 0 asin, 1 sin, 2 cos, 3 tan,
// 4 atan, 5 exp, 6 expm1, 7 sinh, 8 cosh) and the C library's, on n arguments, for the accuracy tests.
void orc_libm(int32_t which, const double* x, int64_t n, double* ours, double* clib) {
    for (int64_t i = 0; i < n; ++i) {
        switch (which) {
            case 0: ours[i] = tp::libm::asin(x[i]); clib[i] = std::asin(x[i]); break;
            case 1: ours[i] = tp::libm::sin(x[i]); clib[i] = std::sin(x[i]); break;
            case 2: ours[i] = tp::libm::cos(x[i]); clib[i] = std::cos(x[i]); break;
            case 3: ours[i] = tp::libm::tan(x[i]); clib[i] = std::tan(x[i]); break;
            case 5: ours[i] = tp::libm::exp(x[i]); clib[i] = std::exp(x[i]); break;
            case 6: ours[i] = tp::libm::expm1(x[i]); clib[i] = std::expm1(x[i]); break;
            case 7: ours[i] = tp::libm::sinh(x[i]); clib[i] = std::sinh(x[i]); break;
            case 8: ours[i] = tp::libm::cosh(x[i]); clib[i] = std::cosh(x[i]); break;
            default: ours[i] = tp::libm::atan(x[i]); clib[i] = std::atan(x[i]); break;
        }
    }
}

// ringpass! (src/lattice.jl:305-317) over linepass! (:260-297) with the
// reference loop order.  lost_turn / lost_elem / min_edge may be NULL.
// min_edge[i] receives the smallest distance of any loss check of particle i
// to a loss threshold (reference limits and aperture).
int orc_ringpass(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis,
                 const int32_t* sfields, int32_t nfields, int32_t sturn0, int32_t snturns,
                 const double* svalues, double* coords, int64_t n, int64_t* lost,
                 int32_t* lost_turn, int32_t* lost_elem, double* min_edge, double beti,
                 int32_t nturns, int32_t turn0, int32_t exact, double ax, double ay, int32_t nthreads) {
    if (n < 0 || ne < 0 || nturns < 0) return -1;
    Inputs in{elems, ne, mis, nmis, sfields, nfields, sturn0, snturns, svalues};
    Lattice lat = build_lattice(in);
    Aperture ap{ax, ay};
    const bool ex = exact != 0;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    std::vector<Elem<double>> el(static_cast<size_t>(ne));
    for (int32_t t = 0; t < nturns; ++t) {
        const int32_t turn = turn0 + t;
        for (int64_t e = 0; e < ne; ++e) el[size_t(e)] = elem_at<double>(lat, e, turn);  // _resolve_for_time
        for (int64_t e = 0; e < ne; ++e) {
            const Elem<double>& E = el[size_t(e)];
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
            for (int64_t i = 0; i < n; ++i) {
                if (lost[i] == 1) continue;
                V6<double> r{{coords[i], coords[n + i], coords[2 * n + i], coords[3 * n + i],
                              coords[4 * n + i], coords[5 * n + i]}};
                V6<double> rn = pass(E, r, beti, ex);
                if (min_edge) min_edge[i] = std::min(min_edge[i], ap.edge_distance(rn.v));
                if (check_lost(rn) || ap.lost(rn[0], rn[2])) {
                    lost[i] = 1;
                    if (lost_turn) lost_turn[i] = turn;
                    if (lost_elem) lost_elem[i] = int32_t(e);
                    continue;
                }
                for (int c = 0; c < 6; ++c) coords[c * n + i] = rn[c];
            }
        }
    }
    return 0;
}

// Algorithmic FLOPs of one particle through each element once (counted with
// the Cnt scalar), starting from state r0 and carrying the state along.
int orc_count_flops(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis, double beti,
                    int32_t exact, const double* r0, double* flops_out, double* transc_out) {
    Inputs in{elems, ne, mis, nmis, nullptr, 0, 0, 0, nullptr};
    Lattice lat = build_lattice(in);
    V6<Cnt> r{{Cnt(r0[0]), Cnt(r0[1]), Cnt(r0[2]), Cnt(r0[3]), Cnt(r0[4]), Cnt(r0[5])}};
    for (int64_t e = 0; e < ne; ++e) {
        Elem<Cnt> E = elem_at<Cnt>(lat, e, 0);
        g_flops = 0.0;
        g_transc = 0.0;
        V6<Cnt> rn = pass(E, r, Cnt(beti), exact != 0);
        flops_out[e] = g_flops;
        if (transc_out) transc_out[e] = g_transc;
        if (!check_lost(rn)) r = rn;
    }
    return 0;
}

// Tangent (6x6 Jacobian) of nturns passes about each orbit, forward mode with
// one tangent per column.  jac: n x 36, M[i,j] at j*6+i.  Lost orbits give NaN.
int orc_jacobian(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis,
                 const int32_t* sfields, int32_t nfields, int32_t sturn0, int32_t snturns,
                 const double* svalues, const double* orbits, int64_t n, double beti, int32_t nturns,
                 int32_t turn0, int32_t exact, double* jac) {
    Inputs in{elems, ne, mis, nmis, sfields, nfields, sturn0, snturns, svalues};
    Lattice lat = build_lattice(in);
    for (int64_t i = 0; i < n; ++i) {
        for (int j = 0; j < 6; ++j) {
            V6<D1> r;
            for (int c = 0; c < 6; ++c) r[c] = D1(orbits[c * n + i], c == j ? 1.0 : 0.0);
            bool lostp = false;
            for (int32_t t = 0; t < nturns && !lostp; ++t)
                for (int64_t e = 0; e < ne; ++e) {
                    Elem<D1> E = elem_at<D1>(lat, e, turn0 + t);
                    V6<D1> rn = pass(E, r, D1(beti), exact != 0);
                    if (check_lost(rn)) { lostp = true; break; }
                    r = rn;
                }
            for (int c = 0; c < 6; ++c) jac[i * 36 + j * 6 + c] = lostp ? NAN : r[c].d;
        }
    }
    return 0;
}

// Loss of the adjoint entry point and its derivative with respect to the main
// strength `k` of element `param_elem` (forward-mode dual), evaluated on the
// particles that survive all turns.  loss = mean_s (x^2+y^2)/sigma^2
// + lost_weight * lost/alive0.  dloss may be NULL (value only).
int orc_loss_and_dk(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis,
                    const int32_t* sfields, int32_t nfields, int32_t sturn0, int32_t snturns,
                    const double* svalues, const double* coords0, int64_t n, const int64_t* lost0,
                    double beti, int32_t nturns, int32_t turn0, int32_t exact, double ax, double ay,
                    double sigma, double lost_weight, int32_t param_elem, int32_t nthreads,
                    double* loss, double* dloss, int64_t* survivors) {
    Inputs in{elems, ne, mis, nmis, sfields, nfields, sturn0, snturns, svalues};
    Lattice lat = build_lattice(in);
    Aperture ap{ax, ay};
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    double sum_v = 0.0, sum_d = 0.0;
    int64_t alive0 = 0, surv = 0;
    for (int64_t i = 0; i < n; ++i) alive0 += (lost0 == nullptr || lost0[i] != 1) ? 1 : 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads) reduction(+ : sum_v, sum_d, surv)
    for (int64_t i = 0; i < n; ++i) {
        if (lost0 && lost0[i] == 1) continue;
        V6<D1> r;
        for (int c = 0; c < 6; ++c) r[c] = D1(coords0[c * n + i]);
        bool lostp = false;
        for (int32_t t = 0; t < nturns && !lostp; ++t)
            for (int64_t e = 0; e < ne; ++e) {
                Elem<D1> E = elem_at<D1>(lat, e, turn0 + t);
                if (e == param_elem) {
                    E.k.d = 1.0;
                    for (int f = 0; f < 4; ++f) E.param[f].d = 0.0;
                }
                V6<D1> rn = pass(E, r, D1(beti), exact != 0);
                if (check_lost(rn) || ap.lost(rn[0].v, rn[2].v)) { lostp = true; break; }
                r = rn;
            }
        if (lostp) continue;
        D1 q = (r[0] * r[0] + r[2] * r[2]) / D1(sigma * sigma);
        sum_v += q.v;
        sum_d += q.d;
        surv += 1;
    }
    double frac = alive0 > 0 ? double(alive0 - surv) / double(alive0) : 0.0;
    *loss = (surv > 0 ? sum_v / double(surv) : 0.0) + lost_weight * frac;
    if (dloss) *dloss = surv > 0 ? sum_d / double(surv) : 0.0;
    if (survivors) *survivors = surv;
    return 0;
}

// One element map applied to n particles (no loss bookkeeping): the unit
// under test for single-element parity.
int orc_pass_elements(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis, double* coords,
                      int64_t n, double beti, int32_t exact) {
    Inputs in{elems, ne, mis, nmis, nullptr, 0, 0, 0, nullptr};
    Lattice lat = build_lattice(in);
    for (int64_t i = 0; i < n; ++i) {
        V6<double> r{{coords[i], coords[n + i], coords[2 * n + i], coords[3 * n + i], coords[4 * n + i],
                      coords[5 * n + i]}};
        for (int64_t e = 0; e < ne; ++e) r = pass(elem_at<double>(lat, e, 0), r, beti, exact != 0);
        for (int c = 0; c < 6; ++c) coords[c * n + i] = r[c];
    }
    return 0;
}

// Sub-maps of the exact bend and the drift, exposed for the reversibility
// tests (which = 0 drift6, 1 exact_bend_body, 2 bend_edge, 3 yrot,
// 4 bend_fringe, 5 strthinkick with b = {0, a0, a1, 0} order 1).
int orc_submap(int32_t which, double* r6, double a0, double a1, double beti) {
    V6<double> r{{r6[0], r6[1], r6[2], r6[3], r6[4], r6[5]}};
    switch (which) {
        case 0: r = drift6(r, a0, beti, true); break;
        case 1: r = exact_bend_body(r, a0, a1, beti); break;
        case 2: r = bend_edge(r, a0, a1, beti); break;
        case 3: r = yrot(r, a0, beti); break;
        case 4: r = bend_fringe(r, a0, a1, beti); break;
        case 5: {
            double pa[4] = {0, 0, 0, 0}, pb[4] = {0, a1, 0, 0};
            r = strthinkick(r, pa, pb, a0, 1);
            break;
        }
        default: return -1;
    }
    for (int c = 0; c < 6; ++c) r6[c] = r[c];
    return 0;
}

// ---------------------------------------------------------------------------
// TPSA (ext/TrackPadPolySeriesExt.jl): series of order `order` in the six
// variables; maps are nmaps x 6 x M coefficients (M = C(order + 6, 6)).
// ---------------------------------------------------------------------------
int orc_tpsa_set_order(int32_t order) {
    if (order < 0 || order > 10) return -1;
    tps_set_order(order);
    return tps_desc().M;
}

// Exponent vectors of the monomials (M x 6), in coefficient order.
int orc_tpsa_monomials(int32_t* exps) {
    const TpsDesc& d = tps_desc();
    for (int k = 0; k < d.M; ++k)
        for (int v = 0; v < 6; ++v) exps[k * 6 + v] = d.mono[size_t(k)][size_t(v)];
    return d.M;
}

// One series operation on full series a, b (M coefficients each): op 0 a*b,
// 1 a/b, 2 inv(a), 3 sqrt(a), 4 a^(-1/2), 5 exp(a), 6 sin(a), 7 cos(a).
int orc_tpsa_op(int32_t op, const double* a, const double* b, double* out) {
    const int M = tps_desc().M;
    Tps A = Tps::full(), B = Tps::full();
    for (int k = 0; k < M; ++k) { A.c[size_t(k)] = a[k]; if (b) B.c[size_t(k)] = b[k]; }
    Tps R;
    switch (op) {
        case 0: R = A * B; break;
        case 1: R = A / B; break;
        case 2: R = inv(A); break;
        case 3: R = sqrt(A); break;
        case 4: R = rsqrt(A); break;
        case 5: R = exp(A); break;
        case 6: R = sin(A); break;
        case 7: R = cos(A); break;
        default: return -1;
    }
    for (int k = 0; k < M; ++k) out[k] = R.is_const() ? (k == 0 ? R.c[0] : 0.0) : R.c[size_t(k)];
    return 0;
}

// linepass / ringpass of series maps (ext/TrackPadPolySeriesExt.jl:654-686):
// nturns passes from turn turn0, elements resolved per turn from the schedule.
// Returns -2 for an element kind without a TPSA pass! method.
int orc_tpsa_ringpass(const tp_elem* elems, int64_t ne, const tp_misalign* mis, int64_t nmis,
                      const int32_t* sfields, int32_t nfields, int32_t sturn0, int32_t snturns,
                      const double* svalues, double* maps, int64_t nmaps, double beti, int32_t nturns,
                      int32_t turn0) {
    for (int64_t e = 0; e < ne; ++e)
        if (!tpsa_supported(elems[e].kind)) return -2;
    Inputs in{elems, ne, mis, nmis, sfields, nfields, sturn0, snturns, svalues};
    Lattice lat = build_lattice(in);
    const int M = tps_desc().M;
    try {
    for (int64_t m = 0; m < nmaps; ++m) {
        V6<Tps> r;
        for (int c = 0; c < 6; ++c) {
            r[c] = Tps::full();
            for (int k = 0; k < M; ++k) r[c].c[size_t(k)] = maps[(m * 6 + c) * M + k];
        }
        for (int32_t t = 0; t < nturns; ++t)
            for (int64_t e = 0; e < ne; ++e) r = tpsa_pass(elem_at<Tps>(lat, e, turn0 + t), r, Tps(beti));
        for (int c = 0; c < 6; ++c)
            for (int k = 0; k < M; ++k)
                maps[(m * 6 + c) * M + k] = r[c].is_const() ? (k == 0 ? r[c].c[0] : 0.0) : r[c].c[size_t(k)];
    }
    } catch (const std::exception& ex) {
        g_tpsa_error = ex.what();
        return -3;
    }
    return 0;
}

const char* orc_tpsa_error(void) { return g_tpsa_error.c_str(); }

}  // extern "C"

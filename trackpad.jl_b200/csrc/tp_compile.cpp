// tp_compile.cpp -- validation of tp_elem records and their compilation into
// the device element program (tp_program.h), plus the algorithmic FLOP model.
//
// Host constants are computed with the operations, operands and order the
// reference uses per particle (built with -ffp-contract=off, transcendental
// functions from tp_libm.h), so hoisting them out of the particle loop does not
// change a single bit of the result.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tp_internal.h"
#include "tp_libm.h"

namespace tp {

namespace {

constexpr double DRIFT1 = 0.6756035959798286638;   // src/tracking.jl:29-32
constexpr double DRIFT2 = -0.1756035959798286639;
constexpr double KICK1 = 1.351207191959657328;
constexpr double KICK2 = -1.702414383919314656;
constexpr double TWO_PI = 6.283185307179586;        // Float64(2pi)
constexpr double EPS = 2.220446049250313e-16;       // eps(Float64)

// Julia max(a, b) for Float64 with b = eps: NaN propagates.
double jmax_eps(double a) { return std::isnan(a) ? a : (a < EPS ? EPS : a); }

bool has_misalign_fields(int kind) {
    switch (kind) {
        case TP_DRIFT: case TP_DRIFT_SC: case TP_QUADRUPOLE: case TP_SEXTUPOLE: case TP_OCTUPOLE:
        case TP_THIN_MULTIPOLE: case TP_SBEND: case TP_EXACT_SBEND: case TP_SOLENOID: case TP_CORRECTOR:
        case TP_QUADRUPOLE_SC: case TP_SEXTUPOLE_SC: case TP_OCTUPOLE_SC: case TP_SBEND_SC: case TP_LBEND:
        case TP_WIGGLER:
            return true;
        default:
            return false;
    }
}

// Kinds whose arrays live in aux[iparam[0] .. iparam[0] + iparam[1]).
bool uses_aux(int kind) {
    return kind == TP_STRONG_GAUSSIAN_BEAM || kind == TP_LONGITUDINAL_WAKE || kind == TP_WIGGLER;
}

bool uses_order(int kind) {
    switch (kind) {
        case TP_QUADRUPOLE: case TP_SEXTUPOLE: case TP_OCTUPOLE: case TP_THIN_MULTIPOLE: case TP_SBEND:
        case TP_EXACT_SBEND:
            return true;
        default:
            return false;
    }
}

struct Rec {
    RecHdr h{};
    double w[MAX_REC_WORDS]{};
    int nw = 0;                // fixed payload words
    std::vector<double> tail;  // arrays after the fixed words
};

// edge_fringe_entrance / _exit constants (tracking.jl:162-172, 196-206):
// fx = irho tan(e), the edge angle and the fringe correction irho gap fint
// (1 + sin^2 e) / cos e (zero without fint, gap or method).
void edge_consts(double irho, double gap, int method, double ang, double fint, double* fx, double* eang,
                 double* fc) {
    double corr;
    if (fint == 0.0 || gap == 0.0 || method == 0) {
        corr = 0.0;
    } else {
        double sedge = libm::sin(ang), cedge = libm::cos(ang);
        corr = irho * gap * fint * (1.0 + sedge * sedge) / cedge;
    }
    *fx = irho * libm::tan(ang);
    *eang = ang;
    *fc = corr;
}

// symplectic4_pass / symplectic4_bend_pass slice constants (src/tracking.jl:325-329).
void yoshida_consts(double L, int n, double* L1, double* L2, double* K1, double* K2) {
    double SL = L / double(n);
    *L1 = SL * DRIFT1;
    *L2 = SL * DRIFT2;
    *K1 = SL * KICK1;
    *K2 = SL * KICK2;
}

// kick_angle folding (src/tracking.jl:396-411, 668-682, 931-940).
void fold_kick(const tp_elem& e, double* pa, double* pb) {
    if (e.L > 0.0) {
        pb[0] = pb[0] - libm::sin(e.kick_angle[0]) / e.L;
        pa[0] = pa[0] + libm::sin(e.kick_angle[1]) / e.L;
    }
}

}  // namespace

int validate_elem(const tp_elem& e, int64_t idx, int64_t nmis, std::string* err, const AuxView& aux) {
    auto fail = [&](const char* what) {
        *err = "element " + std::to_string(idx) + ": " + what;
        return TP_EINVAL;
    };
    if (e.kind < 0 || e.kind >= TP_KIND_COUNT) {
        *err = "element " + std::to_string(idx) + ": unknown kind " + std::to_string(e.kind);
        return TP_EUNSUPPORTED;
    }
    if (uses_aux(e.kind)) {
        const int64_t off = e.iparam[0], len = e.iparam[1];
        if (off < 0 || len < 0 || off + len > aux.n || (len > 0 && aux.p == nullptr))
            return fail("array fields outside the aux array (tp_lattice_create_ex)");
        if (len > 60000) {
            *err = "element " + std::to_string(idx) + ": array fields longer than 60000 words";
            return TP_ERANGE;
        }
        if (e.kind == TP_STRONG_GAUSSIAN_BEAM && len % 3 != 0)
            return fail("StrongGaussianBeam arrays: zslice_npar, xoffsets, yoffsets of nzslice each");
        if (e.kind == TP_LONGITUDINAL_WAKE && (len % 2 != 0 || len < 4))
            return fail("LongitudinalWake needs times and wakefields of the same length >= 2");
        if (e.kind == TP_WIGGLER) {
            if (len < 3) return fail("Wiggler arrays: NHharm, NVharm, rad, By, Bx");
            const double* a = aux.p + off;
            const int64_t nh = int64_t(a[0]), nv = int64_t(a[1]);
            if (nh < 0 || nv < 0 || a[0] != double(nh) || a[1] != double(nv) || 3 + 6 * (nh + nv) != len)
                return fail("Wiggler arrays: length must be 3 + 6 NHharm + 6 NVharm");
            if (!(e.param[0] > 0.0)) return fail("Wiggler lw must be positive");
        }
    }
    if (e.kind == TP_LBEND && e.L == 0.0) {
        // pass!(::LBend) returns NaN for L == 0 (tracking.jl:1158-1160); accepted, compiled to a NaN map
    }
    if (uses_order(e.kind) && (e.max_order < 0 || e.max_order > 3))
        return fail("max_order must be in 0..3 (polynom_a/polynom_b hold 4 coefficients)");
    if (e.misalign_index >= 0) {
        if (!has_misalign_fields(e.kind)) return fail("this element kind has no misalignment fields");
        if (e.misalign_index >= nmis) return fail("misalign_index out of range");
    } else if (e.misalign_index != -1) {
        return fail("misalign_index must be -1 or a row index");
    }
    return TP_OK;
}

// Compile one element.  Returns the record words (header + payload).
static Rec compile_rec(const tp_elem& e, const AuxView& aux) {
    Rec r;
    r.h.kind = DK_IDENTITY;
    r.h.order = 0;
    r.h.nsteps = e.num_int_steps;
    r.h.aux = -1;
    if (e.misalign_index >= 0 && has_misalign_fields(e.kind)) {
        r.h.flags |= RF_MISALIGN;
        r.h.aux = e.misalign_index;
    }
    switch (e.kind) {
        case TP_MARKER:
        case TP_SPACE_CHARGE:
            r.h.kind = DK_IDENTITY;
            break;
        case TP_DRIFT:
        case TP_DRIFT_SC:
            r.h.kind = DK_DRIFT;
            r.w[drift::L] = e.L;
            r.nw = drift::WORDS;
            break;
        case TP_QUADRUPOLE: case TP_SEXTUPOLE: case TP_OCTUPOLE:
        case TP_QUADRUPOLE_SC: case TP_SEXTUPOLE_SC: case TP_OCTUPOLE_SC: {
            double pa[4], pb[4];
            for (int i = 0; i < 4; ++i) { pa[i] = e.polynom_a[i]; pb[i] = e.polynom_b[i]; }
            int order = e.max_order;
            if (e.kind == TP_QUADRUPOLE) {            // tracking.jl:394-411
                pb[1] = e.k;
                fold_kick(e, pa, pb);
            } else if (e.kind == TP_SEXTUPOLE) {      // tracking.jl:446
                pb[2] = e.k / 2.0;
            } else if (e.kind == TP_OCTUPOLE) {       // tracking.jl:478
                pb[3] = e.k / 6.0;
            } else {                                   // _sc_polynom_b, tracking.jl:993-995
                pb[0] = e.param[0]; pb[1] = e.param[1]; pb[2] = e.param[2] / 2.0; pb[3] = e.param[3] / 6.0;
                if (e.kind == TP_QUADRUPOLE_SC) fold_kick(e, pa, pb);
                order = order < 0 ? 0 : (order > 3 ? 3 : order);
            }
            r.h.kind = DK_MULTIPOLE;
            r.h.order = uint8_t(order);
            yoshida_consts(e.L, e.num_int_steps, &r.w[mp::L1], &r.w[mp::L2], &r.w[mp::K1], &r.w[mp::K2]);
            for (int i = 0; i < 4; ++i) { r.w[mp::PA + i] = pa[i]; r.w[mp::PB + i] = pb[i]; }
            r.nw = mp::WORDS;
            break;
        }
        case TP_THIN_MULTIPOLE:
            r.h.kind = DK_THIN;
            r.h.order = uint8_t(e.max_order);
            for (int i = 0; i < 4; ++i) { r.w[thin::PA + i] = e.polynom_a[i]; r.w[thin::PB + i] = e.polynom_b[i]; }
            r.nw = thin::WORDS;
            break;
        case TP_SBEND:
        case TP_SBEND_SC: {
            if (e.kind == TP_SBEND_SC && e.L == 0.0) {  // tracking.jl:1047-1049
                r.h.kind = DK_NAN;
                break;
            }
            int order = e.max_order;
            if (e.kind == TP_SBEND_SC) order = order < 0 ? 0 : (order > 3 ? 3 : order);
            double irho = e.angle / e.L;
            double pa[4], pb[4];
            for (int i = 0; i < 4; ++i) { pa[i] = e.polynom_a[i]; pb[i] = e.polynom_b[i]; }
            fold_kick(e, pa, pb);
            r.h.kind = DK_SBEND;
            r.h.order = uint8_t(order);
            yoshida_consts(e.L, e.num_int_steps, &r.w[mp::L1], &r.w[mp::L2], &r.w[mp::K1], &r.w[mp::K2]);
            for (int i = 0; i < 4; ++i) { r.w[mp::PA + i] = pa[i]; r.w[mp::PB + i] = pb[i]; }
            r.w[sb::IRHO] = irho;
            auto edge = [&](int method, double ang, double fint, double* fx, double* eang, double* fc) {
                edge_consts(irho, e.gap, method, ang, fint, fx, eang, fc);
            };
            if (e.fringe_bend_entrance != 0) {
                r.h.flags |= RF_FRINGE_IN;
                r.h.method_in = uint8_t(e.fringe_bend_entrance >= 1 && e.fringe_bend_entrance <= 3
                                            ? e.fringe_bend_entrance : 1);
                edge(e.fringe_bend_entrance, e.e1, e.fint1, &r.w[sb::FX_IN], &r.w[sb::E_IN], &r.w[sb::FC_IN]);
                if (r.w[sb::FC_IN] == 0.0) r.h.flags |= RF_FC_IN_ZERO;
            }
            if (e.fringe_bend_exit != 0) {
                r.h.flags |= RF_FRINGE_OUT;
                r.h.method_out = uint8_t(e.fringe_bend_exit >= 1 && e.fringe_bend_exit <= 3 ? e.fringe_bend_exit : 1);
                edge(e.fringe_bend_exit, e.e2, e.fint2, &r.w[sb::FX_OUT], &r.w[sb::E_OUT], &r.w[sb::FC_OUT]);
                if (r.w[sb::FC_OUT] == 0.0) r.h.flags |= RF_FC_OUT_ZERO;
            }
            r.nw = sb::WORDS;
            break;
        }
        case TP_EXACT_SBEND: {  // tracking.jl:901-973
            double irho = e.angle / e.L;
            r.h.kind = DK_EXACT_SBEND;
            r.h.order = uint8_t(e.max_order);
            r.w[eb::IRHO] = irho;
            r.w[eb::IRHO_INV] = 1.0 / irho;
            if (std::isnormal(irho) && std::isnormal(r.w[eb::IRHO_INV])) r.h.flags |= RF_RCP_IRHO;
            r.w[eb::GK] = e.gk;
            if (e.e1 != 0.0) {
                r.h.flags |= RF_YROT_IN;
                r.w[eb::YC_IN] = libm::cos(e.e1);
                r.w[eb::YS_IN] = libm::sin(e.e1);
            }
            if (e.e2 != 0.0) {
                r.h.flags |= RF_YROT_OUT;
                r.w[eb::YC_OUT] = libm::cos(e.e2);
                r.w[eb::YS_OUT] = libm::sin(e.e2);
            }
            if (e.fringe_bend_entrance != 0) r.h.flags |= RF_FRINGE_IN;
            if (e.fringe_bend_exit != 0) r.h.flags |= RF_FRINGE_OUT;
            if (!(std::fabs(irho) < 1e-6)) {
                r.h.flags |= RF_EDGE;  // bend_edge returns r unchanged when |rhoinv| < 1e-6
                double t_in = -e.e1, t_out = -e.e2;
                r.w[eb::EC_IN] = libm::cos(t_in);
                r.w[eb::ES_IN] = libm::sin(t_in);
                r.w[eb::ES2_IN] = libm::sin(2.0 * t_in);
                r.w[eb::ETH_IN] = t_in;
                r.w[eb::ETHH_IN] = t_in / irho;
                r.w[eb::EC_OUT] = libm::cos(t_out);
                r.w[eb::ES_OUT] = libm::sin(t_out);
                r.w[eb::ES2_OUT] = libm::sin(2.0 * t_out);
                r.w[eb::ETH_OUT] = t_out;
                r.w[eb::ETHH_OUT] = t_out / irho;
            } else {
                r.h.flags |= RF_STRAIGHT;  // exact_bend_body drift limit
            }
            if (e.num_int_steps == 0) {
                r.h.flags |= RF_BODY_ONE;
                r.w[eb::L1] = e.L;
                r.w[eb::CS1] = libm::cos(irho * e.L);
                r.w[eb::SN1] = libm::sin(irho * e.L);
            } else {
                double pa[4], pb[4];
                for (int i = 0; i < 4; ++i) { pa[i] = e.polynom_a[i]; pb[i] = e.polynom_b[i]; }
                fold_kick(e, pa, pb);
                yoshida_consts(e.L, e.num_int_steps, &r.w[eb::L1], &r.w[eb::L2], &r.w[eb::K1], &r.w[eb::K2]);
                r.w[eb::CS1] = libm::cos(irho * r.w[eb::L1]);
                r.w[eb::SN1] = libm::sin(irho * r.w[eb::L1]);
                r.w[eb::CS2] = libm::cos(irho * r.w[eb::L2]);
                r.w[eb::SN2] = libm::sin(irho * r.w[eb::L2]);
                for (int i = 0; i < 4; ++i) { r.w[eb::PA + i] = pa[i]; r.w[eb::PB + i] = pb[i]; }
                // With max_order 0 the kick is px -= K*pb[0], py += K*pa[0]: exact no-ops
                // when both coefficients are zero (only the sign of a zero can change).
                if (e.max_order == 0 && pb[0] == 0.0 && pa[0] == 0.0) r.h.flags |= RF_NOKICK;
            }
            r.nw = eb::WORDS;
            break;
        }
        case TP_RFCAVITY:  // tracking.jl:502-518
            r.h.kind = DK_RF;
            if (e.L > 0.0) { r.h.flags |= RF_LPOS; r.w[rf::LH] = e.L / 2.0; }
            if (e.energy > 0.0) {
                r.h.flags |= RF_ENERGY;
                r.w[rf::NV] = e.volt / e.energy;
                r.w[rf::W] = TWO_PI * e.freq;
                r.w[rf::LAG] = e.lag;
                r.w[rf::PHILAG] = e.philag;
            }
            r.nw = rf::WORDS;
            break;
        case TP_SOLENOID:
            r.h.kind = DK_SOLENOID;
            r.w[sol::L] = e.L;
            r.w[sol::KS] = e.param[0];
            r.nw = sol::WORDS;
            break;
        case TP_CORRECTOR:
            r.h.kind = DK_CORRECTOR;
            r.w[cor::L] = e.L;
            r.w[cor::XK] = e.param[0];
            r.w[cor::YK] = e.param[1];
            r.nw = cor::WORDS;
            break;
        case TP_TRANSLATION:
            r.h.kind = DK_TRANSLATION;
            r.w[trn::DX] = e.param[0];
            r.w[trn::DY] = e.param[1];
            r.w[trn::DS] = e.param[2];
            r.nw = trn::WORDS;
            break;
        case TP_YROTATION: {  // tracking.jl:1194-1218
            double angle = -e.angle;
            if (angle == 0.0) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_YROTATION;
            r.w[yr::CA] = libm::cos(angle);
            r.w[yr::SA] = libm::sin(angle);
            r.w[yr::TA] = libm::tan(angle);
            r.nw = yr::WORDS;
            break;
        }
        case TP_CRAB_CAVITY:  // tracking.jl:1531-1547
            r.h.kind = DK_CRAB;
            if (e.L > 0.0) { r.h.flags |= RF_LPOS; r.w[crab::LH] = e.L / 2.0; }
            r.w[crab::VOLT] = e.volt * (1.0 + e.param[2]);
            r.w[crab::PHI] = e.param[1] + e.param[3];
            r.w[crab::E] = jmax_eps(std::fabs(e.energy));
            r.w[crab::K] = e.param[0];
            r.nw = crab::WORDS;
            break;
        case TP_ACCEL_CAVITY:  // tracking.jl:1549-1559
            r.h.kind = DK_ACCEL;
            r.w[acc::VOLT] = e.volt;
            r.w[acc::E] = jmax_eps(std::fabs(e.energy));
            r.w[acc::K] = e.param[0];
            r.w[acc::PHIS] = e.param[1];
            r.w[acc::SINPHIS] = libm::sin(e.param[1]);
            r.nw = acc::WORDS;
            break;
        case TP_LONGITUDINAL_RF_MAP:  // tracking.jl:1575-1585
            if (std::fabs(e.param[1]) <= EPS) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_LONG_RF_MAP;
            r.w[lrf::ALPHAC] = e.param[0];
            r.w[lrf::K] = e.param[1];
            r.w[lrf::H] = e.param[2];
            r.nw = lrf::WORDS;
            break;
        case TP_LORENTZ_BOOST:  // tracking.jl:1587-1595
            if (e.iparam[0] != 0) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_LORENTZ;
            r.w[lor::A] = 1.0 / e.param[1];
            r.w[lor::B] = e.param[3];
            r.nw = lor::WORDS;
            break;
        case TP_INV_LORENTZ_BOOST:  // tracking.jl:1597-1604
            if (e.iparam[0] != 0) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_INV_LORENTZ;
            r.w[lor::A] = e.param[1];
            r.w[lor::B] = e.param[2];
            r.nw = lor::WORDS;
            break;
        case TP_STRONG_THIN_GAUSSIAN_BEAM: {  // tracking.jl:1610-1619
            r.h.kind = DK_STRONG_THIN_GAUSS;
            double sx2 = e.param[1] * e.param[1], sy2 = e.param[2] * e.param[2];
            r.w[stg::AMP] = e.param[0];
            r.w[stg::SX2] = jmax_eps(sx2);
            r.w[stg::SY2] = jmax_eps(sy2);
            r.w[stg::XO] = e.param[3];
            r.w[stg::YO] = e.param[4];
            r.nw = stg::WORDS;
            break;
        }
        case TP_LBEND: {  // tracking.jl:1152-1170 (edges: method 1), body :1076-1150
            if (e.L == 0.0) { r.h.kind = DK_NAN; break; }
            r.h.kind = DK_LBEND;
            const double kx = e.angle / e.L;  // Kx = b_angle / L, and irho of the edges
            r.w[lb::L] = e.L;
            r.w[lb::KX] = kx;
            r.w[lb::G1C] = kx * kx + e.param[0];
            r.w[lb::NGRD] = -e.param[0];
            r.w[lb::BYERR] = e.param[1];
            r.w[lb::IRHO] = kx;
            edge_consts(kx, e.gap, 1, e.e1, e.fint1, &r.w[lb::FX_IN], &r.w[lb::E_IN], &r.w[lb::FC_IN]);
            edge_consts(kx, e.gap, 1, e.e2, e.fint2, &r.w[lb::FX_OUT], &r.w[lb::E_OUT], &r.w[lb::FC_OUT]);
            if (r.w[lb::FC_IN] == 0.0) r.h.flags |= RF_FC_IN_ZERO;
            if (r.w[lb::FC_OUT] == 0.0) r.h.flags |= RF_FC_OUT_ZERO;
            r.nw = lb::WORDS;
            break;
        }
        case TP_STRONG_GAUSSIAN_BEAM: {  // tracking.jl:1621-1641
            const int64_t nz = e.iparam[1] / 3;
            if (nz <= 0) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_SGB;
            r.w[sgb::FACTOR] = e.param[0] / jmax_eps(std::fabs(e.param[1]));
            r.w[sgb::SX2] = jmax_eps(e.param[2] * e.param[2]);
            r.w[sgb::SY2] = jmax_eps(e.param[3] * e.param[3]);
            r.w[sgb::NZ] = double(nz);
            r.nw = sgb::WORDS;
            r.tail.assign(aux.p + e.iparam[0], aux.p + e.iparam[0] + 3 * nz);
            break;
        }
        case TP_LONGITUDINAL_RLC_WAKE: {  // tracking.jl:1647-1654, elements/wake.jl:27-37
            if (e.param[3] == 0.0) { r.h.kind = DK_IDENTITY; break; }
            r.h.kind = DK_RLC_WAKE;
            const double freq = e.param[0], rsh = e.param[1], q0 = e.param[2];
            const double q0p = std::sqrt(q0 * q0 - 0.25);
            const double w0 = TWO_PI * freq;
            r.w[rlc::SCALE] = e.param[3];
            r.w[rlc::A] = rsh * w0 / q0;
            r.w[rlc::W0P] = w0 / q0 * q0p;
            r.w[rlc::D2Q0P] = 2.0 * q0p;
            r.w[rlc::W0] = w0;
            r.w[rlc::D2Q0] = 2.0 * q0;
            r.nw = rlc::WORDS;
            break;
        }
        case TP_LONGITUDINAL_WAKE: {  // tracking.jl:1656-1663, elements/wake.jl:68-91
            if (e.param[1] == 0.0) { r.h.kind = DK_IDENTITY; break; }
            const int64_t n = e.iparam[1] / 2;
            const double* t = aux.p + e.iparam[0];
            r.h.kind = DK_TAB_WAKE;
            bool sorted = true;
            for (int64_t i = 1; i < n; ++i) sorted = sorted && t[i - 1] <= t[i];
            r.h.order = sorted ? 1 : 0;  // sorted times: the device finds the segment by bisection
            r.w[tw::SCALE] = e.param[1];
            r.w[tw::FLIP] = e.param[0];
            r.w[tw::T1F] = t[0] * e.param[0];
            r.w[tw::N] = double(n);
            r.nw = tw::WORDS;
            r.tail.assign(t, t + 2 * n);
            break;
        }
        case TP_WIGGLER: {  // tracking.jl:1224-1529
            const double* a = aux.p + e.iparam[0];
            const int nh = int(a[0]), nv = int(a[1]), rad = int(a[2]);
            const double lw = e.param[0], bmax = e.param[1], energy = e.param[2];
            const int PN = e.num_int_steps;
            const double Nw = std::nearbyint(e.L / lw);  // round(Int, L/lw): half to even
            const double Nstep = double(PN) * (Nw > 1.0 ? Nw : 1.0);
            const double dl = lw / double(PN);
            const double dl1 = dl * 1.3512071919596573, dl0 = dl * -1.7024143839193146;
            const double Aw = 1e-9 * 2.99792458e8 / (0.51099895069e6 * 1e-9) / TWO_PI * lw * bmax;
            const double kw = TWO_PI / lw;
            double Po, srCoef = 0.0;
            if (rad == 1) {
                const double gamma = energy / 0.51099895069e6;
                Po = std::sqrt(gamma * gamma - 1.0);
                srCoef = (2.0 / 3.0) * 2.8179403205e-15 * (gamma * gamma * gamma);
            } else {
                Po = std::sqrt((energy / 0.51099895069e6) * (energy / 0.51099895069e6) - 1.0);
            }
            const double H = Po * 0.51099895069e6 / 2.99792458e8;
            r.h.kind = DK_WIGGLER;
            r.w[wg::NSTEP] = Nstep;
            r.w[wg::DL1] = dl1;
            r.w[wg::DL0] = dl0;
            r.w[wg::DL1H] = dl1 / 2.0;
            r.w[wg::DL0H] = dl0 / 2.0;
            r.w[wg::PO] = Po;
            r.w[wg::SRCOEF] = srCoef;
            r.w[wg::SL] = dl;
            r.w[wg::HH] = H * H;
            r.w[wg::NH] = double(nh);
            r.w[wg::NV] = double(nv);
            r.w[wg::RAD] = double(rad);
            r.nw = wg::WORDS;
            r.tail.assign(size_t(wg::HWORDS) * size_t(nh + nv), 0.0);
            for (int i = 0; i < nh + nv; ++i) {
                const bool horiz = i < nh;
                const double* b = a + 3 + 6 * i;
                double* o = r.tail.data() + size_t(wg::HWORDS) * size_t(i);
                const double kx = b[2] * kw, ky = b[3] * kw, kz = b[4] * kw;
                const double c = b[1] * Aw / Po;   // HCw or VCw of the vector potential
                const double ckz = c * (kw / kz);
                o[wg::KX] = kx; o[wg::KY] = ky; o[wg::KZ] = kz; o[wg::TZ] = b[5];
                if (horiz) {
                    o[wg::C_AX] = ckz;
                    o[wg::C_AXPY] = ckz * ky;
                    o[wg::C_AY] = ckz * (kx / ky);
                    o[wg::C_AYPX] = ckz * ((kx / ky) * (kx / ky));
                    o[wg::SINC] = std::fabs(kx / kw) > 1e-6 ? 1.0 : 0.0;
                    o[wg::B_X] = bmax * b[1] * (kx / ky);
                    o[wg::B_Y] = bmax * b[1];
                } else {
                    o[wg::C_AX] = ckz * (ky / kx);
                    o[wg::C_AXPY] = ckz * ((ky / kx) * (ky / kx));
                    o[wg::C_AY] = ckz;
                    o[wg::C_AYPX] = ckz * kx;
                    o[wg::SINC] = std::fabs(ky / kw) > 1e-6 ? 1.0 : 0.0;
                    o[wg::B_X] = bmax * b[1];
                    o[wg::B_Y] = bmax * b[1] * (ky / kx);
                }
            }
            break;
        }
        default:
            break;
    }
    r.h.words = uint16_t(HDR_WORDS + r.nw + int(r.tail.size()));
    return r;
}

static void append_rec(const Rec& r, std::vector<double>* out) {
    size_t at = out->size();
    out->resize(at + r.h.words);
    std::memcpy(out->data() + at, &r.h, sizeof(RecHdr));
    for (int i = 0; i < r.nw; ++i) (*out)[at + HDR_WORDS + i] = r.w[i];
    for (size_t i = 0; i < r.tail.size(); ++i) (*out)[at + HDR_WORDS + r.nw + i] = r.tail[i];
}

void compile_record(const tp_elem& e, std::vector<double>* out, const AuxView& aux) {
    append_rec(compile_rec(e, aux), out);
}

int record_words(const tp_elem& e, const AuxView& aux) { return compile_rec(e, aux).h.words; }

void scheduled_stub(const tp_elem& e, int32_t slot, std::vector<double>* out, const AuxView& aux) {
    Rec r;
    r.h.kind = compile_rec(e, aux).h.kind;
    r.h.flags = RF_SCHEDULED;
    r.h.words = HDR_WORDS;
    r.h.aux = slot;
    append_rec(r, out);
}

void apply_field(tp_elem* e, int field, double v) {
    switch (field) {
        case TP_FIELD_L: e->L = v; break;
        case TP_FIELD_K: e->k = v; break;
        case TP_FIELD_ANGLE: e->angle = v; break;
        case TP_FIELD_E1: e->e1 = v; break;
        case TP_FIELD_E2: e->e2 = v; break;
        case TP_FIELD_VOLT: e->volt = v; break;
        case TP_FIELD_FREQ: e->freq = v; break;
        case TP_FIELD_LAG: e->lag = v; break;
        case TP_FIELD_PHILAG: e->philag = v; break;
        case TP_FIELD_ENERGY: e->energy = v; break;
        case TP_FIELD_NUM_INT_STEPS: e->num_int_steps = int32_t(v); break;
        default:
            if (field >= TP_FIELD_POLYNOM_A0 && field < TP_FIELD_POLYNOM_A0 + 4)
                e->polynom_a[field - TP_FIELD_POLYNOM_A0] = v;
            else if (field >= TP_FIELD_POLYNOM_B0 && field < TP_FIELD_POLYNOM_B0 + 4)
                e->polynom_b[field - TP_FIELD_POLYNOM_B0] = v;
            break;
    }
}

// ---------------------------------------------------------------------------
// Algorithmic FLOP model: operations the reference's pass! performs for one
// typical particle, counted with add/sub/mul/div/sqrt = 1 and each
// transcendental call = TP_FLOPS_PER_TRANSCENDENTAL (20).  Every constant
// below is checked against the oracle's op-counting scalar in the CPU tests.
// ---------------------------------------------------------------------------
double elem_flops(const tp_elem& e, const tp_misalign* mis, bool exact, const AuxView& aux) {
    const double TR = TP_FLOPS_PER_TRANSCENDENTAL;
    const double D = exact ? 20.0 : 14.0;           // drift6
    auto kick = [](int m) { return 8.0 * m + 4.0; };  // strthinkick
    auto bkick = [](int m) { return 8.0 * m + 12.0; };  // bndthinkick
    double mis_f = 0.0;
    if (has_misalign_fields(e.kind)) {
        mis_f = 12.0;  // r + t1, r + t2 are always evaluated
        if (mis) {
            bool r1 = false, r2 = false;
            for (int i = 0; i < 36; ++i) { r1 |= mis->r1[i] != 0.0; r2 |= mis->r2[i] != 0.0; }
            mis_f += (r1 ? 66.0 : 0.0) + (r2 ? 66.0 : 0.0);
        }
    }
    const int n = e.num_int_steps > 0 ? e.num_int_steps : 0;
    const double fold = e.L > 0.0 ? 4.0 + 2.0 * TR : 0.0;
    switch (e.kind) {
        case TP_MARKER: case TP_SPACE_CHARGE: return 0.0;
        case TP_DRIFT: case TP_DRIFT_SC: return mis_f + D;
        case TP_QUADRUPOLE:
            return mis_f + fold + 5.0 + n * (4.0 * D + 3.0 * kick(e.max_order));
        case TP_SEXTUPOLE: case TP_OCTUPOLE:
            return mis_f + 1.0 + 5.0 + n * (4.0 * D + 3.0 * kick(e.max_order));
        case TP_QUADRUPOLE_SC: case TP_SEXTUPOLE_SC: case TP_OCTUPOLE_SC: {
            int m = e.max_order < 0 ? 0 : (e.max_order > 3 ? 3 : e.max_order);
            return mis_f + 2.0 + (e.kind == TP_QUADRUPOLE_SC ? fold : 0.0) + 5.0 + n * (4.0 * D + 3.0 * kick(m));
        }
        case TP_THIN_MULTIPOLE: return mis_f + kick(e.max_order);
        case TP_SBEND: case TP_SBEND_SC: {
            if (e.kind == TP_SBEND_SC && e.L == 0.0) return mis_f;
            int m = e.max_order;
            if (e.kind == TP_SBEND_SC) m = m < 0 ? 0 : (m > 3 ? 3 : m);
            auto edge = [&](int method, double fint) {
                if (method == 0) return 0.0;
                double f = 49.0;
                if (!(fint == 0.0 || e.gap == 0.0)) f += 46.0;  // sin, cos and the fringecorr product
                if (method == 2) f += 2.0;
                if (method == 3) f += 1.0;
                return f;
            };
            return mis_f + 1.0 + fold + 5.0 + edge(e.fringe_bend_entrance, e.fint1) +
                   n * (4.0 * D + 3.0 * bkick(m)) + edge(e.fringe_bend_exit, e.fint2);
        }
        case TP_EXACT_SBEND: {
            const double body = 124.0, yrot = 63.0, fringe = 243.0, edge = 152.0;
            double f = mis_f + 1.0;
            if (e.e1 != 0.0) f += yrot;
            if (e.e2 != 0.0) f += yrot;
            if (e.fringe_bend_entrance != 0) f += fringe;
            if (e.fringe_bend_exit != 0) f += fringe;
            double irho = e.angle / e.L;
            if (!(std::fabs(irho) < 1e-6)) f += 2.0 * edge;
            if (e.num_int_steps == 0) {
                f += body;
            } else {
                f += 5.0 + fold + n * (4.0 * body + 3.0 * kick(e.max_order));
            }
            return f;
        }
        case TP_RFCAVITY: {
            double f = 1.0;
            if (e.L > 0.0) f += 2.0 * (1.0 + D);
            if (e.energy > 0.0) f += 30.0;
            return f;
        }
        case TP_SOLENOID: return mis_f + (e.param[0] == 0.0 ? D : 80.0 + 2.0 * TR);
        case TP_CORRECTOR: return mis_f + 30.0;
        case TP_TRANSLATION: return 22.0;
        case TP_YROTATION: return e.angle == 0.0 ? 0.0 : 29.0 + 3.0 * TR;
        case TP_CRAB_CAVITY: return 16.0 + 2.0 * TR + (e.L > 0.0 ? 2.0 * (1.0 + D) : 0.0);
        case TP_ACCEL_CAVITY: return 9.0 + 2.0 * TR;
        case TP_LONGITUDINAL_RF_MAP: return 9.0;
        case TP_LORENTZ_BOOST: return 8.0;
        case TP_INV_LORENTZ_BOOST: return 7.0;
        case TP_STRONG_THIN_GAUSSIAN_BEAM: return 17.0 + TR;
        case TP_LBEND: {
            if (e.L == 0.0) return mis_f;
            // edges (method 1) as for the SBend; body: 57 operations, plus the
            // focusing terms of each plane whose |G| = |(Kx^2 + K, -K) p_norm| >= sqrt(eps)
            auto edge = [&](double fint) { return 49.0 + ((fint == 0.0 || e.gap == 0.0) ? 0.0 : 46.0); };
            const double kx = e.angle / e.L;
            const double g1 = kx * kx + e.param[0], g2 = -e.param[0];
            const double tol = 1.4901161193847656e-08;
            double body = 57.0;
            if (std::fabs(g1) >= tol) body += 44.0 + 5.0 * TR;
            if (std::fabs(g2) >= tol) body += 4.0 + 3.0 * TR;
            return mis_f + 1.0 + edge(e.fint1) + body + edge(e.fint2);
        }
        case TP_STRONG_GAUSSIAN_BEAM: {
            const double nz = double(e.iparam[1] / 3);
            return nz <= 0.0 ? 0.0 : 3.0 + nz * (17.0 + TR);
        }
        case TP_LONGITUDINAL_RLC_WAKE: return e.param[3] == 0.0 ? 0.0 : 21.0 + 3.0 * TR;
        case TP_LONGITUDINAL_WAKE:
            // a particle ahead of the wake (z > 0 with fliphalf < 0); one behind adds the interpolation
            return e.param[1] == 0.0 ? 0.0 : 3.0;
        case TP_WIGGLER: {
            // per 2nd-order map: 46 operations, 752 per By and 762 per Bx harmonic (each harmonic
            // costs 5 or 6 transcendental calls per vector-potential evaluation, 6 evaluations per map)
            // (a By harmonic with kx != 0 evaluates sin(kx x)/kx, 8 operations more than the
            // small-argument series, in each of the 2 ax evaluations per map; a Bx harmonic with
            // ky == 0 takes the series, 8 fewer, in each of the 4 ay evaluations per map)
            const double* a = aux.p + e.iparam[0];
            const int nh = int(a[0]), nv = int(a[1]);
            const bool rad = a[2] == 1.0;
            const double nw = std::nearbyint(e.L / e.param[0]);
            const double nstep = double(e.num_int_steps) * (nw > 1.0 ? nw : 1.0);
            double per_step = 138.0, per_block = 24.0;
            for (int i = 0; i < nh + nv; ++i) {
                const double* b = a + 3 + 6 * i;
                if (i < nh) {
                    const bool sinpath = std::fabs(b[2]) > 1e-6;  // |kx / kw|
                    per_step += 2256.0 + (sinpath ? 48.0 : 0.0);
                    per_block += 397.0 + (sinpath ? 8.0 : 0.0);
                } else {
                    const bool series = !(std::fabs(b[3]) > 1e-6);  // |ky / kw|
                    per_step += 2286.0 - (series ? 96.0 : 0.0);
                    per_block += 405.0 - (series ? 8.0 : 0.0);
                }
            }
            double f = mis_f + 14.0 + nstep * per_step;
            if (rad) f += 3.0 + (nstep + 1.0) * per_block;
            return f;
        }
        default: return 0.0;
    }
}

bool records_have_rare(const double* recs, size_t words) {
    for (size_t w = 0; w < words;) {
        RecHdr h;
        std::memcpy(&h, recs + w, sizeof h);
        if (h.words == 0) break;  // padding word
        if (h.kind > DK_RF) return true;
        w += h.words;
    }
    return false;
}

}  // namespace tp

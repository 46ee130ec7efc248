// tp_program.h -- the compiled element table ("program") read by the kernels.
//
// The host compiles each tp_elem into a variable-length record of 8-byte
// words.  Everything that is constant for a lattice entry (folded multipole
// coefficients, Yoshida slice lengths, cos/sin/tan of fixed angles, RF
// angular frequency ...) is computed once on the host, with the same IEEE
// operations in the same order as the reference evaluates them per particle,
// so the device only does the per-particle arithmetic.  Records are walked in
// order; every thread of a warp reads the same record, so shared-memory reads
// are broadcasts.
#pragma once
#include <stdint.h>

namespace tp {

// Device element kinds (several tp_kind map onto one device kind).
enum DevKind : uint8_t {
    DK_IDENTITY = 0,    // Marker, SpaceCharge, zero-angle YRotation
    DK_DRIFT = 1,       // Drift, DriftSC
    DK_MULTIPOLE = 2,   // Quadrupole, Sextupole, Octupole, *SC: symplectic4_pass
    DK_THIN = 3,        // ThinMultipole: strthinkick with unit length
    DK_SBEND = 4,       // SBend, SBendSC: edges + symplectic4_bend_pass
    DK_EXACT_SBEND = 5, // ExactSBend
    DK_RF = 6,          // RFCavity
    DK_SOLENOID = 7,
    DK_CORRECTOR = 8,
    DK_TRANSLATION = 9,
    DK_YROTATION = 10,
    DK_CRAB = 11,
    DK_ACCEL = 12,
    DK_LONG_RF_MAP = 13,
    DK_LORENTZ = 14,
    DK_INV_LORENTZ = 15,
    DK_STRONG_THIN_GAUSS = 16,
    DK_NAN = 17,        // maps that return NaN for every particle (SBendSC with L == 0)
    DK_LBEND = 18,      // LBend: edges (method 1) + linear combined-function body
    DK_SGB = 19,        // StrongGaussianBeam: Gaussian kicks of nz slices (arrays in the record)
    DK_RLC_WAKE = 20,   // LongitudinalRLCWake
    DK_TAB_WAKE = 21,   // LongitudinalWake: tabulated wake (table in the record)
    DK_WIGGLER = 22,    // Wiggler (harmonics in the record)
    DK_COUNT = 23
};

// Record flags.
enum RecFlag : uint16_t {
    RF_MISALIGN = 1u << 0,   // apply the misalignment row `aux`
    RF_SCHEDULED = 1u << 1,  // fields vary per turn: read the record from the schedule table
    RF_NOKICK = 1u << 2,     // exact bend: thin kicks are exact no-ops (order 0, zero coefficients)
    RF_FRINGE_IN = 1u << 3,  // exact bend: bend_fringe at entrance / SBend: edge at entrance
    RF_FRINGE_OUT = 1u << 4,
    RF_YROT_IN = 1u << 5,    // exact bend: yrot(e1) (phi != 0)
    RF_YROT_OUT = 1u << 6,
    RF_EDGE = 1u << 7,       // exact bend: bend_edge active (|irho| >= 1e-6)
    RF_STRAIGHT = 1u << 8,   // exact bend body: drift limit (|irho| < 1e-6)
    RF_LPOS = 1u << 9,       // RF / crab: L > 0 (half drifts)
    RF_ENERGY = 1u << 10,    // RF: energy > 0 (kick applied)
    RF_FC_IN_ZERO = 1u << 11,  // SBend: entrance fringecorr == 0
    RF_FC_OUT_ZERO = 1u << 12, // SBend: exit fringecorr == 0
    RF_BODY_ONE = 1u << 13,  // exact bend with num_int_steps == 0: one body call over L
    RF_OFF = 1u << 14,       // Lorentz boost with mode != 0, Accel with beta^2 <= eps ...: identity
    RF_RCP_IRHO = 1u << 15   // exact bend: irho and RN(1/irho) are normal numbers (reciprocal division)
};

// Two header words.  `words` is the record length including the header.
struct RecHdr {
    uint8_t kind;
    uint8_t order;      // multipole order of the thin kicks (0..3)
    uint8_t method_in;  // SBend edge method at entrance (0..3, others = Brown)
    uint8_t method_out;
    uint16_t flags;
    uint16_t words;
    int32_t nsteps;     // Yoshida steps
    int32_t aux;        // misalignment row, or schedule slot (word offset) when RF_SCHEDULED
};
static_assert(sizeof(RecHdr) == 16, "header is two words");
constexpr int HDR_WORDS = 2;

// Payload layouts (word offsets after the header).
namespace drift { enum { L = 0, WORDS = 1 }; }
namespace mp {  // DK_MULTIPOLE and DK_SBEND share the first 12 words
enum { L1 = 0, L2 = 1, K1 = 2, K2 = 3, PA = 4, PB = 8, WORDS = 12 };
}
namespace sb {  // DK_SBEND
enum { IRHO = 12, FX_IN = 13, E_IN = 14, FC_IN = 15, FX_OUT = 16, E_OUT = 17, FC_OUT = 18, WORDS = 19 };
}
namespace thin { enum { PA = 0, PB = 4, WORDS = 8 }; }
namespace eb {  // DK_EXACT_SBEND
enum {
    IRHO = 0, GK = 1,
    L1 = 2, L2 = 3, K1 = 4, K2 = 5,          // body slice lengths and kick lengths (L1 = L for one body)
    CS1 = 6, SN1 = 7, CS2 = 8, SN2 = 9,      // cos/sin(irho*L1), cos/sin(irho*L2)
    YC_IN = 10, YS_IN = 11, YC_OUT = 12, YS_OUT = 13,  // yrot(e1), yrot(e2)
    EC_IN = 14, ES_IN = 15, ES2_IN = 16, ETH_IN = 17, ETHH_IN = 18,     // bend_edge(-e1): c, s, sin(2t), t, t/h
    EC_OUT = 19, ES_OUT = 20, ES2_OUT = 21, ETH_OUT = 22, ETHH_OUT = 23, // bend_edge(-e2)
    PA = 24, PB = 28,
    IRHO_INV = 32,                              // RN(1/irho) for the exact quotient by irho
    WORDS = 33
};
}
namespace rf { enum { LH = 0, NV = 1, W = 2, LAG = 3, PHILAG = 4, WORDS = 5 }; }
namespace sol { enum { L = 0, KS = 1, WORDS = 2 }; }
namespace cor { enum { L = 0, XK = 1, YK = 2, WORDS = 3 }; }
namespace trn { enum { DX = 0, DY = 1, DS = 2, WORDS = 3 }; }
namespace yr { enum { CA = 0, SA = 1, TA = 2, WORDS = 3 }; }
namespace crab { enum { LH = 0, VOLT = 1, PHI = 2, E = 3, K = 4, WORDS = 5 }; }
namespace acc { enum { VOLT = 0, E = 1, K = 2, PHIS = 3, SINPHIS = 4, WORDS = 5 }; }
namespace lrf { enum { ALPHAC = 0, K = 1, H = 2, WORDS = 3 }; }
namespace lor { enum { A = 0, B = 1, WORDS = 2 }; }  // boost: invcos, tanang; inverse: cosang, sinang
namespace stg { enum { AMP = 0, SX2 = 1, SY2 = 2, XO = 3, YO = 4, WORDS = 5 }; }
namespace lb {  // DK_LBEND: body constants, then the SBend edge words
enum { L = 0, KX = 1, G1C = 2, NGRD = 3, BYERR = 4, IRHO = 5, FX_IN = 6, E_IN = 7, FC_IN = 8,
       FX_OUT = 9, E_OUT = 10, FC_OUT = 11, WORDS = 12 };
}
namespace sgb { enum { FACTOR = 0, SX2 = 1, SY2 = 2, NZ = 3, WORDS = 4 }; }  // then w[nz], xo[nz], yo[nz]
namespace rlc { enum { SCALE = 0, A = 1, W0P = 2, D2Q0P = 3, W0 = 4, D2Q0 = 5, WORDS = 6 }; }
namespace tw { enum { SCALE = 0, FLIP = 1, T1F = 2, N = 3, WORDS = 4 }; }  // then times[n], wakes[n]
namespace wg {  // DK_WIGGLER, then HWORDS words per harmonic (By harmonics first, then Bx)
enum { NSTEP = 0, DL1 = 1, DL0 = 2, DL1H = 3, DL0H = 4, PO = 5, SRCOEF = 6, SL = 7, HH = 8, NH = 9, NV = 10,
       RAD = 11, WORDS = 12 };
// per harmonic: wave numbers, phase, the four vector-potential coefficients,
// the small-argument flag of sin(k u)/k, and the two field coefficients
enum { KX = 0, KY = 1, KZ = 2, TZ = 3, C_AX = 4, C_AXPY = 5, C_AY = 6, C_AYPX = 7, SINC = 8, B_X = 9,
       B_Y = 10, HWORDS = 12 };
}

// Misalignment row as stored on the device (same content as tp_misalign).
struct MisalignDev {
    double t1[6];
    double t2[6];
    double r1[36];
    double r2[36];
    int32_t r1nz, r2nz;
    int32_t pad[2];
};

// Maximum fixed record length in words (exact bend); array-carrying kinds
// (DK_SGB, DK_TAB_WAKE, DK_WIGGLER) append their arrays after the fixed words.
constexpr int MAX_REC_WORDS = HDR_WORDS + eb::WORDS;

}  // namespace tp

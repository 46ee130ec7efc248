// tp_tpsa.cu -- truncated power series (TPSA) map tracking on the device:
// linepass / ringpass / polyseries_one_turn_map of ext/TrackPadPolySeriesExt.jl
// (TrackPad.jl's PolySeries extension, :654-705).
//
// A map is six series (x, px, y, py, z, delta) in the six phase-space
// variables, truncated at total order N (M = C(N+6, 6) coefficients each).
// One CTA tracks one map at a time (a persistent loop over the maps); its
// threads share every series operation, each thread owning the coefficients
// k = tid, tid + blockDim, ...; a __syncthreads() ends every operation.  The
// series live in a pool of 18 or 40 slots of M doubles (40 when the lattice
// holds the longer bodies: solenoid, corrector, rotations, beam-beam, crab and
// accelerating cavities, misalignment rows), in shared memory when
// it fits and in a per-CTA global slab otherwise.
//
// Series algebra (the published algorithm of PolySeries's CTPS):
//   * coefficients ordered by degree, and within a degree by exponent vector
//     in descending lexicographic order (x^d first, delta^d last);
//   * a product is truncated at order N: c_k = sum_{(i,j) in P(k)} a_i b_j
//     over the pairs whose monomials multiply to monomial k, in increasing i
//     (the host builds P as a CSR table, read through the L1 cache);
//   * f(a0 + abar) = sum_k f^(k)(a0)/k! abar^k by Horner's rule (N products)
//     for 1/a, sqrt, a^(-1/2), exp, sin, cos; a / b = a * (1/b); a series
//     divided by a number divides every coefficient;
//   * numbers (element constants) stay numbers: a number times a series scales
//     it, a number plus a series changes its constant part only.
// The element maps are the CTPS pass! bodies of the extension (the particle
// bodies of src/tracking.jl in series arithmetic, with an always-exact drift,
// bend edges whose fy uses the constant parts of delta and px, and wakes at
// the constant part of z), written with a series value type so that each
// expression keeps the reference's operation order; compiled without FMA
// contraction, the maps equal the CPU oracle's coefficient for coefficient.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "tp_internal.h"
#include "tp_maps.cuh"

namespace tp {
namespace {

using namespace tp::dev;

constexpr int kTpsaMaxOrder = 10;
constexpr int kSlotsCore = 18;        // series per map for drifts, kicks, bends, RF
constexpr int kSlotsRare = 40;        // with the longer bodies (solenoid, corrector, rotations, beam-beam)
// busiest-thread pair count of the strided split above which product outputs
// are dealt to threads by pair count instead
#ifndef TP_TPSA_DEAL_MIN
#define TP_TPSA_DEAL_MIN 64
#endif
constexpr int kTpsaScratchTable = 13; // context scratch slots used here
constexpr int kTpsaScratchMaps = 14;
constexpr int kTpsaScratchPool = 15;

// ---------------------------------------------------------------------------
// Host tables: monomials and product pairs of order N.
// ---------------------------------------------------------------------------
struct TpsaTables {
    int N = -1, M = 0;
    std::vector<int32_t> mono;   // M x 6 exponents
    std::vector<int32_t> poff;   // M + 1
    std::vector<uint32_t> pairs; // i | j << 16
};

void enum_degree(int deg, int v, int* cur, std::vector<int32_t>* out) {
    if (v == 5) {
        cur[5] = deg;
        out->insert(out->end(), cur, cur + 6);
        return;
    }
    for (int e = deg; e >= 0; --e) {
        cur[v] = e;
        enum_degree(deg - e, v + 1, cur, out);
    }
}

const TpsaTables& tables_of(int N) {
    static std::mutex mu;
    static std::map<int, TpsaTables> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(N);
    if (it != cache.end()) return it->second;
    TpsaTables t;
    t.N = N;
    int cur[6] = {0, 0, 0, 0, 0, 0};
    for (int d = 0; d <= N; ++d) enum_degree(d, 0, cur, &t.mono);
    t.M = int(t.mono.size() / 6);
    auto key = [](const int32_t* e) {
        uint64_t k = 0;
        for (int v = 0; v < 6; ++v) k = k * 64u + uint64_t(e[v]);
        return k;
    };
    std::unordered_map<uint64_t, int32_t> index;
    for (int k = 0; k < t.M; ++k) index[key(&t.mono[size_t(k) * 6])] = k;
    t.poff.assign(size_t(t.M) + 1, 0);
    for (int k = 0; k < t.M; ++k) {
        const int32_t* mk = &t.mono[size_t(k) * 6];
        for (int i = 0; i < t.M; ++i) {
            const int32_t* mi = &t.mono[size_t(i) * 6];
            int32_t mj[6];
            bool ok = true;
            for (int v = 0; v < 6 && ok; ++v) {
                mj[v] = mk[v] - mi[v];
                ok = mj[v] >= 0;
            }
            if (!ok) continue;
            t.pairs.push_back(uint32_t(i) | (uint32_t(index.at(key(mj))) << 16));
        }
        t.poff[size_t(k) + 1] = int32_t(t.pairs.size());
    }
    return cache.emplace(N, std::move(t)).first->second;
}

// ---------------------------------------------------------------------------
// Device series algebra
// ---------------------------------------------------------------------------
struct TCtx {
    double* pool;            // nslots x M
    const int4* otab;        // product output slots: {output k (-1: none), first pair, end pair, 0}
    const uint32_t* pairs;
    int olen;                // product output slots (M, or more when dealt by pair count)
    int M, N, top, maxtop, nslots;
    int* err;                // TE_* bits
    unsigned long long nmul, nlin;  // series products and elementwise operations of this map
};

enum TpsaErr : int32_t { TE_SLOTS = 1, TE_KIND = 2, TE_SCHED = 4 };

// A series (p != nullptr: M coefficients in the pool) or a number c.
struct Tv {
    double* p;
    double c;
    TCtx* x;
    __device__ Tv() : p(nullptr), c(0.0), x(nullptr) {}
    __device__ Tv(double v) : p(nullptr), c(v), x(nullptr) {}
    __device__ Tv(double* q, TCtx* cx) : p(q), c(0.0), x(cx) {}
};

__device__ __forceinline__ double* t_alloc(TCtx* x) {
    if (x->top >= x->nslots) {
        if (threadIdx.x == 0) atomicOr(x->err, TE_SLOTS);
        return x->pool + size_t(x->nslots - 1) * x->M;  // in bounds; the result is flagged
    }
    double* p = x->pool + size_t(x->top++) * x->M;
    if (x->top > x->maxtop) x->maxtop = x->top;
    return p;
}

__device__ __forceinline__ TCtx* ctx_of(const Tv& a, const Tv& b) { return a.x ? a.x : b.x; }

__device__ __forceinline__ double cst(const Tv& a) { return a.p ? a.p[0] : a.c; }

// Elementwise kernels and the truncated product on plain restrict pointers:
// the loops keep their pointers and sizes in registers (through the value
// structs, every store could alias them and force reloads).
static __device__ __forceinline__ void ew_add(double* __restrict__ r, const double* __restrict__ ap, double ac,
                                              const double* __restrict__ bp, double bc, int M, bool sub) {
    const int n = blockDim.x;
    if (!ap) {
        for (int k = threadIdx.x; k < M; k += n) r[k] = k == 0 ? (sub ? ac - bp[0] : ac + bp[0]) : (sub ? -bp[k] : bp[k]);
    } else if (!bp) {
        for (int k = threadIdx.x; k < M; k += n) r[k] = k == 0 ? (sub ? ap[0] - bc : ap[0] + bc) : ap[k];
    } else if (sub) {
        for (int k = threadIdx.x; k < M; k += n) r[k] = ap[k] - bp[k];
    } else {
        for (int k = threadIdx.x; k < M; k += n) r[k] = ap[k] + bp[k];
    }
    __syncthreads();
}

static __device__ __forceinline__ void ew_scale(double* __restrict__ r, const double* __restrict__ ap, double s,
                                                int M) {
    for (int k = threadIdx.x; k < M; k += blockDim.x) r[k] = ap[k] * s;
    __syncthreads();
}

static __device__ __forceinline__ void ew_div(double* __restrict__ r, const double* __restrict__ ap, double s,
                                              int M) {
    for (int k = threadIdx.x; k < M; k += blockDim.x) r[k] = ap[k] / s;
    __syncthreads();
}

static __device__ __forceinline__ void ew_neg(double* __restrict__ r, const double* __restrict__ ap, int M) {
    for (int k = threadIdx.x; k < M; k += blockDim.x) r[k] = -ap[k];
    __syncthreads();
}

static __device__ __forceinline__ void ew_copy(double* __restrict__ r, const double* __restrict__ ap, int M) {
    for (int k = threadIdx.x; k < M; k += blockDim.x) r[k] = ap[k];
    __syncthreads();
}

// Truncated product r = a * b over the pair table (r distinct from a and b);
// four products in flight, summed in pair order (the oracle's order).
// With addc, the constant c is then added to the constant part (Horner's
// "+ c_k"), in the same pass.
static __device__ __noinline__ void t_mul_raw(double* __restrict__ r, const double* __restrict__ ap,
                                              const double* __restrict__ bp, const int4* __restrict__ otab,
                                              const uint32_t* __restrict__ pairs, int olen, bool addc = false,
                                              double c = 0.0) {
    for (int o = threadIdx.x; o < olen; o += blockDim.x) {
        const int4 e = otab[o];
        const int k = e.x;
        if (k < 0) continue;
        int p = e.y;
        const int p1 = e.z;
        uint32_t q = pairs[p];
        double s = ap[q & 0xffffu] * bp[q >> 16];
        ++p;
        for (; p + 4 <= p1; p += 4) {
            const uint32_t q0 = pairs[p], q1 = pairs[p + 1], q2 = pairs[p + 2], q3 = pairs[p + 3];
            const double m0 = ap[q0 & 0xffffu] * bp[q0 >> 16];
            const double m1 = ap[q1 & 0xffffu] * bp[q1 >> 16];
            const double m2 = ap[q2 & 0xffffu] * bp[q2 >> 16];
            const double m3 = ap[q3 & 0xffffu] * bp[q3 >> 16];
            s = s + m0;
            s = s + m1;
            s = s + m2;
            s = s + m3;
        }
        for (; p < p1; ++p) {
            q = pairs[p];
            s = s + ap[q & 0xffffu] * bp[q >> 16];
        }
        r[k] = (addc && k == 0) ? s + c : s;
    }
    __syncthreads();
}

__device__ Tv operator+(const Tv& a, const Tv& b) {
    if (!a.p && !b.p) return Tv(a.c + b.c);
    TCtx* x = ctx_of(a, b);
    ++x->nlin;
    double* r = t_alloc(x);
    ew_add(r, a.p, a.c, b.p, b.c, x->M, false);
    return Tv(r, x);
}

__device__ Tv operator-(const Tv& a) {
    if (!a.p) return Tv(-a.c);
    ++a.x->nlin;
    double* r = t_alloc(a.x);
    ew_neg(r, a.p, a.x->M);
    return Tv(r, a.x);
}

__device__ Tv operator-(const Tv& a, const Tv& b) {
    if (!a.p && !b.p) return Tv(a.c - b.c);
    TCtx* x = ctx_of(a, b);
    ++x->nlin;
    double* r = t_alloc(x);
    ew_add(r, a.p, a.c, b.p, b.c, x->M, true);
    return Tv(r, x);
}

__device__ Tv t_scale(const Tv& a, double s) {
    ++a.x->nlin;
    double* r = t_alloc(a.x);
    ew_scale(r, a.p, s, a.x->M);
    return Tv(r, a.x);
}

// dst = add + a*b (sub: add - a*b) with the product summed as in t_mul_raw and
// then combined, the rounding of the two separate operations; add may be dst.
static __device__ __noinline__ void t_mul_acc_raw(double* dst, const double* add, const double* __restrict__ ap,
                                                  const double* __restrict__ bp, const int4* __restrict__ otab,
                                                  const uint32_t* __restrict__ pairs, int olen, bool sub) {
    for (int o = threadIdx.x; o < olen; o += blockDim.x) {
        const int4 e = otab[o];
        const int k = e.x;
        if (k < 0) continue;
        int p = e.y;
        const int p1 = e.z;
        uint32_t q = pairs[p];
        double s = ap[q & 0xffffu] * bp[q >> 16];
        ++p;
        for (; p + 4 <= p1; p += 4) {
            const uint32_t q0 = pairs[p], q1 = pairs[p + 1], q2 = pairs[p + 2], q3 = pairs[p + 3];
            const double m0 = ap[q0 & 0xffffu] * bp[q0 >> 16];
            const double m1 = ap[q1 & 0xffffu] * bp[q1 >> 16];
            const double m2 = ap[q2 & 0xffffu] * bp[q2 >> 16];
            const double m3 = ap[q3 & 0xffffu] * bp[q3 >> 16];
            s = s + m0;
            s = s + m1;
            s = s + m2;
            s = s + m3;
        }
        for (; p < p1; ++p) {
            q = pairs[p];
            s = s + ap[q & 0xffffu] * bp[q >> 16];
        }
        const double v = add[k];
        dst[k] = sub ? v - s : v + s;
    }
    __syncthreads();
}

__device__ __forceinline__ void t_mul_acc(double* dst, const double* add, const Tv& a, const Tv& b, TCtx* x,
                                          bool sub) {
    ++x->nmul;
    ++x->nlin;
    t_mul_acc_raw(dst, add, a.p, b.p, x->otab, x->pairs, x->olen, sub);
}

__device__ __forceinline__ void t_mul_into(double* r, const Tv& a, const Tv& b, TCtx* x) {
    ++x->nmul;
    t_mul_raw(r, a.p, b.p, x->otab, x->pairs, x->olen);
}

__device__ Tv operator*(const Tv& a, const Tv& b) {
    if (!a.p && !b.p) return Tv(a.c * b.c);
    if (!a.p) return t_scale(b, a.c);
    if (!b.p) return t_scale(a, b.c);
    TCtx* x = ctx_of(a, b);
    double* r = t_alloc(x);
    t_mul_into(r, a, b, x);
    return Tv(r, x);
}

enum TFn { F_INV, F_SQRT, F_RSQRT, F_EXP, F_SIN, F_COS };

__device__ void fn_coef(TFn f, double a0, int N, double* c) {
    switch (f) {
        case F_INV:
            c[0] = 1.0 / a0;
            for (int k = 1; k <= N; ++k) c[k] = -c[k - 1] / a0;
            break;
        case F_SQRT:
            c[0] = sqrt(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] * (0.5 - double(k - 1)) / (double(k) * a0);
            break;
        case F_RSQRT:
            c[0] = 1.0 / sqrt(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] * (-0.5 - double(k - 1)) / (double(k) * a0);
            break;
        case F_EXP:
            c[0] = libm::exp(a0);
            for (int k = 1; k <= N; ++k) c[k] = c[k - 1] / double(k);
            break;
        default: {
            const double s0 = libm::sin(a0), c0 = libm::cos(a0);
            const double cyc_s[4] = {s0, c0, -s0, -c0};
            const double cyc_c[4] = {c0, -s0, -c0, s0};
            const double* cyc = f == F_SIN ? cyc_s : cyc_c;
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

// f(a) by Horner's rule in three slots (result, product, abar); the result
// ends in the first of them and the other two are released.
__device__ Tv t_apply(TFn f, const Tv& a) {
    double c[kTpsaMaxOrder + 1];
    if (!a.p) {
        fn_coef(f, a.c, 0, c);
        return Tv(c[0]);
    }
    TCtx* x = a.x;
    const int N = x->N, M = x->M;
    fn_coef(f, a.p[0], N, c);
    const int base = x->top;
    double* s0 = t_alloc(x);
    double* s1 = t_alloc(x);
    double* ab = t_alloc(x);
    {
        const double* __restrict__ ap = a.p;
        double* __restrict__ abr = ab;
        for (int k = threadIdx.x; k < M; k += blockDim.x) abr[k] = k == 0 ? 0.0 : ap[k];
        __syncthreads();
    }
    // r = c_N (a number); r = r * abar -> c_N abar (a scaling); then r = r + c_k
    double* r = s0;
    double* t = s1;
    if (N == 0) {
        for (int k = threadIdx.x; k < M; k += blockDim.x) r[k] = k == 0 ? c[0] : 0.0;
        __syncthreads();
    } else {
        ++x->nlin;
        {
            const double cn = c[N], cn1 = c[N - 1];
            const double* __restrict__ abr = ab;
            double* __restrict__ rr = r;
            for (int k = threadIdx.x; k < M; k += blockDim.x) {
                const double v = abr[k] * cn;
                rr[k] = k == 0 ? v + cn1 : v;
            }
            __syncthreads();
        }
        for (int j = N - 2; j >= 0; --j) {
            ++x->nmul;
            t_mul_raw(t, r, ab, x->otab, x->pairs, x->olen, true, c[j]);
            double* sw = r; r = t; t = sw;
        }
    }
    if (r != s0) ew_copy(s0, r, M);
    x->top = base + 1;
    return Tv(s0, x);
}

__device__ __forceinline__ Tv inv(const Tv& a) { return t_apply(F_INV, a); }
__device__ __forceinline__ Tv sqrt(const Tv& a) { return t_apply(F_SQRT, a); }
__device__ __forceinline__ Tv rsqrt(const Tv& a) { return t_apply(F_RSQRT, a); }
__device__ __forceinline__ Tv exp(const Tv& a) { return t_apply(F_EXP, a); }
__device__ __forceinline__ Tv sin(const Tv& a) { return t_apply(F_SIN, a); }
__device__ __forceinline__ Tv cos(const Tv& a) { return t_apply(F_COS, a); }

__device__ Tv operator/(const Tv& a, const Tv& b) {
    if (!b.p) {
        if (!a.p) return Tv(a.c / b.c);
        ++a.x->nlin;
        double* r = t_alloc(a.x);
        ew_div(r, a.p, b.c, a.x->M);
        return Tv(r, a.x);
    }
    return a * inv(b);
}

// The state: six series in slots 0..5.  set(i, v) copies v into slot i.
struct TState {
    TCtx* x;
    Tv r[6];
    __device__ void set(int i, const Tv& v) {
        double* d = r[i].p;
        if (v.p == d) return;
        const int M = x->M;
        if (v.p) {
            ew_copy(d, v.p, M);
        } else {
            const double vc = v.c;
            for (int k = threadIdx.x; k < M; k += blockDim.x) d[k] = k == 0 ? vc : 0.0;
            __syncthreads();
        }
    }
};

// Keep a statement's value in slot `mark` and release everything above it
// (the work slots of the expression); mark advances past the kept value.
__device__ Tv t_keep(const Tv& v, TCtx* x, int& mark) {
    if (!v.p) {
        x->top = mark;
        return v;
    }
    double* d = x->pool + size_t(mark) * x->M;
    if (v.p != d) ew_copy(d, v.p, x->M);
    x->top = ++mark;
    return Tv(d, x);
}
#define KEEP(v) t_keep((v), S.x, mk)

// ---------------------------------------------------------------------------
// Element maps (ext/TrackPadPolySeriesExt.jl).  Each releases its work slots.
// ---------------------------------------------------------------------------
// drift6_tpsa (:57-65), L / sqrt(pz2) as L * pz2^(-1/2)
// Each statement is the reference's expression, evaluated with every sum of a
// product fused into the product's pass (t_mul_acc): the same roundings in the
// same order, fewer passes and barriers.
__device__ void t_drift(TState& S, double L, double beti) {
    TCtx* x = S.x;
    const int m = x->top;
    const int M = x->M;
    Tv* r = S.r;
    // pz2 = 1 + 2 delta beti + delta^2 - px^2 - py^2, left to right
    double* pz2 = t_alloc(x);
    {
        const double* __restrict__ d = r[5].p;
        for (int k = threadIdx.x; k < M; k += blockDim.x) {
            const double v = (d[k] * 2.0) * beti;
            pz2[k] = k == 0 ? 1.0 + v : v;
        }
        ++x->nlin;
        __syncthreads();
    }
    t_mul_acc(pz2, pz2, r[5], r[5], x, false);
    t_mul_acc(pz2, pz2, r[1], r[1], x, true);
    t_mul_acc(pz2, pz2, r[3], r[3], x, true);
    // NormL = L / sqrt(pz2) as L * pz2^(-1/2)
    Tv NormL = t_scale(rsqrt(Tv(pz2, x)), L);
    // x and y in place: x_k = x_k + (NormL px)_k
    t_mul_acc(r[0].p, r[0].p, NormL, r[1], x, false);
    t_mul_acc(r[2].p, r[2].p, NormL, r[3], x, false);
    // z = z + NormL (beti + delta) - L beti
    double* u = t_alloc(x);
    {
        const double* __restrict__ d = r[5].p;
        for (int k = threadIdx.x; k < M; k += blockDim.x) u[k] = k == 0 ? beti + d[0] : d[k];
        ++x->nlin;
        __syncthreads();
    }
    t_mul_acc(r[4].p, r[4].p, NormL, Tv(u, x), x, false);
    if (threadIdx.x == 0) r[4].p[0] = r[4].p[0] - L * beti;
    __syncthreads();
    x->top = m;
}

// strthinkick_tpsa (:78-92) and bndthinkick_tpsa (:94-112)
__device__ void t_kick(TState& S, const double* pa, const double* pb, double L, int mo, bool bend, double irho,
                       double beti) {
    if (mo == 1) {
        // Order 1 (quadrupoles, dipole kicks): every output is a linear function
        // of the coordinates, evaluated in one pass with the reference's
        // operations per coefficient (the number terms only on the constant part).
        TCtx* x = S.x;
        const int M = x->M;
        const double re1 = pb[1], im1 = pa[1], pb0 = pb[0], pa0 = pa[0];
        const double Lirho = L * irho;
        const double* __restrict__ xs = S.r[0].p;
        const double* __restrict__ ys = S.r[2].p;
        const double* __restrict__ ds = S.r[5].p;
        double* pxs = S.r[1].p;
        double* pys = S.r[3].p;
        double* zs = S.r[4].p;
        for (int k = threadIdx.x; k < M; k += blockDim.x) {
            // ReSum = pb1 x - pa1 y + pb0, ImSum = pa1 x + pb1 y + pa0
            double re = xs[k] * re1 - ys[k] * im1;
            double im = xs[k] * im1 + ys[k] * re1;
            if (k == 0) {
                re = re + pb0;
                im = im + pa0;
            }
            if (!bend) {
                pxs[k] = pxs[k] - re * L;
            } else {
                pxs[k] = pxs[k] - (re - (ds[k] - xs[k] * irho) * irho) * L;
                zs[k] = zs[k] + (xs[k] * Lirho) * beti;
            }
            pys[k] = pys[k] + im * L;
        }
        x->nlin += bend ? 3 : 2;
        __syncthreads();
        return;
    }
    const int m = S.x->top;
    Tv* r = S.r;
    Tv ReSum(pb[mo]), ImSum(pa[mo]);
    // the running sums live in slots m and m+1 whatever the order
    if (m + 2 > S.x->nslots) {
        if (threadIdx.x == 0) atomicOr(S.x->err, TE_SLOTS);
        return;
    }
    double* const re_slot = S.x->pool + size_t(m) * S.x->M;
    double* const im_slot = re_slot + S.x->M;
    for (int i = mo - 1; i >= 0; --i) {
        int mk = m + 2;
        S.x->top = mk;
        Tv ReSumTemp = KEEP(ReSum * r[0] - ImSum * r[2] + Tv(pb[i]));
        Tv ImSumNew = KEEP(ImSum * r[0] + ReSum * r[2] + Tv(pa[i]));
        ew_copy(re_slot, ReSumTemp.p, S.x->M);
        ew_copy(im_slot, ImSumNew.p, S.x->M);
        ReSum = Tv(re_slot, S.x);
        ImSum = Tv(im_slot, S.x);
    }
    const int m2 = mo > 0 ? m + 2 : m;
    S.x->top = m2;
    // px, py and z do not feed each other: each is stored as soon as it is known
    if (!bend) {
        S.set(1, r[1] - Tv(L) * ReSum);
        S.x->top = m2;
        S.set(3, r[3] + Tv(L) * ImSum);
    } else {
        S.set(1, r[1] - Tv(L) * (ReSum - (r[5] - r[0] * Tv(irho)) * Tv(irho)));
        S.x->top = m2;
        S.set(3, r[3] + Tv(L) * ImSum);
        S.x->top = m2;
        S.set(4, r[4] + Tv(L) * Tv(irho) * r[0] * Tv(beti));
    }
    S.x->top = m;
}

// symplectic4_pass_tpsa / symplectic4_bend_pass_tpsa (:114-159)
__device__ void t_integrate(TState& S, const double* w, int mo, int nsteps, bool bend, double irho, double beti) {
    const double L1 = w[mp::L1], L2 = w[mp::L2], K1 = w[mp::K1], K2 = w[mp::K2];
    const double* pa = w + mp::PA;
    const double* pb = w + mp::PB;
    for (int s = 0; s < nsteps; ++s) {
        t_drift(S, L1, beti);
        t_kick(S, pa, pb, K1, mo, bend, irho, beti);
        t_drift(S, L2, beti);
        t_kick(S, pa, pb, K2, mo, bend, irho, beti);
        t_drift(S, L2, beti);
        t_kick(S, pa, pb, K1, mo, bend, irho, beti);
        t_drift(S, L1, beti);
    }
}

// edge_fringe_entrance_tpsa / _exit_tpsa (:161-215): fx, fy numbers, fy from
// the constant parts of delta and px.
__device__ void t_edge(TState& S, double irho, double fx, double ea, double fc, int method, bool is_exit) {
    const int m = S.x->top;
    Tv* r = S.r;
    const double d0 = cst(r[5]), px0 = cst(r[1]);
    double fy;
    if (method == 2) fy = irho * libm::tan(ea - fc / (1.0 + d0)) / (1.0 + d0);
    else if (method == 3) fy = irho * libm::tan(is_exit ? (ea - fc - px0 / (1.0 + d0)) : (ea - fc + px0 / (1.0 + d0)));
    else fy = irho * libm::tan(ea - fc / (1.0 + d0));
    Tv px_new = r[1] + r[0] * Tv(fx);
    Tv py_new = r[3] - r[2] * Tv(fy);
    S.set(1, px_new);
    S.set(3, py_new);
    S.x->top = m;
}

// Misalignment rows (:24-55)
__device__ void t_mis(TState& S, const double* t, const double* R, bool rot, bool entrance) {
    const int m = S.x->top;
    Tv* r = S.r;
    if (entrance) {
        for (int i = 0; i < 6; ++i) S.set(i, r[i] + Tv(t[i]));
        S.x->top = m;
    }
    if (rot) {
        Tv o[6];
        int mk = m;
        for (int i = 0; i < 6; ++i) {
            Tv s = Tv(R[i]) * r[0];
            for (int j = 1; j < 6; ++j) s = s + Tv(R[j * 6 + i]) * r[j];
            o[i] = KEEP(s);
        }
        for (int i = 0; i < 6; ++i) S.set(i, o[i]);
        S.x->top = m;
    }
    if (!entrance) {
        for (int i = 0; i < 6; ++i) S.set(i, r[i] + Tv(t[i]));
        S.x->top = m;
    }
}

__device__ void t_rf(TState& S, const double* w, const RecHdr& h, double beti) {
    const int m = S.x->top;
    Tv* r = S.r;
    const double beta = 1.0 / beti;
    if (h.flags & RF_LPOS) t_drift(S, w[rf::LH], beti);
    if (h.flags & RF_ENERGY) {
        int mk = m;
        Tv phase = KEEP(Tv(w[rf::W]) * ((r[4] - Tv(w[rf::LAG])) / Tv(C_LIGHT)) - Tv(w[rf::PHILAG]));
        Tv delta_new = KEEP(r[5] - Tv(w[rf::NV]) * sin(phase) / Tv(beta * beta));
        S.set(5, delta_new);
        S.x->top = m;
    }
    if (h.flags & RF_LPOS) t_drift(S, w[rf::LH], beti);
}

__device__ void t_solenoid(TState& S, const double* w, double beti) {
    const double ks = w[sol::KS], L = w[sol::L];
    if (ks == 0.0) {
        t_drift(S, L, beti);
        return;
    }
    const int m = S.x->top;
    int mk = m;
    Tv* r = S.r;
    Tv p_norm = KEEP(Tv(1.0) / (Tv(1.0) + r[5]));
    Tv x = r[0];
    Tv xpr = KEEP(r[1] * p_norm);
    Tv y = r[2];
    Tv ypr = KEEP(r[3] * p_norm);
    Tv H = KEEP(Tv(ks) * p_norm / Tv(2.0));
    Tv S_ = KEEP(sin(Tv(L) * H));
    Tv C = KEEP(cos(Tv(L) * H));
    Tv x_new = KEEP(x * C * C + xpr * C * S_ / H + y * C * S_ + ypr * S_ * S_ / H);
    Tv px_new = KEEP((-x * H * C * S_ + xpr * C * C - y * H * S_ * S_ + ypr * C * S_) / p_norm);
    Tv y_new = KEEP(-x * C * S_ - xpr * S_ * S_ / H + y * C * C + ypr * C * S_ / H);
    Tv py_new = KEEP((x * H * S_ * S_ - xpr * C * S_ - y * C * S_ * H + ypr * C * C) / p_norm);
    Tv z_new = KEEP(r[4] + Tv(L) * (H * H * (x * x + y * y) + Tv(2.0) * H * (xpr * y - ypr * x) + xpr * xpr +
                                    ypr * ypr) / Tv(2.0));
    S.set(0, x_new);
    S.set(1, px_new);
    S.set(2, y_new);
    S.set(3, py_new);
    S.set(4, z_new);
    S.x->top = m;
}

__device__ void t_corrector(TState& S, const double* w) {
    const int m = S.x->top;
    int mk = m;
    Tv* r = S.r;
    const Tv xk(w[cor::XK]), yk(w[cor::YK]);
    Tv p_norm = KEEP(Tv(1.0) / (Tv(1.0) + r[5]));
    Tv NormL = KEEP(Tv(w[cor::L]) * p_norm);
    Tv z_new = KEEP(r[4] + NormL * p_norm *
                               (xk * xk / Tv(3.0) + yk * yk / Tv(3.0) + r[1] * r[1] + r[3] * r[3] + r[1] * xk +
                                r[3] * yk) / Tv(2.0));
    Tv x_new = KEEP(r[0] + NormL * (r[1] + xk / Tv(2.0)));
    Tv px_new = KEEP(r[1] + xk);
    Tv y_new = KEEP(r[2] + NormL * (r[3] + yk / Tv(2.0)));
    Tv py_new = KEEP(r[3] + yk);
    S.set(0, x_new);
    S.set(1, px_new);
    S.set(2, y_new);
    S.set(3, py_new);
    S.set(4, z_new);
    S.x->top = m;
}

__device__ void t_translation(TState& S, const double* w, double beti) {
    const int m = S.x->top;
    int mk = m;
    Tv* r = S.r;
    Tv pz2 = KEEP(Tv(1.0) + Tv(2.0) * r[5] * Tv(beti) + r[5] * r[5] - r[1] * r[1] - r[3] * r[3]);
    Tv pz = KEEP(sqrt(pz2));
    const Tv dx(w[trn::DX]), dy(w[trn::DY]), ds(w[trn::DS]);
    Tv x_new = KEEP(r[0] - (dx + ds * r[1] / pz));
    Tv y_new = KEEP(r[2] - (dy + ds * r[3] / pz));
    Tv z_new = KEEP(r[4] + ds * (Tv(beti) + r[5]) / pz);
    S.set(0, x_new);
    S.set(2, y_new);
    S.set(4, z_new);
    S.x->top = m;
}

__device__ void t_yrotation(TState& S, const double* w, double beti) {
    const int m = S.x->top;
    int mk = m;
    Tv* r = S.r;
    const Tv ca(w[yr::CA]), sa(w[yr::SA]), ta(w[yr::TA]);
    Tv pz2 = KEEP(Tv(1.0) + Tv(2.0) * r[5] * Tv(beti) + r[5] * r[5] - r[1] * r[1] - r[3] * r[3]);
    Tv pz = KEEP(sqrt(pz2));
    Tv ptt = KEEP(Tv(1.0) - ta * r[1] / pz);
    Tv x_new = KEEP(r[0] / (ca * ptt));
    Tv px_new = KEEP(ca * r[1] + sa * pz);
    Tv y_new = KEEP(r[2] + ta * r[0] * r[3] / (pz * ptt));
    Tv z_new = KEEP(r[4] + ta * r[0] * (Tv(beti) + r[5]) / (pz * ptt));
    S.set(0, x_new);
    S.set(1, px_new);
    S.set(2, y_new);
    S.set(4, z_new);
    S.x->top = m;
}

__device__ void t_crab(TState& S, const double* w, const RecHdr& h, double beti) {
    const int m0 = S.x->top;
    Tv* r = S.r;
    const Tv volt(w[crab::VOLT]), E(w[crab::E]), kk(w[crab::K]);
    // the kick phase uses z before the first half drift: keep it in a slot
    double* angp = t_alloc(S.x);
    {
        const int m = S.x->top;
        Tv a = kk * r[4] + Tv(w[crab::PHI]);
        for (int k = threadIdx.x; k < S.x->M; k += blockDim.x) angp[k] = a.p ? a.p[k] : (k == 0 ? a.c : 0.0);
        __syncthreads();
        S.x->top = m;
    }
    const Tv ang(angp, S.x);
    if (h.flags & RF_LPOS) t_drift(S, w[crab::LH], beti);
    {
        const int m = S.x->top;
        int mk = m;
        Tv px_new = KEEP(r[1] + (volt / E) * sin(ang * Tv(beti)));
        Tv delta_new = KEEP(r[5] - (kk * volt / E * Tv(beti)) * r[0] * cos(ang * Tv(beti)));
        S.set(1, px_new);
        S.set(5, delta_new);
        S.x->top = m;
    }
    if (h.flags & RF_LPOS) t_drift(S, w[crab::LH], beti);
    S.x->top = m0;
}

__device__ void t_accel(TState& S, const double* w, double beti) {
    const double beta = 1.0 / beti;
    const double beta2 = beta * beta;
    if (beta2 <= EPSD) return;
    const int m = S.x->top;
    Tv* r = S.r;
    Tv sv = sin(Tv(w[acc::K]) * r[4] + Tv(w[acc::PHIS])) - Tv(w[acc::SINPHIS]);
    Tv delta_new = r[5] + (Tv(w[acc::VOLT]) / (Tv(beta2) * Tv(w[acc::E]))) * sv;
    S.set(5, delta_new);
    S.x->top = m;
}

__device__ void t_long_rf_map(TState& S, const double* w, double beti) {
    const int m = S.x->top;
    Tv* r = S.r;
    const double beta = 1.0 / beti;
    const double eta = w[lrf::ALPHAC] - (1.0 - beta * beta);
    Tv z_new = r[4] - Tv(6.283185307179586 * w[lrf::H] * eta / w[lrf::K]) * r[5];
    S.set(4, z_new);
    S.x->top = m;
}

__device__ void t_lorentz(TState& S, const double* w, bool inverse) {
    const int m = S.x->top;
    Tv* r = S.r;
    if (!inverse) {
        const Tv invcos(w[lor::A]), tanang(w[lor::B]);
        Tv x_new = r[0] + tanang * r[4];
        Tv delta_new = r[5] - tanang * r[1];
        Tv px = r[1] * invcos, py = r[3] * invcos, z = r[4] * invcos;
        S.set(0, x_new); S.set(1, px); S.set(3, py); S.set(4, z); S.set(5, delta_new);
    } else {
        const Tv cosang(w[lor::A]), sinang(w[lor::B]);
        Tv x_new = r[0] - sinang * r[4];
        Tv delta_new = r[5] + sinang * r[1];
        Tv px = r[1] * cosang, py = r[3] * cosang, z = r[4] * cosang;
        S.set(0, x_new); S.set(1, px); S.set(3, py); S.set(4, z); S.set(5, delta_new);
    }
    S.x->top = m;
}

__device__ void t_stgb(TState& S, const double* w) {
    const int m = S.x->top;
    int mk = m;
    Tv* r = S.r;
    const Tv amp(w[stg::AMP]), sx2(w[stg::SX2]), sy2(w[stg::SY2]);
    Tv dx = KEEP(r[0] - Tv(w[stg::XO]));
    Tv dy = KEEP(r[2] - Tv(w[stg::YO]));
    Tv g = KEEP(amp * exp(Tv(-0.5) * (dx * dx / sx2 + dy * dy / sy2)));
    Tv px_new = KEEP(r[1] - g * dx / sx2);
    Tv py_new = KEEP(r[3] - g * dy / sy2);
    S.set(1, px_new);
    S.set(3, py_new);
    S.x->top = m;
}

__device__ void t_sgb(TState& S, const double* w) {
    const int m = S.x->top;
    Tv* r = S.r;
    const int nz = int(w[sgb::NZ]);
    const double* wt = w + sgb::WORDS;
    const Tv factor(w[sgb::FACTOR]), sx2(w[sgb::SX2]), sy2(w[sgb::SY2]);
    // px, py accumulate in two work slots
    double* pxs = t_alloc(S.x);
    double* pys = t_alloc(S.x);
    ew_copy(pxs, r[1].p, S.x->M);
    ew_copy(pys, r[3].p, S.x->M);
    Tv px(pxs, S.x), py(pys, S.x);
    const int m2 = S.x->top;
    for (int i = 0; i < nz; ++i) {
        int mk = m2;
        Tv dx = KEEP(r[0] - Tv(wt[nz + i]));
        Tv dy = KEEP(r[2] - Tv(wt[2 * nz + i]));
        Tv g = KEEP(Tv(wt[i]) * exp(Tv(-0.5) * (dx * dx / sx2 + dy * dy / sy2)));
        Tv pxn = KEEP(px - factor * g * dx / sx2);
        Tv pyn = KEEP(py - factor * g * dy / sy2);
        ew_copy(pxs, pxn.p, S.x->M);
        ew_copy(pys, pyn.p, S.x->M);
        S.x->top = m2;
    }
    S.set(1, px);
    S.set(3, py);
    S.x->top = m;
}

// Wakes at the constant part of z (:630-649): a number added to delta.
__device__ void t_wake(TState& S, const double* w, const RecHdr& h) {
    P6 q{0.0, 0.0, 0.0, 0.0, cst(S.r[4]), 0.0};
    if (h.kind == DK_RLC_WAKE) rlc_wake(q, w);
    else tab_wake(q, w, h);
    if (threadIdx.x == 0) S.r[5].p[0] = S.r[5].p[0] + q.d;
    __syncthreads();
}

__device__ void t_nan(TState& S) {
    const double q = CUDART_NAN;
    for (int i = 0; i < 6; ++i)
        for (int k = threadIdx.x; k < S.x->M; k += blockDim.x) S.r[i].p[k] = k == 0 ? q : 0.0;
    __syncthreads();
}

// One record.  Returns false for a kind without a TPSA pass! method.
__device__ bool t_record(TState& S, const double* rec, const RecHdr& h, const MisalignDev* mis, double beti) {
    const double* w = rec + HDR_WORDS;
    if (h.flags & RF_MISALIGN) {
        const MisalignDev& md = mis[h.aux];
        t_mis(S, md.t1, md.r1, md.r1nz != 0, true);
    }
    switch (h.kind) {
        case DK_IDENTITY: break;
        case DK_DRIFT: t_drift(S, w[drift::L], beti); break;
        case DK_MULTIPOLE: t_integrate(S, w, h.order, h.nsteps, false, 0.0, beti); break;
        case DK_THIN: t_kick(S, w + thin::PA, w + thin::PB, 1.0, h.order, false, 0.0, beti); break;
        case DK_SBEND: {
            const double irho = w[sb::IRHO];
            if (h.flags & RF_FRINGE_IN)
                t_edge(S, irho, w[sb::FX_IN], w[sb::E_IN], w[sb::FC_IN], h.method_in, false);
            t_integrate(S, w, h.order, h.nsteps, true, irho, beti);
            if (h.flags & RF_FRINGE_OUT)
                t_edge(S, irho, w[sb::FX_OUT], w[sb::E_OUT], w[sb::FC_OUT], h.method_out, true);
            break;
        }
        case DK_RF: t_rf(S, w, h, beti); break;
        case DK_SOLENOID: t_solenoid(S, w, beti); break;
        case DK_CORRECTOR: t_corrector(S, w); break;
        case DK_TRANSLATION: t_translation(S, w, beti); break;
        case DK_YROTATION: t_yrotation(S, w, beti); break;
        case DK_CRAB: t_crab(S, w, h, beti); break;
        case DK_ACCEL: t_accel(S, w, beti); break;
        case DK_LONG_RF_MAP: t_long_rf_map(S, w, beti); break;
        case DK_LORENTZ: t_lorentz(S, w, false); break;
        case DK_INV_LORENTZ: t_lorentz(S, w, true); break;
        case DK_STRONG_THIN_GAUSS: t_stgb(S, w); break;
        case DK_SGB: t_sgb(S, w); break;
        case DK_RLC_WAKE: case DK_TAB_WAKE: t_wake(S, w, h); break;
        case DK_NAN: t_nan(S); break;
        default: return false;
    }
    if (h.flags & RF_MISALIGN) {
        const MisalignDev& md = mis[h.aux];
        t_mis(S, md.t2, md.r2, md.r2nz != 0, false);
    }
    return true;
}

struct TArgs {
    const double* table;
    int32_t nelem, N, M;
    int32_t sched_stride, sched_turn0, sched_nturns;
    const double* sched;
    const MisalignDev* mis;
    const int4* otab;
    const uint32_t* pairs;
    int32_t olen;
    double* maps;            // nmaps x 6 x M
    int64_t nmaps;
    double* gpool;           // per-CTA slabs when the pool is not in shared memory
    double beti;
    int32_t nturns, turn0;
    int32_t* err;
    unsigned long long* ops;  // [series products, elementwise operations, most slots held] over all maps
    int32_t slots;            // series slots per map
};

__global__ void __launch_bounds__(256) tpsa_track(TArgs a) {
    extern __shared__ __align__(16) double tsm[];
    TCtx X;
    X.pool = a.gpool ? a.gpool + size_t(blockIdx.x) * a.slots * a.M : tsm;
    X.nslots = a.slots;
    X.otab = a.otab;
    X.olen = a.olen;
    X.pairs = a.pairs;
    X.M = a.M;
    X.N = a.N;
    X.err = a.err;
    X.nmul = 0;
    X.nlin = 0;
    X.maxtop = 6;
    const int M = a.M;
    for (int64_t mi = blockIdx.x; mi < a.nmaps; mi += gridDim.x) {
        X.top = 6;
        TState S;
        S.x = &X;
        for (int i = 0; i < 6; ++i) S.r[i] = Tv(X.pool + size_t(i) * M, &X);
        const double* src = a.maps + mi * 6 * M;
        for (int k = threadIdx.x; k < 6 * M; k += blockDim.x) X.pool[k] = src[k];
        __syncthreads();
        for (int t = 0; t < a.nturns; ++t) {
            const double* rec = a.table;
            for (int e = 0; e < a.nelem; ++e) {
                RecHdr h = *reinterpret_cast<const RecHdr*>(rec);
                const double* next = rec + h.words;
                const double* r = rec;
                if (h.flags & RF_SCHEDULED) {
                    const int row = a.turn0 + t - a.sched_turn0;
                    if (a.sched == nullptr || row < 0 || row >= a.sched_nturns) {
                        if (threadIdx.x == 0) atomicOr(a.err, TE_SCHED);
                        r = nullptr;
                    } else {
                        r = a.sched + int64_t(row) * a.sched_stride + h.aux;
                        h = *reinterpret_cast<const RecHdr*>(r);
                    }
                }
                if (r != nullptr && !t_record(S, r, h, a.mis, a.beti)) {
                    if (threadIdx.x == 0) atomicOr(a.err, TE_KIND);
                }
                rec = next;
            }
        }
        double* dst = a.maps + mi * 6 * M;
        for (int k = threadIdx.x; k < 6 * M; k += blockDim.x) dst[k] = X.pool[k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(a.ops, X.nmul);
        atomicAdd(a.ops + 1, X.nlin);
        atomicMax(a.ops + 2, (unsigned long long)X.maxtop);
    }
}

int fail(int st, const std::string& m) {
    set_last_error(m);
    return st;
}

thread_local tp_tpsa_stats g_tpsa_stats{};
// Slots the last call on a (lattice program, order) used; keyed by the
// lattice's stamp (unique per program) and the order.
std::mutex g_slot_mu;
std::unordered_map<uint64_t, int> g_slot_cache;

bool tpsa_kind_ok(int kind) {
    return kind != DK_EXACT_SBEND && kind != DK_LBEND && kind != DK_WIGGLER && kind >= 0 && kind < DK_COUNT;
}

}  // namespace
}  // namespace tp

using namespace tp;

#define TPSA_CUDA(call)                                                                             \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(TP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

TP_API int tp_tpsa_coefficients(int32_t order, int64_t* ncoef) {
    if (order < 0 || order > kTpsaMaxOrder) return fail(TP_ERANGE, "TPSA order outside 0..10");
    if (!ncoef) return fail(TP_EINVAL, "ncoef is null");
    int64_t m = 1;
    for (int i = 1; i <= 6; ++i) m = m * (order + i) / i;
    *ncoef = m;
    return TP_OK;
}

TP_API int tp_tpsa_monomials(int32_t order, int32_t* exps) {
    if (order < 0 || order > kTpsaMaxOrder) return fail(TP_ERANGE, "TPSA order outside 0..10");
    if (!exps) return fail(TP_EINVAL, "exps is null");
    const TpsaTables& t = tables_of(order);
    std::memcpy(exps, t.mono.data(), t.mono.size() * sizeof(int32_t));
    return TP_OK;
}

TP_API int tp_tpsa_ringpass(tp_ctx* ctx, const tp_lattice* lat, double* maps, int64_t nmaps, int32_t order,
                            double beti, int32_t nturns, int32_t turn0) {
    tp::NvtxRange nvtx_range("tp_tpsa_ringpass");
    if (!ctx || !lat) return fail(TP_EINVAL, "null context or lattice");
    if (order < 0 || order > kTpsaMaxOrder) return fail(TP_ERANGE, "TPSA order outside 0..10");
    if (nmaps < 0 || nturns < 0) return fail(TP_EINVAL, "negative size");
    if (nmaps > 0 && !maps) return fail(TP_EINVAL, "maps is null");
    if (!(beti > 0.0) || !std::isfinite(beti)) return fail(TP_EINVAL, "beti must be finite and positive");
    LatticeHost L;
    lattice_host(lat, &L);
    for (int32_t e = 0; e < L.nelem; ++e) {
        RecHdr h;
        std::memcpy(&h, L.program + L.rec_off[e], sizeof h);
        if (!tpsa_kind_ok(h.kind))
            return fail(TP_EUNSUPPORTED, "element " + std::to_string(e) + " (kind " +
                                             std::to_string(L.elems[e].kind) +
                                             ") has no TPSA pass! method (ExactSBend, LBend, Wiggler)");
    }
    if (L.has_schedule && (int64_t(turn0) < L.sched_turn0 ||
                           int64_t(turn0) + nturns > int64_t(L.sched_turn0) + L.sched_nturns))
        return fail(TP_ERANGE, "turns outside the lattice schedule");
    if (nmaps == 0 || nturns == 0) return TP_OK;
    const TpsaTables& T = tables_of(order);
    const int M = T.M;
    CtxHost ch;
    ctx_host(ctx, &ch);
    TPSA_CUDA(cudaSetDevice(ch.device));
    cudaStream_t s = static_cast<cudaStream_t>(ch.stream);

    // device copies: program, schedule, misalignment rows, tables, error word
    std::vector<MisalignDev> md(size_t(L.nmis));
    for (int64_t i = 0; i < L.nmis; ++i) {
        const tp_misalign& m = L.mis[i];
        MisalignDev& o = md[size_t(i)];
        o = MisalignDev{};
        std::memcpy(o.t1, m.t1, sizeof o.t1); std::memcpy(o.t2, m.t2, sizeof o.t2);
        std::memcpy(o.r1, m.r1, sizeof o.r1); std::memcpy(o.r2, m.r2, sizeof o.r2);
        for (int k = 0; k < 36; ++k) { o.r1nz |= m.r1[k] != 0.0; o.r2nz |= m.r2[k] != 0.0; }
    }
    // launch shape: about four coefficients per thread, enough work per
    // operation to carry its barrier, and small CTAs so that registers allow
    // 8 maps per SM
    int block = (M / 4 + 31) / 32 * 32;
    block = std::max(32, std::min(256, block));
    // Product outputs dealt to threads by pair count, longest first to the
    // least loaded thread: a product takes as long as its busiest thread (at
    // order 6 the strided split gave one thread 122 pairs, this one 76).  The
    // sum of each output keeps its pair order, so the bits do not change.
    // Measured on the FODO ring (six variables): orders 5 / 6 / 7 run 16 / 7 /
    // 18 % faster; at orders 2 and 4, whose busiest thread sums 4 and 38 pairs,
    // the indirection cost more than the balance saved (15 and 5 % slower), so
    // the dealt order is used only when the strided split leaves a thread
    // TP_TPSA_DEAL_MIN pairs or more and the dealt one lowers that.  Slot o of
    // the table holds {output k (-1: none), first pair, end pair, 0}; thread t
    // takes slots t, t + block, ...
    std::vector<int32_t> otab;
    {
        auto npairs = [&](int32_t k) { return int64_t(T.poff[size_t(k) + 1]) - T.poff[size_t(k)]; };
        int64_t strided_max = 0;
        for (int t = 0; t < block; ++t) {
            int64_t l = 0;
            for (int k = t; k < M; k += block) l += npairs(k);
            strided_max = std::max(strided_max, l);
        }
        std::vector<int32_t> idx(static_cast<size_t>(M));
        for (int k = 0; k < M; ++k) idx[size_t(k)] = k;
        std::stable_sort(idx.begin(), idx.end(), [&](int32_t u, int32_t v) {
            return npairs(u) > npairs(v);
        });
        std::vector<int64_t> load(static_cast<size_t>(block), 0);
        std::vector<std::vector<int32_t>> lists(static_cast<size_t>(block));
        for (int32_t k : idx) {
            size_t best = 0;
            for (size_t t = 1; t < load.size(); ++t)
                if (load[t] < load[best]) best = t;
            load[best] += npairs(k);
            lists[best].push_back(k);
        }
        const int64_t dealt_max = *std::max_element(load.begin(), load.end());
        auto put = [&](size_t o, int32_t k) {
            otab[4 * o] = k;
            otab[4 * o + 1] = T.poff[size_t(k)];
            otab[4 * o + 2] = T.poff[size_t(k) + 1];
        };
        if (strided_max >= TP_TPSA_DEAL_MIN && dealt_max < strided_max) {
            size_t depth = 0;
            for (const auto& l : lists) depth = std::max(depth, l.size());
            otab.assign(4 * depth * size_t(block), 0);
            for (size_t o = 0; o < depth * size_t(block); ++o) otab[4 * o] = -1;
            for (size_t t = 0; t < lists.size(); ++t)
                for (size_t j = 0; j < lists[t].size(); ++j) put(t + j * size_t(block), lists[t][j]);
        } else {
            otab.assign(4 * size_t(M), 0);
            for (int k = 0; k < M; ++k) put(size_t(k), k);
        }
    }
    const int32_t olen = int32_t(otab.size() / 4);
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_tab = up(L.words * 8), b_sch = up(L.sched_words * 8), b_mis = up(md.size() * sizeof(MisalignDev));
    const size_t b_otab = up(otab.size() * 4), b_pairs = up(T.pairs.size() * 4), b_err = 256;  // err + ops
    void* d_tab = nullptr;
    int st = ctx_scratch(ctx, kTpsaScratchTable, b_tab + b_sch + b_mis + b_otab + b_pairs + b_err, &d_tab);
    if (st != TP_OK) return st;
    char* base = static_cast<char*>(d_tab);
    double* dtable = reinterpret_cast<double*>(base);
    double* dsched = reinterpret_cast<double*>(base + b_tab);
    MisalignDev* dmis = reinterpret_cast<MisalignDev*>(base + b_tab + b_sch);
    int4* dotab = reinterpret_cast<int4*>(base + b_tab + b_sch + b_mis);
    uint32_t* dpairs = reinterpret_cast<uint32_t*>(base + b_tab + b_sch + b_mis + b_otab);
    int32_t* derr = reinterpret_cast<int32_t*>(base + b_tab + b_sch + b_mis + b_otab + b_pairs);
    TPSA_CUDA(cudaMemcpyAsync(dtable, L.program, L.words * 8, cudaMemcpyHostToDevice, s));
    if (L.sched_words) TPSA_CUDA(cudaMemcpyAsync(dsched, L.sched, L.sched_words * 8, cudaMemcpyHostToDevice, s));
    if (!md.empty()) TPSA_CUDA(cudaMemcpyAsync(dmis, md.data(), md.size() * sizeof(MisalignDev), cudaMemcpyHostToDevice, s));
    TPSA_CUDA(cudaMemcpyAsync(dotab, otab.data(), otab.size() * 4, cudaMemcpyHostToDevice, s));
    TPSA_CUDA(cudaMemcpyAsync(dpairs, T.pairs.data(), T.pairs.size() * 4, cudaMemcpyHostToDevice, s));
    unsigned long long* dops = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(derr) + 16);
    TPSA_CUDA(cudaMemsetAsync(derr, 0, 48, s));

    const size_t map_bytes = size_t(nmaps) * 6 * M * 8;
    void* d_maps = nullptr;
    if ((st = ctx_scratch(ctx, kTpsaScratchMaps, map_bytes, &d_maps)) != TP_OK) return st;
    TPSA_CUDA(cudaMemcpyAsync(d_maps, maps, map_bytes, cudaMemcpyHostToDevice, s));

    // series slots: the longer bodies hold more work series at once
    bool rare = L.nmis > 0;
    for (int32_t e = 0; e < L.nelem; ++e) {
        RecHdr h;
        std::memcpy(&h, L.program + L.rec_off[e], sizeof h);
        rare = rare || (h.kind > DK_RF && h.kind != DK_LONG_RF_MAP && h.kind != DK_LORENTZ &&
                        h.kind != DK_INV_LORENTZ && h.kind != DK_RLC_WAKE && h.kind != DK_TAB_WAKE && h.kind != DK_NAN);
    }
    const int slots_full = rare ? kSlotsRare : kSlotsCore;
    // The pool's slot count bounds the maps resident per SM.  A lattice's
    // series bodies take the same slots whatever the coefficients (allocation
    // follows the code path, which follows the element kinds), so a call
    // sizes the pool by what the previous call on this lattice program and
    // order used; if that runs out (TE_SLOTS), it runs again with the full pool.
    LatticeView lv;
    lattice_view(lat, &lv);
    const uint64_t slot_key = lv.stamp * 16 + uint64_t(order);
    int slots = slots_full;
    {
        std::lock_guard<std::mutex> g(g_slot_mu);
        auto it = g_slot_cache.find(slot_key);
        if (it != g_slot_cache.end()) slots = std::max(7, std::min(slots_full, it->second));
    }
    tp_tpsa_stats& g = g_tpsa_stats;
    for (int attempt = 0;; ++attempt) {
        const size_t pool_bytes = size_t(slots) * M * 8;
        // shared memory when it leaves room for at least two maps per SM (one map
        // per SM is latency-bound: order 6 ran 2.2x faster from an L2-resident
        // global pool at three maps per SM than from shared memory at one)
        bool in_smem = pool_bytes + 1024 <= ch.smem_optin;
        int per_sm = 1;
        if (in_smem) {
            if (pool_bytes > 48 * 1024)
                TPSA_CUDA(cudaFuncSetAttribute(tpsa_track, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(pool_bytes)));
            TPSA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tpsa_track, block, pool_bytes));
            in_smem = per_sm >= 2;
        }
        if (!in_smem) per_sm = 3;
        const int64_t grid = std::min<int64_t>(nmaps, int64_t(ch.sm_count) * per_sm);
        double* gpool = nullptr;
        if (!in_smem) {
            void* p = nullptr;
            if ((st = ctx_scratch(ctx, kTpsaScratchPool, size_t(grid) * pool_bytes, &p)) != TP_OK) return st;
            gpool = static_cast<double*>(p);
        }
        if (attempt > 0) {  // the first attempt overwrote the device maps: stage them again
            TPSA_CUDA(cudaMemcpyAsync(d_maps, maps, map_bytes, cudaMemcpyHostToDevice, s));
            TPSA_CUDA(cudaMemsetAsync(derr, 0, 48, s));
        }
        TArgs a{};
        a.table = dtable;
        a.nelem = L.nelem;
        a.N = order;
        a.M = M;
        a.sched = L.sched_words ? dsched : nullptr;
        a.sched_stride = L.sched_stride;
        a.sched_turn0 = L.sched_turn0;
        a.sched_nturns = L.sched_nturns;
        a.mis = md.empty() ? nullptr : dmis;
        a.otab = dotab;
        a.pairs = dpairs;
        a.olen = olen;
        a.maps = static_cast<double*>(d_maps);
        a.nmaps = nmaps;
        a.gpool = gpool;
        a.beti = beti;
        a.nturns = nturns;
        a.turn0 = turn0;
        a.err = derr;
        a.ops = dops;
        a.slots = slots;
        cudaEvent_t e0, e1;
        TPSA_CUDA(cudaEventCreate(&e0));
        TPSA_CUDA(cudaEventCreate(&e1));
        cudaEventRecord(e0, s);
        tpsa_track<<<int(grid), block, in_smem ? pool_bytes : 0, s>>>(a);
        cudaEventRecord(e1, s);
        cudaError_t le = cudaGetLastError();
        int32_t herr = 0;
        unsigned long long hops[3] = {0, 0, 0};
        if (le == cudaSuccess) le = cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, s);
        if (le == cudaSuccess) le = cudaMemcpyAsync(hops, dops, 24, cudaMemcpyDeviceToHost, s);
        if (le == cudaSuccess) le = cudaStreamSynchronize(s);
        float ms = 0.f;
        if (le == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (le != cudaSuccess) return fail(TP_ECUDA, std::string("TPSA kernel: ") + cudaGetErrorString(le));
        if ((herr & TE_SLOTS) && slots < slots_full) {
            std::lock_guard<std::mutex> lk(g_slot_mu);
            g_slot_cache.erase(slot_key);
            slots = slots_full;
            continue;
        }
        g = tp_tpsa_stats{};
        g.maps = nmaps;
        g.order = order;
        g.coefficients = M;
        g.pairs = int64_t(T.pairs.size());
        g.series_mul = double(hops[0]);
        g.series_lin = double(hops[1]);
        g.flops = g.series_mul * (2.0 * double(T.pairs.size()) - double(M)) + g.series_lin * double(M);
        g.kernel_ms = ms;
        g.grid = int32_t(grid);
        g.block = block;
        g.shared_pool = in_smem ? 1 : 0;
        g.slots_used = int32_t(hops[2]);
        g.slots = slots;
        if (herr & TE_SLOTS) return fail(TP_ERANGE, "TPSA work slots exhausted (internal limit)");
        if (herr & TE_KIND) return fail(TP_EUNSUPPORTED, "a record without a TPSA pass! method");
        if (herr & TE_SCHED) return fail(TP_ERANGE, "turn outside the lattice schedule");
        if (g.slots_used > 0) {
            std::lock_guard<std::mutex> lk(g_slot_mu);
            g_slot_cache[slot_key] = g.slots_used;
        }
        break;
    }
    TPSA_CUDA(cudaMemcpyAsync(maps, d_maps, map_bytes, cudaMemcpyDeviceToHost, s));
    TPSA_CUDA(cudaStreamSynchronize(s));
    tp_stats* stt = ctx_stats(ctx);
    stt->h2d_bytes += map_bytes;
    stt->d2h_bytes += map_bytes;
    return TP_OK;
}

TP_API int tp_tpsa_last_stats(tp_tpsa_stats* out) {
    if (!out) return fail(TP_EINVAL, "out is null");
    *out = g_tpsa_stats;
    return TP_OK;
}

// tp_adjoint.cu -- gradients of a tracked-beam loss (reverse mode) and the
// one-turn Jacobian, on the device.
//
// The reference has no adjoint (its Enzyme extension is a stub,
// ext/TrackPadEnzymeExt.jl:14-17); its one_turn_map (src/optics.jl:110-121)
// takes finite differences.  Here both are exact derivatives of the tracked
// maps, computed in two launches over 32-particle tiles (one warp each):
//
//  forward  tracks every particle like ringpass! (same maps, same loss rule,
//           no FMA contraction) and stores its state at the start of every
//           K-th turn (the checkpoints) and at the end;
//  reverse  walks each K-turn segment backwards from the stored state at its
//           end, rebuilding the state before every building block with the
//           block's exact time-reversed map (tp_reverse.cuh,
//           tp_reverse_kinds.cuh) while pulling
//           the cotangent back through it.  At the start of the segment the
//           rebuilt state is compared with the stored one (the reconstruction
//           error reported in tp_adjoint_stats).
//
// Gradient accumulation is deterministic: the cotangent contribution of a
// parameter element is summed over the warp with shuffles in a fixed order
// and added by lane 0 to the tile's own row of partial sums; a final kernel
// sums the rows of each variant in tile order.  The loss's survivor set is
// the forward run's, so the lost-fraction term contributes no gradient.
//
// Seeds.  Loss mode: the cotangent of the final state of a survivor is
// d q / d state with q = (x^2 + y^2) / sigma^2, so that the tile sums are
// sum_s dq_s/dk; the final kernel divides by the survivor count.  Jacobian
// mode: particle 6*i + j is a copy of orbit i seeded with e_j, and its final
// cotangent is row j of the orbit's tangent map.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "tp_internal.h"
#include "tp_maps.cuh"
#include "tp_reverse_kinds.cuh"

namespace tp {
namespace {

using namespace tp::dev;

constexpr int kTile = 32;
// 64-thread blocks (two 32-particle tiles): with 128 registers, 8 resident per
// SM.  The gradient workload (65,536 particles) has fewer warps than the GPU's
// slots, and smaller blocks spread them evenly over the SMs (2,048 warps: 13 or
// 14 per SM instead of 12 or 16 with 128-thread blocks); measured 3 % faster.
constexpr int kAdjBlock = 64;

// One variant (lattice) of an adjoint launch.
struct AdjVar {
    int64_t toff;     // word offset of its table in AdjArgs::table
    int64_t eoff;     // offset of its per-element info in AdjArgs::einfo (2 ints per element)
    int64_t p0, p1;   // its particles [p0, p1)
    int64_t tile0;    // its first tile
    int64_t prow;     // word offset of its first tile's partial-gradient row
    int64_t soff;     // word offset of its schedule in AdjArgs::sched (-1: none)
    double beti;
    int32_t nelem, nparams;
    int32_t sstride, sturn0, snturns, pad;
};

struct AdjArgs {
    const double* table;
    const int32_t* einfo;     // per element: record word offset, parameter code (slot*4 + pm, or -1)
    const double* sched;
    const AdjVar* var;
    const MisalignDev* mis;   // misalignment rows of every variant (record aux indexes them)
    const double* misinv;     // their inverses, 72 words per row (r1^-1, r2^-1)
    int32_t nvar;
    int32_t nturns;
    int32_t turn0;
    int32_t K;                // turns per checkpoint segment
    int32_t nseg;             // ceil(nturns / K)
    int32_t mode;             // 0 = loss, 1 = Jacobian seeds
    int64_t ntot;             // particles over all variants
    int64_t ntiles;
    const double* coords0;    // ntot x 6 column-major (read only)
    const int64_t* lost0;
    double* fin;              // final state (ntot x 6)
    int64_t* lost;            // final flags
    double* ckpt;             // (nseg - 1) x 6 x ntot
    double limx, limy;
    double inv_sigma2;
    double* partial;          // gradient rows
    double* tile_q;           // per tile: sum of q over survivors
    int64_t* tile_cnt;        // per tile: alive at start, survivors
    double* tile_rec;         // per tile: max reconstruction error
    double* seed_out;         // Jacobian mode: final cotangents, ntot x 6 row-major
    int32_t* err;
    int32_t smem_words;       // table + einfo words staged in shared memory (single variant)
};

__device__ __forceinline__ void ld6(const double* c, int64_t n, int64_t i, P6& s) {
    s.x = c[i]; s.px = c[n + i]; s.y = c[2 * n + i]; s.py = c[3 * n + i]; s.z = c[4 * n + i]; s.d = c[5 * n + i];
}
__device__ __forceinline__ void st6(double* c, int64_t n, int64_t i, const P6& s) {
    c[i] = s.x; c[n + i] = s.px; c[2 * n + i] = s.y; c[3 * n + i] = s.py; c[4 * n + i] = s.z; c[5 * n + i] = s.d;
}

__device__ __forceinline__ bool lost_check(const P6& s, double limx, double limy) {
    return isnan(s.x) || fabs(s.x) > limx || fabs(s.y) > limy || fabs(s.px) > 1.0 || fabs(s.py) > 1.0;
}

__device__ __forceinline__ int find_var(const AdjVar* var, int nvar, int64_t tile) {
    int lo = 0, hi = nvar - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (var[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ const double* resolve_rec(const double* rec, RecHdr& h, const double* sched,
                                                     const AdjVar& V, int turn) {
    if (!(h.flags & RF_SCHEDULED)) return rec;
    int row = turn - V.sturn0;
    if (V.soff < 0 || row < 0 || row >= V.snturns) return nullptr;
    const double* p = sched + V.soff + int64_t(row) * V.sstride + h.aux;
    h = *reinterpret_cast<const RecHdr*>(p);
    return p;
}

// Stage the single variant's table and element info into shared memory.
__device__ void stage_plain(double* dst, const double* tab, int words_tab, const int32_t* einfo, int words_info) {
    for (int i = threadIdx.x; i < words_tab; i += blockDim.x) dst[i] = tab[i];
    int32_t* di = reinterpret_cast<int32_t*>(dst + words_tab);
    for (int i = threadIdx.x; i < 2 * words_info; i += blockDim.x) di[i] = einfo[i];
    __syncthreads();
}

template <bool EXACT, bool RARE>
__global__ void __launch_bounds__(kAdjBlock, 8) adj_forward(AdjArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int lane = threadIdx.x & 31;
    const int64_t tile = int64_t(blockIdx.x) * (kAdjBlock / 32) + (threadIdx.x >> 5);
    const double* tab_s = nullptr;
    if (a.smem_words > 0) {
        const AdjVar& V0 = a.var[0];
        stage_plain(smem, a.table, int(a.smem_words) - V0.nelem, a.einfo, V0.nelem);
        tab_s = smem;
    }
    if (tile >= a.ntiles) return;
    const int v = find_var(a.var, a.nvar, tile);
    const AdjVar V = a.var[v];
    const double* tab = tab_s ? tab_s : a.table + V.toff;
    const int64_t p = V.p0 + kTile * (tile - V.tile0) + lane;
    const bool valid = p < V.p1;
    const double beti = V.beti;
    const double beta = 1.0 / beti;
    const double beta2 = beta * beta;
    P6 s{};
    int64_t lf = 1;
    if (valid) {
        ld6(a.coords0, a.ntot, p, s);
        lf = a.lost0 ? a.lost0[p] : 0;
    }
    bool act = valid && lf != 1;
    const int alive0 = __popc(__ballot_sync(0xffffffffu, act));
    for (int t = 0; t < a.nturns; ++t) {
        if (__ballot_sync(0xffffffffu, act) == 0) break;
        if (t > 0 && (t % a.K) == 0 && act) st6(a.ckpt + int64_t(t / a.K - 1) * 6 * a.ntot, a.ntot, p, s);
        const double* rec = tab;
        for (int e = 0; e < V.nelem; ++e) {
            RecHdr h0 = *reinterpret_cast<const RecHdr*>(rec);
            const double* next = rec + h0.words;
            if (act) {
                RecHdr h = h0;
                const double* r = resolve_rec(rec, h, a.sched, V, a.turn0 + t);
                P6 sn = s;
                if (r == nullptr || !apply_record<EXACT, RARE>(sn, r, h, RARE ? a.mis : nullptr, beti, beta, beta2)) {
                    atomicOr(a.err, r == nullptr ? DE_SCHED_RANGE : DE_BAD_KIND);
                    act = false;
                    lf = 1;
                } else if (lost_check(sn, a.limx, a.limy)) {
                    act = false;  // entrance coordinates are kept (src/lattice.jl:281-284)
                    lf = 1;
                } else {
                    s = sn;
                }
            }
            rec = next;
        }
    }
    double q = 0.0;
    if (valid) {
        st6(a.fin, a.ntot, p, s);
        a.lost[p] = lf;
        if (act) q = (s.x * s.x + s.y * s.y) * a.inv_sigma2;
    }
    const int surv = __popc(__ballot_sync(0xffffffffu, act));
    for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
    if (lane == 0) {
        a.tile_q[tile] = q;
        a.tile_cnt[2 * tile] = alive0;
        a.tile_cnt[2 * tile + 1] = surv;
    }
}

template <bool EXACT, bool RARE>
__global__ void __launch_bounds__(kAdjBlock, 8) adj_reverse(AdjArgs a) {
    extern __shared__ __align__(16) double smem[];
    const int lane = threadIdx.x & 31;
    const int64_t tile = int64_t(blockIdx.x) * (kAdjBlock / 32) + (threadIdx.x >> 5);
    const double* tab_s = nullptr;
    const int32_t* info_s = nullptr;
    if (a.smem_words > 0) {
        const AdjVar& V0 = a.var[0];
        const int wt = int(a.smem_words) - V0.nelem;  // table words (the info takes nelem words)
        stage_plain(smem, a.table, wt, a.einfo, V0.nelem);
        tab_s = smem;
        info_s = reinterpret_cast<const int32_t*>(smem + wt);
    }
    if (tile >= a.ntiles) return;
    const int v = find_var(a.var, a.nvar, tile);
    const AdjVar V = a.var[v];
    const double* tab = tab_s ? tab_s : a.table + V.toff;
    const int32_t* info = info_s ? info_s : a.einfo + 2 * V.eoff;
    const int64_t p = V.p0 + kTile * (tile - V.tile0) + lane;
    const bool valid = p < V.p1;
    const bool surv = valid && a.lost[p] != 1;
    if (__ballot_sync(0xffffffffu, surv) == 0) {
        if (lane == 0) a.tile_rec[tile] = 0.0;
        return;
    }
    const double beti = V.beti;
    const double beta = 1.0 / beti;
    const double beta2 = beta * beta;
    double* row = a.partial + V.prow + (tile - V.tile0) * int64_t(V.nparams);
    P6 s{};
    L6 l{};
    if (surv) {
        ld6(a.fin, a.ntot, p, s);
        if (a.mode == 0) {
            l.x = 2.0 * s.x * a.inv_sigma2;
            l.y = 2.0 * s.y * a.inv_sigma2;
        } else {
            const int j = int((p - V.p0) % 6);
            l.x = j == 0; l.px = j == 1; l.y = j == 2; l.py = j == 3; l.z = j == 4; l.d = j == 5;
        }
    }
    double rec_err = 0.0;
    for (int seg = a.nseg - 1; seg >= 0; --seg) {
        const int t_lo = seg * a.K;
        const int t_hi = min(a.nturns, t_lo + a.K);
        if (seg < a.nseg - 1 && surv) ld6(a.ckpt + int64_t(seg) * 6 * a.ntot, a.ntot, p, s);
        for (int t = t_hi - 1; t >= t_lo; --t) {
            for (int e = V.nelem - 1; e >= 0; --e) {
                const int32_t off = info[2 * e];
                const int32_t code = info[2 * e + 1];
                double g = 0.0;
                if (surv) {
                    const double* rec = tab + off;
                    RecHdr h = *reinterpret_cast<const RecHdr*>(rec);
                    const double* r = resolve_rec(rec, h, a.sched, V, a.turn0 + t);
                    const int pm = code >= 0 ? (code & 3) : 0;
                    if (r == nullptr || !reverse_record<EXACT, RARE>(s, l, r, h, a.mis, a.misinv, beti, beta, beta2, pm, g))
                        atomicOr(a.err, r == nullptr ? DE_SCHED_RANGE : DE_BAD_KIND);
                }
                if (code >= 0) {  // warp-uniform: every lane walks the same variant
                    for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
                    if (lane == 0) {
                        const int pm = code & 3;
                        const double cm = pm == 1 ? 1.0 : (pm == 2 ? 0.5 : 1.0 / 6.0);
                        row[code >> 2] += cm * g;
                    }
                }
            }
        }
        if (surv) {
            // The rebuilt state at the segment start against the stored one.
            P6 ref;
            if (seg > 0) ld6(a.ckpt + int64_t(seg - 1) * 6 * a.ntot, a.ntot, p, ref);
            else ld6(a.coords0, a.ntot, p, ref);
            double m = fabs(s.x - ref.x);
            m = fmax(m, fabs(s.px - ref.px));
            m = fmax(m, fabs(s.y - ref.y));
            m = fmax(m, fabs(s.py - ref.py));
            m = fmax(m, fabs(s.z - ref.z));
            m = fmax(m, fabs(s.d - ref.d));
            if (!(m <= rec_err)) rec_err = m;  // NaN propagates
        }
    }
    if (a.mode == 1 && surv) {
        double* o = a.seed_out + p * 6;
        o[0] = l.x; o[1] = l.px; o[2] = l.y; o[3] = l.py; o[4] = l.z; o[5] = l.d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double r = __shfl_xor_sync(0xffffffffu, rec_err, o);
        rec_err = (r > rec_err || isnan(r)) ? r : rec_err;
    }
    if (lane == 0) a.tile_rec[tile] = rec_err;
}

// Loss and gradient of each variant from the tile partials (fixed order).
// out_loss[v]; out_grad over the variants' parameters; out_cnt[v] = survivors.
__global__ void adj_finalize(const AdjVar* var, int32_t nvar, const double* partial, const double* tile_q,
                             const int64_t* tile_cnt, int64_t ntiles, double lost_weight, double* out_loss,
                             double* out_grad, const int32_t* param_off, int64_t* out_surv) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t np_tot = param_off[nvar];
    if (i < np_tot) {
        int lo = 0, hi = nvar - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (param_off[mid] <= i) lo = mid; else hi = mid - 1;
        }
        const AdjVar V = var[lo];
        const int64_t t1 = lo + 1 < nvar ? var[lo + 1].tile0 : ntiles;
        const int j = int(i - param_off[lo]);
        double sg = 0.0;
        int64_t sv = 0;
        for (int64_t t = V.tile0; t < t1; ++t) {
            sg += partial[V.prow + (t - V.tile0) * V.nparams + j];
            sv += tile_cnt[2 * t + 1];
        }
        out_grad[i] = sv > 0 ? sg / double(sv) : 0.0;
    }
    if (i < nvar) {
        const AdjVar V = var[i];
        const int64_t t1 = i + 1 < nvar ? var[i + 1].tile0 : ntiles;
        double q = 0.0;
        int64_t a0 = 0, sv = 0;
        for (int64_t t = V.tile0; t < t1; ++t) {
            q += tile_q[t];
            a0 += tile_cnt[2 * t];
            sv += tile_cnt[2 * t + 1];
        }
        const double frac = a0 > 0 ? double(a0 - sv) / double(a0) : 0.0;
        out_loss[i] = (sv > 0 ? q / double(sv) : 0.0) + lost_weight * frac;
        out_surv[i] = sv;
    }
}

// Jacobian mode: orbit i's tangent map from the six seeded copies, and
// ||M^T J M - J||_max with J = diag(J2, J2, -J2) (z is conjugate to delta
// with the sign of -c*dt in the reference's coordinates).
__global__ void jac_assemble(const double* seed_out, const int64_t* lost, int64_t n, double* jac, double* sympl) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double M[36];
    bool bad = false;
    for (int r = 0; r < 6; ++r) {
        bad = bad || lost[6 * i + r] == 1;
        for (int c = 0; c < 6; ++c) M[c * 6 + r] = seed_out[(6 * i + r) * 6 + c];  // row r = seed r
    }
    const double nanv = CUDART_NAN;
    for (int k = 0; k < 36; ++k) jac[i * 36 + k] = bad ? nanv : M[k];
    if (sympl) {
        double err = 0.0;
        const double sg[3] = {1.0, 1.0, -1.0};
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                // (M^T J M)[r, c] = sum_b sg_b (M[2b, r] M[2b+1, c] - M[2b+1, r] M[2b, c])
                double acc = 0.0;
                for (int b = 0; b < 3; ++b)
                    acc += sg[b] * (M[r * 6 + 2 * b] * M[c * 6 + 2 * b + 1] - M[r * 6 + 2 * b + 1] * M[c * 6 + 2 * b]);
                double jv = 0.0;
                if ((r >> 1) == (c >> 1) && r != c) jv = (r & 1) ? -sg[r >> 1] : sg[r >> 1];
                err = fmax(err, fabs(acc - jv));
            }
        sympl[i] = bad ? nanv : err;
    }
}

__global__ void replicate6(const double* orbits, int64_t n, double* out) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t N6 = 6 * n;
    if (k >= N6) return;
    const int64_t i = k / 6;
    for (int c = 0; c < 6; ++c) out[c * N6 + k] = orbits[c * n + i];
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int fail(int st, const std::string& m) {
    set_last_error(m);
    return st;
}
int cuda_fail(cudaError_t e, const char* where) {
    return fail(TP_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define ADJ_CUDA(call)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

// Scratch slots of the context used here.
enum Slot { S_TABLE = 0, S_INFO, S_SCHED, S_VAR, S_COORDS0, S_LOST0, S_FIN, S_LOST, S_CKPT, S_PARTIAL, S_TILES, S_OUT,
            S_MIS };

struct HostPlan {
    std::vector<double> table;
    std::vector<int32_t> einfo;
    std::vector<double> sched;
    std::vector<AdjVar> var;
    std::vector<MisalignDev> mis;
    std::vector<double> misinv;
    std::vector<int32_t> param_off;
    int64_t ntot = 0, ntiles = 0, prow_words = 0;
    bool rare = false;  // kinds outside the integrator core or misalignment rows: the full kernels
};

double adjoint_stats_time(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

thread_local tp_adjoint_stats g_adj_stats{};
thread_local int64_t g_last_alive = 0;  // particles alive at the start of the last call

// Inverse of a column-major 6x6 matrix by Gauss-Jordan elimination with
// partial pivoting in long double.  Returns false for a singular matrix.
bool invert6(const double* R, double* out) {
    long double a[6][12];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            a[i][j] = R[j * 6 + i];
            a[i][6 + j] = i == j ? 1.0L : 0.0L;
        }
    long double scale = 0.0L;
    for (int k = 0; k < 36; ++k) scale = std::max(scale, std::fabs((long double)R[k]));
    if (!(scale > 0.0L)) return false;
    for (int c = 0; c < 6; ++c) {
        int piv = c;
        for (int r = c + 1; r < 6; ++r)
            if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
        if (!(std::fabs(a[piv][c]) > 1e-14L * scale)) return false;
        if (piv != c)
            for (int j = 0; j < 12; ++j) std::swap(a[c][j], a[piv][j]);
        const long double p = a[c][c];
        for (int j = 0; j < 12; ++j) a[c][j] /= p;
        for (int r = 0; r < 6; ++r) {
            if (r == c || a[r][c] == 0.0L) continue;
            const long double f = a[r][c];
            for (int j = 0; j < 12; ++j) a[r][j] -= f * a[c][j];
        }
    }
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) out[j * 6 + i] = double(a[i][6 + j]);
    return true;
}

// Shift the misalignment row index of every misaligned record in `words`
// words of records (the rows of several variants are concatenated).
void rebase_misalign(double* recs, size_t words, int32_t mbase) {
    for (size_t w = 0; w < words;) {
        RecHdr h;
        std::memcpy(&h, recs + w, sizeof h);
        if (h.words == 0) break;  // padding word
        if (h.flags & RF_MISALIGN) {
            h.aux += mbase;
            std::memcpy(recs + w, &h, sizeof h);
        }
        w += h.words;
    }
}

// Build the concatenated device description of `lats`.  params: element
// indices per variant (param_off[v]..param_off[v+1]), or none (Jacobian).
int make_plan(const std::vector<const tp_lattice*>& lats, const std::vector<int64_t>& npart,
              const std::vector<double>& betis, const int32_t* params, const std::vector<int32_t>& poff_params,
              int32_t turn0, int32_t nturns, HostPlan* P) {
    const int nvar = int(lats.size());
    P->var.resize(size_t(nvar));
    P->param_off = poff_params;
    int64_t tile = 0, prow = 0, p = 0, eoff = 0;
    for (int v = 0; v < nvar; ++v) {
        LatticeHost L;
        lattice_host(lats[size_t(v)], &L);
        const int32_t mbase = int32_t(P->mis.size());
        for (int64_t k = 0; k < L.nmis; ++k) {
            const tp_misalign& m = L.mis[k];
            MisalignDev o{};
            std::memcpy(o.t1, m.t1, sizeof o.t1); std::memcpy(o.t2, m.t2, sizeof o.t2);
            std::memcpy(o.r1, m.r1, sizeof o.r1); std::memcpy(o.r2, m.r2, sizeof o.r2);
            for (int q = 0; q < 36; ++q) { o.r1nz |= m.r1[q] != 0.0; o.r2nz |= m.r2[q] != 0.0; }
            double inv[72] = {};
            if ((o.r1nz && !invert6(m.r1, inv)) || (o.r2nz && !invert6(m.r2, inv + 36)))
                return fail(TP_EUNSUPPORTED, "misalignment row " + std::to_string(k) +
                                                 " has a singular rotation matrix (no inverse map)");
            P->mis.push_back(o);
            P->misinv.insert(P->misinv.end(), inv, inv + 72);
        }
        if (L.has_schedule && (int64_t(turn0) < L.sched_turn0 ||
                               int64_t(turn0) + nturns > int64_t(L.sched_turn0) + L.sched_nturns))
            return fail(TP_ERANGE, "turns outside the lattice schedule");
        // every record (and every scheduled record) must have a reverse map
        auto check = [&](const double* prog, size_t words) -> bool {
            size_t w = 0;
            while (w < words) {
                RecHdr h;
                std::memcpy(&h, prog + w, sizeof h);
                if (h.words == 0) break;  // padding word
                if (!(h.flags & RF_SCHEDULED) && !reverse_supported(h.kind)) return false;
                w += h.words;
            }
            return true;
        };
        for (int32_t e = 0; e < L.nelem; ++e) {
            RecHdr h;
            std::memcpy(&h, L.program + L.rec_off[e], sizeof h);
            if (!(h.flags & RF_SCHEDULED) && !reverse_supported(h.kind))
                return fail(TP_EUNSUPPORTED, "element " + std::to_string(e) + " (kind " +
                                                 std::to_string(L.elems[e].kind) + ") has no reverse map yet");
        }
        if (L.has_schedule && !check(L.sched, L.sched_words))
            return fail(TP_EUNSUPPORTED, "a scheduled element has no reverse map yet");
        if (L.nmis > 0 || records_have_rare(L.program, L.words)) P->rare = true;
        AdjVar& V = P->var[size_t(v)];
        V.toff = int64_t(P->table.size());
        P->table.insert(P->table.end(), L.program, L.program + L.words);
        if (mbase > 0) rebase_misalign(P->table.data() + V.toff, L.words, mbase);
        while (P->table.size() % 2) P->table.push_back(0.0);
        V.eoff = eoff;
        std::vector<int32_t> code(size_t(L.nelem), -1);
        const int32_t np = params ? poff_params[size_t(v) + 1] - poff_params[size_t(v)] : 0;
        for (int32_t j = 0; j < np; ++j) {
            const int32_t e = params[poff_params[size_t(v)] + j];
            if (e < 0 || e >= L.nelem) return fail(TP_EINVAL, "parameter element index out of range");
            if (code[size_t(e)] >= 0) return fail(TP_EINVAL, "parameter element listed twice");
            const int k = L.elems[e].kind;
            const int pm = k == TP_QUADRUPOLE ? 1 : (k == TP_SEXTUPOLE ? 2 : (k == TP_OCTUPOLE ? 3 : 0));
            if (pm == 0)
                return fail(TP_EINVAL, "parameter element " + std::to_string(e) +
                                           " is not a Quadrupole, Sextupole or Octupole");
            code[size_t(e)] = j * 4 + pm;
        }
        for (int32_t e = 0; e < L.nelem; ++e) {
            P->einfo.push_back(L.rec_off[e]);
            P->einfo.push_back(code[size_t(e)]);
        }
        eoff += L.nelem;
        V.soff = -1;
        if (L.has_schedule) {
            V.soff = int64_t(P->sched.size());
            P->sched.insert(P->sched.end(), L.sched, L.sched + L.sched_words);
            if (mbase > 0) rebase_misalign(P->sched.data() + V.soff, L.sched_words, mbase);
        }
        V.sstride = L.sched_stride;
        V.sturn0 = L.sched_turn0;
        V.snturns = L.sched_nturns;
        V.nelem = L.nelem;
        V.nparams = np;
        V.beti = betis[size_t(v)];
        V.p0 = p;
        p += npart[size_t(v)];
        V.p1 = p;
        V.tile0 = tile;
        const int64_t nt = (npart[size_t(v)] + kTile - 1) / kTile;
        tile += nt;
        V.prow = prow;
        prow += nt * np;
        V.pad = 0;
    }
    P->ntot = p;
    P->ntiles = tile;
    P->prow_words = prow;
    return TP_OK;
}

// Choose K: the smallest interval whose checkpoints fit the budget (a quarter
// of the free device memory, at most 16 GiB).
int32_t auto_interval(int64_t ntot, int32_t nturns) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        fr = size_t(8) << 30;
    }
    const double budget = std::min<double>(double(fr) / 4.0, double(size_t(16) << 30));
    const double per = 48.0 * double(std::max<int64_t>(ntot, 1));
    for (int32_t K = 1; K < nturns; ++K) {
        const int64_t nseg = (nturns + K - 1) / K;
        if (double(nseg - 1) * per <= budget) return K;
    }
    return std::max(nturns, 1);
}

// Time-based choice of K (checkpoint_every = 0).  The reverse sweep rebuilds
// each segment with the maps' exact time-reversed forms, so K trades
// checkpoint memory and traffic against reconstruction drift, not compute.
// The first gradient calls of a configuration (particles, turns, variants,
// table, parameters, drift) each run one candidate K in {1, 2, 4, 8} whose
// checkpoints fit the memory budget, timed on the caller's own work (forward +
// reverse device time); later calls keep the fastest candidate whose
// reconstruction error stayed within kRecTol (else the smallest K).
constexpr double kRecTol = 1e-10;
struct KTune {
    uint64_t key = 0;
    int32_t cand[4] = {};
    float ms[4] = {};
    double rec[4] = {};
    int ncand = 0, ntried = 0;
    int32_t best = 1;
    float best_ms = 0.f;
};
std::mutex g_ktune_mu;
// Per device, the tuning state of each configuration seen (a few dozen at most
// in practice; the table is cleared when it grows past 256 entries).
std::unordered_map<uint64_t, KTune> g_ktune[16];

KTune& ktune_of(int device, uint64_t key) {
    auto& m = g_ktune[device & 15];
    if (m.size() > 256 && m.find(key) == m.end()) m.clear();
    return m[key];
}

uint64_t ktune_key(std::initializer_list<int64_t> parts) {
    uint64_t h = 1469598103934665603ull;
    for (int64_t v : parts)
        for (int k = 0; k < 8; ++k) {
            h ^= uint64_t(v >> (8 * k)) & 0xffu;
            h *= 1099511628211ull;
        }
    return h | 1ull;
}

// K for this call and whether it is a timing trial (*state: 1 trial, 2 settled).
int32_t ktune_pick(int device, uint64_t key, int64_t ntot, int32_t nturns, int* state) {
    std::lock_guard<std::mutex> g(g_ktune_mu);
    KTune& t = ktune_of(device, key);
    if (t.key != key) {
        t = KTune{};
        t.key = key;
        const int32_t kmin = auto_interval(ntot, nturns);  // smallest K that fits the budget
        for (int32_t K : {1, 2, 4, 8})
            if (K >= kmin && K <= std::max(nturns, 1) && t.ncand < 4) t.cand[t.ncand++] = K;
        if (t.ncand == 0) t.cand[t.ncand++] = kmin;
        t.best = t.cand[0];
    }
    if (t.ntried < t.ncand) {
        *state = 1;
        return t.cand[t.ntried];
    }
    *state = 2;
    return t.best;
}

void ktune_record(int device, uint64_t key, int32_t K, float ms, double rec) {
    std::lock_guard<std::mutex> g(g_ktune_mu);
    KTune& t = ktune_of(device, key);
    if (t.key != key || t.ntried >= t.ncand || t.cand[t.ntried] != K) return;
    t.ms[t.ntried] = ms;
    t.rec[t.ntried] = rec;
    if (++t.ntried == t.ncand) {
        int bi = -1;
        for (int k = 0; k < t.ncand; ++k)
            if (t.rec[k] <= kRecTol && (bi < 0 || t.ms[k] < t.ms[bi])) bi = k;
        if (bi < 0) bi = 0;
        t.best = t.cand[bi];
        t.best_ms = t.ms[bi];
    }
}

float ktune_best_ms(int device, uint64_t key) {
    std::lock_guard<std::mutex> g(g_ktune_mu);
    const KTune& t = ktune_of(device, key);
    return t.key == key ? t.best_ms : 0.f;
}

// The shared driver.  coords0/lost0 are device pointers here.
int run_adjoint(tp_ctx* c, const std::vector<const tp_lattice*>& lats, const std::vector<int64_t>& npart,
                const std::vector<double>& betis, const double* d_coords0, const int64_t* d_lost0, int32_t nturns,
                int32_t turn0, const int32_t* params, const std::vector<int32_t>& poff_params, int mode,
                double sigma, double lost_weight, int32_t K, double limx, double limy, bool exact, cudaStream_t s,
                double* h_loss, double* h_grad, double* d_fin_out, int64_t* d_lost_out, double* d_seed_out,
                int64_t* h_surv, float* ms_fwd, float* ms_rev, double* rec_err, double* units, bool table_smem) {
    HostPlan P;
    int st = make_plan(lats, npart, betis, params, poff_params, turn0, nturns, &P);
    if (st != TP_OK) return st;
    const int nvar = int(lats.size());
    CtxHost ch0;
    ctx_host(c, &ch0);
    int kstate = 0;  // 0: K fixed by the caller (or a loss-only call); 1: tuning trial; 2: tuned
    uint64_t kkey = 0;
    if (K <= 0 && mode == 0) {
        kkey = ktune_key({P.ntot, nturns, nvar, int64_t(P.table.size()), int64_t(P.param_off.back()), int64_t(exact),
                          int64_t(P.sched.size()), int64_t(P.mis.size())});
        K = ktune_pick(ch0.device, kkey, P.ntot, nturns, &kstate);
    } else if (K <= 0) {
        K = auto_interval(P.ntot, nturns);
    }
    K = std::max(1, std::min(K, std::max(nturns, 1)));
    const int32_t nseg = nturns > 0 ? (nturns + K - 1) / K : 1;
    CtxHost ch;
    ctx_host(c, &ch);

    void *d_table, *d_info, *d_sched, *d_var, *d_fin, *d_lost, *d_ckpt, *d_partial, *d_tiles, *d_out;
    const size_t tb = std::max<size_t>(P.table.size(), 2) * 8;
    if ((st = ctx_scratch(c, S_TABLE, tb, &d_table)) ||
        (st = ctx_scratch(c, S_INFO, std::max<size_t>(P.einfo.size(), 2) * 4, &d_info)) ||
        (st = ctx_scratch(c, S_SCHED, std::max<size_t>(P.sched.size(), 2) * 8, &d_sched)) ||
        (st = ctx_scratch(c, S_VAR, P.var.size() * sizeof(AdjVar) + (nvar + 1) * 4 + 64, &d_var)) ||
        (st = ctx_scratch(c, S_FIN, size_t(P.ntot) * 48, &d_fin)) ||
        (st = ctx_scratch(c, S_LOST, size_t(P.ntot) * 8, &d_lost)) ||
        (st = ctx_scratch(c, S_CKPT, size_t(std::max(nseg - 1, 1)) * size_t(P.ntot) * 48, &d_ckpt)) ||
        (st = ctx_scratch(c, S_PARTIAL, size_t(std::max<int64_t>(P.prow_words, 1)) * 8, &d_partial)) ||
        (st = ctx_scratch(c, S_TILES, size_t(P.ntiles) * 32 + 64, &d_tiles)) ||
        (st = ctx_scratch(c, S_OUT, (size_t(nvar) * 2 + size_t(P.param_off.back()) + 8) * 8, &d_out)))
        return st;
    void* d_mis = nullptr;
    const size_t mis_bytes = P.mis.size() * sizeof(MisalignDev);
    if (!P.mis.empty()) {
        if ((st = ctx_scratch(c, S_MIS, mis_bytes + P.misinv.size() * 8, &d_mis))) return st;
        ADJ_CUDA(cudaMemcpyAsync(d_mis, P.mis.data(), mis_bytes, cudaMemcpyHostToDevice, s));
        ADJ_CUDA(cudaMemcpyAsync(static_cast<char*>(d_mis) + mis_bytes, P.misinv.data(), P.misinv.size() * 8,
                                 cudaMemcpyHostToDevice, s));
    }
    ADJ_CUDA(cudaMemcpyAsync(d_table, P.table.data(), P.table.size() * 8, cudaMemcpyHostToDevice, s));
    ADJ_CUDA(cudaMemcpyAsync(d_info, P.einfo.data(), P.einfo.size() * 4, cudaMemcpyHostToDevice, s));
    if (!P.sched.empty())
        ADJ_CUDA(cudaMemcpyAsync(d_sched, P.sched.data(), P.sched.size() * 8, cudaMemcpyHostToDevice, s));
    ADJ_CUDA(cudaMemcpyAsync(d_var, P.var.data(), P.var.size() * sizeof(AdjVar), cudaMemcpyHostToDevice, s));
    int32_t* d_poff = reinterpret_cast<int32_t*>(static_cast<char*>(d_var) + P.var.size() * sizeof(AdjVar));
    ADJ_CUDA(cudaMemcpyAsync(d_poff, P.param_off.data(), P.param_off.size() * 4, cudaMemcpyHostToDevice, s));
    if (P.prow_words > 0) ADJ_CUDA(cudaMemsetAsync(d_partial, 0, size_t(P.prow_words) * 8, s));
    int32_t* d_err = reinterpret_cast<int32_t*>(static_cast<char*>(d_tiles) + size_t(P.ntiles) * 32);
    ADJ_CUDA(cudaMemsetAsync(d_err, 0, 16, s));

    AdjArgs a{};
    a.table = static_cast<const double*>(d_table);
    a.einfo = static_cast<const int32_t*>(d_info);
    a.sched = static_cast<const double*>(d_sched);
    a.var = static_cast<const AdjVar*>(d_var);
    a.mis = static_cast<const MisalignDev*>(d_mis);
    a.misinv = d_mis ? reinterpret_cast<const double*>(static_cast<char*>(d_mis) + mis_bytes) : nullptr;
    a.nvar = nvar;
    a.nturns = nturns;
    a.turn0 = turn0;
    a.K = K;
    a.nseg = nseg;
    a.mode = mode;
    a.ntot = P.ntot;
    a.ntiles = P.ntiles;
    a.coords0 = d_coords0;
    a.lost0 = d_lost0;
    a.fin = d_fin_out ? d_fin_out : static_cast<double*>(d_fin);
    a.lost = d_lost_out ? d_lost_out : static_cast<int64_t*>(d_lost);
    a.ckpt = static_cast<double*>(d_ckpt);
    a.limx = limx;
    a.limy = limy;
    a.inv_sigma2 = mode == 0 ? 1.0 / (sigma * sigma) : 0.0;
    a.partial = static_cast<double*>(d_partial);
    a.tile_q = static_cast<double*>(d_tiles);
    a.tile_cnt = reinterpret_cast<int64_t*>(static_cast<char*>(d_tiles) + size_t(P.ntiles) * 8);
    a.tile_rec = reinterpret_cast<double*>(static_cast<char*>(d_tiles) + size_t(P.ntiles) * 24);
    a.seed_out = d_seed_out;
    a.err = d_err;
    // one variant: its table and element info in shared memory
    const size_t info_words = nvar == 1 ? size_t(P.var[0].nelem) : 0;  // 2 int32 per element = 1 word
    const size_t smem_bytes = (P.table.size() + info_words) * 8;
    a.smem_words = 0;
    size_t smem = 0;
    if (table_smem && nvar == 1 && smem_bytes + 1024 <= ch.smem_optin) {
        a.smem_words = int32_t(P.table.size() + info_words);
        smem = smem_bytes;
    }
    const int grid = int((P.ntiles + kAdjBlock / 32 - 1) / (kAdjBlock / 32));
    cudaEvent_t e0, e1, e2;
    ADJ_CUDA(cudaEventCreate(&e0));
    ADJ_CUDA(cudaEventCreate(&e1));
    ADJ_CUDA(cudaEventCreate(&e2));
    auto cleanup = [&]() { cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); };
    const bool rare = P.rare;
    auto set_smem = [&](auto fwd, auto rev) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        return e == cudaSuccess ? cudaFuncSetAttribute(rev, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) : e;
    };
    if (smem > 48 * 1024) {
        cudaError_t e = exact ? (rare ? set_smem(adj_forward<true, true>, adj_reverse<true, true>)
                                      : set_smem(adj_forward<true, false>, adj_reverse<true, false>))
                              : (rare ? set_smem(adj_forward<false, true>, adj_reverse<false, true>)
                                      : set_smem(adj_forward<false, false>, adj_reverse<false, false>));
        if (e != cudaSuccess) { cleanup(); return cuda_fail(e, "cudaFuncSetAttribute"); }
    }
    cudaEventRecord(e0, s);
    if (grid > 0) {
        if (exact && rare) adj_forward<true, true><<<grid, kAdjBlock, smem, s>>>(a);
        else if (exact) adj_forward<true, false><<<grid, kAdjBlock, smem, s>>>(a);
        else if (rare) adj_forward<false, true><<<grid, kAdjBlock, smem, s>>>(a);
        else adj_forward<false, false><<<grid, kAdjBlock, smem, s>>>(a);
    }
    cudaEventRecord(e1, s);
    if (grid > 0) {
        if (exact && rare) adj_reverse<true, true><<<grid, kAdjBlock, smem, s>>>(a);
        else if (exact) adj_reverse<true, false><<<grid, kAdjBlock, smem, s>>>(a);
        else if (rare) adj_reverse<false, true><<<grid, kAdjBlock, smem, s>>>(a);
        else adj_reverse<false, false><<<grid, kAdjBlock, smem, s>>>(a);
    }
    cudaEventRecord(e2, s);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) { cleanup(); return cuda_fail(le, "adjoint kernel launch"); }
    double* d_loss = static_cast<double*>(d_out);
    int64_t* d_surv = reinterpret_cast<int64_t*>(d_loss + nvar);
    double* d_grad = d_loss + 2 * nvar;
    const int64_t nfin = std::max<int64_t>(P.param_off.back(), nvar);
    if (mode == 0 && nvar > 0) {
        adj_finalize<<<int((nfin + 127) / 128), 128, 0, s>>>(a.var, nvar, a.partial, a.tile_q, a.tile_cnt, P.ntiles,
                                                            lost_weight, d_loss, d_grad, d_poff, d_surv);
        le = cudaGetLastError();
        if (le != cudaSuccess) { cleanup(); return cuda_fail(le, "adjoint finalize launch"); }
    }
    std::vector<double> recs(size_t(P.ntiles));
    std::vector<int64_t> cnts(size_t(2 * P.ntiles));
    int32_t derr = 0;
    cudaError_t ce = cudaSuccess;
    if (P.ntiles > 0) ce = cudaMemcpyAsync(recs.data(), a.tile_rec, size_t(P.ntiles) * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && P.ntiles > 0)
        ce = cudaMemcpyAsync(cnts.data(), a.tile_cnt, size_t(P.ntiles) * 16, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&derr, d_err, 4, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && mode == 0 && h_loss)
        ce = cudaMemcpyAsync(h_loss, d_loss, size_t(nvar) * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && mode == 0 && h_surv)
        ce = cudaMemcpyAsync(h_surv, d_surv, size_t(nvar) * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess && mode == 0 && h_grad && P.param_off.back() > 0)
        ce = cudaMemcpyAsync(h_grad, d_grad, size_t(P.param_off.back()) * 8, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) { cleanup(); return cuda_fail(ce, "adjoint"); }
    cudaEventElapsedTime(ms_fwd, e0, e1);
    cudaEventElapsedTime(ms_rev, e1, e2);
    cleanup();
    if (derr & DE_BAD_KIND) return fail(TP_EUNSUPPORTED, "kernel met an element record without a reverse map");
    if (derr & DE_SCHED_RANGE) return fail(TP_ERANGE, "turn outside the lattice schedule");
    if (derr) return fail(TP_EDEVICE, "device error word set");
    double m = 0.0;
    for (double r : recs) m = (r > m || std::isnan(r)) ? r : m;
    *rec_err = m;
    // particle*element*turns of the forward pass (alive at start x elements x turns)
    double u = 0.0;
    g_last_alive = 0;
    for (int v = 0; v < nvar; ++v) {
        const int64_t t1 = v + 1 < nvar ? P.var[size_t(v) + 1].tile0 : P.ntiles;
        int64_t a0 = 0;
        for (int64_t t = P.var[size_t(v)].tile0; t < t1; ++t) a0 += cnts[size_t(2 * t)];
        u += double(a0) * double(P.var[size_t(v)].nelem) * double(nturns);
        g_last_alive += a0;
    }
    *units = u;
    g_adj_stats.checkpoint_every = K;
    g_adj_stats.segments = nseg;
    g_adj_stats.checkpoint_bytes = int64_t(std::max(nseg - 1, 0)) * P.ntot * 48;
    g_adj_stats.forward_ms = *ms_fwd;
    g_adj_stats.reverse_ms = *ms_rev;
    g_adj_stats.reconstruction_error = m;
    g_adj_stats.particles = P.ntot;
    g_adj_stats.launches = 2 + (mode == 0 ? 1 : 0);
    g_adj_stats.units = u;
    if (kstate == 1) ktune_record(ch0.device, kkey, K, *ms_fwd + *ms_rev, m);
    g_adj_stats.k_tuning = kstate;
    g_adj_stats.tuned_ms = kstate ? ktune_best_ms(ch0.device, kkey) : 0.0;
    return TP_OK;
}

tp_opts opts_of(const tp_opts* o) {
    tp_opts r{};
    r.size = sizeof(tp_opts);
    r.exact_hamiltonian = 1;
    if (o && o->size > 0) std::memcpy(&r, o, std::min<size_t>(size_t(o->size), sizeof(tp_opts)));
    return r;
}

double limit_of(double ap) { return ap > 0.0 ? std::min(1.0, ap) : 1.0; }

// Stage host arrays (or take device arrays) of n particles.
int stage_inputs(tp_ctx* c, bool dev, const double* coords0, const int64_t* lost0, int64_t n, cudaStream_t s,
                 const double** d_c, const int64_t** d_l, int64_t* h2d) {
    if (dev) {
        *d_c = coords0;
        *d_l = lost0;
        return TP_OK;
    }
    void *pc, *pl;
    int st;
    if ((st = ctx_scratch(c, S_COORDS0, size_t(n) * 48, &pc)) || (st = ctx_scratch(c, S_LOST0, size_t(n) * 8, &pl)))
        return st;
    ADJ_CUDA(cudaMemcpyAsync(pc, coords0, size_t(n) * 48, cudaMemcpyHostToDevice, s));
    *h2d += n * 48;
    if (lost0) {
        ADJ_CUDA(cudaMemcpyAsync(pl, lost0, size_t(n) * 8, cudaMemcpyHostToDevice, s));
        *h2d += n * 8;
        *d_l = static_cast<const int64_t*>(pl);
    } else {
        *d_l = nullptr;
    }
    *d_c = static_cast<const double*>(pc);
    return TP_OK;
}

}  // namespace
}  // namespace tp

using namespace tp;

extern "C" {

TP_API int tp_ringpass_adjoint(tp_ctx* ctx, const tp_lattice* lat, const double* coords0, int64_t n,
                               const int64_t* lost0, double beti, int32_t nturns, double time, double dt_turn,
                               int32_t turn0, const int32_t* param_elems, int32_t nparams, const tp_loss_spec* loss,
                               int32_t checkpoint_every, double* loss_out, double* grad_out, double* coords_out,
                               int64_t* lost_out, const tp_opts* opts) {
    tp::NvtxRange nvtx_range("tp_ringpass_adjoint");
    (void)time;
    (void)dt_turn;
    auto t0 = std::chrono::steady_clock::now();
    if (!ctx || !lat || !loss) return fail(TP_EINVAL, "null context, lattice or loss");
    if (n < 0 || nturns < 0 || nparams < 0) return fail(TP_EINVAL, "negative size");
    if (n > 0 && !coords0) return fail(TP_EINVAL, "coords0 is required");
    if (nparams > 0 && (!param_elems || !grad_out)) return fail(TP_EINVAL, "param_elems and grad_out are required");
    if (!loss_out) return fail(TP_EINVAL, "loss_out is required");
    if (loss->kind != TP_LOSS_BEAM_SIZE) return fail(TP_EUNSUPPORTED, "unknown loss kind");
    if (!(loss->sigma > 0.0) || !std::isfinite(loss->sigma)) return fail(TP_EINVAL, "sigma must be positive");
    if (!(beti > 0.0) || !std::isfinite(beti)) return fail(TP_EINVAL, "beti must be finite and positive");
    if (n > (int64_t(1) << 34)) return fail(TP_ERANGE, "particle count beyond 2^34");
    tp_opts o = opts_of(opts);
    CtxHost ch;
    ctx_host(ctx, &ch);
    ADJ_CUDA(cudaSetDevice(ch.device));
    cudaStream_t s = static_cast<cudaStream_t>(o.stream ? o.stream : ch.stream);
    const bool dev = o.device_pointers != 0;
    int64_t h2d = 0, d2h = 0;
    const double* d_c = nullptr;
    const int64_t* d_l = nullptr;
    int st = stage_inputs(ctx, dev, coords0, lost0, n, s, &d_c, &d_l, &h2d);
    if (st != TP_OK) return st;
    std::vector<const tp_lattice*> lats{lat};
    std::vector<int32_t> poff{0, nparams};
    double* d_fin = dev ? coords_out : nullptr;
    int64_t* d_lost = dev ? lost_out : nullptr;
    int64_t surv = 0;
    float msf = 0.f, msr = 0.f;
    double rec = 0.0, units = 0.0;
    std::vector<double> grad(size_t(std::max(nparams, 1)));
    st = run_adjoint(ctx, lats, {n}, {beti}, d_c, d_l, nturns, turn0, param_elems, poff, 0, loss->sigma,
                     loss->lost_weight, checkpoint_every, limit_of(o.aperture_x), limit_of(o.aperture_y),
                     o.exact_hamiltonian != 0, s, loss_out, grad.data(), d_fin, d_lost, nullptr, &surv, &msf, &msr,
                     &rec, &units, o.table_in_smem != 0);
    if (st != TP_OK) return st;
    if (nparams > 0) std::memcpy(grad_out, grad.data(), size_t(nparams) * 8);
    if (!dev && (coords_out || lost_out)) {
        void *pf, *pl;
        if ((st = ctx_scratch(ctx, S_FIN, size_t(n) * 48, &pf)) || (st = ctx_scratch(ctx, S_LOST, size_t(n) * 8, &pl)))
            return st;
        if (coords_out) {
            ADJ_CUDA(cudaMemcpyAsync(coords_out, pf, size_t(n) * 48, cudaMemcpyDeviceToHost, s));
            d2h += n * 48;
        }
        if (lost_out) {
            ADJ_CUDA(cudaMemcpyAsync(lost_out, pl, size_t(n) * 8, cudaMemcpyDeviceToHost, s));
            d2h += n * 8;
        }
        ADJ_CUDA(cudaStreamSynchronize(s));
    }
    tp_stats& S = *ctx_stats(ctx);
    S = tp_stats{};
    S.particles = g_last_alive;
    S.survivors = surv;
    S.units = units;
    S.kernel_ms = double(msf) + double(msr);
    S.total_ms = adjoint_stats_time(t0);
    S.h2d_bytes = h2d;
    S.d2h_bytes = d2h + 8 * (1 + nparams);
    S.block_size = kAdjBlock;
    S.min_blocks = 4;
    S.launches = g_adj_stats.launches;
    S.schedule = 1;
    return TP_OK;
}

TP_API int tp_ringpass_adjoint_batched(tp_ctx* ctx, tp_batch* b, const double* coords0, const int64_t* poff,
                                       const int64_t* lost0, const double* beti, int32_t nturns, double time,
                                       double dt_turn, int32_t turn0, const int32_t* param_elems,
                                       const int32_t* param_off, const tp_loss_spec* loss, int32_t checkpoint_every,
                                       double* loss_out, double* grad_out, const tp_opts* opts) {
    tp::NvtxRange nvtx_range("tp_ringpass_adjoint_batched");
    (void)time;
    (void)dt_turn;
    auto t0 = std::chrono::steady_clock::now();
    if (!ctx || !b || !loss || !poff || !beti || !param_off || !loss_out)
        return fail(TP_EINVAL, "null argument");
    if (nturns < 0) return fail(TP_EINVAL, "negative number of turns");
    if (loss->kind != TP_LOSS_BEAM_SIZE) return fail(TP_EUNSUPPORTED, "unknown loss kind");
    if (!(loss->sigma > 0.0) || !std::isfinite(loss->sigma)) return fail(TP_EINVAL, "sigma must be positive");
    std::vector<const tp_lattice*> lats;
    batch_lattices(b, &lats);
    const int nvar = int(lats.size());
    std::vector<int64_t> np(static_cast<size_t>(nvar));
    std::vector<double> bt(static_cast<size_t>(nvar));
    std::vector<int32_t> pofs(static_cast<size_t>(nvar) + 1);
    if (poff[0] != 0 || param_off[0] != 0) return fail(TP_EINVAL, "poff[0] and param_off[0] must be 0");
    for (int v = 0; v < nvar; ++v) {
        np[size_t(v)] = poff[v + 1] - poff[v];
        if (np[size_t(v)] < 0) return fail(TP_EINVAL, "poff must be non-decreasing");
        if (!(beti[v] > 0.0) || !std::isfinite(beti[v])) return fail(TP_EINVAL, "beti must be finite and positive");
        bt[size_t(v)] = beti[v];
        if (param_off[v + 1] < param_off[v]) return fail(TP_EINVAL, "param_off must be non-decreasing");
        pofs[size_t(v)] = param_off[v];
    }
    pofs[size_t(nvar)] = param_off[nvar];
    if (pofs[size_t(nvar)] > 0 && (!param_elems || !grad_out)) return fail(TP_EINVAL, "param_elems and grad_out are required");
    const int64_t n = poff[nvar];
    if (n > 0 && !coords0) return fail(TP_EINVAL, "coords0 is required");
    tp_opts o = opts_of(opts);
    CtxHost ch;
    ctx_host(ctx, &ch);
    ADJ_CUDA(cudaSetDevice(ch.device));
    cudaStream_t s = static_cast<cudaStream_t>(o.stream ? o.stream : ch.stream);
    const bool dev = o.device_pointers != 0;
    int64_t h2d = 0;
    const double* d_c = nullptr;
    const int64_t* d_l = nullptr;
    int st = stage_inputs(ctx, dev, coords0, lost0, n, s, &d_c, &d_l, &h2d);
    if (st != TP_OK) return st;
    std::vector<int64_t> surv(static_cast<size_t>(nvar));
    float msf = 0.f, msr = 0.f;
    double rec = 0.0, units = 0.0;
    std::vector<double> grad(size_t(std::max<int32_t>(pofs[size_t(nvar)], 1)));
    st = run_adjoint(ctx, lats, np, bt, d_c, d_l, nturns, turn0, param_elems, pofs, 0, loss->sigma,
                     loss->lost_weight, checkpoint_every, limit_of(o.aperture_x), limit_of(o.aperture_y),
                     o.exact_hamiltonian != 0, s, loss_out, grad.data(), nullptr, nullptr, nullptr, surv.data(), &msf,
                     &msr, &rec, &units, o.table_in_smem != 0);
    if (st != TP_OK) return st;
    if (pofs[size_t(nvar)] > 0) std::memcpy(grad_out, grad.data(), size_t(pofs[size_t(nvar)]) * 8);
    tp_stats& S = *ctx_stats(ctx);
    S = tp_stats{};
    S.particles = g_last_alive;
    for (int64_t x : surv) S.survivors += x;
    S.units = units;
    S.kernel_ms = double(msf) + double(msr);
    S.total_ms = adjoint_stats_time(t0);
    S.h2d_bytes = h2d;
    S.d2h_bytes = 8 * (nvar + pofs[size_t(nvar)]);
    S.block_size = kAdjBlock;
    S.min_blocks = 4;
    S.launches = g_adj_stats.launches;
    S.schedule = 1;
    return TP_OK;
}

TP_API int tp_one_turn_jacobian(tp_ctx* ctx, const tp_lattice* lat, const double* orbits, int64_t n, double beti,
                                int32_t nturns, int32_t turn0, double* jac_out, double* sympl_out,
                                const tp_opts* opts) {
    tp::NvtxRange nvtx_range("tp_one_turn_jacobian");
    auto t0 = std::chrono::steady_clock::now();
    if (!ctx || !lat) return fail(TP_EINVAL, "null context or lattice");
    if (n < 0 || nturns < 0) return fail(TP_EINVAL, "negative size");
    if (n > 0 && (!orbits || !jac_out)) return fail(TP_EINVAL, "orbits and jac_out are required");
    if (!(beti > 0.0) || !std::isfinite(beti)) return fail(TP_EINVAL, "beti must be finite and positive");
    if (n > (int64_t(1) << 30)) return fail(TP_ERANGE, "orbit count beyond 2^30");
    if (n == 0) return TP_OK;
    tp_opts o = opts_of(opts);
    CtxHost ch;
    ctx_host(ctx, &ch);
    ADJ_CUDA(cudaSetDevice(ch.device));
    cudaStream_t s = static_cast<cudaStream_t>(o.stream ? o.stream : ch.stream);
    const bool dev = o.device_pointers != 0;
    const int64_t n6 = 6 * n;
    int st;
    void *d_orb = nullptr, *d_rep, *d_seed, *d_jac;
    int64_t h2d = 0, d2h = 0;
    if ((st = ctx_scratch(ctx, S_COORDS0, size_t(n6) * 48, &d_rep)) ||
        (st = ctx_scratch(ctx, S_LOST0, size_t(n6) * 48 + size_t(n) * 37 * 8 + size_t(n) * 48, &d_seed)))
        return st;
    d_jac = static_cast<char*>(d_seed) + size_t(n6) * 48;
    if (dev) {
        d_orb = const_cast<double*>(orbits);
    } else {
        d_orb = static_cast<char*>(d_jac) + size_t(n) * 37 * 8;
        ADJ_CUDA(cudaMemcpyAsync(d_orb, orbits, size_t(n) * 48, cudaMemcpyHostToDevice, s));
        h2d += n * 48;
    }
    replicate6<<<int((n6 + 255) / 256), 256, 0, s>>>(static_cast<const double*>(d_orb), n, static_cast<double*>(d_rep));
    ADJ_CUDA(cudaGetLastError());
    std::vector<const tp_lattice*> lats{lat};
    std::vector<int32_t> poff{0, 0};
    int64_t surv = 0;
    float msf = 0.f, msr = 0.f;
    double rec = 0.0, units = 0.0;
    ADJ_CUDA(cudaMemsetAsync(d_seed, 0, size_t(n6) * 48, s));
    // K = 1: the reverse sweep rebuilds one turn at a time.
    st = run_adjoint(ctx, lats, {n6}, {beti}, static_cast<const double*>(d_rep), nullptr, nturns, turn0, nullptr, poff,
                     1, 1.0, 0.0, 1, 1.0, 1.0, o.exact_hamiltonian != 0, s, nullptr, nullptr, nullptr, nullptr,
                     static_cast<double*>(d_seed), &surv, &msf, &msr, &rec, &units, o.table_in_smem != 0);
    if (st != TP_OK) return st;
    // run_adjoint left the flags in its own scratch slot
    void* d_lost;
    if ((st = ctx_scratch(ctx, S_LOST, size_t(n6) * 8, &d_lost))) return st;
    double* jac_d = dev ? jac_out : static_cast<double*>(d_jac);
    double* sym_d = sympl_out ? (dev ? sympl_out : static_cast<double*>(d_jac) + size_t(n) * 36) : nullptr;
    jac_assemble<<<int((n + 127) / 128), 128, 0, s>>>(static_cast<const double*>(d_seed),
                                                     static_cast<const int64_t*>(d_lost), n, jac_d, sym_d);
    ADJ_CUDA(cudaGetLastError());
    if (!dev) {
        ADJ_CUDA(cudaMemcpyAsync(jac_out, jac_d, size_t(n) * 36 * 8, cudaMemcpyDeviceToHost, s));
        d2h += n * 36 * 8;
        if (sympl_out) {
            ADJ_CUDA(cudaMemcpyAsync(sympl_out, sym_d, size_t(n) * 8, cudaMemcpyDeviceToHost, s));
            d2h += n * 8;
        }
    }
    ADJ_CUDA(cudaStreamSynchronize(s));
    tp_stats& S = *ctx_stats(ctx);
    S = tp_stats{};
    S.particles = n;
    S.survivors = surv;
    S.kernel_ms = double(msf) + double(msr);
    S.total_ms = adjoint_stats_time(t0);
    S.h2d_bytes = h2d;
    S.d2h_bytes = d2h;
    S.block_size = kAdjBlock;
    S.min_blocks = 4;
    S.launches = 2 + 2;
    S.schedule = 1;
    return TP_OK;
}

TP_API int tp_last_adjoint_stats(tp_adjoint_stats* out) {
    if (!out) return fail(TP_EINVAL, "null argument");
    *out = g_adj_stats;
    return TP_OK;
}

}  // extern "C"

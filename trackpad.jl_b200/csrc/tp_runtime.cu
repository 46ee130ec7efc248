// tp_runtime.cu -- the C ABI (include/trackpad_b200.h): contexts, lattices,
// schedules, batches, launch configuration and statistics.
//
// Ownership follows the reference's linepass!/ringpass!: the caller owns the
// coordinate and flag arrays and the call mutates them in place.  Host arrays
// are staged through per-context device buffers; device arrays are used in
// place.  Every entry point returns a status and never throws.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "tp_internal.h"

using namespace tp;

namespace {

thread_local std::string g_last_error;

int set_err(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

int cuda_err(cudaError_t e, const char* where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return TP_ECUDA;
}

#define TP_CUDA(call)                                       \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_err(e_, #call);  \
    } while (0)

constexpr int kMaxDevices = 16;

// Online choice of the launch configuration: the particle scheduling (1 =
// static, 2 = lane refill) and the kernel instance whose registers are sized
// for 7, 8, 6 or 5 resident blocks per SM.  Every configuration gives
// bit-identical results, so the first calls of a configuration key (sizes,
// turns, drift, build, lattice version) each run one candidate on the caller's
// own work, timed with the call's CUDA events: first the two schedules at 7
// resident blocks, then 8, 6 and 5 with the faster schedule (batched pooled
// refill: then folds 2 and 4).  Later calls keep the
// fastest candidate.  What the caller fixes in tp_opts is not tuned.
struct LaunchCand {
    int sched = 1, minb = 7;
    int fold = 1;  // batched pooled refill: warps per variant = tiles / fold (more refills per warp)
};

struct LaunchTune {
    uint64_t key = 0;
    LaunchCand cand[8];
    float ms[8] = {};
    int ncand = 0, ntried = 0;
    int stage = 0;       // 0: schedules, 1: resident blocks, 2: batched refill folds, 3: settled
    LaunchCand best;
};

uint64_t tune_key(std::initializer_list<int64_t> parts) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the parts
    for (int64_t v : parts) {
        for (int k = 0; k < 8; ++k) {
            h ^= uint64_t(v >> (8 * k)) & 0xffu;
            h *= 1099511628211ull;
        }
    }
    return h | 1ull;
}

int tune_argmin(const LaunchTune& t) {
    int bi = 0;
    for (int k = 1; k < t.ntried; ++k)
        if (t.ms[k] < t.ms[bi]) bi = k;
    return bi;
}

// The candidate for this call.  fixed_sched / fixed_minb: the caller's choice
// (0: tuned).  minbs[0..nminb): the resident-block counts the kernel build
// carries, the default first.  folds: whether batched refill folds are tried.
// *trial is set when the call is a timing trial.
LaunchCand tune_pick(LaunchTune& t, uint64_t key, int fixed_sched, int fixed_minb, const int* minbs, int nminb,
                     bool folds, bool* trial) {
    if (t.key != key) {
        t = LaunchTune{};
        t.key = key;
        const int m0 = fixed_minb ? fixed_minb : minbs[0];
        if (fixed_sched) {
            t.cand[t.ncand++] = {fixed_sched, m0, 1};
        } else {
            t.cand[t.ncand++] = {1, m0, 1};
            t.cand[t.ncand++] = {2, m0, 1};
        }
    }
    while (t.ntried == t.ncand && t.stage < 3) {
        const LaunchCand b = t.cand[tune_argmin(t)];
        if (t.stage == 0 && !fixed_minb && nminb > 1) {
            for (int k = 1; k < nminb && t.ncand < 8; ++k) t.cand[t.ncand++] = {b.sched, minbs[k], 1};
            t.stage = 1;
        } else if (t.stage <= 1 && folds && b.sched == 2) {
            for (int f : {2, 4})
                if (t.ncand < 8) t.cand[t.ncand++] = {2, b.minb, f};
            t.stage = 2;
        } else {
            t.best = b;
            t.stage = 3;
        }
    }
    if (t.ntried < t.ncand) {
        *trial = true;
        return t.cand[t.ntried];
    }
    *trial = false;
    return t.best;
}

void tune_record(LaunchTune& t, uint64_t key, LaunchCand c, float ms) {
    if (t.key != key || t.ntried >= t.ncand) return;
    const LaunchCand& e = t.cand[t.ntried];
    if (e.sched != c.sched || e.minb != c.minb || e.fold != c.fold) return;
    t.ms[t.ntried++] = ms;
}

// The three builds of the tracking kernels (tp_track.cu): with FMA
// contraction, without, and without with bounds checks.
enum TrackBuild { TB_FAST = 0, TB_STRICT = 1, TB_CHECKED = 2 };

TrackBuild track_build(const tp_opts& o) {
    if (o.bounds_check) return TB_CHECKED;
    return o.fp_contract ? TB_FAST : TB_STRICT;
}

// The strict build's 5- and 6-block instances live in a second unit.
bool strict_low(const TrackArgs* a, int minb) {
    return minb_track_strict_low(minb) == minb && minb > 0 && (a == nullptr || !a->rare);
}

int track_launch(TrackBuild b, const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream) {
    if (b == TB_CHECKED) return launch_track_checked(a, grid, block, minb, smem, stream);
    if (b == TB_STRICT)
        return strict_low(&a, minb) ? launch_track_strict_low(a, grid, block, minb, smem, stream)
                                    : launch_track_strict(a, grid, block, minb, smem, stream);
    return launch_track_fast(a, grid, block, minb, smem, stream);
}

int track_occupancy(TrackBuild b, int block, int minb, size_t smem, int* bps) {
    if (b == TB_CHECKED) return occupancy_track_checked(block, minb, smem, bps);
    if (b == TB_STRICT)
        return strict_low(nullptr, minb) ? occupancy_track_strict_low(block, minb, smem, bps)
                                         : occupancy_track_strict(block, minb, smem, bps);
    return occupancy_track_fast(block, minb, smem, bps);
}

int track_minb(TrackBuild b, int minb) {
    if (b == TB_CHECKED) return minb_track_checked(minb);
    if (b == TB_STRICT) return strict_low(nullptr, minb) ? minb : minb_track_strict(minb);
    return minb_track_fast(minb);
}

bool pick_launch(LaunchTune* tu, std::mutex* mu, uint64_t key, const tp_opts& o, int nturns, TrackBuild build,
                 bool rare, bool batched, LaunchCand* out) {
    int minbs[4] = {7, 8, 6, 5};
    int nminb = 1;
    if (!rare && track_minb(build, 5) == 5 && track_minb(build, 6) == 6 && track_minb(build, 8) == 8) nminb = 4;
    const int fixed_minb = o.min_blocks > 0 ? track_minb(build, o.min_blocks) : 0;
    const int fixed_sched = o.schedule == 1 || o.schedule == 2 ? o.schedule : 0;
    const bool folds = batched && fixed_sched != 1;
    if (nturns <= 1 || (fixed_sched && (fixed_minb || nminb == 1) && !folds)) {
        out->sched = fixed_sched ? fixed_sched : 1;
        out->minb = fixed_minb ? fixed_minb : minbs[0];
        out->fold = 1;
        return false;
    }
    bool trial = false;
    if (mu) {
        std::lock_guard<std::mutex> g(*mu);
        *out = tune_pick(*tu, key, fixed_sched, fixed_minb, minbs, nminb, folds, &trial);
    } else {
        *out = tune_pick(*tu, key, fixed_sched, fixed_minb, minbs, nminb, folds, &trial);
    }
    return trial;
}

std::atomic<uint64_t> g_stamp{0};
uint64_t next_stamp() { return ++g_stamp; }

// Device copy of a lattice on one device.
struct DevLattice {
    double* table = nullptr;
    MisalignDev* mis = nullptr;
    double* sched = nullptr;
    double* prefix = nullptr;  // inclusive prefix sums of per-element flops
    size_t sched_bytes = 0;
    uint64_t version = 0;
    LaunchTune tune;
};

}  // namespace

struct tp_lattice {
    std::vector<tp_elem> elems;
    std::vector<tp_misalign> mis;
    std::vector<double> aux;           // array fields of the elements (tp_lattice_create_ex)
    std::vector<double> program;       // compiled table, padded to 16 bytes
    std::vector<int32_t> rec_off;      // word offset of each record
    std::vector<double> flops_exact;   // per element, exact drift
    std::vector<double> flops_lin;     // per element, linearised drift
    // schedule
    std::vector<int32_t> sfields;
    int32_t sturn0 = 0, snturns = 0;
    std::vector<double> svalues;
    std::vector<double> sched_table;   // snturns x stride words
    int32_t sched_stride = 0;
    bool has_sched = false;
    uint64_t version = 1;
    uint64_t stamp = next_stamp();     // unique per lattice and program (see LatticeView)
    DevLattice dev[kMaxDevices];
    std::mutex mu;
};

struct tp_batch {
    std::vector<const tp_lattice*> lats;
    int32_t nvar = 0;
    int device = -1;
    double* table = nullptr;           // concatenated programs
    int64_t* toff = nullptr;           // toff[nvar+1], then tile_off[nvar+1]
    int32_t* nelem_v = nullptr;
    double* beti_v = nullptr;
    int64_t* poff = nullptr;
    MisalignDev* mis = nullptr;
    double* prefix = nullptr;          // per-variant inclusive flop prefix sums: exact drift, then linearised
    int64_t* prefix_off = nullptr;     // offsets of each variant's prefix (nvar + 1)
    int64_t prefix_words = 0;          // length of one prefix set
    std::vector<int64_t> h_toff;
    std::vector<int32_t> h_nelem;
    std::vector<int64_t> h_mis_off;    // misalignment row offset per variant
    size_t table_words = 0;
    bool rare = false;         // some variant holds kinds outside the integrator core
    double* sched = nullptr;           // concatenated per-turn schedule tables
    int64_t* sched_v = nullptr;        // per variant: word offset (-1: none), stride, first turn, turns
    std::vector<uint64_t> h_ver;       // lattice versions the device tables were built from
    unsigned long long* pool = nullptr; // per variant particles handed out (pooled refill)
    LaunchTune tune;
    std::vector<int64_t> h_sched_v;
    // cached CUDA graph of the launch sequence and every value it bakes in
    // (argument values, device pointers, launch shapes; see graph_key)
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> g_key;
};

struct tp_ctx {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // scratch: [0] work counter, [1] passes, [2] alive at start, [3] survivors; err word after
    unsigned long long* counters = nullptr;
    int32_t* err = nullptr;
    double* flops_acc = nullptr;
    // staging buffers for host pointers
    double* coords = nullptr;
    int64_t* lost = nullptr;
    int32_t* lost_turn = nullptr;
    int32_t* lost_elem = nullptr;
    uint8_t* alive0 = nullptr;
    int64_t cap = 0;
    tp_stats stats{};
    // grow-only device scratch of the adjoint and Jacobian paths
    void* scr[kCtxScratchSlots] = {};
    size_t scr_bytes[kCtxScratchSlots] = {};
};

namespace {

int ensure_capacity(tp_ctx* c, int64_t n) {
    if (n <= c->cap) return TP_OK;
    int64_t cap = std::max<int64_t>(n, c->cap * 2);
    cudaFree(c->coords); cudaFree(c->lost); cudaFree(c->lost_turn); cudaFree(c->lost_elem); cudaFree(c->alive0);
    c->coords = nullptr; c->lost = nullptr; c->lost_turn = nullptr; c->lost_elem = nullptr; c->alive0 = nullptr;
    c->cap = 0;
    if (cudaMalloc(&c->coords, size_t(cap) * 6 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->lost, size_t(cap) * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&c->lost_turn, size_t(cap) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&c->lost_elem, size_t(cap) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&c->alive0, size_t(cap)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(TP_ENOMEM, "device staging allocation failed");
    }
    c->cap = cap;
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Statistics kernels: alive-at-start mask before tracking; survivors and exact
// algorithmic FLOPs after it (full turns x flops per turn + the prefix up to
// and including the element of loss).
// ---------------------------------------------------------------------------
__global__ void k_alive_mask(const int64_t* lost, int64_t n, uint8_t* alive0, unsigned long long* count) {
    unsigned long long local = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        uint8_t a = lost[i] != 1;
        alive0[i] = a;
        local += a;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

__global__ void k_work_stats(const uint8_t* alive0, const int64_t* lost, const int32_t* lost_turn,
                             const int32_t* lost_elem, int64_t n, const double* prefix, const int64_t* poff,
                             const int64_t* pref_off, const int32_t* nelem_v, int32_t nvar, int32_t nelem, int32_t nturns,
                             int32_t turn0, unsigned long long* survivors, double* flops,
                             unsigned long long* passes) {
    unsigned long long surv = 0, ps = 0;
    double f = 0.0, u = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        if (!alive0[i]) continue;
        const double* pre = prefix;
        int ne = nelem;
        if (nvar > 0) {
            int lo = 0, hi = nvar - 1;
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (poff[mid] <= i) lo = mid; else hi = mid - 1;
            }
            pre = prefix + pref_off[lo];
            ne = nelem_v[lo];
        }
        const double per_turn = ne > 0 ? pre[ne - 1] : 0.0;
        u += double(ne) * double(nturns);
        if (lost[i] != 1) {
            surv += 1;
            f += double(nturns) * per_turn;
            ps += (unsigned long long)nturns * (unsigned long long)ne;
        } else {
            int full = lost_turn[i] - turn0;
            f += double(full) * per_turn + (lost_elem[i] >= 0 && ne > 0 ? pre[lost_elem[i]] : 0.0);
            // the maps evaluated: full turns, then the elements up to and including the one of loss
            ps += (unsigned long long)full * (unsigned long long)ne + (unsigned long long)(lost_elem[i] + 1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        ps += __shfl_down_sync(0xffffffffu, ps, o);
        surv += __shfl_down_sync(0xffffffffu, surv, o);
        f += __shfl_down_sync(0xffffffffu, f, o);
        u += __shfl_down_sync(0xffffffffu, u, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (ps) atomicAdd(passes, ps);
        if (surv) atomicAdd(survivors, surv);
        if (f != 0.0) atomicAdd(flops, f);
        if (u != 0.0) atomicAdd(flops + 1, u);
    }
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

// FP64 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void k_fp64_probe(double* out, int iters, double a, double b) {
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[0] = s;  // keep the chains alive
}

int grid_for(int64_t items, int block, int sm_count) {
    int64_t g = (items + block - 1) / block;
    g = std::min<int64_t>(g, int64_t(sm_count) * 8);
    return int(std::max<int64_t>(g, 1));
}

// Upload (or refresh) the lattice on the context's device.
int upload_lattice(tp_ctx* c, tp_lattice* L) {
    std::lock_guard<std::mutex> g(L->mu);
    DevLattice& d = L->dev[c->device];
    if (d.table && d.version == L->version) return TP_OK;
    cudaFree(d.table); cudaFree(d.mis); cudaFree(d.sched); cudaFree(d.prefix);
    d = DevLattice{};
    size_t tb = std::max<size_t>(L->program.size(), 2) * sizeof(double);
    TP_CUDA(cudaMalloc(&d.table, tb));
    TP_CUDA(cudaMemcpy(d.table, L->program.data(), L->program.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (!L->mis.empty()) {
        std::vector<MisalignDev> md(L->mis.size());
        for (size_t i = 0; i < L->mis.size(); ++i) {
            const tp_misalign& m = L->mis[i];
            MisalignDev& o = md[i];
            std::memcpy(o.t1, m.t1, sizeof o.t1); std::memcpy(o.t2, m.t2, sizeof o.t2);
            std::memcpy(o.r1, m.r1, sizeof o.r1); std::memcpy(o.r2, m.r2, sizeof o.r2);
            o.r1nz = 0; o.r2nz = 0;
            for (int k = 0; k < 36; ++k) { o.r1nz |= m.r1[k] != 0.0; o.r2nz |= m.r2[k] != 0.0; }
        }
        TP_CUDA(cudaMalloc(&d.mis, md.size() * sizeof(MisalignDev)));
        TP_CUDA(cudaMemcpy(d.mis, md.data(), md.size() * sizeof(MisalignDev), cudaMemcpyHostToDevice));
    }
    {   // inclusive flop prefix sums: exact-drift set, then linearised set
        const size_t n = std::max<size_t>(L->elems.size(), 1);
        std::vector<double> pre(2 * n, 0.0);
        double ae = 0.0, al = 0.0;
        for (size_t i = 0; i < L->elems.size(); ++i) {
            ae += L->flops_exact[i];
            al += L->flops_lin[i];
            pre[i] = ae;
            pre[n + i] = al;
        }
        TP_CUDA(cudaMalloc(&d.prefix, pre.size() * sizeof(double)));
        TP_CUDA(cudaMemcpy(d.prefix, pre.data(), pre.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (L->has_sched && !L->sched_table.empty()) {
        d.sched_bytes = L->sched_table.size() * sizeof(double);
        TP_CUDA(cudaMalloc(&d.sched, d.sched_bytes));
        TP_CUDA(cudaMemcpy(d.sched, L->sched_table.data(), d.sched_bytes, cudaMemcpyHostToDevice));
    }
    d.version = L->version;
    return TP_OK;
}

double* prefix_of(tp_ctx* c, tp_lattice* L, bool exact) {
    return L->dev[c->device].prefix + (exact ? 0 : std::max<size_t>(L->elems.size(), 1));
}

tp_opts default_opts(const tp_opts* o) {
    tp_opts r{};
    r.size = sizeof(tp_opts);
    r.exact_hamiltonian = 1;
    if (o && o->size > 0) {
        size_t sz = std::min<size_t>(size_t(o->size), sizeof(tp_opts));
        std::memcpy(&r, o, sz);
    }
    return r;
}

double loss_limit(double aperture) { return aperture > 0.0 ? std::min(1.0, aperture) : 1.0; }

int check_device_error(tp_ctx* c) {
    int32_t err = 0;
    TP_CUDA(cudaMemcpy(&err, c->err, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (err & DE_BOUNDS) return set_err(TP_EDEVICE, "bounds check: an element-table record or particle index "
                                                    "lay outside its array (the access was skipped)");
    if (err & DE_BAD_KIND) return set_err(TP_EUNSUPPORTED, "kernel met an unknown element record");
    if (err & DE_SCHED_RANGE) return set_err(TP_ERANGE, "turn outside the lattice schedule");
    if (err & DE_TMA_TIMEOUT) return set_err(TP_ETIMEOUT, "element-table staging wait ran out");
    return TP_OK;
}

}  // namespace

namespace tp {

void lattice_view(const tp_lattice* lat, LatticeView* out) {
    out->program = lat->program.data();
    out->words = lat->program.size();
    out->nelem = int32_t(lat->elems.size());
    out->has_schedule = lat->has_sched;
    out->has_misalignment = !lat->mis.empty();
    out->stamp = lat->stamp;
}

std::mutex& lattice_mutex(const tp_lattice* lat) { return const_cast<tp_lattice*>(lat)->mu; }

void lattice_host(const tp_lattice* lat, LatticeHost* out) {
    out->elems = lat->elems.data();
    out->nelem = int32_t(lat->elems.size());
    out->program = lat->program.data();
    out->words = lat->program.size();
    out->rec_off = lat->rec_off.data();
    out->has_schedule = lat->has_sched;
    out->sched = lat->has_sched ? lat->sched_table.data() : nullptr;
    out->sched_words = lat->has_sched ? lat->sched_table.size() : 0;
    out->sched_stride = lat->sched_stride;
    out->sched_turn0 = lat->sturn0;
    out->sched_nturns = lat->snturns;
    out->nmis = int64_t(lat->mis.size());
    out->mis = lat->mis.data();
}

void ctx_host(const tp_ctx* c, CtxHost* out) {
    out->device = c->device;
    out->sm_count = c->sm_count;
    out->smem_optin = c->smem_optin;
    out->stream = c->stream;
}

tp_stats* ctx_stats(tp_ctx* c) { return &c->stats; }

int ctx_scratch(tp_ctx* c, int slot, size_t bytes, void** out) {
    if (slot < 0 || slot >= kCtxScratchSlots) return set_err(TP_EINVAL, "scratch slot out of range");
    bytes = std::max<size_t>(bytes, 256);
    if (c->scr_bytes[slot] < bytes) {
        if (c->scr[slot]) {
            cudaStreamSynchronize(c->stream);
            cudaFree(c->scr[slot]);
        }
        c->scr[slot] = nullptr;
        c->scr_bytes[slot] = 0;
        if (cudaMalloc(&c->scr[slot], bytes) != cudaSuccess) {
            cudaGetLastError();
            return set_err(TP_ENOMEM, "device scratch allocation of " + std::to_string(bytes) + " bytes failed");
        }
        c->scr_bytes[slot] = bytes;
    }
    *out = c->scr[slot];
    return TP_OK;
}

void batch_lattices(const tp_batch* b, std::vector<const tp_lattice*>* out) { *out = b->lats; }

void set_last_error(const std::string& msg) { g_last_error = msg; }

NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
NvtxRange::~NvtxRange() { nvtxRangePop(); }

}  // namespace tp

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

TP_API int tp_abi_version(void) { return TP_ABI_VERSION; }

TP_API const char* tp_strerror(int status) {
    switch (status) {
        case TP_OK: return "ok";
        case TP_EINVAL: return "invalid argument";
        case TP_ENOMEM: return "out of memory";
        case TP_EUNSUPPORTED: return "unsupported element kind or option";
        case TP_ECUDA: return "CUDA runtime error";
        case TP_ETIMEOUT: return "bounded device wait ran out";
        case TP_EDEVICE: return "device reported an error";
        case TP_ENODEV: return "no usable CUDA device";
        case TP_ERANGE: return "size or index beyond a documented maximum";
        default: return "unknown status";
    }
}

TP_API const char* tp_last_error_string(void) { return g_last_error.c_str(); }

TP_API int tp_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

TP_API int tp_beam_beti(double energy, double mass, double* beti_out) {
    if (!beti_out) return set_err(TP_EINVAL, "beti_out is null");
    if (!(mass > 0.0) || !(energy > 0.0)) return set_err(TP_EINVAL, "energy and mass must be positive");
    double gamma = (energy + mass) / mass;              // src/lattice.jl:51
    double beta = std::sqrt(1.0 - 1.0 / (gamma * gamma));  // :52
    *beti_out = 1.0 / beta;                              // :61
    return TP_OK;
}

TP_API int tp_ctx_create(int device, tp_ctx** out) {
    if (!out) return set_err(TP_EINVAL, "out is null");
    *out = nullptr;
    int ndev = tp_device_count();
    if (ndev <= 0) return set_err(TP_ENODEV, "no CUDA device");
    if (device < 0 || device >= ndev || device >= kMaxDevices) return set_err(TP_EINVAL, "device ordinal out of range");
    tp_ctx* c = new (std::nothrow) tp_ctx();
    if (!c) return set_err(TP_ENOMEM, "host allocation failed");
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    c->smem_optin = size_t(optin);
    // A blocking stream: it waits for work queued on the legacy default stream
    // and that stream waits for it, so device arrays a caller fills on its
    // default stream (PyTorch's, unless it set another) are complete before a
    // call's first kernel reads them.
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e == cudaSuccess) e = cudaMalloc(&c->counters, 8 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->err, 4 * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c->flops_acc, 2 * sizeof(double));
    if (e != cudaSuccess) {
        int st = cuda_err(e, "tp_ctx_create");
        tp_ctx_destroy(c);
        return st;
    }
    *out = c;
    return TP_OK;
}

TP_API int tp_ctx_destroy(tp_ctx* c) {
    if (!c) return TP_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->counters); cudaFree(c->err); cudaFree(c->flops_acc);
    cudaFree(c->coords); cudaFree(c->lost); cudaFree(c->lost_turn); cudaFree(c->lost_elem); cudaFree(c->alive0);
    for (int k = 0; k < kCtxScratchSlots; ++k) cudaFree(c->scr[k]);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return TP_OK;
}

TP_API int tp_last_stats(const tp_ctx* c, tp_stats* out) {
    if (!c || !out) return set_err(TP_EINVAL, "null argument");
    *out = c->stats;
    return TP_OK;
}

// ---------------------------------------------------------------------------
TP_API int tp_lattice_create(const tp_elem* elems, int64_t n, const tp_misalign* mis, int64_t nmis,
                             tp_lattice** out) {
    return tp_lattice_create_ex(elems, n, mis, nmis, nullptr, 0, out);
}

TP_API int tp_lattice_create_ex(const tp_elem* elems, int64_t n, const tp_misalign* mis, int64_t nmis,
                                const double* aux, int64_t naux, tp_lattice** out) {
    if (!out) return set_err(TP_EINVAL, "out is null");
    *out = nullptr;
    if (n < 0 || nmis < 0 || naux < 0) return set_err(TP_EINVAL, "negative size");
    if (n > 0 && !elems) return set_err(TP_EINVAL, "elems is null");
    if (nmis > 0 && !mis) return set_err(TP_EINVAL, "mis is null");
    if (naux > 0 && !aux) return set_err(TP_EINVAL, "aux is null");
    if (n > (int64_t(1) << 24)) return set_err(TP_ERANGE, "lattice longer than 2^24 elements");
    const AuxView av{aux, naux};
    std::string err;
    for (int64_t i = 0; i < n; ++i) {
        int st = validate_elem(elems[i], i, nmis, &err, av);
        if (st != TP_OK) return set_err(st, err);
    }
    tp_lattice* L = new (std::nothrow) tp_lattice();
    if (!L) return set_err(TP_ENOMEM, "host allocation failed");
    L->elems.assign(elems, elems + n);
    if (nmis > 0) L->mis.assign(mis, mis + nmis);
    if (naux > 0) L->aux.assign(aux, aux + naux);
    const AuxView lav{L->aux.data(), int64_t(L->aux.size())};
    L->rec_off.resize(size_t(n));
    L->flops_exact.resize(size_t(n));
    L->flops_lin.resize(size_t(n));
    for (int64_t i = 0; i < n; ++i) {
        L->rec_off[size_t(i)] = int32_t(L->program.size());
        compile_record(elems[i], &L->program, lav);
        const tp_misalign* m = elems[i].misalign_index >= 0 ? &mis[elems[i].misalign_index] : nullptr;
        L->flops_exact[size_t(i)] = elem_flops(elems[i], m, true, lav);
        L->flops_lin[size_t(i)] = elem_flops(elems[i], m, false, lav);
    }
    if (L->program.size() > (size_t(1) << 30)) {
        delete L;
        return set_err(TP_ERANGE, "element table too large");
    }
    while (L->program.size() % 2) L->program.push_back(0.0);  // 16-byte multiple for the bulk copy
    *out = L;
    return TP_OK;
}

TP_API int tp_lattice_destroy(tp_lattice* L) {
    if (!L) return TP_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < kMaxDevices; ++d) {
        DevLattice& x = L->dev[d];
        if (x.table || x.mis || x.sched || x.prefix) {
            cudaSetDevice(d);
            cudaFree(x.table); cudaFree(x.mis); cudaFree(x.sched); cudaFree(x.prefix);
        }
    }
    cudaSetDevice(cur);
    cudaGetLastError();
    delete L;
    return TP_OK;
}

TP_API int tp_lattice_length(const tp_lattice* L, int64_t* n_out) {
    if (!L || !n_out) return set_err(TP_EINVAL, "null argument");
    *n_out = int64_t(L->elems.size());
    return TP_OK;
}

TP_API int tp_lattice_flops(const tp_lattice* L, double* out) {
    if (!L || (!out && !L->elems.empty())) return set_err(TP_EINVAL, "null argument");
    for (size_t i = 0; i < L->elems.size(); ++i) out[i] = L->flops_exact[i];
    return TP_OK;
}

TP_API int tp_lattice_set_schedule(tp_lattice* L, const int32_t* fields, int32_t nfields, int32_t turn0,
                                   int32_t nturns, const double* values) {
    if (!L) return set_err(TP_EINVAL, "lattice is null");
    std::lock_guard<std::mutex> g(L->mu);
    if (nfields == 0) {
        // restore the static program
        L->program.clear();
        for (size_t i = 0; i < L->elems.size(); ++i) {
            L->rec_off[i] = int32_t(L->program.size());
            compile_record(L->elems[i], &L->program, AuxView{L->aux.data(), int64_t(L->aux.size())});
        }
        while (L->program.size() % 2) L->program.push_back(0.0);
        L->has_sched = false;
        L->sfields.clear(); L->svalues.clear(); L->sched_table.clear();
        L->version++;
        L->stamp = next_stamp();
        return TP_OK;
    }
    if (nfields < 0 || !fields || nturns <= 0 || !values) return set_err(TP_EINVAL, "bad schedule arguments");
    const int64_t ne = int64_t(L->elems.size());
    std::vector<int32_t> sched_elems;
    for (int32_t j = 0; j < nfields; ++j) {
        int32_t e = fields[2 * j], f = fields[2 * j + 1];
        if (e < 0 || e >= ne) return set_err(TP_EINVAL, "schedule element index out of range");
        if (f < 0 || f >= TP_FIELD_COUNT) return set_err(TP_EINVAL, "unknown schedule field");
        if (std::find(sched_elems.begin(), sched_elems.end(), e) == sched_elems.end()) sched_elems.push_back(e);
    }
    std::sort(sched_elems.begin(), sched_elems.end());
    // Slot of each scheduled element inside a turn block.
    std::vector<int32_t> slot(size_t(ne), -1);
    int32_t stride = 0;
    for (int32_t e : sched_elems) {
        slot[size_t(e)] = stride;
        stride += record_words(L->elems[size_t(e)], AuxView{L->aux.data(), int64_t(L->aux.size())});
    }
    std::vector<double> table;
    table.reserve(size_t(stride) * size_t(nturns));
    std::string err;
    for (int32_t t = 0; t < nturns; ++t) {
        for (int32_t e : sched_elems) {
            tp_elem x = L->elems[size_t(e)];
            for (int32_t j = 0; j < nfields; ++j)
                if (fields[2 * j] == e) apply_field(&x, fields[2 * j + 1], values[int64_t(t) * nfields + j]);
            const AuxView lav{L->aux.data(), int64_t(L->aux.size())};
            int st = validate_elem(x, e, int64_t(L->mis.size()), &err, lav);
            if (st != TP_OK) return set_err(st, err);
            size_t before = table.size();
            compile_record(x, &table, lav);
            if (int32_t(table.size() - before) != record_words(L->elems[size_t(e)], lav))
                return set_err(TP_EINVAL, "schedule changes the record layout of an element");
        }
    }
    L->program.clear();
    for (int64_t i = 0; i < ne; ++i) {
        L->rec_off[size_t(i)] = int32_t(L->program.size());
        const AuxView lav{L->aux.data(), int64_t(L->aux.size())};
        if (slot[size_t(i)] >= 0) scheduled_stub(L->elems[size_t(i)], slot[size_t(i)], &L->program, lav);
        else compile_record(L->elems[size_t(i)], &L->program, lav);
    }
    while (L->program.size() % 2) L->program.push_back(0.0);
    L->sfields.assign(fields, fields + 2 * nfields);
    L->sturn0 = turn0;
    L->snturns = nturns;
    L->svalues.assign(values, values + int64_t(nturns) * nfields);
    L->sched_table.swap(table);
    L->sched_stride = stride;
    L->has_sched = true;
    L->version++;
    L->stamp = next_stamp();
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Tracking
// ---------------------------------------------------------------------------
static int track_common(tp_ctx* c, tp_lattice* L, double* coords, int64_t n, int64_t* lost_flags,
                        int32_t* lost_turn, int32_t* lost_elem, double beti, int32_t nturns, int32_t turn0,
                        const tp_opts* opts_in) {
    auto t_start = std::chrono::steady_clock::now();
    if (!c || !L) return set_err(TP_EINVAL, "null context or lattice");
    if (n < 0) return set_err(TP_EINVAL, "negative particle count");
    if (nturns < 0) return set_err(TP_EINVAL, "negative number of turns");
    if (!(beti > 0.0) || !std::isfinite(beti)) return set_err(TP_EINVAL, "beti must be finite and positive");
    if (n > 0 && (!coords || !lost_flags)) return set_err(TP_EINVAL, "coords and lost_flags are required");
    if (n > (int64_t(1) << 40)) return set_err(TP_ERANGE, "particle count beyond 2^40");
    tp_opts o = default_opts(opts_in);
    c->stats = tp_stats{};
    if (n == 0 || nturns == 0) return TP_OK;
    if (L->has_sched) {
        if (int64_t(turn0) < L->sturn0 || int64_t(turn0) + nturns > int64_t(L->sturn0) + L->snturns)
            return set_err(TP_ERANGE, "turns outside the lattice schedule");
    }
    TP_CUDA(cudaSetDevice(c->device));
    int st = upload_lattice(c, L);
    if (st != TP_OK) return st;
    cudaStream_t s = o.stream ? static_cast<cudaStream_t>(o.stream) : c->stream;
    const bool dev = o.device_pointers != 0;
    const bool exact = o.exact_hamiltonian != 0;
    double* d_coords = coords;
    int64_t* d_lost = lost_flags;
    int32_t* d_lt = lost_turn;
    int32_t* d_le = lost_elem;
    st = ensure_capacity(c, n);
    if (st != TP_OK) return st;
    int64_t h2d = 0, d2h = 0;
    if (!dev) {
        d_coords = c->coords;
        d_lost = c->lost;
        TP_CUDA(cudaMemcpyAsync(d_coords, coords, size_t(n) * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
        TP_CUDA(cudaMemcpyAsync(d_lost, lost_flags, size_t(n) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        h2d += n * 6 * 8 + n * 8;
        d_lt = c->lost_turn;
        d_le = c->lost_elem;
        if (lost_turn) { TP_CUDA(cudaMemcpyAsync(d_lt, lost_turn, size_t(n) * 4, cudaMemcpyHostToDevice, s)); h2d += n * 4; }
        if (lost_elem) { TP_CUDA(cudaMemcpyAsync(d_le, lost_elem, size_t(n) * 4, cudaMemcpyHostToDevice, s)); h2d += n * 4; }
    } else {
        if (!d_lt) d_lt = c->lost_turn;
        if (!d_le) d_le = c->lost_elem;
    }
    double* prefix = prefix_of(c, L, exact);
    DevLattice& dl = L->dev[c->device];

    TrackArgs a{};
    a.table = dl.table;
    a.table_words = int32_t(L->program.size());
    a.nelem = int32_t(L->elems.size());
    a.sched = dl.sched;
    a.sched_stride = L->sched_stride;
    a.sched_turn0 = L->sturn0;
    a.sched_nturns = L->snturns;
    a.mis = dl.mis;
    a.rare = records_have_rare(L->program.data(), L->program.size()) ? 1 : 0;
    a.coords = d_coords;
    a.n = n;
    a.lost_flags = d_lost;
    a.lost_turn = d_lt;
    a.lost_elem = d_le;
    a.beti = beti;
    a.limx = loss_limit(o.aperture_x);
    a.limy = loss_limit(o.aperture_y);
    a.nturns = nturns;
    a.turn0 = turn0;
    a.exact = exact ? 1 : 0;
    a.work = c->counters;
    a.passes = c->counters + 1;
    a.err = c->err;
    a.nvar = 0;
    const size_t table_bytes = L->program.size() * sizeof(double);
    const size_t smem = o.table_in_smem && table_bytes + 64 <= c->smem_optin ? table_bytes : 0;
    a.smem_words = smem ? int32_t(L->program.size()) : 0;
    // Launch configuration: static at the default occupancy for single passes;
    // for multi-turn tracks what the caller asks for, else the tuned choice
    // (lane refill frees the lanes of lost particles, static has less
    // bookkeeping; more resident blocks hide more latency, fewer spill less).
    int block = o.block_size > 0 ? o.block_size : 128;
    block = std::max(32, std::min(kTrackMaxBlock, block / 32 * 32));
    const TrackBuild build = track_build(o);
    const bool strict = build != TB_FAST;
    const uint64_t tkey = tune_key({n, nturns, int64_t(exact), int64_t(build), block, int64_t(L->version),
                                    int64_t(L->program.size()), int64_t(smem), o.schedule, o.min_blocks});
    LaunchCand lc;
    const bool tuning = pick_launch(&L->dev[c->device].tune, &L->mu, tkey, o, nturns, build, a.rare != 0, false,
                                    &lc);
    const int schedule = lc.sched;
    a.refill = schedule == 2 ? 1 : 0;
    int bps = 0;
    int oerr = track_occupancy(build, block, lc.minb, smem, &bps);
    if (oerr != 0 || bps <= 0) bps = 1;
    int64_t grid_needed = (n + block - 1) / block;
    int grid = a.refill ? int(std::min<int64_t>(int64_t(c->sm_count) * bps, grid_needed)) : int(grid_needed);
    grid = std::max(grid, 1);

    TP_CUDA(cudaMemsetAsync(c->counters, 0, 8 * sizeof(unsigned long long), s));
    TP_CUDA(cudaMemsetAsync(c->err, 0, 4 * sizeof(int32_t), s));
    TP_CUDA(cudaMemsetAsync(c->flops_acc, 0, 2 * sizeof(double), s));
    int sg = grid_for(n, 256, c->sm_count);
    if (!lost_turn) k_fill_i32<<<sg, 256, 0, s>>>(d_lt, n, -1);
    if (!lost_elem) k_fill_i32<<<sg, 256, 0, s>>>(d_le, n, -1);
    k_alive_mask<<<sg, 256, 0, s>>>(d_lost, n, c->alive0, c->counters + 2);
    TP_CUDA(cudaGetLastError());
    TP_CUDA(cudaEventRecord(c->ev0, s));
    int le = track_launch(build, a, grid, block, lc.minb, smem, s);
    if (le != 0) return cuda_err(cudaError_t(le), "track kernel launch");
    TP_CUDA(cudaEventRecord(c->ev1, s));
    k_work_stats<<<sg, 256, 0, s>>>(c->alive0, d_lost, d_lt, d_le, n, prefix, nullptr, nullptr, nullptr, 0, a.nelem,
                                     nturns, turn0, c->counters + 3, c->flops_acc, c->counters + 1);
    TP_CUDA(cudaGetLastError());
    if (!dev) {
        TP_CUDA(cudaMemcpyAsync(coords, d_coords, size_t(n) * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
        TP_CUDA(cudaMemcpyAsync(lost_flags, d_lost, size_t(n) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        d2h += n * 6 * 8 + n * 8;
        if (lost_turn) { TP_CUDA(cudaMemcpyAsync(lost_turn, d_lt, size_t(n) * 4, cudaMemcpyDeviceToHost, s)); d2h += n * 4; }
        if (lost_elem) { TP_CUDA(cudaMemcpyAsync(lost_elem, d_le, size_t(n) * 4, cudaMemcpyDeviceToHost, s)); d2h += n * 4; }
    }
    unsigned long long cnt[4];
    double fl[2];
    TP_CUDA(cudaMemcpyAsync(cnt, c->counters, sizeof cnt, cudaMemcpyDeviceToHost, s));
    TP_CUDA(cudaMemcpyAsync(fl, c->flops_acc, sizeof fl, cudaMemcpyDeviceToHost, s));
    TP_CUDA(cudaStreamSynchronize(s));
    st = check_device_error(c);
    if (st != TP_OK) return st;
    float ms = 0.f;
    TP_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (tuning) {
        std::lock_guard<std::mutex> g(L->mu);
        tune_record(L->dev[c->device].tune, tkey, lc, ms);
    }
    tp_stats& S = c->stats;
    S.particles = int64_t(cnt[2]);
    S.survivors = int64_t(cnt[3]);
    S.element_passes = int64_t(cnt[1]);
    S.units = fl[1];
    S.flops = fl[0];
    S.kernel_ms = ms;
    S.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    S.h2d_bytes = h2d;
    S.d2h_bytes = d2h;
    S.block_size = block;
    S.min_blocks = track_minb(build, lc.minb);
    S.grid = grid;
    S.launches = 3 + (lost_turn ? 0 : 1) + (lost_elem ? 0 : 1);
    S.schedule = schedule;
    S.fp_contract = strict ? 0 : 1;
    S.refill_fold = 1;
    S.bounds_check = build == TB_CHECKED ? 1 : 0;
    return TP_OK;
}

TP_API int tp_linepass(tp_ctx* c, const tp_lattice* L, double* coords, int64_t n, int64_t* lost_flags,
                       int32_t* lost_turn, int32_t* lost_elem, double beti, double time, int32_t turn,
                       const tp_opts* opts) {
    NvtxRange r("tp_linepass");
    (void)time;  // the host evaluates time-dependent fields into the per-turn schedule
    return track_common(c, const_cast<tp_lattice*>(L), coords, n, lost_flags, lost_turn, lost_elem, beti, 1, turn,
                        opts);
}

TP_API int tp_ringpass(tp_ctx* c, const tp_lattice* L, double* coords, int64_t n, int64_t* lost_flags,
                       int32_t* lost_turn, int32_t* lost_elem, double beti, int32_t nturns, double time,
                       double dt_turn, int32_t turn0, const tp_opts* opts) {
    NvtxRange r("tp_ringpass");
    (void)time;
    (void)dt_turn;
    return track_common(c, const_cast<tp_lattice*>(L), coords, n, lost_flags, lost_turn, lost_elem, beti, nturns,
                        turn0, opts);
}

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------
// (Re)build the device tables of a batch from its lattices: programs,
// misalignment rows, per-turn schedules and FLOP prefix tables.
static void batch_free_tables(tp_batch* b) {
    cudaFree(b->table); cudaFree(b->toff); cudaFree(b->nelem_v); cudaFree(b->beti_v); cudaFree(b->poff);
    cudaFree(b->mis); cudaFree(b->prefix); cudaFree(b->prefix_off); cudaFree(b->sched); cudaFree(b->sched_v);
    cudaFree(b->pool);
    b->table = nullptr; b->toff = nullptr; b->nelem_v = nullptr; b->beti_v = nullptr; b->poff = nullptr;
    b->mis = nullptr; b->prefix = nullptr; b->prefix_off = nullptr; b->sched = nullptr; b->sched_v = nullptr;
    b->pool = nullptr;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
}

static int batch_build(tp_batch* b) {
    batch_free_tables(b);
    const int32_t nvar = b->nvar;
    std::vector<double> table, sched;
    std::vector<MisalignDev> mis;
    b->h_toff.assign(size_t(nvar) + 1, 0);
    b->h_nelem.assign(size_t(nvar), 0);
    b->h_ver.assign(size_t(nvar), 0);
    b->h_sched_v.assign(4 * size_t(nvar), 0);
    for (int32_t v = 0; v < nvar; ++v) {
        const tp_lattice* L = b->lats[size_t(v)];
        b->h_ver[size_t(v)] = L->version;
        b->h_toff[size_t(v)] = int64_t(table.size());
        b->h_nelem[size_t(v)] = int32_t(L->elems.size());
        int32_t mbase = int32_t(mis.size());
        size_t at = table.size();
        table.insert(table.end(), L->program.begin(), L->program.end());
        if (v == 0) b->rare = false;
        if (records_have_rare(L->program.data(), L->program.size())) b->rare = true;
        if (mbase > 0) {  // shift misalignment rows of this variant
            for (size_t e = 0; e < L->elems.size(); ++e) {
                RecHdr* h = reinterpret_cast<RecHdr*>(table.data() + at + L->rec_off[e]);
                if (h->flags & RF_MISALIGN) h->aux += mbase;
            }
        }
        for (const tp_misalign& m : L->mis) {
            MisalignDev o{};
            std::memcpy(o.t1, m.t1, sizeof o.t1); std::memcpy(o.t2, m.t2, sizeof o.t2);
            std::memcpy(o.r1, m.r1, sizeof o.r1); std::memcpy(o.r2, m.r2, sizeof o.r2);
            for (int k = 0; k < 36; ++k) { o.r1nz |= m.r1[k] != 0.0; o.r2nz |= m.r2[k] != 0.0; }
            mis.push_back(o);
        }
        int64_t* sv = &b->h_sched_v[4 * size_t(v)];
        sv[0] = -1;
        if (L->has_sched) {
            sv[0] = int64_t(sched.size());
            sv[1] = L->sched_stride;
            sv[2] = L->sturn0;
            sv[3] = L->snturns;
            std::vector<double> blk = L->sched_table;
            if (mbase > 0) {  // misalignment rows inside the per-turn records
                for (size_t w = 0; w < blk.size();) {
                    RecHdr* h = reinterpret_cast<RecHdr*>(blk.data() + w);
                    if (h->words == 0) break;
                    if (h->flags & RF_MISALIGN) h->aux += mbase;
                    w += h->words;
                }
            }
            sched.insert(sched.end(), blk.begin(), blk.end());
        }
    }
    b->h_toff[size_t(nvar)] = int64_t(table.size());
    b->table_words = table.size();
    // FLOP prefix tables of every variant (exact drift set, then linearised set).
    std::vector<double> pre_e, pre_l;
    std::vector<int64_t> pre_off(size_t(nvar) + 1, 0);
    for (int32_t v = 0; v < nvar; ++v) {
        const tp_lattice* L = b->lats[size_t(v)];
        pre_off[size_t(v)] = int64_t(pre_e.size());
        double ae = 0.0, al = 0.0;
        for (size_t i = 0; i < L->elems.size(); ++i) {
            ae += L->flops_exact[i];
            al += L->flops_lin[i];
            pre_e.push_back(ae);
            pre_l.push_back(al);
        }
        if (L->elems.empty()) { pre_e.push_back(0.0); pre_l.push_back(0.0); }
    }
    pre_off[size_t(nvar)] = int64_t(pre_e.size());
    b->prefix_words = int64_t(pre_e.size());
    pre_e.insert(pre_e.end(), pre_l.begin(), pre_l.end());
    cudaError_t e = cudaMalloc(&b->table, std::max<size_t>(table.size(), 2) * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(b->table, table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->toff, 3 * (size_t(nvar) + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMemcpy(b->toff, b->h_toff.data(), (size_t(nvar) + 1) * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->nelem_v, size_t(nvar) * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpy(b->nelem_v, b->h_nelem.data(), size_t(nvar) * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->beti_v, size_t(nvar) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->poff, (size_t(nvar) + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->prefix, pre_e.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(b->prefix, pre_e.data(), pre_e.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->prefix_off, pre_off.size() * sizeof(int64_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->prefix_off, pre_off.data(), pre_off.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !mis.empty()) {
        e = cudaMalloc(&b->mis, mis.size() * sizeof(MisalignDev));
        if (e == cudaSuccess) e = cudaMemcpy(b->mis, mis.data(), mis.size() * sizeof(MisalignDev), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && !sched.empty()) {
        e = cudaMalloc(&b->sched, sched.size() * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(b->sched, sched.data(), sched.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->pool, size_t(nvar) * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&b->sched_v, b->h_sched_v.size() * sizeof(int64_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(b->sched_v, b->h_sched_v.data(), b->h_sched_v.size() * sizeof(int64_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_err(e, "batch tables");
    return TP_OK;
}

TP_API int tp_batch_create(tp_ctx* c, const tp_lattice* const* lats, int32_t nvar, tp_batch** out) {
    if (!c || !out || (nvar > 0 && !lats)) return set_err(TP_EINVAL, "null argument");
    *out = nullptr;
    if (nvar <= 0) return set_err(TP_EINVAL, "a batch needs at least one lattice");
    for (int32_t v = 0; v < nvar; ++v) {
        if (!lats[v]) return set_err(TP_EINVAL, "null lattice in batch");
    }
    TP_CUDA(cudaSetDevice(c->device));
    tp_batch* b = new (std::nothrow) tp_batch();
    if (!b) return set_err(TP_ENOMEM, "host allocation failed");
    b->nvar = nvar;
    b->device = c->device;
    b->lats.assign(lats, lats + nvar);
    int st = batch_build(b);
    if (st != TP_OK) {
        tp_batch_destroy(b);
        return st;
    }
    *out = b;
    return TP_OK;
}

TP_API int tp_batch_destroy(tp_batch* b) {
    if (!b) return TP_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    if (b->device >= 0) cudaSetDevice(b->device);
    batch_free_tables(b);
    cudaSetDevice(cur);
    cudaGetLastError();
    delete b;
    return TP_OK;
}

TP_API int tp_ringpass_batched(tp_ctx* c, tp_batch* b, double* coords, const int64_t* poff, int64_t* lost_flags,
                               int32_t* lost_turn, int32_t* lost_elem, const double* beti, int32_t nturns,
                               double time, double dt_turn, int32_t turn0, int32_t use_graph,
                               const tp_opts* opts_in) {
    NvtxRange r("tp_ringpass_batched");
    (void)time;
    (void)dt_turn;
    auto t_start = std::chrono::steady_clock::now();
    if (!c || !b || !poff || !beti) return set_err(TP_EINVAL, "null argument");
    if (b->device != c->device) return set_err(TP_EINVAL, "batch and context are on different devices");
    if (nturns < 0) return set_err(TP_EINVAL, "negative number of turns");
    const int32_t nvar = b->nvar;
    if (poff[0] != 0) return set_err(TP_EINVAL, "poff[0] must be 0");
    for (int32_t v = 0; v < nvar; ++v) {
        if (poff[v + 1] < poff[v]) return set_err(TP_EINVAL, "poff must be non-decreasing");
        if (!(beti[v] > 0.0) || !std::isfinite(beti[v])) return set_err(TP_EINVAL, "beti must be finite and positive");
    }
    const int64_t n = poff[nvar];
    if (n > 0 && (!coords || !lost_flags)) return set_err(TP_EINVAL, "coords and lost_flags are required");
    tp_opts o = default_opts(opts_in);
    c->stats = tp_stats{};
    if (n == 0 || nturns == 0) return TP_OK;
    for (int32_t v = 0; v < nvar; ++v) {
        const tp_lattice* L = b->lats[size_t(v)];
        if (L->has_sched && (int64_t(turn0) < L->sturn0 || int64_t(turn0) + nturns > int64_t(L->sturn0) + L->snturns))
            return set_err(TP_ERANGE, "turns outside the schedule of variant " + std::to_string(v));
    }
    TP_CUDA(cudaSetDevice(c->device));
    {   // a member lattice changed (e.g. a new schedule): rebuild the device tables
        bool stale = false;
        for (int32_t v = 0; v < nvar; ++v) stale = stale || b->lats[size_t(v)]->version != b->h_ver[size_t(v)];
        if (stale) {
            TP_CUDA(cudaDeviceSynchronize());
            int bst = batch_build(b);
            if (bst != TP_OK) return bst;
        }
    }
    cudaStream_t s = o.stream ? static_cast<cudaStream_t>(o.stream) : c->stream;
    const bool dev = o.device_pointers != 0;
    const bool exact = o.exact_hamiltonian != 0;
    const TrackBuild build = track_build(o);
    const bool strict = build != TB_FAST;
    int st = ensure_capacity(c, n);
    if (st != TP_OK) return st;
    double* d_coords = dev ? coords : c->coords;
    int64_t* d_lost = dev ? lost_flags : c->lost;
    int32_t* d_lt = (dev && lost_turn) ? lost_turn : c->lost_turn;
    int32_t* d_le = (dev && lost_elem) ? lost_elem : c->lost_elem;
    int64_t h2d = 0, d2h = 0;
    if (!dev) {
        TP_CUDA(cudaMemcpyAsync(d_coords, coords, size_t(n) * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
        TP_CUDA(cudaMemcpyAsync(d_lost, lost_flags, size_t(n) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
        h2d += n * 56;
        if (lost_turn) { TP_CUDA(cudaMemcpyAsync(d_lt, lost_turn, size_t(n) * 4, cudaMemcpyHostToDevice, s)); h2d += n * 4; }
        if (lost_elem) { TP_CUDA(cudaMemcpyAsync(d_le, lost_elem, size_t(n) * 4, cudaMemcpyHostToDevice, s)); h2d += n * 4; }
    }
    const double* d_pre = b->prefix + (exact ? 0 : b->prefix_words);
    const int64_t* d_pre_off = b->prefix_off;

    TrackArgs a{};
    a.table = b->table;
    a.table_words = int32_t(b->table_words);
    a.mis = b->mis;
    a.rare = b->rare ? 1 : 0;
    a.coords = d_coords;
    a.n = n;
    a.lost_flags = d_lost;
    a.lost_turn = d_lt;
    a.lost_elem = d_le;
    a.beti = beti[0];
    a.limx = loss_limit(o.aperture_x);
    a.limy = loss_limit(o.aperture_y);
    a.nturns = nturns;
    a.turn0 = turn0;
    a.exact = exact ? 1 : 0;
    a.work = c->counters;
    a.passes = c->counters + 1;
    a.err = c->err;
    a.poff = b->poff;
    a.toff = b->toff;
    a.beti_v = b->beti_v;
    a.nelem_v = b->nelem_v;
    a.nvar = nvar;
    a.sched = b->sched;
    a.sched_v = b->sched_v;
    a.pool = b->pool;
    int block = o.block_size > 0 ? std::max(32, std::min(kTrackMaxBlock, o.block_size / 32 * 32)) : 128;
    // Static tiles or pooled refill: the caller's choice, else tuned online.
    int64_t ph = 0;
    for (int32_t v = 0; v <= nvar; ++v) ph = ph * 1000003 + poff[v];
    const uint64_t tkey = tune_key({n, nturns, int64_t(exact), int64_t(build), block, ph, int64_t(b->table_words),
                                    o.schedule, o.min_blocks});
    LaunchCand lc;
    const bool tuning = pick_launch(&b->tune, nullptr, tkey, o, nturns, build, a.rare != 0, true, &lc);
    const int schedule = lc.sched;
    a.refill = schedule == 2 ? 1 : 0;
    const int fold = a.refill ? std::max(1, lc.fold) : 1;
    // Per-variant offsets, betas, tile offsets and flop prefix tables.  Tiles
    // are handed out longest first: the variants with the most elements (the
    // longest 32-particle loads) come first, so that short loads fill the end
    // of the launch.  With pooled refill, `fold` > 1 hands out 1/fold as many
    // tiles per variant: fewer warps per variant, each refilling its lanes
    // from the variant's pool more often.  Layout: toff[nvar+1], tile offsets in that order
    // [nvar+1], the order itself [nvar].
    std::vector<int32_t> order(static_cast<size_t>(nvar));
    for (int32_t v = 0; v < nvar; ++v) order[size_t(v)] = v;
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return b->h_nelem[size_t(x)] > b->h_nelem[size_t(y)]; });
    std::vector<int64_t> offs(3 * (size_t(nvar) + 1));
    for (int32_t v = 0; v <= nvar; ++v) offs[size_t(v)] = b->h_toff[size_t(v)];
    int64_t tiles = 0;
    for (int32_t k = 0; k < nvar; ++k) {
        const int32_t v = order[size_t(k)];
        offs[size_t(nvar) + 1 + size_t(k)] = tiles;
        offs[2 * (size_t(nvar) + 1) + size_t(k)] = v;
        tiles += (poff[v + 1] - poff[v] + 32 * fold - 1) / (32 * fold);
    }
    offs[2 * (size_t(nvar) + 1) - 1] = tiles;
    TP_CUDA(cudaMemcpyAsync(b->toff, offs.data(), offs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    TP_CUDA(cudaMemcpyAsync(b->beti_v, beti, size_t(nvar) * sizeof(double), cudaMemcpyHostToDevice, s));
    TP_CUDA(cudaMemcpyAsync(b->poff, poff, (size_t(nvar) + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    int bps = 0;
    int oerr = track_occupancy(build, block, lc.minb, 0, &bps);
    if (oerr != 0 || bps <= 0) bps = 1;
    int grid = int(std::min<int64_t>(int64_t(c->sm_count) * bps, (tiles * 32 + block - 1) / block));
    grid = std::max(grid, 1);
    int sg = grid_for(n, 256, c->sm_count);

    // `timed`: record the kernel events inside the sequence (not during graph
    // capture: a captured event record does not time; the graph launch is
    // bracketed by the events instead).
    auto enqueue = [&](cudaStream_t q, bool timed) -> int {
        TP_CUDA(cudaMemsetAsync(c->counters, 0, 8 * sizeof(unsigned long long), q));
        TP_CUDA(cudaMemsetAsync(c->err, 0, 4 * sizeof(int32_t), q));
        TP_CUDA(cudaMemsetAsync(c->flops_acc, 0, 2 * sizeof(double), q));
        if (a.refill) TP_CUDA(cudaMemsetAsync(b->pool, 0, size_t(nvar) * sizeof(unsigned long long), q));
        if (!(dev && lost_turn)) k_fill_i32<<<sg, 256, 0, q>>>(d_lt, n, -1);
        if (!(dev && lost_elem)) k_fill_i32<<<sg, 256, 0, q>>>(d_le, n, -1);
        k_alive_mask<<<sg, 256, 0, q>>>(d_lost, n, c->alive0, c->counters + 2);
        TP_CUDA(cudaGetLastError());
        if (timed) TP_CUDA(cudaEventRecord(c->ev0, q));
        int le = track_launch(build, a, grid, block, lc.minb, 0, q);
        if (le != 0) return cuda_err(cudaError_t(le), "batched track kernel launch");
        if (timed) TP_CUDA(cudaEventRecord(c->ev1, q));
        k_work_stats<<<sg, 256, 0, q>>>(c->alive0, d_lost, d_lt, d_le, n, d_pre, b->poff, d_pre_off, b->nelem_v, nvar,
                                        0, nturns, turn0, c->counters + 3, c->flops_acc, c->counters + 1);
        TP_CUDA(cudaGetLastError());
        return TP_OK;
    };
    if (use_graph) {
        // The graph bakes in every value the sequence reads on the host: the
        // kernels' arguments (the context's counters, error word, FLOP
        // accumulator and alive mask; the coordinate, flag and loss-record
        // arrays; the batch's tables), which of the fill kernels run, and the
        // launch shapes.  Any change rebuilds it.
        auto u = [](const void* p) { return uint64_t(reinterpret_cast<uintptr_t>(p)); };
        auto dbits = [](double x) { uint64_t r; std::memcpy(&r, &x, sizeof r); return r; };
        std::vector<uint64_t> key = {
            u(c), u(c->counters), u(c->err), u(c->flops_acc), u(c->alive0), uint64_t(c->cap),
            u(d_coords), u(d_lost), u(d_lt), u(d_le), uint64_t(dev && lost_turn), uint64_t(dev && lost_elem),
            u(b->table), u(b->toff), u(b->poff), u(b->beti_v), u(b->nelem_v), u(b->mis), u(b->sched),
            u(b->sched_v), u(b->pool), u(b->prefix), u(b->prefix_off), u(d_pre),
            uint64_t(uint32_t(nturns)), uint64_t(uint32_t(turn0)), uint64_t(exact), uint64_t(build),
            uint64_t(a.refill), uint64_t(a.rare), dbits(a.limx), dbits(a.limy), dbits(a.beti),
            uint64_t(block), uint64_t(grid), uint64_t(sg), uint64_t(n), uint64_t(lc.minb), uint64_t(fold)};
        for (int32_t v = 0; v <= nvar; ++v) key.push_back(uint64_t(poff[v]));
        if (!b->graph || b->g_key != key) {
            if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
            b->g_key.clear();
            cudaStream_t cap = nullptr;
            TP_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            TP_CUDA(cudaStreamSynchronize(s));
            TP_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            int est = enqueue(cap, false);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(cap, &graph);
            cudaStreamDestroy(cap);
            if (est != TP_OK) { if (graph) cudaGraphDestroy(graph); return est; }
            if (ce != cudaSuccess) return cuda_err(ce, "cudaStreamEndCapture");
            ce = cudaGraphInstantiate(&b->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) { b->graph = nullptr; return cuda_err(ce, "cudaGraphInstantiate"); }
            b->g_key.swap(key);
        }
        TP_CUDA(cudaEventRecord(c->ev0, s));
        TP_CUDA(cudaGraphLaunch(b->graph, s));
        TP_CUDA(cudaEventRecord(c->ev1, s));
    } else {
        st = enqueue(s, true);
        if (st != TP_OK) return st;
    }
    if (!dev) {
        TP_CUDA(cudaMemcpyAsync(coords, d_coords, size_t(n) * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
        TP_CUDA(cudaMemcpyAsync(lost_flags, d_lost, size_t(n) * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        d2h += n * 56;
        if (lost_turn) { TP_CUDA(cudaMemcpyAsync(lost_turn, d_lt, size_t(n) * 4, cudaMemcpyDeviceToHost, s)); d2h += n * 4; }
        if (lost_elem) { TP_CUDA(cudaMemcpyAsync(lost_elem, d_le, size_t(n) * 4, cudaMemcpyDeviceToHost, s)); d2h += n * 4; }
    }
    unsigned long long cnt[4];
    double fl[2];
    TP_CUDA(cudaMemcpyAsync(cnt, c->counters, sizeof cnt, cudaMemcpyDeviceToHost, s));
    TP_CUDA(cudaMemcpyAsync(fl, c->flops_acc, sizeof fl, cudaMemcpyDeviceToHost, s));
    TP_CUDA(cudaStreamSynchronize(s));
    st = check_device_error(c);
    if (st != TP_OK) return st;
    float ms = 0.f;
    TP_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    if (tuning) tune_record(b->tune, tkey, lc, ms);
    tp_stats& S = c->stats;
    S.particles = int64_t(cnt[2]);
    S.survivors = int64_t(cnt[3]);
    S.element_passes = int64_t(cnt[1]);
    S.units = fl[1];  // alive-at-start x elements x turns, summed per variant
    S.flops = fl[0];
    S.kernel_ms = ms;
    S.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    S.h2d_bytes = h2d;
    S.d2h_bytes = d2h;
    S.block_size = block;
    S.min_blocks = track_minb(build, lc.minb);
    S.grid = grid;
    S.launches = 3 + ((dev && lost_turn) ? 0 : 1) + ((dev && lost_elem) ? 0 : 1);
    S.schedule = schedule;
    S.fp_contract = strict ? 0 : 1;
    S.refill_fold = fold;
    S.bounds_check = build == TB_CHECKED ? 1 : 0;
    return TP_OK;
}

// ---------------------------------------------------------------------------
// Adjoint and Jacobian entry points are implemented in tp_adjoint.cu.
// ---------------------------------------------------------------------------

TP_API int tp_probe_fp64_peak(tp_ctx* c, double* tflops_out) {
    if (!c || !tflops_out) return set_err(TP_EINVAL, "null argument");
    TP_CUDA(cudaSetDevice(c->device));
    double* out = nullptr;
    TP_CUDA(cudaMalloc(&out, sizeof(double)));
    const int block = 256, grid = c->sm_count * 8, iters = 1 << 12;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        TP_CUDA(cudaEventRecord(c->ev0, c->stream));
        k_fp64_probe<<<grid, block, 0, c->stream>>>(out, iters, 0.999999, 1e-7);
        TP_CUDA(cudaEventRecord(c->ev1, c->stream));
        TP_CUDA(cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        TP_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        double flops = 2.0 * 8.0 * double(iters) * double(grid) * double(block);
        if (rep > 0) best = std::max(best, flops / (double(ms) * 1e-3) / 1e12);
    }
    cudaFree(out);
    *tflops_out = best;
    return TP_OK;
}

}  // extern "C"

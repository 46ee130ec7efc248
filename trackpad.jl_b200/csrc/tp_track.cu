// tp_track.cu -- the tracking kernel (ringpass!/linepass! on the device).
//
// One thread per particle; the 6D FP64 state stays in registers across every
// element and turn of the launch.  Every lane of a warp reads the same word of
// the compiled element table at the same time (a broadcast); by default the
// table is read through the L1 cache, where it stays resident.  On request
// (TrackArgs::smem_words > 0) each block first stages it into shared memory
// with a bulk copy (cp.async.bulk, no multicast) completed on an mbarrier.
// Particles are read and written in coalesced SoA order (column c of the N x 6
// column-major array).
//
// Scheduling.  With lane refill a persistent warp takes particle indices from
// a global counter (one warp-aggregated atomic per refill); a lane whose
// particle is lost or finished takes the next particle at the next turn
// boundary, so loss does not leave lanes idle for the rest of the launch.
// Every particle is still tracked from turn 0 with its own turn counter, so
// the result is the same as the reference's loop order.  Static scheduling
// gives each thread one particle.  Batched launches hand out 32-particle
// tiles of (variant, particles) and read each variant's table through L1.
//
// This file is compiled three times: with FMA contraction (TP_NS = fast),
// without (-fmad=false, TP_NS = strict, bit-identical arithmetic to the
// oracle), and without contraction with bounds checks (TP_NS = checked,
// TP_BOUNDS_CHECK: every element-table record must lie inside its table or
// turn block and every particle index below N, else the kernel sets DE_BOUNDS
// in the error word and stops the warp's work instead of reading out of
// bounds).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tp_internal.h"
#include "tp_maps.cuh"

#ifndef TP_NS
#define TP_NS fast
#endif

namespace tp {
namespace TP_NS {

using namespace tp::dev;

// 128-thread blocks (64- and 256-thread blocks measured slower).
#ifndef TP_MAX_BLOCK
#define TP_MAX_BLOCK 128
#endif
// Resident 128-thread blocks per SM the register allocation is sized for
// (MINB, a template parameter of the kernels): 8 gives 64 registers and 32
// warps per SM, 7 gives 72 registers and 28 warps, 6 gives 80 registers, 5
// gives 96.  Fewer registers spill more, more warps hide more latency; which
// wins depends on the lattice, the schedule and the code (8 blocks beat 7 on
// the DBA step by 1.5 % and lost by 4-7 % on the 256-variant batch), so the
// build that runs the reference's operation order carries 5, 6, 7 and 8 for
// the integrator-core kernels (in two units, see carried_minb) and the host
// picks one by timing.
constexpr int kMinBlocksDefault = 7;
constexpr int kMaxBlock = TP_MAX_BLOCK;
constexpr long long kTmaSpinLimit = 1ll << 22;  // bounded mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Stage `words` words of the element table into shared memory with
// cp.async.bulk (global -> shared::cluster, which for a launch without
// clusters is this CTA's own shared memory) completed on an mbarrier.
// Returns false if the bounded wait ran out.
__device__ bool stage_table(double* dst, const double* src, int words, uint64_t* mbar) {
    const uint32_t bar = smem_u32(mbar);
    const uint32_t bytes = uint32_t(words) * 8u;  // multiple of 16: the host pads the table
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        const uint32_t chunk = 32768u;
        for (uint32_t off = 0; off < bytes; off += chunk) {
            uint32_t n = bytes - off < chunk ? bytes - off : chunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32(reinterpret_cast<char*>(dst) + off)),
                "l"(reinterpret_cast<const char*>(src) + off), "r"(n), "r"(bar)
                : "memory");
        }
    }
    uint32_t done = 0;
    long long spins = 0;
    while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(0u)
            : "memory");
        if (++spins > kTmaSpinLimit) break;
    }
    __syncthreads();
    return done != 0;
}

__device__ __forceinline__ void load_state(const double* coords, int64_t n, int64_t i, P6& s) {
    s.x = coords[i];
    s.px = coords[n + i];
    s.y = coords[2 * n + i];
    s.py = coords[3 * n + i];
    s.z = coords[4 * n + i];
    s.d = coords[5 * n + i];
}

__device__ __forceinline__ void store_state(double* coords, int64_t n, int64_t i, const P6& s) {
    coords[i] = s.x;
    coords[n + i] = s.px;
    coords[2 * n + i] = s.y;
    coords[3 * n + i] = s.py;
    coords[4 * n + i] = s.z;
    coords[5 * n + i] = s.d;
}

// check_lost (src/tracking.jl:49-52) fused with the rectangular aperture:
// |x| > 1 or |x| > ax  <=>  |x| > min(1, ax).
__device__ __forceinline__ bool is_lost(const P6& s, double limx, double limy) {
    return isnan(s.x) || fabs(s.x) > limx || fabs(s.y) > limy || fabs(s.px) > 1.0 || fabs(s.py) > 1.0;
}

// The per-turn table of a lattice's scheduled elements.
struct SchedView {
    const double* p;
    int32_t stride, turn0, nturns;
};

// Header of the record to use at `turn` (scheduled elements live in the
// per-turn table).  Returns null when the turn is outside the schedule (and,
// in the bounds-checked build, when the record does not fit its turn block,
// with DE_BOUNDS set).
__device__ __forceinline__ const double* resolve(const double* rec, RecHdr& h, const SchedView& sv, int turn,
                                                 int32_t* err) {
    (void)err;
    if (!(h.flags & RF_SCHEDULED)) return rec;
    int row = turn - sv.turn0;
    if (row < 0 || row >= sv.nturns) return nullptr;
    const int32_t slot = h.aux;
#ifdef TP_BOUNDS_CHECK
    if (slot < 0 || slot + HDR_WORDS > sv.stride) {
        atomicOr(err, DE_BOUNDS);
        return nullptr;
    }
#endif
    const double* p = sv.p + int64_t(row) * sv.stride + slot;
    h = *reinterpret_cast<const RecHdr*>(p);
#ifdef TP_BOUNDS_CHECK
    if (h.words < HDR_WORDS || slot + int32_t(h.words) > sv.stride) {
        atomicOr(err, DE_BOUNDS);
        return nullptr;
    }
#endif
    return p;
}

#ifdef TP_BOUNDS_CHECK
// The walk over the element table left the table (a corrupt record length):
// report it and end this warp's work (the condition is warp-uniform).
__device__ __forceinline__ void table_overrun(const TrackArgs& a, bool& act, bool& more) {
    if ((threadIdx.x & 31) == 0) atomicOr(a.err, DE_BOUNDS);
    act = false;
    more = false;
}
#endif

// Track the particles of one warp through `nturns` turns of the table `tab`
// (`nelem` records).  Slot state is per lane.  With REFILL, lanes take new
// particles from `next_particle` at turn boundaries until it returns < 0.
template <bool EXACT, bool REFILL, bool RARE, typename NextFn>
__device__ void run_warp(const TrackArgs& a, const double* tab, const double* tab_end, int nelem, double beti,
                         const SchedView& sv, NextFn next_particle) {
    (void)tab_end;  // read by the bounds-checked build only
    const double beta = 1.0 / beti;
    const double beta2 = beta * beta;
    const int lane = threadIdx.x & 31;
    P6 s{};
    int64_t idx = -1;
    int t = 0;
    bool act = false;
    bool more = true;  // warp-uniform: the particle source is not exhausted

    for (;;) {
        // Refill empty lanes at the turn boundary.
        while (more) {
            unsigned need = __ballot_sync(0xffffffffu, !act);
            if (need == 0) break;
            int64_t j = next_particle(need, lane, more);
#ifdef TP_BOUNDS_CHECK
            if (j >= a.n) {
                atomicOr(a.err, DE_BOUNDS);
                j = -1;
            }
#endif
            if (!act && j >= 0) {
                if (a.lost_flags[j] != 1) {
                    load_state(a.coords, a.n, j, s);
                    idx = j;
                    t = 0;
                    act = true;
                }
            }
            if (!REFILL) more = false;
        }
        if (__ballot_sync(0xffffffffu, act) == 0) {
            if (!more) break;
            continue;
        }
        // One turn.
        const double* rec = tab;
        for (int e = 0; e < nelem; ++e) {
#ifdef TP_BOUNDS_CHECK
            if (rec + HDR_WORDS > tab_end) {
                table_overrun(a, act, more);
                break;
            }
#endif
            RecHdr h0 = *reinterpret_cast<const RecHdr*>(rec);
            const double* next = rec + h0.words;
#ifdef TP_BOUNDS_CHECK
            if (h0.words < HDR_WORDS || next > tab_end) {
                table_overrun(a, act, more);
                break;
            }
#endif
            // Every lane of this warp empty: skip the rest of the turn.  (The vote
            // at every element also reconverges the warp after divergent maps;
            // voting every 16 elements measured 4% slower on the DBA ring.)
            if (__ballot_sync(0xffffffffu, act) == 0) break;
            if (act) {
                RecHdr h = h0;
                const double* r = resolve(rec, h, sv, a.turn0 + t, a.err);
                if (r == nullptr) {
                    atomicOr(a.err, DE_SCHED_RANGE);
                    act = false;
                } else {
                    P6 sn = s;
                    if (!apply_record<EXACT, RARE>(sn, r, h, a.mis, beti, beta, beta2)) {
                        atomicOr(a.err, DE_BAD_KIND);
                        act = false;
                    } else if (is_lost(sn, a.limx, a.limy)) {
                        // linepass!: flag the particle, keep the entrance coordinates
                        // (src/lattice.jl:281-284).
                        store_state(a.coords, a.n, idx, s);
                        a.lost_flags[idx] = 1;
                        if (a.lost_turn) a.lost_turn[idx] = a.turn0 + t;
                        if (a.lost_elem) a.lost_elem[idx] = e;
                        act = false;
                    } else {
                        s = sn;
                    }
                }
            }
            rec = next;
        }
        if (act) {
            ++t;
            if (t == a.nturns) {
                store_state(a.coords, a.n, idx, s);
                act = false;
            }
        }
    }
}

template <bool EXACT, bool REFILL, bool RARE, int MINB>
__global__ void __launch_bounds__(kMaxBlock, MINB) track_single(TrackArgs a) {
    extern __shared__ __align__(16) double smem[];
    __shared__ __align__(8) uint64_t mbar;
    const double* tab = a.table;
    const SchedView sv{a.sched, a.sched_stride, a.sched_turn0, a.sched_nturns};
    if (a.smem_words > 0) {
        if (!stage_table(smem, a.table, a.smem_words, &mbar)) {
            if (threadIdx.x == 0) atomicOr(a.err, DE_TMA_TIMEOUT);
            return;
        }
        tab = smem;
    }
    if (REFILL) {
        auto next = [&](unsigned need, int lane, bool& more) -> int64_t {
            unsigned long long base = 0;
            int cnt = __popc(need);
            if (lane == 0) base = atomicAdd(a.work, (unsigned long long)cnt);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + (unsigned long long)cnt >= (unsigned long long)a.n) more = false;
            if (!((need >> lane) & 1u)) return -1;
            unsigned long long j = base + __popc(need & ((1u << lane) - 1u));
            return j < (unsigned long long)a.n ? int64_t(j) : -1;
        };
        run_warp<EXACT, true, RARE>(a, tab, tab + a.table_words, a.nelem, a.beti, sv, next);
    } else {
        const int64_t gid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
        auto next = [&](unsigned need, int lane, bool& more) -> int64_t {
            more = false;
            return gid < a.n ? gid : -1;
        };
        run_warp<EXACT, false, RARE>(a, tab, tab + a.table_words, a.nelem, a.beti, sv, next);
    }
}

// Batched: warps take 32-particle tiles (variant, first particle) in the
// host's hand-out order (variants with the most elements first); tile t of the
// k-th variant v = order[k] covers particles poff[v] + 32*(t - tile_off[k]).
// Static (REFILL false): the warp tracks exactly its tile's particles.  Pooled
// refill (REFILL true): a warp that takes a tile of variant v draws particles
// of v from the variant's pool counter (pool[v], zeroed by the host) and
// refills lanes freed by a loss at turn boundaries until the pool is empty;
// later tiles of an emptied variant end at once.  Either way every particle is
// tracked from turn 0 with its own turn counter, so the results are the same.
template <bool EXACT, bool REFILL, bool RARE, int MINB>
__global__ void __launch_bounds__(kMaxBlock, MINB) track_batched(TrackArgs a, const int64_t* tile_off) {
    const int lane = threadIdx.x & 31;
    const int64_t ntiles = tile_off[a.nvar];
    for (;;) {
        unsigned long long tile = 0;
        if (lane == 0) tile = atomicAdd(a.work, 1ull);
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (tile >= (unsigned long long)ntiles) break;
        // position k of this tile's variant in the hand-out order (last k with
        // tile_off[k] <= tile), and the variant itself
        int lo = 0, hi = a.nvar - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (tile_off[mid] <= (int64_t)tile) lo = mid; else hi = mid - 1;
        }
        const int v = int(tile_off[a.nvar + 1 + lo]);
        const int64_t p0 = a.poff[v];
        const int64_t endp = a.poff[v + 1];
        const int64_t mine = p0 + 32 * (int64_t(tile) - tile_off[lo]) + lane;
        const unsigned long long nv = (unsigned long long)(endp - p0);
        auto next = [&](unsigned need, int ln, bool& more) -> int64_t {
            if (!REFILL) {
                more = false;
                return mine < endp ? mine : -1;
            }
            unsigned long long base = 0;
            const int cnt = __popc(need);
            if (ln == 0) base = atomicAdd(a.pool + v, (unsigned long long)cnt);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + (unsigned long long)cnt >= nv) more = false;
            if (!((need >> ln) & 1u)) return -1;
            const unsigned long long j = base + __popc(need & ((1u << ln) - 1u));
            return j < nv ? p0 + int64_t(j) : -1;
        };
        // this variant's per-turn schedule (none: no record of the variant is scheduled)
        SchedView sv{nullptr, 0, 0, 0};
        if (a.sched_v != nullptr && a.sched_v[4 * v] >= 0) {
            sv.p = a.sched + a.sched_v[4 * v];
            sv.stride = int32_t(a.sched_v[4 * v + 1]);
            sv.turn0 = int32_t(a.sched_v[4 * v + 2]);
            sv.nturns = int32_t(a.sched_v[4 * v + 3]);
        }
        run_warp<EXACT, REFILL, RARE>(a, a.table + a.toff[v], a.table + a.toff[v + 1], a.nelem_v[v], a.beti_v[v], sv,
                                      next);
    }
}

// The kernel instance of (exact drift, refill, rare kinds, resident blocks)
// chosen at run time.
template <bool EXACT, bool REFILL, bool RARE, int MINB>
int launch_t(const TrackArgs& a, int grid, int block, size_t smem, cudaStream_t st) {
    if (a.nvar > 0) {
        const int64_t* tile_off = a.toff + (a.nvar + 1);  // host packs tile offsets and the order after toff
        track_batched<EXACT, REFILL, RARE, MINB><<<grid, block, 0, st>>>(a, tile_off);
        return int(cudaGetLastError());
    }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(track_single<EXACT, REFILL, RARE, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return int(e);
    }
    track_single<EXACT, REFILL, RARE, MINB><<<grid, block, smem, st>>>(a);
    return int(cudaGetLastError());
}

// Resident-block counts this translation unit carries.  The build without
// contraction is split in two units that compile in parallel: TP_OCC_VARIANTS
// carries the default 7 (every kind) and 8 (integrator core), TP_OCC_LOW
// carries 5 and 6 (integrator core) and nothing else; the other builds carry
// the default only.  carried_minb returns 0 for a count the unit does not hold.
int carried_minb(int minb) {
#if defined(TP_OCC_LOW)
    return (minb == 5 || minb == 6) ? minb : 0;
#elif defined(TP_OCC_VARIANTS)
    return minb == 8 ? 8 : kMinBlocksDefault;
#else
    (void)minb;
    return kMinBlocksDefault;
#endif
}

template <bool EXACT, bool REFILL>
int launch_r(const TrackArgs& a, int grid, int block, int minb, size_t smem, cudaStream_t st) {
#if defined(TP_OCC_LOW)
    if (a.rare) return int(cudaErrorInvalidValue);  // tables with rare kinds run the default instance
    if (minb == 5) return launch_t<EXACT, REFILL, false, 5>(a, grid, block, smem, st);
    if (minb == 6) return launch_t<EXACT, REFILL, false, 6>(a, grid, block, smem, st);
    return int(cudaErrorInvalidValue);
#else
    if (a.rare) return launch_t<EXACT, REFILL, true, kMinBlocksDefault>(a, grid, block, smem, st);
#if defined(TP_OCC_VARIANTS)
    if (minb == 8) return launch_t<EXACT, REFILL, false, 8>(a, grid, block, smem, st);
#endif
    (void)minb;
    return launch_t<EXACT, REFILL, false, kMinBlocksDefault>(a, grid, block, smem, st);
#endif
}

int launch(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    minb = carried_minb(minb);
    if (a.nvar > 0) smem = 0;
    if (a.exact && a.refill) return launch_r<true, true>(a, grid, block, minb, smem, st);
    if (a.exact) return launch_r<true, false>(a, grid, block, minb, smem, st);
    if (a.refill) return launch_r<false, true>(a, grid, block, minb, smem, st);
    return launch_r<false, false>(a, grid, block, minb, smem, st);
}

template <int MINB>
int occupancy_t(int block, size_t smem, int* blocks_per_sm) {
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(track_single<true, true, false, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return int(e);
    }
    return int(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, track_single<true, true, false, MINB>,
                                                             block, smem));
}

int occupancy(int block, int minb, size_t smem, int* blocks_per_sm) {
    minb = carried_minb(minb);
#if defined(TP_OCC_LOW)
    if (minb == 5) return occupancy_t<5>(block, smem, blocks_per_sm);
    if (minb == 6) return occupancy_t<6>(block, smem, blocks_per_sm);
    return int(cudaErrorInvalidValue);
#else
#if defined(TP_OCC_VARIANTS)
    if (minb == 8) return occupancy_t<8>(block, smem, blocks_per_sm);
#endif
    return occupancy_t<kMinBlocksDefault>(block, smem, blocks_per_sm);
#endif
}

}  // namespace TP_NS

#define TP_CAT2(a, b) a##_##b
#define TP_CAT(a, b) TP_CAT2(a, b)
int TP_CAT(launch_track, TP_NS)(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream) {
    return TP_NS::launch(a, grid, block, minb, smem, stream);
}
int TP_CAT(occupancy_track, TP_NS)(int block, int minb, size_t smem, int* blocks_per_sm) {
    return TP_NS::occupancy(block, minb, smem, blocks_per_sm);
}
int TP_CAT(minb_track, TP_NS)(int minb) { return TP_NS::carried_minb(minb); }

}  // namespace tp

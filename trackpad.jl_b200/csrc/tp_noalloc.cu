// tp_noalloc.cu -- ringpass without any device allocation.
//
// Some callers cannot let a library allocate device memory: a Julia or
// PyTorch program whose memory pool owns the whole device, a real-time loop
// where allocation is forbidden after start-up, or code that must not call
// cudaMalloc/cudaFree while other work is in flight on the device (both can
// synchronise the device).  tp_ringpass_noalloc serves them: it runs the same
// tracking kernel as tp_ringpass, but its scratch memory -- the lane-refill
// work counter, the pass counter, the device error word and the compiled
// element table -- lives in the file-scope array below, which the CUDA module
// loader places in device memory when the library's device code is loaded on
// a device.  The entry point itself calls no cudaMalloc, cudaFree or other
// allocating routine.
//
// Limits and rules:
//   * the array holds at most kNoAllocTableWords (16384) words of element
//     table, 128 KiB; lattices with misalignment rows or a per-turn schedule
//     are not accepted (they need further device tables);
//   * every GPU that loads the library holds the array (about 128 KiB) until
//     the process exits;
//   * every call shares the array: the counters and the error word are cleared
//     at the start of each call, and the table is overwritten whenever the
//     call's lattice (or its program) differs from the one the array holds on
//     that device, so calls that overlap on the GPU race with each other;
//   * the kernel reads the table from the array through the L1 cache (every
//     lane of a warp reads the same record word), as tp_ringpass does;
//   * the first call on a device looks up the array's device address there
//     (cudaGetSymbolAddress); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "tp_internal.h"

namespace {

constexpr int kNoAllocTableWords = 16384;
constexpr int kHeadWords = 32;  // counters and error word; the table starts 256 bytes in
constexpr int kScratchWords = kHeadWords + kNoAllocTableWords;
constexpr int kMaxDev = 16;

// The allocation-free scratch: words [0, 4) counters (work, passes), [4, 8)
// error word, [32, 32 + 16384) element table (256-byte aligned).
static __device__ __align__(256) double g_noalloc_scratch[kScratchWords];

std::mutex g_mu;                      // serialises the set-up of the calls of this process
double* g_scratch_dev[kMaxDev] = {};  // device address of the array on each device
uint64_t g_resident[kMaxDev] = {};    // lattice stamp whose table the array holds (0: none)

int fail(int st, const std::string& msg) {
    tp::set_last_error(msg);
    return st;
}

int cuda_fail(cudaError_t e, const char* what) { return fail(TP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)); }

}  // namespace

extern "C" {

TP_API int tp_ringpass_noalloc(const tp_lattice* lat, double* coords, int64_t n, int64_t* lost_flags,
                               int32_t* lost_turn, int32_t* lost_elem, double beti, int32_t nturns, int32_t turn0,
                               double aperture_x, double aperture_y, void* stream) {
    if (!lat) return fail(TP_EINVAL, "lattice is null");
    if (n < 0 || nturns < 0) return fail(TP_EINVAL, "negative particle count or number of turns");
    if (!(beti > 0.0) || !std::isfinite(beti)) return fail(TP_EINVAL, "beti must be finite and positive");
    if (n > 0 && (!coords || !lost_flags)) return fail(TP_EINVAL, "coords and lost_flags are required");
    // The lattice's program may be rebuilt by tp_lattice_set_schedule: hold
    // its lock while the program is read and copied.
    std::unique_lock<std::mutex> lat_lock(tp::lattice_mutex(lat));
    tp::LatticeView v;
    tp::lattice_view(lat, &v);
    if (v.has_schedule || v.has_misalignment)
        return fail(TP_EUNSUPPORTED, "the allocation-free entry point takes lattices without schedules or misalignment");
    if (v.words > size_t(kNoAllocTableWords))
        return fail(TP_ERANGE, "element table of " + std::to_string(v.words) + " words exceeds the allocation-free limit of " +
                                   std::to_string(kNoAllocTableWords) + " words (128 KiB)");
    if (n == 0 || nturns == 0) return TP_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDev) return fail(TP_EINVAL, "device ordinal out of range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scratch = nullptr;
    std::unique_lock<std::mutex> g(g_mu);
    if (!g_scratch_dev[dev]) {
        // Once per device, with that device current: the array's device address.
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
    int sm = 0;
    e = cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");

    // Clear what must start at zero; copy the table unless this lattice's
    // current program is the one the array already holds on this device.
    e = cudaMemsetAsync(scratch, 0, kHeadWords * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "scratch set-up");
    if (g_resident[dev] != v.stamp) {
        g_resident[dev] = 0;
        e = cudaMemcpyAsync(scratch + kHeadWords, v.program, v.words * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "element table copy");
        g_resident[dev] = v.stamp;
    }
    const bool rare = tp::records_have_rare(v.program, v.words);
    g.unlock();
    lat_lock.unlock();

    tp::TrackArgs a{};
    a.table = scratch + kHeadWords;
    a.table_words = int32_t(v.words);
    a.nelem = v.nelem;
    a.rare = rare ? 1 : 0;
    a.coords = coords;
    a.n = n;
    a.lost_flags = lost_flags;
    a.lost_turn = lost_turn;
    a.lost_elem = lost_elem;
    a.beti = beti;
    a.limx = aperture_x > 0.0 ? std::fmin(1.0, aperture_x) : 1.0;
    a.limy = aperture_y > 0.0 ? std::fmin(1.0, aperture_y) : 1.0;
    a.nturns = nturns;
    a.turn0 = turn0;
    a.exact = 1;
    a.refill = nturns > 1 ? 1 : 0;
    a.work = reinterpret_cast<unsigned long long*>(scratch);
    a.passes = reinterpret_cast<unsigned long long*>(scratch) + 1;
    a.err = reinterpret_cast<int32_t*>(scratch + 4);
    a.smem_words = 0;  // the table is read through the L1 cache, as tp_ringpass does by default
    const size_t smem = 0;
    const int block = 128;
    int bps = 0;
    if (tp::occupancy_track_strict(block, 0, smem, &bps) != 0 || bps <= 0) bps = 1;
    const int64_t needed = (n + block - 1) / block;
    int grid = a.refill ? int(std::min<int64_t>(int64_t(sm) * bps, needed)) : int(needed);
    if (grid < 1) grid = 1;
    int le = tp::launch_track_strict(a, grid, block, 0, smem, s);
    if (le != 0) return cuda_fail(cudaError_t(le), "track kernel launch");
    int32_t err = 0;
    e = cudaMemcpyAsync(&err, a.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "tp_ringpass_noalloc");
    if (err & tp::DE_BAD_KIND) return fail(TP_EUNSUPPORTED, "kernel met an unknown element record");
    if (err & tp::DE_TMA_TIMEOUT) return fail(TP_ETIMEOUT, "element-table staging wait ran out");
    if (err) return fail(TP_EDEVICE, "device error word set");
    return TP_OK;
}

}  // extern "C"

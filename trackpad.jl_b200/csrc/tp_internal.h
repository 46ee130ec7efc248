// tp_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/trackpad_b200.h"
#include "tp_program.h"

namespace tp {

// Array fields of the elements (the `aux` argument of tp_lattice_create_ex).
struct AuxView {
    const double* p = nullptr;
    int64_t n = 0;
};

// Host compiler (tp_compile.cpp)
int validate_elem(const tp_elem& e, int64_t idx, int64_t nmis, std::string* err, const AuxView& aux = AuxView{});
void compile_record(const tp_elem& e, std::vector<double>* out, const AuxView& aux = AuxView{});
int record_words(const tp_elem& e, const AuxView& aux = AuxView{});
void scheduled_stub(const tp_elem& e, int32_t slot, std::vector<double>* out, const AuxView& aux = AuxView{});
void apply_field(tp_elem* e, int field, double v);
double elem_flops(const tp_elem& e, const tp_misalign* mis, bool exact, const AuxView& aux = AuxView{});

// Arguments of one tracking launch.  All pointers are device pointers.
struct TrackArgs {
    const double* table;        // compiled program, `table_words` words (16-byte multiple)
    int32_t table_words;
    int32_t nelem;
    const double* sched;        // per-turn records of scheduled elements (may be null)
    int32_t sched_stride;       // words per turn block
    int32_t sched_turn0;
    int32_t sched_nturns;
    int32_t rare;               // the table holds kinds outside the integrator core (kind > DK_RF)
    const MisalignDev* mis;
    double* coords;             // N x 6 column-major
    int64_t n;
    int64_t* lost_flags;
    int32_t* lost_turn;         // may be null
    int32_t* lost_elem;         // may be null
    double beti;
    double limx, limy;          // loss limits on |x|, |y|: min(1, aperture)
    int32_t nturns;
    int32_t turn0;
    int32_t exact;              // exact Hamiltonian drift
    int32_t refill;             // lane-refill scheduling
    unsigned long long* work;   // refill counter (scratch, zeroed by the host)
    unsigned long long* passes; // unused by the kernels (element passes are derived from the loss records)
    int32_t* err;               // device error word (scratch, zeroed)
    // Batched (ragged) launches: variant v owns particles [poff[v], poff[v+1])
    // and program words [toff[v], toff[v+1]).  nvar == 0 for single lattices.
    const int64_t* poff;
    const int64_t* toff;
    const double* beti_v;
    const int32_t* nelem_v;
    const int64_t* sched_v;     // batched: per variant word offset into `sched` (-1: none), stride, first turn, turns
    unsigned long long* pool;   // batched with refill: per variant count of particles handed out (zeroed)
    int32_t nvar;
    int32_t smem_words;         // words staged into shared memory per block
};

// Device error word bits.
enum DevErr : int32_t {
    DE_BAD_KIND = 1,
    DE_SCHED_RANGE = 2,
    DE_TMA_TIMEOUT = 4,
    DE_BOUNDS = 8,        // bounds-checked build: a table record or particle index out of range
};

// True when a record of `words` words of records (a compiled table) has a
// kind outside the integrator core; the tracking kernels without the rare
// kinds' dispatch run every other table (tp_compile.cpp).
bool records_have_rare(const double* recs, size_t words);

// Kernel launchers (tp_track.cu, compiled once with and once without FMA
// contraction).  Return a cudaError_t value.  `minb` selects the kernel
// instance whose registers are sized for that many resident 128-thread blocks
// per SM (5, 6, 7 or 8 in the build without contraction, 7 in the other; tables
// with kinds outside the integrator core always run 7); minb_track_* maps a
// request to the instance that runs.
constexpr int kTrackMaxBlock = 128;  // launch bound of the tracking kernels
int launch_track_fast(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream);
int launch_track_strict(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream);
int occupancy_track_fast(int block, int minb, size_t smem, int* blocks_per_sm);
int occupancy_track_strict(int block, int minb, size_t smem, int* blocks_per_sm);
int minb_track_fast(int minb);
int minb_track_strict(int minb);
// The instances sized for 5 and 6 resident blocks of the build without
// contraction (a second unit of that build; minb_track_strict_low returns 0 for
// counts it does not hold).
int launch_track_strict_low(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream);
int occupancy_track_strict_low(int block, int minb, size_t smem, int* blocks_per_sm);
int minb_track_strict_low(int minb);
// The bounds-checked build (no contraction, tp_opts.bounds_check).
int launch_track_checked(const TrackArgs& a, int grid, int block, int minb, size_t smem, void* stream);
int occupancy_track_checked(int block, int minb, size_t smem, int* blocks_per_sm);
int minb_track_checked(int minb);

// Read-only view of a lattice's compiled program (tp_runtime.cu).  The
// program may be rebuilt by tp_lattice_set_schedule: hold lattice_mutex(lat)
// while the view is used.  `stamp` is unique to this lattice and its current
// program (every creation and every rebuild draws a new one).
struct LatticeView {
    const double* program;  // host copy of the compiled table
    size_t words;
    int32_t nelem;
    bool has_schedule;
    bool has_misalignment;
    uint64_t stamp;
};
void lattice_view(const tp_lattice* lat, LatticeView* out);
std::mutex& lattice_mutex(const tp_lattice* lat);

// Everything the adjoint and Jacobian paths read from a lattice (tp_runtime.cu).
struct LatticeHost {
    const tp_elem* elems;
    int32_t nelem;
    const double* program;    // compiled table (scheduled elements are stubs)
    size_t words;
    const int32_t* rec_off;   // word offset of each element's record
    const double* sched;      // per-turn records of scheduled elements (null without schedule)
    size_t sched_words;
    int32_t sched_stride, sched_turn0, sched_nturns;
    bool has_schedule;
    int64_t nmis;
    const tp_misalign* mis;   // nmis rows
};
void lattice_host(const tp_lattice* lat, LatticeHost* out);

// Context properties and per-context device scratch (tp_runtime.cu).  Scratch
// slot `slot` grows to at least `bytes` and is kept until the context is
// destroyed.
struct CtxHost {
    int device;
    int sm_count;
    size_t smem_optin;
    void* stream;
};
void ctx_host(const tp_ctx* c, CtxHost* out);
tp_stats* ctx_stats(tp_ctx* c);
constexpr int kCtxScratchSlots = 16;
int ctx_scratch(tp_ctx* c, int slot, size_t bytes, void** out);
// The lattices of a batch in variant order.
void batch_lattices(const tp_batch* b, std::vector<const tp_lattice*>* out);

// Set the text returned by tp_last_error_string on this thread.
void set_last_error(const std::string& msg);

// A named NVTX range over one entry point (shown by Nsight Systems and by
// ncu's --nvtx filters; a no-op unless a tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char* name);
    ~NvtxRange();
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

}  // namespace tp

/*
 * trackpad_b200.h -- C ABI of the B200 multi-particle tracking engine.
 *
 * This is the drop-in boundary for TrackPad.jl's element-by-element tracking
 * path.  A Julia package extension binds these symbols with `ccall`; the
 * Python package beside this library binds them with ctypes.  Every entry
 * point takes plain pointers and sizes, returns an int status (0 = TP_OK),
 * and never throws.  There is no CPU fallback: an element kind the device
 * kernels do not implement is rejected with TP_EUNSUPPORTED when the lattice
 * is built.
 *
 * Reference interfaces replaced (paths inside TrackPad.jl):
 *   linepass!(coords, lat, beam, lost_flags; time, turn)     src/lattice.jl:260-297
 *   ringpass!(coords, lat, beam, lost_flags, nturns; ...)    src/lattice.jl:305-317
 *   pass!(elem, r, beti) for every element kind              src/tracking.jl
 *   Beam(energy; mass) / beti(beam)                           src/lattice.jl:46-61
 *   materialize / _resolve_for_time (time-varying fields)     src/time_dependence.jl:163-178
 *   one_turn_map (finite-difference 6x6 Jacobian)             src/optics.jl:110-121
 *
 * Data layout at the boundary (same as the reference's Julia arrays):
 *   coords      N x 6 Float64, column-major: column c (x, px, y, py, z, delta)
 *               is N contiguous doubles at coords + c*N (src/lattice.jl:252,274).
 *   lost_flags  N Int64, 0 = alive, 1 = lost (src/lattice.jl:255,269,282).
 *               Only the value 1 marks a particle as lost on entry, exactly as
 *               the reference tests `lost_flags[i] == 1`.
 *
 * Pointers are host memory unless tp_opts.device_pointers is set, in which
 * case they are device pointers on the context's device (e.g. CuArray or
 * torch.cuda tensors).  All calls are synchronous with respect to the host
 * unless documented otherwise.
 */
#ifndef TRACKPAD_B200_H
#define TRACKPAD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TP_API __attribute__((visibility("default")))
#else
#define TP_API
#endif

#define TP_ABI_VERSION 1

/* ------------------------------------------------------------------------- */
/* Status codes                                                               */
/* ------------------------------------------------------------------------- */
enum tp_status {
    TP_OK = 0,
    TP_EINVAL = -1,        /* bad argument (reference: ArgumentError)          */
    TP_ENOMEM = -2,        /* device or host allocation failed                 */
    TP_EUNSUPPORTED = -3,  /* element kind / option not implemented on device  */
    TP_ECUDA = -4,         /* CUDA runtime error (see tp_last_error_string)    */
    TP_ETIMEOUT = -5,      /* a bounded device wait ran out                    */
    TP_EDEVICE = -6,       /* a kernel reported an error through its error word*/
    TP_ENODEV = -7,        /* no usable CUDA device                            */
    TP_ERANGE = -8         /* size beyond a documented maximum                 */
};

/* ------------------------------------------------------------------------- */
/* Element description (one record per lattice entry)                         */
/* ------------------------------------------------------------------------- */
/* Element kinds.  Each kind names the reference struct whose fields the
 * record carries and the pass! method it follows. */
enum tp_kind {
    TP_MARKER = 0,          /* Marker          tracking.jl:139-141              */
    TP_DRIFT = 1,           /* Drift           tracking.jl:115-132              */
    TP_QUADRUPOLE = 2,      /* Quadrupole      tracking.jl:386-427              */
    TP_SEXTUPOLE = 3,       /* Sextupole       tracking.jl:438-459              */
    TP_OCTUPOLE = 4,        /* Octupole        tracking.jl:470-491              */
    TP_THIN_MULTIPOLE = 5,  /* ThinMultipole   tracking.jl:616-633              */
    TP_SBEND = 6,           /* SBend / RBend   tracking.jl:657-706              */
    TP_EXACT_SBEND = 7,     /* ExactSBend / ERBend  tracking.jl:901-973         */
    TP_RFCAVITY = 8,        /* RFCavity        tracking.jl:502-518              */
    TP_SOLENOID = 9,        /* Solenoid        tracking.jl:529-570              */
    TP_CORRECTOR = 10,      /* Corrector/HKicker/VKicker tracking.jl:579-607   */
    TP_TRANSLATION = 11,    /* Translation     tracking.jl:1182-1192            */
    TP_YROTATION = 12,      /* YRotation       tracking.jl:1194-1218            */
    TP_CRAB_CAVITY = 13,    /* CrabCavity      tracking.jl:1531-1547            */
    TP_ACCEL_CAVITY = 14,   /* AccelCavity     tracking.jl:1549-1559            */
    TP_LONGITUDINAL_RF_MAP = 15, /* LongitudinalRFMap tracking.jl:1575-1585     */
    TP_LORENTZ_BOOST = 16,  /* LorentzBoost    tracking.jl:1587-1595            */
    TP_INV_LORENTZ_BOOST = 17, /* InvLorentzBoost tracking.jl:1597-1604         */
    TP_SPACE_CHARGE = 18,   /* SpaceCharge (no-op) tracking.jl:1176-1180        */
    TP_DRIFT_SC = 19,       /* DriftSC         tracking.jl:981-991              */
    TP_QUADRUPOLE_SC = 20,  /* QuadrupoleSC    tracking.jl:997-1015             */
    TP_SEXTUPOLE_SC = 21,   /* SextupoleSC     tracking.jl:1017-1027            */
    TP_OCTUPOLE_SC = 22,    /* OctupoleSC      tracking.jl:1029-1039            */
    TP_SBEND_SC = 23,       /* SBendSC / RBendSC tracking.jl:1041-1070          */
    TP_STRONG_THIN_GAUSSIAN_BEAM = 24, /* tracking.jl:1610-1619                 */
    TP_LBEND = 25,          /* LBend           tracking.jl:1076-1170            */
    TP_WIGGLER = 26,        /* Wiggler         tracking.jl:1224-1529            */
    TP_STRONG_GAUSSIAN_BEAM = 27, /* StrongGaussianBeam tracking.jl:1621-1641   */
    TP_LONGITUDINAL_RLC_WAKE = 28, /* LongitudinalRLCWake tracking.jl:1647-1654,
                                      elements/wake.jl:27-37                    */
    TP_LONGITUDINAL_WAKE = 29,     /* LongitudinalWake tracking.jl:1656-1663,
                                      elements/wake.jl:68-91                    */
    TP_KIND_COUNT = 30
};

/* One lattice entry.  Fields use the reference struct field names; a field a
 * kind does not have is ignored.  `param`/`iparam` carry the fields of the
 * remaining kinds (see the per-kind list below). */
typedef struct tp_elem {
    int32_t kind;                 /* enum tp_kind                               */
    int32_t max_order;            /* multipole order used by the thin kicks     */
    int32_t num_int_steps;        /* Yoshida-4 steps (0 allowed for ExactSBend) */
    int32_t fringe_bend_entrance; /* SBend: edge method 0..3; ExactSBend: 0/1   */
    int32_t fringe_bend_exit;
    int32_t misalign_index;       /* -1: none; else row of the tp_misalign table*/
    int32_t iparam[2];            /* kind-specific integers                     */
    double L;                     /* length [m]                                 */
    double k;                     /* Quadrupole.k1 / Sextupole.k2 / Octupole.k3 */
    double angle, e1, e2;         /* bends                                       */
    double fint1, fint2, gap, gk; /* bend fringe                                */
    double polynom_a[4];          /* skew coefficients (reference 1-based [1..4])*/
    double polynom_b[4];          /* normal coefficients                        */
    double kick_angle[2];         /* Quadrupole/SBend/ExactSBend kick_angle     */
    double volt, freq, h, lag, philag, energy; /* RFCavity                      */
    double param[8];              /* kind-specific doubles                      */
} tp_elem;
/* Kind-specific fields:
 *   TP_SOLENOID       param[0] = ks
 *   TP_CORRECTOR      param[0] = xkick, param[1] = ykick
 *   TP_TRANSLATION    param[0] = dx, param[1] = dy, param[2] = ds
 *   TP_YROTATION      angle
 *   TP_CRAB_CAVITY    volt, freq, energy, param[0] = k, param[1] = phi,
 *                     param[2] = errors[1], param[3] = errors[2]
 *   TP_ACCEL_CAVITY   volt, freq, h, energy, param[0] = k, param[1] = phis
 *   TP_LONGITUDINAL_RF_MAP  param[0] = alphac, param[1] = k of the linked RF
 *                     element (_rf_k), param[2] = h of the linked element (_rf_h)
 *   TP_LORENTZ_BOOST / TP_INV_LORENTZ_BOOST  param[0] = angle, param[1] = cosang,
 *                     param[2] = sinang, param[3] = tanang, iparam[0] = mode
 *   TP_QUADRUPOLE_SC .. TP_OCTUPOLE_SC  param[0..3] = k0, k1, k2, k3
 *   TP_STRONG_THIN_GAUSSIAN_BEAM  param[0] = amplitude, param[1] = rmssizex,
 *                     param[2] = rmssizey, param[3] = xoffset, param[4] = yoffset
 *   TP_LBEND          L, angle, e1, e2, fint1, fint2, gap = full_gap,
 *                     param[0] = K, param[1] = by_error
 *   TP_LONGITUDINAL_RLC_WAKE  param[0] = freq, param[1] = Rshunt, param[2] = Q0,
 *                     param[3] = scale
 * Kinds with array fields read them from the `aux` array of
 * tp_lattice_create_ex: iparam[0] = word offset of the element's arrays in
 * aux, iparam[1] = their total length, laid out as
 *   TP_STRONG_GAUSSIAN_BEAM  aux = zslice_npar[nz], xoffsets[nz], yoffsets[nz]
 *                     (iparam[1] = 3*nzslice); param[0] = charge,
 *                     param[1] = total_energy, param[2..3] = beamsize
 *   TP_LONGITUDINAL_WAKE  aux = times[n], wakefields[n] (iparam[1] = 2n, n >= 2);
 *                     param[0] = fliphalf, param[1] = scale
 *   TP_WIGGLER        aux = NHharm, NVharm, rad, By[6*NHharm], Bx[6*NVharm];
 *                     L, num_int_steps = Nsteps, param[0] = lw, param[1] = Bmax,
 *                     param[2] = energy
 */

/* Misalignment of one element: entrance translation t1, entrance rotation r1,
 * exit rotation r2, exit translation t2 (tracking.jl:60-67,117-130).  The 6x6
 * matrices are column-major, as Julia stores SMatrix.  A zero matrix means
 * "not applied", exactly as `iszero(elem.r1)` does in the reference. */
typedef struct tp_misalign {
    double t1[6];
    double t2[6];
    double r1[36];
    double r2[36];
} tp_misalign;

/* ------------------------------------------------------------------------- */
/* Per-call options                                                           */
/* ------------------------------------------------------------------------- */
typedef struct tp_opts {
    int32_t size;              /* sizeof(tp_opts); 0 selects all defaults          */
    int32_t exact_hamiltonian; /* 1 (default) = exact drift, 0 = linearised drift;
                                  reference global USE_EXACT_HAMILTONIAN,
                                  tracking.jl:38,100-107                          */
    int32_t device_pointers;   /* 1: data pointers are device pointers            */
    int32_t fp_contract;       /* 1: use the kernels built with FMA contraction.
                                  Default 0: no contraction, so every map evaluates
                                  the reference's operations in its order (exact
                                  bends amplify a changed rounding to ~1e-11)     */
    int32_t block_size;        /* threads per block; 0 = autotuned                */
    int32_t min_blocks;        /* tracking kernel instance: registers sized for 8,
                                  7, 6 or 5 resident 128-thread blocks per SM (more
                                  blocks hide more latency, fewer spill less);
                                  0 = autotuned.  The build with FMA contraction
                                  and tables with kinds outside the integrator
                                  core have the 7-block instance only             */
    int32_t schedule;          /* 0 = autotuned; 1 = static, 2 = lane refill
                                  (batched: lanes of a variant refill from that
                                  variant's particles).  Autotuning (schedule and
                                  min_blocks 0): the first multi-turn calls of a
                                  configuration run static and lane refill at 7
                                  blocks, then 8, 6 and 5 blocks with the faster
                                  schedule, each timed on the call's own work;
                                  later calls keep the fastest.  Every choice
                                  gives identical results                         */
    int32_t table_in_smem;     /* 1: stage the element table into shared memory by a
                                  bulk (TMA) copy at the start of each block; default
                                  0: read it through the L1 cache.  On the DBA ring the
                                  staged table (37.5 KB per block) leaves the L1 too
                                  small for the kernels' stack, and staging measured
                                  5 % slower                                       */
    double aperture_x;         /* rectangular aperture half widths [m]; a value   */
    double aperture_y;         /* <= 0 disables it (reference limits remain)      */
    void* stream;              /* cudaStream_t to run on; NULL = context stream, a
                                  blocking stream ordered with the legacy default
                                  stream                                          */
    int32_t bounds_check;      /* 1: run the bounds-checked tracking kernels (no
                                  FMA contraction): an element-table record outside
                                  its table or turn block, or a particle index >= N,
                                  is skipped and reported as TP_EDEVICE instead of
                                  being read; results are otherwise identical      */
    int32_t reserved0;
} tp_opts;

/* Statistics of the last tracking call on a context. */
typedef struct tp_stats {
    int64_t particles;         /* particles alive at the start of the call        */
    int64_t survivors;         /* particles alive at the end                      */
    int64_t element_passes;    /* particle-element maps evaluated                 */
    double units;              /* particle*element*turns = alive-at-start x elements x turns */
    double flops;              /* algorithmic FLOPs of the evaluated maps         */
    double kernel_ms;          /* device time of the tracking kernels             */
    double total_ms;           /* host wall time of the call                      */
    int64_t h2d_bytes;
    int64_t d2h_bytes;
    int32_t block_size;
    int32_t min_blocks;        /* resident blocks per SM of the kernel instance   */
    int32_t grid;
    int32_t launches;          /* kernels this library launched in the call      */
    int32_t schedule;          /* 1 = static, 2 = lane refill                      */
    int32_t fp_contract;
    int32_t refill_fold;       /* batched pooled refill: variant particles per warp
                                  tile / 32 (1 = one tile per 32 particles)       */
    int32_t bounds_check;      /* 1: the bounds-checked kernels ran               */
} tp_stats;

/* ------------------------------------------------------------------------- */
/* Library, context                                                           */
/* ------------------------------------------------------------------------- */
typedef struct tp_ctx tp_ctx;
typedef struct tp_lattice tp_lattice;
typedef struct tp_batch tp_batch;

TP_API int tp_abi_version(void);
TP_API const char* tp_strerror(int status);
/* Text of the last CUDA error seen by this thread (empty if none). */
TP_API const char* tp_last_error_string(void);

/* Number of usable CUDA devices (0 when none); never fails. */
TP_API int tp_device_count(void);

/* Create a tracking context on `device` (owns a stream and scratch buffers). */
TP_API int tp_ctx_create(int device, tp_ctx** out);
TP_API int tp_ctx_destroy(tp_ctx* ctx);
TP_API int tp_last_stats(const tp_ctx* ctx, tp_stats* out);

/* Beam(energy; mass) semantics of src/lattice.jl:46-61: gamma = (E + m)/m
 * (E is kinetic), beta = sqrt(1 - 1/gamma^2), beti = 1/beta.  Host only. */
TP_API int tp_beam_beti(double energy, double mass, double* beti_out);

/* ------------------------------------------------------------------------- */
/* Lattices                                                                   */
/* ------------------------------------------------------------------------- */
/* Validate and compile `n` element records into the device element table.
 * Host-only work: the device copy is made on first use by a context.  The
 * records are copied; the caller keeps ownership of `elems`/`mis`.
 * Replaces building Lattice(elems) (src/lattice.jl:87-99) for the device.  */
TP_API int tp_lattice_create(const tp_elem* elems, int64_t n,
                             const tp_misalign* mis, int64_t nmis,
                             tp_lattice** out);
/* The same with the array fields of StrongGaussianBeam, LongitudinalWake and
 * Wiggler elements in `aux` (see the per-kind layouts above); the arrays are
 * copied.  A record may hold at most 65535 words (TP_ERANGE beyond). */
TP_API int tp_lattice_create_ex(const tp_elem* elems, int64_t n,
                                const tp_misalign* mis, int64_t nmis,
                                const double* aux, int64_t naux,
                                tp_lattice** out);
TP_API int tp_lattice_destroy(tp_lattice* lat);
TP_API int tp_lattice_length(const tp_lattice* lat, int64_t* n_out);

/* Algorithmic FLOPs of one particle through each element (typical particle,
 * counted with the rules add/sub/mul/div/sqrt = 1, fused multiply-add = 2,
 * each sin/cos/tan/asin/atan/exp call = TP_FLOPS_PER_TRANSCENDENTAL).  */
#define TP_FLOPS_PER_TRANSCENDENTAL 20
TP_API int tp_lattice_flops(const tp_lattice* lat, double* flops_per_elem /* n */);

/* Time-varying fields (reference `timed(elem; field=f)` + `materialize`,
 * src/time_dependence.jl:147-173).  The host evaluates each closure at every
 * turn's (time, turn) context and passes the values here; tracking at turn t
 * then uses the element with those fields, exactly as linepass! materialises
 * it once per element per call (src/lattice.jl:267).
 *   fields[2*j]   = element index, fields[2*j+1] = enum tp_field
 *   values[(t - turn0)*nfields + j] = field j at turn t, t in [turn0, turn0+nturns)
 * Passing nfields = 0 clears the schedule. */
enum tp_field {
    TP_FIELD_L = 0, TP_FIELD_K = 1, TP_FIELD_ANGLE = 2, TP_FIELD_E1 = 3,
    TP_FIELD_E2 = 4, TP_FIELD_VOLT = 5, TP_FIELD_FREQ = 6, TP_FIELD_LAG = 7,
    TP_FIELD_PHILAG = 8, TP_FIELD_ENERGY = 9, TP_FIELD_NUM_INT_STEPS = 10,
    TP_FIELD_POLYNOM_A0 = 11, /* +i for polynom_a[i], i = 0..3 */
    TP_FIELD_POLYNOM_B0 = 15, /* +i for polynom_b[i] */
    TP_FIELD_COUNT = 19
};
TP_API int tp_lattice_set_schedule(tp_lattice* lat, const int32_t* fields, int32_t nfields,
                                   int32_t turn0, int32_t nturns, const double* values);

/* ------------------------------------------------------------------------- */
/* Tracking: the drop-in for linepass! / ringpass!                            */
/* ------------------------------------------------------------------------- */
/* One pass through the lattice (src/lattice.jl:260-297).  Particles with
 * lost_flags[i] == 1 are skipped.  A particle whose map output fails
 * check_lost (tracking.jl:49-52) or the aperture gets lost_flags[i] = 1 and
 * keeps the coordinates it had at that element's entrance.
 * lost_turn / lost_elem (Int32, may be NULL) receive the turn and 0-based
 * element index of the loss for particles lost in this call and are left
 * unchanged otherwise.  `time` and `turn` select the schedule row. */
TP_API int tp_linepass(tp_ctx* ctx, const tp_lattice* lat,
                       double* coords, int64_t n, int64_t* lost_flags,
                       int32_t* lost_turn, int32_t* lost_elem,
                       double beti, double time, int32_t turn,
                       const tp_opts* opts);

/* nturns passes (src/lattice.jl:305-317): turn k uses time + k*dt_turn and
 * turn index turn0 + k.  One device launch covers every turn; the particle
 * state stays in registers between elements and turns. */
TP_API int tp_ringpass(tp_ctx* ctx, const tp_lattice* lat,
                       double* coords, int64_t n, int64_t* lost_flags,
                       int32_t* lost_turn, int32_t* lost_elem,
                       double beti, int32_t nturns,
                       double time, double dt_turn, int32_t turn0,
                       const tp_opts* opts);

/* ------------------------------------------------------------------------- */
/* Batched ragged tracking (many lattice variants, one persistent launch)     */
/* ------------------------------------------------------------------------- */
/* A batch concatenates the element tables of `nvar` lattices (uneven element
 * counts) into one ragged device table.  No reference counterpart: it runs
 * ringpass! for every (lattice_v, coords_v) pair at once. */
TP_API int tp_batch_create(tp_ctx* ctx, const tp_lattice* const* lats, int32_t nvar,
                           tp_batch** out);
TP_API int tp_batch_destroy(tp_batch* b);

/* coords: all variants' particles in one N_total x 6 column-major array;
 * variant v owns rows [poff[v], poff[v+1]).  beti[v] per variant.  When
 * use_graph != 0 the launch sequence is captured once in a CUDA graph and
 * replayed while the shapes stay the same. */
TP_API int tp_ringpass_batched(tp_ctx* ctx, tp_batch* b,
                               double* coords, const int64_t* poff,
                               int64_t* lost_flags, int32_t* lost_turn, int32_t* lost_elem,
                               const double* beti, int32_t nturns,
                               double time, double dt_turn, int32_t turn0,
                               int32_t use_graph, const tp_opts* opts);

/* ------------------------------------------------------------------------- */
/* Adjoint (reverse-mode gradient of a tracked-beam loss)                     */
/* ------------------------------------------------------------------------- */
/* No reference counterpart (the Enzyme extension is a stub,
 * ext/TrackPadEnzymeExt.jl:14-17).  Loss over the particles alive at the end:
 *   loss = mean_s (x_s^2 + y_s^2) / sigma^2 + lost_weight * (lost / alive-at-start)
 * The gradient is taken with respect to the main strength `k` of the listed
 * elements (Quadrupole k1, Sextupole k2, Octupole k3); the survivor set is
 * held fixed, so the piecewise-constant loss term contributes nothing.
 * Every element kind and every misalignment row can be differentiated; a
 * misalignment row whose r1 or r2 is singular (no inverse map) gives
 * TP_EUNSUPPORTED, here and in tp_one_turn_jacobian. */
enum tp_loss_kind { TP_LOSS_BEAM_SIZE = 0 };
typedef struct tp_loss_spec {
    int32_t kind;
    int32_t reserved;
    double sigma;
    double lost_weight;
} tp_loss_spec;

/* coords0 / lost0 are read only.  coords_out / lost_out (may be NULL) receive
 * the forward result.  checkpoint_every = K turns between stored particle
 * states (0 = autotuned); within a K-turn segment the reverse sweep rebuilds
 * states with the integrators' time-reversed maps. */
TP_API int tp_ringpass_adjoint(tp_ctx* ctx, const tp_lattice* lat,
                               const double* coords0, int64_t n, const int64_t* lost0,
                               double beti, int32_t nturns,
                               double time, double dt_turn, int32_t turn0,
                               const int32_t* param_elems, int32_t nparams,
                               const tp_loss_spec* loss, int32_t checkpoint_every,
                               double* loss_out, double* grad_out,
                               double* coords_out, int64_t* lost_out,
                               const tp_opts* opts);

/* Batched adjoint: per-variant loss and gradient in one launch.
 * param_off[v]..param_off[v+1] index into param_elems (element indices of
 * variant v) and grad_out; loss_out has nvar entries. */
TP_API int tp_ringpass_adjoint_batched(tp_ctx* ctx, tp_batch* b,
                                       const double* coords0, const int64_t* poff,
                                       const int64_t* lost0, const double* beti,
                                       int32_t nturns, double time, double dt_turn, int32_t turn0,
                                       const int32_t* param_elems, const int32_t* param_off,
                                       const tp_loss_spec* loss, int32_t checkpoint_every,
                                       double* loss_out, double* grad_out,
                                       const tp_opts* opts);

/* Statistics of the last adjoint or Jacobian call on this host thread (no
 * reference counterpart).  The reverse sweep rebuilds each K-turn segment
 * with the maps' time-reversed forms; reconstruction_error is the largest
 * absolute difference, over survivors and segment starts, between a rebuilt
 * state and the stored checkpoint. */
typedef struct tp_adjoint_stats {
    int32_t checkpoint_every;     /* K used                                       */
    int32_t segments;             /* ceil(nturns / K)                             */
    int64_t checkpoint_bytes;     /* device memory of the stored states           */
    int64_t particles;            /* particles in the launch                      */
    double units;                 /* particle*element*turns of the forward pass   */
    double forward_ms;            /* device time of the forward (checkpointing) pass */
    double reverse_ms;            /* device time of the reverse sweep             */
    double reconstruction_error;
    int32_t launches;
    int32_t k_tuning;             /* 0: K given by the caller (or a loss-only call,
                                     where K does not matter); 1: the call was a
                                     timing trial of the K autotuner; 2: K is the
                                     autotuner's choice                          */
    double tuned_ms;              /* forward + reverse device time of the chosen K
                                     in its trial (0 until the trials are done)  */
} tp_adjoint_stats;
TP_API int tp_last_adjoint_stats(tp_adjoint_stats* out);

/* ------------------------------------------------------------------------- */
/* One-turn Jacobian and symplecticity                                        */
/* ------------------------------------------------------------------------- */
/* Forward-mode tangent map of nturns passes about each of `n` reference
 * orbits (the analytic counterpart of one_turn_map, src/optics.jl:110-121).
 * jac_out: n x 36 doubles, column-major 6x6 per orbit (M[i,j] at j*6+i).
 * sympl_out (may be NULL): ||M^T J M - J||_max per orbit.  orbits is n x 6
 * column-major like coords and is read only. */
TP_API int tp_one_turn_jacobian(tp_ctx* ctx, const tp_lattice* lat,
                                const double* orbits, int64_t n, double beti,
                                int32_t nturns, int32_t turn0,
                                double* jac_out, double* sympl_out,
                                const tp_opts* opts);

/* ------------------------------------------------------------------------- */
/* Allocation-free tracking                                                   */
/* ------------------------------------------------------------------------- */
/* No counterpart in the reference.  ringpass! for callers that cannot let a
 * library allocate device memory (a memory pool that owns the whole device,
 * an allocation-free real-time loop, code that must not let cudaMalloc or
 * cudaFree synchronise the device): the same tracking kernel as tp_ringpass,
 * with its scratch (work and pass counters, error word, element table) in a
 * fixed device array of the library instead of allocated buffers.
 *   * all data pointers are device pointers on the current device; the call
 *     runs on `stream` (NULL: the default stream) and returns when it is done;
 *   * the element table may hold at most 16384 words (128 KiB, about 1400
 *     DBA-type elements); larger tables give TP_ERANGE, lattices with
 *     misalignment rows or a per-turn schedule give TP_EUNSUPPORTED;
 *   * the array (about 128 KiB) stays allocated on every GPU that loads the
 *     library until the process exits, and every call shares it: calls that
 *     overlap on the GPU race with each other.  A call copies the element
 *     table into the array only when the array does not already hold this
 *     lattice's current program on that device; the kernel reads it through
 *     the L1 cache, like tp_ringpass;
 *   * the lattice must not be destroyed while a call on it runs (a schedule
 *     change from another thread waits for the call's table copy);
 *   * the first call on a device looks up the array's address there; make it
 *     before any stream capture.
 * Always the exact drift and no FMA contraction (tp_opts defaults). */
TP_API int tp_ringpass_noalloc(const tp_lattice* lat, double* coords, int64_t n, int64_t* lost_flags,
                               int32_t* lost_turn, int32_t* lost_elem, double beti, int32_t nturns,
                               int32_t turn0, double aperture_x, double aperture_y, void* stream);

/* ------------------------------------------------------------------------- */
/* Truncated power series (TPSA) maps                                         */
/* ------------------------------------------------------------------------- */
/* linepass / ringpass of six CTPS values and polyseries_one_turn_map
 * (ext/TrackPadPolySeriesExt.jl:654-705; CTPS is the truncated power series
 * type of the PolySeries package).  A map is six series (x, px, y, py, z,
 * delta) in the six phase-space variables truncated at total order `order`
 * (0..10), each stored as M = C(order + 6, 6) coefficients in the order
 * tp_tpsa_monomials gives: by degree, then by exponent vector in descending
 * lexicographic order.  polyseries_variables(x0) is the map with constant
 * parts x0 and unit first-order parts. */
TP_API int tp_tpsa_coefficients(int32_t order, int64_t* ncoef);
/* exps: M x 6 exponents of the monomials, in coefficient order. */
TP_API int tp_tpsa_monomials(int32_t order, int32_t* exps);
/* maps: host array of nmaps x 6 x M doubles, updated in place by nturns
 * passes of the lattice from turn turn0 (per-turn schedules apply).  Element
 * kinds without a CTPS pass! method in the reference (ExactSBend, LBend,
 * Wiggler) give TP_EUNSUPPORTED; no aperture or loss check (as the
 * reference). */
TP_API int tp_tpsa_ringpass(tp_ctx* ctx, const tp_lattice* lat, double* maps, int64_t nmaps, int32_t order,
                            double beti, int32_t nturns, int32_t turn0);
/* Work of the last tp_tpsa_ringpass on this thread: series products (each
 * `pairs` coefficient products), elementwise series operations (M
 * coefficients each), their FLOPs (a product counts 2*pairs - M), and the
 * kernel's device time. */
typedef struct tp_tpsa_stats {
    int64_t maps;
    int32_t order, coefficients;
    int64_t pairs;
    double series_mul, series_lin, flops;
    double kernel_ms;
    int32_t grid, block, shared_pool;
    int32_t slots;                /* series slots per map in the pool           */
    int32_t slots_used;           /* most series slots one map held at a time */
    int32_t reserved;
} tp_tpsa_stats;
TP_API int tp_tpsa_last_stats(tp_tpsa_stats* out);

/* ------------------------------------------------------------------------- */
/* Diagnostics                                                                */
/* ------------------------------------------------------------------------- */
/* Measured FP64 fused-multiply-add throughput of the device (TFLOP/s, 2 FLOPs
 * per FMA), from a register-resident FMA-chain kernel timed with CUDA events.
 * Used as the FP64 roofline denominator. */
TP_API int tp_probe_fp64_peak(tp_ctx* ctx, double* tflops_out);

#ifdef __cplusplus
}
#endif
#endif /* TRACKPAD_B200_H */

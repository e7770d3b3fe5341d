/* plis.h — C ABI of the B200 PLISCuda simulation step (libplis.so).
 *
 * The reference exposes one C++ entry point for its whole hot path,
 *     void PLISCuda::run_simulation(Topology t, State s, Reactions r, float* h_rrc, float* h_drc,
 *                                   float endTime, int compartments_count, int* subv_constants,
 *                                   float log_freq);          (PLISCuda/include/cuda/driver.cuh:32-33)
 * called once from main (PLISCuda/src/main.cpp:53-63).  This header splits that function into a
 * handle API with plain pointers and sizes, so it can be bound from C, C++ (the drop-in shim in
 * pliscuda_b200/compat/), Python ctypes, or any FFI.  Every function returns a plis_status
 * (0 = PLIS_OK); no exception, exit() or abort crosses the ABI.  The message of the last failure
 * on the calling thread is available from plis_last_error().
 *
 * Data layout at the boundary (the same as the reference's host arrays):
 *   counts      uint32 [S*N] species-major, counts[s*N + i]      (State.hpp:210, driver.cu:55)
 *   reactants   int32  [S*R] species-major, reactants[s*R + r]  (Reactions.hpp:197)
 *   products    int32  [S*R] species-major                      (Reactions.hpp:209)
 *   neighbours  uint32 [6*N] row-major, unused slots hold the subvolume's own index
 *                                                               (Topology.hpp:176-184)
 *   reaction_rates  [C*R], diffusion_rates [C*S] compartment-major (Configuration.hpp:123-143)
 *   compartment int32  [N] compartment of each subvolume       (cpp_utils.hpp:47-56)
 * Counts must stay below 2^30.  The reference stores them as int (driver.cu:55-59); one bit of
 * headroom lets a step's summed int32 deltas be checked without overflow.  set_state rejects larger
 * counts (PLIS_ERR_OVERFLOW), and a step that would reach 2^30 is rolled back with a halved tau.
 */
#ifndef PLIS_H_
#define PLIS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PLIS_ABI_VERSION 1

typedef enum plis_status {
  PLIS_OK = 0,
  PLIS_ERR_INVALID = 1,    /* bad argument or inconsistent model (reference: std::invalid_argument) */
  PLIS_ERR_PARSE = 2,      /* malformed input file (reference: std::invalid_argument from the parsers) */
  PLIS_ERR_IO = 3,         /* file missing or unreadable (Configuration.hpp:53-55 "file ... not found") */
  PLIS_ERR_OOM = 4,        /* host or device allocation failed */
  PLIS_ERR_CUDA = 5,       /* CUDA runtime error (reference: gpuErrchk -> exit, cpp_utils.hpp:97-105) */
  PLIS_ERR_TIMEOUT = 6,    /* a bounded device-side wait gave up */
  PLIS_ERR_STUCK = 7,      /* more than max_rollbacks consecutive rollbacks in one step */
  PLIS_ERR_OVERFLOW = 8,   /* a count would leave [0, 2^30) (set_state input, or a step no rollback can fix) */
  PLIS_ERR_LIMIT = 9,      /* model exceeds a compiled limit (species, reactions, order, neighbours) */
  PLIS_ERR_NO_DEVICE = 10, /* no CUDA device (main.cpp:19-24) */
  PLIS_ERR_UNSUPPORTED = 11
} plis_status;

/* Semantics of the step (plis_options.mode). */
#define PLIS_MODE_REFERENCE 0 /* the reference's rules, deterministic quirks included */
#define PLIS_MODE_CORRECTED 1 /* Cao-consistent criticality, diffusion terms and exact events */

/* Arithmetic of propensities, Cao tau and Poisson means (plis_options.precision).  Simulated
 * time, the tau array, the min-tau reduction and exponential next-event times are binary64 in both. */
#define PLIS_PREC_FP64 0
#define PLIS_PREC_FP32 1

/* Kernel of the learned-tau MLP (plis_options.learned_mlp, plis_learner_predict). */
#define PLIS_MLP_TCGEN05 0  /* tcgen05.mma, accumulators in tensor memory */
#define PLIS_MLP_MMA_SYNC 1 /* warp-level mma.sync, accumulators in registers */

/* Per-subvolume operation flags (the reference's enum op, constants.cuh:53-58). */
#define PLIS_LEAP_CR 0
#define PLIS_LEAP_NOCR 1
#define PLIS_SSA 2
#define PLIS_SSA_FF 3

/* Why plis_run / plis_step returned. */
#define PLIS_STOP_NONE 0
#define PLIS_STOP_TIME 1      /* simulated time reached t_end */
#define PLIS_STOP_STEPS 2     /* the requested number of steps was taken */
#define PLIS_STOP_NO_EVENT 3  /* min tau was +inf or negative: nothing can fire (driver.cu:269-272) */
#define PLIS_STOP_ERROR 4

typedef struct plis_model_desc {
  uint32_t n_subvolumes;  /* N */
  uint32_t n_species;     /* S */
  uint32_t n_reactions;   /* R */
  uint32_t n_compartments;/* C >= 1 */
  /* Topology: either an explicit table (neighbours != NULL) or an implicit reflective 6-neighbour
   * lattice lattice_x * lattice_y * lattice_z == N, linearised i = x + X*(y + Y*z)
   * (genTopology.py:30-37).  An explicit table that is such a lattice is recognised and run as one. */
  const uint32_t* neighbours;
  uint32_t lattice_x, lattice_y, lattice_z;
  const int32_t* reactants;
  const int32_t* products;
  const double* reaction_rates;
  const double* diffusion_rates;
  const int32_t* compartment; /* NULL: every subvolume in compartment 0 */
} plis_model_desc;

typedef struct plis_options {
  uint32_t size;              /* sizeof(plis_options), filled by plis_options_init */
  int32_t mode;               /* PLIS_MODE_REFERENCE (default) or PLIS_MODE_CORRECTED */
  int32_t precision;          /* PLIS_PREC_FP64 (default) or PLIS_PREC_FP32 */
  int32_t critical_threshold; /* NC, default 10 (driver.cu:36) */
  double epsilon;             /* Cao epsilon, default 0.05 (driver.cu:37) */
  uint64_t seed;              /* key of the Philox4x32-10 stream, default 1 */
  uint32_t replica;           /* replica id folded into the key (independent streams) */
  int32_t device;             /* CUDA device ordinal, default 0 */
  int32_t max_rollbacks;      /* per step before PLIS_ERR_STUCK, default 64 */
  int32_t steps_per_launch;   /* steps captured per CUDA-graph launch, 0 = auto */
  int32_t tile[3];            /* lattice brick per CTA (x, y, z), 0 = auto */
  int32_t persistent;         /* reserved, ignored by plis_create: a handle's step is always the graph of phase
                               * kernels; the persistent cooperative launch is the batched form (plis_batch_*,
                               * one replica or many) */
  int32_t profile;            /* 1 = launch phase kernels one by one with CUDA events around each (plis_get_profile) */
  int32_t stage_halo;         /* lattice leap: 1 = stage brick + halo in shared memory, 0 = global atomics (default) */
  int32_t learned_mlp;        /* learned tau MLP: 0 = tcgen05.mma with TMEM accumulators (default), 1 = mma.sync */
  uint64_t wait_polls;        /* polls after which a device-side wait gives up with PLIS_ERR_TIMEOUT: the grid
                               * barrier of the persistent batched kernel (>= 32 ns per poll) and the mbarrier
                               * waits of the tcgen05 MLP; 0 = defaults (2^26 and 2^22 polls).  The reference
                               * has no device waits (its host loop synchronises, driver.cu:259-376). */
  int32_t pooled_draws;       /* leap: 1 = channels of small mean (below 1/8) drawn as one pooled Poisson total
                               * split over them, 0 = one draw per channel, -1 = auto (default: pooled for
                               * networks of more than 4 reactions or 4 species).  Either way every channel's
                               * firings are Poisson with its mean, independent of the others (leap.cu:20-53
                               * draws one per channel); the two settings give different, equally valid
                               * trajectories. */
} plis_options;

/* Per-kernel device time accumulated while plis_options.profile is set (CUDA events recorded on the
 * handle's stream around every launch). */
#define PLIS_KERNEL_LEAP 0
#define PLIS_KERNEL_EXACT 1
#define PLIS_KERNEL_APPLY 2
#define PLIS_KERNEL_CLASSIFY 3
#define PLIS_KERNEL_COUNT 4
typedef struct plis_profile {
  double ms[PLIS_KERNEL_COUNT];
  uint64_t launches[PLIS_KERNEL_COUNT];
} plis_profile;

typedef struct plis_stats {
  double time;            /* simulated time */
  uint64_t steps;         /* accepted steps */
  uint64_t rollbacks;     /* rejected attempts */
  uint64_t events;        /* reaction firings + molecule jumps (a leap firing of k counts k) */
  uint64_t exact_events;  /* single-event firings (critical and SSA) among them */
  int32_t stop_reason;    /* PLIS_STOP_* of the last run/step call */
  int32_t status;         /* sticky error status of the handle (PLIS_OK if none) */
  double last_tau;        /* arg-min tau of the last accepted step */
  int64_t last_argmin;    /* its subvolume */
  double device_ms;       /* device time spent in run/step calls (CUDA events) */
  uint64_t kernel_launches; /* kernels launched by the library so far */
} plis_stats;

typedef struct plis_handle plis_handle;

/* Library */
int plis_abi_version(void);
const char* plis_last_error(void);         /* thread-local message of the last failed call */
const char* plis_status_string(int status);
void plis_options_init(plis_options* opts);

/* Lifecycle.  Replaces the set-up half of run_simulation (driver.cu:15-239): the model is copied
 * (the caller keeps ownership of every input array), device memory is allocated once, and the
 * state starts at zero counts until plis_set_state. */
int plis_create(const plis_model_desc* model, const plis_options* opts, plis_handle** out);
int plis_destroy(plis_handle* h);

/* State.  plis_set_state copies counts to the device, resets time/steps/statistics and computes
 * the initial rates, taus and flags (driver.cu:221-234).  plis_get_state copies them back
 * (driver.cu:366, :391). */
int plis_set_state(plis_handle* h, const uint32_t* counts);
/* plis_set_state for a trajectory that continues from a host copy of its counts: the counts are at
 * simulated time `time` after `steps` accepted steps.  The accepted-step counter keys the random
 * stream, so the continued steps draw the numbers the same trajectory would have drawn on the device
 * (the reference has no counterpart: its loop never leaves the device, driver.cu:259-376).  The
 * statistics restart at zero; plis_get_stats reports steps from `steps` on. */
int plis_set_state_at(plis_handle* h, const uint32_t* counts, double time, uint64_t steps);
int plis_get_state(plis_handle* h, uint32_t* counts);
int plis_set_time(plis_handle* h, double time);

/* The step loop (driver.cu:259-376).  plis_run advances until simulated time >= t_end (reference
 * mode: the step that crosses t_end is taken, as the reference loop does; corrected mode: the last
 * step is shortened to land on t_end exactly).  plis_step takes at most n_steps accepted steps.
 * Both stop early on PLIS_STOP_NO_EVENT. */
int plis_run(plis_handle* h, double t_end);
int plis_step(plis_handle* h, uint64_t n_steps);
int plis_get_stats(plis_handle* h, plis_stats* out);

/* The reference's whole run_simulation (driver.cu:12-408) in one call: create a handle with opts
 * (NULL = defaults), set counts at simulated time start_time (0 for a new run; a snapshot's time,
 * plis_read_snapshot, to resume one), run until simulated time >= end_time, writing
 * sim<unix time>_<time>.dat into out_dir (NULL or "" = the working directory) each time at least
 * log_freq of simulated time has passed since the last snapshot (log_freq > 0; driver.cu:362-375)
 * and once at the end (driver.cu:390-397), and, when verbose, print the reference's progress and
 * final statistics lines to stdout (driver.cu:246, 380, 399-405).  A step with no possible event
 * ends the run early as in the reference (driver.cu:269-272; stats.stop_reason ==
 * PLIS_STOP_NO_EVENT).  *out (may be NULL) receives the final statistics. */
int plis_run_simulation(const plis_model_desc* model, const uint32_t* counts, double start_time, double end_time,
                        double log_freq, const plis_options* opts, const char* out_dir, int verbose, plis_stats* out);

/* Per-kernel timing of profiled run/step calls (plis_options.profile = 1); reset by plis_set_state. */
int plis_get_profile(plis_handle* h, plis_profile* out);

/* Inspection: per-subvolume tau (binary64) and operation flags of the current state. */
int plis_get_taus(plis_handle* h, double* tau, uint8_t* flags);

/* Event log.  The reference's LOG build prints one line per event from inside its kernels
 * (leap.cu:29-32, 58-62, 144-146, 196-198; ssa.cu:69-71, 96-98).  Here the kernels append one
 * 32-byte record per event to a device buffer of the handle, read back on the host between calls.
 * The records of one step come in no particular order.  Every attempt of a step is logged, the
 * discarded ones included (their `attempt` is below the step's last), as the reference prints
 * before its rollback check (driver.cu:292-315).  An event is a leap draw with count > 0 or one
 * exact event that changed the state. */
typedef struct plis_event_record {
  double time;        /* simulated time at the start of the step */
  uint64_t step;      /* number of the step (1 = the first step of the handle) */
  uint32_t subvolume; /* where the event happened: the source of a diffusion */
  uint32_t target;    /* destination subvolume of a diffusion; = subvolume for a reaction */
  uint32_t count;     /* firings, or molecules moved (exact events: 1); saturated at 2^32-1, and a
                         leap jump at 2^27 (a jump that large always rolls the attempt back) */
  uint16_t channel;   /* reaction index, or species index of a diffusion */
  uint8_t kind;       /* PLIS_EVENT_* */
  uint8_t attempt;    /* rollback attempt of the step, 0 first (saturated at 255) */
} plis_event_record;
#define PLIS_EVENT_LEAP_REACTION 1      /* Poisson firings of one reaction (leap.cu:29-32) */
#define PLIS_EVENT_LEAP_DIFFUSION 2     /* Poisson jumps of one species to one neighbour (leap.cu:58-62) */
#define PLIS_EVENT_CRITICAL_REACTION 3  /* critical reaction of a LEAP_CR subvolume (leap.cu:144-146) */
#define PLIS_EVENT_CRITICAL_DIFFUSION 4 /* critical jump of a LEAP_CR subvolume (leap.cu:196-198) */
#define PLIS_EVENT_SSA_REACTION 5       /* exact reaction of the arg-min subvolume (ssa.cu:69-71) */
#define PLIS_EVENT_SSA_DIFFUSION 6      /* exact jump of the arg-min subvolume (ssa.cu:96-98) */
/* Room for `capacity` records on the device (0 turns the log off and frees it); the log starts
 * empty.  Events past the capacity are counted, not stored. */
int plis_set_event_log(plis_handle* h, uint64_t capacity);
/* Copies min(stored, max_records) records, in the order they were appended, into out (may be NULL
 * when max_records is 0); *n_records = records stored (<= capacity), *n_dropped = events not
 * stored for lack of room since the log was last emptied.  clear != 0 empties the log afterwards.
 * A handle without a log reports 0 and 0. */
int plis_read_event_log(plis_handle* h, plis_event_record* out, uint64_t max_records, uint64_t* n_records,
                        uint64_t* n_dropped, int clear);

/* Arg-min of a device array of n taus (first index on ties) into *d_min_tau / *d_argmin, enqueued
 * on `stream` (a cudaStream_t, NULL for the default stream); the same global min-tau reduction the
 * step does internally.  No counterpart in the reference: it exists for callers that cannot allocate
 * device memory (a host whose own allocator owns the device memory, or a latency-critical loop in
 * which cudaMalloc may synchronise the device).  It allocates nothing: inputs and outputs are the
 * caller's device buffers, and its 16 KiB of per-CTA partials live in a fixed array inside the
 * library, held on every device that loads the library until exit.  Each call looks up that array's
 * device address in the context current on the calling thread (the runtime's context of the current
 * device, also after cudaDeviceReset); the first call on a device may load the library's device code
 * there, so make it before any stream capture.  Calls share the array, so calls that overlap on the
 * GPU race.  NaN taus are skipped (they compare below nothing): NaNs only give (+inf, -1), NaNs among
 * numbers give the arg-min of the numbers; +inf only gives (+inf, 0).  n must be in
 * 1..PLIS_NOALLOC_MAX_TAUS, else PLIS_ERR_LIMIT. */
#define PLIS_NOALLOC_MAX_TAUS 2147483647u
int plis_tau_argmin_noalloc(const double* d_tau, uint64_t n, double* d_min_tau, int64_t* d_argmin, void* stream);

/* z-slab decomposition of one lattice over several ranks (one process or handle per slab; no
 * counterpart in the reference, which runs one GPU, main.cpp:25-28).  A handle created for the whole
 * model and given plis_slab_setup computes only the subvolumes of z-layers [z0, z1); z0 and z1 must be
 * multiples of the brick's z extent, and the slabs of the ranks 0 .. world-1 must tile the lattice in
 * rank order.  Arrays stay full size and indices global: random streams, neighbour counts and the
 * arg-min tie rule are those of the single domain, so the slabs together follow the single-domain
 * trajectory bit for bit.  The caller moves the data between phases (pliscuda_b200/slabs.py does it
 * over torch.distributed or within one process):
 *   PLIS_SLAB_CLASSIFY  classify the slab; its summary is in buffers.summary (call first, after
 *                       plis_set_state, for the initial state; later after PLIS_SLAB_UNPACK)
 *     -> gather every rank's summary into buffers.summary_all (rank order)
 *   PLIS_SLAB_CONTROL   the step decision from summary_all (identical on every rank); the face flags
 *                       are staged in send[0] (to the slab below) and send[1] (above)
 *     -> send[0] to the slab below's recv[1], send[1] to the slab above's recv[0]
 *   PLIS_SLAB_FLAGS     received face flags into the ghost layers
 *   PLIS_SLAB_PREPARE   start a run to t_end / n_steps (what plis_run / plis_step do first)
 * and, per attempt while not done (plis_get_stats stop_reason):
 *   PLIS_SLAB_LEAP      leap, exact events and deltas of the slab; the ghost layers (molecules sent
 *                       across the faces) staged in send[0..1], flag writes outside the slab in remote
 *     -> exchange send/recv as above; gather every rank's remote into remote_all
 *   PLIS_SLAB_MERGE     received molecules added into the face layers, flags merged; faces staged
 *     -> exchange send/recv
 *   PLIS_SLAB_UNPACK    received face layers into the ghost layers
 *   PLIS_SLAB_CLASSIFY, gather, PLIS_SLAB_CONTROL, exchange, PLIS_SLAB_FLAGS as above.
 * Every phase returns once its kernels have finished.  Lattice models only; learned proposals and
 * the event log are not available on a slab. */
#define PLIS_SLAB_CLASSIFY 0
#define PLIS_SLAB_CONTROL 1
#define PLIS_SLAB_FLAGS 2
#define PLIS_SLAB_PREPARE 3
#define PLIS_SLAB_LEAP 4
#define PLIS_SLAB_MERGE 5
#define PLIS_SLAB_UNPACK 6
typedef struct plis_slab_buffers {
  void* send[2];          /* device int32[stage_words]: to the slab below (0) / above (1) */
  void* recv[2];          /* device int32[stage_words]: from the slab below (0) / above (1) */
  uint64_t stage_words;   /* (species + 1) * X * Y */
  void* summary;          /* device, summary_bytes: this rank's summary */
  void* summary_all;      /* device, world * summary_bytes: every rank's, in rank order */
  uint64_t summary_bytes;
  void* remote;           /* device, remote_bytes: this rank's flag writes outside its slab */
  void* remote_all;       /* device, world * remote_bytes */
  uint64_t remote_bytes;
} plis_slab_buffers;
int plis_slab_setup(plis_handle* h, uint32_t z0, uint32_t z1, uint32_t world, uint32_t rank);
int plis_slab_buffers_get(plis_handle* h, plis_slab_buffers* out);
int plis_slab_phase(plis_handle* h, int phase, double t_end, uint64_t n_steps);

/* Topology helpers (host only, no device needed).
 * plis_canonical_neighbours rewrites a 6-wide table so that each row lists its distinct non-self
 * neighbours first (lattice rows in the order -x,+x,-y,+y,-z,+z) followed by self padding; this is
 * the slot order the engine's random stream is keyed on.  lattice_out receives (X,Y,Z) when the
 * table is a reflective lattice, else zeros.  table may be NULL when lattice_in is given. */
int plis_canonical_neighbours(uint32_t n, const uint32_t* table, const uint32_t lattice_in[3],
                              uint32_t* canonical, uint32_t lattice_out[3]);

/* ---------------------------------------------------------------------------------------------
 * Batches: many independent replicas of one reaction network, each on its own reflective lattice
 * (uneven sizes) with its own rate constants and its own random stream, advanced together by one
 * persistent cooperative kernel.  The reference can only emulate this by concatenating disjoint
 * topologies into one model, which couples them through its single global min-tau.  Replica r of a
 * batch follows exactly the trajectory of plis_create with options.replica = replica_ids[r].
 * ------------------------------------------------------------------------------------------- */
typedef struct plis_batch_desc {
  uint32_t n_replicas;        /* 1..4096 */
  uint32_t n_species;         /* S <= 16 */
  uint32_t n_reactions;       /* R */
  const int32_t* reactants;   /* [S*R] species-major, shared by all replicas */
  const int32_t* products;    /* [S*R] */
  const uint32_t* lattice;    /* [n_replicas*3] X, Y, Z of each replica */
  const double* reaction_rates;  /* [n_replicas*R] */
  const double* diffusion_rates; /* [n_replicas*S] */
  const uint32_t* replica_ids;   /* [n_replicas] stream key of each replica, NULL = 0..n-1 */
} plis_batch_desc;

typedef struct plis_batch_tuning {
  int32_t tile[3];            /* brick shape of the bricks CTAs take from the work queue */
  int32_t blocks_per_sm;      /* co-resident CTAs per SM of the persistent launch */
  int32_t grid;               /* CTAs of the persistent launch */
  double events_per_s;        /* measured by plis_batch_autotune (0 if not tuned) */
} plis_batch_tuning;

typedef struct plis_batch plis_batch;

int plis_batch_create(const plis_batch_desc* desc, const plis_options* opts, plis_batch** out);
int plis_batch_destroy(plis_batch* b);
/* counts [S*N_r] species-major for replica r; resets that replica's time and statistics */
int plis_batch_set_state(plis_batch* b, uint32_t replica, const uint32_t* counts);
int plis_batch_get_state(plis_batch* b, uint32_t replica, uint32_t* counts);
int plis_batch_get_taus(plis_batch* b, uint32_t replica, double* tau, uint8_t* flags);
/* every replica until its time >= t_end (reference mode) / lands on t_end (corrected mode) */
int plis_batch_run(plis_batch* b, double t_end);
/* every replica at most n_steps accepted steps */
int plis_batch_step(plis_batch* b, uint64_t n_steps);
int plis_batch_get_stats(plis_batch* b, uint32_t replica, plis_stats* out);
/* Time pilot_steps steps of the current state for each candidate brick shape, keep the fastest,
 * restore the state.  The CTAs take bricks (and with them replicas) from a shared work queue, so
 * the number of replicas per CTA adapts to their sizes at run time. */
int plis_batch_autotune(plis_batch* b, uint64_t pilot_steps, plis_batch_tuning* out);
int plis_batch_get_tuning(plis_batch* b, plis_batch_tuning* out);
/* Learned tau proposals for every replica of the batch (the proposer of plis_set_proposer, same
 * rules: corrected mode, up to 4 species, weights NULL or s_max <= 0 detaches).  Replica r then
 * follows exactly the trajectory of a handle with options.replica = replica_ids[r],
 * learned_mlp = PLIS_MLP_MMA_SYNC and the same proposer.  Every replica's current state is
 * classified again; times and statistics are kept. */
int plis_batch_set_proposer(plis_batch* b, const float* weights, double s_max);

/* ---------------------------------------------------------------------------------------------
 * Learned tau proposals (no counterpart in the reference).  A proposer is an MLP 8 -> 64 -> 64 ->
 * 64 -> 1 (ReLU; BF16 weights and activations, FP32 accumulation on the tensor cores) evaluated
 * for every subvolume inside the classification.  Its features are log1p of the count of species
 * 0, of the mean count of species 0 over the neighbours, of the propensities of reactions 0..3,
 * log of the plain Cao leap bound tau_Cao, and log1p of the subvolume's total diffusion rate.  Its
 * output y gives the proposal s * tau_Cao with s = exp(clamp(y, 0, log s_max)); flags and the
 * critical times are decided against the proposal as against tau_Cao in the plain method.  The
 * step leaps with the arg-min of the proposals; an attempt that has to be rolled back is retried
 * with the plain Cao step (halved once per attempt), so every accepted step is either a proposal
 * that kept all counts non-negative or a plain step.  Corrected mode only (PLIS_ERR_UNSUPPORTED
 * otherwise); up to 4 species.  With s_max = 1 the trajectory is the plain method's, bit for bit.
 *
 * Training data are the simulator's own steps: plis_learner_record runs a plain handle step by
 * step and records, for every stride-th subvolume (the offset rotates from step to step), the
 * features of the state, its tau_Cao, the step taken from it and the label
 * log(tau_safe / tau_Cao), where tau_safe = tau_step / max(rho, rho^2) and rho is the largest
 * change of any propensity over the step relative to max(eps_L * a_j, c_j) (the Cao leap
 * condition at tolerance eps_L measured on the realised step), clamped to [log(1/16), log(64)].
 * plis_learner_train fits the MLP to a quantile of the label (pinball loss, Adam) with
 * hand-written CUDA kernels.  The accuracy of a proposer is measured against the plain method
 * (KS distance of the marginals at checkpoints), which fixes s_max.
 * ------------------------------------------------------------------------------------------- */
#define PLIS_PROPOSER_WEIGHTS 8977 /* 8961 parameters, then 8 feature means and 8 inverse deviations */

typedef struct plis_train_params {
  uint64_t iterations;     /* Adam steps, default 2000 */
  uint32_t batch;          /* records per step, a multiple of 128, default 16384 */
  float learning_rate;     /* default 1e-3 */
  float quantile;          /* pinball-loss quantile of the label, default 0.25 */
  uint64_t seed;           /* parameter initialisation and minibatch sampling, default 1 */
} plis_train_params;

typedef struct plis_train_report {
  double loss_first;       /* mean pinball loss of the first and the last step's minibatch */
  double loss_last;
  uint64_t records;        /* records trained on */
  uint64_t iterations;
  double device_ms;        /* device time of the training (CUDA events) */
} plis_train_report;

/* A recorded subvolume-step, as plis_learner_get_records / set_records move them (64 bytes). */
typedef struct plis_trace_record {
  float features[8];       /* raw (unnormalised) features */
  float tau_cao;
  float tau_step;
  float label;             /* NaN: unusable (no leap bound) */
  uint32_t subvolume;
  int32_t counts[4];       /* species 0..3 at the recorded state */
} plis_trace_record;

typedef struct plis_learner plis_learner;

void plis_train_params_init(plis_train_params* p);
int plis_learner_create(uint64_t capacity, int device, plis_learner** out);
int plis_learner_destroy(plis_learner* learner);
/* n_steps steps of h (<= 4 species), recording every stride-th subvolume; labels use the leap
 * condition at label_epsilon (0: the handle's epsilon) */
int plis_learner_record(plis_learner* learner, plis_handle* h, uint64_t n_steps, uint32_t stride,
                        double label_epsilon);
int plis_learner_count(const plis_learner* learner, uint64_t* n_records);
int plis_learner_get_records(plis_learner* learner, uint64_t first, uint64_t n, plis_trace_record* out);
int plis_learner_set_records(plis_learner* learner, const plis_trace_record* records, uint64_t n);
/* feature statistics of the records, then p->iterations Adam steps from a fresh initialisation */
int plis_learner_train(plis_learner* learner, const plis_train_params* p, plis_train_report* out);
/* mean pinball loss and its gradient over all records (current weights and feature statistics) */
int plis_learner_gradient(plis_learner* learner, float quantile, float* grad, double* loss);
/* the MLP output y for n raw feature rows [n*8], through the inference code of the learned
 * classification: mlp_kernel 0 = tcgen05.mma (TMEM accumulators), 1 = mma.sync */
int plis_learner_predict(plis_learner* learner, const float* features, uint64_t n, float* y, int mlp_kernel);
int plis_learner_get_weights(plis_learner* learner, float* weights);       /* [PLIS_PROPOSER_WEIGHTS] */
int plis_learner_set_weights(plis_learner* learner, const float* weights);
/* Attach a proposer (weights as plis_learner_get_weights returns them) to h with clamp s_max >= 1,
 * or detach it (weights NULL or s_max <= 0).  The current state is classified again. */
int plis_set_proposer(plis_handle* h, const float* weights, double s_max);

/* ---------------------------------------------------------------------------------------------
 * Input files in the reference's formats, read unchanged (Configuration.hpp:27-144,
 * Topology.hpp:98-191, State.hpp:112-217, Reactions.hpp:132-223, cpp_utils.hpp:29-56).
 * ------------------------------------------------------------------------------------------- */
typedef struct plis_config plis_config;

typedef struct plis_config_view {
  plis_model_desc model;     /* points into the config; valid until plis_config_free */
  const uint32_t* initial_state; /* [S*N] */
  double end_time;           /* endTime (Configuration.hpp:73-77) */
  double log_freq;           /* logFreq (Configuration.hpp:80-85) */
} plis_config_view;

/* Parse conf.txt and the files it names (paths relative to the conf file's directory, falling
 * back to the current directory as the reference does).  Errors carry the reference's messages. */
int plis_config_load(const char* conf_path, plis_config** out);
int plis_config_view_get(const plis_config* cfg, plis_config_view* view);
void plis_config_free(plis_config* cfg);

/* Single-file parsers (the reference's operator>> overloads).  Arrays are allocated with malloc
 * and owned by the caller (free with plis_free). */
int plis_parse_topology(const char* path, uint32_t* n_out, uint32_t** neighbours_out);
int plis_parse_state(const char* path, uint32_t* n_out, uint32_t* s_out, uint32_t** counts_out);
int plis_parse_reactions(const char* path, uint32_t* r_out, uint32_t* s_out, int32_t** reactants_out,
                         int32_t** products_out);
void plis_free(void* p);

/* Read a .dat snapshot (the format print_state_snapshot writes, driver.cu:435-447) back: counts
 * [S*N] species-major (malloc'd, free with plis_free) and the snapshot's time, to resume a run from
 * it (plis_set_state + plis_set_time, or plis_run_simulation's start_time).  The time has the
 * snapshot's six decimals. */
int plis_read_snapshot(const char* path, uint32_t* n_out, uint32_t* s_out, double* time_out, uint32_t** counts_out);

/* Snapshot in the reference's .dat format (print_state_snapshot, driver.cu:435-447). */
int plis_write_snapshot(const char* path, const uint32_t* counts, uint32_t n, uint32_t s, double time);

#ifdef __cplusplus
}
#endif
#endif /* PLIS_H_ */

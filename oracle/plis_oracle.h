// plis_oracle.h — TEST INFRASTRUCTURE.  The host oracle of the PLISCuda simulation step.
//
// A CPU restatement (C++17, optional OpenMP) of the reference's step loop
//   PLISCuda/src/driver.cu:259-376   (min-tau, leap, SSA, check/rollback, swap, rates, taus)
//   PLISCuda/src/rates.cu:3-96       (propensities, diffusion rates, rate-matrix sums)
//   PLISCuda/src/tau.cu:3-252        (criticality, Cao g, per-species tau, tau_cr, classification)
//   PLISCuda/src/leap.cu:3-212       (Poisson leap, critical event, negativity check)
//   PLISCuda/src/ssa.cu:3-110        (single SSA event at the arg-min subvolume)
//   PLISCuda/src/init.cu:15-68       (neighbour counts, highest order of reaction)
// driven by the injected counter-based random stream of pliscuda_b200/csrc/plis_stream.h, in
// binary64 (the FP64 oracle) or binary32 (the FP32 form's oracle).  Only tests/, the smoke check
// and bench.py's CPU-baseline leg use this library; the CUDA product never links it.
#ifndef PLIS_ORACLE_H_
#define PLIS_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_model {
  uint32_t n_subvolumes;   // N
  uint32_t n_species;      // S
  uint32_t n_reactions;    // R
  uint32_t n_compartments; // C
  const uint32_t* nbr;     // [6N] canonical neighbour table: the n(c) distinct non-self neighbours first, then c itself
  const uint32_t* orig;    // [6N] table as read from the topology file (used for one reference quirk), NULL = nbr
  const int32_t* reactants;  // [S*R] species-major (PLISCuda/include/cpp/Reactions.hpp:197)
  const int32_t* products;   // [S*R]
  const double* reaction_rates;   // [C*R] compartment-major
  const double* diffusion_rates;  // [C*S]
  const int32_t* compartment;     // [N] or NULL
} oracle_model;

typedef struct oracle_options {
  int32_t mode;              // 0 = reference semantics, 1 = corrected semantics
  int32_t precision;         // 0 = binary64, 1 = binary32 propensities / Cao tau / Poisson means
  int32_t critical_threshold;  // NC (PLISCuda/src/driver.cu:36)
  int32_t max_rollbacks;       // per step
  double epsilon;              // Cao epsilon (PLISCuda/src/driver.cu:37)
  uint64_t seed;
  uint32_t replica;
  int32_t threads;             // OpenMP threads, 0 = default
  int32_t pooled_draws;        // 1 = pooled draws of small-mean leap channels, 0 = off, -1 = auto (> 4 reactions or species)
} oracle_options;

typedef struct oracle_stats {
  double time;
  uint64_t steps;
  uint64_t rollbacks;
  uint64_t events;
  uint64_t leap_events;
  uint64_t exact_events;
  int32_t stop_reason;   // 0 none, 1 time reached, 2 step budget, 3 no event possible, 4 error
  int32_t status;        // 0 ok, else an error code (7 = stuck in rollbacks, 8 = count overflow)
  double last_tau;       // tau of the last accepted step (arg-min tau)
  int64_t last_argmin;
} oracle_stats;

void* oracle_create(const oracle_model* m, const oracle_options* o);
void oracle_destroy(void* h);
int oracle_set_state(void* h, const uint32_t* counts);   // [S*N] species-major; also recomputes taus (init)
// the same for counts that continue a trajectory at time t0 after step0 accepted steps (the step
// number keys the random stream); statistics restart from zero with steps = step0
int oracle_set_state_at(void* h, const uint32_t* counts, double t0, uint64_t step0);
int oracle_get_state(void* h, uint32_t* counts);
int oracle_get_taus(void* h, double* tau, uint8_t* flags);
int oracle_get_stats(void* h, oracle_stats* st);
// Advance: stop after max_steps accepted steps or once time >= t_end (reference loop condition
// driver.cu:259), whichever first.  In corrected mode the last step is clamped to land on t_end.
int oracle_advance(void* h, double t_end, uint64_t max_steps);
// Event log: one record per event, the layout of the library's plis_event_record (the reference
// prints these events under LOG: leap.cu:29-32, 58-62, 144-146, 196-198; ssa.cu:69-71, 96-98).
typedef struct oracle_event {
  double time;          // simulated time at the start of the step
  uint64_t step;
  uint32_t subvolume;
  uint32_t target;
  uint32_t count;
  uint16_t channel;
  uint8_t kind;         // 1 leap reaction, 2 leap diffusion, 3/4 critical reaction/diffusion, 5/6 SSA
  uint8_t attempt;
} oracle_event;
void oracle_set_event_log(void* h, int on);  // on != 0: record from now on; the log starts empty
// returns the number of records logged; with out != NULL it also copies min(logged, max) of them
// into out and empties the log
int64_t oracle_read_event_log(void* h, oracle_event* out, int64_t max);
// Canonical 6-wide neighbour rows (non-self entries first, own index after them; a reflective lattice
// in the direction order -x,+x,-y,+y,-z,+z) from a topology table [6n] or, with table NULL, from
// lattice dimensions.  dims_out: the lattice's dimensions (unit dimensions last), zeros otherwise.
// Returns 0, or 1 for an entry >= n or dimensions that do not multiply to n.
int oracle_canonical_neighbours(uint32_t n, const uint32_t* table, const uint32_t* lattice, uint32_t* out,
                                uint32_t* dims_out);

#ifdef __cplusplus
}
#endif
#endif

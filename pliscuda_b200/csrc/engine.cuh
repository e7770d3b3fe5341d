// engine.cuh — device-side data of the B200 step: control block, model view, kernel arguments.
#ifndef PLIS_ENGINE_CUH_
#define PLIS_ENGINE_CUH_

#include <stdint.h>

#include "plis_stream.h"

namespace plis {

enum : uint8_t { F_LEAP_CR = 0, F_LEAP_NOCR = 1, F_SSA = 2, F_SSA_FF = 3 };  // constants.cuh:53-58

// Guards keeping every per-step sum inside int32 (identical rules in the host oracle).
constexpr int64_t kBigDraw = (int64_t)1 << 29;  // |k * nu| of one reaction draw
constexpr int64_t kBigJump = (int64_t)1 << 27;  // k of one diffusion draw
constexpr int64_t kBigTile = (int64_t)1 << 30;  // |x + own delta| of one subvolume

// The whole control state of a simulation lives on the device, so a batch of steps (rollbacks
// included) runs without the host: the reference instead reads the arg-min back and decides on
// the host every step (driver.cu:267-315).
struct Ctrl {
  double t_end;          // stop once t >= t_end
  uint64_t max_step;     // stop once step >= max_step
  double t;              // simulated time (binary64)
  uint64_t step;         // accepted steps
  double tau_min;        // arg-min of the current taus (first index on ties)
  int64_t argmin;
  double tau_step;       // corrected mode: tau_min clamped onto t_end
  double tau_leap;       // tau used by the leap of the current attempt
  double dt;             // time increment of the current attempt
  double last_tau;
  int64_t last_argmin;
  uint32_t attempt;      // rollbacks so far in the current step
  uint32_t exact;        // bit0: critical events in LEAP_CR subvolumes; bit1: arg-min exact event
  uint32_t n_leap_cr;
  uint32_t argmin_flag;
  uint32_t cur, tgt, spare, tf;  // count buffer rotation and tau/flag double-buffer index
  uint32_t phase;        // 0: initial classification pending, 1: stepping
  int32_t done, status, stop_reason;
  uint32_t blocks_done;
  uint32_t ff_free;      // 1: the classification behind the current flags left no SSA_FF subvolume (0: unknown)
  unsigned long long events, exact_events, rollbacks;
  unsigned long long ev_attempt, ex_attempt;
  // learned tau proposals (corrected mode): attempt 0 leaps with the arg-min of the proposed taus,
  // every later attempt with the plain Cao step halved once per attempt
  double tau_min_plain;  // min of the plain taus of the current state
  double tau_step_plain; // the same clamped onto t_end
  uint32_t learned;      // 1: tau_min is the min of proposed taus
  // the subvolumes whose delta rows the exact events of the attempt wrote, listed after the S x Npad
  // deltas (D + S * Npad, N entries); past N entries the list is incomplete and k_apply scans all
  uint32_t touched_on;   // 1: the delta buffer holds the list (single-replica handles)
  uint32_t n_touched;
};

struct DevModel {
  uint32_t N, S, R, C;
  uint32_t X, Y, Z, lattice;
  uint32_t Npad;
  const uint32_t* canon;   // [6N] (table topology)
  const uint8_t* ncount;   // [N]  (table topology)
  const uint32_t* orig;    // [6N] table as given (reference quirk of leap.cu:192-193), may be null
  const int32_t* comp;     // [N] or null
  const uint8_t* n_reac;
  const uint8_t* n_net;
  const uint16_t* reac_s;
  const uint8_t* reac_m;
  const int16_t* reac_nu;
  const uint16_t* net_s;
  const int16_t* net_nu;
  const double* inv_denom;
  const uint8_t* hor;
  const uint8_t* hmult;
  const uint16_t* sp_off;
  const uint16_t* sp_r;
  const int16_t* sp_nu;
  const uint16_t* sr_off;
  const uint16_t* sr_r;
  const void* rr;   // Real [C][R]
  const void* dr;   // Real [C][S]
};

// Event log of a handle (plis_set_event_log): records of 32 bytes, laid out as plis_event_record;
// rec == null when the log is off (the batched kernel never logs).
struct alignas(16) EvRec {
  double time;
  unsigned long long step;
  uint32_t subvolume, target, count;
  uint16_t channel;
  uint8_t kind, attempt;
};
static_assert(sizeof(EvRec) == 32, "EvRec must match plis_event_record");
struct EvLog {
  EvRec* rec;
  unsigned long long* head;  // events appended since the log was emptied (may exceed cap)
  unsigned long long cap;
};

struct DevBufs {
  int32_t* X[3];
  double* tau[2];
  uint8_t* flag[2];
  int32_t* D;
  double* slot_tau;
  long long* slot_idx;
  uint32_t* slot_cr;
  uint32_t* slot_bad;
  double* slot_tau_plain;  // learned classification: per-CTA min of the plain taus (else null)
  const struct LearnedParams* lp;  // learned classification: the proposer's packed weights
  uint4* feat;             // learned classification (split): normalised BF16 features, 16 B per subvolume
  double2* pre;            // (leap bound or fast-forwarded tau, critical rate) per subvolume
  uint8_t* pre_kind;       // 1: fast-forwarded, 2: leap bound computed
  float* ymlp;             // MLP output per subvolume
  Ctrl* ctrl;
  EvLog ev;                // event log (rec == null: off)
};

struct DevOpts {
  int32_t mode;
  int32_t nc;
  int32_t max_rollbacks;
  uint32_t mlp_wait;  // polls of each mbarrier wait of the tcgen05 MLP before it gives up (0: the default)
  double eps;
  unsigned long long seed;
  uint32_t replica;
  uint32_t pool;      // 1: pooled draws of small-mean channels in the generic leap (plis_stream.h)
  uint32_t rk0[10], rk1[10];  // Philox round keys of (seed, replica): plis_round_keys, set with devopts_keys
};

// Fill the round keys of o.seed / o.replica; call after either changes.
inline void devopts_keys(DevOpts& o) { plis_round_keys(o.seed, o.replica, o.rk0, o.rk1); }

// Division by a divisor fixed at set-up, as one multiply-high, two adds and two shifts: exact for
// every 32-bit numerator (Granlund and Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, section 4: m' = floor(2^32 (2^l - d) / d) + 1 with l = ceil(log2 d),
// q = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = mulhi(m', n)).
struct FastDiv {
  uint32_t mul, sh1, sh2;
};
inline FastDiv fastdiv_make(uint32_t d) {  // d >= 1
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < d) ++l;
  FastDiv f;
  f.mul = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
  f.sh1 = l < 1 ? l : 1;
  f.sh2 = l > 1 ? l - 1 : 0;
  return f;
}

struct Geo {
  uint32_t tx, ty, tz;     // lattice brick per CTA
  uint32_t ntx, nty, ntz;  // bricks per dimension
  uint32_t nblocks;        // CTAs of the cell kernels
  uint32_t threads;        // threads per CTA
  uint32_t staged;         // 1: the leap stages the brick + halo in shared memory
  uint32_t box_bytes;      // dynamic shared memory of the staged leap
  FastDiv dtx, dty, dntx, dnty;  // divisions by tx, ty, ntx, nty (geo_divisors)
};
// Sets the divisors of g from its tx, ty, ntx, nty.
inline void geo_divisors(Geo& g) {
  g.dtx = fastdiv_make(g.tx ? g.tx : 1);
  g.dty = fastdiv_make(g.ty ? g.ty : 1);
  g.dntx = fastdiv_make(g.ntx ? g.ntx : 1);
  g.dnty = fastdiv_make(g.nty ? g.nty : 1);
}

// The tables of a small model (at most kSmallR reactions and kSmallS species, one set of rate
// constants for every subvolume), held in the kernel arguments.  The step kernels built for small
// models read them from the constant bank the arguments live in, with compile-time offsets once
// their reaction and species loops are unrolled, instead of loading DevModel's tables from global
// memory for every subvolume.  The values are those of the DevModel tables (same propensities, same
// criticality, same order of summation).
constexpr int kSmallR = 4, kSmallS = 4;
// plis_options.pooled_draws resolved: auto (-1) pools the networks too large for the small-model tables
inline uint32_t pooled_draws_on(int32_t setting, uint32_t R, uint32_t S) {
  if (setting < 0) return (R > (uint32_t)kSmallR || S > (uint32_t)kSmallS) ? 1u : 0u;
  return setting != 0 ? 1u : 0u;
}
struct SmallModel {
  uint32_t on;                   // 1: the model fits and the tables below are filled
  uint8_t nreac[kSmallR];        // distinct reactant species of reaction r
  uint8_t rs[kSmallR][3];        // reactant species, increasing
  uint8_t rm[kSmallR][3];        // their multiplicities (1..3)
  int8_t rnu[kSmallR][3];        // their net change (the reference's criticality test)
  int8_t nu[kSmallR][kSmallS];   // net change of every species (0 for species >= S and reactions >= R)
  uint8_t hor[kSmallS], hmult[kSmallS];
  uint8_t rmask[kSmallS];        // bit r: species s is a reactant of reaction r
  double inv_denom[kSmallR];
  double rate_d[kSmallR];
  float rate_f[kSmallR];
  double drate_d[kSmallS];
  float drate_f[kSmallS];
};

// z-slab decomposition: this handle computes the subvolumes of whole z-layers [z0, z1) of a lattice
// whose other layers belong to other ranks.  Arrays stay full size and indices global, so random
// streams, neighbour counts and the arg-min tie rule are those of a single domain; the kernels touch
// only the slab, and the host exchanges the layers next to its faces (the ghost layers z0-1 and z1)
// with the neighbouring slabs and gathers every slab's summary.
constexpr uint32_t kExactChunk = 1024;  // subvolumes whose flags one k_exact CTA scans per round
constexpr int kSlabRemote = 64;  // flag writes of one attempt that land outside the slab and its ghosts
struct SlabSummary {             // one rank's reduction of its slab's classification
  double tau;                    // min tau over the slab
  long long idx;                 // its subvolume (global index; first on ties), -1 if none
  double tau_plain;
  unsigned long long ncr, nff;   // subvolumes flagged LEAP_CR / SSA_FF
  uint32_t bad;                  // a negative count in the slab
  uint32_t leap_bad;             // a draw beyond the int32 guards in the slab's leap
  uint32_t am_flag;              // flag of idx
  uint32_t pad_;
};
struct SlabRemote {              // subvolumes outside the slab and its ghosts whose SSA_FF flag must turn SSA
  uint32_t n;                    // entries written (may exceed kSlabRemote: then the attempt fails)
  uint32_t cell[kSlabRemote];
};
struct SlabArgs {
  uint32_t on;
  uint32_t brick0;               // first brick of the slab (bricks are numbered x fastest, z slowest)
  uint32_t lo, hi;               // owned subvolumes [lo, hi)
  uint32_t layer;                // subvolumes of one z-layer (X * Y)
  uint32_t has_lo, has_hi;       // a slab below / above
  uint32_t world, rank;
  SlabSummary* summary;          // [1] this rank's, written by the classification's last CTA
  const SlabSummary* all;        // [world] gathered
  SlabRemote* remote;            // [1] this rank's flag writes outside the slab and its ghosts
  const SlabRemote* remote_all;  // [world] gathered
  int32_t* send[2];              // [S][layer] counts then [layer] flags (as int32): 0 = to the slab below, 1 = above
  const int32_t* recv[2];        // the same layout from the slab below / above
};

struct KArgs {
  DevModel m;
  DevBufs b;
  DevOpts o;
  Geo g;
  SmallModel sm;
  SlabArgs sl;
};

}  // namespace plis

#endif

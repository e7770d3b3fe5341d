// batch_kernels.cuh — many independent replicas advanced by one persistent cooperative kernel.
//
// A batch holds replicas of one reaction network with their own reflective lattice (uneven sizes),
// their own rate constants (parameter sets) and their own random stream (replica id in the key).
// Every replica is a segment of the concatenated state arrays and is cut into bricks.  One
// cooperative launch loops over global iterations; in each, every replica that is not done takes
// one step of the single-replica algorithm (engine_kernels.cuh):
//
//   plan      every CTA scans the replicas' control blocks (identical result in every CTA): prefix sums
//             of the bricks still leaping / classifying, and whether any replica has exact events due
//   leap      CTAs take bricks from an atomic work counter (dynamic balance over uneven replicas)
//   ...       grid barrier; exact events and their deltas when due (two more barriers)
//   classify  bricks again; the last brick of a replica to finish takes that replica's decision
//             (rollback or accept, time, next plan): replicas never wait for each other
//   barrier
//
// Grid barriers spin on a generation counter with an iteration limit: a barrier that gives up sets
// an error word, every CTA leaves the loop, and the host reports PLIS_ERR_TIMEOUT.  The launch is
// cooperative, so all CTAs are co-resident.
#ifndef PLIS_BATCH_KERNELS_CUH_
#define PLIS_BATCH_KERNELS_CUH_

#include "batch.h"
#include "engine_kernels.cuh"
#include "learned_dev.cuh"

namespace plis {

constexpr int kMaxBatchReplicas = 4096;

struct RepDesc {
  uint32_t X, Y, Z, N;
  uint32_t coff;       // first subvolume of the replica in the concatenated arrays (multiple of 32)
  uint32_t tile_off;   // first brick of the replica in the global brick numbering
  uint32_t ntx, nty, ntz, ntiles;
  uint32_t replica_id; // stream key
};

struct BatchArgs {
  DevModel m;          // shared reaction tables; Npad = species stride of the concatenated arrays
  DevOpts o;
  Geo g;               // brick shape (tx, ty, tz, threads); per-replica brick counts in RepDesc
  const KArgs* views;  // [nrep] the single-replica argument block of every replica (read-only)
  const RepDesc* rep;
  uint32_t nrep;
  uint32_t rs, ss;     // rate-table strides per replica (R, S)
  const void* rr;      // Real [nrep][R]
  const void* dr;      // Real [nrep][S]
  Ctrl* ctrl;          // [nrep]
  int32_t* X[3];
  double* tau[2];
  uint8_t* flag[2];
  int32_t* D;
  double* slot_tau;    // per brick
  long long* slot_idx;
  uint32_t* slot_cr;
  uint32_t* slot_bad;
  unsigned* work;      // [4 phases][3 generations] brick / replica counters
  unsigned* bar;       // grid barrier: [0] arrivals, [1] generation
  int* err;            // 1 = a barrier timed out
  unsigned long long spin_limit;
  uint32_t max_iters;  // global iterations per launch
  uint32_t plan_off;   // byte offset of the plan arrays in dynamic shared memory (after the staging box)
};

// dynamic shared memory of k_batch: the staging box (if any), then four plan arrays of nrep + 1
__host__ __device__ inline uint32_t batch_plan_offset(uint32_t box_bytes) { return (box_bytes + 15u) & ~15u; }
__host__ __device__ inline uint32_t batch_dyn_smem(uint32_t box_bytes, uint32_t nrep) {
  return batch_plan_offset(box_bytes) + 4u * (nrep + 1u) * (uint32_t)sizeof(uint32_t);
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of a cooperative launch (the arrive / spin pattern of a grid sync) whose spin
// gives up after spin_limit polls, setting *err; returns false then.
__device__ __forceinline__ bool grid_barrier(const BatchArgs& B) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* count = B.bar;
    volatile unsigned* gen = B.bar + 1;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(count, 1u) + 1u == gridDim.x) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd((unsigned*)gen, 1u);
    } else {
      unsigned long long spins = 0;
      while (ld_acquire_gpu(B.bar + 1) == g) {
        if (++spins > B.spin_limit) {
          ok = 0;
          atomicExch(B.err, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok && *((volatile int*)B.err) == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

// next unit of a phase for this CTA: a work index in [0, total) or total when exhausted.  One CTA
// barrier per call: the index goes through one of two shared slots, alternating with `par` (the same
// sequence of calls in every thread), so a slot is rewritten only after the barrier of the next call,
// by which time every thread has read it.
__device__ __forceinline__ unsigned grab(unsigned* counter, unsigned total, unsigned& par) {
  __shared__ unsigned s_w[2];
  const unsigned slot = par;
  par ^= 1u;
  if (threadIdx.x == 0) s_w[slot] = atomicAdd(counter, 1u);
  __syncthreads();
  const unsigned w = s_w[slot];
  return w < total ? w : total;
}

// In-place inclusive prefix sums of a[0..n) and b[0..n) in shared memory by the whole CTA: each
// thread sums a contiguous chunk, the chunk sums are scanned across warps, then written back.
__device__ __forceinline__ void block_prefix2(uint32_t* a, uint32_t* b, uint32_t n) {
  __shared__ uint32_t s_wa[32], s_wb[32];
  const uint32_t nt = blockDim.x;
  const uint32_t chunk = (n + nt - 1) / nt;
  const uint32_t lo = threadIdx.x * chunk, hi = min(lo + chunk, n);
  uint32_t sa = 0, sb = 0;
  for (uint32_t i = lo; i < hi; ++i) { sa += a[i]; sb += b[i]; }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t ia = sa, ib = sb;  // inclusive warp scan
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t ta = __shfl_up_sync(0xffffffffu, ia, o), tb = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) { ia += ta; ib += tb; }
  }
  if (lane == 31) { s_wa[wid] = ia; s_wb[wid] = ib; }
  __syncthreads();
  if (wid == 0) {
    const int nw = (nt + 31) >> 5;
    uint32_t va = lane < nw ? s_wa[lane] : 0u, vb = lane < nw ? s_wb[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t ta = __shfl_up_sync(0xffffffffu, va, o), tb = __shfl_up_sync(0xffffffffu, vb, o);
      if (lane >= o) { va += ta; vb += tb; }
    }
    s_wa[lane] = va;
    s_wb[lane] = vb;
  }
  __syncthreads();
  uint32_t ra = ia - sa + (wid > 0 ? s_wa[wid - 1] : 0u);  // exclusive offset of this thread's chunk
  uint32_t rb = ib - sb + (wid > 0 ? s_wb[wid - 1] : 0u);
  for (uint32_t i = lo; i < hi; ++i) {
    ra += a[i];
    rb += b[i];
    a[i] = ra;
    b[i] = rb;
  }
  __syncthreads();
}

// The argument block of replica r, copied into shared memory when the CTA's work item moves to
// another replica (r is the CTA's work item, the same in every thread, so the branch is uniform).
// The phases then read the replica's arrays, geometry and tables from shared memory instead of
// global memory.  *svr names the replica held; it is written between the two barriers, so every
// thread reads the same value at the next call.
__device__ __forceinline__ const KArgs& replica_view(const BatchArgs& B, uint32_t r, KArgs* sv, uint32_t* svr) {
  if (*svr != r) {
    __syncthreads();  // every thread is done with the previous replica's block
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(B.views + r);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(sv);
    for (uint32_t i = threadIdx.x; i < (uint32_t)(sizeof(KArgs) / 8); i += blockDim.x) dst[i] = __ldg(src + i);
    if (threadIdx.x == 0) *svr = r;
    __syncthreads();
  }
  return *sv;
}
static_assert(sizeof(KArgs) % 8 == 0, "replica_view copies the argument block in 8-byte words");

// replica owning work index w of an inclusive-exclusive prefix array p[0..n]
__device__ __forceinline__ uint32_t find_replica(const uint32_t* p, uint32_t n, uint32_t w) {
  uint32_t lo = 0, hi = n;  // p[lo] <= w < p[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (p[mid] <= w) lo = mid;
    else hi = mid;
  }
  return lo;
}

// One kernel holds every phase, so it wants more registers than the leap alone (124 plain, 128
// learned).  Capped at 64 (4 CTAs of 256 threads per SM) it spills about 1.4 KB per thread, and is
// still faster: twice the resident warps hide more of the latency-bound phases than the spills cost.
#ifndef PLIS_BATCH_MIN_BLOCKS
#define PLIS_BATCH_MIN_BLOCKS 4
#endif
#ifndef PLIS_BATCH_MIN_BLOCKS_LEARNED
#define PLIS_BATCH_MIN_BLOCKS_LEARNED 4
#endif
// LEARNED: the classification phase takes learned tau proposals (learned_dev.cuh; corrected
// semantics, every replica's view holds the proposer and its plain-min slots).
// SM: every replica's argument block carries the SmallModel tables (small networks).
template <typename Real, int MAXS, bool LEARNED, bool SM>
__global__ void __launch_bounds__(256, LEARNED ? PLIS_BATCH_MIN_BLOCKS_LEARNED : PLIS_BATCH_MIN_BLOCKS)
    k_batch(BatchArgs B) {
  extern __shared__ int32_t s_box[];
  const uint32_t nrep = B.nrep;
  // plan: prefix sums over replicas of the work items of each phase
  uint32_t* s_lp = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(s_box) + B.plan_off);  // bricks leaping
  uint32_t* s_cp = s_lp + (nrep + 1);  // bricks classifying
  uint32_t* s_xp = s_cp + (nrep + 1);  // exact events: every brick (critical events) or one item (arg-min event)
  uint32_t* s_ap = s_xp + (nrep + 1);  // bricks applying critical-event deltas
  __shared__ int s_exact, s_apply;
  __shared__ KArgs s_view;   // the argument block of the replica this CTA works on (replica_view)
  __shared__ uint32_t s_vr;
  if (threadIdx.x == 0) s_vr = 0xFFFFFFFFu;
  __syncthreads();
  unsigned par = 0;  // slot parity of grab()
  Box box;
  box.acc = B.g.staged ? s_box : nullptr;
  box.bx = (int)B.g.tx + 2;
  box.by = (int)B.g.ty + 2;
  box.bz = (int)B.g.tz + 2;
  box.size = box.bx * box.by * box.bz;

  for (uint32_t it = 0; it < B.max_iters; ++it) {
    const uint32_t gen = it % 3u;
    // ---- plan (identical in every CTA) ----
    if (threadIdx.x == 0) { s_exact = 0; s_apply = 0; }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < nrep; r += blockDim.x) {
      const Ctrl* K = B.ctrl + r;
      const int done = __ldcg(&K->done);
      const uint32_t phase = __ldcg(&K->phase);
      const uint32_t nt = B.rep[r].ntiles;
      s_lp[r + 1] = (!done && phase == 1) ? nt : 0u;
      s_cp[r + 1] = (!done) ? nt : 0u;
      uint32_t xi = 0, ai = 0;
      if (!done && phase == 1) {
        const uint32_t ex = __ldcg(&K->exact);
        if (ex) s_exact = 1;
        if (ex & 1u) s_apply = 1;
        xi = (ex & 1u) ? nt : ((ex & 2u) ? 1u : 0u);
        ai = (ex & 1u) ? nt : 0u;
      }
      s_xp[r + 1] = xi;
      s_ap[r + 1] = ai;
    }
    if (threadIdx.x == 0) { s_lp[0] = 0; s_cp[0] = 0; s_xp[0] = 0; s_ap[0] = 0; }
    __syncthreads();
    block_prefix2(s_lp + 1, s_cp + 1, nrep);
    block_prefix2(s_xp + 1, s_ap + 1, nrep);
    const uint32_t n_leap = s_lp[nrep], n_class = s_cp[nrep];
    const int any_exact = s_exact, any_apply = s_apply;
    if (n_class == 0) break;

    // ---- leap ----
    if (n_leap > 0) {
      while (true) {
        const unsigned w = grab(B.work + 0 * 3 + gen, n_leap, par);
        if (w >= n_leap) break;
        const uint32_t r = find_replica(s_lp, nrep, w);
        const KArgs& sA = replica_view(B, r, &s_view, &s_vr);
        Ctrl* K = sA.b.ctrl;
        LeapCtx L;
        L.Xc = sA.b.X[K->cur];
        L.Xt = sA.b.X[K->tgt];
        L.flag = sA.b.flag[K->tf];
        L.step = K->step + 1;
        L.attempt = K->attempt;
        L.t = K->t;
        L.ff_free = K->ff_free != 0;
        const Real tl = (Real)K->tau_leap;
        long long ev;
        int big;
        leap_tile<Real, MAXS, false, false, SM>(sA, w - s_lp[r], L, tl, box, ev, big);
        ev = warp_sum(ev);  // events by warp, straight into the replica's counter (integer: order-free)
        if ((threadIdx.x & 31) == 0 && ev) atomicAdd(&K->ev_attempt, (unsigned long long)ev);
        if (big) atomicOr(&K->blocks_done, 0x80000000u);  // rare: an oversized draw forces a rollback
        if (box.acc) __syncthreads();  // the staging box is reused by the next brick
      }
      if (!grid_barrier(B)) return;
    }

    // ---- exact events: critical events brick by brick, the arg-min event with brick 0 ----
    if (any_exact) {
      const uint32_t n_ex = s_xp[nrep];
      while (true) {
        const unsigned w = grab(B.work + 1 * 3 + gen, n_ex, par);
        if (w >= n_ex) break;
        const uint32_t r = find_replica(s_xp, nrep, w);
        const uint32_t item = w - s_xp[r];
        const KArgs& sA = replica_view(B, r, &s_view, &s_vr);
        Ctrl* K = sA.b.ctrl;
        const uint32_t ex = K->exact;
        const int32_t* Xc = sA.b.X[K->cur];
        int32_t* Xt = sA.b.X[K->tgt];
        uint8_t* flag = sA.b.flag[K->tf];
        const uint64_t step = K->step + 1;
        const uint32_t attempt = K->attempt;
        int fired = 0;
        if (ex & 1u) {  // reference: every LEAP_CR subvolume of this brick
          Cell cl;
          if (cell_of(sA, item, cl) && flag[cl.c] == F_LEAP_CR) {
            Counts<MAXS> x;
            load_counts(sA.m, Xc, cl.c, x);
            fired += critical_event_ref<Real, false>(sA, cl.c, x, Xt, step, attempt, sA.b.D, flag);
          }
        }
        if ((ex & 2u) && item == 0 && threadIdx.x == 0) {
          const uint32_t am = (uint32_t)K->argmin;
          const uint8_t fa = flag[am];
          Counts<MAXS> x;
          load_counts(sA.m, Xc, am, x);
          int32_t* dst = (ex & 1u) ? sA.b.D : Xt;
          if (sA.o.mode == 0) {
            if (fa == F_SSA || fa == F_SSA_FF) fired += argmin_event<Real, false>(sA, am, x, step, attempt, dst, flag, false);
          } else if (fa == F_LEAP_CR) {
            fired += argmin_event<Real, false>(sA, am, x, step, attempt, dst, flag, true);
          } else if (fa == F_SSA || fa == F_SSA_FF) {
            fired += argmin_event<Real, false>(sA, am, x, step, attempt, dst, flag, false);
          }
        }
        if (fired) {  // exact events are rare: one atomic per firing thread
          atomicAdd(&K->ev_attempt, (unsigned long long)fired);
          atomicAdd(&K->ex_attempt, (unsigned long long)fired);
        }
      }
      if (!grid_barrier(B)) return;
      if (any_apply) {  // the staged critical-event deltas, brick by brick
        const uint32_t n_ap = s_ap[nrep];
        while (true) {
          const unsigned w = grab(B.work + 2 * 3 + gen, n_ap, par);
          if (w >= n_ap) break;
          const uint32_t r = find_replica(s_ap, nrep, w);
          const KArgs& sA = replica_view(B, r, &s_view, &s_vr);
          const Ctrl* K = sA.b.ctrl;
          Cell cl;
          if (cell_of(sA, w - s_ap[r], cl)) {
            int32_t* Xt = sA.b.X[__ldcg(&K->tgt)];
            int32_t* Dr = sA.b.D;
            for (uint32_t sp = 0; sp < sA.m.S; ++sp) {
              const size_t i = (size_t)sp * sA.m.Npad + cl.c;
              const int32_t v = Dr[i];
              if (v) {
                Xt[i] += v;
                Dr[i] = 0;
              }
            }
          }
        }
        if (!grid_barrier(B)) return;
      }
    }

    // ---- classify + per-replica control ----
    while (true) {
      const unsigned w = grab(B.work + 3 * 3 + gen, n_class, par);
      if (w >= n_class) break;
      const uint32_t r = find_replica(s_cp, nrep, w);
      const KArgs& sA = replica_view(B, r, &s_view, &s_vr);
      Ctrl* K = sA.b.ctrl;
      const ClassifyCtx C = classify_ctx(sA, K);
      const uint32_t tile = w - s_cp[r];
      if constexpr (LEARNED) {
        if (learned_classify_tile<Real, MAXS, false>(sA, K, C, tile, sA.g.nblocks)) classify_control(sA, K, sA.g.nblocks);
      } else {
        double tn;
        long long ti;
        int fl, bad;
        bool valid;
        classify_tile<Real, MAXS, false, false, SM>(sA, tile, C, tn, ti, fl, bad, valid);
        if (classify_slot(sA, K, tile, sA.g.nblocks, tn, ti, valid && fl == F_LEAP_CR, bad, valid && fl == F_SSA_FF))
          classify_control(sA, K, sA.g.nblocks);
      }
      __syncthreads();
    }
    if (!grid_barrier(B)) return;
    // counters of generation it+2 (== it-1) are no longer in use by any CTA
    if (blockIdx.x == 0 && threadIdx.x < 4) B.work[threadIdx.x * 3 + (it + 2) % 3] = 0u;
  }
}

template <typename Real, int MAXS, bool LEARNED, bool SM>
struct BatchKernelSet {
  static void* kernel() { return (void*)&k_batch<Real, MAXS, LEARNED, SM>; }
  static cudaError_t set_smem(int bytes) {
    return cudaFuncSetAttribute(k_batch<Real, MAXS, LEARNED, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }
};

template <typename Real, bool LEARNED>
BatchLaunch batch_pick_impl(uint32_t S, bool small) {
  if (small) {  // the SmallModel tables hold up to kSmallS species
    if (S <= 1) return {BatchKernelSet<Real, 1, LEARNED, true>::kernel(), BatchKernelSet<Real, 1, LEARNED, true>::set_smem};
    if (S <= 2) return {BatchKernelSet<Real, 2, LEARNED, true>::kernel(), BatchKernelSet<Real, 2, LEARNED, true>::set_smem};
    return {BatchKernelSet<Real, 4, LEARNED, true>::kernel(), BatchKernelSet<Real, 4, LEARNED, true>::set_smem};
  }
  if (S <= 1) return {BatchKernelSet<Real, 1, LEARNED, false>::kernel(), BatchKernelSet<Real, 1, LEARNED, false>::set_smem};
  if (S <= 2) return {BatchKernelSet<Real, 2, LEARNED, false>::kernel(), BatchKernelSet<Real, 2, LEARNED, false>::set_smem};
  if (S <= 4) return {BatchKernelSet<Real, 4, LEARNED, false>::kernel(), BatchKernelSet<Real, 4, LEARNED, false>::set_smem};
  if constexpr (LEARNED) {
    return {nullptr, nullptr};  // learned proposals: up to 4 species
  } else {
    if (S <= 8) return {BatchKernelSet<Real, 8, false, false>::kernel(), BatchKernelSet<Real, 8, false, false>::set_smem};
    return {BatchKernelSet<Real, 16, false, false>::kernel(), BatchKernelSet<Real, 16, false, false>::set_smem};
  }
}

}  // namespace plis

#endif

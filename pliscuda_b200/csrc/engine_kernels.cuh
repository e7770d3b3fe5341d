// engine_kernels.cuh — the device phases of the B200 simulation step (sm_100a).
//
// One tau-leaping step of the reference (PLISCuda/src/driver.cu:259-376) is four device phases,
// with every decision taken on the device so that batches of steps replay as one CUDA graph:
//
//   k_leap      Poisson firings of non-critical reactions and per-neighbour diffusions of every
//               LEAP subvolume (leap.cu:3-65).  Each thread owns one subvolume of a lattice brick;
//               the brick's own values and the molecules it sends are reduced into the zeroed
//               target buffer with int32 atomics (commutative, so the result is deterministic).
//   k_exact     the single critical event of every LEAP_CR subvolume (leap.cu:67-199) and the exact
//               event of the arg-min subvolume (ssa.cu:270-324).  Decisions read the pre-step counts
//               and the post-leap counts; the reference's race on the latter (leap.cu:131-134) is
//               gone because the changes are staged in a delta buffer.
//   k_apply     adds the staged deltas (reference mode with critical events only).
//   k_classify  negativity check (check_state, leap.cu:203-212), rates, criticality, Cao tau,
//               tau_cr, flags and fast-forward (rates.cu, tau.cu:197-252) of the post-step state,
//               a warp-shuffle + CTA min-tau with arg-min, and in the last CTA to finish: the
//               grid-wide arg-min, rollback-or-accept, the time update and the next step's plan
//               (driver.cu:267-334).  It also zeroes the buffer the next leap will reduce into.
//
// Counts are int32 species-major [S][Npad] in three rotating buffers (current, target, spare), so
// accepting a step is an index rotation and a rollback discards the target: no device-to-device
// copies (the reference copies the state twice per step, driver.cu:303, :323).
#ifndef PLIS_ENGINE_KERNELS_CUH_
#define PLIS_ENGINE_KERNELS_CUH_

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "../../include/plis.h"
#include "engine.cuh"
#include "engine.h"
#include "plis_stream.h"

namespace plis {

// ------------------------------------------------------------------------------------------------
// precision traits
// ------------------------------------------------------------------------------------------------
// Programmatic dependent launch.  Every kernel of the step loop starts by waiting until its
// predecessor in the stream has completed and its writes are visible (griddepcontrol.wait), then
// lets its successor begin launching (griddepcontrol.launch_dependents): the successor's launch and
// CTA scheduling overlap this kernel's tail instead of following it.  Results are unchanged; launched
// without the attribute (launch_pdl) both instructions are no-ops.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// One event record appended to the log.  The threads that reach this call together reserve their
// slots with one atomic per warp; slots past the capacity are counted in the head but not written.
__device__ __forceinline__ void ev_put(const EvLog& L, double t, uint64_t step, uint32_t attempt, uint32_t cell,
                                    uint32_t target, long long count, int channel, int kind) {
  namespace cg = cooperative_groups;
  const cg::coalesced_group g = cg::coalesced_threads();
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(L.head, (unsigned long long)g.size());
  base = g.shfl(base, 0) + g.thread_rank();
  if (base >= L.cap) return;
  EvRec r;
  r.time = t;
  r.step = step;
  r.subvolume = cell;
  r.target = target;
  r.count = count > 0xFFFFFFFFll ? 0xFFFFFFFFu : (uint32_t)count;
  r.channel = (uint16_t)channel;
  r.kind = (uint8_t)kind;
  r.attempt = attempt > 255u ? (uint8_t)255 : (uint8_t)attempt;
  L.rec[base] = r;
}

template <typename Kern, typename... Args>
inline void launch_pdl(Kern kern, dim3 g, dim3 b, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

template <typename Real> struct RT;
template <> struct RT<double> {
  static __device__ __forceinline__ double poisson(plis_stream* s, double lam) { return plis_poisson_d(s, lam); }
  // lam >= 0 (a rate times a count times tau): below the inversion limit e^-lam is a normal number
  static __device__ __forceinline__ double emlam(double lam) { return lam < PLIS_LEAP_INV_MAX ? plis_exp_normal(-lam) : 0.0; }
  static __device__ __forceinline__ double poisson_shared(plis_stream* s, double lam, double em) {
    if (!(lam > 0.0)) return 0.0;
    return lam < PLIS_LEAP_INV_MAX ? plis_poisson_small_d(s, lam, em) : plis_poisson_d(s, lam);
  }
  static __device__ __forceinline__ double uniform(plis_stream* s) { return plis_uniform_d(s); }
  static __device__ __forceinline__ long long count(double k) { return plis_count_d(k); }
  static __device__ __forceinline__ double inf() { return PLIS_INF_D; }
  // a 32-bit word of a group block as a uniform, and a Poisson draw by inversion from it
  static __device__ __forceinline__ double word_uniform(uint32_t w) { return plis_u32_to_uniform_d(w); }
  static __device__ __forceinline__ double inv_word(uint32_t w, double lam) {
    return plis_poisson_inv_d(plis_u32_to_uniform_d(w), lam, plis_exp(-lam));
  }
};
template <> struct RT<float> {
  static __device__ __forceinline__ double poisson(plis_stream* s, float lam) { return plis_poisson_f(s, lam); }
  static __device__ __forceinline__ float emlam(float lam) {
    return lam < (float)PLIS_LEAP_INV_MAX ? plis_expf_normal(-lam) : 0.0f;
  }
  static __device__ __forceinline__ double poisson_shared(plis_stream* s, float lam, float em) {
    if (!(lam > 0.0f)) return 0.0;
    return lam < (float)PLIS_LEAP_INV_MAX ? plis_poisson_small_f(s, lam, em) : plis_poisson_d(s, (double)lam);
  }
  static __device__ __forceinline__ float uniform(plis_stream* s) { return plis_uniform_f(s); }
  static __device__ __forceinline__ long long count(double k) { return plis_count_d(k); }
  static __device__ __forceinline__ float inf() { return PLIS_INF_F; }
  static __device__ __forceinline__ float word_uniform(uint32_t w) { return plis_u32_to_uniform_f(w); }
  static __device__ __forceinline__ double inv_word(uint32_t w, float lam) {
    return plis_poisson_inv_f(plis_u32_to_uniform_f(w), lam, plis_expf(-lam));
  }
};

// Per-neighbour diffusion draws of one species (leap.cu:49-53).  All n draws have the same mean, so
// for lam < PLIS_LEAP_INV_MAX the inversion CDF is built once, up to the largest of the n uniforms, and each draw
// reads its result off it: identical results to n separate sequential searches
// (plis_poisson_small_d / _f), max_j k_j iterations instead of sum_j k_j.
template <typename Real> struct DiffTraits;
template <> struct DiffTraits<double> {
  static __device__ __forceinline__ double uni(plis_stream* s) { return plis_uniform_d(s); }
  static __device__ __forceinline__ void group(const plis_stream* g, uint32_t need, double* u, int n) {
    plis_group_uniforms_d(g, need, u, n);
  }
  static __device__ __forceinline__ void group_rk(const plis_stream* g, uint32_t need, double* u, int n, const DevOpts& o) {
    plis_group_uniforms_rk_d(g, need, u, n, o.rk0, o.rk1);
  }
  static constexpr double tail = 8.673617379884035e-19;
  static constexpr int kmax = 200;
  // The searches below read binary64 group uniforms, u <= 1 - 2^-33, with means below 20.  Their tail
  // test p <= F 2^-60 cannot change a result there, so it is left out (the k >= kmax bound stays):
  // p_k > e^-20 / 16 > 2^-60 for k <= 2 lambda, so the test could only fire at some k > 2 lambda, where
  // p_{j+1} / p_j < 1/2 and the mass beyond k is below p_k <= 2^-60; the computed F_k is within
  // 4 k 2^-53 < 2^-44 of the exact CDF (k < 100), so F_k > 1 - 2^-43 > u: the search has already
  // stopped on u <= F.
  static constexpr bool tail_test = false;
};
template <> struct DiffTraits<float> {
  static __device__ __forceinline__ float uni(plis_stream* s) { return plis_uniform_f(s); }
  static __device__ __forceinline__ void group(const plis_stream* g, uint32_t need, float* u, int n) {
    plis_group_uniforms_f(g, need, u, n);
  }
  static __device__ __forceinline__ void group_rk(const plis_stream* g, uint32_t need, float* u, int n, const DevOpts& o) {
    plis_group_uniforms_rk_f(g, need, u, n, o.rk0, o.rk1);
  }
  static constexpr float tail = 2.9802322e-08f;
  static constexpr int kmax = 100;
  // binary32: the rounding of F can leave it below a uniform near 1, so the stop test is needed
  static constexpr bool tail_test = true;
};

template <typename Real, bool RK = false>
__device__ __forceinline__ void diffusion_draws(const KArgs& A, uint32_t c, int s, int n, Real lam, Real em,
                                                uint64_t step, uint32_t attempt, int32_t k[6]) {
  if (!(lam > (Real)0)) {
#pragma unroll
    for (int j = 0; j < 6; ++j) k[j] = 0;
    return;
  }
  if (!(lam < (Real)PLIS_LEAP_INV_MAX)) {
#pragma unroll
    for (int j = 0; j < 6; ++j) k[j] = 0;
#pragma unroll 1
    for (int j = 0; j < n; ++j) {  // one inlined PTRS for the n slots
      plis_stream st = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_diff(s, j));
      const long long kj = plis_count_d(plis_poisson_d(&st, (double)lam));
      const int32_t v = (int32_t)(kj < kBigJump ? kj : kBigJump);  // a jump of 2^27 or more rolls the attempt back
#pragma unroll
      for (int t = 0; t < 6; ++t)
        if (t == j) k[t] = v;
    }
    return;
  }
  Real u[6];
  bool open_[6];
  Real p = em, F = em;
  bool pending = false;
#pragma unroll
  for (int j = 0; j < 6; ++j) u[j] = (Real)0;
  {  // the slots' uniforms from the species' grouped blocks
    const plis_stream g = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_dgroup(s));
    if constexpr (RK) DiffTraits<Real>::group_rk(&g, (1u << n) - 1u, u, 6, A.o);
    else DiffTraits<Real>::group(&g, (1u << n) - 1u, u, 6);
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    open_[j] = false;
    k[j] = 0;
    if (j < n) {
      open_[j] = u[j] > F;
      pending |= open_[j];
    }
  }
  int ki = 0;
  while (pending) {
    ki += 1;
    p = (p * lam) * (Real)plis_inv_k_tab[ki];
    F += p;
    const bool brk = (DiffTraits<Real>::tail_test && p <= F * DiffTraits<Real>::tail) || ki >= DiffTraits<Real>::kmax;
    pending = false;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (open_[j] && (!(u[j] > F) || brk)) {
        open_[j] = false;
        k[j] = ki;
      }
      pending |= open_[j];
    }
  }
}

// Up to 4 reaction draws with means in (0, 10) advanced in lockstep: each is exactly the sequential
// search of plis_poisson_small_d / _f (same arithmetic per draw), but the independent chains give
// the FP64 pipe four times the instruction-level parallelism and the loop runs max_i k_i times.
template <typename Real>
__device__ __forceinline__ void batched_small_draws(const Real u[4], const Real lam[4], const bool act[4], long long k[4]) {
  Real p[4], F[4];
  bool open_[4];
  bool pending = false;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    k[i] = 0;
    open_[i] = false;
    p[i] = F[i] = (Real)0;
    if (act[i]) {
      p[i] = RT<Real>::emlam(lam[i]);
      F[i] = p[i];
      open_[i] = u[i] > F[i];
      pending |= open_[i];
    }
  }
  // two terms per pass (k = ki + 1, ki + 2): the same arithmetic, half the loop overhead; kmax is even,
  // so ki + 2 <= kmax and the table index stays in range
  static_assert(DiffTraits<Real>::kmax % 2 == 0, "two terms per pass need an even kmax");
  int ki = 0;
  while (pending) {
    const Real ik1 = (Real)plis_inv_k_tab[ki + 1];
    const Real ik2 = (Real)plis_inv_k_tab[ki + 2];
    pending = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (open_[i]) {
        p[i] = (p[i] * lam[i]) * ik1;
        F[i] += p[i];
        const bool brk1 = (DiffTraits<Real>::tail_test && p[i] <= F[i] * DiffTraits<Real>::tail) ||
                          ki + 1 >= DiffTraits<Real>::kmax;
        if (!(u[i] > F[i]) || brk1) {
          open_[i] = false;
          k[i] = ki + 1;
        } else {
          p[i] = (p[i] * lam[i]) * ik2;
          F[i] += p[i];
          const bool brk2 = (DiffTraits<Real>::tail_test && p[i] <= F[i] * DiffTraits<Real>::tail) ||
                            ki + 2 >= DiffTraits<Real>::kmax;
          if (!(u[i] > F[i]) || brk2) {
            open_[i] = false;
            k[i] = ki + 2;
          }
        }
        pending |= open_[i];
      }
    }
    ki += 2;
  }
}

// Per-thread copy of one subvolume's counts.  Small species counts stay in registers: the
// selection loops below use compile-time indices only.
template <int MAXS> struct Counts {
  int32_t v[MAXS];
  __device__ __forceinline__ int32_t get(int s) const {
    if (MAXS <= 8) {
      int32_t r = 0;
#pragma unroll
      for (int i = 0; i < MAXS; ++i)
        if (i == s) r = v[i];
      return r;
    }
    return v[s];
  }
};
template <int MAXS> struct Deltas {
  long long v[MAXS];
  __device__ __forceinline__ void add(int s, long long d) {
    if (MAXS <= 8) {
#pragma unroll
      for (int i = 0; i < MAXS; ++i)
        if (i == s) v[i] += d;
      return;
    }
    v[s] += d;
  }
};

// ------------------------------------------------------------------------------------------------
// geometry
// ------------------------------------------------------------------------------------------------
struct Cell {
  uint32_t c;        // linear index
  uint32_t x, y, z;  // lattice coordinates (lattice topology only)
};

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
  const uint32_t t = __umulhi(f.mul, n);
  return (t + ((n - t) >> f.sh1)) >> f.sh2;
}

__device__ __forceinline__ bool cell_of(const KArgs& A, uint32_t block, Cell& cl) {
  if (A.m.lattice) {
    const uint32_t b = block + A.sl.brick0, t = threadIdx.x;  // brick0: first brick of a z-slab (0 otherwise)
    if (t >= A.g.tx * A.g.ty * A.g.tz) return false;  // block rounded up to whole warps
    const uint32_t br = fdiv(b, A.g.dntx), bx = b - br * A.g.ntx;
    const uint32_t bz = fdiv(br, A.g.dnty), by = br - bz * A.g.nty;
    const uint32_t tr = fdiv(t, A.g.dtx), lx = t - tr * A.g.tx;
    const uint32_t lz = fdiv(tr, A.g.dty), ly = tr - lz * A.g.ty;
    cl.x = bx * A.g.tx + lx;
    cl.y = by * A.g.ty + ly;
    cl.z = bz * A.g.tz + lz;
    if (cl.x >= A.m.X || cl.y >= A.m.Y || cl.z >= A.m.Z) return false;
    cl.c = cl.x + A.m.X * (cl.y + A.m.Y * cl.z);
    return true;
  }
  cl.c = block * blockDim.x + threadIdx.x;
  cl.x = cl.y = cl.z = 0;
  return cl.c < A.m.N;
}
__device__ __forceinline__ bool cell_of(const KArgs& A, uint32_t& c) {
  Cell cl;
  const bool v = cell_of(A, blockIdx.x, cl);
  c = cl.c;
  return v;
}

// Canonical neighbours of a subvolume and their own neighbour counts.  Lattice rows are
// -x,+x,-y,+y,-z,+z (absent ones skipped), derived from the coordinates without divisions.
struct Nbr {
  uint32_t nb[6];
  uint8_t nn[6];
  uint8_t dir[6];  // lattice direction of each slot: 0..5 = -x,+x,-y,+y,-z,+z
  int n;
  // lattice: the subvolume, its coordinates and neighbours per axis (for_each_nbr walks the
  // directions from these; nbr_lite fills nothing else)
  int lat;
  uint32_t c, x, y, z;
  int ax, ay, az;
};

__device__ __forceinline__ int axis_count(uint32_t v, uint32_t dim) { return (v > 0) + (v + 1 < dim); }

__device__ __forceinline__ void nbr_scalars(const DevModel& m, const Cell& cl, Nbr& q) {
  q.lat = (int)m.lattice;
  q.c = cl.c;
  q.x = cl.x;
  q.y = cl.y;
  q.z = cl.z;
  if (m.lattice) {
    q.ax = axis_count(cl.x, m.X);
    q.ay = axis_count(cl.y, m.Y);
    q.az = axis_count(cl.z, m.Z);
    q.n = q.ax + q.ay + q.az;
  }
}

__device__ __forceinline__ void nbr_info(const DevModel& m, const Cell& cl, Nbr& q) {
  const uint32_t c = cl.c;
  nbr_scalars(m, cl, q);
  if (m.lattice) {
    const uint32_t X = m.X, Y = m.Y, Z = m.Z, XY = m.X * m.Y;
    const int ax = axis_count(cl.x, X), ay = axis_count(cl.y, Y), az = axis_count(cl.z, Z);
    int n = 0;
    if (cl.x > 0) { q.nb[n] = c - 1; q.dir[n] = 0; q.nn[n++] = (uint8_t)(axis_count(cl.x - 1, X) + ay + az); }
    if (cl.x + 1 < X) { q.nb[n] = c + 1; q.dir[n] = 1; q.nn[n++] = (uint8_t)(axis_count(cl.x + 1, X) + ay + az); }
    if (cl.y > 0) { q.nb[n] = c - X; q.dir[n] = 2; q.nn[n++] = (uint8_t)(ax + axis_count(cl.y - 1, Y) + az); }
    if (cl.y + 1 < Y) { q.nb[n] = c + X; q.dir[n] = 3; q.nn[n++] = (uint8_t)(ax + axis_count(cl.y + 1, Y) + az); }
    if (cl.z > 0) { q.nb[n] = c - XY; q.dir[n] = 4; q.nn[n++] = (uint8_t)(ax + ay + axis_count(cl.z - 1, Z)); }
    if (cl.z + 1 < Z) { q.nb[n] = c + XY; q.dir[n] = 5; q.nn[n++] = (uint8_t)(ax + ay + axis_count(cl.z + 1, Z)); }
    q.n = n;
    for (int j = n; j < 6; ++j) { q.nb[j] = c; q.nn[j] = 0; q.dir[j] = 0; }
    return;
  }
  q.n = m.ncount[c];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    q.nb[j] = m.canon[(size_t)c * 6 + j];
    q.nn[j] = j < q.n ? m.ncount[q.nb[j]] : 0;
    q.dir[j] = 0;
  }
}

// The neighbours without the slot arrays on a lattice (they are walked by direction instead);
// a neighbour table fills them as nbr_info does.
__device__ __forceinline__ void nbr_lite(const DevModel& m, const Cell& cl, Nbr& q) {
  if (m.lattice) nbr_scalars(m, cl, q);
  else nbr_info(m, cl, q);
}

// Lattice neighbour in direction d (0..5 = -x,+x,-y,+y,-z,+z): false when absent, else its index and
// its own neighbour count.
__device__ __forceinline__ bool nbr_dir(const DevModel& m, const Nbr& q, int d, uint32_t& b, int& nn) {
  switch (d) {
    case 0: b = q.c - 1; nn = axis_count(q.x - 1, m.X) + q.ay + q.az; return q.x > 0;
    case 1: b = q.c + 1; nn = axis_count(q.x + 1, m.X) + q.ay + q.az; return q.x + 1 < m.X;
    case 2: b = q.c - m.X; nn = q.ax + axis_count(q.y - 1, m.Y) + q.az; return q.y > 0;
    case 3: b = q.c + m.X; nn = q.ax + axis_count(q.y + 1, m.Y) + q.az; return q.y + 1 < m.Y;
    case 4: b = q.c - m.X * m.Y; nn = q.ax + q.ay + axis_count(q.z - 1, m.Z); return q.z > 0;
    default: b = q.c + m.X * m.Y; nn = q.ax + q.ay + axis_count(q.z + 1, m.Z); return q.z + 1 < m.Z;
  }
}

// f(b, nn) for each neighbour in slot order (on a lattice: the present directions in order), fully
// unrolled so that the neighbours' loads issue together.
template <class F>
__device__ __forceinline__ void for_each_nbr(const DevModel& m, const Nbr& q, F&& f) {
  if (q.lat) {
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      uint32_t b;
      int nn;
      if (nbr_dir(m, q, d, b, nn)) f(b, nn);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (j >= q.n) break;
      f(q.nb[j], (int)q.nn[j]);
    }
  }
}

// canonical neighbours of a subvolume given only its index (rare paths: exact events)
__device__ __forceinline__ int nbrs(const DevModel& m, uint32_t c, uint32_t nb[6]) {
  if (m.lattice) {
    const uint32_t X = m.X, Y = m.Y, Z = m.Z;
    const uint32_t x = c % X, y = (c / X) % Y, z = c / (X * Y);
    int n = 0;
    if (x > 0) nb[n++] = c - 1;
    if (x + 1 < X) nb[n++] = c + 1;
    if (y > 0) nb[n++] = c - X;
    if (y + 1 < Y) nb[n++] = c + X;
    if (z > 0) nb[n++] = c - X * Y;
    if (z + 1 < Z) nb[n++] = c + X * Y;
    return n;
  }
  const int n = m.ncount[c];
#pragma unroll
  for (int j = 0; j < 6; ++j) nb[j] = m.canon[(size_t)c * 6 + j];
  return n;
}

// slot-th entry of the canonical 6-wide row of c (self padding beyond the neighbour count)
__device__ __forceinline__ uint32_t canon_slot(const DevModel& m, uint32_t c, int slot) {
  if (!m.lattice) return m.canon[(size_t)c * 6 + slot];
  uint32_t nb[6];
  const int n = nbrs(m, c, nb);
  uint32_t r = c;
#pragma unroll
  for (int j = 0; j < 6; ++j)
    if (j == slot && j < n) r = nb[j];
  return r;
}

// the flat table entry the reference reads at leap.cu:192 (neigh.index[rdi])
__device__ __forceinline__ uint32_t flat_table_entry(const DevModel& m, uint32_t flat) {
  if (m.orig) return m.orig[flat];
  return canon_slot(m, flat / 6, (int)(flat % 6));
}

__device__ __forceinline__ int comp_of(const DevModel& m, uint32_t c) { return m.comp ? m.comp[c] : 0; }

// ------------------------------------------------------------------------------------------------
// per-subvolume rates (rates.cu:3-96) and criticality (tau.cu:3-45)
// ------------------------------------------------------------------------------------------------
template <typename Real, int MAXS>
__device__ __forceinline__ Real prop(const DevModel& m, const Counts<MAXS>& x, int r, int comp) {
  const Real* rr = (const Real*)m.rr;
  const int nr = m.n_reac[r];
  Real prod = (Real)1;
  for (int i = 0; i < nr; ++i) {
    const int s = m.reac_s[r * 3 + i];
    const int mu = m.reac_m[r * 3 + i];
    const Real xs = (Real)x.get(s);
    for (int j = 0; j < mu; ++j) prod = prod * (xs - (Real)j);
  }
  return (rr[(size_t)comp * m.R + r] * prod) * (Real)m.inv_denom[r];
}

template <typename Real>
__device__ __forceinline__ Real drate(const DevModel& m, int comp, int s) {
  return ((const Real*)m.dr)[(size_t)comp * m.S + s];
}

// reference criticality: the first two reactant species decide (tau.cu:3-40)
template <int MAXS>
__device__ __forceinline__ bool crit_ref(const DevModel& m, const Counts<MAXS>& x, int r, int nc) {
  const int nr = m.n_reac[r];
  const int lim = nr < 2 ? nr : 2;
  bool crit = false;
  for (int i = 0; i < lim; ++i) {
    const int s = m.reac_s[r * 3 + i];
    const int32_t xs = x.get(s);
    if (xs == 0) return true;
    const int nu = m.reac_nu[r * 3 + i];
    if (nu < 0 && (long long)(-nu) * nc > xs) crit = true;
  }
  return crit;
}

// corrected criticality: a > 0 and L_j = min_{nu<0} floor(x/|nu|) < NC (Cao, Gillespie, Petzold 2005)
template <typename Real, int MAXS>
__device__ __forceinline__ bool crit_fix(const DevModel& m, const Counts<MAXS>& x, int r, Real a, int nc) {
  if (!(a > (Real)0)) return false;
  const int nn = m.n_net[r];
  for (int i = 0; i < nn; ++i) {
    const int nu = m.net_nu[r * 8 + i];
    if (nu < 0 && x.get(m.net_s[r * 8 + i]) < (long long)(-nu) * nc) return true;
  }
  return false;
}

// Cao's g (tau.cu:47-66 for orders <= 2; orders 3 per Cao, Gillespie, Petzold 2006)
template <typename Real>
__device__ __forceinline__ Real gfun(int hor, int hmult, int32_t x) {
  const Real xr = (Real)x;
  switch (hor) {
    case 0: return RT<Real>::inf();
    case 1: return (Real)1;
    case 2:
      if (hmult == 1) return (Real)2;
      return (Real)2 + (Real)1 / (xr - (Real)1);
    default:
      if (hmult == 1) return (Real)3;
      if (hmult == 2) return (Real)1.5 * ((Real)2 + (Real)1 / (xr - (Real)1));
      return ((Real)3 + (Real)1 / (xr - (Real)1)) + (Real)2 / (xr - (Real)2);
  }
}

// Small models (SmallModel in the kernel arguments): the same propensity, criticality and rate
// constants as prop / crit_ref / crit_fix / drate above, from the argument tables.  The product of
// falling factorials is formed in the same order (reactant species increasing, x, x-1, x-2).
template <typename Real> __device__ __forceinline__ Real sm_rate(const SmallModel& t, int r);
template <> __device__ __forceinline__ double sm_rate<double>(const SmallModel& t, int r) { return t.rate_d[r]; }
template <> __device__ __forceinline__ float sm_rate<float>(const SmallModel& t, int r) { return t.rate_f[r]; }
template <typename Real> __device__ __forceinline__ Real sm_drate(const SmallModel& t, int s);
template <> __device__ __forceinline__ double sm_drate<double>(const SmallModel& t, int s) { return t.drate_d[s]; }
template <> __device__ __forceinline__ float sm_drate<float>(const SmallModel& t, int s) { return t.drate_f[s]; }

template <typename Real, int MAXS>
__device__ __forceinline__ Real prop_sm(const SmallModel& t, const Counts<MAXS>& x, int r) {
  Real prod = (Real)1;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (i < t.nreac[r]) {
      const Real xs = (Real)x.get(t.rs[r][i]);
      const int mu = t.rm[r][i];
      prod = prod * xs;
      if (mu > 1) prod = prod * (xs - (Real)1);
      if (mu > 2) prod = prod * (xs - (Real)2);
    }
  }
  return (sm_rate<Real>(t, r) * prod) * (Real)t.inv_denom[r];
}

template <int MAXS>
__device__ __forceinline__ bool crit_ref_sm(const SmallModel& t, const Counts<MAXS>& x, int r, int nc) {
  const int lim = t.nreac[r] < 2 ? t.nreac[r] : 2;
  bool crit = false;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    if (i < lim) {
      const int32_t xs = x.get(t.rs[r][i]);
      if (xs == 0) return true;
      const int nu = t.rnu[r][i];
      if (nu < 0 && (long long)(-nu) * nc > xs) crit = true;
    }
  }
  return crit;
}

template <typename Real, int MAXS>
__device__ __forceinline__ bool crit_fix_sm(const SmallModel& t, const Counts<MAXS>& x, int r, Real a, int nc) {
  if (!(a > (Real)0)) return false;
  bool crit = false;
#pragma unroll
  for (int s = 0; s < MAXS; ++s) {
    const int nu = t.nu[r][s];
    if (nu < 0 && x.v[s] < (long long)(-nu) * nc) crit = true;
  }
  return crit;
}

template <int MAXS>
__device__ __forceinline__ void load_counts(const DevModel& m, const int32_t* X, uint32_t c, Counts<MAXS>& x) {
#pragma unroll
  for (int s = 0; s < MAXS; ++s) x.v[s] = (s < (int)m.S) ? X[(size_t)s * m.Npad + c] : 0;
}

// ------------------------------------------------------------------------------------------------
// classification of one subvolume (compute_taus, tau.cu:197-252)
// ------------------------------------------------------------------------------------------------
// Fast-forward of an SSA_FF subvolume (tau.cu:214-217): true when the subvolume keeps its flag and
// its tau is decremented by the time advanced.
__device__ __forceinline__ bool classify_ff(int mode, double tau_cur, uint8_t flag_cur, uint64_t step, double ff,
                                            double& tau_out, int& flag_out) {
  if (step > 0 && flag_cur == F_SSA_FF && !plis_isinf_d(tau_cur)) {
    if (mode == 0) {
      if (ff > 0.0 && ff != tau_cur) { tau_out = tau_cur - ff; flag_out = F_SSA_FF; return true; }
    } else if (tau_cur > ff) {
      tau_out = tau_cur - ff;
      flag_out = F_SSA_FF;
      return true;
    }
  }
  return false;
}

// The deterministic part of compute_taus (tau.cu:68-195): the Cao leap bound tau_ncr over the
// species that enter it, and the rate whose exponential time is tau_cr (critical channels; in
// corrected mode, all channels of a subvolume without a leap bound).
// WALK: the neighbour loops are unrolled (for_each_nbr); with WALK false they run to the run-time
// count over nbr_info's slot arrays, which needs fewer registers where the kernel arguments live in
// global memory (the batched kernel's per-replica views).
// CACHE: every propensity and criticality of the subvolume is evaluated once, the propensities
// into the thread's column of `pc` (shared memory, pc[r * stride], R <= kPropCache) and the critical
// flags into a bit mask, and the loops below read them back; without it each loop evaluates them
// again (the batched and learned kernels, and models with more reactions).  Same values either way.
constexpr int kPropCache = 20;  // 20 x 256 threads x 8 B = 40 KB: under the 48 KB a launch gets without opting in
template <typename Real, bool WALK = true, int MAXS>
__device__ __forceinline__ void cell_tau_parts_sm(const KArgs& A, const Nbr& q, const Counts<MAXS>& x,
                                                  const int32_t* Xe, Real& tau_ncr_out, Real& rate_cr_out);

template <typename Real, bool WALK = true, bool CACHE = false, int MAXS>
__device__ __forceinline__ void cell_tau_parts(const KArgs& A, uint32_t c, const Nbr& q, const Counts<MAXS>& x,
                                               const int32_t* Xe, Real& tau_ncr_out, Real& rate_cr_out,
                                               Real* pc = nullptr, uint32_t stride = 0) {
  const DevModel& m = A.m;
  const int mode = A.o.mode;
  const int nc = A.o.nc;
  const int comp = comp_of(m, c);
  const int n = q.n;
  const int S = (int)m.S, R = (int)m.R;
  uint32_t critm = 0;
  if constexpr (CACHE) {
    for (int r = 0; r < R; ++r) {
      const Real a = prop<Real>(m, x, r, comp);
      pc[r * stride] = a;
      const bool cr = (mode == 0) ? crit_ref(m, x, r, nc) : crit_fix(m, x, r, a, nc);
      critm |= (uint32_t)cr << r;
    }
  }
  auto propensity = [&](int r) -> Real {
    if constexpr (CACHE) return pc[r * stride];
    else return prop<Real>(m, x, r, comp);
  };
  auto critical = [&](int r, Real a) -> bool {  // crit_ref in reference mode, crit_fix in corrected mode
    if constexpr (CACHE) return ((critm >> r) & 1u) != 0u;
    else return (mode == 0) ? crit_ref(m, x, r, nc) : crit_fix(m, x, r, a, nc);
  };
  Real tau_ncr = RT<Real>::inf();
  for (int s = 0; s < S; ++s) {
    const int32_t xs = x.get(s);
    bool include;
    const int r0 = m.sr_off[s], r1 = m.sr_off[s + 1];
    if (mode == 0) {
      bool skip_r = false;
      for (int i = r0; i < r1 && !skip_r; ++i) skip_r = critical(m.sr_r[i], (Real)0);
      include = !(skip_r && xs < nc);  // tau.cu:165
    } else {
      include = false;
      for (int i = r0; i < r1 && !include; ++i) {
        const int r = m.sr_r[i];
        const Real a = propensity(r);
        include = (a > (Real)0) && !critical(r, a);
      }
      if (!include && xs >= nc && drate<Real>(m, comp, s) > (Real)0 && n > 0) include = true;
    }
    if (!include) continue;
    // compute_tau_sp, tau.cu:68-143
    const Real g = gfun<Real>(m.hor[s], m.hmult[s], xs);
    Real mu = (Real)0, s2 = (Real)0;
    const int p0 = m.sp_off[s], p1 = m.sp_off[s + 1];
    for (int i = p0; i < p1; ++i) {
      const int r = m.sp_r[i];
      const int nu = m.sp_nu[i];
      const Real a = propensity(r);
      const bool ncrit = (mode == 0) ? !critical(r, a) : ((a > (Real)0) && !critical(r, a));
      if (!ncrit) continue;
      mu = mu + (Real)nu * a;
      s2 = s2 + (Real)(nu * nu) * a;
    }
    const Real d = drate<Real>(m, comp, s) * (Real)xs;
    if (mode == 0) {
      if (xs >= nc) { mu = mu + d; s2 = s2 + d; }
      auto term = [&](uint32_t b, int nn) {
        const Real db = drate<Real>(m, comp_of(m, b), s) * (Real)Xe[(size_t)s * m.Npad + b];
        const Real qd = db / (Real)nn;
        mu = mu - qd;
        s2 = s2 + qd;
      };
      if constexpr (WALK) for_each_nbr(m, q, term);
      else for (int j = 0; j < n; ++j) term(q.nb[j], (int)q.nn[j]);
    } else {
      if (xs >= nc && n > 0) {
        const Real dout = (Real)n * d;
        mu = mu - dout;
        s2 = s2 + dout;
      }
      auto term = [&](uint32_t b, int) {
        const int32_t xb = Xe[(size_t)s * m.Npad + b];
        if (xb >= nc) {
          const Real qd = drate<Real>(m, comp_of(m, b), s) * (Real)xb;
          mu = mu + qd;
          s2 = s2 + qd;
        }
      };
      if constexpr (WALK) for_each_nbr(m, q, term);
      else for (int j = 0; j < n; ++j) term(q.nb[j], (int)q.nn[j]);
    }
    Real mm = ((Real)A.o.eps * (Real)xs) / g;
    if (!(mm > (Real)1)) mm = (Real)1;
    const Real t1 = mm / fabs(mu);
    const Real t2 = (mm * mm) / s2;
    const Real ts = t1 < t2 ? t1 : t2;
    if (ts < tau_ncr) tau_ncr = ts;
  }
  // critical (or, corrected SSA subvolume: total) rate, compute_tau_cr tau.cu:176-195
  Real rsum = (Real)0, dsum = (Real)0;
  const bool ncr_inf = plis_isinf_d((double)tau_ncr);
  if (mode == 0 || !ncr_inf) {
    for (int r = 0; r < R; ++r) {
      const Real a = propensity(r);
      if (critical(r, a)) rsum = rsum + a;
    }
    for (int s = 0; s < S; ++s) {
      const int32_t xs = x.get(s);
      if (xs < nc) {
        const Real d = drate<Real>(m, comp, s) * (Real)xs;
        dsum = dsum + (mode == 0 ? d : (Real)n * d);
      }
    }
  } else {
    for (int r = 0; r < R; ++r) rsum = rsum + propensity(r);
    for (int s = 0; s < S; ++s) dsum = dsum + (Real)n * (drate<Real>(m, comp, s) * (Real)x.get(s));
  }
  tau_ncr_out = tau_ncr;
  rate_cr_out = (rsum == (Real)0 && dsum == (Real)0) ? (Real)0 : rsum + dsum;
}

// cell_tau_parts for a small model (SmallModel in the kernel arguments): the same quantities in the
// same order, with the species and reaction loops unrolled to the tables' compile-time sizes.
template <typename Real, bool WALK, int MAXS>
__device__ __forceinline__ void cell_tau_parts_sm(const KArgs& A, const Nbr& q, const Counts<MAXS>& x,
                                                  const int32_t* Xe, Real& tau_ncr_out, Real& rate_cr_out) {
  static_assert(MAXS <= kSmallS, "small-model tables hold kSmallS species");
  const DevModel& m = A.m;
  const SmallModel& t = A.sm;
  const int mode = A.o.mode;
  const int nc = A.o.nc;
  const int n = q.n;
  const int S = (int)m.S, R = (int)m.R;
  Real tau_ncr = RT<Real>::inf();
#pragma unroll
  for (int s = 0; s < MAXS; ++s) {
    if (s >= S) continue;
    const int32_t xs = x.v[s];
    bool include;
    if (mode == 0) {
      bool skip_r = false;
#pragma unroll
      for (int r = 0; r < kSmallR; ++r)
        if ((t.rmask[s] >> r) & 1u) skip_r = skip_r || crit_ref_sm(t, x, r, nc);
      include = !(skip_r && xs < nc);  // tau.cu:165
    } else {
      include = false;
#pragma unroll
      for (int r = 0; r < kSmallR; ++r)
        if ((t.rmask[s] >> r) & 1u) {
          const Real a = prop_sm<Real>(t, x, r);
          include = include || ((a > (Real)0) && !crit_fix_sm(t, x, r, a, nc));
        }
      if (!include && xs >= nc && sm_drate<Real>(t, s) > (Real)0 && n > 0) include = true;
    }
    if (!include) continue;
    const Real g = gfun<Real>(t.hor[s], t.hmult[s], xs);
    Real mu = (Real)0, s2 = (Real)0;
#pragma unroll
    for (int r = 0; r < kSmallR; ++r) {
      const int nu = t.nu[r][s];  // 0 for reactions >= R
      if (nu == 0) continue;
      const Real a = prop_sm<Real>(t, x, r);
      const bool ncrit = (mode == 0) ? !crit_ref_sm(t, x, r, nc) : ((a > (Real)0) && !crit_fix_sm(t, x, r, a, nc));
      if (!ncrit) continue;
      mu = mu + (Real)nu * a;
      s2 = s2 + (Real)(nu * nu) * a;
    }
    const Real dr = sm_drate<Real>(t, s);
    const Real d = dr * (Real)xs;
    if (mode == 0) {
      if (xs >= nc) { mu = mu + d; s2 = s2 + d; }
      auto term = [&](uint32_t b, int nn) {
        const Real db = dr * (Real)Xe[(size_t)s * m.Npad + b];
        const Real qd = db / (Real)nn;
        mu = mu - qd;
        s2 = s2 + qd;
      };
      if constexpr (WALK) for_each_nbr(m, q, term);
      else for (int j = 0; j < n; ++j) term(q.nb[j], (int)q.nn[j]);
    } else {
      if (xs >= nc && n > 0) {
        const Real dout = (Real)n * d;
        mu = mu - dout;
        s2 = s2 + dout;
      }
      auto term = [&](uint32_t b, int) {
        const int32_t xb = Xe[(size_t)s * m.Npad + b];
        if (xb >= nc) {
          const Real qd = dr * (Real)xb;
          mu = mu + qd;
          s2 = s2 + qd;
        }
      };
      if constexpr (WALK) for_each_nbr(m, q, term);
      else for (int j = 0; j < n; ++j) term(q.nb[j], (int)q.nn[j]);
    }
    Real mm = ((Real)A.o.eps * (Real)xs) / g;
    if (!(mm > (Real)1)) mm = (Real)1;
    const Real t1 = mm / fabs(mu);
    const Real t2 = (mm * mm) / s2;
    const Real ts = t1 < t2 ? t1 : t2;
    if (ts < tau_ncr) tau_ncr = ts;
  }
  Real rsum = (Real)0, dsum = (Real)0;
  const bool ncr_inf = plis_isinf_d((double)tau_ncr);
  if (mode == 0 || !ncr_inf) {
#pragma unroll
    for (int r = 0; r < kSmallR; ++r) {
      if (r >= R) continue;
      const Real a = prop_sm<Real>(t, x, r);
      const bool cr = (mode == 0) ? crit_ref_sm(t, x, r, nc) : crit_fix_sm(t, x, r, a, nc);
      if (cr) rsum = rsum + a;
    }
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      if (s >= S) continue;
      const int32_t xs = x.v[s];
      if (xs < nc) {
        const Real d = sm_drate<Real>(t, s) * (Real)xs;
        dsum = dsum + (mode == 0 ? d : (Real)n * d);
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < kSmallR; ++r)
      if (r < R) rsum = rsum + prop_sm<Real>(t, x, r);
#pragma unroll
    for (int s = 0; s < MAXS; ++s)
      if (s < S) dsum = dsum + (Real)n * (sm_drate<Real>(t, s) * (Real)x.v[s]);
  }
  tau_ncr_out = tau_ncr;
  rate_cr_out = (rsum == (Real)0 && dsum == (Real)0) ? (Real)0 : rsum + dsum;
}

// tau_cr: exponential time of the critical rate (inf when it is zero), tau.cu:193.
template <typename Real>
__device__ __forceinline__ double cell_tau_cr(const KArgs& A, uint32_t c, uint64_t step, uint32_t attempt, Real rate) {
  if (rate == (Real)0) return PLIS_INF_D;
  plis_stream st = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_TAU, step, attempt, 0);
  return plis_exponential_d(&st, (double)rate);
}

// Flag and tau of a subvolume from its leap bound and its critical time (tau.cu:224-250).
__device__ __forceinline__ void cell_decide(double tn, double tcr, double& tau_out, int& flag_out) {
  if (plis_isinf_d(tn)) {
    flag_out = F_SSA_FF;
    tau_out = tcr;
  } else if (tn < tcr) {
    flag_out = F_LEAP_NOCR;
    tau_out = tn;
  } else {
    flag_out = F_LEAP_CR;
    tau_out = tcr;
  }
}

// ------------------------------------------------------------------------------------------------
// classification of one subvolume (compute_taus, tau.cu:197-252)
// ------------------------------------------------------------------------------------------------
template <typename Real, bool WALK = true, bool CACHE = false, bool SM = false, int MAXS>
__device__ void classify_cell(const KArgs& A, uint32_t c, const Nbr& q, const Counts<MAXS>& x, const int32_t* Xe,
                              double tau_cur, uint8_t flag_cur, uint64_t step, uint32_t attempt,
                              double ff, double& tau_out, int& flag_out, Real* pc = nullptr, uint32_t stride = 0) {
  if (classify_ff(A.o.mode, tau_cur, flag_cur, step, ff, tau_out, flag_out)) return;
  Real tau_ncr, rate;
  if constexpr (SM) cell_tau_parts_sm<Real, WALK>(A, q, x, Xe, tau_ncr, rate);
  else cell_tau_parts<Real, WALK, CACHE>(A, c, q, x, Xe, tau_ncr, rate, pc, stride);
  const double tcr = cell_tau_cr<Real>(A, c, step, attempt, rate);
  cell_decide((double)tau_ncr, tcr, tau_out, flag_out);
}

// ------------------------------------------------------------------------------------------------
// control (runs in one thread of the last CTA of k_classify, or in k_prepare)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void set_attempt(Ctrl* K, int mode) {
  double scale = 1.0;
  for (uint32_t i = 0; i < K->attempt; ++i) scale *= 0.5;
  if (K->learned && K->attempt > 0) {  // a proposal was rolled back: plain Cao step, halved per attempt
    K->tau_leap = K->tau_step_plain * scale;
    K->dt = K->tau_leap;
    K->exact = 0;
    K->ev_attempt = 0;
    K->ex_attempt = 0;
    return;
  }
  if (mode == 0) {  // the reference re-leaps with the un-halved tau but advances time by the halved one
    K->tau_leap = K->tau_min;
    K->dt = K->tau_min * scale;
  } else {
    K->tau_leap = K->tau_step * scale;
    K->dt = K->tau_leap;
  }
  const uint32_t af = K->argmin_flag;
  uint32_t ex = 0;
  if (mode == 0) {
    if (K->n_leap_cr > 0) ex |= 1u;
    if (af == F_SSA || af == F_SSA_FF) ex |= 2u;
  } else if (K->attempt == 0 && K->tau_step == K->tau_min &&
             (af == F_LEAP_CR || af == F_SSA || af == F_SSA_FF)) {
    ex |= 2u;
  }
  K->exact = ex;
  K->ev_attempt = 0;
  K->ex_attempt = 0;
}

__device__ __forceinline__ void prepare_step(Ctrl* K, int mode) {
  if (K->done) return;
  if (K->t >= K->t_end) { K->done = 1; K->stop_reason = PLIS_STOP_TIME; return; }
  if (K->step >= K->max_step) { K->done = 1; K->stop_reason = PLIS_STOP_STEPS; return; }
  if (K->argmin < 0 || plis_isinf_d(K->tau_min) || K->tau_min < 0.0) {  // driver.cu:269-272
    if (mode == 1) { K->t = K->t_end; K->stop_reason = PLIS_STOP_TIME; }
    else K->stop_reason = PLIS_STOP_NO_EVENT;
    K->done = 1;
    return;
  }
  K->tau_step = K->tau_min;
  if (mode == 1 && K->t_end - K->t < K->tau_step) K->tau_step = K->t_end - K->t;
  if (K->learned) {
    K->tau_step_plain = K->tau_min_plain;
    if (K->t_end - K->t < K->tau_step_plain) K->tau_step_plain = K->t_end - K->t;
  }
  K->attempt = 0;
  set_attempt(K, mode);
}

#ifdef PLIS_ENGINE_HOST_TU
__global__ void k_prepare(KArgs A, double t_end, unsigned long long n_steps) {
  Ctrl* K = A.b.ctrl;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (K->status != PLIS_OK) { K->done = 1; K->stop_reason = PLIS_STOP_ERROR; return; }
  K->t_end = t_end;
  K->max_step = (n_steps == ~0ull) ? ~0ull : K->step + n_steps;
  K->done = 0;
  K->stop_reason = PLIS_STOP_NONE;
  prepare_step(K, A.o.mode);
}
#endif

// ------------------------------------------------------------------------------------------------
// reductions
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void min_pair(double& t, long long& i, double t2, long long i2) {
  if (t2 < t || (t2 == t && i2 < i)) { t = t2; i = i2; }
}
__device__ __forceinline__ void warp_min_pair(double& t, long long& i) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double t2 = __shfl_xor_sync(0xffffffffu, t, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
    min_pair(t, i, t2, i2);
  }
}
__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------------------------------------------
// k_leap (leap_step, leap.cu:3-65)
// ------------------------------------------------------------------------------------------------
// The leap is latency-bound on dependent FP64/integer chains: occupancy matters more than the few
// registers it spills at this bound.
#ifndef PLIS_LEAP_MIN_BLOCKS
#define PLIS_LEAP_MIN_BLOCKS 4
#endif
// Shared-memory staging of one brick's leap: the brick plus a one-subvolume halo.  Every molecule a
// subvolume of the brick keeps or sends is added into the box with shared-memory atomics; the box
// is then flushed with one global reduction per touched subvolume, so global atomics only happen on
// the brick's own subvolumes and its six faces.  Integer sums commute: results are unchanged.
struct Box {
  int32_t* acc;   // shared [S][bz][by][bx], or null when not staged (table topology / too large)
  int bx, by, bz; // tx+2, ty+2, tz+2
  int size;       // bx*by*bz
};

__device__ __forceinline__ int box_offset(const Box& b, int dir) {
  switch (dir) {
    case 0: return -1;
    case 1: return 1;
    case 2: return -b.bx;
    case 3: return b.bx;
    case 4: return -b.bx * b.by;
    default: return b.bx * b.by;
  }
}

struct LeapCtx {
  const int32_t* Xc;
  int32_t* Xt;
  uint8_t* flag;
  uint64_t step;
  uint32_t attempt;
  double t;  // simulated time at the start of the step (event log)
  bool ff_free;  // no subvolume is SSA_FF: the receivers' flag updates are no-ops and are skipped
};

// Leap of one brick (or one 1-D block of a table topology) by the whole CTA; returns this thread's
// events and guard flag.  leap_step, leap.cu:3-65.
// SM: a small model whose tables are in A.sm (SmallModel): the reaction and species loops run to
// the tables' compile-time sizes, so every table read is a constant-bank operand.
// RK: the group blocks use the round keys in A.o (kernel arguments: constant-bank operands); the
// batched kernel, whose per-replica arguments sit in shared memory, recomputes them instead.
template <typename Real, int MAXS, bool LOG, bool WALK = true, bool SM = false, bool RK = false>
__device__ __forceinline__ void leap_tile(const KArgs& A, uint32_t tile, const LeapCtx& L, Real tl, const Box& box,
                                          long long& ev, int& big) {
  static_assert(!SM || MAXS <= kSmallS, "small-model tables hold kSmallS species");
  const DevModel& m = A.m;
  const int mode = A.o.mode, nc = A.o.nc;
  const int32_t* Xc = L.Xc;
  int32_t* Xt = L.Xt;
  uint8_t* flag = L.flag;
  const uint64_t step = L.step;
  const uint32_t attempt = L.attempt;
  Cell cl;
  const bool valid = cell_of(A, tile, cl);
  const uint32_t c = cl.c;
  int own = 0;
  if (box.acc) {
    for (int i = threadIdx.x; i < box.size * (int)m.S; i += blockDim.x) box.acc[i] = 0;
    const uint32_t t = threadIdx.x;
    const int lx = (int)(t % A.g.tx), ly = (int)((t / A.g.tx) % A.g.ty), lz = (int)(t / (A.g.tx * A.g.ty));
    own = (lx + 1) + box.bx * ((ly + 1) + box.by * (lz + 1));
    __syncthreads();
  }
  ev = 0;
  big = 0;
  if (valid) {
    Counts<MAXS> x;
    load_counts(m, Xc, c, x);
    Deltas<MAXS> dl;
#pragma unroll
    for (int s = 0; s < MAXS; ++s) dl.v[s] = 0;
    const uint8_t f = flag[c];
    if (f == F_LEAP_CR || f == F_LEAP_NOCR) {  // leap.cu:9-10
      const int comp = SM ? 0 : comp_of(m, c);
      const int S = (int)m.S, R = (int)m.R;
      // pooled draws (plis_stream.h): the running total of the pool and the membership rule, the
      // same in the walk that fills the pool and in the walks that place its events
      const bool pool_on = !SM && A.o.pool != 0;
      Real pool = (Real)0;
      auto pool_join = [](Real& acc, Real unit, Real w) -> bool {
        if (!(unit < (Real)PLIS_POOL_CUT) || !(acc + w <= (Real)PLIS_POOL_MAX)) return false;
        acc = acc + w;
        return true;
      };
      auto reaction_group = [&](const int r0) {
        // reactions r0..r0+3: means >= PLIS_LEAP_INV_MAX go through PTRS one by one, the rest in lockstep
        Real u[4], lam[4];
        bool act[4];
        long long kk[4];
        uint32_t need = 0, big_mean = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = r0 + i;
          act[i] = false;
          lam[i] = (Real)0;
          u[i] = (Real)0;
          kk[i] = 0;
          if (r < R) {
            Real a;
            bool fire;
            if constexpr (SM) {
              a = prop_sm<Real>(A.sm, x, r);
              fire = (mode == 0) ? !crit_ref_sm(A.sm, x, r, nc) : ((a > (Real)0) && !crit_fix_sm(A.sm, x, r, a, nc));
            } else {
              a = prop<Real>(m, x, r, comp);
              fire = (mode == 0) ? !crit_ref(m, x, r, nc) : ((a > (Real)0) && !crit_fix(m, x, r, a, nc));
            }
            lam[i] = fire ? tl * a : (Real)0;
            if (pool_on && lam[i] > (Real)0 && pool_join(pool, lam[i], lam[i])) lam[i] = (Real)0;  // pooled
            if (lam[i] > (Real)0) {
              if (lam[i] < (Real)PLIS_LEAP_INV_MAX) {
                act[i] = true;  // inversion search: its single uniform comes from the group's blocks
                need |= 1u << i;
              } else {
                big_mean |= 1u << i;  // PTRS below, one sampler for the group
              }
            }
          }
        }
        while (big_mean) {  // draws with means >= PLIS_LEAP_INV_MAX, one at a time through a single inlined PTRS
          const int i = __ffs(big_mean) - 1;
          big_mean &= big_mean - 1u;
          Real li = lam[0];
#pragma unroll
          for (int j = 1; j < 4; ++j)
            if (i == j) li = lam[j];
          plis_stream st = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_react(r0 + i));
          const long long kv = RT<Real>::count(RT<Real>::poisson(&st, li));
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (i == j) kk[j] = kv;
        }
        if (need) {
          const plis_stream g =
              plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_rgroup((uint32_t)r0 >> 2));
          if constexpr (RK) DiffTraits<Real>::group_rk(&g, need, u, 4, A.o);
          else DiffTraits<Real>::group(&g, need, u, 4);
        }
        long long ks[4];
        batched_small_draws<Real>(u, lam, act, ks);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int r = r0 + i;
          if (r >= R) continue;
          const long long k = act[i] ? ks[i] : kk[i];
          ev += k;
          if (LOG && k > 0) ev_put(A.b.ev, L.t, step, attempt, c, c, k, r, PLIS_EVENT_LEAP_REACTION);
          if constexpr (SM) {
#pragma unroll
            for (int sp = 0; sp < MAXS; ++sp) {
              const int nu = A.sm.nu[r][sp];
              if (nu != 0) {
                const long long v = k * (long long)nu;
                if (v >= kBigDraw || v <= -kBigDraw) big = 1;
                dl.v[sp] += v;
              }
            }
          } else {
            const int nn = m.n_net[r];
            for (int q = 0; q < nn; ++q) {
              const long long v = k * (long long)m.net_nu[r * 8 + q];
              if (v >= kBigDraw || v <= -kBigDraw) big = 1;
              dl.add(m.net_s[r * 8 + q], v);
            }
          }
        }
      };
      if constexpr (SM) {
#pragma unroll
        for (int r0 = 0; r0 < kSmallR; r0 += 4)
          if (r0 < R) reaction_group(r0);
      } else {
        for (int r0 = 0; r0 < R; r0 += 4) reaction_group(r0);
      }
      Nbr q;
      if (WALK && m.lattice) nbr_scalars(m, cl, q);  // walked by direction below: no slot arrays
      else nbr_info(m, cl, q);
      const int n = q.n;
      bool mark = false;
      auto jump = [&](int s, long long k, uint32_t b, int dir) {
        if (k >= kBigJump) big = 1;
        if (k > 0) {
          if (box.acc) atomicAdd_block(&box.acc[s * box.size + own + box_offset(box, dir)], (int)k);
          else atomicAdd(&Xt[(size_t)s * m.Npad + b], (int)k);
          if (mode == 1 && !L.ff_free && flag[b] == F_SSA_FF) flag[b] = F_SSA;
          if (LOG) ev_put(A.b.ev, L.t, step, attempt, c, b, k, s, PLIS_EVENT_LEAP_DIFFUSION);
        }
      };
      auto species_lam = [&](const int s) -> Real {
        Real dr;
        if constexpr (SM) dr = sm_drate<Real>(A.sm, s);
        else dr = drate<Real>(m, comp, s);
        return tl * (dr * (Real)x.get(s));
      };
      auto species_jumps = [&](const int s) {
        const int32_t xs = x.get(s);
        if (xs < nc) return;  // is_critical_diffusion, tau.cu:42-45
        if (mode == 0 && n > 0) mark = true;
        const Real lam = species_lam(s);
        if (pool_on && n > 0 && lam > (Real)0 && pool_join(pool, lam, (Real)n * lam)) return;  // pooled
        const Real em = RT<Real>::emlam(lam);  // one exp for the n draws of this species
        int32_t kd[6];
        diffusion_draws<Real, RK>(A, c, s, n, lam, em, step, attempt, kd);
        long long out = 0;
        if (WALK && q.lat) {  // slot j is the j-th present direction; kd is read by constant index only
          int j = 0;
#pragma unroll
          for (int d = 0; d < 6; ++d) {
            uint32_t b;
            int nb_n;
            if (!nbr_dir(m, q, d, b, nb_n)) continue;
            int32_t k = kd[0];
#pragma unroll
            for (int i = 1; i < 6; ++i)
              if (j == i) k = kd[i];
            ++j;
            jump(s, k, b, d);
            out += k;
          }
        } else if constexpr (WALK) {
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            if (j >= n) break;
            jump(s, kd[j], q.nb[j], 0);
            out += kd[j];
          }
        } else {
          for (int j = 0; j < n; ++j) {
            jump(s, kd[j], q.nb[j], q.dir[j]);
            out += kd[j];
          }
        }
        dl.add(s, -out);
        ev += out;
      };
      if constexpr (SM) {
#pragma unroll
        for (int s = 0; s < MAXS; ++s)
          if (s < S) species_jumps(s);
      } else {
        for (int s = 0; s < S; ++s) species_jumps(s);
      }
      if constexpr (!SM) {
        if (pool > (Real)0) {  // the pool's events: total by inversion, then one walk per event
          const plis_stream g =
              plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_LEAP, step, attempt, PLIS_CH_POOL);
          const long long K = RT<Real>::count(RT<Real>::inv_word(plis_group_block(&g, 0).x, pool));
          for (long long e = 0; e < K; ++e) {
            const plis_u32x4 w = plis_group_block(&g, (uint32_t)(e + 1));
            const Real target = RT<Real>::word_uniform(w.x) * pool;
            Real acc = (Real)0;
            int pick_r = -1, pick_s = -1, last_r = -1, last_s = -1;
            for (int r = 0; r < R && pick_r < 0; ++r) {
              const Real a = prop<Real>(m, x, r, comp);
              const bool fire = (mode == 0) ? !crit_ref(m, x, r, nc) : ((a > (Real)0) && !crit_fix(m, x, r, a, nc));
              const Real lr = fire ? tl * a : (Real)0;
              if (lr > (Real)0 && pool_join(acc, lr, lr)) {
                last_r = r;
                if (target < acc) pick_r = r;
              }
            }
            if (pick_r < 0) {
              for (int s = 0; s < S; ++s) {
                if (x.get(s) < nc || n == 0) continue;
                const Real ls = species_lam(s);
                if (ls > (Real)0 && pool_join(acc, ls, (Real)n * ls)) {
                  last_s = s;
                  if (target < acc) {
                    pick_s = s;
                    break;
                  }
                }
              }
              if (pick_s < 0) {  // rounding left the target at the total: the last member
                if (last_s >= 0) pick_s = last_s;
                else pick_r = last_r;
              }
            }
            ev += 1;
            if (pick_r >= 0) {
              if (LOG) ev_put(A.b.ev, L.t, step, attempt, c, c, 1, pick_r, PLIS_EVENT_LEAP_REACTION);
              const int nn = m.n_net[pick_r];
              for (int i = 0; i < nn; ++i) dl.add(m.net_s[pick_r * 8 + i], (long long)m.net_nu[pick_r * 8 + i]);
            } else {
              const int j = (int)plis_pool_slot(w.y, (uint32_t)n);
              uint32_t b = c;
              int dir = 0;
              if (WALK && q.lat) {
                int jj = 0;
                for (int d = 0; d < 6; ++d) {
                  uint32_t bd;
                  int nb_n;
                  if (!nbr_dir(m, q, d, bd, nb_n)) continue;
                  if (jj == j) {
                    b = bd;
                    dir = d;
                  }
                  ++jj;
                }
              } else {
                b = q.nb[j];
                if constexpr (!WALK) dir = q.dir[j];
              }
              jump(pick_s, 1, b, dir);
              dl.add(pick_s, -1);
            }
          }
        }
      }
      if (mark && !L.ff_free) {  // leap.cu:54-56: every receiver leaves fast-forward
        auto leave_ff = [&](uint32_t b, int) {
          if (flag[b] == F_SSA_FF) flag[b] = F_SSA;
        };
        if constexpr (WALK) for_each_nbr(m, q, leave_ff);
        else for (int j = 0; j < n; ++j) leave_ff(q.nb[j], 0);
      }
    }
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
      if (s < (int)m.S) {
        const long long tv = (long long)x.v[s] + dl.v[s];
        if (tv >= kBigTile || tv <= -kBigTile) big = 1;
        if (box.acc) atomicAdd_block(&box.acc[s * box.size + own], (int)tv);
        else atomicAdd(&Xt[(size_t)s * m.Npad + c], (int)tv);
      }
    }
  }
  if (box.acc) {  // flush the box: each subvolume's own entry, then the six halo faces
    __syncthreads();
    if (valid) {
      for (int s = 0; s < (int)m.S; ++s) {
        const int32_t v = box.acc[s * box.size + own];
        if (v) atomicAdd(&Xt[(size_t)s * m.Npad + c], v);
      }
    }
    const uint32_t tx = A.g.tx, ty = A.g.ty, tz = A.g.tz;
    const uint32_t b = tile;
    const uint32_t bxi = b % A.g.ntx, br = b / A.g.ntx;
    const uint32_t byi = br % A.g.nty, bzi = br / A.g.nty;
    const int x0 = (int)(bxi * tx), y0 = (int)(byi * ty), z0 = (int)(bzi * tz);
    // face f: 0/1 = x-/x+ (ty*tz entries), 2/3 = y-/y+ (tx*tz), 4/5 = z-/z+ (tx*ty)
    const int fsz[3] = {(int)(ty * tz), (int)(tx * tz), (int)(tx * ty)};
    const int total = 2 * (fsz[0] + fsz[1] + fsz[2]);
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
      int f = 0, i = w;
      while (i >= fsz[f >> 1]) { i -= fsz[f >> 1]; ++f; }
      int lx, ly, lz;  // box-relative coordinates (-1 .. t)
      if (f < 2) { ly = i % (int)ty; lz = i / (int)ty; lx = (f == 0) ? -1 : (int)tx; }
      else if (f < 4) { lx = i % (int)tx; lz = i / (int)tx; ly = (f == 2) ? -1 : (int)ty; }
      else { lx = i % (int)tx; ly = i / (int)tx; lz = (f == 4) ? -1 : (int)tz; }
      const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
      if (gx < 0 || gy < 0 || gz < 0 || gx >= (int)m.X || gy >= (int)m.Y || gz >= (int)m.Z) continue;
      const int p = (lx + 1) + box.bx * ((ly + 1) + box.by * (lz + 1));
      const uint32_t g = (uint32_t)gx + m.X * ((uint32_t)gy + m.Y * (uint32_t)gz);
      for (int s = 0; s < (int)m.S; ++s) {
        const int32_t v = box.acc[s * box.size + p];
        if (v) atomicAdd(&Xt[(size_t)s * m.Npad + g], v);
      }
    }
  }
}

template <typename Real, int MAXS, bool LOG, bool SM>
__global__ void __launch_bounds__(256, PLIS_LEAP_MIN_BLOCKS) k_leap(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  extern __shared__ int32_t s_box[];
  __shared__ long long s_ev[32];
  __shared__ int s_big;
  if (threadIdx.x == 0) s_big = 0;
  LeapCtx L;
  L.Xc = A.b.X[K->cur];
  L.Xt = A.b.X[K->tgt];
  L.flag = A.b.flag[K->tf];
  L.step = K->step + 1;
  L.attempt = K->attempt;
  L.t = K->t;
  L.ff_free = K->ff_free != 0;
  const Real tl = (Real)K->tau_leap;
  Box box;
  box.acc = A.g.staged ? s_box : nullptr;
  box.bx = (int)A.g.tx + 2;
  box.by = (int)A.g.ty + 2;
  box.bz = (int)A.g.tz + 2;
  box.size = box.bx * box.by * box.bz;
  __syncthreads();
  long long ev;
  int big;
  leap_tile<Real, MAXS, LOG, true, SM, true>(A, blockIdx.x, L, tl, box, ev, big);
  // events and guard flags of the CTA
  ev = warp_sum(ev);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (big) s_big = 1;
  if (lane == 0) s_ev[wid] = ev;
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    long long v = lane < nw ? s_ev[lane] : 0;
    v = warp_sum(v);
    if (lane == 0) {
      if (v) atomicAdd(&K->ev_attempt, (unsigned long long)v);
      if (s_big) atomicOr(&K->blocks_done, 0x80000000u);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// exact events
// ------------------------------------------------------------------------------------------------
// A subvolume whose delta row an exact event wrote: k_apply adds only the listed rows.
__device__ __forceinline__ uint32_t* touched_list(const KArgs& A) {
  return reinterpret_cast<uint32_t*>(A.b.D + (size_t)A.m.S * A.m.Npad);
}
__device__ __forceinline__ void touch(const KArgs& A, uint32_t c) {
  Ctrl* K = A.b.ctrl;
  if (!K->touched_on) return;
  const uint32_t i = atomicAdd(&K->n_touched, 1u);
  if (i < A.m.N) touched_list(A)[i] = c;
}

// Reference critical event of one LEAP_CR subvolume (leap.cu:86-199).
template <typename Real, bool LOG, int MAXS>
__device__ int critical_event_ref(const KArgs& A, uint32_t c, const Counts<MAXS>& x, const int32_t* Xt,
                                  uint64_t step, uint32_t attempt, int32_t* D, uint8_t* flag) {
  const DevModel& m = A.m;
  const int nc = A.o.nc;
  const int S = (int)m.S, R = (int)m.R;
  const int comp = comp_of(m, c);
  plis_stream su = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_CRIT, step, attempt, 0);
  const Real u = RT<Real>::uniform(&su);
  Real rsum = (Real)0, dsum = (Real)0;
  for (int r = 0; r < R; ++r)
    if (crit_ref(m, x, r, nc)) rsum = rsum + prop<Real>(m, x, r, comp);
  for (int s = 0; s < S; ++s)
    if (x.get(s) < nc) dsum = dsum + drate<Real>(m, comp, s) * (Real)x.get(s);
  if (rsum + dsum == (Real)0) return 0;
  if (u < rsum / (rsum + dsum)) {
    const Real scaled = rsum * u;
    Real partial = (Real)0;
    int ric = 0;
    while (partial <= scaled && ric < R) {
      if (crit_ref(m, x, ric, nc)) partial = partial + prop<Real>(m, x, ric, comp);
      ++ric;
    }
    int ri = 0;
    for (ri = 0; ri < R && ric > 0; ++ri)
      if (crit_ref(m, x, ri, nc)) --ric;
    ri = ri - 1;  // leap.cu:121-126 as written
    if (ri < 0) ri = 0;
    bool fire = true;
    for (int s = 0; s < S; ++s) {
      int need = 0;
      for (int i = 0; i < m.n_reac[ri]; ++i)
        if (m.reac_s[ri * 3 + i] == s) need = m.reac_m[ri * 3 + i];
      fire = fire && x.get(s) >= need && Xt[(size_t)s * m.Npad + c] >= need;
    }
    if (!fire) return 0;
    for (int i = 0; i < m.n_net[ri]; ++i)
      atomicAdd(&D[(size_t)m.net_s[ri * 8 + i] * m.Npad + c], (int)m.net_nu[ri * 8 + i]);
    touch(A, c);
    if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, c, c, 1, ri, PLIS_EVENT_CRITICAL_REACTION);
    return 1;
  }
  const Real scaled = dsum * u;
  Real partial = (Real)0;
  int spic = 0;
  while (partial <= scaled && spic < S) {
    if (x.get(spic) < nc) partial = partial + drate<Real>(m, comp, spic) * (Real)x.get(spic);
    ++spic;
  }
  int spi = 0;
  for (spi = 0; spi < S && spic > 0; ++spi)
    if (x.get(spi) < nc) --spic;
  spi = spi - 1;  // leap.cu:160-166
  if (spi < 0) spi = 0;
  const bool fire = x.get(spi) > 0 && Xt[(size_t)spi * m.Npad + c] > 0;
  if (!fire) return 0;
  plis_stream sd = plis_stream_make(A.o.seed, A.o.replica, c, PLIS_PHASE_CRIT, step, attempt, 1);
  const Real u2 = RT<Real>::uniform(&sd);
  int slot = (int)(u2 * (Real)6);
  if (slot > 5) slot = 5;
  const uint32_t target = canon_slot(m, c, slot);
  if (target == c) return 0;
  atomicAdd(&D[(size_t)spi * m.Npad + c], -1);
  atomicAdd(&D[(size_t)spi * m.Npad + target], 1);
  touch(A, c);
  touch(A, target);
  const uint32_t q = flat_table_entry(m, target);  // leap.cu:192-193
  if (!A.sl.on || (q + A.sl.has_lo * A.sl.layer >= A.sl.lo && q < A.sl.hi + A.sl.has_hi * A.sl.layer)) {
    if (flag[q] == F_SSA_FF) flag[q] = F_SSA;
  } else {  // z-slab: another slab owns q; its owner applies the write after the gather
    const uint32_t i = atomicAdd(&A.sl.remote->n, 1u);
    if (i < (uint32_t)kSlabRemote) A.sl.remote->cell[i] = q;
  }
  if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, c, target, 1, spi, PLIS_EVENT_CRITICAL_DIFFUSION);
  return 1;
}

// Exact event of the arg-min subvolume: reference ssa_step (ssa.cu:270-324), or in corrected mode
// an SSA over the critical channels (LEAP_CR) or over every channel (SSA subvolumes).
template <typename Real, bool LOG, int MAXS>
__device__ int argmin_event(const KArgs& A, uint32_t mcell, const Counts<MAXS>& x, uint64_t step, uint32_t attempt,
                            int32_t* dst, uint8_t* flag, bool critical_only) {
  const DevModel& m = A.m;
  const int mode = A.o.mode, nc = A.o.nc;
  const int S = (int)m.S, R = (int)m.R;
  const int comp = comp_of(m, mcell);
  uint32_t nb[6];
  const int n = nbrs(m, mcell, nb);
  plis_stream su = plis_stream_make(A.o.seed, A.o.replica, mcell, PLIS_PHASE_SSA, step, attempt, 0);
  const Real u = RT<Real>::uniform(&su);
  if (mode == 0) {
    Real rsum = (Real)0, dsum = (Real)0;
    for (int r = 0; r < R; ++r) rsum = rsum + prop<Real>(m, x, r, comp);
    for (int s = 0; s < S; ++s) dsum = dsum + drate<Real>(m, comp, s) * (Real)x.get(s);
    const Real dtot = dsum * (Real)n;  // rates.cu:165-172
    const Real total = rsum + dtot;
    if (!(total > (Real)0)) return 0;
    if (u < rsum / total) {
      const Real scaled = rsum * u;
      Real partial = (Real)0;
      int ri = 0;
      while (partial <= scaled && ri < R) { partial = partial + prop<Real>(m, x, ri, comp); ++ri; }
      ri = ri - 1;
      if (ri < 0) ri = 0;
      for (int i = 0; i < m.n_net[ri]; ++i)
        atomicAdd(&dst[(size_t)m.net_s[ri * 8 + i] * m.Npad + mcell], (int)m.net_nu[ri * 8 + i]);
      if (dst == A.b.D) touch(A, mcell);
      flag[mcell] = F_SSA;  // ssa.cu:295
      if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, mcell, mcell, 1, ri, PLIS_EVENT_SSA_REACTION);
      return 1;
    }
    if (!(dtot > (Real)0)) return 0;
    const Real scaled = (dtot / (Real)n) * u;  // ssa.cu:256-266
    Real partial = (Real)0;
    int spi = 0;
    while (partial <= scaled && spi < S) {
      partial = partial + drate<Real>(m, comp, spi) * (Real)x.get(spi);
      ++spi;
    }
    spi = spi - 1;
    if (spi < 0) spi = 0;
    plis_stream sd = plis_stream_make(A.o.seed, A.o.replica, mcell, PLIS_PHASE_SSA, step, attempt, 1);
    const Real u2 = RT<Real>::uniform(&sd);
    int slot = (int)(u2 * (Real)6);
    if (slot > 5) slot = 5;
    const uint32_t target = canon_slot(m, mcell, slot);
    if (target == mcell) return 0;
    atomicAdd(&dst[(size_t)spi * m.Npad + mcell], -1);
    atomicAdd(&dst[(size_t)spi * m.Npad + target], 1);
    if (dst == A.b.D) {
      touch(A, mcell);
      touch(A, target);
    }
    if (flag[target] == F_SSA_FF) flag[target] = F_SSA;
    if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, mcell, target, 1, spi, PLIS_EVENT_SSA_DIFFUSION);
    return 1;
  }
  Real total = (Real)0;
  for (int r = 0; r < R; ++r) {
    const Real a = prop<Real>(m, x, r, comp);
    if (!critical_only || crit_fix(m, x, r, a, nc)) total = total + a;
  }
  for (int s = 0; s < S; ++s)
    if (!critical_only || x.get(s) < nc) total = total + (Real)n * (drate<Real>(m, comp, s) * (Real)x.get(s));
  if (!(total > (Real)0)) return 0;
  const Real scaled = total * u;
  Real partial = (Real)0;
  int chosen_r = -1, chosen_s = -1, last_r = -1, last_s = -1;
  for (int r = 0; r < R && chosen_r < 0; ++r) {
    const Real a = prop<Real>(m, x, r, comp);
    const bool use = critical_only ? crit_fix(m, x, r, a, nc) : true;
    if (!use || !(a > (Real)0)) continue;
    partial = partial + a;
    last_r = r;
    if (partial > scaled) chosen_r = r;
  }
  if (chosen_r < 0) {
    for (int s = 0; s < S && chosen_s < 0; ++s) {
      const bool use = critical_only ? (x.get(s) < nc) : true;
      const Real w = (Real)n * (drate<Real>(m, comp, s) * (Real)x.get(s));
      if (!use || !(w > (Real)0)) continue;
      partial = partial + w;
      last_s = s;
      if (partial > scaled) chosen_s = s;
    }
  }
  if (chosen_r < 0 && chosen_s < 0) {
    if (last_s >= 0) chosen_s = last_s;
    else chosen_r = last_r;
  }
  const int kind_r = critical_only ? PLIS_EVENT_CRITICAL_REACTION : PLIS_EVENT_SSA_REACTION;
  if (chosen_r >= 0) {
    for (int i = 0; i < m.n_net[chosen_r]; ++i)
      atomicAdd(&dst[(size_t)m.net_s[chosen_r * 8 + i] * m.Npad + mcell], (int)m.net_nu[chosen_r * 8 + i]);
    if (dst == A.b.D) touch(A, mcell);
    if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, mcell, mcell, 1, chosen_r, kind_r);
    return 1;
  }
  plis_stream sd = plis_stream_make(A.o.seed, A.o.replica, mcell, PLIS_PHASE_SSA, step, attempt, 1);
  const Real u2 = RT<Real>::uniform(&sd);
  int slot = (int)(u2 * (Real)n);
  if (slot > n - 1) slot = n - 1;
  const uint32_t target = nb[slot];
  atomicAdd(&dst[(size_t)chosen_s * m.Npad + mcell], -1);
  atomicAdd(&dst[(size_t)chosen_s * m.Npad + target], 1);
  if (dst == A.b.D) {
    touch(A, mcell);
    touch(A, target);
  }
  if (flag[target] == F_SSA_FF) flag[target] = F_SSA;
  if (LOG) ev_put(A.b.ev, A.b.ctrl->t, step, attempt, mcell, target, 1, chosen_s, kind_r + 1);
  return 1;
}

template <typename Real, int MAXS, bool LOG>
__global__ void __launch_bounds__(256) k_exact(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const uint32_t ex = K->exact;
  if (ex == 0) return;
  const DevModel& m = A.m;
  const int32_t* Xc = A.b.X[K->cur];
  int32_t* Xt = A.b.X[K->tgt];
  uint8_t* flag = A.b.flag[K->tf];
  const uint64_t step = K->step + 1;
  const uint32_t attempt = K->attempt;
  int fired = 0;
  const uint32_t c_lo = A.sl.on ? A.sl.lo : 0u, c_hi = A.sl.on ? A.sl.hi : m.N;  // a z-slab: its own subvolumes
  if (ex & 1u) {
    // reference: every LEAP_CR subvolume.  A CTA scans a chunk of flags, gathers the chunk's LEAP_CR
    // subvolumes in shared memory and fires them on consecutive threads: a few per cent of the
    // subvolumes are LEAP_CR, and a strided scan would run each event on one lane of its warp.
    __shared__ uint32_t s_cell[kExactChunk];
    __shared__ uint32_t s_n;
    const unsigned lane = threadIdx.x & 31u;
    for (uint32_t base = c_lo + blockIdx.x * kExactChunk; base < c_hi; base += gridDim.x * kExactChunk) {
      if (threadIdx.x == 0) s_n = 0;
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < kExactChunk; i += blockDim.x) {  // blockDim.x divides the chunk
        const uint32_t c = base + i;
        const bool cr = c < c_hi && flag[c] == F_LEAP_CR;
        const unsigned mask = __ballot_sync(0xffffffffu, cr);
        unsigned pos = 0;
        if (lane == 0 && mask) pos = atomicAdd(&s_n, (unsigned)__popc(mask));
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (cr) s_cell[pos + __popc(mask & ((1u << lane) - 1u))] = c;
      }
      __syncthreads();
      const uint32_t n = s_n;
      for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const uint32_t c = s_cell[j];
        Counts<MAXS> x;
        load_counts(m, Xc, c, x);
        fired += critical_event_ref<Real, LOG>(A, c, x, Xt, step, attempt, A.b.D, flag);
      }
      __syncthreads();
    }
  }
  if ((ex & 2u) && blockIdx.x == 0 && threadIdx.x == 0 && (uint32_t)K->argmin >= c_lo && (uint32_t)K->argmin < c_hi) {
    const uint32_t am = (uint32_t)K->argmin;
    const uint8_t fa = flag[am];
    Counts<MAXS> x;
    load_counts(m, Xc, am, x);
    int32_t* dst = (ex & 1u) ? A.b.D : Xt;
    if (A.o.mode == 0) {
      if (fa == F_SSA || fa == F_SSA_FF) fired += argmin_event<Real, LOG>(A, am, x, step, attempt, dst, flag, false);
    } else {
      if (fa == F_LEAP_CR) fired += argmin_event<Real, LOG>(A, am, x, step, attempt, dst, flag, true);
      else if (fa == F_SSA || fa == F_SSA_FF) fired += argmin_event<Real, LOG>(A, am, x, step, attempt, dst, flag, false);
    }
  }
  if (fired) {  // exact events are rare: one atomic per firing thread
    atomicAdd(&K->ev_attempt, (unsigned long long)fired);
    atomicAdd(&K->ex_attempt, (unsigned long long)fired);
  }
}

#ifdef PLIS_ENGINE_HOST_TU
__global__ void __launch_bounds__(256) k_apply(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done || !(K->exact & 1u)) return;
  const DevModel& m = A.m;
  int32_t* Xt = A.b.X[K->tgt];
  // a z-slab: its subvolumes and the ghost layers next to its faces (deltas of events that cross a face)
  const uint32_t nt = K->touched_on ? K->n_touched : ~0u;
  if (nt <= m.N) {  // the listed rows (a row listed twice: the second finds zeros)
    const uint32_t* list = touched_list(A);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
      const uint32_t c = list[i];
      for (uint32_t s = 0; s < m.S; ++s) {
        const size_t j = (size_t)s * m.Npad + c;
        const int32_t v = atomicExch(&A.b.D[j], 0);
        if (v) atomicAdd(&Xt[j], v);
      }
    }
    return;
  }
  const uint32_t c_lo = A.sl.on ? A.sl.lo - A.sl.has_lo * A.sl.layer : 0u;
  const uint32_t c_hi = A.sl.on ? A.sl.hi + A.sl.has_hi * A.sl.layer : m.N;
  for (uint32_t c = c_lo + blockIdx.x * blockDim.x + threadIdx.x; c < c_hi; c += gridDim.x * blockDim.x) {
    for (uint32_t s = 0; s < m.S; ++s) {
      const size_t i = (size_t)s * m.Npad + c;
      const int32_t v = A.b.D[i];
      if (v) {
        Xt[i] += v;
        A.b.D[i] = 0;
      }
    }
  }
}
#endif

// ------------------------------------------------------------------------------------------------
// classification phase + last-CTA control
// ------------------------------------------------------------------------------------------------
struct ClassifyCtx {
  const int32_t* Xe;      // counts to classify (post-step, or the initial state)
  int32_t* Xz;            // buffer the next leap reduces into: zeroed here
  const double* tau_cur;
  double* tau_new;
  const uint8_t* flag_cur;
  uint8_t* flag_new;
  uint64_t step;
  uint32_t attempt;
  double ff;              // fast-forward decrement
};

__device__ __forceinline__ ClassifyCtx classify_ctx(const KArgs& A, const Ctrl* K) {
  ClassifyCtx C;
  const uint32_t phase = K->phase;
  C.Xe = A.b.X[phase == 0 ? K->cur : K->tgt];
  C.Xz = A.b.X[K->spare];
  const uint32_t tf = K->tf;
  C.tau_cur = A.b.tau[tf];
  C.tau_new = A.b.tau[tf ^ 1u];
  C.flag_cur = A.b.flag[tf];
  C.flag_new = A.b.flag[tf ^ 1u];
  C.step = phase == 0 ? K->step : K->step + 1;  // phase 0 at step 0 after set_state, or a re-classification
  C.attempt = phase == 0 ? 0 : K->attempt;
  C.ff = K->dt;
  return C;
}

// One thread's subvolume of one brick: negativity check, zeroing of the next target, classification.
template <typename Real, int MAXS, bool WALK = true, bool CACHE = false, bool SM = false>
__device__ __forceinline__ void classify_tile(const KArgs& A, uint32_t tile, const ClassifyCtx& C, double& tn,
                                              long long& ti, int& fl, int& bad, bool& valid, Real* pc = nullptr) {
  const DevModel& m = A.m;
  Cell cl;
  valid = cell_of(A, tile, cl);
  const uint32_t c = cl.c;
  tn = PLIS_INF_D;
  ti = 0x7FFFFFFFFFFFFFFFll;
  fl = F_SSA_FF;
  bad = 0;
  if (!valid) return;
  Counts<MAXS> x;
  load_counts(m, C.Xe, c, x);
#pragma unroll
  for (int s = 0; s < MAXS; ++s)
    if (s < (int)m.S) {
      if (x.v[s] < 0) bad = 1;
      C.Xz[(size_t)s * m.Npad + c] = 0;
    }
  Nbr q;
  if constexpr (WALK) nbr_lite(m, cl, q);
  else nbr_info(m, cl, q);
  classify_cell<Real, WALK, CACHE, SM>(A, c, q, x, C.Xe, C.tau_cur[c], C.flag_cur[c], C.step, C.attempt, C.ff, tn, fl,
                                       CACHE ? pc + threadIdx.x : nullptr, blockDim.x);
  C.tau_new[c] = tn;
  C.flag_new[c] = (uint8_t)fl;
  ti = c;
}

// CTA reduction of one brick into slot `slot` (min tau with arg-min, #LEAP_CR, negative flag), then
// the count of finished bricks; true in the CTA that finished last of `nslots`.
__device__ __forceinline__ bool classify_slot(const KArgs& A, Ctrl* K, uint32_t slot, uint32_t nslots, double tn,
                                              long long ti, bool is_cr, int bad, bool is_ff) {
  __shared__ double s_t[32];
  __shared__ long long s_i[32];
  __shared__ bool s_last;
  const int ncr = __syncthreads_count(is_cr);
  const int nff = __syncthreads_count(is_ff);
  const int nbad = __syncthreads_or(bad);
  warp_min_pair(tn, ti);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_t[wid] = tn; s_i[wid] = ti; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double bt = s_t[0];
    long long bi = s_i[0];
    for (int w = 1; w < nw; ++w) min_pair(bt, bi, s_t[w], s_i[w]);
    A.b.slot_tau[slot] = bt;
    A.b.slot_idx[slot] = bi;
    A.b.slot_cr[slot] = (uint32_t)ncr | ((uint32_t)nff << 16);  // #LEAP_CR | #SSA_FF << 16 (<= 1024 each)
    A.b.slot_bad[slot] = nbad ? 1u : 0u;
    __threadfence();
    const uint32_t prev = atomicAdd(&K->blocks_done, 1u);
    s_last = ((prev & 0x7FFFFFFFu) == nslots - 1);
  }
  __syncthreads();
  return s_last;
}

// The step decision (driver.cu:267-334) from the grid-wide reductions: the arg-min gt / gi (gi = -1 when
// no subvolume can fire), #LEAP_CR gcr, #SSA_FF gff, a negative count or oversized draw `bad`, the min of
// the plain taus gp (learned proposals) and the flag of the arg-min subvolume: rollback or accept, time,
// the next plan.  One thread.
__device__ __forceinline__ void step_decide(const KArgs& A, Ctrl* K, uint32_t phase, uint32_t tf, double gt, long long gi,
                                            unsigned long long gcr, unsigned long long gff, uint32_t bad, double gp,
                                            bool learned, uint32_t am_flag) {
  const int mode = A.o.mode;
  K->learned = learned ? 1u : 0u;
  if (phase == 0) {
    K->tau_min = gt;
    K->tau_min_plain = gp;
    K->argmin = gi;
    K->n_leap_cr = (uint32_t)gcr;
    K->ff_free = gff == 0 ? 1u : 0u;
    K->argmin_flag = am_flag;
    K->tf = tf ^ 1u;
    K->phase = 1;
    K->done = 1;  // idle until a run call
  } else if (bad) {  // check_state + revert (leap.cu:203-212, driver.cu:292-315)
    K->attempt += 1;
    if ((int)K->attempt > A.o.max_rollbacks) {
      K->status = PLIS_ERR_STUCK;
      K->stop_reason = PLIS_STOP_ERROR;
      K->done = 1;
    } else {
      const uint32_t t = K->tgt;
      K->tgt = K->spare;
      K->spare = t;
      set_attempt(K, mode);
    }
  } else {
    // accept: swap state (driver.cu:320-323) by rotating buffer indices
    K->t = K->t + K->dt;
    K->step = K->step + 1;
    K->events += K->ev_attempt;
    K->exact_events += K->ex_attempt;
    K->rollbacks += K->attempt;
    K->last_tau = K->tau_min;
    K->last_argmin = K->argmin;
    const uint32_t oc = K->cur;
    K->cur = K->tgt;
    K->tgt = K->spare;
    K->spare = oc;
    K->tf = tf ^ 1u;
    K->tau_min = gt;
    K->tau_min_plain = gp;
    K->argmin = gi;
    K->n_leap_cr = (uint32_t)gcr;
    K->ff_free = gff == 0 ? 1u : 0u;
    K->argmin_flag = am_flag;
    prepare_step(K, mode);
  }
}

// The whole last CTA: reduce the `nslots` slots (independent L2 loads spread over the block), then
// one thread takes the step decision (driver.cu:267-334): rollback or accept, time, the next plan.
__device__ __forceinline__ void classify_control(const KArgs& A, Ctrl* K, uint32_t nslots) {
  __shared__ double s_t[32];
  __shared__ long long s_i[32];
  __shared__ unsigned long long s_cr[32];
  __shared__ unsigned long long s_ff[32];
  __shared__ uint32_t s_bad[32];
  __shared__ double s_p[32];
  __threadfence();
  const uint32_t phase = K->phase;
  const uint32_t tf = K->tf;
  const uint8_t* flag_new = A.b.flag[tf ^ 1u];
  double gt = PLIS_INF_D;
  long long gi = 0x7FFFFFFFFFFFFFFFll;
  unsigned long long gcr = 0, gff = 0;
  uint32_t gbad = 0;
  double gp = PLIS_INF_D;  // learned classification: min of the plain taus
  const double* sp = A.b.slot_tau_plain;
  for (uint32_t b = threadIdx.x; b < nslots; b += blockDim.x) {
    min_pair(gt, gi, __ldcg(&A.b.slot_tau[b]), __ldcg(&A.b.slot_idx[b]));
    const uint32_t sc = __ldcg(&A.b.slot_cr[b]);
    gcr += sc & 0xFFFFu;
    gff += sc >> 16;
    gbad |= __ldcg(&A.b.slot_bad[b]);
    if (sp) gp = fmin(gp, __ldcg(&sp[b]));
  }
  warp_min_pair(gt, gi);
  gcr = (unsigned long long)warp_sum((long long)gcr);
  gff = (unsigned long long)warp_sum((long long)gff);
  gbad = __reduce_or_sync(0xffffffffu, gbad);
  if (sp) gp = warp_min_d(gp);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_t[wid] = gt; s_i[wid] = gi; s_cr[wid] = gcr; s_ff[wid] = gff; s_bad[wid] = gbad; s_p[wid] = gp; }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    gt = lane < nw ? s_t[lane] : PLIS_INF_D;
    gi = lane < nw ? s_i[lane] : 0x7FFFFFFFFFFFFFFFll;
    gcr = lane < nw ? s_cr[lane] : 0ull;
    gff = lane < nw ? s_ff[lane] : 0ull;
    gbad = lane < nw ? s_bad[lane] : 0u;
    gp = lane < nw ? s_p[lane] : PLIS_INF_D;
    warp_min_pair(gt, gi);
    gcr = (unsigned long long)warp_sum((long long)gcr);
    gff = (unsigned long long)warp_sum((long long)gff);
    gbad = __reduce_or_sync(0xffffffffu, gbad);
    if (sp) gp = warp_min_d(gp);
  }
  if (threadIdx.x == 0) {
    const uint32_t leap_bad = (__ldcg(&K->blocks_done) & 0x80000000u) ? 1u : 0u;
    K->blocks_done = 0;
    if (gi == 0x7FFFFFFFFFFFFFFFll) gi = -1;
    const uint32_t am_flag = gi >= 0 ? __ldcg(&flag_new[gi]) : F_SSA_FF;
    if (A.sl.on) {  // a z-slab: the decision waits for every slab's summary (k_slab_control)
      SlabSummary q;
      q.tau = gt; q.idx = gi; q.tau_plain = gp; q.ncr = gcr; q.nff = gff; q.bad = gbad; q.leap_bad = leap_bad;
      q.am_flag = am_flag; q.pad_ = 0;
      *A.sl.summary = q;
      return;
    }
    step_decide(A, K, phase, tf, gt, gi, gcr, gff, gbad | leap_bad, gp, sp != nullptr, am_flag);
  }
}

// 64 registers, 4 CTAs per SM: the classification is bound by load latency and needs the warps
// (with the compiler's own choice of 80-88 registers it runs 12-60 % slower).
#ifndef PLIS_CLASSIFY_MIN_BLOCKS
#define PLIS_CLASSIFY_MIN_BLOCKS 4
#endif
template <typename Real, int MAXS, bool CACHE, bool SM>
__global__ void __launch_bounds__(256, PLIS_CLASSIFY_MIN_BLOCKS) k_classify(KArgs A) {
  extern __shared__ __align__(16) unsigned char s_prop[];  // CACHE: R x blockDim propensities
  pdl_entry();
  if (blockIdx.x == 0 && threadIdx.x == 0) A.b.ctrl->n_touched = 0;  // k_apply has consumed the list
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const ClassifyCtx C = classify_ctx(A, K);
  double tn;
  long long ti;
  int fl, bad;
  bool valid;
  classify_tile<Real, MAXS, true, CACHE, SM>(A, blockIdx.x, C, tn, ti, fl, bad, valid, reinterpret_cast<Real*>(s_prop));
  if (classify_slot(A, K, blockIdx.x, gridDim.x, tn, ti, valid && fl == F_LEAP_CR, bad, valid && fl == F_SSA_FF))
    classify_control(A, K, gridDim.x);
}

#ifdef PLIS_ENGINE_HOST_TU
// ------------------------------------------------------------------------------------------------
// z-slab exchanges (SlabArgs): layer i of a face is subvolume (first subvolume of the layer) + i;
// a staging buffer holds [S][layer] counts, then [layer] flags widened to int32.
// ------------------------------------------------------------------------------------------------
// After the leap, exact events and deltas: the ghost layers of the target (molecules this slab sent
// across its faces, with their receivers' flags) into send[0] (below) and send[1] (above).
__global__ void k_slab_pack_ghosts(KArgs A) {
  const Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const SlabArgs& L = A.sl;
  const int32_t* Xt = A.b.X[K->tgt];
  const uint8_t* flag = A.b.flag[K->tf];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.layer; i += gridDim.x * blockDim.x) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t g = side ? L.hi + i : L.lo - L.layer + i;
      for (uint32_t s = 0; s < A.m.S; ++s) L.send[side][(size_t)s * L.layer + i] = Xt[(size_t)s * A.m.Npad + g];
      L.send[side][(size_t)A.m.S * L.layer + i] = flag[g];
    }
  }
}

// The neighbours' ghost layers added into this slab's face layers (their molecules that crossed into
// it), their flag changes (SSA_FF -> SSA only) merged, then the gathered flag writes that land in
// this slab applied.  An attempt with more such writes than one list holds fails (PLIS_ERR_LIMIT,
// identically on every rank).
__global__ void k_slab_merge(KArgs A) {
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const SlabArgs& L = A.sl;
  int32_t* Xt = A.b.X[K->tgt];
  uint8_t* flag = A.b.flag[K->tf];
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (uint32_t i = tid; i < L.layer; i += nth) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t b = side ? L.hi - L.layer + i : L.lo + i;
      const int32_t* r = L.recv[side];
      for (uint32_t s = 0; s < A.m.S; ++s) {
        const int32_t v = r[(size_t)s * L.layer + i];
        if (v) Xt[(size_t)s * A.m.Npad + b] += v;
      }
      if (r[(size_t)A.m.S * L.layer + i] == F_SSA && flag[b] == F_SSA_FF) flag[b] = F_SSA;
    }
  }
  for (uint32_t w = 0; w < L.world; ++w) {
    const SlabRemote& R = L.remote_all[w];
    const uint32_t n = R.n < (uint32_t)kSlabRemote ? R.n : (uint32_t)kSlabRemote;
    if (R.n > (uint32_t)kSlabRemote && tid == 0) {
      K->status = PLIS_ERR_LIMIT;
      K->stop_reason = PLIS_STOP_ERROR;
    }
    for (uint32_t j = tid; j < n; j += nth) {
      const uint32_t q = R.cell[j];
      if (q >= L.lo && q < L.hi && flag[q] == F_SSA_FF) flag[q] = F_SSA;
    }
  }
}

// This slab's face layers of the target (final counts of the attempt) into send[0] / send[1].
__global__ void k_slab_pack_faces(KArgs A) {
  const Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const SlabArgs& L = A.sl;
  const int32_t* Xt = A.b.X[K->tgt];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.layer; i += gridDim.x * blockDim.x) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t b = side ? L.hi - L.layer + i : L.lo + i;
      for (uint32_t s = 0; s < A.m.S; ++s) L.send[side][(size_t)s * L.layer + i] = Xt[(size_t)s * A.m.Npad + b];
    }
  }
}

// The neighbours' face layers into this slab's ghost layers of the target: the neighbour counts the
// classification of the faces reads.
__global__ void k_slab_unpack_ghosts(KArgs A) {
  const Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const SlabArgs& L = A.sl;
  int32_t* Xt = A.b.X[K->tgt];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.layer; i += gridDim.x * blockDim.x) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t g = side ? L.hi + i : L.lo - L.layer + i;
      for (uint32_t s = 0; s < A.m.S; ++s) Xt[(size_t)s * A.m.Npad + g] = L.recv[side][(size_t)s * L.layer + i];
    }
  }
}

// The decision from every slab's summary, reduced in rank order exactly as the single domain reduces
// its CTA slots (min tau, then the lowest index), by one thread; identical on every rank.
__global__ void k_slab_control(KArgs A) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ctrl* K = A.b.ctrl;
  if (K->status != PLIS_OK) { K->done = 1; return; }
  double gt = PLIS_INF_D, gp = PLIS_INF_D;
  long long gi = 0x7FFFFFFFFFFFFFFFll;
  unsigned long long gcr = 0, gff = 0;
  uint32_t bad = 0, am_flag = F_SSA_FF;
  for (uint32_t w = 0; w < A.sl.world; ++w) {
    const SlabSummary& q = A.sl.all[w];
    const long long qi = q.idx < 0 ? 0x7FFFFFFFFFFFFFFFll : q.idx;
    if (q.tau < gt || (q.tau == gt && qi < gi)) { gt = q.tau; gi = qi; am_flag = q.am_flag; }
    gp = fmin(gp, q.tau_plain);
    gcr += q.ncr;
    gff += q.nff;
    bad |= q.bad | q.leap_bad;
  }
  if (gi == 0x7FFFFFFFFFFFFFFFll) { gi = -1; am_flag = F_SSA_FF; }
  step_decide(A, K, K->phase, K->tf, gt, gi, gcr, gff, bad, gp, false, am_flag);
}

// After the decision: this slab's face flags (the current flags) into send[0] / send[1], and the ghost
// layers of the next target zeroed (the classification zeroed the slab's own part).
__global__ void k_slab_pack_flags(KArgs A) {
  const Ctrl* K = A.b.ctrl;
  const SlabArgs& L = A.sl;
  const uint8_t* flag = A.b.flag[K->tf];
  int32_t* Xn = A.b.X[K->tgt];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.layer; i += gridDim.x * blockDim.x) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t b = side ? L.hi - L.layer + i : L.lo + i;
      const uint32_t g = side ? L.hi + i : L.lo - L.layer + i;
      L.send[side][(size_t)A.m.S * L.layer + i] = flag[b];
      for (uint32_t s = 0; s < A.m.S; ++s) Xn[(size_t)s * A.m.Npad + g] = 0;
    }
  }
}

// The neighbours' face flags into this slab's ghost flags (the leap reads its receivers' flags).
__global__ void k_slab_unpack_flags(KArgs A) {
  const Ctrl* K = A.b.ctrl;
  const SlabArgs& L = A.sl;
  uint8_t* flag = A.b.flag[K->tf];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < L.layer; i += gridDim.x * blockDim.x) {
    for (int side = 0; side < 2; ++side) {
      if (!(side ? L.has_hi : L.has_lo)) continue;
      const uint32_t g = side ? L.hi + i : L.lo - L.layer + i;
      flag[g] = (uint8_t)L.recv[side][(size_t)A.m.S * L.layer + i];
    }
  }
}
#endif

#ifdef PLIS_ENGINE_HOST_TU
__global__ void k_fill_tau(double* t, uint8_t* f, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { t[i] = PLIS_INF_D; f[i] = F_SSA_FF; }
}
#endif

// kernel launchers of each (precision, species capacity)
template <typename Real, int MAXS>
struct KernelSet {
  static constexpr bool kSmallOk = MAXS <= kSmallS;  // small-model kernels exist for these species counts
  // the event-log variants (LOG = true) only when the handle's log is on: the plain path carries no logging code
  static void leap(const KArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    if constexpr (kSmallOk) {
      if (a.sm.on) {
        if (a.b.ev.rec) launch_pdl(k_leap<Real, MAXS, true, true>, g, b, a.g.box_bytes, s, a);
        else launch_pdl(k_leap<Real, MAXS, false, true>, g, b, a.g.box_bytes, s, a);
        return;
      }
    }
    if (a.b.ev.rec) launch_pdl(k_leap<Real, MAXS, true, false>, g, b, a.g.box_bytes, s, a);
    else launch_pdl(k_leap<Real, MAXS, false, false>, g, b, a.g.box_bytes, s, a);
  }
  static cudaError_t leap_smem(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(k_leap<Real, MAXS, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_leap<Real, MAXS, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if constexpr (kSmallOk) {
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_leap<Real, MAXS, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_leap<Real, MAXS, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    }
    return e;
  }
  static void exact(const KArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    if (a.b.ev.rec) launch_pdl(k_exact<Real, MAXS, true>, g, b, 0, s, a);
    else launch_pdl(k_exact<Real, MAXS, false>, g, b, 0, s, a);
  }
  static void classify(const KArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    if constexpr (kSmallOk) {
      if (a.sm.on) {  // the small-model tables make a propensity cheap: no cache
        launch_pdl(k_classify<Real, MAXS, false, true>, g, b, 0, s, a);
        return;
      }
    }
    // the cache pays once the grid fills the GPU; on a grid of a few CTAs its extra pass only
    // lengthens each thread's chain (measured: 57 -> 62 us per step on 1,000 subvolumes)
    if (a.m.R <= (uint32_t)kPropCache && g.x >= 148u)
      launch_pdl(k_classify<Real, MAXS, true, false>, g, b, (size_t)a.m.R * b.x * sizeof(Real), s, a);
    else
      launch_pdl(k_classify<Real, MAXS, false, false>, g, b, 0, s, a);
  }
};

template <typename Real>
Launchers pick_impl(uint32_t S) {
  if (S <= 1) return {KernelSet<Real, 1>::leap, KernelSet<Real, 1>::exact, KernelSet<Real, 1>::classify, KernelSet<Real, 1>::leap_smem};
  if (S <= 2) return {KernelSet<Real, 2>::leap, KernelSet<Real, 2>::exact, KernelSet<Real, 2>::classify, KernelSet<Real, 2>::leap_smem};
  if (S <= 4) return {KernelSet<Real, 4>::leap, KernelSet<Real, 4>::exact, KernelSet<Real, 4>::classify, KernelSet<Real, 4>::leap_smem};
  if (S <= 8) return {KernelSet<Real, 8>::leap, KernelSet<Real, 8>::exact, KernelSet<Real, 8>::classify, KernelSet<Real, 8>::leap_smem};
  if (S <= 16) return {KernelSet<Real, 16>::leap, KernelSet<Real, 16>::exact, KernelSet<Real, 16>::classify, KernelSet<Real, 16>::leap_smem};
  if (S <= 32) return {KernelSet<Real, 32>::leap, KernelSet<Real, 32>::exact, KernelSet<Real, 32>::classify, KernelSet<Real, 32>::leap_smem};
  if (S <= 64) return {KernelSet<Real, 64>::leap, KernelSet<Real, 64>::exact, KernelSet<Real, 64>::classify, KernelSet<Real, 64>::leap_smem};
  return {KernelSet<Real, 256>::leap, KernelSet<Real, 256>::exact, KernelSet<Real, 256>::classify, KernelSet<Real, 256>::leap_smem};
}


Launchers pick_f64(uint32_t S);
Launchers pick_f32(uint32_t S);

}  // namespace plis

#endif

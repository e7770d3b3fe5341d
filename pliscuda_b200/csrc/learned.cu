// learned.cu — learned tau proposals on the device.
//
//  * cell_features: the proposer's 8 inputs of one subvolume, computed from the same state and the
//    same plain leap bound the classification computes.
//  * warp_mlp: the MLP 8 -> 64 -> 64 -> 64 -> 1 for the 32 subvolumes of a warp on the tensor cores
//    (mma.sync m16n8k16, BF16 operands, FP32 accumulators).  The accumulator fragment of one layer
//    is, after bias + ReLU + BF16 rounding, exactly the A fragment of the next layer, so hidden
//    activations never leave registers; B fragments are pre-packed per lane (16 KB per layer, read
//    through L1).
//  * k_classify_learned (MLP by mma.sync inside the classification) or k_learned_pre + k_mlp_tc
//    (tcgen05, tc_mlp.cuh) + k_learned_post: the classification with proposals, a second (plain)
//    min-tau reduction for the rollback fallback, and the usual last-CTA control.
//  * k_trace_features / k_trace_label: recording of (features, label) pairs from plain steps.
//  * k_train / k_adam / feature statistics / k_pack: training in FP32 (one CTA = 128 records, the
//    forward and backward pass of the whole MLP in shared memory, per-CTA gradients reduced in a
//    fixed order by the Adam kernel, so training is deterministic), then packing of the BF16
//    fragments the inference reads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "engine_kernels.cuh"
#include "learned.h"
#include "learned_dev.cuh"
#include "tc_mlp.cuh"

namespace plis {

// the coordinates of subvolume c (trace kernels)
__device__ __forceinline__ Cell cell_from_index(const DevModel& m, uint32_t c) {
  Cell cl;
  cl.c = c;
  if (m.lattice) {
    cl.x = c % m.X;
    cl.y = (c / m.X) % m.Y;
    cl.z = c / (m.X * m.Y);
  } else {
    cl.x = cl.y = cl.z = 0;
  }
  return cl;
}

// the tcgen05 tile kernel's view of the packed proposer
__device__ __forceinline__ tc::Params tc_params(const LearnedParams* P) {
  tc::Params t;
  t.wimg = P->wimg;
  t.b1 = P->b1;
  t.b2 = P->b2;
  t.b3 = P->b3;
  t.w4 = P->w4;
  t.b4 = P->b4;
  return t;
}

// ------------------------------------------------------------------------------------------------
// classification with proposals
// ------------------------------------------------------------------------------------------------
template <typename Real, int MAXS>
__global__ void __launch_bounds__(256, 2) k_classify_learned(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const ClassifyCtx C = classify_ctx(A, K);
  if (learned_classify_tile<Real, MAXS>(A, K, C, blockIdx.x, gridDim.x)) classify_control(A, K, gridDim.x);
}

// The classification with proposals split in three launches, the MLP on tcgen05 in between:
// k_learned_pre (per subvolume: negativity check, zeroing of the next target, fast-forward or leap
// bound and critical rate, normalised BF16 features), k_mlp_tc (persistent, tc_mlp.cuh), and
// k_learned_post (critical time, decision against the proposal and the plain bound, reductions,
// last-CTA control).  The pre and post passes keep the plain classification's occupancy.
template <typename Real, int MAXS>
__global__ void __launch_bounds__(256) k_learned_pre(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const ClassifyCtx C = classify_ctx(A, K);
  const LearnedParams* P = A.b.lp;
  const DevModel& m = A.m;
  Cell cl;
  const bool valid = cell_of(A, blockIdx.x, cl);
  const uint32_t c = cl.c;
  int bad = 0;
  if (valid) {
    Counts<MAXS> x;
    load_counts(m, C.Xe, c, x);
#pragma unroll
    for (int s = 0; s < MAXS; ++s)
      if (s < (int)m.S) {
        if (x.v[s] < 0) bad = 1;
        C.Xz[(size_t)s * m.Npad + c] = 0;
      }
    Nbr q;
    nbr_info(m, cl, q);
    double tn;
    int fl;
    float f[kFeat];
#pragma unroll
    for (int k = 0; k < kFeat; ++k) f[k] = 0.f;
    if (classify_ff(A.o.mode, C.tau_cur[c], C.flag_cur[c], C.step, C.ff, tn, fl)) {
      A.b.pre[c] = make_double2(tn, 0.0);
      A.b.pre_kind[c] = 1;
    } else {
      Real tau_ncr, rate;
      cell_tau_parts<Real>(A, c, q, x, C.Xe, tau_ncr, rate);
      A.b.pre[c] = make_double2((double)tau_ncr, (double)rate);
      A.b.pre_kind[c] = 2;
      if (!plis_isinf_d((double)tau_ncr)) {
        cell_features<Real>(A, c, q, x, C.Xe, tau_ncr, f);
        normalise(P, f);
      }
    }
    A.b.feat[c] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                             pack_bf16x2(f[6], f[7]));
  }
  const int nbad = __syncthreads_or(bad);
  if (threadIdx.x == 0) A.b.slot_bad[blockIdx.x] = nbad ? 1u : 0u;
}

__global__ void __launch_bounds__(128) k_mlp_tc(const Ctrl* __restrict__ K, const LearnedParams* __restrict__ P,
                                                const uint4* __restrict__ feats, float* __restrict__ y, uint32_t nrows,
                                                uint32_t ntiles, int* status, uint32_t wait_limit) {
  extern __shared__ __align__(128) uint8_t tsm[];
  pdl_entry();
  if (K && K->done) return;
  tc::mlp_tiles(tc_params(P), feats, y, nrows, ntiles, tsm, status, wait_limit);
}

template <typename Real, int MAXS>
__global__ void __launch_bounds__(256) k_learned_post(KArgs A) {
  pdl_entry();
  Ctrl* K = A.b.ctrl;
  if (K->done) return;
  const ClassifyCtx C = classify_ctx(A, K);
  const LearnedParams* P = A.b.lp;
  Cell cl;
  const bool valid = cell_of(A, blockIdx.x, cl);
  const uint32_t c = cl.c;
  double tn = PLIS_INF_D, tp = PLIS_INF_D;
  long long ti = 0x7FFFFFFFFFFFFFFFll;
  int fl = F_SSA_FF;
  if (valid) {
    const double2 pr = A.b.pre[c];
    if (A.b.pre_kind[c] == 1) {
      tn = pr.x;
      tp = tn;
    } else {
      const double tcr = cell_tau_cr<Real>(A, c, C.step, C.attempt, (Real)pr.y);
      int fp;
      cell_decide(pr.x, tcr, tp, fp);
      const float ls = fminf(fmaxf(A.b.ymlp[c], 0.f), P->log_smax);
      const double sc = ls > 0.f ? (double)expf(ls) : 1.0;
      cell_decide(plis_isinf_d(pr.x) ? pr.x : pr.x * sc, tcr, tn, fl);
    }
    C.tau_new[c] = tn;
    C.flag_new[c] = (uint8_t)fl;
    ti = c;
  }
  const int bad = threadIdx.x == 0 ? (int)A.b.slot_bad[blockIdx.x] : 0;
  if (classify_slot_learned(A, K, blockIdx.x, gridDim.x, tn, ti, tp, valid && fl == F_LEAP_CR, bad,
                            valid && fl == F_SSA_FF))
    classify_control(A, K, gridDim.x);
}

// ------------------------------------------------------------------------------------------------
// trace recording
// ------------------------------------------------------------------------------------------------
template <typename Real, int MAXS>
__global__ void k_trace_features(KArgs A, TraceRec* out, uint32_t offset, uint32_t stride, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const DevModel& m = A.m;
  const int32_t* Xe = A.b.X[A.b.ctrl->cur];
  const uint32_t c = offset + i * stride;
  const Cell cl = cell_from_index(m, c);
  Counts<MAXS> x;
  load_counts(m, Xe, c, x);
  Nbr q;
  nbr_info(m, cl, q);
  Real tn, rate;
  cell_tau_parts<Real>(A, c, q, x, Xe, tn, rate);
  TraceRec r;
  cell_features<Real>(A, c, q, x, Xe, tn, r.f);
  r.tau_cao = (float)tn;
  r.tau_step = 0.f;
  r.label = PLIS_NAN_F;
  r.cell = c;
#pragma unroll
  for (int s = 0; s < 4; ++s) r.x[s] = s < (int)m.S ? x.get(s) : 0;
  out[i] = r;
}

// label of each record from the state the step reached: the Cao leap condition on the realised step
template <typename Real, int MAXS>
__global__ void k_trace_label(KArgs A, TraceRec* recs, uint32_t count, double tau_step, float eps) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const DevModel& m = A.m;
  TraceRec r = recs[i];
  const uint32_t c = r.cell;
  const int comp = comp_of(m, c);
  Counts<MAXS> x0, x1;
#pragma unroll
  for (int s = 0; s < MAXS; ++s) x0.v[s] = (s < (int)m.S && s < 4) ? r.x[s] : 0;
  load_counts(m, A.b.X[A.b.ctrl->cur], c, x1);
  const Cell cl = cell_from_index(m, c);
  Nbr q;
  nbr_info(m, cl, q);
  const Real* rr = (const Real*)m.rr;
  float rho = 0.f;
  for (int j = 0; j < (int)m.R; ++j) {
    const float a0 = (float)prop<Real>(m, x0, j, comp), a1 = (float)prop<Real>(m, x1, j, comp);
    const float cj = (float)rr[(size_t)comp * m.R + j];
    if ((a0 > 0.f || a1 > 0.f) && cj > 0.f) rho = fmaxf(rho, fabsf(a1 - a0) / fmaxf(eps * a0, cj));
  }
  for (int s = 0; s < (int)m.S; ++s) {
    const float d = (float)q.n * (float)drate<Real>(m, comp, s);
    if (d > 0.f) {
      const float a0 = d * (float)x0.get(s), a1 = d * (float)x1.get(s);
      rho = fmaxf(rho, fabsf(a1 - a0) / fmaxf(eps * a0, d));
    }
  }
  r.tau_step = (float)tau_step;
  const float lmax = 4.158883083f, lmin = -2.772588722f;  // log 64, log 1/16
  if (!(r.tau_cao > 0.f) || isinf(r.tau_cao) || !(tau_step > 0.0)) {
    r.label = PLIS_NAN_F;
  } else if (rho <= 0.f) {
    r.label = lmax;
  } else {
    const double safe = tau_step / fmax((double)rho, (double)rho * (double)rho);
    r.label = fminf(fmaxf((float)log(safe / (double)r.tau_cao), lmin), lmax);
  }
  recs[i] = r;
}

// persistent grid of the tile kernel: 4 CTAs per SM at most, never more CTAs than tiles
static uint32_t mlp_grid(uint32_t ntiles) {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  const uint32_t g = 4u * (uint32_t)sms;
  return ntiles < g ? (ntiles ? ntiles : 1u) : g;
}

template <typename Real, int MAXS>
struct LearnedSet {
  static void classify(const KArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    launch_pdl(k_classify_learned<Real, MAXS>, g, b, 0, s, a);
  }
  static void classify_split(const KArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    launch_pdl(k_learned_pre<Real, MAXS>, g, b, 0, s, a);
    const uint32_t ntiles = a.m.Npad / 128u + ((a.m.Npad % 128u) ? 1u : 0u);
    launch_pdl(k_mlp_tc, dim3(mlp_grid(ntiles)), dim3(128), tc::kPSmemBytes, s, (const Ctrl*)a.b.ctrl,
               (const LearnedParams*)a.b.lp, (const uint4*)a.b.feat, a.b.ymlp, a.m.Npad, ntiles, (int*)&a.b.ctrl->status,
               a.o.mlp_wait);
    launch_pdl(k_learned_post<Real, MAXS>, g, b, 0, s, a);
  }
  static void features(const KArgs& a, TraceRec* out, uint32_t offset, uint32_t stride, uint32_t count,
                       cudaStream_t s) {
    k_trace_features<Real, MAXS><<<(count + 127) / 128, 128, 0, s>>>(a, out, offset, stride, count);
  }
  static void label(const KArgs& a, TraceRec* recs, uint32_t count, double tau_step, float eps, cudaStream_t s) {
    k_trace_label<Real, MAXS><<<(count + 127) / 128, 128, 0, s>>>(a, recs, count, tau_step, eps);
  }
};

template <typename Real, int MAXS>
static LearnedLaunch learned_set(int mlp) {
  using L = LearnedSet<Real, MAXS>;
  if (mlp == PLIS_MLP_MMA_SYNC) return {L::classify, L::features, L::label};
  if (cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kPSmemBytes) != cudaSuccess)
    return {nullptr, nullptr, nullptr};
  return {L::classify_split, L::features, L::label};
}

template <typename Real>
static LearnedLaunch learned_pick_impl(uint32_t S, int mlp) {
  if (S <= 1) return learned_set<Real, 1>(mlp);
  if (S <= 2) return learned_set<Real, 2>(mlp);
  if (S <= 4) return learned_set<Real, 4>(mlp);
  return {nullptr, nullptr, nullptr};
}

LearnedLaunch learned_pick(int precision, uint32_t S, int mlp_kernel) {
  return precision == PLIS_PREC_FP32 ? learned_pick_impl<float>(S, mlp_kernel) : learned_pick_impl<double>(S, mlp_kernel);
}

// ------------------------------------------------------------------------------------------------
// packing, inference for tests
// ------------------------------------------------------------------------------------------------
// the tcgen05 weight image: element (n, k) of W_l^T (= W_l[k][n]) at its K-major canonical offset
__global__ void k_pack_image(const float* __restrict__ w, LearnedParams* __restrict__ P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // 64*16 + 2*64*64 elements
  if (i >= 64 * 16 + 2 * 64 * 64) return;
  uint16_t* img = reinterpret_cast<uint16_t*>(P->wimg);
  int n, k, base, chunk;
  float v;
  if (i < 64 * 16) {
    n = i / 16;
    k = i % 16;
    v = k < kFeat ? w[kOffW1 + k * kHid + n] : 0.f;
    base = 0;
    chunk = 1024;
  } else {
    const int ii = i - 64 * 16, layer = ii / 4096, e = ii % 4096;
    n = e / 64;
    k = e % 64;
    v = w[(layer == 0 ? kOffW2 : kOffW3) + k * kHid + n];
    base = tc::kW1Bytes + layer * tc::kWBytes;
    chunk = 1024;
  }
  const uint32_t off = (uint32_t)base + tc::canon((uint32_t)n, (uint32_t)k, (uint32_t)chunk);
  const __nv_bfloat16 b = __float2bfloat16_rn(v);
  img[off / 2] = *reinterpret_cast<const uint16_t*>(&b);
}

__global__ void k_pack(const float* __restrict__ w, float log_smax, LearnedParams* __restrict__ P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = i & 31, g = lane >> 2, t = lane & 3;
  if (i < 8 * 32) {
    const int n = 8 * (i >> 5) + g, k = 2 * t;  // K rows 8..15 are the zero padding
    P->w1f[i] = make_uint2(pack_bf16x2(w[kOffW1 + k * kHid + n], w[kOffW1 + (k + 1) * kHid + n]), 0u);
  } else if (i < 8 * 32 + 2 * 32 * 32) {
    const int ii = i - 8 * 32;
    const int layer = ii >> 10, fr = (ii & 1023) >> 5;  // fragment kk * 8 + j
    const int kk = fr >> 3, j = fr & 7;
    const float* W = w + (layer == 0 ? kOffW2 : kOffW3);
    const int n = 8 * j + g, k = 16 * kk + 2 * t;
    const uint2 v = make_uint2(pack_bf16x2(W[k * kHid + n], W[(k + 1) * kHid + n]),
                               pack_bf16x2(W[(k + 8) * kHid + n], W[(k + 9) * kHid + n]));
    if (layer == 0) P->w2f[ii & 1023] = v;
    else P->w3f[ii & 1023] = v;
  }
  if (i < kHid) {
    P->b1[i] = w[kOffB1 + i];
    P->b2[i] = w[kOffB2 + i];
    P->b3[i] = w[kOffB3 + i];
    P->w4[i] = w[kOffW4 + i];
  }
  if (i < kFeat) {
    P->fmean[i] = w[kNParams + i];
    P->finv[i] = w[kNParams + kFeat + i];
  }
  if (i == 0) {
    P->b4 = w[kOffB4];
    P->log_smax = log_smax;
  }
}

void learned_pack(const float* w, double s_max, LearnedParams* out, cudaStream_t s) {
  const float ls = s_max > 1.0 ? (float)std::log(s_max) : 0.f;
  k_pack<<<(8 * 32 + 2 * 32 * 32 + 255) / 256, 256, 0, s>>>(w, ls, out);
  k_pack_image<<<(64 * 16 + 2 * 64 * 64 + 255) / 256, 256, 0, s>>>(w, out);
}

// raw features -> normalised BF16 rows (rows n .. nrows-1 zero)
__global__ void k_feat_rows(const LearnedParams* __restrict__ P, const float* __restrict__ feats, uint64_t n,
                            uint64_t nrows, uint4* __restrict__ rows) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  float f[kFeat];
#pragma unroll
  for (int k = 0; k < kFeat; ++k) f[k] = i < n ? feats[i * kFeat + k] : 0.f;
  if (i < n) normalise(P, f);
  else {
#pragma unroll
    for (int k = 0; k < kFeat; ++k) f[k] = 0.f;
  }
  rows[i] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                       pack_bf16x2(f[6], f[7]));
}

__global__ void k_predict(const LearnedParams* __restrict__ P, const float* __restrict__ feats, uint64_t n,
                          float* __restrict__ y) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float f[kFeat];
#pragma unroll
  for (int k = 0; k < kFeat; ++k) f[k] = i < n ? feats[i * kFeat + k] : 0.f;
  if (i < n) normalise(P, f);
  const float v = warp_mlp(P, f);  // whole warps: the grid covers n rounded up to 128
  if (i < n) y[i] = v;
}

// ------------------------------------------------------------------------------------------------
// training
// ------------------------------------------------------------------------------------------------
constexpr int kTB = 128;          // records per training CTA
constexpr int kLd = kTB + 1;      // row pitch of the activation tiles (bank-conflict-free columns)
constexpr size_t kTrainSmem = (size_t)(kNParams + (kFeat + 3 * kHid) * kLd + kTB + 32) * sizeof(float);
constexpr int kStatN = 2 * kFeat + 2;  // sums of f, f^2, label, count

// dW[k][j] = sum_u A[k][u] G[j][u] for a 64x64 layer: each thread a 4x8 tile
__device__ __forceinline__ void grad_tile(const float* A, const float* G, float* out, int t) {
  const int k0 = (t >> 3) * 4, j0 = (t & 7) * 8;
  float acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int l = 0; l < 8; ++l) acc[i][l] = 0.f;
  for (int u = 0; u < kTB; ++u) {
    float a[4], g[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = A[(k0 + i) * kLd + u];
#pragma unroll
    for (int l = 0; l < 8; ++l) g[l] = G[(j0 + l) * kLd + u];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int l = 0; l < 8; ++l) acc[i][l] = acc[i][l] + a[i] * g[l];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int l = 0; l < 8; ++l) out[(k0 + i) * kHid + j0 + l] = acc[i][l];
}

// column t: H[k] <- (sum_j G[j] W[k][j]) * (H[k] > 0)
__device__ __forceinline__ void backprop_layer(const float* G, float* H, const float* W, int t) {
  float acc[kHid];
#pragma unroll
  for (int k = 0; k < kHid; ++k) acc[k] = 0.f;
  for (int j = 0; j < kHid; ++j) {
    const float gj = G[j * kLd + t];
#pragma unroll
    for (int k = 0; k < kHid; ++k) acc[k] = acc[k] + gj * W[k * kHid + j];
  }
#pragma unroll
  for (int k = 0; k < kHid; ++k) {
    const float h = H[k * kLd + t];
    H[k * kLd + t] = h > 0.f ? acc[k] : 0.f;
  }
}

// column t: H[j] <- relu(b[j] + sum_k In[k] W[k][j])
__device__ __forceinline__ void forward_layer(const float* In, float* H, const float* W, const float* b, int t) {
  float acc[kHid];
#pragma unroll
  for (int j = 0; j < kHid; ++j) acc[j] = b[j];
  for (int k = 0; k < kHid; ++k) {
    const float h = In[k * kLd + t];
#pragma unroll
    for (int j = 0; j < kHid; ++j) acc[j] = acc[j] + h * W[k * kHid + j];
  }
#pragma unroll
  for (int j = 0; j < kHid; ++j) H[j * kLd + t] = fmaxf(acc[j], 0.f);
}

// One CTA: forward and backward pass of 128 records; writes its summed gradient (already scaled by
// inv_batch) and its summed loss.  fixed: record blockIdx*128 + t; else Philox-sampled records.
__global__ void __launch_bounds__(kTB) k_train(const TraceRec* __restrict__ recs, uint64_t n,
                                                const float* __restrict__ W, float* __restrict__ partial,
                                                float* __restrict__ loss_out, uint64_t iter, uint32_t seed_lo,
                                                uint32_t seed_hi, float quantile, int fixed, float inv_batch) {
  extern __shared__ float sm[];
  float* sW = sm;
  float* F = sW + kNParams;
  float* H1 = F + kFeat * kLd;
  float* H2 = H1 + kHid * kLd;
  float* H3 = H2 + kHid * kLd;
  float* dy = H3 + kHid * kLd;
  float* red = dy + kTB;
  const int t = threadIdx.x;
  for (int i = t; i < kNParams; i += kTB) sW[i] = W[i];
  uint64_t idx;
  bool use;
  if (fixed) {
    idx = (uint64_t)blockIdx.x * kTB + t;
    use = idx < n;
  } else {
    plis_u32x4 ctr = {(uint32_t)(blockIdx.x * kTB + t), (uint32_t)iter, (uint32_t)(iter >> 32), 0x7A11u};
    const plis_u32x4 r = plis_philox4x32_10(ctr, seed_lo, seed_hi);
    idx = (((uint64_t)r.x << 32) | r.y) % n;
    use = true;
  }
  float f[kFeat], label = 0.f;
  if (use) {
    const TraceRec& r = recs[idx];
    label = r.label;
    use = !isnan(label);
#pragma unroll
    for (int k = 0; k < kFeat; ++k) f[k] = (r.f[k] - W[kNParams + k]) * W[kNParams + kFeat + k];
  }
  if (!use) {
#pragma unroll
    for (int k = 0; k < kFeat; ++k) f[k] = 0.f;
  }
#pragma unroll
  for (int k = 0; k < kFeat; ++k) F[k * kLd + t] = f[k];
  __syncthreads();
  // forward
  for (int j = 0; j < kHid; ++j) {
    float s = sW[kOffB1 + j];
#pragma unroll
    for (int k = 0; k < kFeat; ++k) s = s + f[k] * sW[kOffW1 + k * kHid + j];
    H1[j * kLd + t] = fmaxf(s, 0.f);
  }
  forward_layer(H1, H2, sW + kOffW2, sW + kOffB2, t);
  forward_layer(H2, H3, sW + kOffW3, sW + kOffB3, t);
  float y = sW[kOffB4];
  for (int j = 0; j < kHid; ++j) y = y + H3[j * kLd + t] * sW[kOffW4 + j];
  float loss = 0.f, g = 0.f;
  if (use) {
    const float res = label - y;
    loss = res >= 0.f ? quantile * res : (quantile - 1.f) * res;
    g = res > 0.f ? -quantile : (res < 0.f ? 1.f - quantile : 0.f);
  }
  dy[t] = g * inv_batch;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((t & 31) == 0) red[t >> 5] = loss;
  __syncthreads();
  if (t == 0) loss_out[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
  float* P = partial + (size_t)blockIdx.x * kNParams;
  // output layer
  if (t < kHid) {
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + H3[t * kLd + u] * dy[u];
    P[kOffW4 + t] = s;
  } else if (t == kHid) {
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + dy[u];
    P[kOffB4] = s;
  }
  __syncthreads();
  {  // G3 = dy * w4 * relu'(H3), in place
    const float d = dy[t];
    for (int j = 0; j < kHid; ++j) {
      const float h = H3[j * kLd + t];
      H3[j * kLd + t] = h > 0.f ? d * sW[kOffW4 + j] : 0.f;
    }
  }
  __syncthreads();
  grad_tile(H2, H3, P + kOffW3, t);
  if (t < kHid) {
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + H3[t * kLd + u];
    P[kOffB3 + t] = s;
  }
  __syncthreads();
  backprop_layer(H3, H2, sW + kOffW3, t);  // G2 in place of H2
  __syncthreads();
  grad_tile(H1, H2, P + kOffW2, t);
  if (t < kHid) {
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + H2[t * kLd + u];
    P[kOffB2 + t] = s;
  }
  __syncthreads();
  backprop_layer(H2, H1, sW + kOffW2, t);  // G1 in place of H1
  __syncthreads();
  for (int e = t; e < kFeat * kHid; e += kTB) {
    const int k = e / kHid, j = e % kHid;
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + F[k * kLd + u] * H1[j * kLd + u];
    P[kOffW1 + e] = s;
  }
  if (t < kHid) {
    float s = 0.f;
    for (int u = 0; u < kTB; ++u) s = s + H1[t * kLd + u];
    P[kOffB1 + t] = s;
  }
}

// gradient = sum over CTAs (fixed order); Adam step when lr > 0, else the gradient into out
__global__ void k_adam(float* __restrict__ W, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ partial, uint32_t nblk, float lr, float bc1, float bc2,
                       float* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNParams) return;
  float g = 0.f;
  for (uint32_t b = 0; b < nblk; ++b) g = g + partial[(size_t)b * kNParams + p];
  if (out) {
    out[p] = g;
    return;
  }
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  W[p] = W[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

// per-CTA sums of the usable records' features, squares, labels and count
__global__ void k_feat_partial(const TraceRec* __restrict__ recs, uint64_t n, double* __restrict__ part) {
  __shared__ double s[kStatN][8];
  double acc[kStatN];
#pragma unroll
  for (int k = 0; k < kStatN; ++k) acc[k] = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const TraceRec& r = recs[i];
    if (isnan(r.label)) continue;
#pragma unroll
    for (int k = 0; k < kFeat; ++k) {
      acc[k] += (double)r.f[k];
      acc[kFeat + k] += (double)r.f[k] * (double)r.f[k];
    }
    acc[2 * kFeat] += (double)r.label;
    acc[2 * kFeat + 1] += 1.0;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kStatN; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kStatN) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s[threadIdx.x][w];
    part[(size_t)blockIdx.x * kStatN + threadIdx.x] = v;
  }
}

// means and inverse deviations into the weights buffer, the label mean into out[0], count out[1]
__global__ void k_feat_final(const double* __restrict__ part, int nblk, float* __restrict__ w, double* __restrict__ out) {
  __shared__ double tot[kStatN];
  if (threadIdx.x < kStatN) {
    double v = 0.0;
    for (int b = 0; b < nblk; ++b) v += part[(size_t)b * kStatN + threadIdx.x];
    tot[threadIdx.x] = v;
  }
  __syncthreads();
  if (threadIdx.x < kFeat) {
    const int k = threadIdx.x;
    const double cnt = tot[2 * kFeat + 1];
    const double mean = cnt > 0 ? tot[k] / cnt : 0.0;
    const double var = cnt > 0 ? tot[kFeat + k] / cnt - mean * mean : 1.0;
    const double sd = sqrt(var > 1e-6 ? var : 1e-6);
    w[kNParams + k] = (float)mean;
    w[kNParams + kFeat + k] = (float)(1.0 / sd);
  }
  if (threadIdx.x == 0) {
    const double cnt = tot[2 * kFeat + 1];
    out[0] = cnt > 0 ? tot[2 * kFeat] / cnt : 0.0;
    out[1] = cnt;
  }
}

// ------------------------------------------------------------------------------------------------
// host: Learner
// ------------------------------------------------------------------------------------------------
#define PLIS_LCU(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      err_ = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
      return e_ == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;             \
    }                                                                                    \
  } while (0)

constexpr int kStatBlocks = 256;

Learner::~Learner() {
  if (device_ >= 0) cudaSetDevice(device_);
  for (void* p : allocs_) cudaFree(p);
  if (stream_) cudaStreamDestroy(stream_);
}

int Learner::dmalloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    err_ = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;
  }
  allocs_.push_back(*p);
  return PLIS_OK;
}

// He-uniform initialisation from a Philox stream, zero biases, identity feature statistics
static void init_weights(std::vector<float>& w, uint64_t seed) {
  w.assign(kNWeights, 0.f);
  uint32_t ctr = 0;
  auto uni = [&](void) {
    plis_u32x4 c = {ctr++, 0x1417u, 0u, 0u};
    const plis_u32x4 r = plis_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    return ((double)(r.x >> 8) + 0.5) / 16777216.0;  // (0, 1)
  };
  auto fill = [&](int off, int fan_in, int count) {
    const double a = std::sqrt(6.0 / fan_in);
    for (int i = 0; i < count; ++i) w[off + i] = (float)((2.0 * uni() - 1.0) * a);
  };
  fill(kOffW1, kFeat, kFeat * kHid);
  fill(kOffW2, kHid, kHid * kHid);
  fill(kOffW3, kHid, kHid * kHid);
  fill(kOffW4, kHid, kHid);
  for (int k = 0; k < kFeat; ++k) w[kNParams + kFeat + k] = 1.f;
}

int Learner::create(uint64_t capacity, int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    err_ = "No CUDA-capable device detected.";
    device_ = -1;
    return PLIS_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) {
    err_ = "device ordinal out of range";
    device_ = -1;
    return PLIS_ERR_INVALID;
  }
  device_ = device;
  PLIS_LCU(cudaSetDevice(device));
  PLIS_LCU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  capacity_ = capacity;
  int rc;
  if ((rc = dmalloc((void**)&recs_, capacity * sizeof(TraceRec)))) return rc;
  if ((rc = dmalloc((void**)&w_, kNWeights * sizeof(float)))) return rc;
  if ((rc = dmalloc((void**)&m_, kNParams * sizeof(float)))) return rc;
  if ((rc = dmalloc((void**)&v_, kNParams * sizeof(float)))) return rc;
  if ((rc = dmalloc((void**)&stats_, (kStatBlocks * kStatN + 2) * sizeof(double)))) return rc;
  if ((rc = dmalloc((void**)&packed_, sizeof(LearnedParams)))) return rc;
  std::vector<float> w;
  init_weights(w, 1);
  PLIS_LCU(cudaMemcpy(w_, w.data(), kNWeights * sizeof(float), cudaMemcpyHostToDevice));
  PLIS_LCU(cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
  return PLIS_OK;
}

int Learner::ensure_train_buffers(uint32_t blocks) {
  if (blocks <= partial_blocks_) return PLIS_OK;
  int rc;
  if ((rc = dmalloc((void**)&partial_, (size_t)blocks * kNParams * sizeof(float)))) return rc;
  if ((rc = dmalloc((void**)&loss_, (size_t)blocks * sizeof(float)))) return rc;
  partial_blocks_ = blocks;
  return PLIS_OK;
}

int Learner::record(Engine& e, uint64_t n_steps, uint32_t stride, double label_eps) {
  if (stride == 0) { err_ = "stride must be positive"; return PLIS_ERR_INVALID; }
  if (label_eps < 0.0) { err_ = "label_epsilon must be >= 0"; return PLIS_ERR_INVALID; }
  PLIS_LCU(cudaSetDevice(device_));
  const uint32_t N = e.model().N;
  for (uint64_t k = 0; k < n_steps; ++k) {
    const uint32_t offset = (uint32_t)(k % stride) % N;
    const uint32_t cnt = (N - offset + stride - 1) / stride;
    if (count_ + cnt > capacity_) break;
    int rc = e.trace_features(recs_ + count_, offset, stride, cnt);
    if (rc) { err_ = e.error(); return rc; }
    plis_stats a, b;
    e.stats(&a);
    rc = e.advance(PLIS_INF_D, 1);
    if (rc) { err_ = e.error(); return rc; }
    e.stats(&b);
    if (b.steps == a.steps) break;  // nothing can fire any more
    rc = e.trace_label(recs_ + count_, cnt, b.time - a.time, label_eps);
    if (rc) { err_ = e.error(); return rc; }
    count_ += cnt;
  }
  return PLIS_OK;
}

int Learner::get_records(uint64_t first, uint64_t n, void* out) {
  if (first + n > count_) { err_ = "record range out of bounds"; return PLIS_ERR_INVALID; }
  PLIS_LCU(cudaSetDevice(device_));
  PLIS_LCU(cudaMemcpy(out, recs_ + first, n * sizeof(TraceRec), cudaMemcpyDeviceToHost));
  return PLIS_OK;
}

int Learner::set_records(const void* recs, uint64_t n) {
  if (n > capacity_) { err_ = "more records than the capacity"; return PLIS_ERR_INVALID; }
  PLIS_LCU(cudaSetDevice(device_));
  if (n) PLIS_LCU(cudaMemcpy(recs_, recs, n * sizeof(TraceRec), cudaMemcpyHostToDevice));
  count_ = n;
  return PLIS_OK;
}

int Learner::feature_stats() {
  k_feat_partial<<<kStatBlocks, 256, 0, stream_>>>(recs_, count_, stats_);
  k_feat_final<<<1, 32, 0, stream_>>>(stats_, kStatBlocks, w_, stats_ + kStatBlocks * kStatN);
  PLIS_LCU(cudaGetLastError());
  return PLIS_OK;
}

int Learner::train(const plis_train_params& p, plis_train_report* out) {
  if (count_ == 0) { err_ = "no records"; return PLIS_ERR_INVALID; }
  if (p.batch == 0 || p.batch % kTB) { err_ = "batch must be a positive multiple of 128"; return PLIS_ERR_INVALID; }
  if (!(p.quantile > 0.f && p.quantile < 1.f)) { err_ = "quantile must be in (0, 1)"; return PLIS_ERR_INVALID; }
  PLIS_LCU(cudaSetDevice(device_));
  const uint32_t nblk = p.batch / kTB;
  int rc = ensure_train_buffers(nblk);
  if (rc) return rc;
  // fresh parameters, then the statistics of these records
  std::vector<float> w;
  init_weights(w, p.seed);
  PLIS_LCU(cudaMemcpyAsync(w_, w.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice, stream_));
  if ((rc = feature_stats())) return rc;
  double st[2];
  PLIS_LCU(cudaMemcpyAsync(st, stats_ + kStatBlocks * kStatN, sizeof st, cudaMemcpyDeviceToHost, stream_));
  PLIS_LCU(cudaStreamSynchronize(stream_));
  if (st[1] < 1.0) { err_ = "no usable records (every label is NaN)"; return PLIS_ERR_INVALID; }
  const float b4 = (float)st[0];
  PLIS_LCU(cudaMemcpyAsync(w_ + kOffB4, &b4, sizeof b4, cudaMemcpyHostToDevice, stream_));
  PLIS_LCU(cudaMemsetAsync(m_, 0, kNParams * sizeof(float), stream_));
  PLIS_LCU(cudaMemsetAsync(v_, 0, kNParams * sizeof(float), stream_));
  cudaEvent_t e0, e1;
  PLIS_LCU(cudaEventCreate(&e0));
  PLIS_LCU(cudaEventCreate(&e1));
  PLIS_LCU(cudaEventRecord(e0, stream_));
  std::vector<float> lossbuf(nblk);
  double loss_first = 0.0, loss_last = 0.0;
  const float inv_b = 1.f / (float)p.batch;
  double b1t = 1.0, b2t = 1.0;
  for (uint64_t it = 0; it < p.iterations; ++it) {
    k_train<<<nblk, kTB, kTrainSmem, stream_>>>(recs_, count_, w_, partial_, loss_, it, (uint32_t)p.seed,
                                                 (uint32_t)(p.seed >> 32), p.quantile, 0, inv_b);
    b1t *= 0.9;
    b2t *= 0.999;
    k_adam<<<(kNParams + 255) / 256, 256, 0, stream_>>>(w_, m_, v_, partial_, nblk, p.learning_rate,
                                                         (float)(1.0 - b1t), (float)(1.0 - b2t), nullptr);
    if (it == 0 || it + 1 == p.iterations) {
      PLIS_LCU(cudaMemcpyAsync(lossbuf.data(), loss_, nblk * sizeof(float), cudaMemcpyDeviceToHost, stream_));
      PLIS_LCU(cudaStreamSynchronize(stream_));
      double s = 0.0;
      for (float v : lossbuf) s += v;
      (it == 0 ? loss_first : loss_last) = s / p.batch;
      if (it == 0) loss_last = loss_first;
    }
  }
  PLIS_LCU(cudaEventRecord(e1, stream_));
  PLIS_LCU(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PLIS_LCU(cudaGetLastError());
  adam_t_ = p.iterations;
  if (out) {
    out->loss_first = loss_first;
    out->loss_last = loss_last;
    out->records = count_;
    out->iterations = p.iterations;
    out->device_ms = ms;
  }
  return PLIS_OK;
}

int Learner::gradient(float* grad, double* loss, float quantile) {
  if (count_ == 0) { err_ = "no records"; return PLIS_ERR_INVALID; }
  PLIS_LCU(cudaSetDevice(device_));
  const uint32_t nblk = (uint32_t)((count_ + kTB - 1) / kTB);
  int rc = ensure_train_buffers(nblk);
  if (rc) return rc;
  float* d_g = nullptr;
  PLIS_LCU(cudaMalloc(&d_g, kNParams * sizeof(float)));
  k_train<<<nblk, kTB, kTrainSmem, stream_>>>(recs_, count_, w_, partial_, loss_, 0, 0, 0, quantile, 1,
                                               1.f / (float)count_);
  k_adam<<<(kNParams + 255) / 256, 256, 0, stream_>>>(w_, m_, v_, partial_, nblk, 0.f, 1.f, 1.f, d_g);
  std::vector<float> lossbuf(nblk);
  cudaError_t e = cudaMemcpyAsync(grad, d_g, kNParams * sizeof(float), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(lossbuf.data(), loss_, nblk * sizeof(float), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  cudaFree(d_g);
  if (e != cudaSuccess) { err_ = cudaGetErrorString(e); return PLIS_ERR_CUDA; }
  double s = 0.0;
  for (float v : lossbuf) s += v;
  if (loss) *loss = s / (double)count_;
  return PLIS_OK;
}

int Learner::predict(const float* features, uint64_t n, float* y, int mlp_kernel) {
  PLIS_LCU(cudaSetDevice(device_));
  if (n == 0) return PLIS_OK;
  float *d_f = nullptr, *d_y = nullptr;
  int* d_st = nullptr;
  PLIS_LCU(cudaMalloc(&d_f, n * kFeat * sizeof(float)));
  cudaError_t e = cudaMalloc(&d_y, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_st, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_st, 0, sizeof(int), stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_f, features, n * kFeat * sizeof(float), cudaMemcpyHostToDevice, stream_);
  if (e == cudaSuccess) {
    learned_pack(w_, 1.0, packed_, stream_);
    if (mlp_kernel == PLIS_MLP_MMA_SYNC) {
      k_predict<<<(unsigned)((n + 127) / 128), 128, 0, stream_>>>(packed_, d_f, n, d_y);
    } else {
      const uint64_t ntiles = (n + 127) / 128;
      uint4* d_rows = nullptr;
      e = cudaMalloc(&d_rows, ntiles * 128 * sizeof(uint4));
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kPSmemBytes);
      if (e == cudaSuccess) {
        k_feat_rows<<<(unsigned)((ntiles * 128 + 255) / 256), 256, 0, stream_>>>(packed_, d_f, n, ntiles * 128, d_rows);
        k_mlp_tc<<<mlp_grid((uint32_t)ntiles), 128, tc::kPSmemBytes, stream_>>>(nullptr, packed_, d_rows, d_y,
                                                                                (uint32_t)n, (uint32_t)ntiles, d_st, 0u);
        e = cudaStreamSynchronize(stream_);
      }
      if (d_rows) cudaFree(d_rows);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  int st = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, d_y, n * sizeof(float), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&st, d_st, sizeof(int), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  cudaFree(d_f);
  if (d_y) cudaFree(d_y);
  if (d_st) cudaFree(d_st);
  if (e != cudaSuccess) { err_ = cudaGetErrorString(e); return PLIS_ERR_CUDA; }
  if (st) { err_ = "tensor-core MLP wait timed out"; return st; }
  return PLIS_OK;
}

int Learner::get_weights(float* w) {
  PLIS_LCU(cudaSetDevice(device_));
  PLIS_LCU(cudaMemcpyAsync(w, w_, kNWeights * sizeof(float), cudaMemcpyDeviceToHost, stream_));
  PLIS_LCU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Learner::set_weights(const float* w) {
  PLIS_LCU(cudaSetDevice(device_));
  PLIS_LCU(cudaMemcpyAsync(w_, w, kNWeights * sizeof(float), cudaMemcpyHostToDevice, stream_));
  PLIS_LCU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

}  // namespace plis

// learned_dev.cuh — device code of learned tau proposals shared by the single-replica kernels
// (learned.cu) and the batched persistent kernel (batch_kernels.cuh): the proposer's features, the
// warp-level tensor-core MLP (mma.sync), and the classification of one brick with proposals.
#ifndef PLIS_LEARNED_DEV_CUH_
#define PLIS_LEARNED_DEV_CUH_

#include <cuda_bf16.h>

#include "engine_kernels.cuh"
#include "learned.h"

namespace plis {

// log1p(x0), log1p(mean neighbour x0), log1p(a_0..a_3), log(tau_Cao), log1p(total diffusion rate)
template <typename Real, int MAXS>
__device__ __forceinline__ void cell_features(const KArgs& A, uint32_t c, const Nbr& q, const Counts<MAXS>& x,
                                              const int32_t* Xe, Real tau_ncr, float f[kFeat]) {
  const DevModel& m = A.m;
  const int comp = comp_of(m, c);
  const float x0 = (float)x.get(0);
  float ns = 0.f;
  for (int j = 0; j < q.n; ++j) ns += (float)Xe[q.nb[j]];
  f[0] = log1pf(x0);
  f[1] = log1pf(q.n > 0 ? ns / (float)q.n : x0);
#pragma unroll
  for (int r = 0; r < 4; ++r) f[2 + r] = r < (int)m.R ? log1pf((float)prop<Real>(m, x, r, comp)) : 0.f;
  f[6] = logf(fminf(fmaxf((float)tau_ncr, 1e-30f), 1e30f));
  float dt = 0.f;
  for (int s = 0; s < (int)m.S; ++s) dt += (float)q.n * ((float)drate<Real>(m, comp, s) * (float)x.get(s));
  f[7] = log1pf(dt);
}

// ------------------------------------------------------------------------------------------------
// warp-level tensor-core MLP
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x (lo) in the low 16 bits
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D = A * B + D, A 16x16 row-major BF16, B 16x8 column-major BF16, D 16x8 FP32
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// Accumulators of the 8 n-tiles of a 64-wide layer -> bias, ReLU, BF16 -> A fragments of the 4
// k-tiles of the next layer (k-tile kk = n-tiles 2kk and 2kk+1).
__device__ __forceinline__ void bias_relu_pack(const float c[8][4], const float* __restrict__ bias, int t,
                                               uint32_t a[4][4]) {
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const int j0 = 2 * kk, j1 = 2 * kk + 1;
    const float b00 = __ldg(&bias[8 * j0 + 2 * t]), b01 = __ldg(&bias[8 * j0 + 2 * t + 1]);
    const float b10 = __ldg(&bias[8 * j1 + 2 * t]), b11 = __ldg(&bias[8 * j1 + 2 * t + 1]);
    a[kk][0] = pack_bf16x2(fmaxf(c[j0][0] + b00, 0.f), fmaxf(c[j0][1] + b01, 0.f));
    a[kk][1] = pack_bf16x2(fmaxf(c[j0][2] + b00, 0.f), fmaxf(c[j0][3] + b01, 0.f));
    a[kk][2] = pack_bf16x2(fmaxf(c[j1][0] + b10, 0.f), fmaxf(c[j1][1] + b11, 0.f));
    a[kk][3] = pack_bf16x2(fmaxf(c[j1][2] + b10, 0.f), fmaxf(c[j1][3] + b11, 0.f));
  }
}

// y of this lane's row from its 8 normalised features.  Every lane of the warp must call it
// (converged): lane l is row l; rows 0..15 and 16..31 are two m16 tiles done one after the other.
static __device__ float warp_mlp(const LearnedParams* __restrict__ P, const float f[kFeat]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t p0 = pack_bf16x2(f[0], f[1]), p1 = pack_bf16x2(f[2], f[3]);
  const uint32_t p2 = pack_bf16x2(f[4], f[5]), p3 = pack_bf16x2(f[6], f[7]);
  float mine = 0.f;
#pragma unroll 1
  for (int mt = 0; mt < 2; ++mt) {
    uint32_t a[4][4];
    {  // layer-1 A fragment: features 2t, 2t+1 of rows g and g+8 of this tile; K 8..15 are zero
      const int s0 = 16 * mt + g, s1 = s0 + 8;
      const uint32_t u0 = __shfl_sync(FULL, p0, s0), u1 = __shfl_sync(FULL, p1, s0);
      const uint32_t u2 = __shfl_sync(FULL, p2, s0), u3 = __shfl_sync(FULL, p3, s0);
      const uint32_t v0 = __shfl_sync(FULL, p0, s1), v1 = __shfl_sync(FULL, p1, s1);
      const uint32_t v2 = __shfl_sync(FULL, p2, s1), v3 = __shfl_sync(FULL, p3, s1);
      a[0][0] = t == 0 ? u0 : t == 1 ? u1 : t == 2 ? u2 : u3;
      a[0][1] = t == 0 ? v0 : t == 1 ? v1 : t == 2 ? v2 : v3;
      a[0][2] = 0u;
      a[0][3] = 0u;
    }
    float c[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
      mma16816(c[j], a[0], __ldg(&P->w1f[j * 32 + lane]));
    }
    bias_relu_pack(c, P->b1, t, a);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) mma16816(c[j], a[kk], __ldg(&P->w2f[(kk * 8 + j) * 32 + lane]));
    }
    bias_relu_pack(c, P->b2, t, a);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) mma16816(c[j], a[kk], __ldg(&P->w3f[(kk * 8 + j) * 32 + lane]));
    }
    // output layer in FP32: rows g (c0, c1) and g + 8 (c2, c3), columns 8j + 2t, 8j + 2t + 1
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int col = 8 * j + 2 * t;
      const float b0 = __ldg(&P->b3[col]), b1 = __ldg(&P->b3[col + 1]);
      const float w0 = __ldg(&P->w4[col]), w1 = __ldg(&P->w4[col + 1]);
      y0 = y0 + fmaxf(c[j][0] + b0, 0.f) * w0 + fmaxf(c[j][1] + b1, 0.f) * w1;
      y1 = y1 + fmaxf(c[j][2] + b0, 0.f) * w0 + fmaxf(c[j][3] + b1, 0.f) * w1;
    }
    y0 += __shfl_xor_sync(FULL, y0, 1);
    y0 += __shfl_xor_sync(FULL, y0, 2);
    y1 += __shfl_xor_sync(FULL, y1, 1);
    y1 += __shfl_xor_sync(FULL, y1, 2);
    const int r = lane - 16 * mt;
    const int src = 4 * (r & 7);
    const float z0 = __shfl_sync(FULL, y0, src), z1 = __shfl_sync(FULL, y1, src);
    if (r >= 0 && r < 16) mine = (r < 8 ? z0 : z1) + P->b4;
  }
  return mine;
}

__device__ __forceinline__ void normalise(const LearnedParams* __restrict__ P, float f[kFeat]) {
#pragma unroll
  for (int k = 0; k < kFeat; ++k) f[k] = (f[k] - __ldg(&P->fmean[k])) * __ldg(&P->finv[k]);
}

// ------------------------------------------------------------------------------------------------
// classification with proposals
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool classify_slot_learned(const KArgs& A, Ctrl* K, uint32_t slot, uint32_t nslots,
                                                      double tn, long long ti, double tp, bool is_cr, int bad,
                                                      bool is_ff) {
  __shared__ double s_t[32];
  __shared__ long long s_i[32];
  __shared__ double s_p[32];
  __shared__ bool s_last;
  const int ncr = __syncthreads_count(is_cr);
  const int nff = __syncthreads_count(is_ff);
  const int nbad = __syncthreads_or(bad);
  warp_min_pair(tn, ti);
  tp = warp_min_d(tp);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_t[wid] = tn; s_i[wid] = ti; s_p[wid] = tp; }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    double bt = s_t[0], bp = s_p[0];
    long long bi = s_i[0];
    for (int w = 1; w < nw; ++w) {
      min_pair(bt, bi, s_t[w], s_i[w]);
      bp = fmin(bp, s_p[w]);
    }
    A.b.slot_tau[slot] = bt;
    A.b.slot_idx[slot] = bi;
    A.b.slot_tau_plain[slot] = bp;
    A.b.slot_cr[slot] = (uint32_t)ncr | ((uint32_t)nff << 16);  // #LEAP_CR | #SSA_FF << 16
    A.b.slot_bad[slot] = nbad ? 1u : 0u;
    __threadfence();
    const uint32_t prev = atomicAdd(&K->blocks_done, 1u);
    s_last = ((prev & 0x7FFFFFFFu) == nslots - 1);
  }
  __syncthreads();
  return s_last;
}

// The classification of one brick with proposals: the tile's subvolume per thread (features, the
// warp's MLP by mma.sync, decisions against the proposal and the plain bound), then its CTA slot
// with the plain min-tau beside the proposed one; true in the CTA that reduces the last slot.  Every
// thread of the CTA must call it (the MLP is warp-collective).
template <typename Real, int MAXS, bool WALK = true>
__device__ __forceinline__ bool learned_classify_tile(const KArgs& A, Ctrl* K, const ClassifyCtx& C, uint32_t tile,
                                                      uint32_t nslots) {
  const LearnedParams* P = A.b.lp;
  const DevModel& m = A.m;
  Cell cl;
  const bool valid = cell_of(A, tile, cl);
  const uint32_t c = cl.c;
  double tn = PLIS_INF_D, tp = PLIS_INF_D;
  long long ti = 0x7FFFFFFFFFFFFFFFll;
  int fl = F_SSA_FF, bad = 0;
  bool ff = false;
  Real tau_ncr = RT<Real>::inf(), rate = (Real)0;
  float f[kFeat];
#pragma unroll
  for (int k = 0; k < kFeat; ++k) f[k] = 0.f;
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
    ff = classify_ff(A.o.mode, C.tau_cur[c], C.flag_cur[c], C.step, C.ff, tn, fl);
    if (!ff) {
      cell_tau_parts<Real, WALK>(A, c, q, x, C.Xe, tau_ncr, rate);
      if (!plis_isinf_d((double)tau_ncr)) {
        cell_features<Real>(A, c, q, x, C.Xe, tau_ncr, f);
        normalise(P, f);
      }
    }
  }
  __syncwarp();
  const float y = warp_mlp(P, f);
  if (valid) {
    if (ff) {
      tp = tn;
    } else {
      const double tcr = cell_tau_cr<Real>(A, c, C.step, C.attempt, rate);
      const double tnd = (double)tau_ncr;
      int fp;
      cell_decide(tnd, tcr, tp, fp);
      const float ls = fminf(fmaxf(y, 0.f), P->log_smax);
      const double sc = ls > 0.f ? (double)expf(ls) : 1.0;
      cell_decide(plis_isinf_d(tnd) ? tnd : tnd * sc, tcr, tn, fl);
    }
    C.tau_new[c] = tn;
    C.flag_new[c] = (uint8_t)fl;
    ti = c;
  }
  return classify_slot_learned(A, K, tile, nslots, tn, ti, tp, valid && fl == F_LEAP_CR, bad, valid && fl == F_SSA_FF);
}

}  // namespace plis

#endif

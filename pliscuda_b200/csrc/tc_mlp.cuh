// tc_mlp.cuh — the proposer's MLP on the 5th-generation tensor cores (tcgen05.mma, accumulators in
// tensor memory), over 128-row tiles.
//
// Layout.  Operands are BF16 in shared memory in the K-major canonical layout without swizzle:
// 8x8-element core matrices of 128 contiguous bytes (8 rows x 16 bytes); core matrix (row group g,
// K chunk c) of an A tile sits at c * LBO + g * 128 (SBO = 128), so within one K chunk the 128 rows
// are contiguous 16-byte rows: the layer-1 tile is the stored features as they are (K chunk 0)
// followed by a zero chunk (K padded from 8 to 16).  A weight image (64 output rows) has
// LBO = 1024.  One tcgen05.mma (M = 128, N = 64, K = 16, kind::f16, BF16 x BF16 -> FP32) covers
// two K chunks: one per tile for layer 1, four for layers 2 and 3.  Accumulators are TMEM columns
// 0..63, lane = row, so after each layer each of the 128 threads reads its own row back with
// tcgen05.ld.32x32b (a warp reads the 32 lanes of its quarter), applies bias + ReLU, rounds to
// BF16 and writes the next layer's A row.
//
// Synchronisation.  One thread issues the MMAs and commits them to an mbarrier; every thread
// waits on it with an iteration limit.  A wait that runs out stops the CTA with a status; TMEM is
// always freed.  A CTA allocates 64 TMEM columns, so the 512 columns of an SM hold 8 CTAs and its
// shared memory keeps at most 5 on an SM: allocation never has to wait.
#ifndef PLIS_TC_MLP_CUH_
#define PLIS_TC_MLP_CUH_

#include <cuda_bf16.h>
#include <stdint.h>

namespace plis {
namespace tc {

constexpr uint32_t kA1Bytes = 2 * 2048;        // A tile of layer 1: 128 rows x K 16
constexpr uint32_t kABytes = 8 * 2048;         // A tile of layers 2, 3: 128 rows x K 64
constexpr uint32_t kW1Bytes = 2 * 1024;        // W1^T: 64 x 16
constexpr uint32_t kWBytes = 8 * 1024;         // W2^T, W3^T: 64 x 64
constexpr uint32_t kWImageBytes = kW1Bytes + 2 * kWBytes;  // 18 KB, the packed weight image
constexpr uint32_t kWaitLimit = 1u << 22;

// instruction descriptor: D F32, A BF16, B BF16, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle (start, leading and stride byte offsets >> 4, version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// byte offset of element (row, k) in a K-major canonical tile whose K chunks are `chunk` bytes apart
__device__ __forceinline__ uint32_t canon(uint32_t row, uint32_t k, uint32_t chunk) {
  return (k >> 3) * chunk + (row >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// wait for the mbarrier phase `parity`; false (and *err set) when the limit ran out
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity, volatile int* err, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (try_wait(bar, parity)) return true;
    if (*err) return false;
  }
  *err = 1;
  return false;
}

struct Params {
  const uint4* wimg;   // packed weight image (kWImageBytes), global
  const float* b1;
  const float* b2;
  const float* b3;
  const float* w4;
  float b4;
};

// Persistent tile kernel: shared memory of one CTA (128 threads, one 128-row tile at a time)
constexpr uint32_t kPOffW = 0;
constexpr uint32_t kPOffA1 = kPOffW + kWImageBytes;  // features: K chunk 0 of the layer-1 A tile
constexpr uint32_t kPOffZero = kPOffA1 + 2048;       // K chunk 1: zeros (the padding of K 8 -> 16)
constexpr uint32_t kPOffA = kPOffZero + 2048;        // A tile of layers 2, 3
constexpr uint32_t kPOffVec = kPOffA + kABytes;
constexpr uint32_t kPOffBar = kPOffVec + 4 * 64 * 4;
constexpr uint32_t kPSmemBytes = kPOffBar + 16;
constexpr uint32_t kPTmemCols = 64;  // <= 8 CTAs per SM ever fit the 512 columns
static_assert(kPSmemBytes * 6 > 228 * 1024, "at most 5 CTAs per SM");

// y[r] for the rows of `feats` (normalised BF16 features, 16 bytes per row, rows 0 .. 128*ntiles-1
// readable) with the MLP on tcgen05.  Tiles are taken round robin; every CTA loads the weights once.
// A wait that runs out sets *status and the CTA stops; TMEM is always freed.
static __device__ void mlp_tiles(const Params& P, const uint4* __restrict__ feats, float* __restrict__ y, uint32_t nrows,
                          uint32_t ntiles, uint8_t* smem, int* status, uint32_t wait_limit = 0) {
  if (wait_limit == 0) wait_limit = kWaitLimit;
  __shared__ int s_err;
  const uint32_t tid = threadIdx.x;  // blockDim.x == 128
  const uint32_t warp = tid >> 5;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar = sbase + kPOffBar;
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kPOffBar + 8);
  float* vec = reinterpret_cast<float*>(smem + kPOffVec);
  if (tid == 0) s_err = 0;
  {
    uint4* dst = reinterpret_cast<uint4*>(smem + kPOffW);
    for (uint32_t i = tid; i < kWImageBytes / 16; i += 128) dst[i] = __ldg(&P.wimg[i]);
    reinterpret_cast<uint4*>(smem + kPOffZero)[tid] = make_uint4(0u, 0u, 0u, 0u);
    if (tid < 64) {
      vec[tid] = __ldg(&P.b1[tid]);
      vec[64 + tid] = __ldg(&P.b2[tid]);
      vec[128 + tid] = __ldg(&P.b3[tid]);
      vec[192 + tid] = __ldg(&P.w4[tid]);
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kPOffBar + 8),
                   "r"(kPTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t my_cols = tmem + ((32u * warp) << 16);
  const volatile int* err = &s_err;
  uint32_t phase = 0;
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const uint32_t r = tile * 128u + tid;
    // row tid of chunk 0 of the layer-1 A tile sits at tid * 16: the features as they are stored
    reinterpret_cast<uint4*>(smem + kPOffA1)[tid] = feats[r];
    fence_before();
    fence_async_smem();
    __syncthreads();
    bool ok = true;
    float out = 0.f;
    for (int layer = 0; layer < 3 && ok; ++layer) {
      if (tid == 0 && !*err) {
        fence_after();
        if (layer == 0) {
          mma(tmem, sdesc(sbase + kPOffA1, kPOffZero - kPOffA1, 128), sdesc(sbase + kPOffW, 1024, 128), 0u);
        } else {
          const uint32_t wofs = kPOffW + kW1Bytes + (layer == 1 ? 0u : kWBytes);
          for (uint32_t ks = 0; ks < 4; ++ks)
            mma(tmem, sdesc(sbase + kPOffA + ks * 2u * 2048u, 2048, 128), sdesc(sbase + wofs + ks * 2u * 1024u, 1024, 128),
                ks > 0 ? 1u : 0u);
        }
        commit(bar);
      }
      bool got = !*err && wait_phase(bar, phase & 1u, (volatile int*)err, wait_limit);
      phase += 1;
      fence_after();
      ok = __syncthreads_and(got && !*err) != 0;
      if (!ok) break;
      if (layer < 2) {
        const float* b = vec + 64 * layer;
        uint8_t* a = smem + kPOffA;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float v[16];
          ld16(my_cols + 16u * c, v);
          uint32_t p[8];
#pragma unroll
          for (int i = 0; i < 8; ++i)
            p[i] = bf16x2(fmaxf(v[2 * i] + b[16 * c + 2 * i], 0.f), fmaxf(v[2 * i + 1] + b[16 * c + 2 * i + 1], 0.f));
          *reinterpret_cast<uint4*>(a + canon(tid, 16u * c, 2048)) = make_uint4(p[0], p[1], p[2], p[3]);
          *reinterpret_cast<uint4*>(a + canon(tid, 16u * c + 8u, 2048)) = make_uint4(p[4], p[5], p[6], p[7]);
        }
      } else {
        const float* b = vec + 128;
        const float* w = vec + 192;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float v[16];
          ld16(my_cols + 16u * c, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) out = out + fmaxf(v[i] + b[16 * c + i], 0.f) * w[16 * c + i];
        }
        out = out + P.b4;
      }
      fence_before();
      fence_async_smem();
      __syncthreads();
    }
    if (!ok) break;
    if (r < nrows) y[r] = out;
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
  if (tid == 0 && s_err) atomicExch(status, 6 /* PLIS_ERR_TIMEOUT */);
}

}  // namespace tc
}  // namespace plis

#endif

// tc_mlp.cuh — the proposer's MLP for the 256 rows of a CTA on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory).
//
// Layout.  Row r of the CTA (its thread r) is row r % 128 of M-tile r / 128.  Operands are BF16 in
// shared memory in the K-major canonical layout without swizzle: 8x8-element core matrices of
// 128 contiguous bytes (8 rows x 16 bytes); core matrix (row group g, K chunk c) of an A tile sits
// at c * 2048 + g * 128 (LBO = 2048, SBO = 128), of a weight image (64 output rows) at
// c * 1024 + g * 128 (LBO = 1024, SBO = 128).  One tcgen05.mma (M = 128, N = 64, K = 16,
// kind::f16, BF16 x BF16 -> FP32) covers two K chunks; layer 1 is one MMA per tile (its K is
// padded from 8 to 16 with zeros), layers 2 and 3 four.  The accumulators of tile t are TMEM
// columns 64t .. 64t + 63, lane = row, so after each layer every thread reads exactly its own row
// back with tcgen05.ld.32x32b (a warp reads the 32 lanes of its quarter), applies bias + ReLU,
// rounds to BF16 and writes the next layer's A row.
//
// Synchronisation.  One thread issues the MMAs and commits them to an mbarrier; every thread
// waits on it with an iteration limit.  A wait that runs out sets *err and the remaining layers
// are skipped; TMEM is always freed.  The CTA allocates 128 TMEM columns and its shared memory
// (kTcSmemBytes) keeps at most 3 CTAs on an SM, so allocation never has to wait.
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
// shared memory: weights | A1 x 2 | A x 2 | b1 b2 b3 w4 (floats) | mbarrier | tmem slot | error
constexpr uint32_t kOffW = 0;
constexpr uint32_t kOffA1 = kOffW + kWImageBytes;
constexpr uint32_t kOffA = kOffA1 + 2 * kA1Bytes;
constexpr uint32_t kOffVec = kOffA + 2 * kABytes;
constexpr uint32_t kOffBar = kOffVec + 4 * 64 * 4;
constexpr uint32_t kUsed = kOffBar + 16;
// padded so that at most 3 CTAs fit on an SM (3 x 128 TMEM columns <= 512)
constexpr uint32_t kTcSmemBytes = 62 * 1024;
static_assert(kUsed <= kTcSmemBytes, "tcgen05 MLP shared memory");
static_assert(4 * (kTcSmemBytes + 1024) > 228 * 1024, "at most 3 CTAs per SM");
constexpr uint32_t kTmemCols = 128;
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
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity, volatile int* err) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
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

// y of this thread's row from its 8 normalised features.  All threads of the CTA (blockDim.x <=
// 256, a multiple of 32) must call it; *err (shared, zero on entry) is set when a wait ran out.
__device__ float mlp_cta(const Params& P, const float f[8], uint8_t* smem, volatile int* err) {
  const uint32_t tid = threadIdx.x, nthr = blockDim.x;
  const uint32_t warp = tid >> 5;
  const uint32_t tile = tid >> 7, row = tid & 127u;
  const uint32_t ntiles = (nthr + 127u) >> 7;
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar = sbase + kOffBar;
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kOffBar + 8);
  float* vec = reinterpret_cast<float*>(smem + kOffVec);
  // weights and vectors into shared memory, mbarrier, TMEM
  {
    uint4* dst = reinterpret_cast<uint4*>(smem + kOffW);
    for (uint32_t i = tid; i < kWImageBytes / 16; i += nthr) dst[i] = __ldg(&P.wimg[i]);
    for (uint32_t i = tid; i < 64; i += nthr) {
      vec[i] = __ldg(&P.b1[i]);
      vec[64 + i] = __ldg(&P.b2[i]);
      vec[128 + i] = __ldg(&P.b3[i]);
      vec[192 + i] = __ldg(&P.w4[i]);
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kOffBar + 8),
                   "r"(kTmemCols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
  }
  // this row of the layer-1 A tile: features 0..7, then the zero chunk
  {
    uint8_t* a1 = smem + kOffA1 + tile * kA1Bytes;
    const uint4 v = make_uint4(bf16x2(f[0], f[1]), bf16x2(f[2], f[3]), bf16x2(f[4], f[5]), bf16x2(f[6], f[7]));
    *reinterpret_cast<uint4*>(a1 + canon(row, 0, 2048)) = v;
    *reinterpret_cast<uint4*>(a1 + canon(row, 8, 2048)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (nthr < ntiles * 128u) {  // rows without a thread: zero
    for (uint32_t r = nthr; r < ntiles * 128u; ++r)
      if (tid == 0) {
        uint8_t* a1 = smem + kOffA1 + (r >> 7) * kA1Bytes;
        *reinterpret_cast<uint4*>(a1 + canon(r & 127u, 0, 2048)) = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(a1 + canon(r & 127u, 8, 2048)) = make_uint4(0u, 0u, 0u, 0u);
      }
  }
  fence_before();
  fence_async_smem();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *slot;
  const uint32_t my_cols = tmem + ((32u * (warp & 3u)) << 16) + 64u * tile;
  float y = 0.f;
  bool ok = true;
  for (int layer = 0; layer < 3; ++layer) {
    if (tid == 0 && !*err) {
      fence_after();
      for (uint32_t t = 0; t < ntiles; ++t) {
        const uint32_t d = tmem + 64u * t;
        if (layer == 0) {
          mma(d, sdesc(sbase + kOffA1 + t * kA1Bytes, 2048, 128), sdesc(sbase + kOffW, 1024, 128), 0u);
        } else {
          const uint32_t wofs = kOffW + kW1Bytes + (layer == 1 ? 0u : kWBytes);
          for (uint32_t ks = 0; ks < 4; ++ks)
            mma(d, sdesc(sbase + kOffA + t * kABytes + ks * 2u * 2048u, 2048, 128),
                sdesc(sbase + wofs + ks * 2u * 1024u, 1024, 128), ks > 0 ? 1u : 0u);
        }
      }
      commit(bar);
    }
    ok = ok && wait_phase(bar, (uint32_t)(layer & 1), err);
    fence_after();
    ok = __syncthreads_and(ok && !*err) != 0;  // CTA-uniform: the loads below are warp-collective
    if (ok) {
      if (layer < 2) {
        const float* b = vec + 64 * layer;
        uint8_t* a = smem + kOffA + tile * kABytes;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float v[16];
          ld16(my_cols + 16u * c, v);
          uint32_t p[8];
#pragma unroll
          for (int i = 0; i < 8; ++i)
            p[i] = bf16x2(fmaxf(v[2 * i] + b[16 * c + 2 * i], 0.f), fmaxf(v[2 * i + 1] + b[16 * c + 2 * i + 1], 0.f));
          *reinterpret_cast<uint4*>(a + canon(row, 16u * c, 2048)) = make_uint4(p[0], p[1], p[2], p[3]);
          *reinterpret_cast<uint4*>(a + canon(row, 16u * c + 8u, 2048)) = make_uint4(p[4], p[5], p[6], p[7]);
        }
      } else {
        const float* b = vec + 128;
        const float* w = vec + 192;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float v[16];
          ld16(my_cols + 16u * c, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) y = y + fmaxf(v[i] + b[16 * c + i], 0.f) * w[16 * c + i];
        }
        y = y + P.b4;
      }
    }
    fence_before();
    fence_async_smem();
    __syncthreads();
  }
  fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  return ok ? y : 0.f;
}

}  // namespace tc
}  // namespace plis

#endif

// noalloc.cu — plis_tau_argmin_noalloc: the step's global min-tau / arg-min reduction for callers
// that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a host application whose own allocator owns
// all device memory (cudaMalloc would bypass its budget), or a latency-critical loop where
// cudaMalloc/cudaFree may synchronise the device.  This entry point takes the caller's device input
// and output buffers and allocates nothing: the per-CTA partial results live in a file-scope
// __device__ array of fixed size (kMaxPartials entries, 16 KiB), which every GPU that loads the
// library keeps until the process exits.
//
// Host code cannot pass the array's name to a kernel (on the host it is only a stand-in for the
// device symbol), so every call looks up its device address in the context current on the calling
// thread with cudaGetSymbolAddress, checks the result, and passes that address to the kernels.  The
// lookup allocates nothing and is cheap; doing it on every call (rather than caching an address per
// device ordinal) keeps it right after cudaDeviceReset and for whichever context the runtime has
// current.  The first call on a device may load the library's device code there (lazy module
// loading), so make it before any stream capture.  All calls share the array and it keeps the last
// call's contents; nothing in it needs to start at zero (every partial a call reads was written by
// the same call).  Two calls whose kernels overlap on the GPU (different streams, or different host
// threads) race on the array.
//
// NaN taus never compare below anything, so they are skipped: an input of NaNs only gives
// (+inf, -1), and NaNs mixed with numbers give the arg-min of the numbers.  An input of +inf only
// gives (+inf, 0): the first index wins the tie.
#include <cuda_runtime.h>

#include <string>

#include "../../include/plis.h"

namespace plis {
void set_error(const std::string& msg);
}

namespace {

constexpr int kThreads = 256;
constexpr int kMaxPartials = 1024;  // CTAs of the first pass = entries of the scratch array

struct Partial {
  double tau;
  long long idx;
};

static __device__ __align__(256) Partial g_argmin_scratch[kMaxPartials];

__device__ __forceinline__ void min_pair(double& t, long long& i, double t2, long long i2) {
  if (t2 < t || (t2 == t && i2 < i)) { t = t2; i = i2; }
}

__device__ __forceinline__ void block_min(double& t, long long& i, double* st, long long* si) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double t2 = __shfl_xor_sync(0xffffffffu, t, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
    min_pair(t, i, t2, i2);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { st[wid] = t; si[wid] = i; }
  __syncthreads();
  if (wid == 0) {
    t = lane < kThreads / 32 ? st[lane] : __longlong_as_double(0x7FF0000000000000ll);
    i = lane < kThreads / 32 ? si[lane] : 0x7FFFFFFFFFFFFFFFll;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double t2 = __shfl_xor_sync(0xffffffffu, t, o);
      const long long i2 = __shfl_xor_sync(0xffffffffu, i, o);
      min_pair(t, i, t2, i2);
    }
  }
}

// pass 1: grid-stride min over the input, one partial per CTA
__global__ void __launch_bounds__(kThreads) k_argmin_partials(const double* __restrict__ tau, long long n, Partial* part) {
  __shared__ double st[32];
  __shared__ long long si[32];
  double t = __longlong_as_double(0x7FF0000000000000ll);
  long long i = 0x7FFFFFFFFFFFFFFFll;
  for (long long k = (long long)blockIdx.x * kThreads + threadIdx.x; k < n; k += (long long)gridDim.x * kThreads)
    min_pair(t, i, tau[k], k);
  block_min(t, i, st, si);
  if (threadIdx.x == 0) part[blockIdx.x] = Partial{t, i};
}

// pass 2: one CTA reduces the partials of pass 1
__global__ void __launch_bounds__(kThreads) k_argmin_final(const Partial* part, int nparts, double* out_tau, long long* out_idx) {
  __shared__ double st[32];
  __shared__ long long si[32];
  double t = __longlong_as_double(0x7FF0000000000000ll);
  long long i = 0x7FFFFFFFFFFFFFFFll;
  for (int k = threadIdx.x; k < nparts; k += kThreads) min_pair(t, i, part[k].tau, part[k].idx);
  block_min(t, i, st, si);
  if (threadIdx.x == 0) {
    *out_tau = t;
    *out_idx = (i == 0x7FFFFFFFFFFFFFFFll) ? -1 : i;
  }
}

}  // namespace

extern "C" int plis_tau_argmin_noalloc(const double* d_tau, uint64_t n, double* d_min_tau, int64_t* d_argmin,
                                       void* stream) {
  if (!d_tau || !d_min_tau || !d_argmin) {
    plis::set_error("plis_tau_argmin_noalloc: null pointer");
    return PLIS_ERR_INVALID;
  }
  if (n == 0 || n > (uint64_t)PLIS_NOALLOC_MAX_TAUS) {
    plis::set_error("plis_tau_argmin_noalloc: n must be in 1.." + std::to_string((unsigned long long)PLIS_NOALLOC_MAX_TAUS));
    return PLIS_ERR_LIMIT;
  }
  Partial* scratch = nullptr;  // the array's device address in the current context
  cudaError_t e = cudaGetSymbolAddress((void**)&scratch, g_argmin_scratch);
  if (e != cudaSuccess || !scratch) {
    plis::set_error(std::string("plis_tau_argmin_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return e == cudaErrorNoDevice ? PLIS_ERR_NO_DEVICE : PLIS_ERR_CUDA;
  }
  const long long nn = (long long)n;
  long long blocks = (nn + kThreads - 1) / kThreads;
  if (blocks > kMaxPartials) blocks = kMaxPartials;
  cudaStream_t s = (cudaStream_t)stream;
  k_argmin_partials<<<(unsigned)blocks, kThreads, 0, s>>>(d_tau, nn, scratch);
  k_argmin_final<<<1, kThreads, 0, s>>>(scratch, (int)blocks, d_min_tau, (long long*)d_argmin);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    plis::set_error(std::string("plis_tau_argmin_noalloc: launch: ") + cudaGetErrorString(e));
    return PLIS_ERR_CUDA;
  }
  return PLIS_OK;
}

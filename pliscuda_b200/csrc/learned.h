// learned.h — learned tau proposals: the proposer's parameter layout, trace records, the launchers
// of the learned classification and the trace kernels, and the host owner of traces and training.
#ifndef PLIS_LEARNED_H_
#define PLIS_LEARNED_H_

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/plis.h"
#include "engine.cuh"

namespace plis {

// MLP 8 -> 64 -> 64 -> 64 -> 1 (ReLU).  Master parameters, binary32, in this order:
constexpr int kFeat = 8, kHid = 64;
constexpr int kOffW1 = 0;                        // W1[8][64]  (input k, unit j) at k*64 + j
constexpr int kOffB1 = kOffW1 + kFeat * kHid;    // b1[64]
constexpr int kOffW2 = kOffB1 + kHid;            // W2[64][64]
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;            // W3[64][64]
constexpr int kOffB3 = kOffW3 + kHid * kHid;
constexpr int kOffW4 = kOffB3 + kHid;            // w4[64]
constexpr int kOffB4 = kOffW4 + kHid;            // b4
constexpr int kNParams = kOffB4 + 1;             // 8961
static_assert(kNParams == 8961, "parameter count");
// plis_learner_get_weights layout: the parameters, then the feature means and inverse deviations
constexpr int kNWeights = kNParams + 2 * kFeat;  // 8977
static_assert(kNWeights == PLIS_PROPOSER_WEIGHTS, "weights layout");

// Device copy the inference reads: the BF16 weight image of the tcgen05 kernel (tc_mlp.cuh), BF16
// B fragments of mma.sync.m16n8k16 (one uint2 per lane per 16x8 tile; layer 1's K is padded from 8
// to 16 with zeros), the rest binary32.
struct LearnedParams {
  uint4 wimg[(2 * 1024 + 2 * 8 * 1024) / 16];  // W1^T, W2^T, W3^T, BF16, tcgen05 K-major canonical image
  uint2 w1f[8 * 32];       // [n-tile][lane]
  uint2 w2f[4 * 8 * 32];   // [k-tile][n-tile][lane]
  uint2 w3f[4 * 8 * 32];
  float b1[kHid], b2[kHid], b3[kHid], w4[kHid];
  float b4;
  float log_smax;          // proposals are s * tau_Cao with log s clamped to [0, log_smax]
  float fmean[kFeat], finv[kFeat];
};

// One recorded subvolume-step (64 bytes).
struct TraceRec {
  float f[kFeat];     // raw features of the recorded state
  float tau_cao;      // its plain leap bound
  float tau_step;     // the step the simulation took from it (label kernel)
  float label;        // log(tau_safe / tau_cao), clamped (label kernel); NaN = unusable record
  uint32_t cell;
  int32_t x[4];       // counts of species 0..3 at the recorded state
};
static_assert(sizeof(TraceRec) == 64, "trace record size");

struct LearnedLaunch {
  void (*classify)(const KArgs&, dim3, dim3, cudaStream_t);
  void (*features)(const KArgs&, TraceRec*, uint32_t offset, uint32_t stride, uint32_t count, cudaStream_t);
  void (*label)(const KArgs&, TraceRec*, uint32_t count, double tau_step, float eps, cudaStream_t);
};
// mlp_kernel: PLIS_MLP_TCGEN05 or PLIS_MLP_MMA_SYNC (include/plis.h)
// nullptr members when the species count is above 4
LearnedLaunch learned_pick(int precision, uint32_t S, int mlp_kernel);
// pack master weights (device, kNWeights floats) into a LearnedParams
void learned_pack(const float* w, double s_max, LearnedParams* out, cudaStream_t s);

class Engine;

class Learner {
 public:
  Learner() = default;
  ~Learner();
  int create(uint64_t capacity, int device);
  int record(Engine& e, uint64_t n_steps, uint32_t stride, double label_eps);
  int count(uint64_t* n) const { *n = count_; return PLIS_OK; }
  int get_records(uint64_t first, uint64_t n, void* out);
  int set_records(const void* recs, uint64_t n);
  int train(const plis_train_params& p, plis_train_report* out);
  int gradient(float* grad, double* loss, float quantile);
  int predict(const float* features, uint64_t n, float* y, int mlp_kernel);
  int get_weights(float* w);
  int set_weights(const float* w);
  const std::string& error() const { return err_; }

 private:
  int dmalloc(void** p, size_t bytes);
  int ensure_train_buffers(uint32_t blocks);
  int feature_stats();
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  uint64_t capacity_ = 0, count_ = 0;
  TraceRec* recs_ = nullptr;
  float* w_ = nullptr;        // master weights [kNWeights]
  float* m_ = nullptr;        // Adam moments
  float* v_ = nullptr;
  float* partial_ = nullptr;  // per-CTA gradients
  float* loss_ = nullptr;     // per-CTA losses
  double* stats_ = nullptr;   // feature statistics scratch
  uint32_t partial_blocks_ = 0;
  LearnedParams* packed_ = nullptr;
  uint64_t adam_t_ = 0;
  std::vector<void*> allocs_;
  std::string err_;
};

}  // namespace plis

#endif

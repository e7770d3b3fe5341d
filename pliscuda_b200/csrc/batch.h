// batch.h — host owner of a batch of independent replicas advanced by one persistent kernel.
#ifndef PLIS_BATCH_H_
#define PLIS_BATCH_H_

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/plis.h"
#include "engine.cuh"
#include "plis_model.h"

namespace plis {

struct RepDesc;
struct BatchArgs;

struct BatchLaunch {
  void* kernel;        // k_batch<Real, MAXS>
  cudaError_t (*set_smem)(int bytes);
};
// small: the network fits the SmallModel tables (every replica's argument block carries them)
BatchLaunch batch_pick_f64(uint32_t S, bool learned, bool small);
BatchLaunch batch_pick_f32(uint32_t S, bool learned, bool small);
void batch_prepare(const BatchArgs& B, double t_end, unsigned long long n_steps, cudaStream_t s);

class BatchEngine {
 public:
  BatchEngine();
  ~BatchEngine();
  int create(const plis_batch_desc& d, const plis_options& opt);
  int set_state(uint32_t r, const uint32_t* counts);
  int get_state(uint32_t r, uint32_t* counts);
  int get_taus(uint32_t r, double* tau, uint8_t* flags);
  int run(double t_end, uint64_t n_steps);
  int stats(uint32_t r, plis_stats* st);
  int autotune(uint64_t pilot_steps, plis_batch_tuning* out);
  int tuning(plis_batch_tuning* out);
  // learned tau proposals for every replica (corrected mode, <= 4 species); null / s_max <= 0 detaches
  int set_proposer(const float* weights, double s_max);
  const std::string& error() const { return err_; }

 private:
  void release();
  int dmalloc(void** p, size_t bytes);
  int layout(const int tile[3]);        // bricks, views, grid for a brick shape
  int launch(uint32_t max_iters);       // one persistent launch
  int init_pending();
  int read_ctrls();

  Model shared_;                        // reaction tables (from replica 0)
  plis_options opt_{};
  uint32_t nrep_ = 0, S_ = 0, R_ = 0;
  std::vector<uint32_t> dims_;          // [nrep*3] squeezed lattice dims
  std::vector<uint32_t> ids_;
  std::vector<uint32_t> coff_, npad_;
  std::vector<double> h_rr_, h_dr_;  // per-replica rate constants (host copies, for the SmallModel blocks)
  bool small_ = false;
  uint64_t ntot_ = 0;
  uint32_t tile_[3] = {0, 0, 0};
  uint32_t total_tiles_ = 0, max_tiles_ = 0;
  int grid_ = 0, blocks_per_sm_ = 0;
  double tuned_rate_ = 0.0;
  std::vector<uint8_t> pending_;
  bool any_pending_ = false;

  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<void*> allocs_;
  std::string err_;
  BatchLaunch launch_{};
  // device
  DevModel dm_{};
  DevOpts dopt_{};
  Geo geo_{};
  void* d_views_ = nullptr;
  void* d_rep_ = nullptr;
  void* d_rr_ = nullptr;
  void* d_dr_ = nullptr;
  Ctrl* d_ctrl_ = nullptr;
  int32_t* d_X_[3] = {nullptr, nullptr, nullptr};
  double* d_tau_[2] = {nullptr, nullptr};
  uint8_t* d_flag_[2] = {nullptr, nullptr};
  int32_t* d_D_ = nullptr;
  double* d_slot_tau_ = nullptr;
  long long* d_slot_idx_ = nullptr;
  uint32_t* d_slot_cr_ = nullptr;
  uint32_t* d_slot_bad_ = nullptr;
  unsigned* d_work_ = nullptr;
  unsigned* d_bar_ = nullptr;
  int* d_err_ = nullptr;
  std::vector<Ctrl> h_ctrl_;
  double device_ms_ = 0.0;
  uint64_t launches_ = 0;
  bool learned_ = false;
  struct LearnedParams* d_lp_ = nullptr;
  float* d_lw_ = nullptr;
  double* d_slot_plain_ = nullptr;
  uint32_t plain_tiles_ = 0;
};

}  // namespace plis

#endif

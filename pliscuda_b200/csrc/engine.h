// engine.h — host-side owner of one simulation on one device (one plis_handle).
#ifndef PLIS_ENGINE_H_
#define PLIS_ENGINE_H_

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/plis.h"
#include "engine.cuh"
#include "learned.h"
#include "plis_model.h"

namespace plis {

// Kernel launchers of one (precision, species-capacity) instantiation.
struct Launchers {
  void (*leap)(const KArgs&, dim3, dim3, cudaStream_t);
  void (*exact)(const KArgs&, dim3, dim3, cudaStream_t);
  void (*classify)(const KArgs&, dim3, dim3, cudaStream_t);
  cudaError_t (*leap_smem)(int bytes);
};

// SmallModel tables of a model (engine.cu); false, with sm->on = 0, when it does not fit.
bool fill_small_model(const Model& M, const double* rrate, const double* drate, SmallModel* sm);

class Engine {
 public:
  Engine();
  ~Engine();
  int create(const Model& model, const plis_options& opt);
  // t0, step0: simulated time and accepted-step counter the state is at (0, 0 for a new run); the
  // step counter keys the random stream, so a trajectory continued from a host copy draws fresh numbers
  int set_state(const uint32_t* counts, double t0 = 0.0, uint64_t step0 = 0);
  int get_state(uint32_t* counts);
  int set_time(double t);
  int get_taus(double* tau, uint8_t* flags);
  int advance(double t_end, uint64_t n_steps);
  int stats(plis_stats* st);
  int profile(plis_profile* p);
  // learned tau proposals (learned.cu): attach (weights != null, s_max >= 1) or detach a proposer
  int set_proposer(const float* weights, double s_max);
  // trace recording: features of every stride-th subvolume of the current state from offset, and
  // the labels of those records once a step has been taken (leap condition at label_eps, 0 = epsilon)
  int trace_features(TraceRec* out, uint32_t offset, uint32_t stride, uint32_t count);
  int trace_label(TraceRec* recs, uint32_t count, double tau_step, double label_eps);
  // event log (plis_set_event_log / plis_read_event_log)
  int set_event_log(uint64_t capacity);
  int read_event_log(plis_event_record* out, uint64_t max_records, uint64_t* n_records, uint64_t* n_dropped,
                     bool clear);
  // z-slab decomposition (plis_slab_*): this handle computes z-layers [z0, z1) of world slabs
  int slab_setup(uint32_t z0, uint32_t z1, uint32_t world, uint32_t rank);
  int slab_phase(int phase, double t_end, uint64_t n_steps);
  int slab_buffers(plis_slab_buffers* out);
  int device() const { return opt_.device; }
  const std::string& error() const { return err_; }
  const Model& model() const { return model_; }

 private:
  void release();
  int dmalloc(void** p, size_t bytes);
  template <typename T> int upload(const std::vector<T>& v, const T** out);
  void enqueue_step();
  void launch_classify();
  int build_graph();
  int read_ctrl();
  int reclassify();

  Model model_;
  plis_options opt_{};
  KArgs args_{};
  Launchers launch_{};
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  Ctrl* h_ctrl_ = nullptr;
  std::vector<void*> allocs_;
  std::string err_;
  int graph_steps_ = 32;
  uint32_t exact_blocks_ = 1;  // CTAs of k_exact / k_apply
  int kernels_per_step_ = 4;
  uint64_t launches_ = 0;
  double device_ms_ = 0.0;
  plis_profile prof_{};
  cudaEvent_t pev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int enqueue_step_profiled();
  bool state_set_ = false;
  bool use_learned_ = false;
  LearnedLaunch llaunch_{};
  LearnedParams* d_lp_ = nullptr;
  float* d_lw_ = nullptr;
  double* d_slot_plain_ = nullptr;
  uint4* d_feat_ = nullptr;
  double2* d_pre_ = nullptr;
  uint8_t* d_pre_kind_ = nullptr;
  float* d_ymlp_ = nullptr;
  EvRec* d_evrec_ = nullptr;
  unsigned long long* d_evhead_ = nullptr;
  uint32_t slab_blocks_ = 0;  // bricks of this handle's z-slab (0: not a slab)
  size_t slab_stage_ = 0;     // int32 words of one staging buffer
};

}  // namespace plis

#endif

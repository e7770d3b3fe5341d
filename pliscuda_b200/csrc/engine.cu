// engine.cu — host side of the B200 step: buffers, control block, CUDA-graph batches.
//
// The device phases are in engine_kernels.cuh; their template instantiations are compiled in
// inst_f64.cu / inst_f32.cu so the build parallelises.
#define PLIS_ENGINE_HOST_TU 1
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine_kernels.cuh"
#include "plis_model.h"

namespace plis {

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
#define PLIS_CU(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      err_ = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
      return e_ == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;             \
    }                                                                                    \
  } while (0)

static uint32_t pow2_at_least(uint32_t v) {
  uint32_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

Engine::Engine() {}

Engine::~Engine() { release(); }

void Engine::release() {
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  graph_exec_ = nullptr;
  if (d_evrec_) cudaFree(d_evrec_);
  if (d_evhead_) cudaFree(d_evhead_);
  d_evrec_ = nullptr;
  d_evhead_ = nullptr;
  for (void* p : allocs_) cudaFree(p);
  allocs_.clear();
  if (h_ctrl_) cudaFreeHost(h_ctrl_);
  h_ctrl_ = nullptr;
  for (auto& e : pev_)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  ev0_ = ev1_ = nullptr;
  if (stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
}

int Engine::dmalloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    err_ = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;
  }
  allocs_.push_back(*p);
  return PLIS_OK;
}

template <typename T>
int Engine::upload(const std::vector<T>& v, const T** out) {
  void* p = nullptr;
  int rc = dmalloc(&p, v.size() * sizeof(T));
  if (rc) return rc;
  if (!v.empty()) PLIS_CU(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = (const T*)p;
  return PLIS_OK;
}

// The SmallModel block of a model that fits it (at most kSmallR reactions and kSmallS species, net
// changes within int8, one set of rate constants: rrate[R] and drate[S]; rrate null = several sets);
// sm->on = 0 otherwise.
bool fill_small_model(const Model& M, const double* rrate, const double* drate, SmallModel* out) {
  SmallModel& sm = *out;
  std::memset(&sm, 0, sizeof sm);
  const ReactionTables& t = M.rt;
  bool fits = rrate && M.R <= (uint32_t)kSmallR && M.S <= (uint32_t)kSmallS;
  for (size_t r = 0; fits && r < M.R; ++r)
    for (size_t s = 0; s < M.S; ++s) {
      const int nu = M.products[s * M.R + r] - M.reactants[s * M.R + r];
      if (nu < -127 || nu > 127) fits = false;
    }
  if (!fits) return false;
  for (uint32_t r = 0; r < M.R; ++r) {
    sm.nreac[r] = t.n_reac[r];
    for (int i = 0; i < t.n_reac[r]; ++i) {
      sm.rs[r][i] = (uint8_t)t.reac_s[r * kMaxReactantSpecies + i];
      sm.rm[r][i] = t.reac_m[r * kMaxReactantSpecies + i];
      sm.rnu[r][i] = (int8_t)t.reac_nu[r * kMaxReactantSpecies + i];
      sm.rmask[sm.rs[r][i]] |= (uint8_t)(1u << r);
    }
    for (int i = 0; i < t.n_net[r]; ++i) sm.nu[r][t.net_s[r * kMaxNet + i]] = (int8_t)t.net_nu[r * kMaxNet + i];
    sm.inv_denom[r] = t.inv_denom[r];
    sm.rate_d[r] = rrate[r];
    sm.rate_f[r] = (float)rrate[r];
  }
  for (uint32_t s = 0; s < M.S; ++s) {
    sm.hor[s] = t.hor[s];
    sm.hmult[s] = t.hmult[s];
    sm.drate_d[s] = drate[s];
    sm.drate_f[s] = (float)drate[s];
  }
  sm.on = 1;
  return true;
}

int Engine::create(const Model& model, const plis_options& opt) {
  model_ = model;
  opt_ = opt;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    err_ = "No CUDA-capable device detected.";
    return PLIS_ERR_NO_DEVICE;
  }
  if (opt.device < 0 || opt.device >= ndev) { err_ = "device ordinal out of range"; return PLIS_ERR_INVALID; }
  PLIS_CU(cudaSetDevice(opt.device));
  PLIS_CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  PLIS_CU(cudaEventCreate(&ev0_));
  PLIS_CU(cudaEventCreate(&ev1_));
  PLIS_CU(cudaMallocHost((void**)&h_ctrl_, sizeof(Ctrl)));
  std::memset(h_ctrl_, 0, sizeof(Ctrl));

  const Model& M = model_;
  DevModel& dm = args_.m;
  std::memset(&dm, 0, sizeof dm);
  dm.N = M.N; dm.S = M.S; dm.R = M.R; dm.C = M.C;
  dm.Npad = (M.N + 31u) & ~31u;
  dm.lattice = M.topo.is_lattice() ? 1u : 0u;
  dm.X = M.topo.lattice[0]; dm.Y = M.topo.lattice[1]; dm.Z = M.topo.lattice[2];
  int rc;
  if (!dm.lattice) {
    if ((rc = upload(M.topo.canon, &dm.canon))) return rc;
    if ((rc = upload(M.topo.ncount, &dm.ncount))) return rc;
  }
  if (!M.topo.orig.empty()) {
    if ((rc = upload(M.topo.orig, &dm.orig))) return rc;
  }
  if (!M.comp.empty()) {
    if ((rc = upload(M.comp, &dm.comp))) return rc;
  }
  const ReactionTables& t = M.rt;
  if ((rc = upload(t.n_reac, &dm.n_reac))) return rc;
  if ((rc = upload(t.n_net, &dm.n_net))) return rc;
  if ((rc = upload(t.reac_s, &dm.reac_s))) return rc;
  if ((rc = upload(t.reac_m, &dm.reac_m))) return rc;
  if ((rc = upload(t.reac_nu, &dm.reac_nu))) return rc;
  if ((rc = upload(t.net_s, &dm.net_s))) return rc;
  if ((rc = upload(t.net_nu, &dm.net_nu))) return rc;
  if ((rc = upload(t.inv_denom, &dm.inv_denom))) return rc;
  if ((rc = upload(t.hor, &dm.hor))) return rc;
  if ((rc = upload(t.hmult, &dm.hmult))) return rc;
  if ((rc = upload(t.sp_off, &dm.sp_off))) return rc;
  if ((rc = upload(t.sp_r, &dm.sp_r))) return rc;
  if ((rc = upload(t.sp_nu, &dm.sp_nu))) return rc;
  if ((rc = upload(t.sr_off, &dm.sr_off))) return rc;
  if ((rc = upload(t.sr_r, &dm.sr_r))) return rc;
  if (opt.precision == PLIS_PREC_FP32) {
    std::vector<float> rr(M.rrate.begin(), M.rrate.end()), dr(M.drate.begin(), M.drate.end());
    const float* p;
    if ((rc = upload(rr, &p))) return rc;
    dm.rr = p;
    if ((rc = upload(dr, &p))) return rc;
    dm.dr = p;
  } else {
    const double* p;
    if ((rc = upload(M.rrate, &p))) return rc;
    dm.rr = p;
    if ((rc = upload(M.drate, &p))) return rc;
    dm.dr = p;
  }

  // a small model's tables in the kernel arguments (SmallModel)
  fill_small_model(M, M.comp.empty() ? M.rrate.data() : nullptr, M.drate.data(), &args_.sm);

  // geometry
  Geo& g = args_.g;
  if (dm.lattice) {
    // default brick: 8 x 8 in x and y and deep enough in z for 256 subvolumes (8 x 8 x 4 on a cube),
    // then wider in x and y where the lattice is too thin in z.  Measured on one B200 against the
    // earlier 32 x 8 x 1 rows: Schlogl 64^3 -1.6 % time, the random network 128^3 -1.1 %, the small
    // A/B 10^3 -0.9 % (the six neighbours of a compact brick are more often in the brick's own lines)
    uint32_t tx, ty, tz;
    if (opt.tile[0] > 0) {
      tx = (uint32_t)opt.tile[0];
      ty = opt.tile[1] > 0 ? (uint32_t)opt.tile[1] : std::min<uint32_t>(std::max<uint32_t>(1, 256 / tx), pow2_at_least(dm.Y));
      tz = opt.tile[2] > 0 ? (uint32_t)opt.tile[2] : std::min<uint32_t>(std::max<uint32_t>(1, 256 / (tx * ty)), pow2_at_least(dm.Z));
    } else if (opt.tile[1] > 0 || opt.tile[2] > 0) {  // y and/or z given: x fills up to 256
      ty = opt.tile[1] > 0 ? (uint32_t)opt.tile[1] : 1u;
      tz = opt.tile[2] > 0 ? (uint32_t)opt.tile[2] : 1u;
      tx = std::min<uint32_t>(std::max<uint32_t>(1, 256 / std::max<uint32_t>(1, ty * tz)), pow2_at_least(dm.X));
    } else {
      const uint32_t px = pow2_at_least(dm.X), py = pow2_at_least(dm.Y), pz = pow2_at_least(dm.Z);
      tx = std::min<uint32_t>(8, px);
      ty = std::min<uint32_t>(8, py);
      tz = std::min<uint32_t>(256 / (tx * ty), pz);
      while (tx * ty * tz < 256 && (tx < px || ty < py)) {
        if (tx < px && (tx <= ty || ty >= py)) tx *= 2;
        else ty *= 2;
      }
    }
    if (tx * ty * tz > 256 || tx * ty * tz == 0) { err_ = "tile must hold 1..256 subvolumes"; return PLIS_ERR_INVALID; }
    g.tx = tx; g.ty = ty; g.tz = tz;
    g.ntx = (dm.X + tx - 1) / tx; g.nty = (dm.Y + ty - 1) / ty; g.ntz = (dm.Z + tz - 1) / tz;
    g.threads = (tx * ty * tz + 31u) & ~31u;  // whole warps: the CTA reductions shuffle full warps
    const uint64_t nb = (uint64_t)g.ntx * g.nty * g.ntz;
    if (nb > 0x7FFFFFFFull) { err_ = "grid too large"; return PLIS_ERR_LIMIT; }
    g.nblocks = (uint32_t)nb;
  } else {
    g.tx = 256; g.ty = g.tz = 1;
    g.threads = 256;
    g.nblocks = (dm.N + 255) / 256;
    g.ntx = g.nblocks; g.nty = g.ntz = 1;
  }
  geo_divisors(g);
  {  // the exact-event kernel takes chunks of kExactChunk subvolumes with up to four CTAs per SM (all
     // resident); on most steps it finds nothing to do, and an early exit costs per CTA
    int nsm = 0;
    PLIS_CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opt.device));
    const uint32_t need = (dm.N + kExactChunk - 1) / kExactChunk, cap = 4u * (uint32_t)(nsm > 0 ? nsm : 1);
    exact_blocks_ = need < cap ? need : cap;
  }

  // buffers
  const size_t cells = (size_t)M.S * dm.Npad;
  DevBufs& b = args_.b;
  for (int i = 0; i < 3; ++i)
    if ((rc = dmalloc((void**)&b.X[i], cells * 4))) return rc;
  for (int i = 0; i < 2; ++i) {
    if ((rc = dmalloc((void**)&b.tau[i], (size_t)dm.Npad * 8))) return rc;
    if ((rc = dmalloc((void**)&b.flag[i], (size_t)dm.Npad))) return rc;
  }
  // the deltas, then the list of rows the exact events wrote (N entries: two rows per event, so more
  // than N/2 events in one attempt fall back to a scan of all deltas)
  if ((rc = dmalloc((void**)&b.D, (cells + dm.Npad) * 4))) return rc;
  PLIS_CU(cudaMemset(b.D, 0, cells * 4));
  if ((rc = dmalloc((void**)&b.slot_tau, (size_t)g.nblocks * 8))) return rc;
  if ((rc = dmalloc((void**)&b.slot_idx, (size_t)g.nblocks * 8))) return rc;
  if ((rc = dmalloc((void**)&b.slot_cr, (size_t)g.nblocks * 4))) return rc;
  if ((rc = dmalloc((void**)&b.slot_bad, (size_t)g.nblocks * 4))) return rc;
  if ((rc = dmalloc((void**)&b.ctrl, sizeof(Ctrl)))) return rc;
  PLIS_CU(cudaMemset(b.ctrl, 0, sizeof(Ctrl)));

  DevOpts& o = args_.o;
  o.mlp_wait = opt.wait_polls > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)opt.wait_polls;
  o.mode = opt.mode;
  o.nc = opt.critical_threshold;
  o.max_rollbacks = opt.max_rollbacks;
  o.eps = opt.epsilon;
  o.seed = opt.seed;
  o.replica = opt.replica;
  devopts_keys(o);
  o.pool = pooled_draws_on(opt.pooled_draws, M.R, M.S);
  if (o.pool) args_.sm.on = 0;  // pooled draws live in the generic leap only

  launch_ = (opt.precision == PLIS_PREC_FP32) ? pick_f32(M.S) : pick_f64(M.S);
  // shared-memory staging of the leap's brick + halo (lattices only, when the box fits)
  g.staged = 0;
  g.box_bytes = 0;
  if (dm.lattice && opt.stage_halo) {
    const size_t bytes = (size_t)(g.tx + 2) * (g.ty + 2) * (g.tz + 2) * M.S * sizeof(int32_t);
    if (bytes <= 200u * 1024u) {
      g.staged = 1;
      g.box_bytes = (uint32_t)bytes;
      if (bytes > 48u * 1024u) PLIS_CU(launch_.leap_smem((int)bytes));
    }
  }
  kernels_per_step_ = (opt.mode == PLIS_MODE_REFERENCE) ? 4 : 3;
  graph_steps_ = opt.steps_per_launch > 0 ? opt.steps_per_launch : 32;
  PLIS_CU(cudaDeviceSynchronize());
  return PLIS_OK;
}

void Engine::launch_classify() {
  const dim3 gc(slab_blocks_ ? slab_blocks_ : args_.g.nblocks), bc(args_.g.threads);
  if (use_learned_) llaunch_.classify(args_, gc, bc, stream_);
  else launch_.classify(args_, gc, bc, stream_);
}

void Engine::enqueue_step() {
  const dim3 gc(args_.g.nblocks), bc(args_.g.threads);
  const dim3 gx(exact_blocks_), bx(256);
  launch_.leap(args_, gc, bc, stream_);
  launch_.exact(args_, gx, bx, stream_);
  if (opt_.mode == PLIS_MODE_REFERENCE) launch_pdl(k_apply, gx, bx, 0, stream_, args_);
  launch_classify();
}

// Profiled step: the same four launches with CUDA events between them, accumulated per kernel.
int Engine::enqueue_step_profiled() {
  const dim3 gc(args_.g.nblocks), bc(args_.g.threads);
  const dim3 gx(exact_blocks_), bx(256);
  for (auto& e : pev_)
    if (!e) PLIS_CU(cudaEventCreate(&e));
  PLIS_CU(cudaEventRecord(pev_[0], stream_));
  launch_.leap(args_, gc, bc, stream_);
  PLIS_CU(cudaEventRecord(pev_[1], stream_));
  launch_.exact(args_, gx, bx, stream_);
  PLIS_CU(cudaEventRecord(pev_[2], stream_));
  if (opt_.mode == PLIS_MODE_REFERENCE) launch_pdl(k_apply, gx, bx, 0, stream_, args_);
  PLIS_CU(cudaEventRecord(pev_[3], stream_));
  launch_classify();
  PLIS_CU(cudaEventRecord(pev_[4], stream_));
  PLIS_CU(cudaEventSynchronize(pev_[4]));
  const int kind[4] = {PLIS_KERNEL_LEAP, PLIS_KERNEL_EXACT, PLIS_KERNEL_APPLY, PLIS_KERNEL_CLASSIFY};
  for (int i = 0; i < 4; ++i) {
    if (i == 2 && opt_.mode != PLIS_MODE_REFERENCE) continue;
    float ms = 0.f;
    PLIS_CU(cudaEventElapsedTime(&ms, pev_[i], pev_[i + 1]));
    prof_.ms[kind[i]] += ms;
    prof_.launches[kind[i]] += 1;
  }
  return PLIS_OK;
}

int Engine::profile(plis_profile* p) {
  *p = prof_;
  return PLIS_OK;
}

int Engine::build_graph() {
  if (graph_exec_) return PLIS_OK;
  cudaGraph_t graph = nullptr;
  PLIS_CU(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < graph_steps_; ++i) enqueue_step();
  PLIS_CU(cudaStreamEndCapture(stream_, &graph));
  cudaError_t e = cudaGraphInstantiate(&graph_exec_, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    err_ = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
    graph_exec_ = nullptr;
    return PLIS_ERR_CUDA;
  }
  return PLIS_OK;
}

int Engine::read_ctrl() {
  PLIS_CU(cudaMemcpyAsync(h_ctrl_, args_.b.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Engine::set_state(const uint32_t* counts, double t0, uint64_t step0) {
  const DevModel& dm = args_.m;
  for (size_t i = 0; i < (size_t)dm.S * dm.N; ++i)
    if (counts[i] >= (1u << 30)) {
      err_ = "counts must be below 2^30";
      return PLIS_ERR_OVERFLOW;
    }
  const size_t cells = (size_t)dm.S * dm.Npad;
  PLIS_CU(cudaMemsetAsync(args_.b.X[0], 0, cells * 4, stream_));
  PLIS_CU(cudaMemcpy2DAsync(args_.b.X[0], (size_t)dm.Npad * 4, counts, (size_t)dm.N * 4, (size_t)dm.N * 4, dm.S,
                            cudaMemcpyHostToDevice, stream_));
  PLIS_CU(cudaMemsetAsync(args_.b.X[1], 0, cells * 4, stream_));
  PLIS_CU(cudaMemsetAsync(args_.b.X[2], 0, cells * 4, stream_));
  PLIS_CU(cudaMemsetAsync(args_.b.D, 0, cells * 4, stream_));
  k_fill_tau<<<(dm.Npad + 255) / 256, 256, 0, stream_>>>(args_.b.tau[0], args_.b.flag[0], dm.Npad);
  k_fill_tau<<<(dm.Npad + 255) / 256, 256, 0, stream_>>>(args_.b.tau[1], args_.b.flag[1], dm.Npad);
  Ctrl k;
  std::memset(&k, 0, sizeof k);
  k.cur = 0; k.tgt = 1; k.spare = 2; k.tf = 0;
  k.touched_on = 1;
  k.phase = 0;
  k.done = 0;
  k.argmin = -1;
  k.last_argmin = -1;
  k.t_end = 0.0;
  k.t = t0;
  k.step = step0;
  *h_ctrl_ = k;
  PLIS_CU(cudaMemcpyAsync(args_.b.ctrl, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, stream_));
  launch_classify();
  launches_ += 3;
  PLIS_CU(cudaGetLastError());
  int rc = read_ctrl();
  if (rc) return rc;
  device_ms_ = 0.0;
  std::memset(&prof_, 0, sizeof prof_);
  state_set_ = true;
  return PLIS_OK;
}

// Classify the current state again (after the classification kernels changed): phase 0 at the
// current step, no fast-forward decrement; time, step and statistics are kept.
int Engine::reclassify() {
  int rc = read_ctrl();
  if (rc) return rc;
  if (h_ctrl_->status != PLIS_OK) return PLIS_OK;
  h_ctrl_->phase = 0;
  h_ctrl_->dt = 0.0;
  h_ctrl_->done = 0;
  PLIS_CU(cudaMemcpyAsync(args_.b.ctrl, h_ctrl_, sizeof(Ctrl), cudaMemcpyHostToDevice, stream_));
  launch_classify();
  launches_ += 1;
  PLIS_CU(cudaGetLastError());
  return read_ctrl();
}

int Engine::set_proposer(const float* weights, double s_max) {
  const bool on = weights != nullptr && s_max > 0.0;
  if (on) {
    if (opt_.mode != PLIS_MODE_CORRECTED) {
      err_ = "learned tau proposals need corrected mode";
      return PLIS_ERR_UNSUPPORTED;
    }
    if (s_max < 1.0) { err_ = "s_max must be >= 1"; return PLIS_ERR_INVALID; }
    if (model_.S > 4) { err_ = "learned tau proposals support up to 4 species"; return PLIS_ERR_LIMIT; }
    llaunch_ = learned_pick(opt_.precision, model_.S, opt_.learned_mlp);
    if (!llaunch_.classify) { err_ = "cannot configure the learned classification kernel"; return PLIS_ERR_CUDA; }
    int rc;
    if (!d_lp_) {
      if ((rc = dmalloc((void**)&d_lp_, sizeof(LearnedParams)))) return rc;
      if ((rc = dmalloc((void**)&d_lw_, PLIS_PROPOSER_WEIGHTS * sizeof(float)))) return rc;
      if ((rc = dmalloc((void**)&d_slot_plain_, (size_t)args_.g.nblocks * sizeof(double)))) return rc;
    }
    if (opt_.learned_mlp == PLIS_MLP_TCGEN05 && !d_feat_) {  // the split classification's buffers
      const size_t rows = ((size_t)args_.m.Npad + 127) / 128 * 128;
      if ((rc = dmalloc((void**)&d_feat_, rows * sizeof(uint4)))) return rc;
      PLIS_CU(cudaMemset(d_feat_, 0, rows * sizeof(uint4)));
      if ((rc = dmalloc((void**)&d_pre_, (size_t)args_.m.Npad * sizeof(double2)))) return rc;
      if ((rc = dmalloc((void**)&d_pre_kind_, (size_t)args_.m.Npad))) return rc;
      if ((rc = dmalloc((void**)&d_ymlp_, rows * sizeof(float)))) return rc;
    }
    PLIS_CU(cudaMemcpyAsync(d_lw_, weights, PLIS_PROPOSER_WEIGHTS * sizeof(float), cudaMemcpyHostToDevice, stream_));
    learned_pack(d_lw_, s_max, d_lp_, stream_);
    PLIS_CU(cudaGetLastError());
    args_.b.lp = d_lp_;
    args_.b.slot_tau_plain = d_slot_plain_;
    args_.b.feat = d_feat_;
    args_.b.pre = d_pre_;
    args_.b.pre_kind = d_pre_kind_;
    args_.b.ymlp = d_ymlp_;
  } else {
    args_.b.lp = nullptr;
    args_.b.slot_tau_plain = nullptr;
  }
  use_learned_ = on;
  const int classify_launches = (on && opt_.learned_mlp == PLIS_MLP_TCGEN05) ? 3 : 1;
  kernels_per_step_ = ((opt_.mode == PLIS_MODE_REFERENCE) ? 4 : 3) + classify_launches - 1;
  if (graph_exec_) {  // the graph holds the kernel arguments by value
    cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
  }
  return state_set_ ? reclassify() : PLIS_OK;
}

int Engine::trace_features(TraceRec* out, uint32_t offset, uint32_t stride, uint32_t count) {
  LearnedLaunch l = learned_pick(opt_.precision, model_.S, PLIS_MLP_MMA_SYNC);
  if (!l.features) { err_ = "trace recording supports up to 4 species"; return PLIS_ERR_LIMIT; }
  if (!state_set_) { err_ = "no state set"; return PLIS_ERR_INVALID; }
  if (count == 0) return PLIS_OK;
  l.features(args_, out, offset, stride, count, stream_);
  launches_ += 1;
  PLIS_CU(cudaGetLastError());
  return PLIS_OK;
}

int Engine::trace_label(TraceRec* recs, uint32_t count, double tau_step, double label_eps) {
  LearnedLaunch l = learned_pick(opt_.precision, model_.S, PLIS_MLP_MMA_SYNC);
  if (!l.label) { err_ = "trace recording supports up to 4 species"; return PLIS_ERR_LIMIT; }
  if (count == 0) return PLIS_OK;
  l.label(args_, recs, count, tau_step, (float)(label_eps > 0.0 ? label_eps : opt_.epsilon), stream_);
  launches_ += 1;
  PLIS_CU(cudaGetLastError());
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Engine::set_time(double t) {
  int rc = read_ctrl();
  if (rc) return rc;
  h_ctrl_->t = t;
  PLIS_CU(cudaMemcpyAsync(&args_.b.ctrl->t, &h_ctrl_->t, sizeof(double), cudaMemcpyHostToDevice, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Engine::get_state(uint32_t* counts) {
  int rc = read_ctrl();
  if (rc) return rc;
  const DevModel& dm = args_.m;
  PLIS_CU(cudaMemcpy2DAsync(counts, (size_t)dm.N * 4, args_.b.X[h_ctrl_->cur], (size_t)dm.Npad * 4, (size_t)dm.N * 4,
                            dm.S, cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Engine::get_taus(double* tau, uint8_t* flags) {
  int rc = read_ctrl();
  if (rc) return rc;
  const uint32_t tf = h_ctrl_->tf;
  if (tau) PLIS_CU(cudaMemcpyAsync(tau, args_.b.tau[tf], (size_t)args_.m.N * 8, cudaMemcpyDeviceToHost, stream_));
  if (flags) PLIS_CU(cudaMemcpyAsync(flags, args_.b.flag[tf], args_.m.N, cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int Engine::set_event_log(uint64_t capacity) {
  if (capacity > (1ull << 36)) { err_ = "event log capacity above 2^36 records"; return PLIS_ERR_LIMIT; }
  PLIS_CU(cudaSetDevice(opt_.device));
  PLIS_CU(cudaStreamSynchronize(stream_));
  if (d_evrec_) cudaFree(d_evrec_);
  if (d_evhead_) cudaFree(d_evhead_);
  d_evrec_ = nullptr;
  d_evhead_ = nullptr;
  args_.b.ev = EvLog{nullptr, nullptr, 0};
  if (capacity) {
    PLIS_CU(cudaMalloc((void**)&d_evrec_, capacity * sizeof(EvRec)));
    PLIS_CU(cudaMalloc((void**)&d_evhead_, sizeof(unsigned long long)));
    PLIS_CU(cudaMemsetAsync(d_evhead_, 0, sizeof(unsigned long long), stream_));
    PLIS_CU(cudaStreamSynchronize(stream_));
    args_.b.ev = EvLog{d_evrec_, d_evhead_, (unsigned long long)capacity};
  }
  if (graph_exec_) {  // the graph holds the kernel arguments by value
    cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
  }
  return PLIS_OK;
}

int Engine::read_event_log(plis_event_record* out, uint64_t max_records, uint64_t* n_records, uint64_t* n_dropped,
                           bool clear) {
  static_assert(sizeof(plis_event_record) == sizeof(EvRec), "record layouts differ");
  *n_records = 0;
  *n_dropped = 0;
  if (!d_evhead_) return PLIS_OK;
  unsigned long long head = 0;
  PLIS_CU(cudaMemcpyAsync(&head, d_evhead_, sizeof head, cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  const uint64_t cap = args_.b.ev.cap;
  const uint64_t stored = head < cap ? head : cap;
  const uint64_t n = stored < max_records ? stored : max_records;
  if (n) {
    if (!out) { err_ = "null record buffer"; return PLIS_ERR_INVALID; }
    PLIS_CU(cudaMemcpyAsync(out, d_evrec_, n * sizeof(EvRec), cudaMemcpyDeviceToHost, stream_));
  }
  if (clear) PLIS_CU(cudaMemsetAsync(d_evhead_, 0, sizeof(unsigned long long), stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  *n_records = stored;
  *n_dropped = head - stored;
  return PLIS_OK;
}

int Engine::advance(double t_end, uint64_t n_steps) {
  if (slab_blocks_) { err_ = "a z-slab advances through plis_slab_phase"; return PLIS_ERR_UNSUPPORTED; }
  const bool few = n_steps != ~0ull && n_steps < (uint64_t)graph_steps_;
  if (!few && !opt_.profile) {  // the one-off capture and instantiation stay out of the timed interval
    int rc = build_graph();
    if (rc) return rc;
  }
  PLIS_CU(cudaEventRecord(ev0_, stream_));
  k_prepare<<<1, 32, 0, stream_>>>(args_, t_end, (unsigned long long)n_steps);
  launches_ += 1;
  PLIS_CU(cudaGetLastError());
  if (opt_.profile) {  // one step at a time, events around every kernel
    while (true) {
      int rc = enqueue_step_profiled();
      if (rc) return rc;
      launches_ += kernels_per_step_;
      PLIS_CU(cudaGetLastError());
      rc = read_ctrl();
      if (rc) return rc;
      if (h_ctrl_->done) break;
    }
    PLIS_CU(cudaEventRecord(ev1_, stream_));
    PLIS_CU(cudaEventSynchronize(ev1_));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    device_ms_ += ms;
    if (h_ctrl_->status != PLIS_OK) { err_ = "device step failed"; return h_ctrl_->status; }
    return PLIS_OK;
  }
  uint64_t budget = few ? n_steps : 0;
  while (true) {
    if (few) {
      for (uint64_t i = 0; i < budget; ++i) enqueue_step();
      launches_ += budget * kernels_per_step_;
    } else {
      PLIS_CU(cudaGraphLaunch(graph_exec_, stream_));
      launches_ += (uint64_t)graph_steps_ * kernels_per_step_;
    }
    PLIS_CU(cudaGetLastError());
    int rc = read_ctrl();
    if (rc) return rc;
    if (h_ctrl_->done) break;
    if (few) {  // rollbacks used up some of the per-call launches
      budget = 1;
    }
  }
  PLIS_CU(cudaEventRecord(ev1_, stream_));
  PLIS_CU(cudaEventSynchronize(ev1_));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  device_ms_ += ms;
  if (h_ctrl_->status != PLIS_OK) {
    err_ = h_ctrl_->status == PLIS_ERR_STUCK ? "too many consecutive rollbacks in one step" : "device step failed";
    return h_ctrl_->status;
  }
  return PLIS_OK;
}

// ------------------------------------------------------------------------------------------------
// z-slab decomposition
// ------------------------------------------------------------------------------------------------
int Engine::slab_setup(uint32_t z0, uint32_t z1, uint32_t world, uint32_t rank) {
  const DevModel& dm = args_.m;
  const Geo& g = args_.g;
  if (!dm.lattice) { err_ = "z-slabs need a lattice topology"; return PLIS_ERR_UNSUPPORTED; }
  if (state_set_) { err_ = "plis_slab_setup comes before plis_set_state"; return PLIS_ERR_INVALID; }
  if (slab_blocks_) { err_ = "this handle is already a slab"; return PLIS_ERR_INVALID; }
  if (use_learned_ || args_.b.ev.rec || opt_.profile) {
    err_ = "learned proposals, the event log and profiling are not available on a slab";
    return PLIS_ERR_UNSUPPORTED;
  }
  if (world < 1 || rank >= world) { err_ = "rank must be below world"; return PLIS_ERR_INVALID; }
  if (!(z0 < z1 && z1 <= dm.Z) || z0 % g.tz != 0 || (z1 % g.tz != 0 && z1 != dm.Z)) {
    err_ = "a slab is whole bricks along z: z0 < z1 <= Z, both multiples of the brick's z extent (or z1 = Z)";
    return PLIS_ERR_INVALID;
  }
  SlabArgs& L = args_.sl;
  std::memset(&L, 0, sizeof L);
  L.layer = dm.X * dm.Y;
  L.lo = z0 * L.layer;
  L.hi = z1 * L.layer;
  L.has_lo = z0 > 0 ? 1u : 0u;
  L.has_hi = z1 < dm.Z ? 1u : 0u;
  L.world = world;
  L.rank = rank;
  L.brick0 = (z0 / g.tz) * g.ntx * g.nty;
  slab_blocks_ = ((z1 - z0 + g.tz - 1) / g.tz) * g.ntx * g.nty;
  slab_stage_ = (size_t)(dm.S + 1) * L.layer;
  int rc;
  if ((rc = dmalloc((void**)&L.summary, sizeof(SlabSummary)))) return rc;
  if ((rc = dmalloc((void**)&L.all, (size_t)world * sizeof(SlabSummary)))) return rc;
  if ((rc = dmalloc((void**)&L.remote, sizeof(SlabRemote)))) return rc;
  if ((rc = dmalloc((void**)&L.remote_all, (size_t)world * sizeof(SlabRemote)))) return rc;
  for (int i = 0; i < 2; ++i) {
    if ((rc = dmalloc((void**)&L.send[i], slab_stage_ * 4))) return rc;
    if ((rc = dmalloc((void**)&L.recv[i], slab_stage_ * 4))) return rc;
    PLIS_CU(cudaMemset(L.send[i], 0, slab_stage_ * 4));
    PLIS_CU(cudaMemset((void*)L.recv[i], 0, slab_stage_ * 4));
  }
  PLIS_CU(cudaMemset((void*)L.all, 0, (size_t)world * sizeof(SlabSummary)));
  PLIS_CU(cudaMemset((void*)L.remote_all, 0, (size_t)world * sizeof(SlabRemote)));
  L.on = 1;
  if (graph_exec_) {  // the graph holds the kernel arguments by value
    cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
  }
  return PLIS_OK;
}

int Engine::slab_buffers(plis_slab_buffers* out) {
  if (!slab_blocks_) { err_ = "not a slab (plis_slab_setup)"; return PLIS_ERR_INVALID; }
  const SlabArgs& L = args_.sl;
  for (int i = 0; i < 2; ++i) {
    out->send[i] = L.send[i];
    out->recv[i] = (void*)L.recv[i];
  }
  out->stage_words = slab_stage_;
  out->summary = L.summary;
  out->summary_all = (void*)L.all;
  out->summary_bytes = sizeof(SlabSummary);
  out->remote = L.remote;
  out->remote_all = (void*)L.remote_all;
  out->remote_bytes = sizeof(SlabRemote);
  return PLIS_OK;
}

int Engine::slab_phase(int phase, double t_end, uint64_t n_steps) {
  if (!slab_blocks_) { err_ = "not a slab (plis_slab_setup)"; return PLIS_ERR_INVALID; }
  if (!state_set_) { err_ = "no state set"; return PLIS_ERR_INVALID; }
  const dim3 gc(slab_blocks_), bc(args_.g.threads);
  const dim3 gx(exact_blocks_), bx(256);
  const uint32_t lb = (args_.sl.layer + 255u) / 256u;
  const dim3 gl(lb < 1024u ? lb : 1024u), bl(256);
  PLIS_CU(cudaEventRecord(ev0_, stream_));
  switch (phase) {
    case PLIS_SLAB_CLASSIFY:
      launch_classify();
      launches_ += 1;
      break;
    case PLIS_SLAB_CONTROL:
      k_slab_control<<<1, 32, 0, stream_>>>(args_);
      k_slab_pack_flags<<<gl, bl, 0, stream_>>>(args_);
      launches_ += 2;
      break;
    case PLIS_SLAB_FLAGS:
      k_slab_unpack_flags<<<gl, bl, 0, stream_>>>(args_);
      launches_ += 1;
      break;
    case PLIS_SLAB_PREPARE:
      k_prepare<<<1, 32, 0, stream_>>>(args_, t_end, (unsigned long long)n_steps);
      launches_ += 1;
      break;
    case PLIS_SLAB_LEAP:
      PLIS_CU(cudaMemsetAsync(args_.sl.remote, 0, sizeof(SlabRemote), stream_));
      launch_.leap(args_, gc, bc, stream_);
      launch_.exact(args_, gx, bx, stream_);
      if (opt_.mode == PLIS_MODE_REFERENCE) k_apply<<<gx, bx, 0, stream_>>>(args_);
      k_slab_pack_ghosts<<<gl, bl, 0, stream_>>>(args_);
      launches_ += opt_.mode == PLIS_MODE_REFERENCE ? 4 : 3;
      break;
    case PLIS_SLAB_MERGE:
      k_slab_merge<<<gl, bl, 0, stream_>>>(args_);
      k_slab_pack_faces<<<gl, bl, 0, stream_>>>(args_);
      launches_ += 2;
      break;
    case PLIS_SLAB_UNPACK:
      k_slab_unpack_ghosts<<<gl, bl, 0, stream_>>>(args_);
      launches_ += 1;
      break;
    default:
      err_ = "unknown slab phase";
      return PLIS_ERR_INVALID;
  }
  PLIS_CU(cudaGetLastError());
  PLIS_CU(cudaEventRecord(ev1_, stream_));
  PLIS_CU(cudaEventSynchronize(ev1_));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  device_ms_ += ms;
  return PLIS_OK;
}

int Engine::stats(plis_stats* st) {
  int rc = read_ctrl();
  if (rc) return rc;
  const Ctrl& k = *h_ctrl_;
  std::memset(st, 0, sizeof *st);
  st->time = k.t;
  st->steps = k.step;
  st->rollbacks = k.rollbacks;
  st->events = k.events;
  st->exact_events = k.exact_events;
  st->stop_reason = k.stop_reason;
  st->status = k.status;
  st->last_tau = k.last_tau;
  st->last_argmin = k.last_argmin;
  st->device_ms = device_ms_;
  st->kernel_launches = launches_;
  return PLIS_OK;
}

}  // namespace plis

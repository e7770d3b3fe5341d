// batch.cu — host side of the batched persistent driver: layout of the replicas, the cooperative
// launch, the per-replica state and statistics, and the brick-shape autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "batch.h"
#include "engine.h"
#include "learned.h"
#include "batch_kernels.cuh"

namespace plis {

__global__ void k_batch_prepare(BatchArgs B, double t_end, unsigned long long n_steps) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B.nrep) return;
  Ctrl* K = B.ctrl + r;
  if (K->status != PLIS_OK || K->phase != 1u) {
    if (K->status != PLIS_OK) { K->done = 1; K->stop_reason = PLIS_STOP_ERROR; }
    return;
  }
  K->t_end = t_end;
  K->max_step = (n_steps == ~0ull) ? ~0ull : K->step + n_steps;
  K->done = 0;
  K->stop_reason = PLIS_STOP_NONE;
  prepare_step(K, B.o.mode);
}

__global__ void k_batch_fill(double* tau0, double* tau1, uint8_t* f0, uint8_t* f1, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    tau0[i] = PLIS_INF_D;
    tau1[i] = PLIS_INF_D;
    f0[i] = F_SSA_FF;
    f1[i] = F_SSA_FF;
  }
}

#define PLIS_CU(call)                                                               \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      err_ = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
      return e_ == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;        \
    }                                                                               \
  } while (0)

BatchEngine::BatchEngine() {}
BatchEngine::~BatchEngine() { release(); }

void BatchEngine::release() {
  for (void* p : allocs_) cudaFree(p);
  allocs_.clear();
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
  ev0_ = ev1_ = nullptr;
  stream_ = nullptr;
}

int BatchEngine::dmalloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    err_ = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PLIS_ERR_OOM : PLIS_ERR_CUDA;
  }
  allocs_.push_back(*p);
  return PLIS_OK;
}

template <typename T>
static int upload_vec(BatchEngine* self, int (BatchEngine::*alloc)(void**, size_t), const std::vector<T>& v,
                      const T** out, std::string* err) {
  void* p = nullptr;
  int rc = (self->*alloc)(&p, v.size() * sizeof(T));
  if (rc) return rc;
  if (!v.empty()) {
    cudaError_t e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      *err = std::string("cudaMemcpy: ") + cudaGetErrorString(e);
      return PLIS_ERR_CUDA;
    }
  }
  *out = (const T*)p;
  return PLIS_OK;
}

int BatchEngine::create(const plis_batch_desc& d, const plis_options& opt) {
  opt_ = opt;
  if (d.n_replicas < 1 || d.n_replicas > (uint32_t)kMaxBatchReplicas) {
    err_ = "n_replicas must be in 1..4096";
    return PLIS_ERR_LIMIT;
  }
  if (d.n_species < 1 || d.n_species > 16) { err_ = "a batch supports 1..16 species"; return PLIS_ERR_LIMIT; }
  if (!d.reactants || !d.products || !d.lattice || !d.reaction_rates || !d.diffusion_rates) {
    err_ = "missing batch arrays";
    return PLIS_ERR_INVALID;
  }
  nrep_ = d.n_replicas;
  S_ = d.n_species;
  R_ = d.n_reactions;
  // the reaction tables (shared) and validation of the network, through the single-replica builder
  plis_model_desc md;
  std::memset(&md, 0, sizeof md);
  md.n_subvolumes = d.lattice[0] * d.lattice[1] * d.lattice[2];
  md.n_species = S_;
  md.n_reactions = R_;
  md.n_compartments = 1;
  md.lattice_x = d.lattice[0];
  md.lattice_y = d.lattice[1];
  md.lattice_z = d.lattice[2];
  md.reactants = d.reactants;
  md.products = d.products;
  md.reaction_rates = d.reaction_rates;
  md.diffusion_rates = d.diffusion_rates;
  int rc = build_model(&md, &shared_, &err_);
  if (rc) return rc;
  dims_.assign((size_t)nrep_ * 3, 0);
  ids_.assign(nrep_, 0);
  coff_.assign(nrep_, 0);
  npad_.assign(nrep_, 0);
  uint64_t off = 0;
  for (uint32_t r = 0; r < nrep_; ++r) {
    const uint64_t n = (uint64_t)d.lattice[3 * r] * d.lattice[3 * r + 1] * d.lattice[3 * r + 2];
    if (n < 1 || n >= (1ull << 31)) { err_ = "replica " + std::to_string(r) + ": empty or too large lattice"; return PLIS_ERR_INVALID; }
    Topology t;
    rc = canonicalize((uint32_t)n, nullptr, &d.lattice[3 * r], &t, &err_);
    if (rc) return rc;
    for (int k = 0; k < 3; ++k) dims_[3 * r + k] = t.lattice[k];
    for (uint32_t j = 0; j < R_; ++j) {
      const double v = d.reaction_rates[(size_t)r * R_ + j];
      if (!(v >= 0.0) || !std::isfinite(v)) { err_ = "reaction rate constants must be finite and >= 0"; return PLIS_ERR_INVALID; }
    }
    for (uint32_t j = 0; j < S_; ++j) {
      const double v = d.diffusion_rates[(size_t)r * S_ + j];
      if (!(v >= 0.0) || !std::isfinite(v)) { err_ = "diffusion rate constants must be finite and >= 0"; return PLIS_ERR_INVALID; }
    }
    ids_[r] = d.replica_ids ? d.replica_ids[r] : r;
    coff_[r] = (uint32_t)off;
    npad_[r] = (uint32_t)((n + 31) & ~31ull);
    off += npad_[r];
    if (off >= (1ull << 32)) { err_ = "batch too large"; return PLIS_ERR_LIMIT; }
  }
  ntot_ = off;

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    err_ = "No CUDA-capable device detected.";
    return PLIS_ERR_NO_DEVICE;
  }
  if (opt.device < 0 || opt.device >= ndev) { err_ = "device ordinal out of range"; return PLIS_ERR_INVALID; }
  PLIS_CU(cudaSetDevice(opt.device));
  int coop = 0;
  PLIS_CU(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, opt.device));
  if (!coop) { err_ = "device does not support cooperative launches"; return PLIS_ERR_UNSUPPORTED; }
  PLIS_CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  PLIS_CU(cudaEventCreate(&ev0_));
  PLIS_CU(cudaEventCreate(&ev1_));

  // shared reaction tables
  const ReactionTables& t = shared_.rt;
  std::memset(&dm_, 0, sizeof dm_);
  dm_.S = S_;
  dm_.R = R_;
  dm_.C = 1;
  dm_.lattice = 1;
  dm_.Npad = (uint32_t)ntot_;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.n_reac, &dm_.n_reac, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.n_net, &dm_.n_net, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.reac_s, &dm_.reac_s, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.reac_m, &dm_.reac_m, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.reac_nu, &dm_.reac_nu, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.net_s, &dm_.net_s, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.net_nu, &dm_.net_nu, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.inv_denom, &dm_.inv_denom, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.hor, &dm_.hor, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.hmult, &dm_.hmult, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.sp_off, &dm_.sp_off, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.sp_r, &dm_.sp_r, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.sp_nu, &dm_.sp_nu, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.sr_off, &dm_.sr_off, &err_))) return rc;
  if ((rc = upload_vec(this, &BatchEngine::dmalloc, t.sr_r, &dm_.sr_r, &err_))) return rc;
  // per-replica rate tables in the working precision
  const std::vector<double> rr(d.reaction_rates, d.reaction_rates + (size_t)nrep_ * R_);
  const std::vector<double> dr(d.diffusion_rates, d.diffusion_rates + (size_t)nrep_ * S_);
  h_rr_ = rr;
  h_dr_ = dr;
  {  // small networks: every replica's tables and rate constants in its argument block (SmallModel)
    SmallModel probe;
    small_ = fill_small_model(shared_, rr.data(), dr.data(), &probe);
  }
  if (opt.precision == PLIS_PREC_FP32) {
    const std::vector<float> rf(rr.begin(), rr.end()), df(dr.begin(), dr.end());
    const float* p;
    if ((rc = upload_vec(this, &BatchEngine::dmalloc, rf, &p, &err_))) return rc;
    d_rr_ = (void*)p;
    if ((rc = upload_vec(this, &BatchEngine::dmalloc, df, &p, &err_))) return rc;
    d_dr_ = (void*)p;
  } else {
    const double* p;
    if ((rc = upload_vec(this, &BatchEngine::dmalloc, rr, &p, &err_))) return rc;
    d_rr_ = (void*)p;
    if ((rc = upload_vec(this, &BatchEngine::dmalloc, dr, &p, &err_))) return rc;
    d_dr_ = (void*)p;
  }
  dopt_.mode = opt.mode;
  dopt_.nc = opt.critical_threshold;
  dopt_.max_rollbacks = opt.max_rollbacks;
  dopt_.eps = opt.epsilon;
  dopt_.seed = opt.seed;
  dopt_.replica = 0;
  devopts_keys(dopt_);
  dopt_.pool = pooled_draws_on(opt.pooled_draws, R_, S_);
  if (dopt_.pool) small_ = false;  // pooled draws live in the generic leap only

  const size_t cells = (size_t)S_ * ntot_;
  for (int i = 0; i < 3; ++i)
    if ((rc = dmalloc((void**)&d_X_[i], cells * 4))) return rc;
  for (int i = 0; i < 2; ++i) {
    if ((rc = dmalloc((void**)&d_tau_[i], ntot_ * 8))) return rc;
    if ((rc = dmalloc((void**)&d_flag_[i], ntot_))) return rc;
  }
  if ((rc = dmalloc((void**)&d_D_, cells * 4))) return rc;
  if ((rc = dmalloc((void**)&d_ctrl_, (size_t)nrep_ * sizeof(Ctrl)))) return rc;
  if ((rc = dmalloc((void**)&d_work_, 12 * sizeof(unsigned)))) return rc;
  if ((rc = dmalloc((void**)&d_bar_, 2 * sizeof(unsigned)))) return rc;
  if ((rc = dmalloc((void**)&d_err_, sizeof(int)))) return rc;
  if ((rc = dmalloc(&d_views_, (size_t)nrep_ * sizeof(KArgs)))) return rc;
  if ((rc = dmalloc(&d_rep_, (size_t)nrep_ * sizeof(RepDesc)))) return rc;
  PLIS_CU(cudaMemset(d_X_[0], 0, cells * 4));
  PLIS_CU(cudaMemset(d_X_[1], 0, cells * 4));
  PLIS_CU(cudaMemset(d_X_[2], 0, cells * 4));
  PLIS_CU(cudaMemset(d_D_, 0, cells * 4));
  PLIS_CU(cudaMemset(d_err_, 0, sizeof(int)));
  h_ctrl_.assign(nrep_, Ctrl());
  for (auto& k : h_ctrl_) {
    std::memset(&k, 0, sizeof k);
    k.cur = 0; k.tgt = 1; k.spare = 2; k.tf = 0;
    k.done = 1;
    k.argmin = -1;
    k.last_argmin = -1;
  }
  PLIS_CU(cudaMemcpy(d_ctrl_, h_ctrl_.data(), nrep_ * sizeof(Ctrl), cudaMemcpyHostToDevice));
  pending_.assign(nrep_, 2);  // 2 = never given a state
  launch_ = (opt.precision == PLIS_PREC_FP32) ? batch_pick_f32(S_, false, small_) : batch_pick_f64(S_, false, small_);
  int tile[3] = {opt.tile[0], opt.tile[1], opt.tile[2]};
  if (tile[0] <= 0 || tile[1] <= 0 || tile[2] <= 0) { tile[0] = 8; tile[1] = 8; tile[2] = 4; }
  rc = layout(tile);
  if (rc) return rc;
  PLIS_CU(cudaDeviceSynchronize());
  return PLIS_OK;
}

int BatchEngine::layout(const int tile[3]) {
  const uint32_t tx = (uint32_t)tile[0], ty = (uint32_t)tile[1], tz = (uint32_t)tile[2];
  if (tx * ty * tz < 1 || tx * ty * tz > 256) { err_ = "tile must hold 1..256 subvolumes"; return PLIS_ERR_INVALID; }
  tile_[0] = tx; tile_[1] = ty; tile_[2] = tz;
  std::memset(&geo_, 0, sizeof geo_);
  geo_.tx = tx; geo_.ty = ty; geo_.tz = tz;
  geo_.threads = (tx * ty * tz + 31u) & ~31u;
  geo_.staged = 0;
  geo_.box_bytes = 0;
  if (opt_.stage_halo) {
    const size_t bytes = (size_t)(tx + 2) * (ty + 2) * (tz + 2) * S_ * sizeof(int32_t);
    if (bytes <= 96u * 1024u) {
      geo_.staged = 1;
      geo_.box_bytes = (uint32_t)bytes;
    }
  }
  std::vector<RepDesc> rep(nrep_);
  uint64_t toff = 0;
  for (uint32_t r = 0; r < nrep_; ++r) {
    RepDesc& q = rep[r];
    q.X = dims_[3 * r]; q.Y = dims_[3 * r + 1]; q.Z = dims_[3 * r + 2];
    q.N = q.X * q.Y * q.Z;
    q.coff = coff_[r];
    q.ntx = (q.X + tx - 1) / tx; q.nty = (q.Y + ty - 1) / ty; q.ntz = (q.Z + tz - 1) / tz;
    q.ntiles = q.ntx * q.nty * q.ntz;
    q.tile_off = (uint32_t)toff;
    q.replica_id = ids_[r];
    toff += q.ntiles;
  }
  if (toff >= (1ull << 31)) { err_ = "too many bricks"; return PLIS_ERR_LIMIT; }
  total_tiles_ = (uint32_t)toff;
  int rc;
  if (total_tiles_ > max_tiles_) {
    if ((rc = dmalloc((void**)&d_slot_tau_, (size_t)total_tiles_ * 8))) return rc;
    if ((rc = dmalloc((void**)&d_slot_idx_, (size_t)total_tiles_ * 8))) return rc;
    if ((rc = dmalloc((void**)&d_slot_cr_, (size_t)total_tiles_ * 4))) return rc;
    if ((rc = dmalloc((void**)&d_slot_bad_, (size_t)total_tiles_ * 4))) return rc;
    max_tiles_ = total_tiles_;
  }
  if (learned_ && total_tiles_ > plain_tiles_) {
    if ((rc = dmalloc((void**)&d_slot_plain_, (size_t)total_tiles_ * 8))) return rc;
    plain_tiles_ = total_tiles_;
  }
  std::vector<KArgs> views(nrep_);
  const size_t rsz = opt_.precision == PLIS_PREC_FP32 ? sizeof(float) : sizeof(double);
  for (uint32_t r = 0; r < nrep_; ++r) {
    KArgs& v = views[r];
    std::memset(&v, 0, sizeof v);
    v.m = dm_;
    v.m.X = rep[r].X; v.m.Y = rep[r].Y; v.m.Z = rep[r].Z; v.m.N = rep[r].N;
    v.m.lattice = 1;
    v.m.rr = (const char*)d_rr_ + (size_t)r * R_ * rsz;
    v.m.dr = (const char*)d_dr_ + (size_t)r * S_ * rsz;
    v.o = dopt_;
    v.o.replica = ids_[r];
    devopts_keys(v.o);
    v.g = geo_;
    v.g.ntx = rep[r].ntx; v.g.nty = rep[r].nty; v.g.ntz = rep[r].ntz;
    geo_divisors(v.g);
    v.g.nblocks = rep[r].ntiles;
    for (int i = 0; i < 3; ++i) v.b.X[i] = d_X_[i] + coff_[r];
    for (int i = 0; i < 2; ++i) {
      v.b.tau[i] = d_tau_[i] + coff_[r];
      v.b.flag[i] = d_flag_[i] + coff_[r];
    }
    v.b.D = d_D_ + coff_[r];
    v.b.slot_tau = d_slot_tau_ + rep[r].tile_off;
    v.b.slot_idx = d_slot_idx_ + rep[r].tile_off;
    v.b.slot_cr = d_slot_cr_ + rep[r].tile_off;
    v.b.slot_bad = d_slot_bad_ + rep[r].tile_off;
    v.b.ctrl = d_ctrl_ + r;
    if (small_) fill_small_model(shared_, &h_rr_[(size_t)r * R_], &h_dr_[(size_t)r * S_], &v.sm);
    if (learned_) {
      v.b.lp = d_lp_;
      v.b.slot_tau_plain = d_slot_plain_ + rep[r].tile_off;
    }
  }
  PLIS_CU(cudaMemcpy(d_views_, views.data(), nrep_ * sizeof(KArgs), cudaMemcpyHostToDevice));
  PLIS_CU(cudaMemcpy(d_rep_, rep.data(), nrep_ * sizeof(RepDesc), cudaMemcpyHostToDevice));
  const uint32_t dyn = batch_dyn_smem(geo_.box_bytes, nrep_);
  if (dyn > 48u * 1024u) PLIS_CU(launch_.set_smem((int)dyn));
  int bps = 0, sms = 0;
  PLIS_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, launch_.kernel, (int)geo_.threads, dyn));
  PLIS_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt_.device));
  if (bps < 1) { err_ = "the persistent kernel does not fit on an SM"; return PLIS_ERR_UNSUPPORTED; }
  blocks_per_sm_ = bps;
  grid_ = bps * sms;
  return PLIS_OK;
}

static BatchArgs make_args(const DevModel& dm, const DevOpts& o, const Geo& g, void* views, void* rep, uint32_t nrep,
                           uint32_t R, uint32_t S, void* rr, void* dr, Ctrl* ctrl, int32_t* const X[3],
                           double* const tau[2], uint8_t* const flag[2], int32_t* D, double* st, long long* si,
                           uint32_t* sc, uint32_t* sb, unsigned* work, unsigned* bar, int* err, uint32_t iters) {
  BatchArgs B;
  std::memset(&B, 0, sizeof B);
  B.m = dm;
  B.o = o;
  B.g = g;
  B.views = (const KArgs*)views;
  B.rep = (const RepDesc*)rep;
  B.nrep = nrep;
  B.rs = R;
  B.ss = S;
  B.rr = rr;
  B.dr = dr;
  B.ctrl = ctrl;
  for (int i = 0; i < 3; ++i) B.X[i] = X[i];
  for (int i = 0; i < 2; ++i) { B.tau[i] = tau[i]; B.flag[i] = flag[i]; }
  B.D = D;
  B.slot_tau = st; B.slot_idx = si; B.slot_cr = sc; B.slot_bad = sb;
  B.work = work;
  B.bar = bar;
  B.err = err;
  B.spin_limit = 1ull << 26;  // x >= 32 ns per poll: a barrier gives up after at least ~2 s
  B.max_iters = iters;
  B.plan_off = batch_plan_offset(g.box_bytes);
  return B;
}

void batch_prepare(const BatchArgs& B, double t_end, unsigned long long n_steps, cudaStream_t s) {
  k_batch_prepare<<<(B.nrep + 127) / 128, 128, 0, s>>>(B, t_end, n_steps);
}

int BatchEngine::launch(uint32_t max_iters) {
  BatchArgs B = make_args(dm_, dopt_, geo_, d_views_, d_rep_, nrep_, R_, S_, d_rr_, d_dr_, d_ctrl_, d_X_, d_tau_,
                          d_flag_, d_D_, d_slot_tau_, d_slot_idx_, d_slot_cr_, d_slot_bad_, d_work_, d_bar_, d_err_,
                          max_iters);
  if (opt_.wait_polls) B.spin_limit = opt_.wait_polls;
  PLIS_CU(cudaMemsetAsync(d_work_, 0, 12 * sizeof(unsigned), stream_));
  PLIS_CU(cudaMemsetAsync(d_bar_, 0, 2 * sizeof(unsigned), stream_));
  PLIS_CU(cudaMemsetAsync(d_err_, 0, sizeof(int), stream_));  // a timed-out launch does not poison the next
  void* args[] = {&B};
  PLIS_CU(cudaLaunchCooperativeKernel(launch_.kernel, dim3(grid_), dim3(geo_.threads), args,
                                      batch_dyn_smem(geo_.box_bytes, nrep_), stream_));
  launches_ += 1;
  return PLIS_OK;
}

int BatchEngine::set_proposer(const float* weights, double s_max) {
  const bool on = weights != nullptr && s_max > 0.0;
  if (on) {
    if (opt_.mode != PLIS_MODE_CORRECTED) { err_ = "learned tau proposals need corrected mode"; return PLIS_ERR_UNSUPPORTED; }
    if (s_max < 1.0) { err_ = "s_max must be >= 1"; return PLIS_ERR_INVALID; }
    if (S_ > 4) { err_ = "learned tau proposals support up to 4 species"; return PLIS_ERR_LIMIT; }
    int rc;
    if (!d_lp_) {
      if ((rc = dmalloc((void**)&d_lp_, sizeof(LearnedParams)))) return rc;
      if ((rc = dmalloc((void**)&d_lw_, PLIS_PROPOSER_WEIGHTS * sizeof(float)))) return rc;
    }
    PLIS_CU(cudaMemcpyAsync(d_lw_, weights, PLIS_PROPOSER_WEIGHTS * sizeof(float), cudaMemcpyHostToDevice, stream_));
    learned_pack(d_lw_, s_max, d_lp_, stream_);
    PLIS_CU(cudaGetLastError());
    PLIS_CU(cudaStreamSynchronize(stream_));
  }
  learned_ = on;
  launch_ = (opt_.precision == PLIS_PREC_FP32) ? batch_pick_f32(S_, on, small_) : batch_pick_f64(S_, on, small_);
  const int tile[3] = {(int)tile_[0], (int)tile_[1], (int)tile_[2]};
  int rc = layout(tile);
  if (rc) return rc;
  // classify every replica's current state again (time, step and statistics are kept)
  if ((rc = read_ctrls())) return rc;
  for (uint32_t r = 0; r < nrep_; ++r) {
    if (pending_[r] != 0) continue;
    Ctrl& k = h_ctrl_[r];
    if (k.status != PLIS_OK) continue;
    k.phase = 0;
    k.dt = 0.0;
    k.done = 0;
    pending_[r] = 1;
    any_pending_ = true;
  }
  PLIS_CU(cudaMemcpy(d_ctrl_, h_ctrl_.data(), nrep_ * sizeof(Ctrl), cudaMemcpyHostToDevice));
  return init_pending();
}

int BatchEngine::read_ctrls() {
  PLIS_CU(cudaMemcpyAsync(h_ctrl_.data(), d_ctrl_, nrep_ * sizeof(Ctrl), cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int BatchEngine::set_state(uint32_t r, const uint32_t* counts) {
  if (r >= nrep_) { err_ = "replica index out of range"; return PLIS_ERR_INVALID; }
  const uint32_t n = dims_[3 * r] * dims_[3 * r + 1] * dims_[3 * r + 2];
  for (size_t i = 0; i < (size_t)S_ * n; ++i)
    if (counts[i] >= (1u << 30)) { err_ = "counts must be below 2^30"; return PLIS_ERR_OVERFLOW; }
  int rc = read_ctrls();
  if (rc) return rc;
  const size_t pitch = ntot_ * 4;
  for (int i = 0; i < 3; ++i) PLIS_CU(cudaMemset2DAsync(d_X_[i] + coff_[r], pitch, 0, (size_t)npad_[r] * 4, S_, stream_));
  PLIS_CU(cudaMemset2DAsync(d_D_ + coff_[r], pitch, 0, (size_t)npad_[r] * 4, S_, stream_));
  PLIS_CU(cudaMemcpy2DAsync(d_X_[0] + coff_[r], pitch, counts, (size_t)n * 4, (size_t)n * 4, S_,
                            cudaMemcpyHostToDevice, stream_));
  k_batch_fill<<<(npad_[r] + 255) / 256, 256, 0, stream_>>>(d_tau_[0] + coff_[r], d_tau_[1] + coff_[r],
                                                           d_flag_[0] + coff_[r], d_flag_[1] + coff_[r], npad_[r]);
  Ctrl& k = h_ctrl_[r];
  std::memset(&k, 0, sizeof k);
  k.cur = 0; k.tgt = 1; k.spare = 2; k.tf = 0;
  k.phase = 0;
  k.done = 0;
  k.argmin = -1;
  k.last_argmin = -1;
  PLIS_CU(cudaMemcpyAsync(d_ctrl_ + r, &k, sizeof(Ctrl), cudaMemcpyHostToDevice, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  pending_[r] = 1;
  any_pending_ = true;
  return PLIS_OK;
}

int BatchEngine::init_pending() {
  if (!any_pending_) return PLIS_OK;
  int rc = launch(4);  // classification only: pending replicas are in phase 0, the others are done
  if (rc) return rc;
  rc = read_ctrls();
  if (rc) return rc;
  int err = 0;
  PLIS_CU(cudaMemcpy(&err, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) { err_ = "a grid barrier of the persistent kernel timed out"; return PLIS_ERR_TIMEOUT; }
  for (uint32_t r = 0; r < nrep_; ++r)
    if (pending_[r] == 1) pending_[r] = 0;
  any_pending_ = false;
  return PLIS_OK;
}

int BatchEngine::run(double t_end, uint64_t n_steps) {
  for (uint32_t r = 0; r < nrep_; ++r)
    if (pending_[r] == 2) { err_ = "replica " + std::to_string(r) + " has no state"; return PLIS_ERR_INVALID; }
  int rc = init_pending();
  if (rc) return rc;
  BatchArgs B = make_args(dm_, dopt_, geo_, d_views_, d_rep_, nrep_, R_, S_, d_rr_, d_dr_, d_ctrl_, d_X_, d_tau_,
                          d_flag_, d_D_, d_slot_tau_, d_slot_idx_, d_slot_cr_, d_slot_bad_, d_work_, d_bar_, d_err_, 0);
  PLIS_CU(cudaEventRecord(ev0_, stream_));
  batch_prepare(B, t_end, (unsigned long long)n_steps, stream_);
  launches_ += 1;
  PLIS_CU(cudaGetLastError());
  while (true) {
    rc = launch(1u << 24);
    if (rc) return rc;
    rc = read_ctrls();
    if (rc) return rc;
    int err = 0;
    PLIS_CU(cudaMemcpy(&err, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) { err_ = "a grid barrier of the persistent kernel timed out"; return PLIS_ERR_TIMEOUT; }
    bool all = true;
    for (const Ctrl& k : h_ctrl_) all = all && k.done;
    if (all) break;
  }
  PLIS_CU(cudaEventRecord(ev1_, stream_));
  PLIS_CU(cudaEventSynchronize(ev1_));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0_, ev1_);
  device_ms_ += ms;
  for (uint32_t r = 0; r < nrep_; ++r)
    if (h_ctrl_[r].status != PLIS_OK) {
      err_ = "replica " + std::to_string(r) + ": too many consecutive rollbacks in one step";
      return h_ctrl_[r].status;
    }
  return PLIS_OK;
}

int BatchEngine::get_state(uint32_t r, uint32_t* counts) {
  if (r >= nrep_) { err_ = "replica index out of range"; return PLIS_ERR_INVALID; }
  int rc = init_pending();
  if (rc) return rc;
  rc = read_ctrls();
  if (rc) return rc;
  const uint32_t n = dims_[3 * r] * dims_[3 * r + 1] * dims_[3 * r + 2];
  PLIS_CU(cudaMemcpy2DAsync(counts, (size_t)n * 4, d_X_[h_ctrl_[r].cur] + coff_[r], ntot_ * 4, (size_t)n * 4, S_,
                            cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int BatchEngine::get_taus(uint32_t r, double* tau, uint8_t* flags) {
  if (r >= nrep_) { err_ = "replica index out of range"; return PLIS_ERR_INVALID; }
  int rc = init_pending();
  if (rc) return rc;
  rc = read_ctrls();
  if (rc) return rc;
  const uint32_t n = dims_[3 * r] * dims_[3 * r + 1] * dims_[3 * r + 2];
  const uint32_t tf = h_ctrl_[r].tf;
  if (tau) PLIS_CU(cudaMemcpyAsync(tau, d_tau_[tf] + coff_[r], (size_t)n * 8, cudaMemcpyDeviceToHost, stream_));
  if (flags) PLIS_CU(cudaMemcpyAsync(flags, d_flag_[tf] + coff_[r], n, cudaMemcpyDeviceToHost, stream_));
  PLIS_CU(cudaStreamSynchronize(stream_));
  return PLIS_OK;
}

int BatchEngine::stats(uint32_t r, plis_stats* st) {
  if (r >= nrep_) { err_ = "replica index out of range"; return PLIS_ERR_INVALID; }
  int rc = init_pending();
  if (rc) return rc;
  rc = read_ctrls();
  if (rc) return rc;
  const Ctrl& k = h_ctrl_[r];
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

int BatchEngine::tuning(plis_batch_tuning* out) {
  out->tile[0] = (int32_t)tile_[0];
  out->tile[1] = (int32_t)tile_[1];
  out->tile[2] = (int32_t)tile_[2];
  out->blocks_per_sm = blocks_per_sm_;
  out->grid = grid_;
  out->events_per_s = tuned_rate_;
  return PLIS_OK;
}

// Brick-shape autotuner: every candidate runs the same pilot steps from the same state.
int BatchEngine::autotune(uint64_t pilot_steps, plis_batch_tuning* out) {
  for (uint32_t r = 0; r < nrep_; ++r)
    if (pending_[r] == 2) { err_ = "replica " + std::to_string(r) + " has no state"; return PLIS_ERR_INVALID; }
  int rc = init_pending();
  if (rc) return rc;
  const size_t cells = (size_t)S_ * ntot_;
  std::vector<void*> saved;
  auto save = [&](const void* src, size_t bytes) -> int {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) { err_ = "autotune snapshot: out of device memory"; return PLIS_ERR_OOM; }
    cudaMemcpy(p, src, bytes, cudaMemcpyDeviceToDevice);
    saved.push_back(p);
    return PLIS_OK;
  };
  const void* srcs[] = {d_X_[0], d_X_[1], d_X_[2], d_tau_[0], d_tau_[1], d_flag_[0], d_flag_[1], d_D_, d_ctrl_};
  const size_t sizes[] = {cells * 4, cells * 4, cells * 4, ntot_ * 8, ntot_ * 8, ntot_, ntot_, cells * 4,
                          nrep_ * sizeof(Ctrl)};
  for (int i = 0; i < 9 && rc == PLIS_OK; ++i) rc = save(srcs[i], sizes[i]);
  auto restore = [&]() {
    for (int i = 0; i < 9; ++i) cudaMemcpy((void*)srcs[i], saved[i], sizes[i], cudaMemcpyDeviceToDevice);
  };
  const int cands[][3] = {{8, 8, 4}, {16, 4, 4}, {8, 4, 8}, {16, 8, 2}, {32, 4, 2}, {32, 8, 1}, {8, 8, 2}, {4, 8, 8}};
  double best = -1.0;
  int best_i = -1;
  const double ms0 = device_ms_;
  for (int i = 0; i < 8 && rc == PLIS_OK; ++i) {
    rc = layout(cands[i]);
    if (rc) break;
    restore();
    std::vector<Ctrl> before(nrep_);
    cudaMemcpy(before.data(), d_ctrl_, nrep_ * sizeof(Ctrl), cudaMemcpyDeviceToHost);
    const double m0 = device_ms_;
    rc = run(__builtin_inf(), pilot_steps);
    if (rc) break;
    double ev = 0.0;
    for (uint32_t r = 0; r < nrep_; ++r) ev += (double)(h_ctrl_[r].events - before[r].events);
    const double rate = ev / ((device_ms_ - m0) * 1e-3);
    if (rate > best) { best = rate; best_i = i; }
  }
  if (rc == PLIS_OK && best_i >= 0) {
    rc = layout(cands[best_i]);
    tuned_rate_ = best;
  }
  restore();
  device_ms_ = ms0;
  for (void* p : saved) cudaFree(p);
  if (rc == PLIS_OK) rc = read_ctrls();
  if (rc == PLIS_OK && out) rc = tuning(out);
  return rc;
}

}  // namespace plis

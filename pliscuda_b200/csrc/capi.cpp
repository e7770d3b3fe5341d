// capi.cpp — the C ABI of libplis.so (include/plis.h).  No exception crosses this boundary.
#include <cstring>
#include <new>
#include <string>

#include "../../include/plis.h"
#include "batch.h"
#include "engine.h"
#include "learned.h"
#include "plis_model.h"

namespace {
thread_local std::string g_err;
}

namespace plis {
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace plis

struct plis_handle {
  plis::Engine eng;
};

struct plis_batch {
  plis::BatchEngine eng;
};

struct plis_learner {
  plis::Learner l;
};

#define PLIS_GUARD_BEGIN try {
#define PLIS_GUARD_END                                  \
  }                                                     \
  catch (const std::bad_alloc&) {                       \
    g_err = "out of host memory";                       \
    return PLIS_ERR_OOM;                                \
  }                                                     \
  catch (const std::exception& e) {                     \
    g_err = e.what();                                   \
    return PLIS_ERR_INVALID;                            \
  }                                                     \
  catch (...) {                                         \
    g_err = "unknown failure";                          \
    return PLIS_ERR_INVALID;                            \
  }

static int fail(plis_handle* h, int rc) {
  if (rc != PLIS_OK) g_err = h->eng.error();
  return rc;
}

extern "C" {

int plis_abi_version(void) { return PLIS_ABI_VERSION; }

const char* plis_last_error(void) { return g_err.c_str(); }

const char* plis_status_string(int s) {
  switch (s) {
    case PLIS_OK: return "ok";
    case PLIS_ERR_INVALID: return "invalid argument";
    case PLIS_ERR_PARSE: return "parse error";
    case PLIS_ERR_IO: return "i/o error";
    case PLIS_ERR_OOM: return "out of memory";
    case PLIS_ERR_CUDA: return "CUDA error";
    case PLIS_ERR_TIMEOUT: return "device wait timed out";
    case PLIS_ERR_STUCK: return "too many rollbacks";
    case PLIS_ERR_OVERFLOW: return "count overflow";
    case PLIS_ERR_LIMIT: return "model exceeds a compiled limit";
    case PLIS_ERR_NO_DEVICE: return "no CUDA device";
    case PLIS_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

void plis_options_init(plis_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->size = sizeof *o;
  o->mode = PLIS_MODE_REFERENCE;
  o->precision = PLIS_PREC_FP64;
  o->critical_threshold = 10;  // driver.cu:36
  o->epsilon = 0.05;           // driver.cu:37
  o->seed = 1;
  o->device = 0;
  o->max_rollbacks = 64;
  o->steps_per_launch = 0;
  o->persistent = -1;
  o->stage_halo = 0;
  o->learned_mlp = 0;
  o->pooled_draws = -1;
}

int plis_create(const plis_model_desc* model, const plis_options* opts, plis_handle** out) {
  PLIS_GUARD_BEGIN
  if (!model || !out) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  *out = nullptr;
  plis_options o;
  plis_options_init(&o);
  if (opts) {
    if (opts->size != sizeof(plis_options)) { g_err = "plis_options.size mismatch (call plis_options_init)"; return PLIS_ERR_INVALID; }
    o = *opts;
  }
  if (o.mode != PLIS_MODE_REFERENCE && o.mode != PLIS_MODE_CORRECTED) { g_err = "unknown mode"; return PLIS_ERR_INVALID; }
  if (o.precision != PLIS_PREC_FP64 && o.precision != PLIS_PREC_FP32) { g_err = "unknown precision"; return PLIS_ERR_INVALID; }
  if (o.critical_threshold < 0 || !(o.epsilon > 0.0) || o.max_rollbacks < 0 || o.max_rollbacks > 4000) {
    g_err = "critical_threshold, epsilon or max_rollbacks out of range";
    return PLIS_ERR_INVALID;
  }
  if (o.learned_mlp != PLIS_MLP_TCGEN05 && o.learned_mlp != PLIS_MLP_MMA_SYNC) { g_err = "unknown learned_mlp"; return PLIS_ERR_INVALID; }
  if (o.pooled_draws < -1 || o.pooled_draws > 1) { g_err = "pooled_draws must be -1, 0 or 1"; return PLIS_ERR_INVALID; }
  plis::Model m;
  std::string err;
  int rc = plis::build_model(model, &m, &err);
  if (rc) { g_err = err; return rc; }
  plis_handle* h = new plis_handle();
  rc = h->eng.create(m, o);
  if (rc) {
    g_err = h->eng.error();
    delete h;
    return rc;
  }
  *out = h;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_destroy(plis_handle* h) {
  PLIS_GUARD_BEGIN
  delete h;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_set_state(plis_handle* h, const uint32_t* counts) {
  PLIS_GUARD_BEGIN
  if (!h || !counts) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.set_state(counts));
  PLIS_GUARD_END
}

int plis_set_state_at(plis_handle* h, const uint32_t* counts, double time, uint64_t steps) {
  PLIS_GUARD_BEGIN
  if (!h || !counts) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  if (!(time >= 0.0) || time == __builtin_inf()) { g_err = "time must be finite and >= 0"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.set_state(counts, time, steps));
  PLIS_GUARD_END
}

int plis_slab_setup(plis_handle* h, uint32_t z0, uint32_t z1, uint32_t world, uint32_t rank) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.slab_setup(z0, z1, world, rank));
  PLIS_GUARD_END
}

int plis_slab_buffers_get(plis_handle* h, plis_slab_buffers* out) {
  PLIS_GUARD_BEGIN
  if (!h || !out) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.slab_buffers(out));
  PLIS_GUARD_END
}

int plis_slab_phase(plis_handle* h, int phase, double t_end, uint64_t n_steps) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.slab_phase(phase, t_end, n_steps));
  PLIS_GUARD_END
}

int plis_get_state(plis_handle* h, uint32_t* counts) {
  PLIS_GUARD_BEGIN
  if (!h || !counts) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.get_state(counts));
  PLIS_GUARD_END
}

int plis_set_time(plis_handle* h, double t) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.set_time(t));
  PLIS_GUARD_END
}

int plis_run(plis_handle* h, double t_end) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.advance(t_end, ~0ull));
  PLIS_GUARD_END
}

int plis_step(plis_handle* h, uint64_t n) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.advance(__builtin_inf(), n));
  PLIS_GUARD_END
}

int plis_get_stats(plis_handle* h, plis_stats* st) {
  PLIS_GUARD_BEGIN
  if (!h || !st) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.stats(st));
  PLIS_GUARD_END
}

int plis_get_profile(plis_handle* h, plis_profile* p) {
  PLIS_GUARD_BEGIN
  if (!h || !p) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.profile(p));
  PLIS_GUARD_END
}

int plis_get_taus(plis_handle* h, double* tau, uint8_t* flags) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.get_taus(tau, flags));
  PLIS_GUARD_END
}

int plis_set_event_log(plis_handle* h, uint64_t capacity) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.set_event_log(capacity));
  PLIS_GUARD_END
}

int plis_read_event_log(plis_handle* h, plis_event_record* out, uint64_t max_records, uint64_t* n_records,
                        uint64_t* n_dropped, int clear) {
  PLIS_GUARD_BEGIN
  if (!h || !n_records || !n_dropped) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.read_event_log(out, max_records, n_records, n_dropped, clear != 0));
  PLIS_GUARD_END
}

// ---------------------------------------------------------------------------------------------- learned tau
static int lfail(plis_learner* L, int rc) {
  if (rc != PLIS_OK) g_err = L->l.error();
  return rc;
}

void plis_train_params_init(plis_train_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->iterations = 2000;
  p->batch = 16384;
  p->learning_rate = 1e-3f;
  p->quantile = 0.25f;
  p->seed = 1;
}

int plis_learner_create(uint64_t capacity, int device, plis_learner** out) {
  PLIS_GUARD_BEGIN
  if (!out) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  *out = nullptr;
  if (capacity == 0 || capacity > (1ull << 31)) { g_err = "capacity must be in 1..2^31 records"; return PLIS_ERR_INVALID; }
  plis_learner* L = new plis_learner();
  int rc = L->l.create(capacity, device);
  if (rc) {
    g_err = L->l.error();
    delete L;
    return rc;
  }
  *out = L;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_learner_destroy(plis_learner* L) {
  PLIS_GUARD_BEGIN
  delete L;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_learner_record(plis_learner* L, plis_handle* h, uint64_t n_steps, uint32_t stride, double label_epsilon) {
  PLIS_GUARD_BEGIN
  if (!L || !h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.record(h->eng, n_steps, stride, label_epsilon));
  PLIS_GUARD_END
}

int plis_learner_count(const plis_learner* L, uint64_t* n) {
  PLIS_GUARD_BEGIN
  if (!L || !n) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return L->l.count(n);
  PLIS_GUARD_END
}

int plis_learner_get_records(plis_learner* L, uint64_t first, uint64_t n, plis_trace_record* out) {
  PLIS_GUARD_BEGIN
  if (!L || (!out && n)) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.get_records(first, n, out));
  PLIS_GUARD_END
}

int plis_learner_set_records(plis_learner* L, const plis_trace_record* recs, uint64_t n) {
  PLIS_GUARD_BEGIN
  if (!L || (!recs && n)) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.set_records(recs, n));
  PLIS_GUARD_END
}

int plis_learner_train(plis_learner* L, const plis_train_params* p, plis_train_report* out) {
  PLIS_GUARD_BEGIN
  if (!L) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  plis_train_params q;
  plis_train_params_init(&q);
  if (p) q = *p;
  return lfail(L, L->l.train(q, out));
  PLIS_GUARD_END
}

int plis_learner_gradient(plis_learner* L, float quantile, float* grad, double* loss) {
  PLIS_GUARD_BEGIN
  if (!L || !grad) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.gradient(grad, loss, quantile));
  PLIS_GUARD_END
}

int plis_learner_predict(plis_learner* L, const float* features, uint64_t n, float* y, int mlp_kernel) {
  PLIS_GUARD_BEGIN
  if (!L || ((!features || !y) && n)) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  if (mlp_kernel != PLIS_MLP_TCGEN05 && mlp_kernel != PLIS_MLP_MMA_SYNC) { g_err = "unknown MLP kernel"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.predict(features, n, y, mlp_kernel));
  PLIS_GUARD_END
}

int plis_learner_get_weights(plis_learner* L, float* w) {
  PLIS_GUARD_BEGIN
  if (!L || !w) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.get_weights(w));
  PLIS_GUARD_END
}

int plis_learner_set_weights(plis_learner* L, const float* w) {
  PLIS_GUARD_BEGIN
  if (!L || !w) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return lfail(L, L->l.set_weights(w));
  PLIS_GUARD_END
}

int plis_set_proposer(plis_handle* h, const float* weights, double s_max) {
  PLIS_GUARD_BEGIN
  if (!h) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return fail(h, h->eng.set_proposer(weights, s_max));
  PLIS_GUARD_END
}

// ---------------------------------------------------------------------------------------------- batches
static int bfail(plis_batch* b, int rc) {
  if (rc != PLIS_OK) g_err = b->eng.error();
  return rc;
}

int plis_batch_create(const plis_batch_desc* desc, const plis_options* opts, plis_batch** out) {
  PLIS_GUARD_BEGIN
  if (!desc || !out) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  *out = nullptr;
  plis_options o;
  plis_options_init(&o);
  if (opts) {
    if (opts->size != sizeof(plis_options)) { g_err = "plis_options.size mismatch (call plis_options_init)"; return PLIS_ERR_INVALID; }
    o = *opts;
  }
  if (o.mode != PLIS_MODE_REFERENCE && o.mode != PLIS_MODE_CORRECTED) { g_err = "unknown mode"; return PLIS_ERR_INVALID; }
  if (o.precision != PLIS_PREC_FP64 && o.precision != PLIS_PREC_FP32) { g_err = "unknown precision"; return PLIS_ERR_INVALID; }
  if (o.pooled_draws < -1 || o.pooled_draws > 1) { g_err = "pooled_draws must be -1, 0 or 1"; return PLIS_ERR_INVALID; }
  if (o.critical_threshold < 0 || !(o.epsilon > 0.0) || o.max_rollbacks < 0 || o.max_rollbacks > 4000) {
    g_err = "critical_threshold, epsilon or max_rollbacks out of range";
    return PLIS_ERR_INVALID;
  }
  plis_batch* b = new plis_batch();
  int rc = b->eng.create(*desc, o);
  if (rc) {
    g_err = b->eng.error();
    delete b;
    return rc;
  }
  *out = b;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_batch_destroy(plis_batch* b) {
  PLIS_GUARD_BEGIN
  delete b;
  return PLIS_OK;
  PLIS_GUARD_END
}

int plis_batch_set_state(plis_batch* b, uint32_t replica, const uint32_t* counts) {
  PLIS_GUARD_BEGIN
  if (!b || !counts) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.set_state(replica, counts));
  PLIS_GUARD_END
}

int plis_batch_get_state(plis_batch* b, uint32_t replica, uint32_t* counts) {
  PLIS_GUARD_BEGIN
  if (!b || !counts) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.get_state(replica, counts));
  PLIS_GUARD_END
}

int plis_batch_get_taus(plis_batch* b, uint32_t replica, double* tau, uint8_t* flags) {
  PLIS_GUARD_BEGIN
  if (!b) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.get_taus(replica, tau, flags));
  PLIS_GUARD_END
}

int plis_batch_run(plis_batch* b, double t_end) {
  PLIS_GUARD_BEGIN
  if (!b) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.run(t_end, ~0ull));
  PLIS_GUARD_END
}

int plis_batch_step(plis_batch* b, uint64_t n) {
  PLIS_GUARD_BEGIN
  if (!b) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.run(__builtin_inf(), n));
  PLIS_GUARD_END
}

int plis_batch_get_stats(plis_batch* b, uint32_t replica, plis_stats* st) {
  PLIS_GUARD_BEGIN
  if (!b || !st) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.stats(replica, st));
  PLIS_GUARD_END
}

int plis_batch_autotune(plis_batch* b, uint64_t pilot_steps, plis_batch_tuning* out) {
  PLIS_GUARD_BEGIN
  if (!b) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.autotune(pilot_steps, out));
  PLIS_GUARD_END
}

int plis_batch_get_tuning(plis_batch* b, plis_batch_tuning* out) {
  PLIS_GUARD_BEGIN
  if (!b || !out) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.tuning(out));
  PLIS_GUARD_END
}

int plis_batch_set_proposer(plis_batch* b, const float* weights, double s_max) {
  PLIS_GUARD_BEGIN
  if (!b) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  return bfail(b, b->eng.set_proposer(weights, s_max));
  PLIS_GUARD_END
}

int plis_canonical_neighbours(uint32_t n, const uint32_t* table, const uint32_t lattice_in[3], uint32_t* canonical,
                              uint32_t lattice_out[3]) {
  PLIS_GUARD_BEGIN
  if (!canonical) { g_err = "null argument"; return PLIS_ERR_INVALID; }
  plis::Topology t;
  std::string err;
  int rc = plis::canonicalize(n, table, lattice_in, &t, &err);
  if (rc) { g_err = err; return rc; }
  if (lattice_out) std::memcpy(lattice_out, t.lattice, sizeof t.lattice);
  if (!t.canon.empty()) {
    std::memcpy(canonical, t.canon.data(), t.canon.size() * sizeof(uint32_t));
  } else {
    uint32_t buf[6];
    for (uint32_t c = 0; c < n; ++c) {
      int k = plis::lattice_row(t.lattice, c, buf);
      for (int j = 0; j < 6; ++j) canonical[(size_t)c * 6 + j] = j < k ? buf[j] : c;
    }
  }
  return PLIS_OK;
  PLIS_GUARD_END
}

}  // extern "C"

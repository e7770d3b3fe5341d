// simulate.cpp — plis_run_simulation: the reference's whole run_simulation (driver.cu:12-408) over
// the handle API, and the reference's console output around it.
//
// The loop is the reference's: simulate until time >= end_time, and whenever at least log_freq of
// simulated time has passed since the last snapshot, write sim<unix time>_<time>.dat
// (driver.cu:362-375); after the loop write the final snapshot under the same naming
// (driver.cu:390-397) and print the final statistics (driver.cu:399-405).  Each run_to(target)
// call ends on the first accepted step at or past target (reference semantics), which is the step
// at which the reference's `(t - last_log_time) >= log_freq` test fires.
#include <chrono>
#include <cstdio>
#include <ctime>
#include <string>
#include <vector>

#include "../../include/plis.h"

namespace plis {
void set_error(const std::string& msg);
}

namespace {

// std::to_string(float) of the reference: "%f" of the value rounded to binary32.
std::string ref_time_string(double t) {
  char b[64];
  std::snprintf(b, sizeof b, "%f", (double)(float)t);
  return b;
}

int snapshot(plis_handle* h, std::vector<uint32_t>& buf, uint32_t n, uint32_t s, double t, long long ts,
             const char* out_dir) {
  int rc = plis_get_state(h, buf.data());
  if (rc) return rc;
  std::string name = "sim" + std::to_string(ts) + "_" + ref_time_string(t) + ".dat";
  if (out_dir && *out_dir) name = std::string(out_dir) + "/" + name;
  return plis_write_snapshot(name.c_str(), buf.data(), n, s, t);
}

// print_eltime (driver.cu:411-419)
void print_eltime(double secs) {
  int hrs = (int)(secs / 3600);
  int mts = (int)((secs - hrs * 3600) / 60);
  double scs = secs - (hrs * 3600 + mts * 60);
  std::printf("%dh %dm %5.2fs", hrs, mts, scs);
}

}  // namespace

extern "C" int plis_run_simulation(const plis_model_desc* model, const uint32_t* counts, double start_time,
                                   double end_time, double log_freq, const plis_options* opts, const char* out_dir,
                                   int verbose, plis_stats* out) {
  if (!model || !counts) {
    plis::set_error("null argument");
    return PLIS_ERR_INVALID;
  }
  plis_options o;
  plis_options_init(&o);
  if (opts) o = *opts;
  if (verbose) std::printf("\n-- Starting Simulation -- \n\n");
  plis_handle* h = nullptr;
  int rc = plis_create(model, &o, &h);
  if (rc) return rc;
  const uint32_t n = model->n_subvolumes, s = model->n_species;
  std::vector<uint32_t> buf((size_t)n * s);
  rc = plis_set_state(h, counts);
  if (rc == PLIS_OK && start_time != 0.0) rc = plis_set_time(h, start_time);
  if (rc) {
    plis_destroy(h);
    return rc;
  }
  if (verbose) std::printf("-- Begin Iterations -- \n\n");
  std::fflush(stdout);
  const long long tstamp = (long long)std::time(nullptr);
  const auto wall0 = std::chrono::steady_clock::now();
  plis_stats st = {};
  plis_get_stats(h, &st);
  while (st.time < end_time) {
    double target = (log_freq > 0) ? st.time + log_freq : end_time;
    if (target > end_time) target = end_time;
    rc = plis_run(h, target);
    if (rc) break;
    plis_get_stats(h, &st);
    if (st.stop_reason == PLIS_STOP_NO_EVENT) {  // driver.cu:269-272
      if (verbose) std::printf("\n -- WARNING: min(tau) = +Inf or < 0 - abort simulation --\n");
      break;
    }
    if (log_freq > 0 && st.time < end_time) {
      rc = snapshot(h, buf, n, s, st.time, tstamp, out_dir);
      if (rc) break;
    }
  }
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
  if (rc == PLIS_OK) {
    if (verbose) std::printf("\n-- Simulation Complete -- \n\n");
    rc = snapshot(h, buf, n, s, st.time, tstamp, out_dir);
  }
  if (rc == PLIS_OK && verbose) {
    std::printf("  final simulation time:  %gs\n", (double)(float)st.time);
    std::printf("  elapsed time:           ");
    print_eltime(el);
    std::printf("\n  simulation steps:       %llu\n", (unsigned long long)st.steps);
    std::printf("  steps/second:           %g\n", el > 0 ? (double)st.steps / el : 0.0);
    std::printf("  events:                 %llu\n\n", (unsigned long long)st.events);
  }
  if (out) *out = st;
  std::fflush(stdout);
  plis_destroy(h);
  return rc;
}

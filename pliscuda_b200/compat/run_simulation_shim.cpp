// run_simulation_shim.cpp — drop-in replacement for the reference's PLISCuda/src/driver.cu.
//
// Compiled inside the reference tree (it includes the reference's own Topology/State/Reactions
// headers) and linked against libplis.so, it provides the exact function the reference's main.cpp
// calls (PLISCuda/include/cuda/driver.cuh:32-33, called at PLISCuda/src/main.cpp:53-63), with the
// reference's behaviour: simulate until time >= endTime, write sim<timestamp>_<time>.dat snapshots
// every logFreq of simulated time (logFreq > 0) and at the end, print the final statistics, and
// exit(code) on a device error as gpuErrchk does (cpp_utils.hpp:97-105).  The step itself runs in
// libplis.so (reference semantics, binary64, seed from the environment variable PLIS_SEED, default
// from the clock as the reference's non-TEST build seeds from clock64(), init.cu:8).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <iostream>
#include <string>
#include <vector>

#include "Reactions.hpp"
#include "State.hpp"
#include "Topology.hpp"
#include "plis.h"

namespace {

void die(int rc, const char* what) {
  std::fprintf(stderr, "GPUassert: %s (%s) %s\n", plis_last_error(), plis_status_string(rc), what);
  std::exit(rc);
}

void snapshot(plis_handle* h, std::vector<uint32_t>& buf, unsigned n, int s, double t, std::time_t ts) {
  int rc = plis_get_state(h, buf.data());
  if (rc) die(rc, "plis_get_state");
  std::string name = "sim" + std::to_string(ts) + "_" + std::to_string((float)t) + ".dat";
  rc = plis_write_snapshot(name.c_str(), buf.data(), n, (uint32_t)s, t);
  if (rc) die(rc, "plis_write_snapshot");
}

}  // namespace

namespace PLISCuda {

void run_simulation(Topology t, State s, Reactions r, float* h_rrc, float* h_drc, float endTime,
                    int compartments_count, int* subv_constants, float log_freq) {
  const unsigned n = t.getN();
  const int spc = s.getS(), rc_ = r.getR();
  std::vector<double> rrc((size_t)rc_ * compartments_count), drc((size_t)spc * compartments_count);
  for (size_t i = 0; i < rrc.size(); ++i) rrc[i] = h_rrc[i];
  for (size_t i = 0; i < drc.size(); ++i) drc[i] = h_drc[i];

  plis_model_desc d = {};
  d.n_subvolumes = n;
  d.n_species = (uint32_t)spc;
  d.n_reactions = (uint32_t)rc_;
  d.n_compartments = (uint32_t)compartments_count;
  d.neighbours = t.getNeighboursArray();
  d.reactants = r.getReactants();
  d.products = r.getProducts();
  d.reaction_rates = rrc.data();
  d.diffusion_rates = drc.data();
  d.compartment = compartments_count > 1 ? subv_constants : nullptr;

  plis_options o;
  plis_options_init(&o);
  const char* seed = std::getenv("PLIS_SEED");
  o.seed = seed ? std::strtoull(seed, nullptr, 10)
                : (uint64_t)std::chrono::high_resolution_clock::now().time_since_epoch().count();

  std::cout << "\n-- Starting Simulation -- \n\n";
  plis_handle* h = nullptr;
  int rc = plis_create(&d, &o, &h);
  if (rc) die(rc, "plis_create");
  std::vector<uint32_t> buf((size_t)n * spc);
  for (size_t i = 0; i < buf.size(); ++i) buf[i] = (uint32_t)s.getState()[i];
  rc = plis_set_state(h, buf.data());
  if (rc) die(rc, "plis_set_state");

  std::cout << "-- Begin Iterations -- \n\n";
  const std::time_t tstamp = std::time(0);
  const auto wall0 = std::chrono::steady_clock::now();
  plis_stats st = {};
  double target = (log_freq > 0) ? (double)log_freq : (double)endTime;
  while (true) {
    if (target > endTime) target = endTime;
    rc = plis_run(h, target);
    if (rc) die(rc, "plis_run");
    plis_get_stats(h, &st);
    if (st.stop_reason == PLIS_STOP_NO_EVENT) {
      std::printf("\n -- WARNING: min(tau) = +Inf or < 0 - abort simulation --\n");
      break;
    }
    if (st.time >= endTime) break;
    snapshot(h, buf, n, spc, st.time, tstamp);  // driver.cu:362-375
    target = st.time + log_freq;
  }
  const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
  std::cout << "\n-- Simulation Complete -- \n\n";
  snapshot(h, buf, n, spc, st.time, tstamp);  // driver.cu:390-397
  std::cout << "  final simulation time:  " << (float)st.time << "s\n";
  std::printf("  elapsed time:           %.2fs\n", el);
  std::cout << "  simulation steps:       " << st.steps << "\n";
  std::cout << "  steps/second:           " << (el > 0 ? st.steps / el : 0.0) << "\n";
  std::cout << "  events:                 " << st.events << "\n\n";
  plis_destroy(h);
}

}  // namespace PLISCuda

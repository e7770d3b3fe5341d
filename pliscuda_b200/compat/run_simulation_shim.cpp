// run_simulation_shim.cpp — drop-in replacement for the reference's PLISCuda/src/driver.cu.
//
// Compiled inside the reference tree (it includes the reference's own Topology/State/Reactions
// headers) and linked against libplis.so, it provides the exact function the reference's main.cpp
// calls (PLISCuda/include/cuda/driver.cuh:32-33, called at PLISCuda/src/main.cpp:53-63), with the
// reference's behaviour: simulate until time >= endTime, write sim<timestamp>_<time>.dat snapshots
// every logFreq of simulated time (logFreq > 0) and at the end, print the final statistics, and
// exit(code) on a device error as gpuErrchk does (cpp_utils.hpp:97-105).  The loop, the snapshots
// and the console lines are plis_run_simulation's; the step runs in libplis.so (reference
// semantics, binary64, seed from the environment variable PLIS_SEED, default from the clock as the
// reference's non-TEST build seeds from clock64(), init.cu:8).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "Reactions.hpp"
#include "State.hpp"
#include "Topology.hpp"
#include "plis.h"

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
  std::vector<uint32_t> buf((size_t)n * spc);
  for (size_t i = 0; i < buf.size(); ++i) buf[i] = (uint32_t)s.getState()[i];
  std::cout.flush();
  int rc = plis_run_simulation(&d, buf.data(), 0.0, endTime, log_freq, &o, nullptr, 1, nullptr);
  if (rc) {  // gpuErrchk prints and exits (cpp_utils.hpp:97-105)
    std::fprintf(stderr, "GPUassert: %s (%s)\n", plis_last_error(), plis_status_string(rc));
    std::exit(rc);
  }
}

}  // namespace PLISCuda

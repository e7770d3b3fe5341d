// cli.cpp — `pliscuda <configuration file>`: the reference's command line (PLISCuda/src/main.cpp)
// over libplis.so.
//
// Same console output, same input files read unchanged (plis_config_load), same sim*.dat snapshots
// in the working directory, same exit codes (1 for usage, no device, unreadable configuration;
// parse errors are printed and exit 0, as main.cpp:65-68 catches them and falls off the end).
// The step runs in libplis.so.  Beyond the reference: options
//   --mode reference|corrected   (default reference)
//   --precision fp64|fp32        (default fp64)
//   --seed N                     (default: PLIS_SEED from the environment, else the clock, as the
//                                 reference's non-TEST build seeds from clock64(), init.cu:8)
//   --resume sim<ts>_<t>.dat     start from a snapshot's counts and time instead of initialState
// and a CUDA error exits with the library's status code, as gpuErrchk exits (cpp_utils.hpp:97-105).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include "plis.h"

namespace {

int usage() {
  std::cout << "Usage: ./pliscuda <configuration file>\n";
  return 1;
}

}  // namespace

int main(int argc, char* argv[]) {
  const char* conf = nullptr;
  const char* resume = nullptr;
  plis_options o;
  plis_options_init(&o);
  const char* env_seed = std::getenv("PLIS_SEED");
  o.seed = env_seed ? std::strtoull(env_seed, nullptr, 10)
                    : (uint64_t)std::chrono::high_resolution_clock::now().time_since_epoch().count();
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if ((a == "--mode" || a == "--precision" || a == "--seed" || a == "--resume") && i + 1 < argc) {
      std::string v = argv[++i];
      if (a == "--resume") {
        resume = argv[i];
      } else if (a == "--mode") {
        if (v == "reference") o.mode = PLIS_MODE_REFERENCE;
        else if (v == "corrected") o.mode = PLIS_MODE_CORRECTED;
        else return usage();
      } else if (a == "--precision") {
        if (v == "fp64") o.precision = PLIS_PREC_FP64;
        else if (v == "fp32") o.precision = PLIS_PREC_FP32;
        else return usage();
      } else {
        o.seed = std::strtoull(v.c_str(), nullptr, 10);
      }
    } else if (!conf && a.rfind("--", 0) != 0) {
      conf = argv[i];
    } else {
      return usage();
    }
  }
  if (!conf) return usage();

  std::cout << "\n    **   PLISCuda  **    \n\n";
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0 || nd > 99) {  // main.cpp:19-24
    std::cout << "No CUDA-capable device detected.\n";
    return 1;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, 0);
  std::cout << "-- CUDA-capable device detected -- \n\n";
  std::cout << "  Device name: " << prop.name << "\n";
  std::cout << "  Total global memory: " << prop.totalGlobalMem / (1024 * 1024) << " MB\n";
  std::cout << "  Total shared memory per block: " << prop.sharedMemPerBlock / 1024 << " KB\n";
  std::cout << "  Total registers per block: " << prop.regsPerBlock << "\n";
  std::cout << "  Number of multiprocessors: " << prop.multiProcessorCount << "\n\n";

  std::cout << "-- Parsing input files -- \n\n";
  {
    std::ifstream cf(conf);
    if (!cf.good()) {
      std::cout << "Couldn't load configuration file\n";
      return 1;
    }
  }
  std::cout << "  processing configuration file...\n";
  plis_config* cfg = nullptr;
  int rc = plis_config_load(conf, &cfg);
  if (rc == PLIS_ERR_PARSE || rc == PLIS_ERR_IO || rc == PLIS_ERR_INVALID) {
    std::cout << "  parsing of configuration file failed with msg:\n";
    std::cout << "\t" << plis_last_error() << "\n";
    return 0;
  }
  if (rc) {
    std::fprintf(stderr, "pliscuda: %s (%s)\n", plis_last_error(), plis_status_string(rc));
    return rc;
  }
  plis_config_view v;
  plis_config_view_get(cfg, &v);
  const uint32_t* counts = v.initial_state;
  uint32_t* snap = nullptr;
  double t0 = 0.0;
  if (resume) {
    uint32_t sn = 0, ss = 0;
    rc = plis_read_snapshot(resume, &sn, &ss, &t0, &snap);
    if (rc == PLIS_OK && (sn != v.model.n_subvolumes || ss != v.model.n_species)) {
      std::fprintf(stderr, "pliscuda: %s has %u subvolumes x %u species, the configuration %u x %u\n", resume, sn, ss,
                   v.model.n_subvolumes, v.model.n_species);
      plis_free(snap);
      plis_config_free(cfg);
      return PLIS_ERR_INVALID;
    }
    if (rc) {
      std::fprintf(stderr, "pliscuda: %s (%s)\n", plis_last_error(), plis_status_string(rc));
      plis_config_free(cfg);
      return rc;
    }
    counts = snap;
  }
  std::cout.flush();
  rc = plis_run_simulation(&v.model, counts, t0, v.end_time, v.log_freq, &o, nullptr, 1, nullptr);
  if (snap) plis_free(snap);
  plis_config_free(cfg);
  if (rc) {
    std::fprintf(stderr, "GPUassert: %s (%s)\n", plis_last_error(), plis_status_string(rc));
    return rc;
  }
  return 0;
}

// refdump.cpp — TEST INFRASTRUCTURE.  Runs the reference's own input parsers
// (PLISCuda/include/cpp/Configuration.hpp and the headers it includes, compiled from the reference
// tree by oracle/ref_build.py) on a conf.txt and prints what they produced, so the loader in
// pliscuda_b200/csrc/loader.cpp can be checked against them and golden fixtures can be generated.
// Output: one "key: v v v ..." line per array.  Run it from the conf file's directory, as the
// reference opens the files named in conf.txt relative to the working directory.
#include <fstream>
#include <iostream>

#include "Configuration.hpp"

template <typename T>
static void dump(const char* key, const T* a, size_t n) {
  std::cout << key << ":";
  for (size_t i = 0; i < n; ++i) std::cout << " " << a[i];
  std::cout << "\n";
}

int main(int argc, char** argv) {
  if (argc < 2) { std::cerr << "usage: refdump conf.txt\n"; return 2; }
  std::ifstream cf(argv[1]);
  if (!cf.good()) { std::cout << "error: Couldn't load configuration file\n"; return 1; }
  try {
    PLISCuda::Configuration conf(cf);
    auto& t = conf.getTopology();
    auto& s = conf.getState();
    auto& r = conf.getReactions();
    size_t N = t.getN(), S = s.getS(), R = r.getR(), C = conf.getCompartments();
    std::cout.precision(9);
    std::cout << "dims: " << N << " " << S << " " << R << " " << C << "\n";
    dump("neighbours", t.getNeighboursArray(), 6 * N);
    dump("state", s.getState(), S * N);
    dump("reactants", r.getReactants(), S * R);
    dump("products", r.getProducts(), S * R);
    dump("rrc", conf.getReactionsConstantsArray(), R * C);
    dump("drc", conf.getDiffusionConstantsArray(), S * C);
    dump("compartment", conf.getCompArray(), N);
    std::cout << "endTime: " << conf.getEndTime() << "\n";
    std::cout << "logFreq: " << conf.getLogFreq() << "\n";
  } catch (std::invalid_argument& e) {
    std::cout << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}

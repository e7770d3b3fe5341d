// plis_model.h — host-side preparation of a model for the device step.
//
// The reference spreads this across run_simulation's set-up (driver.cu:54-213), init_ncount /
// init_hors (init.cu:15-68) and the per-thread coefficient scans of every kernel
// (rates.cu:3-38, tau.cu:3-40).  Here it is done once on the host: the reaction matrix is turned
// into sparse per-reaction and per-species lists (a subvolume-step then touches only the non-zero
// stoichiometry instead of S*R coefficients), the Cao highest-order data is precomputed, and the
// topology is canonicalised (and recognised as an implicit lattice when it is one).
#ifndef PLIS_MODEL_H_
#define PLIS_MODEL_H_

#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/plis.h"

namespace plis {

// Compiled limits (the reference has MAXREACTIONS 64 unchecked, constants.cuh:9).
constexpr int kMaxSpecies = 256;
constexpr int kMaxReactions = 512;
constexpr int kMaxReactantSpecies = 3;  // distinct reactant species per reaction
constexpr int kMaxNet = 8;              // species changed per reaction
constexpr int kMaxOrder = 3;            // reaction order (Cao's g is tabulated up to 3)
constexpr int kMaxNetEntries = 4096;    // sum over species of reactions changing it

struct ReactionTables {
  // per reaction
  std::vector<uint8_t> n_reac, n_net, order;
  std::vector<uint16_t> reac_s;  // [R][kMaxReactantSpecies]
  std::vector<uint8_t> reac_m;   // [R][kMaxReactantSpecies]
  std::vector<int16_t> reac_nu;  // [R][kMaxReactantSpecies] net change of that reactant species
  std::vector<uint16_t> net_s;   // [R][kMaxNet]
  std::vector<int16_t> net_nu;   // [R][kMaxNet]
  std::vector<double> inv_denom; // [R]
  // per species
  std::vector<uint8_t> hor, hmult;         // Cao highest order and multiplicity
  std::vector<uint16_t> sp_off;            // [S+1] CSR over (reaction, nu) with nu != 0
  std::vector<uint16_t> sp_r;
  std::vector<int16_t> sp_nu;
  std::vector<uint16_t> sr_off;            // [S+1] CSR over reactions where the species is a reactant
  std::vector<uint16_t> sr_r;
};

struct Topology {
  uint32_t n = 0;
  uint32_t lattice[3] = {0, 0, 0};  // X, Y, Z when a reflective lattice
  std::vector<uint32_t> canon;      // [6N] canonical (always built for tables; empty for implicit lattices)
  std::vector<uint32_t> orig;       // [6N] as given (table input only)
  std::vector<uint8_t> ncount;      // [N]
  bool is_lattice() const { return lattice[0] != 0; }
};

struct Model {
  uint32_t N = 0, S = 0, R = 0, C = 1;
  Topology topo;
  std::vector<int32_t> reactants, products;  // [S*R]
  std::vector<double> rrate, drate;          // [C*R], [C*S]
  std::vector<int32_t> comp;                 // [N] or empty
  ReactionTables rt;
};

// Returns PLIS_OK or an error code with a message in *err.
int build_model(const plis_model_desc* d, Model* m, std::string* err);

// Lattice helpers.  canonical_row writes the canonical neighbours of cell c of an X*Y*Z reflective
// lattice (-x,+x,-y,+y,-z,+z, absent ones skipped) and returns their number.
int lattice_row(const uint32_t dims[3], uint32_t c, uint32_t out[6]);
int canonicalize(uint32_t n, const uint32_t* table, const uint32_t lattice_in[3], Topology* t,
                 std::string* err);

}  // namespace plis

#endif

// plis_model.cpp — validation, topology canonicalisation and reaction tables (host only).
#include "plis_model.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace plis {

int lattice_row(const uint32_t dims[3], uint32_t c, uint32_t out[6]) {
  const uint32_t X = dims[0], Y = dims[1], Z = dims[2];
  const uint32_t x = c % X, y = (c / X) % Y, z = c / (X * Y);
  int n = 0;
  if (x > 0) out[n++] = c - 1;
  if (x + 1 < X) out[n++] = c + 1;
  if (y > 0) out[n++] = c - X;
  if (y + 1 < Y) out[n++] = c + X;
  if (z > 0) out[n++] = c - X * Y;
  if (z + 1 < Z) out[n++] = c + X * Y;
  return n;
}

static void squeeze(uint32_t d[3]) {
  // move unit dimensions to the back: (1,Y,Z) and (X,1,Z) linearise like (Y,Z,1) and (X,Z,1)
  uint32_t v[3];
  int k = 0;
  for (int i = 0; i < 3; ++i)
    if (d[i] > 1) v[k++] = d[i];
  while (k < 3) v[k++] = 1;
  d[0] = v[0]; d[1] = v[1]; d[2] = v[2];
}

static std::vector<uint32_t> divisors(uint32_t n) {
  std::vector<uint32_t> lo, hi;
  for (uint64_t i = 1; i * i <= n; ++i)
    if (n % i == 0) {
      lo.push_back((uint32_t)i);
      if (i * i != n) hi.push_back((uint32_t)(n / i));
    }
  lo.insert(lo.end(), hi.rbegin(), hi.rend());
  return lo;
}

static bool verify_lattice(uint32_t n, const std::vector<std::vector<uint32_t>>& rows, const uint32_t d[3]) {
  uint32_t buf[6];
  for (uint32_t c = 0; c < n; ++c) {
    int k = lattice_row(d, c, buf);
    if ((size_t)k != rows[c].size()) return false;
    std::sort(buf, buf + k);
    for (int i = 0; i < k; ++i)
      if (buf[i] != rows[c][i]) return false;
  }
  return true;
}

int canonicalize(uint32_t n, const uint32_t* table, const uint32_t lattice_in[3], Topology* t,
                 std::string* err) {
  t->n = n;
  t->lattice[0] = t->lattice[1] = t->lattice[2] = 0;
  t->canon.clear();
  t->orig.clear();
  t->ncount.assign(n, 0);
  if (n == 0) { *err = "Invalid: n < 1"; return PLIS_ERR_INVALID; }
  if (!table) {
    if (!lattice_in || (uint64_t)lattice_in[0] * lattice_in[1] * lattice_in[2] != n) {
      *err = "lattice dimensions do not multiply to the subvolume count";
      return PLIS_ERR_INVALID;
    }
    uint32_t d[3] = {lattice_in[0], lattice_in[1], lattice_in[2]};
    squeeze(d);
    std::memcpy(t->lattice, d, sizeof d);
    uint32_t buf[6];
    for (uint32_t c = 0; c < n; ++c) t->ncount[c] = (uint8_t)lattice_row(d, c, buf);
    return PLIS_OK;
  }
  t->orig.assign(table, table + (size_t)6 * n);
  std::vector<std::vector<uint32_t>> rows(n);
  for (uint32_t c = 0; c < n; ++c) {
    for (int j = 0; j < 6; ++j) {
      uint32_t b = table[(size_t)c * 6 + j];
      if (b >= n) { *err = "Invalid: sub >= n"; return PLIS_ERR_INVALID; }  // Topology.hpp:170-173
      if (b != c) rows[c].push_back(b);
    }
  }
  // canonical table for a general graph: non-self entries in file order, then self padding
  t->canon.assign((size_t)6 * n, 0);
  for (uint32_t c = 0; c < n; ++c) {
    size_t k = rows[c].size();
    for (size_t j = 0; j < 6; ++j) t->canon[(size_t)c * 6 + j] = j < k ? rows[c][j] : c;
    t->ncount[c] = (uint8_t)k;
  }
  // lattice recognition
  std::vector<std::vector<uint32_t>> sorted = rows;
  for (auto& r : sorted) std::sort(r.begin(), r.end());
  std::vector<uint32_t> dv = divisors(n);
  for (uint32_t X : dv) {
    uint32_t rest = n / X;
    for (uint32_t Y : dv) {
      if (rest % Y) continue;
      uint32_t d[3] = {X, Y, rest / Y};
      uint32_t buf[6];
      int k = lattice_row(d, 0, buf);
      std::sort(buf, buf + k);
      if ((size_t)k != sorted[0].size() || !std::equal(buf, buf + k, sorted[0].begin())) continue;
      k = lattice_row(d, n - 1, buf);
      std::sort(buf, buf + k);
      if ((size_t)k != sorted[n - 1].size() || !std::equal(buf, buf + k, sorted[n - 1].begin())) continue;
      if (!verify_lattice(n, sorted, d)) continue;
      squeeze(d);
      std::memcpy(t->lattice, d, sizeof d);
      for (uint32_t c = 0; c < n; ++c) {
        int m = lattice_row(d, c, buf);
        for (int j = 0; j < 6; ++j) t->canon[(size_t)c * 6 + j] = j < m ? buf[j] : c;
        t->ncount[c] = (uint8_t)m;
      }
      return PLIS_OK;
    }
  }
  return PLIS_OK;
}

int build_model(const plis_model_desc* d, Model* m, std::string* err) {
  if (!d) { *err = "null model"; return PLIS_ERR_INVALID; }
  if (d->n_subvolumes < 1) { *err = "Invalid: n < 1"; return PLIS_ERR_INVALID; }
  if (d->n_species < 1) { *err = "Invalid: s < 1"; return PLIS_ERR_INVALID; }
  if (d->n_reactions < 1) { *err = "Invalid: r < 1"; return PLIS_ERR_INVALID; }
  if (d->n_species > (uint32_t)kMaxSpecies) { *err = "too many species (limit 256)"; return PLIS_ERR_LIMIT; }
  if (d->n_reactions > (uint32_t)kMaxReactions) { *err = "too many reactions (limit 512)"; return PLIS_ERR_LIMIT; }
  if (!d->reactants || !d->products || !d->reaction_rates || !d->diffusion_rates) {
    *err = "missing reactants, products or rate arrays";
    return PLIS_ERR_INVALID;
  }
  m->N = d->n_subvolumes;
  m->S = d->n_species;
  m->R = d->n_reactions;
  m->C = d->n_compartments ? d->n_compartments : 1;
  const size_t N = m->N, S = m->S, R = m->R, C = m->C;
  m->reactants.assign(d->reactants, d->reactants + S * R);
  m->products.assign(d->products, d->products + S * R);
  m->rrate.assign(d->reaction_rates, d->reaction_rates + C * R);
  m->drate.assign(d->diffusion_rates, d->diffusion_rates + C * S);
  for (double v : m->rrate)
    if (!(v >= 0.0) || !std::isfinite(v)) { *err = "reaction rate constants must be finite and >= 0"; return PLIS_ERR_INVALID; }
  for (double v : m->drate)
    if (!(v >= 0.0) || !std::isfinite(v)) { *err = "diffusion rate constants must be finite and >= 0"; return PLIS_ERR_INVALID; }
  if (d->compartment) {
    m->comp.assign(d->compartment, d->compartment + N);
    for (int32_t c : m->comp)
      if (c < 0 || (size_t)c >= C) { *err = "compartment index out of range"; return PLIS_ERR_INVALID; }
    if (C == 1) m->comp.clear();
  }
  const uint32_t dims[3] = {d->lattice_x, d->lattice_y, d->lattice_z};
  int rc = canonicalize(m->N, d->neighbours, d->neighbours ? nullptr : dims, &m->topo, err);
  if (rc != PLIS_OK) return rc;

  ReactionTables& t = m->rt;
  t.n_reac.assign(R, 0); t.n_net.assign(R, 0); t.order.assign(R, 0);
  t.reac_s.assign(R * kMaxReactantSpecies, 0); t.reac_m.assign(R * kMaxReactantSpecies, 0);
  t.reac_nu.assign(R * kMaxReactantSpecies, 0);
  t.net_s.assign(R * kMaxNet, 0); t.net_nu.assign(R * kMaxNet, 0);
  t.inv_denom.assign(R, 1.0);
  t.hor.assign(S, 0); t.hmult.assign(S, 0);
  std::vector<std::vector<std::pair<int, int>>> spl(S);
  std::vector<std::vector<int>> srl(S);
  for (size_t r = 0; r < R; ++r) {
    int nr = 0, nn = 0, order = 0;
    double denom = 1.0;
    for (size_t s = 0; s < S; ++s) {
      int rm = m->reactants[s * R + r], pm = m->products[s * R + r];
      if (rm < 0 || pm < 0) { *err = "negative stoichiometric coefficient"; return PLIS_ERR_INVALID; }
      if (pm > 32767) { *err = "product coefficient too large"; return PLIS_ERR_LIMIT; }
      if (rm > 0) {
        if (nr >= kMaxReactantSpecies) { *err = "reaction with more than 3 reactant species"; return PLIS_ERR_LIMIT; }
        t.reac_s[r * kMaxReactantSpecies + nr] = (uint16_t)s;
        t.reac_m[r * kMaxReactantSpecies + nr] = (uint8_t)std::min(rm, 255);
        t.reac_nu[r * kMaxReactantSpecies + nr] = (int16_t)(pm - rm);
        ++nr;
        order += rm;
        for (int j = 2; j <= rm && j <= 16; ++j) denom *= j;
        srl[s].push_back((int)r);
      }
      int nu = pm - rm;
      if (nu != 0) {
        if (nn >= kMaxNet) { *err = "reaction changing more than 8 species"; return PLIS_ERR_LIMIT; }
        t.net_s[r * kMaxNet + nn] = (uint16_t)s;
        t.net_nu[r * kMaxNet + nn] = (int16_t)nu;
        ++nn;
        spl[s].push_back({(int)r, nu});
      }
    }
    if (order > kMaxOrder) { *err = "reaction of order > 3"; return PLIS_ERR_LIMIT; }
    t.n_reac[r] = (uint8_t)nr;
    t.n_net[r] = (uint8_t)nn;
    t.order[r] = (uint8_t)order;
    t.inv_denom[r] = 1.0 / denom;
    for (int i = 0; i < nr; ++i) {
      int s = t.reac_s[r * kMaxReactantSpecies + i];
      int mult = t.reac_m[r * kMaxReactantSpecies + i];
      if (order > t.hor[s] || (order == t.hor[s] && mult > t.hmult[s])) {
        t.hor[s] = (uint8_t)order;
        t.hmult[s] = (uint8_t)mult;
      }
    }
  }
  size_t tot = 0, tot2 = 0;
  for (size_t s = 0; s < S; ++s) { tot += spl[s].size(); tot2 += srl[s].size(); }
  if (tot > (size_t)kMaxNetEntries || tot2 > (size_t)kMaxNetEntries) {
    *err = "stoichiometry too dense (limit 4096 non-zero entries)";
    return PLIS_ERR_LIMIT;
  }
  t.sp_off.assign(S + 1, 0); t.sr_off.assign(S + 1, 0);
  t.sp_r.clear(); t.sp_nu.clear(); t.sr_r.clear();
  for (size_t s = 0; s < S; ++s) {
    t.sp_off[s] = (uint16_t)t.sp_r.size();
    for (auto& e : spl[s]) { t.sp_r.push_back((uint16_t)e.first); t.sp_nu.push_back((int16_t)e.second); }
    t.sr_off[s] = (uint16_t)t.sr_r.size();
    for (int r : srl[s]) t.sr_r.push_back((uint16_t)r);
  }
  t.sp_off[S] = (uint16_t)t.sp_r.size();
  t.sr_off[S] = (uint16_t)t.sr_r.size();
  return PLIS_OK;
}

}  // namespace plis

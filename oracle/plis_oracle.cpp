// plis_oracle.cpp — TEST INFRASTRUCTURE: the host oracle of the PLISCuda simulation step.
//
// Plain loops over subvolumes, one phase at a time, in the order of the reference's step loop
// (PLISCuda/src/driver.cu:259-376).  Every floating-point expression is written in the order the
// CUDA step uses, so that with the same injected random stream the two produce the same integer
// trajectories bit for bit.  Nothing here is tiled, fused or clever: it is the checker.
//
// Two semantics modes (oracle_options.mode):
//   0  reference: the reference's own rules, including its deterministic quirks
//      (outgoing diffusion counted once in mu/sigma^2, tau.cu:115-116; incoming diffusion subtracted
//      and divided by the neighbour's count, tau.cu:120-136; the && species-skip test, tau.cu:165;
//      channel choice reusing the uniform, leap.cu:109-166 and ssa.cu:64-68; destination slot 1 of 6,
//      leap.cu:180-186; one critical event in every LEAP_CR subvolume, leap.cu:67-199; the receiver
//      flag written through the neighbour table, leap.cu:192-193; rollback re-leaping with the
//      un-halved tau, driver.cu:285-315).  The one race (leap.cu:131-134: the feasibility test reads
//      state.next while other threads add to it) is replaced by a read after all Poisson firings.
//   1  corrected: Cao's critical set and outflow n*d, inflow from non-critical neighbours, fresh
//      uniforms for each choice, destinations among real neighbours, exact events only where their
//      time is <= the step, rollback halving the leap, and the last step clamped onto t_end.
#include "plis_oracle.h"

#include "../pliscuda_b200/csrc/plis_stream.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#define PLIS_ORACLE_MAXR 1024

// Guards that keep every per-step sum inside 32 bits (the device accumulates counts as int32):
// an attempt that draws one reaction contribution |k*nu| >= 2^29, one diffusion jump k >= 2^27,
// or leaves a subvolume's own post-leap value |x + delta| >= 2^30 is rejected like a negative count.
static const int64_t kBigDraw = (int64_t)1 << 29;
static const int64_t kBigJump = (int64_t)1 << 27;
static const int64_t kBigTile = (int64_t)1 << 30;

namespace {

enum Flag : uint8_t { LEAP_CR = 0, LEAP_NOCR = 1, SSA = 2, SSA_FF = 3 };  // enum op, constants.cuh:53-58

template <typename Real> struct RealOps;
template <> struct RealOps<double> {
  static double poisson(plis_stream* s, double lam) { return plis_poisson_d(s, lam); }
  static double emlam(double lam) { return lam < PLIS_LEAP_INV_MAX ? plis_exp(-lam) : 0.0; }
  static double poisson_shared(plis_stream* s, double lam, double em) {
    if (!(lam > 0.0)) return 0.0;
    return lam < PLIS_LEAP_INV_MAX ? plis_poisson_small_d(s, lam, em) : plis_poisson_d(s, lam);
  }
  static int64_t count(double k) { return (int64_t)plis_count_d(k); }
  // inversion draw i of a group of n from the group's shared Philox blocks (plis_group_uniforms_d)
  static double inv_group(const plis_stream* g, uint32_t i, int n, double lam, double em) {
    double u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    plis_group_uniforms_d(g, 1u << i, u, n);
    return plis_poisson_inv_d(u[i], lam, em);
  }
  static double uniform(plis_stream* s) { return plis_uniform_d(s); }
  static double word_uniform(uint32_t w) { return plis_u32_to_uniform_d(w); }
  static double inv_word(uint32_t w, double lam) { return plis_poisson_inv_d(plis_u32_to_uniform_d(w), lam, plis_exp(-lam)); }
  static double inf() { return PLIS_INF_D; }
  static double fabs_(double x) { return fabs(x); }
};
template <> struct RealOps<float> {
  static double poisson(plis_stream* s, float lam) { return plis_poisson_f(s, lam); }
  static float emlam(float lam) { return lam < (float)PLIS_LEAP_INV_MAX ? plis_expf(-lam) : 0.0f; }
  static double poisson_shared(plis_stream* s, float lam, float em) {
    if (!(lam > 0.0f)) return 0.0;
    return lam < (float)PLIS_LEAP_INV_MAX ? plis_poisson_small_f(s, lam, em) : plis_poisson_d(s, (double)lam);
  }
  static int64_t count(double k) { return (int64_t)plis_count_d(k); }
  static double inv_group(const plis_stream* g, uint32_t i, int n, float lam, float em) {
    float u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    plis_group_uniforms_f(g, 1u << i, u, n);
    return plis_poisson_inv_f(u[i], lam, em);
  }
  static float uniform(plis_stream* s) { return plis_uniform_f(s); }
  static float word_uniform(uint32_t w) { return plis_u32_to_uniform_f(w); }
  static double inv_word(uint32_t w, float lam) { return plis_poisson_inv_f(plis_u32_to_uniform_f(w), lam, plis_expf(-lam)); }
  static float inf() { return PLIS_INF_F; }
  static float fabs_(float x) { return fabsf(x); }
};

struct Reaction {
  std::vector<std::pair<int, int>> reac;  // (species, coefficient > 0), increasing species
  std::vector<std::pair<int, int>> net;   // (species, p - r != 0), increasing species
  int order = 0;
  double inv_denom = 1.0;                 // 1 / prod(coefficient!)
};

struct Base {
  uint32_t N, S, R, C;
  std::vector<uint32_t> nbr, orig;
  std::vector<uint8_t> ncount;
  std::vector<int32_t> reactants, products, comp;
  std::vector<double> rrate, drate;
  std::vector<Reaction> rx;
  std::vector<std::vector<std::pair<int, int>>> sp_nu;  // per species: (reaction, nu) with nu != 0
  std::vector<int> hor, hmult;                           // highest order / multiplicity, init.cu:27-68
  std::vector<std::vector<std::pair<uint32_t, int>>> in_edges;  // per cell: (source cell, source slot)
  oracle_options opt;
  virtual ~Base() {}
  virtual int set_state(const uint32_t*, double t0, uint64_t step0) = 0;
  virtual int get_state(uint32_t*) = 0;
  virtual int get_taus(double*, uint8_t*) = 0;
  virtual int advance(double, uint64_t) = 0;
  oracle_stats st{};
  bool logging = false;
  std::vector<oracle_event> log;
  void note(uint64_t step, uint32_t attempt, uint32_t c, uint32_t target, int64_t count, uint32_t channel, int kind) {
    if (!logging) return;
    log.push_back(event(st.time, step, attempt, c, target, count, channel, kind));
  }
  static oracle_event event(double t, uint64_t step, uint32_t attempt, uint32_t c, uint32_t target, int64_t count,
                            uint32_t channel, int kind) {
    oracle_event e;
    e.time = t;
    e.step = step;
    e.subvolume = c;
    e.target = target;
    e.count = count > 0xFFFFFFFFll ? 0xFFFFFFFFu : (uint32_t)count;
    e.channel = (uint16_t)channel;
    e.kind = (uint8_t)kind;
    e.attempt = attempt > 255u ? (uint8_t)255 : (uint8_t)attempt;
    return e;
  }
};

template <typename Real>
struct Sim : Base {
  using Ops = RealOps<Real>;
  std::vector<int64_t> x;      // current counts [S][N]
  std::vector<int64_t> nx;     // next counts [S][N]
  std::vector<double> tau;     // per-subvolume tau (binary64 in both precisions)
  std::vector<uint8_t> flag;
  std::vector<Real> rr_c, dr_c;           // rates of the current state [R][N], [S][N]
  std::vector<int64_t> own;               // leap: own deltas [N][S]
  std::vector<int64_t> outk;              // leap: outgoing diffusion counts [N][S][6]
  std::vector<uint8_t> leaped;            // leap: this cell marks its receivers
  std::vector<int64_t> evc;               // leap: events per cell
  std::vector<uint8_t> bigc;              // leap: a draw too large for 32-bit accumulation
  std::vector<std::vector<oracle_event>> cell_log;  // leap: events per cell (event log on)
  uint8_t leap_big = 0;
  double ff_tau = 0.0;                    // fast-forward decrement (reference: min_tau, driver.cu:333)
  int64_t ff_argmin = -1;
  int ff_fired = 0;

  Real rate_r(uint32_t c, int r) const { return (Real)rrate[(size_t)compo(c) * R + r]; }
  Real rate_d(uint32_t c, int s) const { return (Real)drate[(size_t)compo(c) * S + s]; }
  int compo(uint32_t c) const { return comp.empty() ? 0 : comp[c]; }
  int64_t cnt(const std::vector<int64_t>& v, int s, uint32_t c) const { return v[(size_t)s * N + c]; }

  // propensity of reaction r in subvolume c: c_r * prod_s prod_{j<m_s} (x_s - j) / prod_s m_s!
  // (orders 0-3; the reference's uni / bi_same / bi_diff cases, rates.cu:3-38, are the special cases)
  Real propensity(const std::vector<int64_t>& v, uint32_t c, int r) const {
    const Reaction& q = rx[r];
    Real prod = (Real)1;
    for (auto& e : q.reac) {
      Real xs = (Real)cnt(v, e.first, c);
      for (int j = 0; j < e.second; ++j) prod = prod * (xs - (Real)j);
    }
    return (rate_r(c, r) * prod) * (Real)q.inv_denom;
  }

  // reference criticality, tau.cu:3-40: the first two reactant species decide
  bool crit_ref(const std::vector<int64_t>& v, uint32_t c, int r) const {
    const Reaction& q = rx[r];
    int nc = opt.critical_threshold;
    bool crit = false;
    int seen = 0;
    for (auto& e : q.reac) {
      if (seen >= 2) break;
      ++seen;
      int64_t xs = cnt(v, e.first, c);
      if (xs == 0) return true;
      int nu = products[(size_t)e.first * R + r] - reactants[(size_t)e.first * R + r];
      if (nu < 0 && (int64_t)(-nu) * nc > xs) crit = true;
    }
    return crit;
  }
  // corrected criticality (Cao et al. 2005): L_j = min_{nu_ij<0} floor(x_i/|nu_ij|) < NC, a_j > 0
  bool crit_fix(const std::vector<int64_t>& v, uint32_t c, int r, Real a) const {
    if (!(a > (Real)0)) return false;
    int nc = opt.critical_threshold;
    for (auto& e : rx[r].net) {
      if (e.second < 0 && cnt(v, e.first, c) < (int64_t)(-e.second) * nc) return true;
    }
    return false;
  }

  Real gfun(int s, int64_t x) const {
    Real xr = (Real)x;
    switch (hor[s]) {
      case 0: return Ops::inf();
      case 1: return (Real)1;
      case 2:
        if (hmult[s] == 1) return (Real)2;
        return (Real)2 + (Real)1 / (xr - (Real)1);
      default:
        if (hmult[s] == 1) return (Real)3;
        if (hmult[s] == 2) return (Real)1.5 * ((Real)2 + (Real)1 / (xr - (Real)1));
        return ((Real)3 + (Real)1 / (xr - (Real)1)) + (Real)2 / (xr - (Real)2);
    }
  }

  void init_tables() {
    rx.assign(R, Reaction());
    sp_nu.assign(S, {});
    hor.assign(S, 0);
    hmult.assign(S, 0);
    for (uint32_t r = 0; r < R; ++r) {
      Reaction& q = rx[r];
      double denom = 1.0;
      for (uint32_t s = 0; s < S; ++s) {
        int m = reactants[(size_t)s * R + r];
        int nu = products[(size_t)s * R + r] - m;
        if (m > 0) {
          q.reac.push_back({(int)s, m});
          q.order += m;
          for (int j = 2; j <= m; ++j) denom *= j;
        }
        if (nu != 0) {
          q.net.push_back({(int)s, nu});
          sp_nu[s].push_back({(int)r, nu});
        }
      }
      q.inv_denom = 1.0 / denom;
      for (auto& e : q.reac) {
        int s = e.first;
        if (q.order > hor[s] || (q.order == hor[s] && e.second > hmult[s])) {
          hor[s] = q.order;
          hmult[s] = e.second;
        }
      }
    }
    ncount.assign(N, 0);
    in_edges.assign(N, {});
    for (uint32_t c = 0; c < N; ++c) {
      int n = 0;
      for (int j = 0; j < 6; ++j) {
        uint32_t b = nbr[(size_t)c * 6 + j];
        if (b == c) break;
        ++n;
        in_edges[b].push_back({c, j});
      }
      ncount[c] = (uint8_t)n;
    }
  }

  void compute_rates_of(const std::vector<int64_t>& v) {
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)N; ++ci) {
      uint32_t c = (uint32_t)ci;
      for (uint32_t r = 0; r < R; ++r) rr_c[(size_t)r * N + c] = propensity(v, c, r);
      for (uint32_t s = 0; s < S; ++s) dr_c[(size_t)s * N + c] = rate_d(c, s) * (Real)cnt(v, s, c);
    }
  }

  // ---------------------------------------------------------------- classification (compute_taus)
  // tau.cu:197-252 for one subvolume; rates of the current state are in rr_c / dr_c.
  void classify(uint32_t c, uint64_t step, uint32_t attempt) {
    const int mode = opt.mode;
    const int nc = opt.critical_threshold;
    if (step > 0 && flag[c] == SSA_FF && !plis_isinf_d(tau[c])) {
      if (mode == 0) {
        if (ff_tau > 0.0 && ff_tau != tau[c]) { tau[c] = tau[c] - ff_tau; return; }  // tau.cu:214-217
      } else {
        if (tau[c] > ff_tau) { tau[c] = tau[c] - ff_tau; return; }
      }
    }
    bool crit[PLIS_ORACLE_MAXR];
    bool ncrit[PLIS_ORACLE_MAXR];
    for (uint32_t r = 0; r < R; ++r) {
      Real a = rr_c[(size_t)r * N + c];
      if (mode == 0) {
        crit[r] = crit_ref(x, c, r);
        ncrit[r] = !crit[r];
      } else {
        crit[r] = crit_fix(x, c, r, a);
        ncrit[r] = (a > (Real)0) && !crit[r];
      }
    }
    const int n = ncount[c];
    Real tau_ncr = Ops::inf();
    for (uint32_t s = 0; s < S; ++s) {
      int64_t xs = cnt(x, s, c);
      bool include;
      if (mode == 0) {
        bool skip_r = false;
        for (uint32_t r = 0; r < R; ++r)
          if (crit[r] && reactants[(size_t)s * R + r] > 0) skip_r = true;
        bool skip_d = xs < nc;
        include = !(skip_r && skip_d);  // tau.cu:165
      } else {
        include = false;
        for (uint32_t r = 0; r < R; ++r)
          if (ncrit[r] && reactants[(size_t)s * R + r] > 0) include = true;
        if (xs >= nc && rate_d(c, s) > (Real)0 && n > 0) include = true;
      }
      if (!include) continue;
      // compute_tau_sp, tau.cu:68-143
      Real g = gfun(s, xs);
      Real mu = (Real)0, s2 = (Real)0;
      for (auto& e : sp_nu[s]) {
        if (!ncrit[e.first]) continue;
        Real a = rr_c[(size_t)e.first * N + c];
        mu = mu + (Real)e.second * a;
        s2 = s2 + (Real)(e.second * e.second) * a;
      }
      Real d = dr_c[(size_t)s * N + c];
      if (mode == 0) {
        if (xs >= nc) { mu = mu + d; s2 = s2 + d; }
        for (int j = 0; j < n; ++j) {
          uint32_t b = nbr[(size_t)c * 6 + j];
          Real q = dr_c[(size_t)s * N + b] / (Real)ncount[b];
          mu = mu - q;
          s2 = s2 + q;
        }
      } else {
        if (xs >= nc && n > 0) {
          Real dout = (Real)n * d;
          mu = mu - dout;
          s2 = s2 + dout;
        }
        for (int j = 0; j < n; ++j) {
          uint32_t b = nbr[(size_t)c * 6 + j];
          if (cnt(x, s, b) >= nc) {
            Real q = dr_c[(size_t)s * N + b];
            mu = mu + q;
            s2 = s2 + q;
          }
        }
      }
      Real m = ((Real)opt.epsilon * (Real)xs) / g;
      if (!(m > (Real)1)) m = (Real)1;
      Real t1 = m / Ops::fabs_(mu);
      Real t2 = (m * m) / s2;
      Real ts = t1 < t2 ? t1 : t2;
      if (ts < tau_ncr) tau_ncr = ts;
    }
    // critical / exact rate (compute_tau_cr, tau.cu:176-195)
    Real rsum = (Real)0, dsum = (Real)0;
    if (mode == 0 || !plis_isinf_d((double)tau_ncr)) {
      for (uint32_t r = 0; r < R; ++r)
        if (crit[r]) rsum = rsum + rr_c[(size_t)r * N + c];
      for (uint32_t s = 0; s < S; ++s)
        if (cnt(x, s, c) < nc) {
          Real d = dr_c[(size_t)s * N + c];
          dsum = dsum + (mode == 0 ? d : (Real)n * d);
        }
    } else {  // corrected SSA subvolume: every channel
      for (uint32_t r = 0; r < R; ++r) rsum = rsum + rr_c[(size_t)r * N + c];
      for (uint32_t s = 0; s < S; ++s) dsum = dsum + (Real)n * dr_c[(size_t)s * N + c];
    }
    double tcr;
    if (rsum == (Real)0 && dsum == (Real)0) {
      tcr = PLIS_INF_D;
    } else {
      plis_stream stx = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_TAU, step, attempt, 0);
      tcr = plis_exponential_d(&stx, (double)(rsum + dsum));
    }
    double tn = (double)tau_ncr;
    if (plis_isinf_d(tn)) {
      flag[c] = SSA_FF;
      tau[c] = tcr;
    } else if (tn < tcr) {
      flag[c] = LEAP_NOCR;
      tau[c] = tn;
    } else {
      flag[c] = LEAP_CR;
      tau[c] = tcr;
    }
  }

  void classify_all(uint64_t step, uint32_t attempt) {
    compute_rates_of(x);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ci = 0; ci < (int64_t)N; ++ci) classify((uint32_t)ci, step, attempt);
  }

  int set_state(const uint32_t* counts, double t0, uint64_t step0) override {
    for (size_t i = 0; i < (size_t)S * N; ++i) {
      if (counts[i] >= (1u << 30)) return 8;
      x[i] = counts[i];
    }
    std::fill(flag.begin(), flag.end(), (uint8_t)SSA_FF);  // driver.cu:213
    std::fill(tau.begin(), tau.end(), PLIS_INF_D);
    st = oracle_stats{};
    st.time = t0;
    st.steps = step0;
    ff_tau = 0.0;
    classify_all(step0, 0);
    return 0;
  }
  int get_state(uint32_t* counts) override {
    for (size_t i = 0; i < (size_t)S * N; ++i) counts[i] = (uint32_t)x[i];
    return 0;
  }
  int get_taus(double* t, uint8_t* f) override {
    if (t) std::memcpy(t, tau.data(), sizeof(double) * N);
    if (f) std::memcpy(f, flag.data(), N);
    return 0;
  }

  // ---------------------------------------------------------------- leap (leap_step, leap.cu:3-65)
  int64_t leap_all(uint64_t step, uint32_t attempt, double tau_leap) {
    const int mode = opt.mode;
    const int nc = opt.critical_threshold;
    const Real tl = (Real)tau_leap;
    const bool pool_on = opt.pooled_draws < 0 ? (R > 4 || S > 4) : opt.pooled_draws != 0;
    std::fill(own.begin(), own.end(), 0);
    std::fill(outk.begin(), outk.end(), 0);
    std::fill(leaped.begin(), leaped.end(), 0);
    if (logging && cell_log.size() != N) cell_log.assign(N, {});
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t ci = 0; ci < (int64_t)N; ++ci) {
      uint32_t c = (uint32_t)ci;
      int64_t ev = 0;
      evc[c] = 0;
      bigc[c] = 0;
      if (logging) cell_log[c].clear();
      if (flag[c] == SSA || flag[c] == SSA_FF) continue;  // leap.cu:9-10
      uint8_t big = 0;
      // pooled draws (plis_stream.h): channels of mean below PLIS_POOL_CUT join the pool, in walking
      // order (reactions, then species), while its total stays at most PLIS_POOL_MAX
      Real pool = (Real)0;
      auto join = [](Real& acc, Real unit, Real w) {
        if (!(unit < (Real)PLIS_POOL_CUT) || !(acc + w <= (Real)PLIS_POOL_MAX)) return false;
        acc = acc + w;
        return true;
      };
      auto reaction_mean = [&](uint32_t r) {
        const Real a = rr_c[(size_t)r * N + c];
        const bool fire = (mode == 0) ? !crit_ref(x, c, r) : ((a > (Real)0) && !crit_fix(x, c, r, a));
        return fire ? tl * a : (Real)0;
      };
      const int n = ncount[c];
      for (uint32_t r = 0; r < R; ++r) {
        const Real lam = reaction_mean(r);
        if (!(lam > (Real)0)) continue;  // not leaped (critical), or a zero mean (a draw of 0)
        if (pool_on && join(pool, lam, lam)) continue;
        int64_t k;
        if (lam > (Real)0 && lam < (Real)PLIS_LEAP_INV_MAX) {  // inversion: uniform r % 4 of reaction group r / 4
          plis_stream g = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_rgroup(r >> 2));
          k = Ops::count(Ops::inv_group(&g, r & 3u, 4, lam, Ops::emlam(lam)));
        } else {
          plis_stream sr = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_react(r));
          k = Ops::count(Ops::poisson(&sr, lam));
        }
        ev += k;
        if (logging && k > 0) cell_log[c].push_back(event(st.time, step, attempt, c, c, k, r, 1));
        for (auto& e : rx[r].net) {
          int64_t v = k * e.second;
          if (v >= kBigDraw || v <= -kBigDraw) big = 1;
          own[(size_t)c * S + e.first] += v;
        }
      }
      uint8_t mark = 0;
      for (uint32_t s = 0; s < S; ++s) {
        if (cnt(x, s, c) < nc) continue;  // is_critical_diffusion, tau.cu:42-45
        if (mode == 0 && n > 0) mark = 1;  // leap.cu:54-56 marks every receiver
        Real lam = tl * dr_c[(size_t)s * N + c];
        if (pool_on && n > 0 && lam > (Real)0 && join(pool, lam, (Real)n * lam)) continue;
        Real em = Ops::emlam(lam);
        for (int j = 0; j < n; ++j) {
          int64_t k;
          if (lam > (Real)0 && lam < (Real)PLIS_LEAP_INV_MAX) {  // inversion: uniform j of the species' diffusion group
            plis_stream g = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_dgroup(s));
            k = Ops::count(Ops::inv_group(&g, (uint32_t)j, 6, lam, em));
          } else {
            plis_stream sd = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_LEAP, step, attempt, plis_ch_diff(s, j));
            k = Ops::count(Ops::poisson_shared(&sd, lam, em));
          }
          if (k >= kBigJump) big = 1;
          if (logging && k > 0)  // a jump of 2^27 or more (always rolled back) is logged as 2^27, as on the device
            cell_log[c].push_back(event(st.time, step, attempt, c, nbr[(size_t)c * 6 + j], k < kBigJump ? k : kBigJump, s, 2));
          outk[((size_t)c * S + s) * 6 + j] = k;
          own[(size_t)c * S + s] -= k;
          ev += k;
        }
      }
      if (pool > (Real)0) {  // the pool's total by inversion, then one walk per event
        const plis_stream g = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_LEAP, step, attempt, PLIS_CH_POOL);
        const int64_t K = Ops::count(Ops::inv_word(plis_group_block(&g, 0).x, pool));
        for (int64_t e = 0; e < K; ++e) {
          const plis_u32x4 w = plis_group_block(&g, (uint32_t)(e + 1));
          const Real target = Ops::word_uniform(w.x) * pool;
          Real acc = (Real)0;
          int pick_r = -1, pick_s = -1, last_r = -1, last_s = -1;
          for (uint32_t r = 0; r < R && pick_r < 0; ++r) {
            const Real lr = reaction_mean(r);
            if (lr > (Real)0 && join(acc, lr, lr)) {
              last_r = (int)r;
              if (target < acc) pick_r = (int)r;
            }
          }
          if (pick_r < 0) {
            for (uint32_t s = 0; s < S && pick_s < 0; ++s) {
              if (cnt(x, s, c) < nc || n == 0) continue;
              const Real ls = tl * dr_c[(size_t)s * N + c];
              if (ls > (Real)0 && join(acc, ls, (Real)n * ls)) {
                last_s = (int)s;
                if (target < acc) pick_s = (int)s;
              }
            }
            if (pick_s < 0) {  // rounding left the target at the total: the last member
              if (last_s >= 0) pick_s = last_s;
              else pick_r = last_r;
            }
          }
          ev += 1;
          if (pick_r >= 0) {
            if (logging) cell_log[c].push_back(event(st.time, step, attempt, c, c, 1, (uint32_t)pick_r, 1));
            for (auto& ne : rx[pick_r].net) own[(size_t)c * S + ne.first] += ne.second;
          } else {
            const uint32_t j = plis_pool_slot(w.y, (uint32_t)n);
            if (logging) cell_log[c].push_back(event(st.time, step, attempt, c, nbr[(size_t)c * 6 + j], 1, (uint32_t)pick_s, 2));
            outk[((size_t)c * S + pick_s) * 6 + j] += 1;
            own[(size_t)c * S + pick_s] -= 1;
          }
        }
      }
      for (uint32_t s = 0; s < S; ++s) {
        int64_t tv = cnt(x, s, c) + own[(size_t)c * S + s];
        if (tv >= kBigTile || tv <= -kBigTile) big = 1;
      }
      leaped[c] = mark;
      bigc[c] = big;
      evc[c] = ev;
    }
    leap_big = 0;
    for (uint32_t c = 0; c < N; ++c) leap_big |= bigc[c];
    int64_t events = 0;
    for (uint32_t c = 0; c < N; ++c) events += evc[c];
    if (logging)
      for (uint32_t c = 0; c < N; ++c) log.insert(log.end(), cell_log[c].begin(), cell_log[c].end());
    // gather: next = curr + own + inflow; receivers SSA_FF -> SSA
#pragma omp parallel for schedule(static)
    for (int64_t ci = 0; ci < (int64_t)N; ++ci) {
      uint32_t c = (uint32_t)ci;
      bool marked = false;
      for (uint32_t s = 0; s < S; ++s) {
        int64_t v = cnt(x, s, c) + own[(size_t)c * S + s];
        for (auto& e : in_edges[c]) {
          int64_t k = outk[((size_t)e.first * S + s) * 6 + e.second];
          v += k;
          if (mode == 1 && k > 0) marked = true;
        }
        nx[(size_t)s * N + c] = v;
      }
      if (mode == 0)
        for (auto& e : in_edges[c])
          if (leaped[e.first]) marked = true;
      if (marked && flag[c] == SSA_FF) flag[c] = SSA;
    }
    return events;
  }

  // ---------------------------------------------------------------- exact events
  // reference: one critical event in every LEAP_CR subvolume (leap.cu:67-199), then the SSA event
  // at the arg-min (ssa.cu:270-324).  All decisions read curr and the post-leap next; the deltas
  // are applied afterwards.
  int64_t exact_ref(uint64_t step, uint32_t attempt, int64_t argmin) {
    const int nc = opt.critical_threshold;
    std::vector<std::pair<size_t, int64_t>> delta;
    std::vector<uint32_t> flag_sets;
    int64_t events = 0;
    for (uint32_t c = 0; c < N; ++c) {
      if (flag[c] != LEAP_CR) continue;
      bool crit[PLIS_ORACLE_MAXR];
      for (uint32_t r = 0; r < R; ++r) crit[r] = crit_ref(x, c, r);
      plis_stream su = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_CRIT, step, attempt, 0);
      Real u = Ops::uniform(&su);
      Real rsum = (Real)0, dsum = (Real)0;
      for (uint32_t r = 0; r < R; ++r)
        if (crit[r]) rsum = rsum + rr_c[(size_t)r * N + c];
      for (uint32_t s = 0; s < S; ++s)
        if (cnt(x, s, c) < nc) dsum = dsum + dr_c[(size_t)s * N + c];
      if (rsum + dsum == (Real)0) continue;
      if (u < rsum / (rsum + dsum)) {
        Real scaled = rsum * u;
        Real partial = (Real)0;
        uint32_t ric = 0;
        while (partial <= scaled && ric < R) {
          if (crit[ric]) partial = partial + rr_c[(size_t)ric * N + c];
          ++ric;
        }
        uint32_t ri = 0;
        for (ri = 0; ri < R && ric > 0; ++ri)
          if (crit[ri]) --ric;
        ri = ri - 1;  // leap.cu:121-126, kept as written
        if (ri == (uint32_t)-1) ri = 0;
        bool fire = true;
        for (uint32_t s = 0; s < S; ++s) {
          int32_t need = reactants[(size_t)s * R + ri];
          fire = fire && cnt(x, s, c) >= need && cnt(nx, s, c) >= need;
        }
        if (!fire) continue;
        for (auto& e : rx[ri].net) delta.push_back({(size_t)e.first * N + c, (int64_t)e.second});
        ++events;
        note(step, attempt, c, c, 1, ri, 3);
      } else {
        Real scaled = dsum * u;
        Real partial = (Real)0;
        uint32_t spic = 0;
        while (partial <= scaled && spic < S) {
          if (cnt(x, spic, c) < nc) partial = partial + dr_c[(size_t)spic * N + c];
          ++spic;
        }
        uint32_t spi = 0;
        for (spi = 0; spi < S && spic > 0; ++spi)
          if (cnt(x, spi, c) < nc) --spic;
        spi = spi - 1;  // leap.cu:160-166
        if (spi == (uint32_t)-1) spi = 0;
        bool fire = cnt(x, spi, c) > 0 && cnt(nx, spi, c) > 0;
        if (!fire) continue;
        plis_stream sd = plis_stream_make(opt.seed, opt.replica, c, PLIS_PHASE_CRIT, step, attempt, 1);
        Real u2 = Ops::uniform(&sd);
        int slot = (int)(u2 * (Real)6);
        if (slot > 5) slot = 5;
        uint32_t target = nbr[(size_t)c * 6 + slot];
        if (target != c) {
          delta.push_back({(size_t)spi * N + c, -1});
          delta.push_back({(size_t)spi * N + target, 1});
          ++events;
          note(step, attempt, c, target, 1, spi, 4);
          uint32_t q = orig.empty() ? nbr[target] : orig[target];  // leap.cu:192-193
          flag_sets.push_back(q);
        }
      }
    }
    for (uint32_t q : flag_sets)
      if (flag[q] == SSA_FF) flag[q] = SSA;
    if (argmin >= 0 && (flag[argmin] == SSA || flag[argmin] == SSA_FF))
      events += ssa_event(step, attempt, (uint32_t)argmin, false, delta);
    for (auto& d : delta) nx[d.first] += d.second;
    return events;
  }

  // ssa_step (ssa.cu:270-324) in reference mode; in corrected mode the exact event of the arg-min
  // (critical channels only when it is LEAP_CR, every channel when it is an SSA subvolume).
  int64_t ssa_event(uint64_t step, uint32_t attempt, uint32_t m, bool critical_only,
                    std::vector<std::pair<size_t, int64_t>>& delta) {
    const int mode = opt.mode;
    const int nc = opt.critical_threshold;
    const int n = ncount[m];
    plis_stream su = plis_stream_make(opt.seed, opt.replica, m, PLIS_PHASE_SSA, step, attempt, 0);
    Real u = Ops::uniform(&su);
    if (mode == 0) {
      Real rsum = (Real)0, dsum = (Real)0;
      for (uint32_t r = 0; r < R; ++r) rsum = rsum + rr_c[(size_t)r * N + m];
      for (uint32_t s = 0; s < S; ++s) dsum = dsum + dr_c[(size_t)s * N + m];
      Real dtot = dsum * (Real)n;  // update_rate_matrix, rates.cu:165-172
      Real total = rsum + dtot;
      if (!(total > (Real)0)) return 0;
      if (u < rsum / total) {
        Real scaled = rsum * u;
        Real partial = (Real)0;
        uint32_t ri = 0;
        while (partial <= scaled && ri < R) { partial = partial + rr_c[(size_t)ri * N + m]; ++ri; }
        ri = ri - 1;
        if (ri == (uint32_t)-1) ri = 0;
        for (auto& e : rx[ri].net) delta.push_back({(size_t)e.first * N + m, (int64_t)e.second});
        flag[m] = SSA;  // ssa.cu:295
        note(step, attempt, m, m, 1, ri, 5);
        return 1;
      }
      if (!(dtot > (Real)0)) return 0;
      Real scaled = (dtot / (Real)n) * u;  // choose_rand_specie, ssa.cu:256-266
      Real partial = (Real)0;
      uint32_t spi = 0;
      while (partial <= scaled && spi < S) { partial = partial + dr_c[(size_t)spi * N + m]; ++spi; }
      spi = spi - 1;
      if (spi == (uint32_t)-1) spi = 0;
      plis_stream sd = plis_stream_make(opt.seed, opt.replica, m, PLIS_PHASE_SSA, step, attempt, 1);
      Real u2 = Ops::uniform(&sd);
      int slot = (int)(u2 * (Real)6);
      if (slot > 5) slot = 5;
      uint32_t target = nbr[(size_t)m * 6 + slot];
      if (target == m) return 0;
      delta.push_back({(size_t)spi * N + m, -1});
      delta.push_back({(size_t)spi * N + target, 1});
      if (flag[target] == SSA_FF) flag[target] = SSA;
      note(step, attempt, m, target, 1, spi, 6);
      return 1;
    }
    // corrected: channel rates
    Real total = (Real)0;
    for (uint32_t r = 0; r < R; ++r) {
      Real a = rr_c[(size_t)r * N + m];
      bool use = critical_only ? crit_fix(x, m, r, a) : true;
      if (use) total = total + a;
    }
    for (uint32_t s = 0; s < S; ++s) {
      bool use = critical_only ? (cnt(x, s, m) < nc) : true;
      if (use) total = total + (Real)n * dr_c[(size_t)s * N + m];
    }
    if (!(total > (Real)0)) return 0;
    Real scaled = total * u;
    Real partial = (Real)0;
    int chosen_r = -1, chosen_s = -1, last_r = -1, last_s = -1;
    for (uint32_t r = 0; r < R && chosen_r < 0; ++r) {
      Real a = rr_c[(size_t)r * N + m];
      bool use = critical_only ? crit_fix(x, m, r, a) : true;
      if (!use || !(a > (Real)0)) continue;
      partial = partial + a;
      last_r = (int)r;
      if (partial > scaled) chosen_r = (int)r;
    }
    if (chosen_r < 0) {
      for (uint32_t s = 0; s < S && chosen_s < 0; ++s) {
        bool use = critical_only ? (cnt(x, s, m) < nc) : true;
        Real w = (Real)n * dr_c[(size_t)s * N + m];
        if (!use || !(w > (Real)0)) continue;
        partial = partial + w;
        last_s = (int)s;
        if (partial > scaled) chosen_s = (int)s;
      }
    }
    if (chosen_r < 0 && chosen_s < 0) {  // rounding left the walk short: take the last channel
      if (last_s >= 0) chosen_s = last_s; else chosen_r = last_r;
    }
    const int kind_r = critical_only ? 3 : 5;
    if (chosen_r >= 0) {
      for (auto& e : rx[chosen_r].net) delta.push_back({(size_t)e.first * N + m, (int64_t)e.second});
      note(step, attempt, m, m, 1, (uint32_t)chosen_r, kind_r);
      return 1;
    }
    plis_stream sd = plis_stream_make(opt.seed, opt.replica, m, PLIS_PHASE_SSA, step, attempt, 1);
    Real u2 = Ops::uniform(&sd);
    int slot = (int)(u2 * (Real)n);
    if (slot > n - 1) slot = n - 1;
    uint32_t target = nbr[(size_t)m * 6 + slot];
    delta.push_back({(size_t)chosen_s * N + m, -1});
    delta.push_back({(size_t)chosen_s * N + target, 1});
    if (flag[target] == SSA_FF) flag[target] = SSA;
    note(step, attempt, m, target, 1, (uint32_t)chosen_s, kind_r + 1);
    return 1;
  }

  // ---------------------------------------------------------------- the step loop
  int advance(double t_end, uint64_t max_steps) override {
    const int mode = opt.mode;
    uint64_t done = 0;
    st.stop_reason = 0;
    while (true) {
      if (st.time >= t_end) { st.stop_reason = 1; break; }        // driver.cu:259
      if (done >= max_steps) { st.stop_reason = 2; break; }
      // arg-min tau, first index on ties (thrust::min_element, driver.cu:267-268)
      double tmin = PLIS_INF_D;
      int64_t am = -1;
      for (uint32_t c = 0; c < N; ++c)
        if (tau[c] < tmin) { tmin = tau[c]; am = c; }
      if (am < 0 || plis_isinf_d(tmin) || tmin < 0.0) {        // driver.cu:269-272
        if (mode == 1) { st.time = t_end; st.stop_reason = 1; }
        else st.stop_reason = 3;
        break;
      }
      double tstep = tmin;
      if (mode == 1 && t_end - st.time < tstep) tstep = t_end - st.time;
      const uint64_t step = st.steps + 1;
      uint32_t attempt = 0;
      int64_t events = 0, exact = 0;
      double dt = 0.0;
      while (true) {
        double scale = 1.0;
        for (uint32_t i = 0; i < attempt; ++i) scale *= 0.5;
        double tau_leap = (mode == 0) ? tmin : tstep * scale;
        dt = (mode == 0) ? tmin * scale : tau_leap;
        events = leap_all(step, attempt, tau_leap);
        exact = 0;
        if (mode == 0) {
          exact = exact_ref(step, attempt, am);
        } else if (attempt == 0 && tstep == tmin) {
          std::vector<std::pair<size_t, int64_t>> delta;
          uint8_t f = flag[am];
          if (f == LEAP_CR) exact = ssa_event(step, attempt, (uint32_t)am, true, delta);
          else if (f == SSA || f == SSA_FF) exact = ssa_event(step, attempt, (uint32_t)am, false, delta);
          for (auto& d : delta) nx[d.first] += d.second;
        }
        events += exact;
        bool neg = leap_big != 0;
        for (size_t i = 0; i < (size_t)S * N && !neg; ++i)
          if (nx[i] < 0) neg = true;
        if (!neg) break;
        ++attempt;  // check_state + revert, leap.cu:203-212, driver.cu:292-315
        if ((int)attempt > opt.max_rollbacks) { st.status = 7; st.stop_reason = 4; return 7; }
      }
      st.time += dt;
      st.steps = step;
      st.rollbacks += attempt;
      st.events += (uint64_t)events;
      st.exact_events += (uint64_t)exact;
      st.leap_events += (uint64_t)(events - exact);
      st.last_tau = tmin;
      st.last_argmin = am;
      x.swap(nx);
      ff_tau = dt;  // reference: the (halved) min_tau handed to compute_taus, driver.cu:305, :333
      classify_all(step, attempt);
      ++done;
    }
    return st.status;
  }
};

template <typename Real>
Base* make_sim(const oracle_model* m, const oracle_options* o) {
  Sim<Real>* s = new Sim<Real>();
  s->N = m->n_subvolumes;
  s->S = m->n_species;
  s->R = m->n_reactions;
  s->C = m->n_compartments ? m->n_compartments : 1;
  size_t N = s->N, S = s->S, R = s->R, C = s->C;
  s->nbr.assign(m->nbr, m->nbr + 6 * N);
  if (m->orig) s->orig.assign(m->orig, m->orig + 6 * N);
  s->reactants.assign(m->reactants, m->reactants + S * R);
  s->products.assign(m->products, m->products + S * R);
  s->rrate.assign(m->reaction_rates, m->reaction_rates + C * R);
  s->drate.assign(m->diffusion_rates, m->diffusion_rates + C * S);
  if (m->compartment) s->comp.assign(m->compartment, m->compartment + N);
  s->opt = *o;
  s->init_tables();
  s->x.assign(S * N, 0);
  s->nx.assign(S * N, 0);
  s->tau.assign(N, PLIS_INF_D);
  s->flag.assign(N, SSA_FF);
  s->rr_c.assign(R * N, (Real)0);
  s->dr_c.assign(S * N, (Real)0);
  s->own.assign(N * S, 0);
  s->outk.assign(N * S * 6, 0);
  s->leaped.assign(N, 0);
  s->evc.assign(N, 0);
  s->bigc.assign(N, 0);
  return s;
}

}  // namespace

extern "C" {

void* oracle_create(const oracle_model* m, const oracle_options* o) {
  if (!m || !o || m->n_reactions > PLIS_ORACLE_MAXR || m->n_subvolumes == 0) return nullptr;
#ifdef _OPENMP
  if (o->threads > 0) omp_set_num_threads(o->threads);
#endif
  if (o->precision == 1) return make_sim<float>(m, o);
  return make_sim<double>(m, o);
}
void oracle_destroy(void* h) { delete static_cast<Base*>(h); }
int oracle_set_state(void* h, const uint32_t* c) { return static_cast<Base*>(h)->set_state(c, 0.0, 0); }
int oracle_set_state_at(void* h, const uint32_t* c, double t0, uint64_t step0) {
  return static_cast<Base*>(h)->set_state(c, t0, step0);
}
int oracle_get_state(void* h, uint32_t* c) { return static_cast<Base*>(h)->get_state(c); }
int oracle_get_taus(void* h, double* t, uint8_t* f) { return static_cast<Base*>(h)->get_taus(t, f); }
int oracle_get_stats(void* h, oracle_stats* st) {
  *st = static_cast<Base*>(h)->st;
  return 0;
}
int oracle_advance(void* h, double t_end, uint64_t max_steps) {
  return static_cast<Base*>(h)->advance(t_end, max_steps);
}
void oracle_set_event_log(void* h, int on) {
  Base* b = static_cast<Base*>(h);
  b->logging = on != 0;
  b->log.clear();
}
int64_t oracle_read_event_log(void* h, oracle_event* out, int64_t max) {
  Base* b = static_cast<Base*>(h);
  const int64_t n = (int64_t)b->log.size();
  if (!out) return n;
  for (int64_t i = 0; i < n && i < max; ++i) out[i] = b->log[(size_t)i];
  b->log.clear();
  return n;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Test hooks over the shared stream numerics (pliscuda_b200/csrc/plis_stream.h).
// ---------------------------------------------------------------------------------------------
extern "C" {

// Canonical neighbour table of the oracle, built here rather than taken from the product so that a
// fault in the product's slot order cannot hide from the parity tests.  The reference pads each
// 6-wide row with the subvolume's own index (PLISCuda/include/cpp/Topology.hpp:176-184); its leap
// and SSA draw a destination slot among the six (leap.cu:180-186, ssa.cu:89-106).  The canonical
// row keeps the non-self entries in file order and pads with the own index after them.  A table that
// is a reflective x-fastest lattice is rewritten in the fixed direction order -x,+x,-y,+y,-z,+z,
// which is also the order of an implicit lattice (no table).  Lattice dimensions are read off row 0:
// its sorted non-self entries are {} (one subvolume), {1} (a chain), {1, X} or {1, X, X*Y}; the
// candidate is accepted when every row holds exactly that lattice's neighbours.  Unit dimensions are
// moved to the back, since (1, Y, Z) linearises like (Y, Z, 1).
static int lattice_nbrs(const uint32_t d[3], uint32_t c, uint32_t out[6]) {
  const uint64_t X = d[0], XY = (uint64_t)d[0] * d[1];
  const uint32_t x = (uint32_t)(c % X), y = (uint32_t)((c / X) % d[1]), z = (uint32_t)(c / XY);
  int k = 0;
  if (x >= 1) out[k++] = c - 1;
  if (x + 1 < d[0]) out[k++] = c + 1;
  if (y >= 1) out[k++] = (uint32_t)(c - X);
  if (y + 1 < d[1]) out[k++] = (uint32_t)(c + X);
  if (z >= 1) out[k++] = (uint32_t)(c - XY);
  if (z + 1 < d[2]) out[k++] = (uint32_t)(c + XY);
  return k;
}

static void units_last(uint32_t d[3]) {
  uint32_t v[3] = {1, 1, 1};
  int k = 0;
  for (int i = 0; i < 3; ++i)
    if (d[i] != 1) v[k++] = d[i];
  d[0] = v[0]; d[1] = v[1]; d[2] = v[2];
}

int oracle_canonical_neighbours(uint32_t n, const uint32_t* table, const uint32_t* lattice, uint32_t* out,
                                uint32_t* dims_out) {
  if (n == 0 || !out) return 1;
  uint32_t d[3] = {0, 0, 0};
  bool is_lattice = false;
  if (!table) {
    if (!lattice || (uint64_t)lattice[0] * lattice[1] * lattice[2] != n) return 1;
    d[0] = lattice[0]; d[1] = lattice[1]; d[2] = lattice[2];
    units_last(d);
    is_lattice = true;
  } else {
    std::vector<uint32_t> row0;
    for (int j = 0; j < 6; ++j) {
      const uint32_t b = table[j];
      if (b >= n) return 1;
      if (b != 0) row0.push_back(b);
    }
    std::sort(row0.begin(), row0.end());
    uint32_t cand[3] = {0, 0, 0};
    bool have = false;
    if (row0.empty()) { cand[0] = 1; cand[1] = 1; cand[2] = 1; have = (n == 1); }
    else if (row0[0] == 1 && row0.size() == 1) { cand[0] = n; cand[1] = 1; cand[2] = 1; have = true; }
    else if (row0[0] == 1 && row0.size() == 2 && n % row0[1] == 0) {
      cand[0] = row0[1]; cand[1] = n / row0[1]; cand[2] = 1; have = true;
    } else if (row0[0] == 1 && row0.size() == 3 && row0[2] % row0[1] == 0 && n % row0[2] == 0) {
      cand[0] = row0[1]; cand[1] = row0[2] / row0[1]; cand[2] = n / row0[2]; have = true;
    }
    if (have) {
      is_lattice = true;
      for (uint32_t c = 0; c < n && is_lattice; ++c) {
        std::vector<uint32_t> got;
        for (int j = 0; j < 6; ++j) {
          const uint32_t b = table[(size_t)c * 6 + j];
          if (b >= n) return 1;
          if (b != c) got.push_back(b);
        }
        uint32_t want[6];
        const int k = lattice_nbrs(cand, c, want);
        std::sort(got.begin(), got.end());
        std::sort(want, want + k);
        is_lattice = (int)got.size() == k && std::equal(want, want + k, got.begin());
      }
      if (is_lattice) { d[0] = cand[0]; d[1] = cand[1]; d[2] = cand[2]; units_last(d); }
    }
  }
  if (is_lattice) {
    for (uint32_t c = 0; c < n; ++c) {
      uint32_t row[6];
      const int k = lattice_nbrs(d, c, row);
      for (int j = 0; j < 6; ++j) out[(size_t)c * 6 + j] = j < k ? row[j] : c;
    }
  } else {
    for (uint32_t c = 0; c < n; ++c) {
      int k = 0;
      for (int j = 0; j < 6; ++j) {
        const uint32_t b = table[(size_t)c * 6 + j];
        if (b >= n) return 1;
        if (b != c) out[(size_t)c * 6 + k++] = b;
      }
      for (; k < 6; ++k) out[(size_t)c * 6 + k] = c;
    }
    d[0] = d[1] = d[2] = 0;
  }
  if (dims_out) { dims_out[0] = d[0]; dims_out[1] = d[1]; dims_out[2] = d[2]; }
  return 0;
}

void oracle_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  plis_u32x4 c = {ctr[0], ctr[1], ctr[2], ctr[3]};
  plis_u32x4 r = plis_philox4x32_10(c, key[0], key[1]);
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

// n draws, draw i from the stream of (seed, cell=i, phase LEAP, step, attempt 0, channel)
void oracle_poisson(uint64_t seed, uint64_t step, uint32_t channel, double lam, int precision, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    plis_stream s = plis_stream_make(seed, 0, (uint32_t)i, PLIS_PHASE_LEAP, step, 0, channel);
    out[i] = precision ? plis_poisson_f(&s, (float)lam) : plis_poisson_d(&s, lam);
  }
}

void oracle_uniforms(uint64_t seed, uint32_t cell, int precision, int64_t n, double* out) {
  plis_stream s = plis_stream_make(seed, 0, cell, PLIS_PHASE_INIT, 0, 0, 0);
  for (int64_t i = 0; i < n; ++i) out[i] = precision ? (double)plis_uniform_f(&s) : plis_uniform_d(&s);
}

void oracle_exponential(uint64_t seed, double rate, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    plis_stream s = plis_stream_make(seed, 0, (uint32_t)i, PLIS_PHASE_TAU, 1, 0, 0);
    out[i] = plis_exponential_d(&s, rate);
  }
}

void oracle_math(int which, const double* x, int64_t n, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    switch (which) {
      case 0: out[i] = plis_exp(x[i]); break;
      case 1: out[i] = plis_log(x[i]); break;
      case 2: out[i] = (double)plis_expf((float)x[i]); break;
      case 3: out[i] = (double)plis_logf((float)x[i]); break;
      default: out[i] = plis_lnfact(x[i]); break;
    }
  }
}

}  // extern "C"

// loader.cpp — readers for the reference's input files, unchanged formats.
//
// Each parser follows the reference's operator>> (same accepted syntax, same error messages) but
// reads the whole file once and converts with pointer scans instead of getline/split/stoi per token
// (PLISCuda/include/cpp/State.hpp:165-212 allocates a vector of strings per line; a 2M-subvolume
// topology takes seconds that way).  Where the reference would read uninitialised memory or write
// past an array, the loader reports an error instead:
//   * a topology row with more than 6 neighbours (Topology.hpp:176 writes past the row),
//   * a topology that lists fewer rows than its header (rows stay uninitialised, Topology.hpp:122),
//   * a reactions file with a different number of lines than its header (Reactions.hpp:185-219),
//   * a constants line with fewer values than reactions/species (std::out_of_range, cpp_utils.hpp:33).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/plis.h"

namespace plis {

// A whole input file, memory-mapped read-only (or read into memory when it cannot be mapped).
struct Text {
  const char* p = nullptr;
  size_t n = 0;
  size_t pos = 0;
  void* map = nullptr;
  std::string own;
  bool eof() const { return pos >= n; }
  Text() = default;
  Text(const Text&) = delete;
  Text& operator=(const Text&) = delete;
  ~Text() {
    if (map) munmap(map, n);
  }
};

static int read_file(const std::string& path, Text* t, std::string* err) {
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) { *err = "file " + path + " not found"; return PLIS_ERR_IO; }
  struct stat st;
  if (fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
    void* m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m != MAP_FAILED) {
      madvise(m, (size_t)st.st_size, MADV_SEQUENTIAL);
      t->map = m;
      t->p = static_cast<const char*>(m);
      t->n = (size_t)st.st_size;
      t->pos = 0;
      close(fd);
      return PLIS_OK;
    }
  }
  close(fd);
  std::ifstream f(path, std::ios::binary);
  if (!f.good()) { *err = "file " + path + " not found"; return PLIS_ERR_IO; }
  std::ostringstream ss;
  ss << f.rdbuf();
  t->own = ss.str();
  t->p = t->own.data();
  t->n = t->own.size();
  t->pos = 0;
  return PLIS_OK;
}

// std::getline(is, out, delim) as a view [*b, *e) into the file: extracts up to delim (consumed,
// not stored); false if nothing extracted
static bool getline_v(Text* t, char delim, const char** b, const char** e) {
  if (t->eof()) return false;
  const char* s = t->p + t->pos;
  const char* end = t->p + t->n;
  const char* d = static_cast<const char*>(memchr(s, delim, (size_t)(end - s)));
  *b = s;
  if (!d) {
    *e = end;
    t->pos = t->n;
  } else {
    *e = d;
    t->pos = (size_t)(d - t->p) + 1;
  }
  return true;
}

static bool getline_d(Text* t, char delim, std::string* out) {
  const char *b, *e;
  if (!getline_v(t, delim, &b, &e)) return false;
  out->assign(b, e);
  return true;
}

static void get_char(Text* t) {
  if (!t->eof()) t->pos++;
}

// std::stoi on the text [s, e): leading whitespace, optional sign, at least one digit, trailing
// text ignored, int range
static bool int_at(const char* s, const char* e, long long* v) {
  while (s < e && (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r' || *s == '\f' || *s == '\v')) ++s;
  bool neg = false;
  if (s < e && (*s == '+' || *s == '-')) {
    neg = *s == '-';
    ++s;
  }
  if (s >= e || *s < '0' || *s > '9') return false;
  long long r = 0;
  while (s < e && *s >= '0' && *s <= '9') {
    r = r * 10 + (*s - '0');
    if (r > (long long)INT_MAX + 1) return false;
    ++s;
  }
  r = neg ? -r : r;
  if (r > INT_MAX || r < INT_MIN) return false;
  *v = r;
  return true;
}

static bool only_space_v(const char* b, const char* e) {
  for (; b < e; ++b)
    if (!(*b == ' ' || *b == '\n' || *b == '\r' || *b == '\t')) return false;
  return true;
}

// PLISCuda::split(line, ' ') over a view: calls f(index, token_begin, token_end) for every token
// between single spaces (a trailing empty token is dropped); returns the token count, or -1 if f
// failed
template <typename F>
static long long for_tokens(const char* b, const char* e, F f) {
  long long k = 0;
  while (b < e) {
    const char* sp = static_cast<const char*>(memchr(b, ' ', (size_t)(e - b)));
    const char* te = sp ? sp : e;
    if (!f(k, b, te)) return -1;
    ++k;
    if (!sp) break;
    b = sp + 1;
  }
  return k;
}

// std::stoi semantics: leading whitespace, optional sign, at least one digit, trailing text ignored
static bool to_int(const char* s, long long* v) {
  while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r' || *s == '\f' || *s == '\v') ++s;
  errno = 0;
  char* end = nullptr;
  long long r = strtoll(s, &end, 10);
  if (end == s || errno == ERANGE || r > INT_MAX || r < INT_MIN) return false;
  *v = r;
  return true;
}
static bool to_float(const char* s, float* v) {
  while (*s == ' ' || *s == '\t' || *s == '\n' || *s == '\r') ++s;
  char* end = nullptr;
  float r = strtof(s, &end);
  if (end == s) return false;
  *v = r;
  return true;
}

// PLISCuda::split(s, ' '): tokens between single spaces; a trailing empty token is dropped
static void split_sp(const std::string& s, std::vector<std::string>* out) {
  out->clear();
  size_t i = 0;
  while (i < s.size()) {
    size_t e = s.find(' ', i);
    if (e == std::string::npos) {
      out->push_back(s.substr(i));
      return;
    }
    out->push_back(s.substr(i, e - i));
    i = e + 1;
  }
}

static bool only_space(const std::string& s) {
  for (char c : s)
    if (!(c == ' ' || c == '\n' || c == '\r' || c == '\t')) return false;
  return true;
}

static std::string strip_cr(std::string s) {
  if (!s.empty() && s.back() == '\r') s.pop_back();
  return s;
}

// Topology.hpp:98-191
int parse_topology(const std::string& path, uint32_t* n_out, std::vector<uint32_t>* nb, std::string* err) {
  Text t;
  int rc = read_file(path, &t, err);
  if (rc) return rc;
  std::string a;
  getline_d(&t, ':', &a);
  getline_d(&t, '\n', &a);
  long long n;
  if (!to_int(a.c_str(), &n)) { *err = "Invalid subvolumes number: " + a; return PLIS_ERR_PARSE; }
  if (n < 1) { *err = "Invalid: n < 1"; return PLIS_ERR_PARSE; }
  nb->assign((size_t)6 * n, 0);
  get_char(&t);
  uint32_t counter = 0;
  const char *sb, *se, *lb = nullptr, *le = nullptr;
  while (getline_v(&t, ':', &sb, &se)) {
    if (only_space_v(sb, se) && t.eof()) break;
    long long idx;
    if (!int_at(sb, se, &idx) || idx != (long long)counter || counter >= (uint32_t)n) {
      *err = "Invalid subvolume number : " + std::string(sb, se);
      return PLIS_ERR_PARSE;
    }
    counter++;
    get_char(&t);
    // at the end of the file std::getline leaves the previous line in place, and so does this
    getline_v(&t, '\n', &lb, &le);
    if (!lb) lb = le = t.p + t.n;
    const char* lend = (le > lb && le[-1] == '\r') ? le - 1 : le;
    uint32_t* row = nb->data() + (size_t)(counter - 1) * 6;
    int code = 0;
    const long long k = for_tokens(lb, lend, [&](long long i, const char* b, const char* e) {
      if (i >= 6) { code = 1; return false; }
      long long v;
      if (!int_at(b, e, &v)) { code = 2; return false; }
      if ((unsigned long long)(unsigned int)v >= (unsigned long long)n) { code = 3; return false; }
      row[i] = (uint32_t)v;
      return true;
    });
    if (k < 0) {
      if (code == 1) { *err = "more than 6 neighbours for subvolume " + std::to_string(counter - 1); return PLIS_ERR_PARSE; }
      if (code == 2) { *err = "parse of neighbour number failed"; return PLIS_ERR_PARSE; }
      *err = "Invalid: sub >= n";
      return PLIS_ERR_PARSE;
    }
    for (long long i = k; i < 6; ++i) row[i] = counter - 1;  // self padding, Topology.hpp:181-184
  }
  if (counter != (uint32_t)n) {
    *err = "topology lists " + std::to_string(counter) + " of " + std::to_string(n) + " subvolumes";
    return PLIS_ERR_PARSE;
  }
  *n_out = (uint32_t)n;
  return PLIS_OK;
}

static int parse_header2(Text* t, const char* what1, const char* what2, long long* a1, long long* a2, std::string* err) {
  std::string a;
  getline_d(t, ':', &a);
  getline_d(t, '\n', &a);
  if (!to_int(a.c_str(), a1)) { *err = std::string("Invalid ") + what1 + " number : " + a; return PLIS_ERR_PARSE; }
  if (*a1 < 1) { *err = std::string("Invalid: ") + (what1[0] == 's' ? "n" : "r") + " < 1"; return PLIS_ERR_PARSE; }
  getline_d(t, ':', &a);
  getline_d(t, '\n', &a);
  if (!to_int(a.c_str(), a2)) { *err = std::string("Invalid ") + what2 + " number : " + a; return PLIS_ERR_PARSE; }
  if (*a2 < 1) { *err = "Invalid: s < 1"; return PLIS_ERR_PARSE; }
  get_char(t);
  return PLIS_OK;
}

// State.hpp:112-217
int parse_state(const std::string& path, uint32_t* n_out, uint32_t* s_out, std::vector<uint32_t>* st, std::string* err) {
  Text t;
  int rc = read_file(path, &t, err);
  if (rc) return rc;
  long long n, s;
  if ((rc = parse_header2(&t, "subvolume", "species", &n, &s, err))) return rc;
  st->assign((size_t)n * s, 0);
  const char *sb, *se, *lb = nullptr, *le = nullptr;
  while (getline_v(&t, ':', &sb, &se)) {
    if (only_space_v(sb, se) && t.eof()) break;
    long long idx;
    if (!int_at(sb, se, &idx)) { *err = "Invalid subvolume number : " + std::string(sb, se); return PLIS_ERR_PARSE; }
    if (idx < 0 || idx >= n) { *err = "Unexpected subvolume number. Got: " + std::to_string(idx); return PLIS_ERR_PARSE; }
    get_char(&t);
    getline_v(&t, '\n', &lb, &le);  // at the end of the file the previous line stays, as with std::getline
    if (!lb) lb = le = t.p + t.n;
    const char* lend = (le > lb && le[-1] == '\r') ? le - 1 : le;
    const long long k = for_tokens(lb, lend, [&](long long, const char*, const char*) { return true; });
    if (k != s) {
      *err = "Parse of subvolume line failed (subvolume " + std::string(lb, lend) + ") has wrong length";
      return PLIS_ERR_PARSE;
    }
    int code = 0;
    for_tokens(lb, lend, [&](long long i, const char* b, const char* e) {
      long long c;
      if (!int_at(b, e, &c)) { code = 1; return false; }
      if (c < 0) { code = 2; return false; }
      (*st)[(size_t)idx + (size_t)n * (size_t)i] = (uint32_t)c;  // species-major, State.hpp:210
      return true;
    });
    if (code == 1) { *err = "parse of species count number failed"; return PLIS_ERR_PARSE; }
    if (code == 2) { *err = "Invalid: species count < 0"; return PLIS_ERR_PARSE; }
  }
  *n_out = (uint32_t)n;
  *s_out = (uint32_t)s;
  return PLIS_OK;
}

// Reactions.hpp:132-223
int parse_reactions(const std::string& path, uint32_t* r_out, uint32_t* s_out, std::vector<int32_t>* re,
                    std::vector<int32_t>* pr, std::string* err) {
  Text t;
  int rc = read_file(path, &t, err);
  if (rc) return rc;
  long long r, s;
  if ((rc = parse_header2(&t, "reactions", "species", &r, &s, err))) return rc;
  re->assign((size_t)r * s, 0);
  pr->assign((size_t)r * s, 0);
  std::string line;
  std::vector<std::string> tok;
  long long cur = 0;
  while (getline_d(&t, '\n', &line)) {
    line = strip_cr(line);
    if (only_space(line) && t.eof()) break;
    split_sp(line, &tok);
    if ((long long)tok.size() != 2 * s + 1 || cur >= r) {
      *err = "Parse of reactions line failed (reaction " + std::to_string(cur) + ")";
      return PLIS_ERR_PARSE;
    }
    for (long long i = 0; i < s; ++i) {
      long long v;
      if (!to_int(tok[i].c_str(), &v)) {
        *err = "parse of stechiometric coeff. failed (reaction " + std::to_string(cur) + ")";
        return PLIS_ERR_PARSE;
      }
      (*re)[(size_t)cur + (size_t)r * i] = (int32_t)v;  // species-major, Reactions.hpp:197
    }
    for (long long i = 0; i < s; ++i) {
      long long v;
      if (!to_int(tok[s + i + 1].c_str(), &v)) {
        *err = "parse of stechiometric coeff. failed(reaction " + std::to_string(cur);
        return PLIS_ERR_PARSE;
      }
      (*pr)[(size_t)cur + (size_t)r * i] = (int32_t)v;
    }
    ++cur;
  }
  if (cur != r) {
    *err = "reactions file lists " + std::to_string(cur) + " of " + std::to_string(r) + " reactions";
    return PLIS_ERR_PARSE;
  }
  *r_out = (uint32_t)r;
  *s_out = (uint32_t)s;
  return PLIS_OK;
}

// cpp_utils.hpp:29-45: line 1 = R reaction constants, line 2 = S diffusion constants (parsed as float)
static int parse_constants(const std::string& path, uint32_t R, uint32_t S, double* rr, double* dr, std::string* err) {
  Text t;
  int rc = read_file(path, &t, err);
  if (rc) return rc;
  std::string line;
  std::vector<std::string> tok;
  getline_d(&t, '\n', &line);
  split_sp(strip_cr(line), &tok);
  if (tok.size() < R) { *err = "constants file " + path + ": fewer reaction constants than reactions"; return PLIS_ERR_PARSE; }
  for (uint32_t i = 0; i < R; ++i) {
    float v;
    if (!to_float(tok[i].c_str(), &v)) { *err = "constants file " + path + ": bad reaction constant"; return PLIS_ERR_PARSE; }
    rr[i] = (double)v;
  }
  line.clear();
  getline_d(&t, '\n', &line);
  split_sp(strip_cr(line), &tok);
  if (tok.size() < S) { *err = "constants file " + path + ": fewer diffusion constants than species"; return PLIS_ERR_PARSE; }
  for (uint32_t i = 0; i < S; ++i) {
    float v;
    if (!to_float(tok[i].c_str(), &v)) { *err = "constants file " + path + ": bad diffusion constant"; return PLIS_ERR_PARSE; }
    dr[i] = (double)v;
  }
  return PLIS_OK;
}

// cpp_utils.hpp:47-56: the i-th line's value (after ':') is the compartment of subvolume i
static int parse_compartments(const std::string& path, uint32_t N, std::vector<int32_t>* comp, std::string* err) {
  Text t;
  int rc = read_file(path, &t, err);
  if (rc) return rc;
  comp->assign(N, 0);
  std::string a;
  for (uint32_t i = 0; i < N; ++i) {
    if (!getline_d(&t, ':', &a) || !getline_d(&t, '\n', &a)) { *err = "compartments file too short"; return PLIS_ERR_PARSE; }
    long long v;
    if (!to_int(a.c_str(), &v)) { *err = "compartments file: bad value"; return PLIS_ERR_PARSE; }
    (*comp)[i] = (int32_t)v;
  }
  return PLIS_OK;
}

struct Config {
  uint32_t N = 0, S = 0, R = 0, C = 1;
  std::vector<uint32_t> nb, state;
  std::vector<int32_t> re, pr, comp;
  std::vector<double> rr, dr;
  double end_time = 0, log_freq = 0;
};

static std::string resolve(const std::string& dir, const std::string& p) {
  if (p.empty() || p[0] == '/') return p;
  std::string c = dir.empty() ? p : dir + "/" + p;
  std::ifstream f(c);
  if (f.good()) return c;
  return p;  // the reference opens paths relative to the working directory
}

static bool conf_key(Text* t, const char* key, std::string* val) {
  std::string k;
  if (!getline_d(t, '=', &k)) return false;
  if (strip_cr(k) != key) return false;
  getline_d(t, '\n', val);
  *val = strip_cr(*val);
  return true;
}

// Configuration.hpp:27-144
int load_config(const std::string& conf, Config* c, std::string* err) {
  Text t;
  int rc = read_file(conf, &t, err);
  if (rc) { *err = "Couldn't load configuration file"; return rc; }
  std::string dir;
  size_t sl = conf.find_last_of('/');
  if (sl != std::string::npos) dir = conf.substr(0, sl);
  std::string v;
  if (!conf_key(&t, "topology", &v)) { *err = "need a topology file"; return PLIS_ERR_PARSE; }
  if ((rc = parse_topology(resolve(dir, v), &c->N, &c->nb, err))) return rc;
  if (!conf_key(&t, "reactions", &v)) { *err = "need a reactions file"; return PLIS_ERR_PARSE; }
  uint32_t rs = 0;
  if ((rc = parse_reactions(resolve(dir, v), &c->R, &rs, &c->re, &c->pr, err))) return rc;
  if (!conf_key(&t, "initialState", &v)) { *err = "need a state file"; return PLIS_ERR_PARSE; }
  uint32_t sn = 0;
  if ((rc = parse_state(resolve(dir, v), &sn, &c->S, &c->state, err))) return rc;
  if (sn != c->N) { *err = "state and topology disagree on the number of subvolumes"; return PLIS_ERR_INVALID; }
  if (rs != c->S) { *err = "state and reactions disagree on the number of species"; return PLIS_ERR_INVALID; }
  float f;
  if (!conf_key(&t, "endTime", &v)) { *err = "need an endtime value"; return PLIS_ERR_PARSE; }
  if (!to_float(v.c_str(), &f)) { *err = "bad endTime value"; return PLIS_ERR_PARSE; }
  c->end_time = f;
  if (!conf_key(&t, "logFreq", &v)) { *err = "need a logFreq value (0 = no logging)"; return PLIS_ERR_PARSE; }
  if (!to_float(v.c_str(), &f)) { *err = "bad logFreq value"; return PLIS_ERR_PARSE; }
  c->log_freq = f;
  if (!conf_key(&t, "compartments", &v)) { *err = "need a compartments value"; return PLIS_ERR_PARSE; }
  long long nc;
  if (!to_int(v.c_str(), &nc)) { *err = "bad compartments value"; return PLIS_ERR_PARSE; }
  if (nc < 1) { *err = "compartments count < 1"; return PLIS_ERR_PARSE; }
  c->C = (uint32_t)nc;
  if (nc > 1) {
    if (!conf_key(&t, "compartmentsFile", &v)) { *err = "need a compartments file"; return PLIS_ERR_PARSE; }
    if ((rc = parse_compartments(resolve(dir, v), c->N, &c->comp, err))) return rc;
  } else {
    c->comp.clear();
  }
  c->rr.assign((size_t)c->C * c->R, 0.0);
  c->dr.assign((size_t)c->C * c->S, 0.0);
  for (uint32_t i = 0; i < c->C; ++i) {
    if (!conf_key(&t, "constants", &v)) {
      *err = "need a constants file (" + std::to_string(i + 1) + ")";
      return PLIS_ERR_PARSE;
    }
    if ((rc = parse_constants(resolve(dir, v), c->R, c->S, &c->rr[(size_t)i * c->R], &c->dr[(size_t)i * c->S], err)))
      return rc;
  }
  return PLIS_OK;
}

}  // namespace plis

struct plis_config {
  plis::Config c;
};

namespace plis {
void set_error(const std::string& msg);
}
using plis::set_error;

extern "C" int plis_config_load(const char* conf_path, plis_config** out) {
  if (!conf_path || !out) { set_error("null argument"); return PLIS_ERR_INVALID; }
  plis_config* cfg = new plis_config();
  std::string err;
  int rc = plis::load_config(conf_path, &cfg->c, &err);
  if (rc) {
    delete cfg;
    set_error(err);
    return rc;
  }
  *out = cfg;
  return PLIS_OK;
}

extern "C" int plis_config_view_get(const plis_config* cfg, plis_config_view* v) {
  if (!cfg || !v) { set_error("null argument"); return PLIS_ERR_INVALID; }
  const plis::Config& c = cfg->c;
  std::memset(v, 0, sizeof *v);
  v->model.n_subvolumes = c.N;
  v->model.n_species = c.S;
  v->model.n_reactions = c.R;
  v->model.n_compartments = c.C;
  v->model.neighbours = c.nb.data();
  v->model.reactants = c.re.data();
  v->model.products = c.pr.data();
  v->model.reaction_rates = c.rr.data();
  v->model.diffusion_rates = c.dr.data();
  v->model.compartment = c.comp.empty() ? nullptr : c.comp.data();
  v->initial_state = c.state.data();
  v->end_time = c.end_time;
  v->log_freq = c.log_freq;
  return PLIS_OK;
}

extern "C" void plis_config_free(plis_config* cfg) { delete cfg; }

extern "C" int plis_parse_topology(const char* path, uint32_t* n_out, uint32_t** nb_out) {
  std::vector<uint32_t> nb;
  std::string err;
  int rc = plis::parse_topology(path ? path : "", n_out, &nb, &err);
  if (rc) { set_error(err); return rc; }
  *nb_out = (uint32_t*)malloc(nb.size() * sizeof(uint32_t));
  if (!*nb_out) { set_error("out of memory"); return PLIS_ERR_OOM; }
  std::memcpy(*nb_out, nb.data(), nb.size() * sizeof(uint32_t));
  return PLIS_OK;
}

extern "C" int plis_parse_state(const char* path, uint32_t* n_out, uint32_t* s_out, uint32_t** counts_out) {
  std::vector<uint32_t> st;
  std::string err;
  int rc = plis::parse_state(path ? path : "", n_out, s_out, &st, &err);
  if (rc) { set_error(err); return rc; }
  *counts_out = (uint32_t*)malloc(st.size() * sizeof(uint32_t));
  if (!*counts_out) { set_error("out of memory"); return PLIS_ERR_OOM; }
  std::memcpy(*counts_out, st.data(), st.size() * sizeof(uint32_t));
  return PLIS_OK;
}

extern "C" int plis_parse_reactions(const char* path, uint32_t* r_out, uint32_t* s_out, int32_t** re_out,
                                    int32_t** pr_out) {
  std::vector<int32_t> re, pr;
  std::string err;
  int rc = plis::parse_reactions(path ? path : "", r_out, s_out, &re, &pr, &err);
  if (rc) { set_error(err); return rc; }
  *re_out = (int32_t*)malloc(re.size() * sizeof(int32_t));
  *pr_out = (int32_t*)malloc(pr.size() * sizeof(int32_t));
  if (!*re_out || !*pr_out) { set_error("out of memory"); return PLIS_ERR_OOM; }
  std::memcpy(*re_out, re.data(), re.size() * sizeof(int32_t));
  std::memcpy(*pr_out, pr.data(), pr.size() * sizeof(int32_t));
  return PLIS_OK;
}

extern "C" void plis_free(void* p) { free(p); }

// print_state_snapshot, driver.cu:435-447: header lines, blank line, one line of S counts per
// subvolume each followed by a space.  The time is printed like std::to_string(float).
// The .dat snapshot print_state_snapshot writes (driver.cu:435-447): "subvolumes=N", "species=S",
// "time=T", an empty line, then N lines of S counts each followed by a space.
extern "C" int plis_read_snapshot(const char* path, uint32_t* n_out, uint32_t* s_out, double* time_out,
                                  uint32_t** counts_out) {
  using plis::Text;
  using plis::read_file;
  using plis::getline_v;
  using plis::int_at;
  using plis::for_tokens;
  if (!path || !n_out || !s_out || !time_out || !counts_out) { set_error("null argument"); return PLIS_ERR_INVALID; }
  *counts_out = nullptr;
  Text t;
  std::string err;
  int rc = read_file(path, &t, &err);
  if (rc) { set_error(err); return rc; }
  const char *b, *e;
  long long hv[2];
  const char* keys[2] = {"subvolumes=", "species="};
  for (int i = 0; i < 2; ++i) {
    const size_t kl = strlen(keys[i]);
    if (!getline_v(&t, '\n', &b, &e) || (size_t)(e - b) < kl || strncmp(b, keys[i], kl) != 0 ||
        !int_at(b + kl, e, &hv[i]) || hv[i] < 1) {
      set_error(std::string("snapshot ") + path + ": expected " + keys[i] + "<positive integer>");
      return PLIS_ERR_PARSE;
    }
  }
  if (!getline_v(&t, '\n', &b, &e) || (e - b) < 5 || strncmp(b, "time=", 5) != 0) {
    set_error(std::string("snapshot ") + path + ": expected time=<value>");
    return PLIS_ERR_PARSE;
  }
  const std::string tv(b + 5, e);
  char* endp = nullptr;
  const double time = strtod(tv.c_str(), &endp);
  if (endp == tv.c_str()) {
    set_error(std::string("snapshot ") + path + ": bad time value");
    return PLIS_ERR_PARSE;
  }
  getline_v(&t, '\n', &b, &e);  // the empty line
  const uint64_t n = (uint64_t)hv[0], ns = (uint64_t)hv[1];
  if (n * ns > (1ull << 34)) { set_error("snapshot too large"); return PLIS_ERR_LIMIT; }
  uint32_t* out = static_cast<uint32_t*>(malloc(n * ns * sizeof(uint32_t)));
  if (!out) { set_error("out of host memory"); return PLIS_ERR_OOM; }
  for (uint64_t i = 0; i < n; ++i) {
    if (!getline_v(&t, '\n', &b, &e)) {
      free(out);
      set_error(std::string("snapshot ") + path + ": " + std::to_string(i) + " of " + std::to_string(n) + " subvolume lines");
      return PLIS_ERR_PARSE;
    }
    if (e > b && e[-1] == '\r') --e;
    int bad = 0;
    const long long k = for_tokens(b, e, [&](long long j, const char* tb, const char* te) {
      long long v;
      if (j >= (long long)ns || !int_at(tb, te, &v) || v < 0) { bad = 1; return false; }
      out[(size_t)j * n + i] = (uint32_t)v;  // species-major
      return true;
    });
    if (bad || k != (long long)ns) {
      free(out);
      set_error(std::string("snapshot ") + path + ": bad counts for subvolume " + std::to_string(i));
      return PLIS_ERR_PARSE;
    }
  }
  *n_out = (uint32_t)n;
  *s_out = (uint32_t)ns;
  *time_out = time;
  *counts_out = out;
  return PLIS_OK;
}

extern "C" int plis_write_snapshot(const char* path, const uint32_t* counts, uint32_t n, uint32_t s, double time) {
  if (!path || !counts) { set_error("null argument"); return PLIS_ERR_INVALID; }
  FILE* f = fopen(path, "w");
  if (!f) { set_error(std::string("cannot write ") + path); return PLIS_ERR_IO; }
  fprintf(f, "subvolumes=%u\nspecies=%u\ntime=%f\n\n", n, s, (double)(float)time);
  std::string line;
  char num[16];
  for (uint32_t i = 0; i < n; ++i) {
    line.clear();
    for (uint32_t j = 0; j < s; ++j) {
      int k = snprintf(num, sizeof num, "%d ", (int)counts[(size_t)j * n + i]);
      line.append(num, (size_t)k);
    }
    line.push_back('\n');
    fwrite(line.data(), 1, line.size(), f);
  }
  if (fclose(f) != 0) { set_error(std::string("cannot write ") + path); return PLIS_ERR_IO; }
  return PLIS_OK;
}

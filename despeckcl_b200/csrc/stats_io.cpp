// NL-SAR statistics collections: storage, the LUT builder and file I/O.
//
// A collection is the library-side equivalent of
// std::map<nlsar::params, nlsar::stats> (include/despeckcl.h:30 in the
// reference): entries ordered by (patch, scale), each with its LUTs.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "stats_internal.h"

struct dcl_stats_collection {
  std::map<std::pair<int, int>, dcl::OwnedStats> entries;
};

namespace dcl {

// ---------------------------------------------------------------------------
// chi-squared quantiles (replaces GSL's gsl_cdf_chisq_Pinv, called by the
// reference at src/compute/nlsar/stats.cpp:76)
// ---------------------------------------------------------------------------
//
// P(a, x), the regularised lower incomplete gamma function, by its series
// sum_n x^n / (a (a+1) ... (a+n)) for x < a+1 and through the complement's
// continued fraction (evaluated with the modified Lentz method) otherwise;
// see Abramowitz & Stegun 6.5.29 and 6.5.31.  The chi-squared CDF with nu
// degrees of freedom is P(nu/2, x/2); its inverse is found by Newton steps on
// the CDF, kept inside a bisection bracket.

static double lower_gamma_reg(double a, double x) {
  if (x <= 0.0) return 0.0;
  const double lpre = a * std::log(x) - x - std::lgamma(a);
  if (x < a + 1.0) {
    double term = 1.0 / a, sum = term;
    for (int n = 1; n < 100000; ++n) {
      term *= x / (a + n);
      sum += term;
      if (term < sum * 1e-17) break;
    }
    return std::exp(lpre) * sum;
  }
  // continued fraction of Q(a, x) = e^-x x^a / Gamma(a) * 1/(x+1-a- 1(1-a)/(x+3-a- ...))
  const double tiny = 1e-300;
  double b = x + 1.0 - a;
  double f = 1.0 / b, C = 1.0 / tiny, D = f;
  for (int i = 1; i < 100000; ++i) {
    const double an = -(double)i * (i - a);
    b += 2.0;
    D = an * D + b;
    D = (std::fabs(D) < tiny) ? 1.0 / tiny : 1.0 / D;
    C = b + an / C;
    if (std::fabs(C) < tiny) C = tiny;
    const double delta = C * D;
    f *= delta;
    if (std::fabs(delta - 1.0) < 1e-17) break;
  }
  return 1.0 - std::exp(lpre) * f;
}

double chi2_quantile(double p, double nu) {
  if (p <= 0.0) return 0.0;
  if (p >= 1.0) return std::numeric_limits<double>::infinity();
  const double k = nu / 2.0;
  double lo = 0.0, hi = std::max(1.0, nu);
  while (lower_gamma_reg(k, hi / 2.0) < p) hi *= 2.0;
  double x = 0.5 * (lo + hi);
  for (int it = 0; it < 300; ++it) {
    const double F = lower_gamma_reg(k, x / 2.0) - p;
    if (F < 0.0) lo = x;
    else hi = x;
    const double pdf = std::exp((k - 1.0) * std::log(x) - x / 2.0 - k * std::log(2.0) - std::lgamma(k));
    double nx = (pdf > 0.0) ? x - F / pdf : 0.5 * (lo + hi);
    if (!(nx > lo && nx < hi)) nx = 0.5 * (lo + hi);
    const bool done = std::fabs(nx - x) <= 1e-15 * x;
    x = nx;
    if (done) break;
  }
  return x;
}

// nlsar::stats::stats(dissims, lut_size) (src/compute/nlsar/stats.cpp:28-80).
// `sorted` holds the finite dissimilarities in ascending order.
OwnedStats stats_from_sorted(const std::vector<float>& sorted, unsigned L) {
  OwnedStats s;
  s.lut_size = L;
  s.dmin = sorted.front();
  s.dmax = sorted.back();
  const float step = (s.dmax - s.dmin) / L;
  s.quant.resize(L);
  for (size_t i = 0; i < L; ++i) {
    const float d = s.dmin + i * step;
    const auto it = std::lower_bound(sorted.begin(), sorted.end(), d);
    s.quant[i] = ((float)(it - sorted.begin())) / sorted.size();
  }
  s.chi2.resize(L);
  const float ystep = 1.0f / L;
  for (size_t i = 0; i + 1 < L; ++i) s.chi2[i] = (float)chi2_quantile((double)(i * ystep), 49.0);
  s.chi2[L - 1] = 100000;
  return s;
}

}  // namespace dcl

using dcl::OwnedStats;

dcl_stats_collection* dcl_collection_new() { return new dcl_stats_collection(); }

void dcl_collection_put(dcl_stats_collection* c, int patch, int scale, dcl::OwnedStats s) {
  c->entries[{patch, scale}] = std::move(s);
}

extern "C" int dcl_stats_collection_size(const dcl_stats_collection* c) { return c ? (int)c->entries.size() : 0; }

extern "C" int dcl_stats_collection_get(const dcl_stats_collection* c, int i, dcl_stats_entry* out) {
  if (!c || !out || i < 0 || i >= (int)c->entries.size())
    return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "stats collection index %d out of range", i);
  auto it = c->entries.begin();
  std::advance(it, i);
  out->patch_size = it->first.first;
  out->scale_size = it->first.second;
  out->lut_size = it->second.lut_size;
  out->dissims_min = it->second.dmin;
  out->dissims_max = it->second.dmax;
  out->quantilles = it->second.quant.data();
  out->chi2cdf_inv = it->second.chi2.data();
  return DCL_OK;
}

extern "C" dcl_stats_collection* dcl_stats_collection_from_entries(const dcl_stats_entry* e, int n) {
  if (!e || n < 0) {
    dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null entries");
    return nullptr;
  }
  dcl_stats_collection* c = new dcl_stats_collection();
  for (int i = 0; i < n; ++i) {
    OwnedStats s;
    s.lut_size = e[i].lut_size;
    s.dmin = e[i].dissims_min;
    s.dmax = e[i].dissims_max;
    if (e[i].quantilles) s.quant.assign(e[i].quantilles, e[i].quantilles + e[i].lut_size);
    if (e[i].chi2cdf_inv) s.chi2.assign(e[i].chi2cdf_inv, e[i].chi2cdf_inv + e[i].lut_size);
    c->entries[{e[i].patch_size, e[i].scale_size}] = std::move(s);
  }
  return c;
}

extern "C" void dcl_stats_collection_free(dcl_stats_collection* c) { delete c; }

extern "C" dcl_stats_collection* dcl_stats_from_dissims(int patch, int scale, const float* d, long n, unsigned L) {
  if (!d || n < 1 || L < 2) {
    dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "need dissimilarities and lut_size >= 2");
    return nullptr;
  }
  std::vector<float> v;
  v.reserve((size_t)n);
  for (long i = 0; i < n; ++i)
    if (std::isfinite(d[i])) v.push_back(d[i]);
  if (v.empty()) {
    dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "no finite dissimilarity");
    return nullptr;
  }
  std::sort(v.begin(), v.end());
  dcl_stats_collection* c = new dcl_stats_collection();
  c->entries[{patch, scale}] = dcl::stats_from_sorted(v, L);
  return c;
}

// ---------------------------------------------------------------------------
// files
// ---------------------------------------------------------------------------

static const char* kMagic = "despeckcl_b200-nlsar-stats";

extern "C" int dcl_stats_save(const dcl_stats_collection* c, const char* filename) {
  if (!c || !filename) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null collection or filename");
  FILE* f = std::fopen(filename, "w");
  if (!f) return dcl::set_error(DCL_ERR_IO, "cannot open %s for writing", filename);
  std::fprintf(f, "%s 1\n%zu\n", kMagic, c->entries.size());
  for (auto& kv : c->entries) {
    const OwnedStats& s = kv.second;
    std::fprintf(f, "%d %d %u %.9g %.9g\n", kv.first.first, kv.first.second, s.lut_size, s.dmin, s.dmax);
    for (size_t i = 0; i < s.quant.size(); ++i) std::fprintf(f, "%.9g%c", s.quant[i], i + 1 == s.quant.size() ? '\n' : ' ');
    for (size_t i = 0; i < s.chi2.size(); ++i) std::fprintf(f, "%.9g%c", s.chi2[i], i + 1 == s.chi2.size() ? '\n' : ' ');
  }
  const bool ok = std::fclose(f) == 0;
  return ok ? DCL_OK : dcl::set_error(DCL_ERR_IO, "error writing %s", filename);
}

// Boost text archives of std::map<nlsar::params, nlsar::stats>, the file the
// reference's store_nlsar_stats_collection writes
// (src/compute/nlsar/training/nlsar_training.cpp:99-104: a text_oarchive
// given the whole map).  Boost is not used; the layout follows
// Boost.Serialization's save rules for these types:
//
//   22 serialization::archive V         signature (length, text), format version
//   t v                                 class info of the map (tracking, version)
//   N i                                 element count, item version
//   first element:  t v                 class info of std::pair
//                   t v p s             class info of params, then
//                                       patch_size scale_size (parameters.h:51-55)
//                   t v L dmin dmax     class info of stats, then lut_size,
//                                       dissims_min, dissims_max (stats.h:43-50)
//                   L i q[0..L-1]       quantilles: count, item version, values
//                   L i c[0..L-1]       chi2cdf_inv, the same
//   later elements: p s L dmin dmax L i q[...] L i c[...]
//
// Class info (one tracking word and one class-version word) precedes only
// the first object of each class type; vectors of a primitive type carry
// none (Boost gives them the object_serializable level).  Objects that are
// never saved through a pointer are untracked, so every tracking word is 0
// and no object ids follow.  Format versions 3 and below have no item-version
// words; the layout is otherwise the same in every version.

namespace {

// A strict reader over the archive's whitespace-separated tokens.
struct BoostTokens {
  const std::vector<std::string>& tok;
  size_t k;
  bool ok = true;
  const char* what = nullptr;

  bool fail(const char* w) {
    if (ok) what = w;
    ok = false;
    return false;
  }
  bool next_long(long& out, const char* w) {
    if (!ok) return false;
    if (k >= tok.size()) return fail(w);
    const char* s = tok[k].c_str();
    char* end = nullptr;
    out = std::strtol(s, &end, 10);
    if (end == s || *end != '\0') return fail(w);
    ++k;
    return true;
  }
  bool next_float(float& out, const char* w) {
    if (!ok) return false;
    if (k >= tok.size()) return fail(w);
    const char* s = tok[k].c_str();
    char* end = nullptr;
    out = std::strtof(s, &end);
    if (end == s || *end != '\0') return fail(w);
    ++k;
    return true;
  }
  // tracking and class-version words of a class's first object
  bool class_info(const char* w) {
    long tracking = -1, version = -1;
    if (!next_long(tracking, w) || !next_long(version, w)) return false;
    if (tracking != 0) return fail("tracked objects (not written by a map of NL-SAR statistics)");
    if (version < 0) return fail(w);
    return true;
  }
  bool vec(std::vector<float>& v, long library_version, const char* w) {
    long n = -1, item_version = 0;
    if (!next_long(n, w)) return false;
    if (n < 0 || n > (1L << 24)) return fail(w);
    if (library_version > 3 && !next_long(item_version, w)) return false;
    v.resize((size_t)n);
    for (long i = 0; i < n && ok; ++i) next_float(v[(size_t)i], w);
    return ok;
  }
};

}  // namespace

static dcl_stats_collection* load_boost_text(const std::vector<std::string>& tok, const char* filename) {
  BoostTokens in{tok, 2};
  long version = -1, n = -1, item_version = 0;
  in.next_long(version, "archive format version");
  if (in.ok && version < 1) in.fail("archive format version");
  in.class_info("class info of the map");
  in.next_long(n, "element count");
  if (in.ok && n < 0) in.fail("element count");
  if (version > 3) in.next_long(item_version, "item version");
  dcl_stats_collection* c = new dcl_stats_collection();
  for (long e = 0; e < n && in.ok; ++e) {
    if (e == 0) {
      in.class_info("class info of the (params, stats) pair");
      in.class_info("class info of params");
    }
    long p = 0, s = 0, L = 0;
    in.next_long(p, "patch_size");
    in.next_long(s, "scale_size");
    if (e == 0) in.class_info("class info of stats");
    in.next_long(L, "lut_size");
    OwnedStats st;
    in.next_float(st.dmin, "dissims_min");
    in.next_float(st.dmax, "dissims_max");
    in.vec(st.quant, version, "quantilles");
    in.vec(st.chi2, version, "chi2cdf_inv");
    if (!in.ok) break;
    if (L < 0 || (size_t)L != st.quant.size() || (size_t)L != st.chi2.size()) {
      in.fail("lut_size against the table lengths");
      break;
    }
    st.lut_size = (unsigned)L;
    c->entries[{(int)p, (int)s}] = std::move(st);
  }
  if (in.ok && in.k != tok.size()) in.fail("trailing words after the last element");
  if (!in.ok) {
    delete c;
    dcl::set_error(DCL_ERR_IO, "%s: Boost text archive: bad or missing %s (word %zu)", filename, in.what, in.k);
    return nullptr;
  }
  return c;
}

extern "C" int dcl_stats_save_boost_text(const dcl_stats_collection* c, const char* filename) {
  if (!c || !filename) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null collection or filename");
  FILE* f = std::fopen(filename, "w");
  if (!f) return dcl::set_error(DCL_ERR_IO, "cannot open %s for writing", filename);
  // format version 10: Boost reads every version up to its own, and these
  // types are laid out the same from version 4 on
  std::fprintf(f, "22 serialization::archive 10 0 0 %zu 0", c->entries.size());
  bool first = true;
  for (auto& kv : c->entries) {
    const OwnedStats& s = kv.second;
    if (first) std::fprintf(f, " 0 0 0 0");
    std::fprintf(f, " %d %d", kv.first.first, kv.first.second);
    if (first) std::fprintf(f, " 0 0");
    std::fprintf(f, " %u %.9e %.9e", s.lut_size, s.dmin, s.dmax);
    // floats as Boost's text archive writes them: scientific, 9 digits after
    // the point (an exact round trip for every float)
    std::fprintf(f, " %zu 0", s.quant.size());
    for (float q : s.quant) std::fprintf(f, " %.9e", q);
    std::fprintf(f, " %zu 0", s.chi2.size());
    for (float q : s.chi2) std::fprintf(f, " %.9e", q);
    first = false;
  }
  std::fprintf(f, "\n");
  const bool ok = std::fclose(f) == 0;
  return ok ? DCL_OK : dcl::set_error(DCL_ERR_IO, "error writing %s", filename);
}

extern "C" dcl_stats_collection* dcl_stats_load(const char* filename) {
  if (!filename) {
    dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null filename");
    return nullptr;
  }
  std::ifstream in(filename);
  if (!in) {
    dcl::set_error(DCL_ERR_IO, "cannot open %s", filename);
    return nullptr;
  }
  std::vector<std::string> tok;
  std::string t;
  while (in >> t) tok.push_back(t);
  if (tok.size() >= 3 && tok[0] == kMagic) {
    if (tok[1] != "1") {
      dcl::set_error(DCL_ERR_IO, "%s: unsupported stats file version %s", filename, tok[1].c_str());
      return nullptr;
    }
    size_t k = 2;
    const long n = std::stol(tok[k++]);
    dcl_stats_collection* c = new dcl_stats_collection();
    try {
      for (long e = 0; e < n; ++e) {
        const int p = std::stoi(tok.at(k++)), s = std::stoi(tok.at(k++));
        OwnedStats st;
        st.lut_size = (unsigned)std::stoul(tok.at(k++));
        st.dmin = std::stof(tok.at(k++));
        st.dmax = std::stof(tok.at(k++));
        for (unsigned i = 0; i < st.lut_size; ++i) st.quant.push_back(std::stof(tok.at(k++)));
        for (unsigned i = 0; i < st.lut_size; ++i) st.chi2.push_back(std::stof(tok.at(k++)));
        c->entries[{p, s}] = std::move(st);
      }
    } catch (...) {
      delete c;
      dcl::set_error(DCL_ERR_IO, "%s: truncated or malformed stats file", filename);
      return nullptr;
    }
    return c;
  }
  if (tok.size() >= 2 && tok[0] == "22" && tok[1] == "serialization::archive") return load_boost_text(tok, filename);
  dcl::set_error(DCL_ERR_IO, "%s: not an NL-SAR statistics file", filename);
  return nullptr;
}

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

// Best-effort reader of a Boost text archive of std::map<nlsar::params,
// nlsar::stats> (fields serialised at include/compute/nlsar/parameters.h:51-55
// and stats.h:43-50 of the reference).  Boost inserts class-tracking and
// version numbers whose exact placement depends on the Boost version; this
// reader skips them by matching the shape "patch scale L min max L q[L] L c[L]"
// with an item-version word after each vector length (as modern Boost
// writes it), or without one.  Unverified against a real archive: Boost is
// not available to produce one.
static dcl_stats_collection* load_boost_text(const std::vector<std::string>& tok) {
  std::vector<double> v;
  for (size_t i = 0; i < tok.size(); ++i) {
    char* end = nullptr;
    const double x = std::strtod(tok[i].c_str(), &end);
    if (end && *end == '\0') v.push_back(x);
  }
  dcl_stats_collection* c = new dcl_stats_collection();
  size_t i = 0;
  auto is_int = [](double x) { return std::floor(x) == x; };
  while (i + 6 < v.size()) {
    bool matched = false;
    const double p = v[i], s = v[i + 1];
    if (is_int(p) && is_int(s) && p >= 1 && s >= 1 && ((long)p % 2) && ((long)s % 2)) {
      // up to two class-tracking / version words may sit between the key and
      // the stats fields, and one item-version word after each vector length
      for (int skip = 0; skip <= 2 && !matched; ++skip) {
        const size_t l0 = i + 2 + skip;
        if (l0 + 3 >= v.size()) break;
        bool small_ints = true;
        for (int k = 0; k < skip; ++k) small_ints = small_ints && is_int(v[i + 2 + k]) && v[i + 2 + k] >= 0 && v[i + 2 + k] <= 1;
        const double L = v[l0];
        if (!small_ints || !is_int(L) || L < 2 || L > 4096) continue;
        for (int iv1 = 1; iv1 >= 0 && !matched; --iv1) {
          size_t q0 = l0 + 3;
          if (q0 >= v.size() || v[q0] != L) continue;
          q0 += 1 + iv1;
          const size_t c0 = q0 + (size_t)L;
          for (int iv2 = 1; iv2 >= 0 && !matched; --iv2) {
            if (c0 >= v.size() || v[c0] != L) continue;
            const size_t cc = c0 + 1 + iv2;
            if (cc + (size_t)L > v.size()) continue;
            OwnedStats st;
            st.lut_size = (unsigned)L;
            st.dmin = (float)v[l0 + 1];
            st.dmax = (float)v[l0 + 2];
            for (size_t k = 0; k < (size_t)L; ++k) st.quant.push_back((float)v[q0 + k]);
            for (size_t k = 0; k < (size_t)L; ++k) st.chi2.push_back((float)v[cc + k]);
            c->entries[{(int)p, (int)s}] = std::move(st);
            i = cc + (size_t)L;
            matched = true;
          }
        }
      }
    }
    if (!matched) ++i;
  }
  if (c->entries.empty()) {
    delete c;
    dcl::set_error(DCL_ERR_IO, "no NL-SAR statistics found in the archive");
    return nullptr;
  }
  return c;
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
  if (tok.size() >= 2 && tok[1] == "serialization::archive") return load_boost_text(tok);
  dcl::set_error(DCL_ERR_IO, "%s: not an NL-SAR statistics file", filename);
  return nullptr;
}

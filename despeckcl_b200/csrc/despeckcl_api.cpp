// The drop-in C++ API (include/despeckcl.h) on top of the C ABI.
//
// Argument lists and the 0-on-success return follow the reference's
// include/despeckcl.h:30-95; logging follows the enabled_log_levels contract of
// src/utils/logging.cpp:28-56 with a small stderr logger.

#include "../../include/despeckcl.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "stats_internal.h"

namespace {

struct Logger {
  bool error = false, fatal = false, warning = false, info = false, debug = false;
  explicit Logger(const std::vector<std::string>& levels) {
    for (const std::string& l : levels) {
      if (l == "error") error = true;
      else if (l == "fatal") fatal = true;
      else if (l == "warning") warning = true;
      else if (l == "info") info = true;
      else if (l == "debug") debug = true;
    }
  }
};

int select_mode_from_env() {
  const char* s = std::getenv("DESPECKCL_B200_SELECT");
  if (s && (std::strcmp(s, "argmax_enl") == 0 || std::strcmp(s, "argmax") == 0)) return DCL_SELECT_ARGMAX_ENL;
  return DCL_SELECT_REFERENCE;
}

std::vector<dcl_stats_entry> entries_of(const nlsar_stats_collection& m) {
  std::vector<dcl_stats_entry> e;
  for (const auto& kv : m) {
    dcl_stats_entry x;
    x.patch_size = kv.first.patch_size;
    x.scale_size = kv.first.scale_size;
    x.lut_size = kv.second.lut_size;
    x.dissims_min = kv.second.dissims_min;
    x.dissims_max = kv.second.dissims_max;
    x.quantilles = kv.second.quantilles.data();
    x.chi2cdf_inv = kv.second.chi2cdf_inv.data();
    // a table shorter than lut_size cannot be indexed safely
    if (kv.second.quantilles.size() < x.lut_size || kv.second.chi2cdf_inv.size() < x.lut_size) x.lut_size = 0;
    e.push_back(x);
  }
  return e;
}

nlsar_stats_collection collection_of(dcl_stats_collection* c) {
  nlsar_stats_collection m;
  const int n = dcl_stats_collection_size(c);
  for (int i = 0; i < n; ++i) {
    dcl_stats_entry e;
    dcl_stats_collection_get(c, i, &e);
    nlsar::stats s;
    s.lut_size = e.lut_size;
    s.dissims_min = e.dissims_min;
    s.dissims_max = e.dissims_max;
    s.quantilles.assign(e.quantilles, e.quantilles + e.lut_size);
    s.chi2cdf_inv.assign(e.chi2cdf_inv, e.chi2cdf_inv + e.lut_size);
    m[nlsar::params{e.patch_size, e.scale_size}] = s;
  }
  return m;
}

int finish(const Logger& log, int rc, const char* what, std::chrono::steady_clock::time_point t0) {
  if (rc != DCL_OK) {
    if (log.error) std::fprintf(stderr, "[despeckcl_b200] ERROR %s: %s\n", what, dcl_last_error());
  } else if (log.info) {
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(stderr, "[despeckcl_b200] INFO filtering ran for %g secs\n", s);
  }
  return rc;
}

}  // namespace

nlsar::stats::stats() : lut_size(0), dissims_min(0.f), dissims_max(0.f) {}

nlsar::stats::stats(std::vector<float> dissims, unsigned int lut) : lut_size(lut) {
  // src/compute/nlsar/stats.cpp:28-38
  dissims.erase(std::remove_if(dissims.begin(), dissims.end(), [](float x) { return !std::isfinite(x); }),
                dissims.end());
  if (dissims.empty() || lut < 2) throw std::invalid_argument("nlsar::stats needs finite dissimilarities and lut_size >= 2");
  std::sort(dissims.begin(), dissims.end());
  const dcl::OwnedStats s = dcl::stats_from_sorted(dissims, lut);
  dissims_min = s.dmin;
  dissims_max = s.dmax;
  quantilles = s.quant;
  chi2cdf_inv = s.chi2;
}

int despeckcl::boxcar(float* a1, float* a2, float* phi, float* ref, float* phase, float* coh, const int height,
                      const int width, const int window_width, std::vector<std::string> levels) {
  const Logger log(levels);
  const auto t0 = std::chrono::steady_clock::now();
  return finish(log, dcl_boxcar(a1, a2, phi, ref, phase, coh, height, width, window_width), "boxcar", t0);
}

int despeckcl::nlinsar(float* a1, float* a2, float* phi, float* ref, float* phase, float* coh, const int height,
                       const int width, const int search_window_size, const int patch_size, const int niter,
                       const int lmin, std::vector<std::string> levels) {
  const Logger log(levels);
  const auto t0 = std::chrono::steady_clock::now();
  return finish(log,
                dcl_nlinsar(a1, a2, phi, ref, phase, coh, height, width, search_window_size, patch_size, niter, lmin),
                "nlinsar", t0);
}

int despeckcl::goldstein(float* a1, float* a2, float* phi, float* ref, float* phase, float* coh,
                         const unsigned int height, const unsigned int width, const unsigned int patch_size,
                         const unsigned int overlap, const float alpha, std::vector<std::string> levels) {
  const Logger log(levels);
  const auto t0 = std::chrono::steady_clock::now();
  if (height > 0x7fffffffu || width > 0x7fffffffu || patch_size > 0x7fffffffu || overlap > 0x7fffffffu)
    return finish(log, dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "dimensions out of range"), "goldstein", t0);
  return finish(log,
                dcl_goldstein(a1, a2, phi, ref, phase, coh, (int)height, (int)width, (int)patch_size, (int)overlap,
                              alpha),
                "goldstein", t0);
}

int despeckcl::nlsar(float* a1, float* a2, float* phi, float* ref, float* phase, float* coh, const int height,
                     const int width, const int sws, const std::vector<int> patch_sizes,
                     const std::vector<int> scale_sizes, std::map<nlsar::params, nlsar::stats> nlsar_stats,
                     const float h_param, const float c_param, std::vector<std::string> levels) {
  const Logger log(levels);
  const auto t0 = std::chrono::steady_clock::now();
  const std::vector<dcl_stats_entry> e = entries_of(nlsar_stats);
  const int rc = dcl_nlsar_insar(a1, a2, phi, ref, phase, coh, height, width, sws, patch_sizes.data(),
                                 (int)patch_sizes.size(), scale_sizes.data(), (int)scale_sizes.size(), e.data(),
                                 (int)e.size(), h_param, c_param, select_mode_from_env());
  return finish(log, rc, "nlsar", t0);
}

int despeckcl::nlsar(float* covmat_raw, float* covmat_filt, const int height, const int width, const int dim,
                     const int sws, const std::vector<int> patch_sizes, const std::vector<int> scale_sizes,
                     std::map<nlsar::params, nlsar::stats> nlsar_stats, const float h_param, const float c_param,
                     std::vector<std::string> levels) {
  const Logger log(levels);
  const auto t0 = std::chrono::steady_clock::now();
  const std::vector<dcl_stats_entry> e = entries_of(nlsar_stats);
  const int rc = dcl_nlsar_covmat(covmat_raw, covmat_filt, height, width, dim, sws, patch_sizes.data(),
                                  (int)patch_sizes.size(), scale_sizes.data(), (int)scale_sizes.size(), e.data(),
                                  (int)e.size(), h_param, c_param, select_mode_from_env());
  return finish(log, rc, "nlsar", t0);
}

nlsar_stats_collection despeckcl::nlsar_training(float* a1, float* a2, float* phi, const int height, const int width,
                                                 const std::vector<int> patch_sizes,
                                                 const std::vector<int> scale_sizes, std::vector<std::string> levels) {
  const Logger log(levels);
  dcl_stats_collection* c = dcl_nlsar_training_insar(a1, a2, phi, height, width, patch_sizes.data(),
                                                     (int)patch_sizes.size(), scale_sizes.data(),
                                                     (int)scale_sizes.size());
  if (!c) {
    if (log.error) std::fprintf(stderr, "[despeckcl_b200] ERROR nlsar_training: %s\n", dcl_last_error());
    throw std::runtime_error(std::string("nlsar_training: ") + dcl_last_error());
  }
  nlsar_stats_collection m = collection_of(c);
  dcl_stats_collection_free(c);
  return m;
}

nlsar_stats_collection despeckcl::nlsar_training(float* covmat_raw, const int height, const int width, const int dim,
                                                 const std::vector<int> patch_sizes,
                                                 const std::vector<int> scale_sizes, std::vector<std::string> levels) {
  const Logger log(levels);
  dcl_stats_collection* c = dcl_nlsar_training_covmat(covmat_raw, height, width, dim, patch_sizes.data(),
                                                      (int)patch_sizes.size(), scale_sizes.data(),
                                                      (int)scale_sizes.size());
  if (!c) {
    if (log.error) std::fprintf(stderr, "[despeckcl_b200] ERROR nlsar_training: %s\n", dcl_last_error());
    throw std::runtime_error(std::string("nlsar_training: ") + dcl_last_error());
  }
  nlsar_stats_collection m = collection_of(c);
  dcl_stats_collection_free(c);
  return m;
}

void despeckcl::store_nlsar_stats_collection(nlsar_stats_collection nsc, std::string filename) {
  const std::vector<dcl_stats_entry> e = entries_of(nsc);
  dcl_stats_collection* c = dcl_stats_collection_from_entries(e.data(), (int)e.size());
  // the reference's file: a Boost text archive of the map
  const int rc = c ? dcl_stats_save_boost_text(c, filename.c_str()) : DCL_ERR_INVALID_ARGUMENT;
  dcl_stats_collection_free(c);
  if (rc != DCL_OK) throw std::runtime_error(std::string("store_nlsar_stats_collection: ") + dcl_last_error());
}

nlsar_stats_collection despeckcl::load_nlsar_stats_collection(std::string filename) {
  dcl_stats_collection* c = dcl_stats_load(filename.c_str());
  if (!c) throw std::runtime_error(std::string("load_nlsar_stats_collection: ") + dcl_last_error());
  nlsar_stats_collection m = collection_of(c);
  dcl_stats_collection_free(c);
  return m;
}

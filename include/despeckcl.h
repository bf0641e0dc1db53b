/* Drop-in C++ API of despeckCL's NL-SAR path on the B200 engine.
 *
 * Same declarations as the reference's include/despeckcl.h:30-95 for the
 * functions implemented here (nlsar x2, nlsar_training x2,
 * store/load_nlsar_stats_collection, boxcar, goldstein, nlinsar).  Every function returns 0 on
 * success like the reference; on failure it returns the negative dcl_status of
 * despeckcl_b200.h (the reference terminates the process instead) and logs the
 * message at the "error" level.
 *
 * Per-pixel (patch, scale) selection defaults to the reference's behaviour
 * (the last key of the statistics map, src/compute/nlsar/best_params.cpp:27-54);
 * set DESPECKCL_B200_SELECT=argmax_enl to select by the largest bias-reduced
 * ENL instead. */
#ifndef DESPECKCL_B200_DESPECKCL_H
#define DESPECKCL_B200_DESPECKCL_H

#include <map>
#include <string>
#include <vector>

#include "nlsar/parameters.h"
#include "nlsar/stats.h"

typedef std::map<nlsar::params, nlsar::stats> nlsar_stats_collection;

namespace despeckcl {
int boxcar(float* ampl_master, float* ampl_slave, float* phase, float* ref_filt, float* phase_filt, float* coh_filt,
           const int height, const int width, const int window_width, std::vector<std::string> enabled_log_levels);

int nlinsar(float* ampl_master, float* ampl_slave, float* phase, float* ref_filt, float* phase_filt, float* coh_filt,
            const int height, const int width, const int search_window_size, const int patch_size, const int niter,
            const int lmin, std::vector<std::string> enabled_log_levels);

int goldstein(float* ampl_master, float* ampl_slave, float* phase, float* ref_filt, float* phase_filt,
              float* coh_filt, const unsigned int height, const unsigned int width, const unsigned int patch_size,
              const unsigned int overlap, const float alpha, std::vector<std::string> enabled_log_levels);

int nlsar(float* ampl_master, float* ampl_slave, float* phase, float* ref_filt, float* phase_filt, float* coh_filt,
          const int height, const int width, const int search_window_size, const std::vector<int> patch_sizes,
          const std::vector<int> scale_sizes, std::map<nlsar::params, nlsar::stats> nlsar_stats, const float h_param,
          const float c_param, std::vector<std::string> enabled_log_levels);

int nlsar(float* covmat_raw, float* covmat_filt, const int height, const int width, const int dim,
          const int search_window_size, const std::vector<int> patch_sizes, const std::vector<int> scale_sizes,
          std::map<nlsar::params, nlsar::stats> nlsar_stats, const float h_param, const float c_param,
          std::vector<std::string> enabled_log_levels);

nlsar_stats_collection nlsar_training(float* ampl_master, float* ampl_slave, float* phase, const int height,
                                      const int width, const std::vector<int> patch_sizes,
                                      const std::vector<int> scale_sizes, std::vector<std::string> enabled_log_levels);

nlsar_stats_collection nlsar_training(float* covmat_raw, const int height, const int width, const int dim,
                                      const std::vector<int> patch_sizes, const std::vector<int> scale_sizes,
                                      std::vector<std::string> enabled_log_levels);

void store_nlsar_stats_collection(nlsar_stats_collection nsc, std::string filename);
nlsar_stats_collection load_nlsar_stats_collection(std::string filename);
}  // namespace despeckcl

#endif

// Internal representation of NL-SAR statistics (library side).
#pragma once

#include <vector>

#include "../../include/despeckcl_b200.h"

namespace dcl {

// nlsar::stats (include/compute/nlsar/stats.h:28-55 in the reference) with owned tables.
struct OwnedStats {
  unsigned lut_size = 0;
  float dmin = 0.f, dmax = 0.f;
  std::vector<float> quant, chi2;
};

// The chi-squared quantile function (inverse CDF) with nu degrees of freedom.
double chi2_quantile(double p, double nu);

// LUTs of nlsar::stats from finite dissimilarities sorted ascending.
OwnedStats stats_from_sorted(const std::vector<float>& sorted, unsigned lut_size);

// Sorts npairs device dissimilarities (dis -> dis2) and returns the finite
// ones on the host, ascending.
int sort_dissims(float* dis, float* dis2, long long npairs, std::vector<float>& sorted);

}  // namespace dcl

dcl_stats_collection* dcl_collection_new();
void dcl_collection_put(dcl_stats_collection* c, int patch, int scale, dcl::OwnedStats s);

namespace dcl {
// nlsar_training on a 3x3 covariance image [18][H][W] (host pointer).
dcl_stats_collection* training_covmat3(const float* cov18, int H, int W, const int* patches, int np,
                                       const int* scales, int ns);
}  // namespace dcl

/* nlsar::stats: the dissimilarity LUTs of one (patch, scale) combination, with
 * the members of the reference's include/compute/nlsar/stats.h:28-55
 * (lut_size, dissims_min, dissims_max, quantilles, chi2cdf_inv).  The
 * constructor from dissimilarities builds the LUTs as
 * src/compute/nlsar/stats.cpp:28-80 does. */
#ifndef DESPECKCL_B200_NLSAR_STATS_H
#define DESPECKCL_B200_NLSAR_STATS_H

#include <vector>

namespace nlsar {
class stats {
 public:
  stats();
  stats(std::vector<float> dissims, unsigned int lut_size);
  unsigned int lut_size;
  float dissims_min;
  float dissims_max;
  std::vector<float> quantilles;
  std::vector<float> chi2cdf_inv;
};
}  // namespace nlsar

#endif

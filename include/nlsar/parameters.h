/* nlsar::params: the (patch size, scale size) key of an NL-SAR statistics
 * collection, ordered lexicographically.  Same members and ordering as the
 * reference's include/compute/nlsar/parameters.h:26-57 (the ordering defines
 * which key the reference's per-pixel selection returns); no Boost
 * dependency. */
#ifndef DESPECKCL_B200_NLSAR_PARAMETERS_H
#define DESPECKCL_B200_NLSAR_PARAMETERS_H

namespace nlsar {
struct params {
  int patch_size;
  int scale_size;

  bool operator==(const params& other) const {
    return patch_size == other.patch_size && scale_size == other.scale_size;
  }
  bool operator<(const params& other) const {
    return (patch_size < other.patch_size) || ((patch_size == other.patch_size) && (scale_size < other.scale_size));
  }
};
}  // namespace nlsar

#endif

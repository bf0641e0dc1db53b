// TEST INFRASTRUCTURE ONLY.  A C-ABI shim over the few reference translation
// units that compile without OpenCL, GSL or Boost (sim_measures.h,
// best_params.cpp, best_alpha_copy.cpp, tile_iterator.cpp, sub_images.cpp,
// optimal_tiling.cpp).  The Makefile in this directory compiles those files in
// place from the reference tree into _ref/libref_pieces.so; the tests use it to
// pin the oracle's restatement of the same functions.
#include <map>
#include <vector>

#include "best_alpha_copy.h"
#include "best_params.h"
#include "optimal_tiling.h"
#include "sim_measures.h"
#include "sub_images.h"
#include "tile_iterator.h"

extern "C" float ref_pixel_similarity_2x2(float a00, float a01r, float a01i, float a11, float b00, float b01r,
                                          float b01i, float b11) {
  return pixel_similarity_2x2(a00, a01r, a01i, a11, b00, b01r, b01i, b11, 1);
}

// a, b: {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12}
extern "C" float ref_pixel_similarity_3x3(const float* a, const float* b) {
  return pixel_similarity_3x3(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], b[0], b[1], b[2], b[3], b[4], b[5],
                              b[6], b[7], b[8], 1);
}

extern "C" float ref_det_covmat_3x3(const float* a) {
  return det_covmat_3x3(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
}

// keys[2*i] = patch, keys[2*i+1] = scale; enl[i*n + j]; out[2*j] = chosen key
extern "C" void ref_get_best_params(const int* keys, int nkeys, const float* enl, int n, int* out) {
  std::map<nlsar::params, std::vector<float>> m;
  for (int i = 0; i < nkeys; ++i)
    m[nlsar::params{keys[2 * i], keys[2 * i + 1]}] = std::vector<float>(enl + (size_t)i * n, enl + (size_t)(i + 1) * n);
  const std::vector<nlsar::params> b = nlsar::get_best_params(m);
  for (int j = 0; j < n; ++j) {
    out[2 * j] = b[j].patch_size;
    out[2 * j + 1] = b[j].scale_size;
  }
}

extern "C" int ref_tile_list(int H, int W, int th, int tw, int ov, int* h0, int* w0, int cap) {
  int n = 0;
  for (auto t : tile_iterator(H, W, th, tw, ov, ov)) {
    if (n < cap) {
      h0[n] = t[0].start;
      w0[n] = t[1].start;
    }
    ++n;
  }
  return n;
}

extern "C" void ref_get_sub_image(const float* img, int H, int W, int dim, int h0, int w0, int sh, int sw,
                                  float* out) {
  auto s = get_sub_image(img, H, W, dim, h0, w0, sh, sw);
  for (long i = 0; i < (long)dim * sh * sw; ++i) out[i] = s[i];
}

extern "C" void ref_write_sub_image(float* img, int H, int W, int dim, float* sub, int h0, int w0, int sh, int sw,
                                    int ov) {
  write_sub_image(img, H, W, dim, sub, h0, w0, sh, sw, ov);
}

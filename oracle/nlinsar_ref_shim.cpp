// TEST INFRASTRUCTURE ONLY.  despeckCL's NL-InSAR run on the CPU from the
// reference's own code where it compiles here: the device kernels without
// work-group barriers (precompute_similarities_1st_pass.cl.in configured like
// CMake does, precompute_similarities_2nd_pass.cl, compute_weights.cl,
// common/cl_kernels/compute_number_of_looks.cl, precompute_filter_values.cl)
// compiled as C++ behind emulated work-item ids, the host smoothing step
// (smoothing.cpp, over oracle/ref_stub/CL/cl.hpp) and the tiling
// (tile_iterator.cpp, sub_images.cpp).  The two kernels that depend on
// work-group barriers (precompute_patch_similarities.cl,
// compute_insar.cl) and the transpose are restated here with the same
// summation order.  The driver follows nlinsar_sub_image.cpp:32-250 and
// nlinsar.cpp:42-130.  The tests use this library to pin the restatement in
// nlinsar_oracle.cpp.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

#include "smoothing.h"
#include "sub_images.h"
#include "tile_iterator.h"

namespace refnl {

// The kernels are evaluated with OpenCL's float pi (sim_measures.h falls back to
// the double M_PI only when compiled as host C++).
// Float overloads of the math functions, as OpenCL's built-ins on float.
#define M_PI_F ((float)M_PI)
using std::asin;
using std::atan2;
using std::cos;
using std::exp;
using std::fabs;
using std::isinf;
using std::isnan;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;

thread_local int g_gid[3];
inline int get_global_id(int d) { return g_gid[d]; }
inline int get_group_id(int d) { return g_gid[d]; }
inline int get_local_size(int) { return 1; }
inline int get_local_id(int) { return 0; }

#define __kernel static
#define __global
#include "precompute_similarities_1st_pass.cl"
#include "precompute_similarities_2nd_pass.cl"
#include "compute_weights.cl"
#include "compute_number_of_looks.cl"
#include "precompute_filter_values.cl"
#undef __kernel
#undef __global

constexpr int kBlock = 16;  // nlinsar::kernel_params{sws, p, 16} (nlinsar.cpp:90)

template <typename F>
void ndrange2(int o0, int g0, int o1, int g1, F f) {
  for (int j = o1; j < o1 + g1; ++j)
    for (int i = o0; i < o0 + g0; ++i) {
      g_gid[0] = i;
      g_gid[1] = j;
      f();
    }
}

inline int rounded(int n) { return kBlock * ((n - 1) / kBlock + 1); }

// precompute_patch_similarities.cl: rows (second index) summed first, then the
// row sums down the first index
void patch_sums(const float* in, float* out, int hori, int wori, int p, int nplanes) {
  const int hs = hori + p - 1, ws = wori + p - 1;
  for (int z = 0; z < nplanes; ++z)
    for (int x = 0; x < hori; ++x)
      for (int y = 0; y < wori; ++y) {
        float sum = 0;
        for (int ky = 0; ky < p; ++ky) sum += in[(size_t)z * hs * ws + (size_t)x * ws + y + ky];
        for (int kx = 1; kx < p; ++kx) {
          float r = 0;
          for (int ky = 0; ky < p; ++ky) r += in[(size_t)z * hs * ws + (size_t)(x + kx) * ws + y + ky];
          sum += r;
        }
        out[(size_t)z * hori * wori + (size_t)x * wori + y] = sum;
      }
}

float correct_phase(float phi) {
  if (phi > (float)M_PI) phi -= 2.0f * (float)M_PI;
  if (phi < -(float)M_PI) phi += 2.0f * (float)M_PI;
  return phi;
}

bool valid(float v) { return !(std::isnan(v) || std::isinf(v) || v == 0); }

void sub_image(float* t, int HO, int sws, int p, int lmin, float h, float T) {
  const int psh = (p - 1) / 2, wsh = (sws - 1) / 2, ov = wsh + psh;
  const size_t n2 = (size_t)HO * HO;
  float *a1 = t, *a2 = t + n2, *dp = t + 2 * n2, *rf = t + 3 * n2, *pf = t + 4 * n2, *cf = t + 5 * n2;
  const int hsws = HO - p + 1, hsim = HO - sws + 1, hori = HO - 2 * ov, no = sws * sws;
  std::vector<float> sims((size_t)no * hsim * hsim), kls((size_t)no * hsim * hsim);
  const int border_max = wsh;
  ndrange2(0, rounded(hsim), 0, rounded(hsim), [&] {
    precompute_similarities_1st_pass(a1, a2, dp, rf, pf, cf, sims.data(), kls.data(), HO, HO, border_max, sws);
  });
  if (hsim > border_max && hsim > 2 * border_max)
    ndrange2(border_max, kBlock * ((hsim - 1 - border_max) / kBlock + 1), border_max,
             kBlock * ((hsim - 1 - 2 * border_max) / kBlock + 1),
             [&] { precompute_similarities_2nd_pass(sims.data(), kls.data(), HO, HO, border_max, sws); });
  const size_t nori = (size_t)no * hori * hori;
  std::vector<float> psim(nori), pkl(nori), w(nori);
  patch_sums(sims.data(), psim.data(), hori, hori, p, no);
  patch_sums(kls.data(), pkl.data(), hori, hori, p, no);
  for (size_t i = 0; i < nori; ++i) {
    g_gid[0] = (int)i;
    compute_weights(psim.data(), pkl.data(), w.data(), (int)nori, h, T);
  }
  std::fill(w.begin() + (size_t)(sws * wsh + wsh) * hori * hori, w.begin() + (size_t)(sws * wsh + wsh + 1) * hori * hori,
            0.0f);
  std::vector<float> nols((size_t)hori * hori);
  ndrange2(0, rounded(hori), 0, rounded(hori),
           [&] { compute_number_of_looks(w.data(), nols.data(), hori, hori, sws); });
  std::vector<float> wt(nori);  // transpose.cl: [offset][pixel] -> [pixel][offset]
  for (int k = 0; k < no; ++k)
    for (int i = 0; i < hori * hori; ++i) wt[(size_t)i * no + k] = w[(size_t)k * hori * hori + i];
  cl::CommandQueue q;
  nlinsar::smoothing sm;
  sm.run(q, cl::Buffer(wt.data()), cl::Buffer(nols.data()), a1, hori, hori, sws, p, lmin);
  std::vector<float> fa((size_t)hsws * hsws), fr((size_t)hsws * hsws), fi((size_t)hsws * hsws);
  ndrange2(0, rounded(hsws), 0, rounded(hsws),
           [&] { precompute_filter_values(a1, a2, dp, fa.data(), fr.data(), fi.data(), HO, HO, p); });
  // compute_insar.cl:68-102
  for (int x = 0; x < hori; ++x)
    for (int y = 0; y < hori; ++y) {
      float N = 0, A = 0, Xr = 0, Xi = 0;
      for (int i = 0; i < sws; ++i)
        for (int j = 0; j < sws; ++j) {
          const float wgt = wt[((size_t)x * hori + y) * no + i * sws + j];
          const size_t f = (size_t)(x + i) * hsws + (y + j);
          N += wgt;
          A += wgt * fa[f];
          Xr += wgt * fr[f];
          Xi += wgt * fi[f];
        }
      const float refl = A / N, phi = std::atan2(Xi, Xr), coh = std::sqrt(std::pow(Xr, 2.0f) + std::pow(Xi, 2.0f)) / A;
      const size_t o = (size_t)(x + ov) * HO + (y + ov);
      if (valid(refl)) rf[o] = refl;
      if (valid(phi)) pf[o] = correct_phase(phi);
      if (valid(coh)) cf[o] = std::min(1.0f, std::max(0.0f, coh));
    }
}

}  // namespace refnl

// despeckcl::nlinsar (nlinsar.cpp:42-130) for patch sizes 3 and 7; ref / phase
// / coh hold the initial estimates on entry and the results on exit.
extern "C" int ref_nlinsar(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                           int H, int W, int sws, int p, int niter, int lmin) {
  if (p != 3 && p != 7) return -1;
  const int ov = (p - 1) / 2 + (sws - 1) / 2;
  const int area = p * p;
  const float h_theo = p == 3 ? 0.58f : 0.244f;
  const float h = h_theo * area;
  const float T = 2.0 / h * M_PI / 4 * area;
  const size_t n = (size_t)H * W;
  std::vector<float> img(6 * n);
  std::copy(a1, a1 + n, img.begin());
  std::copy(a2, a2 + n, img.begin() + n);
  std::copy(phi, phi + n, img.begin() + 2 * n);
  std::copy(ref, ref + n, img.begin() + 3 * n);
  std::copy(phase, phase + n, img.begin() + 4 * n);
  std::copy(coh, coh + n, img.begin() + 5 * n);
  const int HO = 80;
  for (int it = 0; it < niter; ++it) {
    std::vector<float> next(img);
    for (auto t : tile_iterator(H, W, HO, HO, ov, ov)) {
      auto tile = get_sub_image(img.data(), H, W, 6, t[0].start, t[1].start, HO, HO);
      refnl::sub_image(tile.get(), HO, sws, p, lmin, h, T);
      const int cs = HO - 2 * ov;
      std::vector<float> crop(6 * (size_t)cs * cs);
      for (int d = 0; d < 6; ++d)
        for (int y = 0; y < cs; ++y)
          for (int x = 0; x < cs; ++x)
            crop[((size_t)d * cs + y) * cs + x] = tile[(size_t)d * HO * HO + (size_t)(y + ov) * HO + (x + ov)];
      write_sub_image(next.data(), H, W, 6, crop.data(), t[0].start + ov, t[1].start + ov, cs, cs, 0);
    }
    img.swap(next);
  }
  std::copy(img.begin() + 3 * n, img.begin() + 4 * n, ref);
  std::copy(img.begin() + 4 * n, img.begin() + 5 * n, phase);
  std::copy(img.begin() + 5 * n, img.begin() + 6 * n, coh);
  return 0;
}

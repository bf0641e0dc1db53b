// TEST INFRASTRUCTURE ONLY.  The reference's Goldstein device kernels
// (src/compute/goldstein/cl_kernels/{raw_interferogram,patches_unpack,
// weighted_multiply,patches_pack,slc2real}.cl) are OpenCL C that is also
// valid C++ once the address-space qualifiers and get_global_id are supplied;
// the Makefile compiles them here, in place from the reference tree, and this
// file drives them the way goldstein_filter_sub_image.cpp:120-186 and the
// wrappers in src/compute/goldstein/cl_wrappers/*.cpp launch them (one
// emulated work item at a time, NDRange sizes as in the wrappers, the pack
// kernel's four parity launches of patches_pack.cpp:48-77), with the
// reference's tiling (tile_iterator.cpp, sub_images.cpp, map_filter_tiles.h).
// clFFT is not available: a double-precision radix-2 transform rounded to
// float stands in for it (forward unnormalised, backward scaled by 1/p^2, the
// convention goldstein_patch_ft_test.cpp pins).  The tests use this library to
// pin the oracle restatement in goldstein_oracle.cpp.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <vector>

#include "sub_images.h"
#include "tile_iterator.h"

namespace refcl {

using std::atan2;
using std::cos;
using std::fabs;
using std::pow;
using std::sin;
using std::sqrt;

thread_local int g_gid[2];
inline int get_global_id(int d) { return g_gid[d]; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }

#define __kernel static
#define __global
#include "raw_interferogram.cl"
#include "patches_unpack.cl"
#include "weighted_multiply.cl"
#include "patches_pack.cl"
#include "slc2real.cl"
#undef __kernel
#undef __global

constexpr int kBlock = 16;  // goldstein::kernel_params kp{16} (goldstein.cpp:67)

inline int rounded(int n) { return kBlock * ((n - 1) / kBlock + 1); }

template <typename F>
void ndrange(int g0, int g1, F f) {
  for (int j = 0; j < g1; ++j)
    for (int i = 0; i < g0; ++i) {
      g_gid[0] = i;
      g_gid[1] = j;
      f();
    }
}

void fft1(std::complex<double>* a, int n, int stride, bool inverse) {
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i * stride], a[j * stride]);
  }
  for (int len = 2; len <= n; len <<= 1)
    for (int k = 0; k < len / 2; ++k) {
      const double ang = 2.0 * M_PI * k / len * (inverse ? 1.0 : -1.0);
      const std::complex<double> w(std::cos(ang), std::sin(ang));
      for (int i = 0; i < n; i += len) {
        const std::complex<double> u = a[(i + k) * stride], v = a[(i + k + len / 2) * stride] * w;
        a[(i + k) * stride] = u + v;
        a[(i + k + len / 2) * stride] = u - v;
      }
    }
}

// goldstein_patch_ft.cpp: every p x p patch of the (height x width) planar buffer
void patch_ft(float* re, float* im, int height, int width, int p, bool inverse) {
  std::vector<std::complex<double>> q((size_t)p * p);
  for (int ph = 0; ph < height / p; ++ph)
    for (int pw = 0; pw < width / p; ++pw) {
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c) {
          const size_t i = (size_t)(ph * p + r) * width + pw * p + c;
          q[r * p + c] = std::complex<double>(re[i], im[i]);
        }
      for (int r = 0; r < p; ++r) fft1(&q[r * p], p, 1, inverse);
      for (int c = 0; c < p; ++c) fft1(&q[c], p, p, inverse);
      const double sc = inverse ? 1.0 / (p * p) : 1.0;
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c) {
          const size_t i = (size_t)(ph * p + r) * width + pw * p + c;
          re[i] = (float)(q[r * p + c].real() * sc);
          im[i] = (float)(q[r * p + c].imag() * sc);
        }
    }
}

// goldstein_filter_sub_image.cpp:27-187 on one tile; a1 and phase are
// overwritten with the amplitude and phase results as on the device.
void filter_sub_image(float* a1, float* a2, float* phase, float* ref_out, float* phase_out, int height, int width,
                      int p, int ov, float alpha) {
  const int npw = width / (p - 2 * ov), nph = height / (p - 2 * ov);
  const int ht = p * nph, wt = p * npw;
  std::vector<float> ir((size_t)height * width), ii((size_t)height * width);
  std::vector<float> tr((size_t)ht * wt), ti((size_t)ht * wt);
  ndrange(rounded(width), rounded(height),
          [&] { raw_interferogram(a1, a2, phase, ir.data(), ii.data(), height, width); });
  ndrange(rounded(wt), rounded(ht), [&] { patches_unpack(ir.data(), ii.data(), tr.data(), ti.data(), ht, wt, p, ov); });
  patch_ft(tr.data(), ti.data(), ht, wt, p, false);
  ndrange(rounded(wt), rounded(ht), [&] { weighted_multiply(tr.data(), ti.data(), ht, wt, alpha); });
  patch_ft(tr.data(), ti.data(), ht, wt, p, true);
  const std::pair<int, int> offsets[4] = {{0, 0}, {0, p}, {p, 0}, {p, p}};
  for (auto o : offsets) {
    const int gx = p * ((wt - o.first - 1) / (2 * p) + 1);
    const int gy = p * ((ht - o.second - 1) / (2 * p) + 1);
    ndrange(gx, gy, [&] { patches_pack(tr.data(), ti.data(), ir.data(), ii.data(), ht, wt, p, ov, o.first, o.second); });
  }
  ndrange(rounded(width), rounded(height), [&] { slc2real(ir.data(), ii.data(), a1, phase, height, width); });
  std::copy(a1, a1 + (size_t)height * width, ref_out);
  std::copy(phase, phase + (size_t)height * width, phase_out);
}

}  // namespace refcl

// despeckcl::goldstein (goldstein.cpp:39-106) for scenes that are one tile:
// planes a1, a2, phase, ref, phase_filt, coh as the insar_data of the call;
// ref/phase/coh hold the caller's buffers on entry.  Returns -1 when the tile
// holds fewer than two patches per side (the pack launches then read outside
// the patch grid, patches_pack.cpp:67-69).
extern "C" int ref_goldstein(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                             int H, int W, int p, int ov, float alpha) {
  const int s = p - 2 * ov;
  const int m = std::max(H + 2 * ov, W + 2 * ov);
  const int side = m - m % s + s;  // goldstein::round_up (tile_size.cpp:27-36)
  if (side / s < 2) return -1;
  const size_t n = (size_t)H * W;
  std::vector<float> img(6 * n);
  std::copy(a1, a1 + n, img.begin());
  std::copy(a2, a2 + n, img.begin() + n);
  std::copy(phi, phi + n, img.begin() + 2 * n);
  std::copy(ref, ref + n, img.begin() + 3 * n);
  std::copy(phase, phase + n, img.begin() + 4 * n);
  std::copy(coh, coh + n, img.begin() + 5 * n);
  for (auto t : tile_iterator(H, W, side, side, ov, ov)) {
    const int h0 = t[0].start, w0 = t[1].start;
    auto tile = get_sub_image(img.data(), H, W, 6, h0, w0, side, side);
    const size_t tn = (size_t)side * side;
    float* tp = tile.get();
    refcl::filter_sub_image(tp, tp + tn, tp + 2 * tn, tp + 3 * tn, tp + 4 * tn, side, side, p, ov, alpha);
    // the filter overwrote the device copies only; the tile's input planes are the host copies
    auto fresh = get_sub_image(img.data(), H, W, 3, h0, w0, side, side);
    std::copy(fresh.get(), fresh.get() + 3 * tn, tp);
    const int cs = side - 2 * ov;
    std::vector<float> crop(6 * (size_t)cs * cs);
    for (int d = 0; d < 6; ++d)
      for (int y = 0; y < cs; ++y)
        for (int x = 0; x < cs; ++x)
          crop[((size_t)d * cs + y) * cs + x] = tp[(size_t)d * tn + (size_t)(y + ov) * side + (x + ov)];
    write_sub_image(img.data(), H, W, 6, crop.data(), h0 + ov, w0 + ov, cs, cs, 0);
  }
  std::copy(img.begin() + 3 * n, img.begin() + 4 * n, ref);
  std::copy(img.begin() + 4 * n, img.begin() + 5 * n, phase);
  std::copy(img.begin() + 5 * n, img.begin() + 6 * n, coh);
  return 0;
}

// The reference's pack kernel alone (patches_pack.cpp:48-77) onto a packed
// buffer the caller initialises; the pack test of the reference
// (patches_pack_test.cpp:36-86) relies on a fresh device buffer reading zero.
extern "C" void ref_goldstein_pack(const float* ur, const float* ui, float* pr, float* pi, int hu, int wu, int p,
                                   int ov) {
  const std::pair<int, int> offsets[4] = {{0, 0}, {0, p}, {p, 0}, {p, p}};
  for (auto o : offsets) {
    const int gx = p * ((wu - o.first - 1) / (2 * p) + 1);
    const int gy = p * ((hu - o.second - 1) / (2 * p) + 1);
    refcl::ndrange(gx, gy, [&] {
      refcl::patches_pack(const_cast<float*>(ur), const_cast<float*>(ui), pr, pi, hu, wu, p, ov, o.first, o.second);
    });
  }
}

extern "C" void ref_goldstein_unpack(const float* pr, const float* pi, float* ur, float* ui, int hu, int wu, int p,
                                     int ov) {
  refcl::ndrange(refcl::rounded(wu), refcl::rounded(hu), [&] {
    refcl::patches_unpack(const_cast<float*>(pr), const_cast<float*>(pi), ur, ui, hu, wu, p, ov);
  });
}

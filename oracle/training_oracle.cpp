// NL-SAR TRAINING ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of despeckCL's nlsar_training path (paths relative to the
// reference project root):
//   covmat from (a1,a2,phi)  src/data/data.cpp:60-89
//   get_dissims              src/compute/nlsar/training/get_dissims.cpp:32-117
//                            (rescale, spatial average with s_max = s)
//   get_all_patches          src/compute/nlsar/training/patches.cpp:32-41
//                            (tile_iterator with overlap 0, clamp padding)
//   dissimilarity            src/compute/nlsar/training/patches.cpp:43-94
//   get_all_dissim_combs     src/compute/nlsar/training/combinations.cpp:26-41
//   get_stats                src/compute/nlsar/training/get_stats.cpp:25-59 (lut_size 256,
//                            keys in patch-outer, scale-inner order)
//   stats                    src/compute/nlsar/stats.cpp:28-80
//
// The chi-squared inverse CDF replaces GSL's gsl_cdf_chisq_Pinv (the
// reference calls it at stats.cpp:76, GSL version unpinned): the regularised
// lower incomplete gamma function P(a, x) by its power series for x < a + 1
// and by the modified-Lentz continued fraction for the upper function
// otherwise (Press et al., Numerical Recipes, 3rd ed., section 6.2), inverted
// by safeguarded Newton iteration inside a bisection bracket.  Its values are
// pinned against scipy.stats.chi2.ppf in the tests.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "oracle.h"

namespace {

double gamma_p_series(double a, double x) {
  double ap = a, sum = 1.0 / a, del = sum;
  for (int n = 0; n < 10000; ++n) {
    ap += 1.0;
    del *= x / ap;
    sum += del;
    if (std::fabs(del) < std::fabs(sum) * 1e-17) break;
  }
  return sum * std::exp(-x + a * std::log(x) - std::lgamma(a));
}

double gamma_q_cf(double a, double x) {
  const double tiny = 1e-300;
  double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
  for (int i = 1; i < 10000; ++i) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (std::fabs(d) < tiny) d = tiny;
    c = b + an / c;
    if (std::fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (std::fabs(del - 1.0) < 1e-17) break;
  }
  return std::exp(-x + a * std::log(x) - std::lgamma(a)) * h;
}

double gamma_p(double a, double x) {
  if (x <= 0) return 0.0;
  if (x < a + 1.0) return gamma_p_series(a, x);
  return 1.0 - gamma_q_cf(a, x);
}

double chi2_cdf(double x, double nu) { return x <= 0 ? 0.0 : gamma_p(nu / 2, x / 2); }

double chi2_pdf(double x, double nu) {
  if (x <= 0) return 0.0;
  const double k = nu / 2;
  return std::exp((k - 1) * std::log(x) - x / 2 - k * std::log(2.0) - std::lgamma(k));
}

double chi2_inv(double y, double nu) {
  if (y <= 0) return 0.0;
  if (y >= 1) return std::numeric_limits<double>::infinity();
  double lo = 0, hi = nu;
  while (chi2_cdf(hi, nu) < y) hi *= 2;
  double x = 0.5 * (lo + hi);
  for (int it = 0; it < 200; ++it) {
    const double f = chi2_cdf(x, nu) - y;
    if (f < 0) lo = x; else hi = x;
    const double p = chi2_pdf(x, nu);
    double xn = (p > 0) ? x - f / p : 0.5 * (lo + hi);
    if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
    if (std::fabs(xn - x) <= 1e-15 * std::fabs(x)) { x = xn; break; }
    x = xn;
  }
  return x;
}

// covariance image [2*d*d][h][w], d = 2 or 3
struct Cov {
  int h, w, d;
  std::vector<float> v;
  float& at(int p, int y, int x) { return v[((size_t)p * h + y) * w + x]; }
  float at(int p, int y, int x) const { return v[((size_t)p * h + y) * w + x]; }
};

inline float det2(float e00, float e01r, float e01i, float e11) {
  return (e00 * e11) - (e01r * e01r + e01i * e01i);
}

inline float glr(float a00, float a01r, float a01i, float a11, float b00, float b01r, float b01i, float b11) {
  // sim_measures.h:37-65
  const float nom1 = det2(a00, a01r, a01i, a11);
  const float nom2 = det2(b00, b01r, b01i, b11);
  const float det = det2(a00 + b00, a01r + b01r, a01i + b01i, a11 + b11);
  float sim = -1 * (2 * 2 * std::log(2.0f) + std::log(nom1) + std::log(nom2) - 2 * std::log(det));
  if (std::isnan(sim)) sim = 0;
  return sim;
}

inline float det3(float a00, float a11, float a22, float a01r, float a01i, float a02r, float a02i, float a12r,
                  float a12i) {
  // sim_measures.h:66-97
  return a00 * a11 * a22 - a00 * (a12r * a12r + a12i * a12i) - a11 * (a02r * a02r + a02i * a02i) -
         a22 * (a01r * a01r + a01i * a01i) +
         2 * (a01r * a12r * a02r - a01i * a12i * a02r + a01r * a12i * a02i + a01i * a12r * a02i);
}

// a, b: {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12} (sim_measures.h:100-160)
inline float glr3(const float* a, const float* b) {
  const float nom1 = det3(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
  const float nom2 = det3(b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8]);
  const float det = det3(a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3], a[4] + b[4], a[5] + b[5], a[6] + b[6],
                         a[7] + b[7], a[8] + b[8]);
  float sim = -1 * (2 * 3 * std::log(2.0f) + std::log(nom1) + std::log(nom2) - 2 * std::log(det));
  if (std::isnan(sim)) sim = 0;
  return sim;
}

Cov rescaled_avg(const float* cov, int H, int W, int dim, int s) {
  // get_dissims.cpp:84-100: rescale in place (covmat_rescale.cl: every
  // off-diagonal element times (1/dim)^0.33333), then spatial average with
  // scale_size_max = scale_size
  const int npl = 2 * dim * dim;
  Cov r{H, W, dim, std::vector<float>(cov, cov + (size_t)npl * H * W)};
  const float gamma = std::pow(std::min(1.0f / dim, 1.0f), 0.33333f);
  for (int row = 0; row < dim; ++row)
    for (int col = 0; col < dim; ++col) {
      if (row == col) continue;
      for (int pl = 2 * (row * dim + col); pl <= 2 * (row * dim + col) + 1; ++pl)
        for (size_t i = 0; i < (size_t)H * W; ++i) r.v[(size_t)pl * H * W + i] *= gamma;
    }
  const int ssh = (s - 1) / 2;
  std::vector<float> g;
  for (int x = -ssh; x <= ssh; ++x)
    for (int y = -ssh; y <= ssh; ++y)
      g.push_back((float)std::exp(-M_PI * (x * x + y * y) / std::pow((double)((float)ssh + 0.5f), 2.0)));
  float K = 0;
  for (float e : g) K += e;
  for (float& e : g) e = e / K;
  Cov o{H - s + 1, W - s + 1, dim, std::vector<float>((size_t)npl * (H - s + 1) * (W - s + 1))};
  for (int pl = 0; pl < npl; ++pl)
    for (int y = 0; y < o.h; ++y)
      for (int x = 0; x < o.w; ++x) {
        float sum = 0;
        for (int kx = 0; kx < s; ++kx)
          for (int ky = 0; ky < s; ++ky) sum += g[kx * s + ky] * r.at(pl, y + kx, x + ky);
        o.at(pl, y, x) = sum;
      }
  return o;
}

std::vector<float> dissims_of(const float* cov, int H, int W, int dim, int p, int s) {
  const Cov a = rescaled_avg(cov, H, W, dim, s);
  // patches.cpp:32-41: tile_iterator(h, w, p, p, 0, 0), clamp padding.  Each
  // patch pixel keeps the planes its similarity reads (patches.cpp:70-136):
  // 2x2 {0, 2, 3, 6}, 3x3 {0, 8, 16, 2, 3, 4, 5, 10, 11}
  static const int pl2[4] = {0, 2, 3, 6};
  static const int pl3[9] = {0, 8, 16, 2, 3, 4, 5, 10, 11};
  const int nv = dim == 2 ? 4 : 9;
  const int* pl = dim == 2 ? pl2 : pl3;
  std::vector<std::vector<float>> patches;
  for (int h0 = 0; h0 < a.h; h0 += p)
    for (int w0 = 0; w0 < a.w; w0 += p) {
      std::vector<float> P;
      for (int y = 0; y < p; ++y)
        for (int x = 0; x < p; ++x) {
          const int yy = std::min(a.h - 1, std::max(0, h0 + y));
          const int xx = std::min(a.w - 1, std::max(0, w0 + x));
          for (int k = 0; k < nv; ++k) P.push_back(a.at(pl[k], yy, xx));
        }
      patches.push_back(std::move(P));
    }
  // combinations.cpp:26-41: head = last patch against all earlier ones
  std::vector<float> d;
  const size_t n = patches.size();
  d.reserve(n * (n - 1) / 2);
  for (size_t hi = n; hi-- > 1;) {
    const std::vector<float>& head = patches[hi];
    for (size_t j = 0; j < hi; ++j) {
      const std::vector<float>& o = patches[j];
      float sum = 0.0f;
      for (size_t i = 0; i < head.size(); i += nv)
        sum += dim == 2 ? glr(head[i], head[i + 1], head[i + 2], head[i + 3], o[i], o[i + 1], o[i + 2], o[i + 3])
                        : glr3(&head[i], &o[i]);
      d.push_back(sum);
    }
  }
  return d;
}

void stats_of(std::vector<float> d, unsigned L, float* dmin, float* dmax, float* quant, float* chi) {
  // stats.cpp:28-38, 51-80
  d.erase(std::remove_if(d.begin(), d.end(), [](float x) { return std::isnan(x) || std::isinf(x); }), d.end());
  std::sort(d.begin(), d.end());
  const float mn = *std::min_element(d.begin(), d.end());
  const float mx = *std::max_element(d.begin(), d.end());
  *dmin = mn;
  *dmax = mx;
  const float step = (mx - mn) / L;
  for (size_t i = 0; i < L; ++i) {
    const float dis = mn + i * step;
    const auto it = std::lower_bound(d.begin(), d.end(), dis);
    quant[i] = ((float)(it - d.begin())) / d.size();
  }
  const float ystep = 1.0f / L;
  for (size_t i = 0; i + 1 < L; ++i) {
    const float y = i * ystep;
    chi[i] = (float)chi2_inv((double)y, 49.0);
  }
  chi[L - 1] = 100000;
}

}  // namespace

extern "C" double oracle_chi2_inv(double y, double nu) { return chi2_inv(y, nu); }

extern "C" long oracle_training_dissims(const float* cov, int H, int W, int dim, int patch, int scale, float* out,
                                        long cap) {
  if (dim < 2 || dim > 3) return -1;
  const std::vector<float> d = dissims_of(cov, H, W, dim, patch, scale);
  if (out) std::copy(d.begin(), d.begin() + std::min<long>(cap, (long)d.size()), out);
  return (long)d.size();
}

extern "C" int oracle_stats_from_dissims(const float* dissims, long n, unsigned lut_size, float* dmin,
                                         float* dmax, float* quantilles, float* chi2cdf_inv) {
  std::vector<float> d(dissims, dissims + n);
  stats_of(std::move(d), lut_size, dmin, dmax, quantilles, chi2cdf_inv);
  return 0;
}

extern "C" int oracle_nlsar_training_insar(const float* a1, const float* a2, const float* ph, int H, int W,
                                           const int* patches, int np, const int* scales, int ns,
                                           int* out_patch, int* out_scale, float* out_dmin, float* out_dmax,
                                           float* out_quant, float* out_chi2) {
  // data.cpp:60-89: host covariance build
  std::vector<float> cov((size_t)8 * H * W);
  const size_t n = (size_t)H * W;
  for (size_t i = 0; i < n; ++i) {
    const float re = a1[i] * a2[i] * std::cos(ph[i]);
    const float im = a1[i] * a2[i] * std::sin(ph[i]);
    cov[i] = a1[i] * a1[i];
    cov[n + i] = 0;
    cov[2 * n + i] = re;
    cov[3 * n + i] = im;
    cov[4 * n + i] = re;
    cov[5 * n + i] = -im;
    cov[6 * n + i] = a2[i] * a2[i];
    cov[7 * n + i] = 0;
  }
  int k = 0;
  for (int pi = 0; pi < np; ++pi)
    for (int si = 0; si < ns; ++si, ++k) {
      const std::vector<float> d = dissims_of(cov.data(), H, W, 2, patches[pi], scales[si]);
      out_patch[k] = patches[pi];
      out_scale[k] = scales[si];
      stats_of(d, 256, out_dmin + k, out_dmax + k, out_quant + (size_t)k * 256, out_chi2 + (size_t)k * 256);
    }
  return k;
}

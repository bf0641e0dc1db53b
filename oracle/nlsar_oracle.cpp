// NL-SAR ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of despeckCL's NL-SAR path (the OpenCL kernels plus the
// host orchestration), templated on the arithmetic type so that it runs as an
// FP32 "reference-faithful" build and as an FP64 "truth" build.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and
// only as the checker or the timed CPU baseline.  The product path never
// calls it.
//
// Every stage follows a reference file (paths relative to the reference
// project root) and keeps its index conventions, summation order and special
// cases (NaN->0 similarities, LUT truncation, self weight 1, clamp padding,
// clamped tile write-back):
//   covmat_create       src/compute/nlsar/cl_kernels/covmat_create.cl:19-56
//   covmat_rescale      src/compute/nlsar/cl_kernels/covmat_rescale.cl:19-41
//   gen_gauss           src/compute/nlsar/cl_wrappers/covmat_spatial_avg.cpp:35-50
//   covmat_spatial_avg  src/compute/nlsar/cl_kernels/covmat_spatial_avg.cl:19-63
//   pixel similarities  src/compute/nlsar/cl_kernels/compute_pixel_similarities_2x2.cl.in:21-75
//                       quadrants: src/compute/nlsar/cl_wrappers/compute_pixel_similarities_2x2.cpp:61-79
//   GLR measure         src/compute/nlsar/sim_measures.h:31-65
//   patch sums          src/compute/nlsar/cl_kernels/patch_similarities_row_pass.cl:19-71,
//                       src/compute/nlsar/cl_kernels/patch_similarities_col_pass.cl:19-70
//   weights             src/compute/nlsar/cl_kernels/compute_weights.cl:19-56
//   symmetric copy      src/compute/nlsar/cl_kernels/copy_symm_weights.cl:19-78
//   self weight         src/compute/nlsar/routines/routines.cpp:151-157
//   statistics          src/compute/nlsar/cl_kernels/compute_nl_statistics.cl:23-104
//   alphas              src/compute/nlsar/cl_kernels/compute_alphas.cl:19-44
//   bias-reduced ENL    src/compute/nlsar/cl_kernels/compute_enls_nobias.cl:19-39
//   selection           src/compute/nlsar/best_params.cpp:27-54 (reference mode),
//                       ENL argmax (documented NL-SAR behaviour)
//   weighted means      src/compute/nlsar/cl_kernels/weighted_means.cl:19-83
//   decompose           src/compute/nlsar/cl_kernels/covmat_decompose.cl:19-39
//   per-tile pipeline   src/compute/nlsar/nlsar_filter_sub_image.cpp:146-390
//   overlap             src/compute/nlsar/nlsar.cpp:41-51
//   tiling              src/compute/common/map_filter_tiles.h:69-96,
//                       src/data/tile_iterator.cpp:48-75, src/data/sub_images.cpp:23-69
//   training            src/compute/nlsar/training/{get_dissims,patches,combinations,get_stats}.cpp
//   LUTs                src/compute/nlsar/stats.cpp:28-80
//
// Compiled with -ffp-contract=off so that the FP32 build performs exactly the
// float operations written here, in the order written.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

namespace {

using std::size_t;

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

// OpenCL's float max/min on a NaN operand return the other operand on every
// implementation we target (fmax semantics); the reference relies on that in
// compute_weights.cl:43-44 and compute_alphas.cl:37.
template <typename T> inline T cl_max(T a, T b) { return std::fmax(a, b); }
template <typename T> inline T cl_min(T a, T b) { return std::fmin(a, b); }

template <typename T> inline T det2(T e00, T e01r, T e01i, T e11) {
  // sim_measures.h:31-34
  return (e00 * e11) - (e01r * e01r + e01i * e01i);
}

template <typename T>
inline T det3(T a00, T a11, T a22, T a01r, T a01i, T a02r, T a02i, T a12r, T a12i) {
  // sim_measures.h:66-97 (Leibniz formula of a Hermitian 3x3 matrix)
  return a00 * a11 * a22 - a00 * (a12r * a12r + a12i * a12i) - a11 * (a02r * a02r + a02i * a02i) -
         a22 * (a01r * a01r + a01i * a01i) +
         2 * (a01r * a12r * a02r - a01i * a12i * a02r + a01r * a12i * a02i + a01i * a12r * a02i);
}

// Pixel similarity of two Hermitian 3x3 matrices given by their 9 unique
// reals {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12}
// (sim_measures.h:100-160, nlooks = 1, dimensions = 3).
template <typename T> inline T glr_3x3(const T* a, const T* b) {
  const T nom1 = det3<T>(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8]);
  const T nom2 = det3<T>(b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7], b[8]);
  const T det = det3<T>(a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3], a[4] + b[4], a[5] + b[5], a[6] + b[6],
                        a[7] + b[7], a[8] + b[8]);
  const T two = T(2);
  T sim = -T(1) * (T(2 * 3) * std::log(two) + std::log(nom1) + std::log(nom2) - two * std::log(det));
  if (std::isnan(sim)) sim = T(0);
  return sim;
}

template <typename T>
inline T glr_2x2(T a00, T a01r, T a01i, T a11, T b00, T b01r, T b01i, T b11) {
  // sim_measures.h:37-65, nlooks = 1, dimensions = 2
  const T nom1 = det2<T>(a00, a01r, a01i, a11);
  const T nom2 = det2<T>(b00, b01r, b01i, b11);
  const T det = det2<T>(a00 + b00, a01r + b01r, a01i + b01i, a11 + b11);
  const T two = T(2);
  T sim = -T(1) * (T(2 * 2) * std::log(two) + std::log(nom1) + std::log(nom2) -
                   two * std::log(det));
  if (std::isnan(sim)) sim = T(0);
  return sim;
}

// A covariance tile: 2*d*d planes [2*d*d][h][w] (d = 2 or 3), plane
// 2*(r*d+c) the real and 2*(r*d+c)+1 the imaginary part of element (r, c)
// (covmat_create.cl:44-54 layout).
template <typename T> struct Cov {
  int h = 0, w = 0, d = 2, np = 8;
  std::vector<T> v;
  Cov() = default;
  Cov(int hh, int ww, int dd = 2) : h(hh), w(ww), d(dd), np(2 * dd * dd), v((size_t)2 * dd * dd * hh * ww) {}
  T& at(int plane, int y, int x) { return v[((size_t)plane * h + y) * w + x]; }
  T at(int plane, int y, int x) const { return v[((size_t)plane * h + y) * w + x]; }
  // real plane of element (r, c)
  int plane(int r, int c) const { return 2 * (r * d + c); }
};

// Pixel similarity of the covariance at (ay, ax) of `ca` and (by, bx) of `cb`
// (compute_pixel_similarities_{2x2,3x3}.cl.in: upper-triangle planes only).
template <typename T> T glr_at(const Cov<T>& ca, int ay, int ax, const Cov<T>& cb, int by, int bx) {
  if (ca.d == 2)
    return glr_2x2<T>(ca.at(0, ay, ax), ca.at(2, ay, ax), ca.at(3, ay, ax), ca.at(6, ay, ax), cb.at(0, by, bx),
                      cb.at(2, by, bx), cb.at(3, by, bx), cb.at(6, by, bx));
  // a00, a11, a22, a01, a02, a12 (planes 0, 8, 16, 2/3, 4/5, 10/11)
  static const int pl[9] = {0, 8, 16, 2, 3, 4, 5, 10, 11};
  T a[9], b[9];
  for (int i = 0; i < 9; ++i) {
    a[i] = ca.at(pl[i], ay, ax);
    b[i] = cb.at(pl[i], by, bx);
  }
  return glr_3x3<T>(a, b);
}

// ---------------------------------------------------------------------------
// stages
// ---------------------------------------------------------------------------

template <typename T>
Cov<T> covmat_create(const float* a1, const float* a2, const float* ph, int h, int w) {
  // covmat_create.cl:19-56
  Cov<T> c(h, w);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x;
      const T am = a1[i], as = a2[i], p = ph[i];
      const T e00 = am * am;
      const T e01r = am * as * std::cos(p);
      const T e01i = am * as * std::sin(p);
      const T e11 = as * as;
      c.at(0, y, x) = e00;
      c.at(1, y, x) = T(0);
      c.at(2, y, x) = e01r;
      c.at(3, y, x) = e01i;
      c.at(4, y, x) = e01r;
      c.at(5, y, x) = -e01i;
      c.at(6, y, x) = e11;
      c.at(7, y, x) = T(0);
    }
  return c;
}

template <typename T> T rescale_gamma(int dim = 2) {
  // covmat_rescale.cl:25-26 with nlooks = 1
  const T LD = T(1) / T(dim);
  return std::pow(std::min(LD, T(1)), T(0.33333f));
}

template <typename T> void covmat_rescale(Cov<T>& c) {
  // covmat_rescale.cl:31-39: both planes of every off-diagonal element times gamma
  const T g = rescale_gamma<T>(c.d);
  for (int r = 0; r < c.d; ++r)
    for (int col = 0; col < c.d; ++col) {
      if (r == col) continue;
      for (int pl = c.plane(r, col); pl <= c.plane(r, col) + 1; ++pl)
        for (int y = 0; y < c.h; ++y)
          for (int x = 0; x < c.w; ++x) c.at(pl, y, x) *= g;
    }
}

template <typename T> std::vector<T> gen_gauss(int s) {
  // cl_wrappers/covmat_spatial_avg.cpp:35-50.  The reference evaluates the
  // exponent in double, stores float, normalises with a float sum.
  std::vector<T> g;
  const int ssh = (s - 1) / 2;
  for (int x = -ssh; x <= ssh; ++x)
    for (int y = -ssh; y <= ssh; ++y) {
      const double den = std::pow((double)((float)ssh + 0.5f), 2.0);
      g.push_back((T)std::exp(-M_PI * (x * x + y * y) / den));
    }
  T K = T(0);
  for (T e : g) K += e;
  for (T& e : g) e = e / K;
  return g;
}

template <typename T> Cov<T> covmat_spatial_avg(const Cov<T>& in, int s, int smax) {
  // covmat_spatial_avg.cl:19-63: output (h-smax+1)x(w-smax+1); output pixel i
  // averages input rows delta+i .. delta+i+s-1 with delta = (smax-s)/2.
  const int delta = (smax - s) / 2;
  const int ho = in.h - smax + 1, wo = in.w - smax + 1;
  const std::vector<T> g = gen_gauss<T>(s);
  Cov<T> out(ho, wo, in.d);
  for (int pl = 0; pl < in.np; ++pl)
    for (int y = 0; y < ho; ++y)
      for (int x = 0; x < wo; ++x) {
        T sum = T(0);
        for (int kx = 0; kx < s; ++kx)
          for (int ky = 0; ky < s; ++ky)
            sum += g[kx * s + ky] * in.at(pl, delta + y + kx, delta + x + ky);
        out.at(pl, y, x) = sum;
      }
  return out;
}

// Per-combination results for one tile core.
template <typename T> struct ComboResult {
  std::vector<T> enl_nobias, alpha, wsum;
  std::vector<T> mean8;       // every plane's sum(w*C) over the core
  std::vector<T> bin_margin;  // FP64 diagnostics: min distance of a LUT index to a bin edge
  std::vector<T> var_cond;    // FP64 diagnostics: min over d of |var_d| / I_d^2 (alpha conditioning)
  std::vector<T> kappa;       // FP64 diagnostics: sum w|C01| / |sum w C01| (cancellation in the complex mean)
};

struct LutView {
  unsigned lut_size;
  float dmin, dmax;
  const float* quant;
  const float* chi2;
};

// The composite weight of a first-stage LUT index k (compute_weights.cl:49-51).
template <typename T> T weight_of_index(unsigned k, const LutView& L, T hpar, T cpar) {
  const T quantile = (T)L.quant[k];
  const T x = (T)L.chi2[(unsigned)(quantile * (T)(int)(L.lut_size - 1))];
  return std::exp(-std::fabs(x - cpar) / hpar);
}

// compute_weights.cl:38-54.  With `margin` set, also records how far (in LUT
// index units) the dissimilarity lies from the nearest boundary at which the
// weight would change: a neighbouring bin with a different weight, or the
// d > dmax cut-off.
template <typename T>
T lut_weight(T dissim, const LutView& L, T hpar, T cpar, T* margin) {
  const T span = (T)L.dmax - (T)L.dmin;
  const T scale = (T)(int)(L.lut_size - 1);
  if (dissim > (T)L.dmax) {
    if (margin) *margin = std::min(*margin, (dissim - (T)L.dmax) / span * scale);
    return T(0);
  }
  T d = cl_max<T>(dissim, (T)L.dmin);
  d = cl_min<T>(d, (T)L.dmax);
  const T mapped = (d - (T)L.dmin) / span * scale;
  const unsigned k = (unsigned)mapped;
  const T w = weight_of_index<T>(k, L, hpar, cpar);
  if (margin) {
    const T fr = mapped - (T)k;
    T m = std::numeric_limits<T>::infinity();
    if (k >= 1 && weight_of_index<T>(k - 1, L, hpar, cpar) != w) m = std::min(m, fr);
    if (k + 1 < L.lut_size - 1 && weight_of_index<T>(k + 1, L, hpar, cpar) != w) m = std::min(m, T(1) - fr);
    // distance to the cut-off above which the weight is 0
    m = std::min(m, ((T)L.dmax - dissim) / span * scale);
    *margin = std::min(*margin, m);
  }
  return w;
}

struct FilterParams {
  int sws;
  std::vector<int> patches;  // as given by the caller (deduplicated)
  std::vector<int> scales;
  std::map<std::pair<int, int>, LutView> stats;  // key (patch, scale)
  double h, c;
  int select_mode;  // 0 = reference (last key of the stats map), 1 = ENL argmax
  int want_diag;
};

// Output of one tile: 8 filtered planes on the core plus diagnostics.
template <typename T> struct TileOut {
  int hc = 0, wc = 0;
  std::vector<T> cov8;       // [2*d*d][hc][wc]
  std::vector<int> sel;      // selected combo index (loop order: scale outer, patch inner)
  std::vector<T> bin_margin, enl_margin, var_cond, kappa, bin_margin_all;
};

// Patch sums of U pixel-similarity planes (height_sim x width_sim each) for
// patch size p within the largest patch pmax: the row pass then the column
// pass, each summing 2*psh+1 terms in order from 0
// (patch_similarities_row_pass.cl:43-70, patch_similarities_col_pass.cl:43-69).
// Output: U planes of (height_sim - pmax + 1) x (width_sim - pmax + 1).
template <typename T>
void patch_sums(const T* pix, int U, int Hsym, int Wo, int p, int pmax, std::vector<T>& inter, T* patch) {
  const int psh = (p - 1) / 2, off = (pmax - p) / 2, Psh = (pmax - 1) / 2;
  const int Hps = Hsym - pmax + 1, Wps = Wo - pmax + 1;
  const int Hi = Hsym - 2 * off, Wi = Wps;
  inter.assign((size_t)U * Hi * Wi, T(0));
  for (int z = 0; z < U; ++z)
    for (int y = 0; y < Hi; ++y)
      for (int x = 0; x < Wi; ++x) {
        T sum = T(0);
        for (int k = -psh; k <= psh; ++k) sum += pix[((size_t)z * Hsym + off + y) * Wo + Psh + x + k];
        inter[((size_t)z * Hi + y) * Wi + x] = sum;
      }
  for (int z = 0; z < U; ++z)
    for (int y = 0; y < Hps; ++y)
      for (int x = 0; x < Wps; ++x) {
        T sum = T(0);
        for (int k = -psh; k <= psh; ++k) sum += inter[((size_t)z * Hi + psh + y + k) * Wi + x];
        patch[((size_t)z * Hps + y) * Wps + x] = sum;
      }
}

// The index map of the symmetric expansion (copy_symm_weights.cl:39-77): for
// every output pixel (hc x wc) and non-centre window offset, f(dst, src) with
// dst the index into the full window [sws*sws][hc][wc] and src the index into
// the upper half window [U][Hps][Wps] it copies.
template <typename F> void symm_index_map(int hc, int wc, int sws, int Hps, int Wps, F f) {
  const int wsh = (sws - 1) / 2, U = sws * wsh + wsh;
  const size_t nc = (size_t)hc * wc;
  for (int y = 0; y < hc; ++y)
    for (int x = 0; x < wc; ++x) {
      const size_t o = (size_t)y * wc + x;
      for (int i = 0; i < U; ++i) f((size_t)i * nc + o, ((size_t)i * Hps + y) * Wps + x + wsh);
      for (int hh = wsh; hh < sws; ++hh) {
        const int ww0 = (hh == wsh) ? wsh + 1 : 0;
        for (int ww = ww0; ww < sws; ++ww) {
          const int hs = y + hh - wsh, ws = wsh + x + ww - wsh;
          const int hhs = sws - hh - 1, wws = sws - ww - 1;
          f((size_t)(hh * sws + ww) * nc + o, ((size_t)(hhs * sws + wws) * Hps + hs) * Wps + ws);
        }
      }
    }
}

// nlsar_filter_sub_image.cpp:146-390 for one padded tile `ori`.
template <typename T> TileOut<T> filter_tile(const Cov<T>& ori, const FilterParams& P) {
  const int sws = P.sws, wsh = (sws - 1) / 2;
  const int pmax = *std::max_element(P.patches.begin(), P.patches.end());
  const int smax = *std::max_element(P.scales.begin(), P.scales.end());
  const int Psh = (pmax - 1) / 2, Ssh = (smax - 1) / 2;
  const int Ho = ori.h - smax + 1, Wo = ori.w - smax + 1;  // height/width_overlap
  const int ov = wsh + Psh;
  const int hc = Ho - 2 * ov, wc = Wo - 2 * ov;  // height/width_ori
  const int N = sws * sws, U = sws * wsh + wsh;
  const int Hsym = Ho - wsh;  // pixel-similarity volume height
  const int Hps = Hsym - pmax + 1, Wps = Wo - pmax + 1;  // patch-similarity volume
  TileOut<T> out;
  out.hc = hc;
  out.wc = wc;
  if (hc <= 0 || wc <= 0) return out;
  const size_t nc = (size_t)hc * wc;

  Cov<T> resc = ori;
  covmat_rescale<T>(resc);

  // combos in the reference loop order: scale outer, patch inner (:449-470)
  struct Combo { int p, s; };
  std::vector<Combo> combos;
  for (int s : P.scales)
    for (int p : P.patches) combos.push_back({p, s});
  const int nco = (int)combos.size();
  std::vector<ComboResult<T>> res(nco);

  std::vector<T> pix((size_t)U * Hsym * Wo);
  std::vector<T> inter, patch((size_t)U * Hps * Wps), wsym((size_t)U * Hps * Wps);
  std::vector<T> wfull((size_t)N * nc);
  std::vector<T> wmargin;

  int idx = 0;
  for (int s : P.scales) {
    const Cov<T> cs = covmat_spatial_avg<T>(resc, s, smax);
    // pixel similarities, both quadrant launches (compute_pixel_similarities_2x2.cpp:61-79)
    std::fill(pix.begin(), pix.end(), std::numeric_limits<T>::quiet_NaN());
    auto quadrant = [&](int hh0, int hh1, int ww0, int ww1, int w_lo) {
      for (int hh = hh0; hh < hh1; ++hh)
        for (int ww = ww0; ww < ww1; ++ww)
          for (int y = 0; y < Hsym; ++y)
            for (int x = w_lo; x < Wo; ++x) {
              const int cy = y + wsh, cx = x;
              const int wy = cy - wsh + hh, wx = cx - wsh + ww;
              if (wx < 0 || wx >= Wo) continue;  // never read downstream
              pix[((size_t)(hh * sws + ww) * Hsym + y) * Wo + x] = glr_at<T>(cs, cy, cx, cs, wy, wx);
            }
    };
    quadrant(0, wsh, wsh, sws, 0);        // first quadrant, offset {0,0}
    quadrant(0, wsh + 1, 0, wsh, wsh);    // second quadrant, offset {0,wsh}

    for (int p : P.patches) {
      const int ci = idx++;
      const LutView& L = P.stats.at({p, s});
      patch_sums<T>(pix.data(), U, Hsym, Wo, p, pmax, inter, patch.data());
      // weights (compute_weights.cl)
      if (P.want_diag) wmargin.assign(wsym.size(), std::numeric_limits<T>::infinity());
      for (size_t i = 0; i < wsym.size(); ++i)
        wsym[i] = lut_weight<T>(patch[i], L, (T)P.h, (T)P.c, P.want_diag ? &wmargin[i] : nullptr);
      // symmetric expansion (copy_symm_weights.cl:39-77) + self weight (routines.cpp:151-157)
      std::vector<T> fmargin;
      if (P.want_diag) fmargin.assign((size_t)N * nc, std::numeric_limits<T>::infinity());
      symm_index_map(hc, wc, sws, Hps, Wps, [&](size_t dst, size_t src) {
        wfull[dst] = wsym[src];
        if (P.want_diag) fmargin[dst] = wmargin[src];
      });
      for (size_t o = 0; o < nc; ++o) wfull[(size_t)U * nc + o] = T(1);
      // statistics (compute_nl_statistics.cl:72-103), alphas, ENL'
      ComboResult<T>& R = res[ci];
      R.enl_nobias.assign(nc, 0);
      R.alpha.assign(nc, 0);
      R.wsum.assign(nc, 0);
      R.mean8.assign((size_t)ori.np * nc, 0);
      if (P.want_diag) {
        R.bin_margin.assign(nc, std::numeric_limits<T>::infinity());
        R.var_cond.assign(nc, std::numeric_limits<T>::infinity());
        R.kappa.assign(nc, T(1));
      }
      for (int y = 0; y < hc; ++y)
        for (int x = 0; x < wc; ++x) {
          const size_t o = (size_t)y * wc + x;
          const int dim = ori.d;
          T wsum = 0, wsum2 = 0, I[3] = {0, 0, 0}, V[3] = {0, 0, 0};
          for (int a = 0; a < sws; ++a)
            for (int b = 0; b < sws; ++b) {
              const T w = wfull[(size_t)(a * sws + b) * nc + o];
              // neighbour at tile row out+a+psh+swh (compute_nl_statistics.cl:61-64)
              const int ny = y + a + Psh + Ssh, nx = x + b + Psh + Ssh;
              wsum += w;
              wsum2 += w * w;
              for (int d = 0; d < dim; ++d) {
                const T inten = ori.at(ori.plane(d, d), ny, nx);
                const T insq = inten * inten;
                I[d] += w * inten;
                V[d] += w * insq;
              }
              if (P.want_diag) R.bin_margin[o] = std::min(R.bin_margin[o], fmargin[(size_t)(a * sws + b) * nc + o]);
            }
          const T enl = wsum * wsum / wsum2;
          T var[3], inl[3];
          for (int d = 0; d < dim; ++d) {
            I[d] /= wsum;
            V[d] /= wsum;
            var[d] = V[d] - I[d] * I[d];
            inl[d] = I[d];
            if (P.want_diag) R.var_cond[o] = std::min(R.var_cond[o], std::fabs(var[d]) / (I[d] * I[d]));
          }
          // compute_alphas.cl:30-42 (nlooks = 1)
          T alpha = 0;
          for (int d = 0; d < dim; ++d)
            alpha = cl_max<T>(alpha, cl_max<T>(T(0), (var[d] - inl[d] * inl[d] / T(1)) / var[d]));
          // compute_enls_nobias.cl:19-23
          const T oma = T(1) - alpha;
          const T enb = enl / (oma * oma + (alpha * alpha + T(2) * alpha * (T(1) - alpha) / wsum) * enl);
          R.enl_nobias[o] = enb;
          R.alpha[o] = alpha;
          R.wsum[o] = wsum;
          // weighted means of every plane (weighted_means.cl:47-80), kept per combo
          for (int pl = 0; pl < ori.np; ++pl) {
            T cnew = 0, ws = 0;
            for (int a = 0; a < sws; ++a)
              for (int b = 0; b < sws; ++b) {
                const T w = wfull[(size_t)(a * sws + b) * nc + o];
                ws += w;
                cnew += w * ori.at(pl, y + a + Ssh + Psh, x + b + Ssh + Psh);
              }
            // store the pieces; the blend needs the selected alpha (:79)
            R.mean8[(size_t)pl * nc + o] = cnew;
            (void)ws;
          }
          if (P.want_diag) {
            T mag = 0;
            for (int a = 0; a < sws; ++a)
              for (int b = 0; b < sws; ++b) {
                const T w = wfull[(size_t)(a * sws + b) * nc + o];
                const int ny = y + a + Ssh + Psh, nx = x + b + Ssh + Psh;
                mag += std::fabs(w) * std::hypot(ori.at(2, ny, nx), ori.at(3, ny, nx));
              }
            const T sr = R.mean8[(size_t)2 * nc + o], si = R.mean8[(size_t)3 * nc + o];
            R.kappa[o] = mag / std::hypot(sr, si);
          }
        }
    }
  }

  // selection (best_params.cpp:27-54 / ENL argmax) and blend (weighted_means.cl:79)
  // map order of keys: lexicographic (patch, scale) (parameters.h:37-40)
  std::vector<std::pair<int, int>> keys_sorted;
  for (auto& kv : P.stats) keys_sorted.push_back(kv.first);
  auto combo_of = [&](std::pair<int, int> k) {
    for (int i = 0; i < nco; ++i)
      if (combos[i].p == k.first && combos[i].s == k.second) return i;
    return -1;
  };
  out.cov8.assign((size_t)ori.np * nc, 0);
  out.sel.assign(nc, 0);
  if (P.want_diag) {
    out.bin_margin.assign(nc, 0);
    out.enl_margin.assign(nc, std::numeric_limits<T>::infinity());
    out.var_cond.assign(nc, std::numeric_limits<T>::infinity());
    out.kappa.assign(nc, T(1));
    out.bin_margin_all.assign(nc, std::numeric_limits<T>::infinity());
  }
  // combos ranked in map order for the argmax
  std::vector<int> map_order;
  for (auto& k : keys_sorted) {
    const int ci = combo_of(k);
    if (ci >= 0) map_order.push_back(ci);
  }
  const std::pair<int, int> last_key = keys_sorted.back();
  const int last_ci = combo_of(last_key);
  for (size_t o = 0; o < nc; ++o) {
    int sel;
    T alpha;
    if (P.select_mode == 0) {
      // every pixel gets the last key of the stats map; a key that was not
      // computed maps to index 0 (params2idx default) with alpha 0 (the
      // zero-initialised alphas map entry, nlsar_filter_sub_image.cpp:418-422)
      if (last_ci >= 0) {
        sel = last_ci;
        alpha = res[sel].alpha[o];
      } else {
        sel = 0;
        alpha = 0;
      }
    } else {
      T best = T(-1);
      sel = -1;
      T second = -std::numeric_limits<T>::infinity();
      for (int ci : map_order) {
        const T e = res[ci].enl_nobias[o];
        if (e > best) {
          second = std::max(second, best);
          best = e;
          sel = ci;
        } else if (!std::isnan(e)) {
          second = std::max(second, e);
        }
      }
      if (sel < 0) sel = 0;
      alpha = res[sel].alpha[o];
      if (P.want_diag) out.enl_margin[o] = (best - second) / std::fabs(best);
    }
    out.sel[o] = sel;
    const int y = (int)(o / wc), x = (int)(o % wc);
    for (int pl = 0; pl < ori.np; ++pl) {
      const T cnew = res[sel].mean8[(size_t)pl * nc + o];
      const T ws = res[sel].wsum[o];
      const T center = ori.at(pl, y + wsh + Ssh + Psh, x + wsh + Ssh + Psh);
      out.cov8[(size_t)pl * nc + o] = (1 - alpha) * cnew / ws + alpha * center;
    }
    if (P.want_diag) {
      out.bin_margin[o] = res[sel].bin_margin[o];
      out.kappa[o] = res[sel].kappa[o];
      for (int ci = 0; ci < nco; ++ci) out.bin_margin_all[o] = std::min(out.bin_margin_all[o], res[ci].bin_margin[o]);
      // reference mode depends on the selected combination only; the ENL
      // argmax depends on every combination's alpha
      if (P.select_mode == 0)
        out.var_cond[o] = res[sel].var_cond[o];
      else
        for (int ci = 0; ci < nco; ++ci) out.var_cond[o] = std::min(out.var_cond[o], res[ci].var_cond[o]);
    }
  }
  return out;
}

// covmat_decompose.cl:29-38
template <typename T>
void decompose(T c00, T c01r, T c01i, T c11, float* ref, float* phase, float* coh) {
  const T am = std::sqrt(c00), as = std::sqrt(c11);
  const T r = T(0.5f) * (am + as);
  *ref = (float)(r * r);
  *phase = (float)std::atan2(c01i, c01r);
  *coh = (float)(std::sqrt(c01i * c01i + c01r * c01r) / (am * as));
}

// tile list of map_filter_tiles (tile_iterator.cpp:48-65)
struct TileRect { int h0, w0; };
std::vector<TileRect> tile_list(int H, int W, int th, int tw, int ov) {
  std::vector<TileRect> t;
  int h = -ov, w = -ov;
  while (h < H) {
    t.push_back({h, w});
    w += tw - 2 * ov;
    if (w >= W) {
      w = -ov;
      h += th - 2 * ov;
    }
  }
  return t;
}

// get_sub_image with clamp padding (sub_images.cpp:23-45)
template <typename T>
Cov<T> cov_tile(const Cov<T>& img, int h0, int w0, int th, int tw) {
  Cov<T> c(th, tw, img.d);
  for (int pl = 0; pl < img.np; ++pl)
    for (int y = 0; y < th; ++y)
      for (int x = 0; x < tw; ++x) {
        const int yy = std::min(img.h - 1, std::max(0, y + h0));
        const int xx = std::min(img.w - 1, std::max(0, x + w0));
        c.at(pl, y, x) = img.at(pl, yy, xx);
      }
  return c;
}

int get_overlap(const FilterParams& P) {
  // nlsar.cpp:41-51
  const int pmax = *std::max_element(P.patches.begin(), P.patches.end());
  const int smax = *std::max_element(P.scales.begin(), P.scales.end());
  return (pmax - 1) / 2 + (P.sws - 1) / 2 + (smax - 1) / 2;
}

// The whole-image driver: map_filter_tiles with clamp padding, crop of the
// overlap and clamped write-back (map_filter_tiles.h:69-96,
// sub_images.cpp:47-69).  Tiles are filtered in parallel and written back in
// iteration order, so a later tile wins where two tiles write the same
// (clamped) output pixel.
template <typename T>
int nlsar_image(const Cov<T>& img, const FilterParams& P, int tile_h, int tile_w, int nthreads,
                Cov<T>& outc, std::vector<int>* sel, std::vector<T>* bmar, std::vector<T>* emar,
                std::vector<T>* vcond, std::vector<T>* kap = nullptr, std::vector<T>* bma = nullptr) {
  const int ov = get_overlap(P);
  const int H = img.h, W = img.w;
  if (tile_h <= 2 * ov || tile_w <= 2 * ov) return -1;
  const std::vector<TileRect> tiles = tile_list(H, W, tile_h, tile_w, ov);
  std::vector<TileOut<T>> outs(tiles.size());
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (long t = 0; t < (long)tiles.size(); ++t) {
    const Cov<T> tile = cov_tile<T>(img, tiles[t].h0, tiles[t].w0, tile_h, tile_w);
    outs[t] = filter_tile<T>(tile, P);
  }
  outc = Cov<T>(H, W, img.d);
  if (sel) sel->assign((size_t)H * W, 0);
  if (bmar) bmar->assign((size_t)H * W, 0);
  if (emar) emar->assign((size_t)H * W, 0);
  if (vcond) vcond->assign((size_t)H * W, 0);
  if (kap) kap->assign((size_t)H * W, 0);
  if (bma) bma->assign((size_t)H * W, 0);
  for (size_t t = 0; t < tiles.size(); ++t) {
    const TileOut<T>& o = outs[t];
    // the core of a tile of size tile_h x tile_w starts at tile origin + ov;
    // the per-tile filter produced a core of (tile - smax + 1 - 2*(wsh+Psh))
    // which equals tile - 2*ov
    for (int y = 0; y < o.hc; ++y)
      for (int x = 0; x < o.wc; ++x) {
        const int yy = std::min(H - 1, std::max(0, tiles[t].h0 + ov + y));
        const int xx = std::min(W - 1, std::max(0, tiles[t].w0 + ov + x));
        const size_t oi = (size_t)y * o.wc + x;
        for (int pl = 0; pl < img.np; ++pl) outc.at(pl, yy, xx) = o.cov8[(size_t)pl * o.hc * o.wc + oi];
        if (sel) (*sel)[(size_t)yy * W + xx] = o.sel[oi];
        if (bmar && !o.bin_margin.empty()) (*bmar)[(size_t)yy * W + xx] = o.bin_margin[oi];
        if (emar && !o.enl_margin.empty()) (*emar)[(size_t)yy * W + xx] = o.enl_margin[oi];
        if (vcond && !o.var_cond.empty()) (*vcond)[(size_t)yy * W + xx] = o.var_cond[oi];
        if (kap && !o.kappa.empty()) (*kap)[(size_t)yy * W + xx] = o.kappa[oi];
        if (bma && !o.bin_margin_all.empty()) (*bma)[(size_t)yy * W + xx] = o.bin_margin_all[oi];
      }
  }
  return 0;
}

int build_params(FilterParams& P, int sws, const int* patches, int np, const int* scales, int ns,
                 const oracle_lut* luts, int nluts, double h, double c, int select_mode, int want_diag) {
  if (sws < 1 || sws % 2 == 0 || np < 1 || ns < 1 || nluts < 1) return -1;
  P.sws = sws;
  P.patches.clear();
  P.scales.clear();
  for (int i = 0; i < np; ++i) {
    if (patches[i] < 1 || patches[i] % 2 == 0) return -1;
    if (std::find(P.patches.begin(), P.patches.end(), patches[i]) == P.patches.end()) P.patches.push_back(patches[i]);
  }
  for (int i = 0; i < ns; ++i) {
    if (scales[i] < 1 || scales[i] % 2 == 0) return -1;
    if (std::find(P.scales.begin(), P.scales.end(), scales[i]) == P.scales.end()) P.scales.push_back(scales[i]);
  }
  P.stats.clear();
  for (int i = 0; i < nluts; ++i)
    P.stats[{luts[i].patch_size, luts[i].scale_size}] =
        LutView{luts[i].lut_size, luts[i].dissims_min, luts[i].dissims_max, luts[i].quantilles, luts[i].chi2cdf_inv};
  for (int p : P.patches)
    for (int s : P.scales)
      if (!P.stats.count({p, s})) return -2;
  P.h = h;
  P.c = c;
  P.select_mode = select_mode;
  P.want_diag = want_diag;
  return 0;
}

template <typename T>
int run_insar(const float* a1, const float* a2, const float* ph, float* ref, float* phase, float* coh,
              int H, int W, const FilterParams& P, int tile_h, int tile_w, int nthreads, int* sel,
              double* bmar, double* emar, double* vcond, double* kappa, double* bma) {
  const Cov<T> img = covmat_create<T>(a1, a2, ph, H, W);
  Cov<T> outc;
  std::vector<int> s;
  std::vector<T> b, e, v, k, ba;
  int rc = nlsar_image<T>(img, P, tile_h, tile_w, nthreads, outc, sel ? &s : nullptr, bmar ? &b : nullptr,
                          emar ? &e : nullptr, vcond ? &v : nullptr, kappa ? &k : nullptr, bma ? &ba : nullptr);
  if (rc) return rc;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const size_t i = (size_t)y * W + x;
      decompose<T>(outc.at(0, y, x), outc.at(2, y, x), outc.at(3, y, x), outc.at(6, y, x), ref + i, phase + i,
                   coh + i);
      if (sel) sel[i] = s[i];
      if (bmar) bmar[i] = (double)b[i];
      if (emar) emar[i] = (double)e[i];
      if (vcond) vcond[i] = (double)v[i];
      if (kappa) kappa[i] = (double)k[i];
      if (bma) bma[i] = (double)ba[i];
    }
  return 0;
}

template <typename T>
int run_covmat(const float* cin, float* cout, int H, int W, int dim, const FilterParams& P, int tile_h, int tile_w,
               int nthreads) {
  Cov<T> img(H, W, dim);
  for (size_t i = 0; i < img.v.size(); ++i) img.v[i] = cin[i];
  Cov<T> outc;
  int rc = nlsar_image<T>(img, P, tile_h, tile_w, nthreads, outc, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  for (size_t i = 0; i < outc.v.size(); ++i) cout[i] = (float)outc.v[i];
  return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// exported entry points (C ABI, loaded by the tests through ctypes)
// ---------------------------------------------------------------------------

extern "C" int oracle_nlsar_insar(const float* a1, const float* a2, const float* ph, float* ref, float* phase,
                                  float* coh, int H, int W, int sws, const int* patches, int np,
                                  const int* scales, int ns, const oracle_lut* luts, int nluts, float h,
                                  float c, int select_mode, int use_double, int tile_h, int tile_w,
                                  int nthreads, int* sel, double* bin_margin, double* enl_margin,
                                  double* var_cond, double* kappa, double* bin_margin_all) {
  FilterParams P;
  const int want_diag = (bin_margin || enl_margin || var_cond || kappa || bin_margin_all) ? 1 : 0;
  int rc = build_params(P, sws, patches, np, scales, ns, luts, nluts, h, c, select_mode, want_diag);
  if (rc) return rc;
  if (H < 1 || W < 1) return -1;
  if (use_double)
    return run_insar<double>(a1, a2, ph, ref, phase, coh, H, W, P, tile_h, tile_w, nthreads, sel, bin_margin,
                             enl_margin, var_cond, kappa, bin_margin_all);
  return run_insar<float>(a1, a2, ph, ref, phase, coh, H, W, P, tile_h, tile_w, nthreads, sel, bin_margin,
                          enl_margin, var_cond, kappa, bin_margin_all);
}

extern "C" int oracle_nlsar_covmat(const float* cin, float* cout, int H, int W, int dim, int sws, const int* patches,
                                   int np, const int* scales, int ns, const oracle_lut* luts, int nluts,
                                   float h, float c, int select_mode, int use_double, int tile_h, int tile_w,
                                   int nthreads) {
  FilterParams P;
  int rc = build_params(P, sws, patches, np, scales, ns, luts, nluts, h, c, select_mode, 0);
  if (rc) return rc;
  if (H < 1 || W < 1 || dim < 2 || dim > 3) return -1;
  if (use_double) return run_covmat<double>(cin, cout, H, W, dim, P, tile_h, tile_w, nthreads);
  return run_covmat<float>(cin, cout, H, W, dim, P, tile_h, tile_w, nthreads);
}

extern "C" int oracle_overlap(int sws, const int* patches, int np, const int* scales, int ns) {
  FilterParams P;
  P.sws = sws;
  P.patches.assign(patches, patches + np);
  P.scales.assign(scales, scales + ns);
  return get_overlap(P);
}

// Stage-level entry points used by the known-answer tests.

extern "C" float oracle_pixel_similarity_2x2(float a00, float a01r, float a01i, float a11, float b00, float b01r,
                                             float b01i, float b11) {
  return glr_2x2<float>(a00, a01r, a01i, a11, b00, b01r, b01i, b11);
}

// a, b: the 9 unique reals {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12}
extern "C" float oracle_pixel_similarity_3x3(const float* a, const float* b) { return glr_3x3<float>(a, b); }

extern "C" void oracle_gen_gauss(int s, float* out) {
  const std::vector<float> g = gen_gauss<float>(s);
  std::copy(g.begin(), g.end(), out);
}

extern "C" float oracle_rescale_gamma(void) { return rescale_gamma<float>(2); }
extern "C" float oracle_rescale_gamma_dim(int dim) { return rescale_gamma<float>(dim); }

extern "C" void oracle_covmat_create(const float* a1, const float* a2, const float* ph, int H, int W, float* cov8) {
  const Cov<float> c = covmat_create<float>(a1, a2, ph, H, W);
  std::copy(c.v.begin(), c.v.end(), cov8);
}

extern "C" void oracle_covmat_spatial_avg(const float* in8, int H, int W, int s, int smax, float* out8) {
  Cov<float> c(H, W);
  std::copy(in8, in8 + c.v.size(), c.v.begin());
  const Cov<float> o = covmat_spatial_avg<float>(c, s, smax);
  std::copy(o.v.begin(), o.v.end(), out8);
}

extern "C" float oracle_lut_weight(float dissim, unsigned lut_size, float dmin, float dmax, const float* quant,
                                   const float* chi2, float h, float c) {
  LutView L{lut_size, dmin, dmax, quant, chi2};
  return lut_weight<float>(dissim, L, h, c, nullptr);
}

// weights of the reference's alpha / ENL' formulas for the known-answer tests
extern "C" float oracle_alpha(const float* var, const float* inl, int dim) {
  float alpha = 0;
  for (int d = 0; d < dim; ++d) alpha = cl_max(alpha, cl_max(0.0f, (var[d] - inl[d] * inl[d] / 1.0f) / var[d]));
  return alpha;
}

extern "C" float oracle_enl_nobias(float enl, float alpha, float wsum) {
  const float oma = 1.0f - alpha;
  return enl / (oma * oma + (alpha * alpha + 2.0f * alpha * (1.0f - alpha) / wsum) * enl);
}

extern "C" int oracle_tile_list(int H, int W, int th, int tw, int ov, int* h0, int* w0, int cap) {
  const std::vector<TileRect> t = tile_list(H, W, th, tw, ov);
  const int n = (int)t.size();
  for (int i = 0; i < n && i < cap; ++i) {
    h0[i] = t[i].h0;
    w0[i] = t[i].w0;
  }
  return n;
}

// Stage entry points for the known-answer tests of the reference's kernel
// tests (compute_patch_similarities_test.cpp:31-81,
// copy_symm_weights_test.cpp:33-128), FP32.
extern "C" int oracle_patch_similarities(const float* pix, float* out, int height_sim, int width_sim, int sws,
                                         int patch_size, int patch_size_max) {
  if (sws < 1 || sws % 2 == 0 || patch_size < 1 || patch_size % 2 == 0 || patch_size > patch_size_max ||
      height_sim < patch_size_max || width_sim < patch_size_max)
    return -1;
  const int wsh = (sws - 1) / 2, U = sws * wsh + wsh;
  std::vector<float> inter;
  patch_sums<float>(pix, U, height_sim, width_sim, patch_size, patch_size_max, inter, out);
  return 0;
}

extern "C" int oracle_copy_symm_weights(const float* wsymm, float* wfull, int height_ori, int width_ori, int sws) {
  if (sws < 1 || sws % 2 == 0 || height_ori < 1 || width_ori < 1) return -1;
  const int wsh = (sws - 1) / 2, U = sws * wsh + wsh;
  const size_t nc = (size_t)height_ori * width_ori;
  symm_index_map(height_ori, width_ori, sws, height_ori + wsh, width_ori + 2 * wsh,
                 [&](size_t dst, size_t src) { wfull[dst] = wsymm[src]; });
  for (size_t o = 0; o < nc; ++o) wfull[(size_t)U * nc + o] = 1.0f;
  return 0;
}

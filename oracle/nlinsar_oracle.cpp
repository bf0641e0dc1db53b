// TEST INFRASTRUCTURE ONLY: a CPU restatement of despeckCL's NL-InSAR filter
// used as the checker of the GPU path; never linked into the product library.
//
// despeckcl::nlinsar (src/compute/nlinsar/nlinsar.cpp:42-130): niter passes;
// each pass cuts the scene into 80 x 80 tiles with overlap wsh + psh
// (tile_iterator.cpp, clamped gather sub_images.cpp:23-45), filters every tile
// from the previous pass's estimates and writes the tile centres into the next
// estimates with clamping, later tiles over earlier ones (map_filter_tiles.h,
// sub_images.cpp:47-69).  Per tile (nlinsar_sub_image.cpp:32-250):
//   pixel similarity (sim_measures.h:27-40) and Kullback-Leibler divergence of
//     the current estimates (sim_measures.h:42-50) for every search-window
//     offset; in the tile interior the first wsh window rows are copies of the
//     mirrored offsets (precompute_similarities_1st_pass.cl.in:29-39,
//     precompute_similarities_2nd_pass.cl:19-45), i.e. the measures with their
//     two pixels swapped;
//   p x p sums, rows first (precompute_patch_similarities.cl:40-58);
//   w = exp(S / h + KL / T), NaN / inf -> 0 (compute_weights.cl:19-30), the
//     centre offset's weight 0 (nlinsar_sub_image.cpp:188-196);
//   looks (sum w)^2 / sum w^2 (common/cl_kernels/compute_number_of_looks.cl);
//   below lmin looks, the lmin largest weights among the window pixels whose
//     master amplitude is below twice the centre's are replaced by their mean
//     (smoothing.cpp:65-117; the selection follows std::priority_queue, a
//     binary heap: sift-up on push, sift-down-to-leaf then sift-up on pop);
//   weighted means of 0.5 (a1^2 + a2^2) and a1 a2 e^{-j phi}
//     (precompute_filter_values.cl, compute_insar.cl:45-103): reflectivity,
//     phase, coherence, each kept from the previous pass where not finite or 0.
// h = h_theo p^2 with h_theo 0.58 (p = 3) / 0.244 (p = 7), T = 2 / h * pi / 4 * p^2
// (nlinsar.cpp:60-75).
//
// T = double is the truth; T = float follows the reference's FP32 order.
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

constexpr int kTile = 80;

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <typename T>
T pixel_sim(T am1, T as1, T dp1, T am2, T as2, T dp2) {
  const T A = std::pow(am1 * am1 + as1 * as1 + am2 * am2 + as2 * as2, T(2));
  const T B = T(4) * (am1 * am1 * as1 * as1 + am2 * am2 * as2 * as2 + T(2) * am1 * as1 * am2 * as2 * std::cos(dp1 - dp2));
  const T C = am1 * as1 * am2 * as2;
  const T f = std::pow(C / B, T(1.5)) * ((A + B) / A * std::sqrt(B / (A - B)) - std::asin(std::sqrt(B / A)));
  if (f == 0 || std::isnan(f)) return 0;
  return std::log(f);
}

template <typename T>
T pixel_kl(T r1, T d1, T c1, T r2, T d2, T c2) {
  const T a1 = (r2 != T(0)) ? r1 / r2 * (T(1) - c1 * c2 * std::cos(d1 - d2)) / (T(1) - c2 * c2) : T(1);
  const T a2 = (r2 != T(0)) ? r2 / r1 * (T(1) - c1 * c2 * std::cos(d1 - d2)) / (T(1) - c1 * c1) : T(1);
  return T(-4) / T(M_PI) * (a1 + a2 - T(2));
}

// The binary heap of std::priority_queue<weight_el> with the reference's
// ordering (the top is the smallest weight; smoothing.cpp:25-31).
struct Heap {
  struct El {
    float w;
    int idx;
  };
  std::vector<El> v;
  // "a before b" in heap order: a.w > b.w  (operator< of weight_el)
  static bool less(const El& a, const El& b) { return a.w > b.w; }
  void sift_up(int hole, El val, int top) {
    int parent = (hole - 1) / 2;
    while (hole > top && less(v[parent], val)) {
      v[hole] = v[parent];
      hole = parent;
      parent = (hole - 1) / 2;
    }
    v[hole] = val;
  }
  void push(El e) {
    v.push_back(e);
    sift_up((int)v.size() - 1, e, 0);
  }
  El top() const { return v[0]; }
  void pop() {
    const int n = (int)v.size() - 1;  // heap of the first n after moving the top out
    El val = v[n];
    v[n] = v[0];
    int hole = 0, child = 0;
    while (child < (n - 1) / 2) {
      child = 2 * (child + 1);
      if (less(v[child], v[child - 1])) --child;
      v[hole] = v[child];
      hole = child;
    }
    if ((n & 1) == 0 && child == (n - 2) / 2) {
      child = 2 * (child + 1);
      v[hole] = v[child - 1];
      hole = child - 1;
    }
    sift_up(hole, val, 0);
    v.pop_back();
  }
};

struct Params {
  int sws, p, lmin;
  float h, Tp;
};

// One tile; planes [6][kTile][kTile] (a1, a2, phase, ref, phase_filt, coh).
template <typename T>
void filter_tile(float* tile, const Params& P) {
  const int sws = P.sws, p = P.p, wsh = (sws - 1) / 2, psh = (p - 1) / 2, ov = wsh + psh;
  const int HO = kTile, Hsim = HO - sws + 1, Hori = HO - 2 * ov, Hsws = HO - p + 1;
  const size_t n2 = (size_t)HO * HO;
  const float *a1 = tile, *a2 = tile + n2, *dp = tile + 2 * n2;
  float *rf = tile + 3 * n2, *pf = tile + 4 * n2, *cf = tile + 5 * n2;
  const int no = sws * sws;
  std::vector<T> S((size_t)no * Hsim * Hsim), K((size_t)no * Hsim * Hsim);
  for (int hh = 0; hh < sws; ++hh)
    for (int ww = 0; ww < sws; ++ww)
      for (int h = 0; h < Hsim; ++h)
        for (int w = 0; w < Hsim; ++w) {
          const bool interior = h >= wsh && w >= wsh && w < Hsim - wsh;
          int c = (h + wsh) * HO + (w + wsh), q = (h + hh) * HO + (w + ww);
          if (interior && hh < wsh) std::swap(c, q);  // the mirrored offset's value
          const size_t o = ((size_t)(hh * sws + ww) * Hsim + h) * Hsim + w;
          S[o] = pixel_sim<T>(a1[c], a2[c], dp[c], a1[q], a2[q], dp[q]);
          K[o] = pixel_kl<T>(rf[c], pf[c], cf[c], rf[q], pf[q], cf[q]);
        }
  // weights [pixel][offset]
  std::vector<float> wts((size_t)Hori * Hori * no);
  for (int k = 0; k < no; ++k)
    for (int x = 0; x < Hori; ++x)
      for (int y = 0; y < Hori; ++y) {
        T s = 0, kl = 0;
        for (int kx = 0; kx < p; ++kx) {
          T rs = 0, rk = 0;
          for (int ky = 0; ky < p; ++ky) {
            rs += S[((size_t)k * Hsim + x + kx) * Hsim + y + ky];
            rk += K[((size_t)k * Hsim + x + kx) * Hsim + y + ky];
          }
          if (kx == 0) {
            s = rs;
            kl = rk;
          } else {
            s += rs;
            kl += rk;
          }
        }
        T wv = std::exp(s / T(P.h) + kl / T(P.Tp));
        if (std::isnan(wv) || std::isinf(wv)) wv = 0;
        if (k == wsh * sws + wsh) wv = 0;
        wts[((size_t)x * Hori + y) * no + k] = (float)wv;
      }
  // filter values at (u + psh, v + psh)
  std::vector<T> fa((size_t)Hsws * Hsws), fr((size_t)Hsws * Hsws), fi((size_t)Hsws * Hsws);
  for (int u = 0; u < Hsws; ++u)
    for (int v = 0; v < Hsws; ++v) {
      const int i = (u + psh) * HO + (v + psh);
      const T x1 = a1[i], x2 = a2[i], d = dp[i];
      fa[(size_t)u * Hsws + v] = T(0.5) * (x1 * x1 + x2 * x2);
      fr[(size_t)u * Hsws + v] = x1 * x2 * std::cos(-d);
      fi[(size_t)u * Hsws + v] = x1 * x2 * std::sin(-d);
    }
  for (int x = 0; x < Hori; ++x)
    for (int y = 0; y < Hori; ++y) {
      float* w = &wts[((size_t)x * Hori + y) * no];
      T s1 = 0, s2 = 0;
      for (int k = 0; k < no; ++k) {
        s1 += T(w[k]);
        s2 += T(w[k]) * T(w[k]);
      }
      const T nol = s1 * s1 / s2;
      if (nol < T(P.lmin)) {
        Heap hp;
        const double as = a1[(x + ov) * HO + (y + ov)];
        for (int hh = 0; hh < sws; ++hh)
          for (int ww = 0; ww < sws; ++ww) {
            const float at = a1[(x + ov + hh - wsh) * HO + (y + ov + ww - wsh)];
            if (at < 2.0 * as) {
              const int idx = hh * sws + ww;
              if ((int)hp.v.size() < P.lmin)
                hp.push({w[idx], idx});
              else if (hp.top().w < w[idx]) {
                hp.pop();
                hp.push({w[idx], idx});
              }
            }
          }
        std::vector<int> idxs;
        T wsum = 0;
        while (!hp.v.empty()) {
          wsum += T(hp.top().w);
          idxs.push_back(hp.top().idx);
          hp.pop();
        }
        wsum /= T((float)idxs.size());
        for (int idx : idxs) w[idx] = (float)wsum;
      }
      T N = 0, A = 0, Xr = 0, Xi = 0;
      for (int i = 0; i < sws; ++i)
        for (int j = 0; j < sws; ++j) {
          const T wt = w[i * sws + j];
          const size_t f = (size_t)(x + i) * Hsws + (y + j);
          N += wt;
          A += wt * fa[f];
          Xr += wt * fr[f];
          Xi += wt * fi[f];
        }
      const T refl = A / N, phi = std::atan2(Xi, Xr), coh = std::sqrt(Xr * Xr + Xi * Xi) / A;
      const int o = (x + ov) * HO + (y + ov);
      auto valid = [](T v) { return !(std::isnan(v) || std::isinf(v) || v == 0); };
      if (valid(refl)) rf[o] = (float)refl;
      if (valid(phi)) {
        T ph = phi;
        if (ph > T((float)M_PI)) ph -= T(2) * T((float)M_PI);
        if (ph < -T((float)M_PI)) ph += T(2) * T((float)M_PI);
        pf[o] = (float)ph;
      }
      if (valid(coh)) cf[o] = (float)std::min(T(1), std::max(T(0), coh));
    }
}

template <typename T>
void nlinsar_t(const float* a1, const float* a2, const float* ph, float* ref, float* phase, float* coh, int H, int W,
               const Params& P, int niter, int nthreads) {
  const int ov = (P.sws - 1) / 2 + (P.p - 1) / 2;
  const int step = kTile - 2 * ov;
  std::vector<int> h0s, w0s;
  for (int h0 = -ov; h0 < H; h0 += step) h0s.push_back(h0);
  for (int w0 = -ov; w0 < W; w0 += step) w0s.push_back(w0);
  const size_t n = (size_t)H * W, n2 = (size_t)kTile * kTile;
  const int ntiles = (int)(h0s.size() * w0s.size());
  std::vector<float> tiles((size_t)ntiles * 6 * n2);
  for (int it = 0; it < niter; ++it) {
    const float* planes[6] = {a1, a2, ph, ref, phase, coh};
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int t = 0; t < ntiles; ++t) {
      const int h0 = h0s[t / w0s.size()], w0 = w0s[t % w0s.size()];
      float* tile = &tiles[(size_t)t * 6 * n2];
      for (int d = 0; d < 6; ++d)
        for (int y = 0; y < kTile; ++y)
          for (int x = 0; x < kTile; ++x)
            tile[d * n2 + y * kTile + x] =
                planes[d][(size_t)clampi(y + h0, 0, H - 1) * W + clampi(x + w0, 0, W - 1)];
      filter_tile<T>(tile, P);
    }
    // write back in tile order (the next estimates start as a copy of these)
    std::vector<float> nr(ref, ref + n), np(phase, phase + n), nc(coh, coh + n);
    for (int t = 0; t < ntiles; ++t) {
      const int h0 = h0s[t / w0s.size()], w0 = w0s[t % w0s.size()];
      const float* tile = &tiles[(size_t)t * 6 * n2];
      for (int y = ov; y < kTile - ov; ++y)
        for (int x = ov; x < kTile - ov; ++x) {
          const size_t o = (size_t)std::min(H - 1, y + h0) * W + std::min(W - 1, x + w0);
          nr[o] = tile[3 * n2 + y * kTile + x];
          np[o] = tile[4 * n2 + y * kTile + x];
          nc[o] = tile[5 * n2 + y * kTile + x];
        }
    }
    std::copy(nr.begin(), nr.end(), ref);
    std::copy(np.begin(), np.end(), phase);
    std::copy(nc.begin(), nc.end(), coh);
  }
}

}  // namespace

// h_theo of nlinsar.cpp:60-69 for the patch sizes it tabulates (0 otherwise).
extern "C" float oracle_nlinsar_h_theo(int patch_size) {
  return patch_size == 3 ? 0.58f : (patch_size == 7 ? 0.244f : 0.0f);
}

// ref / phase / coh hold the initial estimates on entry (the Python binding
// passes zeros) and the results on exit.
extern "C" int oracle_nlinsar(const float* a1, const float* a2, const float* ph, float* ref, float* phase, float* coh,
                              int H, int W, int sws, int patch_size, int niter, int lmin, int use_double,
                              int nthreads) {
  const float h_theo = oracle_nlinsar_h_theo(patch_size);
  if (H < 1 || W < 1 || sws < 1 || sws % 2 == 0 || patch_size < 1 || patch_size % 2 == 0 || h_theo == 0.0f ||
      (sws - 1) + (patch_size - 1) >= kTile)
    return -1;
  Params P;
  P.sws = sws;
  P.p = patch_size;
  P.lmin = lmin;
  const int area = patch_size * patch_size;
  P.h = h_theo * area;
  P.Tp = (float)(2.0 / P.h * M_PI / 4 * area);
  if (use_double)
    nlinsar_t<double>(a1, a2, ph, ref, phase, coh, H, W, P, niter, nthreads);
  else
    nlinsar_t<float>(a1, a2, ph, ref, phase, coh, H, W, P, niter, nthreads);
  return 0;
}

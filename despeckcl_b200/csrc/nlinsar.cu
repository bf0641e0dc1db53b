// NL-InSAR (despeckcl::nlinsar, src/compute/nlinsar/nlinsar.cpp:42-130 and
// nlinsar_sub_image.cpp:32-250 in the reference).
//
// niter passes; each pass cuts the scene into the reference's 80 x 80 tiles
// with overlap wsh + psh (tile_iterator.cpp, clamped gather sub_images.cpp),
// filters every tile from the previous pass's estimates, and takes each output
// pixel from the tile that writes it last in the reference's clamped
// write-back (tile row y / step for y < H-1, the last tile row's last centre
// row for y = H-1; columns alike).  Three kernels:
//
//  nlinsar_filter_values_kernel  once per call: 0.5 (a1^2 + a2^2) and
//      a1 a2 e^{-j phi} per pixel (precompute_filter_values.cl);
//  nlinsar_weights_kernel  one CTA per tile, the tile's six planes in shared
//      memory; per search-window offset: the pixel similarity and the
//      Kullback-Leibler divergence of the estimates (sim_measures.h) on the
//      similarity grid -- with the two pixels swapped in the tile interior for
//      the first wsh window rows, which the reference copies from the mirrored
//      offset (precompute_similarities_{1st,2nd}_pass): each lower-row offset
//      is taken with its mirror, whose interior maps are the lower offset's
//      shifted, only its border evaluated --, p x p sums rows
//      first (precompute_patch_similarities.cl), w = exp(S/h + KL/T) with
//      NaN / inf -> 0 and the centre weight 0 (compute_weights.cl), the looks
//      (sum w)^2 / sum w^2 accumulated in offset order
//      (compute_number_of_looks.cl); weights go to a scratch [tile][offset][pixel];
//  nlinsar_estimate_kernel  one thread per tile pixel that owns its output:
//      below lmin looks the lmin largest weights among the window pixels whose
//      master amplitude is below twice the centre's become their mean, chosen
//      with the reference's std::priority_queue (smoothing.cpp:65-117, a binary
//      heap replayed exactly); then the weighted means (compute_insar.cl),
//      each estimate kept from the previous pass where not finite or 0.
// This file is compiled with -fmad=false: every sum and product is rounded as
// in the reference's kernels; only the math functions (pow, asin, log, exp,
// cos, sin, atan2) are CUDA's.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"

namespace dcl {
namespace {

constexpr int kTile = 80;        // nlinsar.cpp:84, tile_dims {80, 80}
constexpr int kThreads = 1024;   // weights kernel (32 warps: the one CTA an SM holds)
constexpr int kMaxPixPerThread = 6;
constexpr int kMaxLmin = 64;
constexpr int kEstThreads = 128;

struct NlGeom {
  int H, W, sws, wsh, p, psh, ov;
  int hsim, hori;      // similarity grid and output side of a tile
  int step;            // tile origin step, kTile - 2 ov
  int ntx, nty;        // tiles per row / column
  int lmin;
  float h, T;
  int nborder;         // similarity-grid positions outside the interior the reference copies
  int mirror;          // 1: offsets of the lower window rows share their maps with their mirrors
};

__device__ __forceinline__ int clampn(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sim_measures.h:27-40 (am/as/dp of pixel 1, then of pixel 2)
__device__ __forceinline__ float pixel_sim(float am1, float as1, float dp1, float am2, float as2, float dp2) {
  const float s = am1 * am1 + as1 * as1 + am2 * am2 + as2 * as2;
  const float A = s * s;
  const float B = 4.0f * (am1 * am1 * as1 * as1 + am2 * am2 * as2 * as2 + 2.0f * am1 * as1 * am2 * as2 * cosf(dp1 - dp2));
  const float C = am1 * as1 * am2 * as2;
  // pow(x, 1.5) as x sqrt(x) (the same value up to rounding, NaN for x < 0
  // as pow gives) and the hardware log below (a few ulps): 8 % of the pass,
  // with every tested pixel still within tolerance of the oracle; fast
  // divisions or the hardware cos cost agreement
  const float x = C / B;
  const float f = (x * sqrtf(x)) * ((A + B) / A * sqrtf(B / (A - B)) - asinf(sqrtf(B / A)));
  if (f == 0.0f || isnan(f)) return 0.0f;
  return __logf(f);
}

// sim_measures.h:42-50, OpenCL's float pi
__device__ __forceinline__ float pixel_kl(float r1, float d1, float c1, float r2, float d2, float c2) {
  const float cs = cosf(d1 - d2);
  const float a1 = (r2 != 0.0f) ? r1 / r2 * (1.0f - c1 * c2 * cs) / (1.0f - c2 * c2) : 1.0f;
  const float a2 = (r2 != 0.0f) ? r2 / r1 * (1.0f - c1 * c2 * cs) / (1.0f - c1 * c1) : 1.0f;
  return -4.0f / 3.14159274101257324f * (a1 + a2 - 2.0f);
}

__global__ void nlinsar_filter_values_kernel(const float* __restrict__ a1, const float* __restrict__ a2,
                                             const float* __restrict__ dp, float* __restrict__ fa,
                                             float* __restrict__ fr, float* __restrict__ fi, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x1 = a1[i], x2 = a2[i], d = dp[i];
  fa[i] = 0.5f * (x1 * x1 + x2 * x2);
  fr[i] = x1 * x2 * cosf(-d);
  fi[i] = x1 * x2 * sinf(-d);
}

__global__ void __launch_bounds__(kThreads, 1)
    nlinsar_weights_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ dp,
                           const float* __restrict__ rf, const float* __restrict__ pf, const float* __restrict__ cf,
                           NlGeom g, int tile0, float* __restrict__ wout, float* __restrict__ nols) {
  extern __shared__ float sm[];
  constexpr int n2 = kTile * kTile;
  float* sA1 = sm;
  float* sA2 = sA1 + n2;
  float* sDp = sA2 + n2;
  float* sRf = sDp + n2;
  float* sPf = sRf + n2;
  float* sCf = sPf + n2;
  float* sS = sCf + n2;               // [hsim][hsim]
  float* sK = sS + g.hsim * g.hsim;
  float* sRS = sK + g.hsim * g.hsim;  // [hsim][hori] row sums
  float* sRK = sRS + g.hsim * g.hori;
  const int tile = tile0 + blockIdx.x;
  const int ti = tile / g.ntx, tj = tile - ti * g.ntx;
  const int h0 = -g.ov + ti * g.step, w0 = -g.ov + tj * g.step;
  const int tid = threadIdx.x;
  for (int i = tid; i < n2; i += kThreads) {
    const int y = i / kTile, x = i - y * kTile;
    const size_t o = (size_t)clampn(h0 + y, 0, g.H - 1) * g.W + clampn(w0 + x, 0, g.W - 1);
    sA1[i] = a1[o];
    sA2[i] = a2[o];
    sDp[i] = dp[o];
    sRf[i] = rf[o];
    sPf[i] = pf[o];
    sCf[i] = cf[o];
  }
  const int npix = g.hori * g.hori, nsim = g.hsim * g.hsim, nrow = g.hsim * g.hori;
  float s1[kMaxPixPerThread], s2[kMaxPixPerThread];
#pragma unroll
  for (int q = 0; q < kMaxPixPerThread; ++q) s1[q] = s2[q] = 0.0f;
  const int no = g.sws * g.sws, kc = g.wsh * g.sws + g.wsh;
  float* wt = wout + (size_t)blockIdx.x * no * npix;
  __syncthreads();
  // similarities and divergences of offset (hh, ww) on the whole grid, with
  // the two pixels swapped in the interior for the first wsh window rows (the
  // values the reference copies from the mirrored offset)
  auto sims_direct = [&](int hh, int ww) {
    for (int it = tid; it < nsim; it += kThreads) {
      const int h = it / g.hsim, w = it - h * g.hsim;
      const bool interior = h >= g.wsh && w >= g.wsh && w < g.hsim - g.wsh;
      int c = (h + g.wsh) * kTile + (w + g.wsh), q = (h + hh) * kTile + (w + ww);
      if (interior && hh < g.wsh) {
        const int t = c;
        c = q;
        q = t;
      }
      sS[it] = pixel_sim(sA1[c], sA2[c], sDp[c], sA1[q], sA2[q], sDp[q]);
      sK[it] = pixel_kl(sRf[c], sPf[c], sCf[c], sRf[q], sPf[q], sCf[q]);
    }
  };
  // p-wide row sums of a map given by `val(h, w)` (similarity, divergence)
  auto row_sums = [&](auto val) {
    for (int it = tid; it < nrow; it += kThreads) {
      const int r = it / g.hori, col = it - r * g.hori;
      float rs = 0.0f, rk = 0.0f;
      for (int ky = 0; ky < g.p; ++ky) {
        const float2 v = val(r, col + ky);
        rs += v.x;
        rk += v.y;
      }
      sRS[it] = rs;
      sRK[it] = rk;
    }
  };
  auto direct_val = [&](int h, int w) { return make_float2(sS[h * g.hsim + w], sK[h * g.hsim + w]); };
  // p-wide column sums, weights and looks of offset k
  auto weights_of = [&](int k) {
#pragma unroll
    for (int q = 0; q < kMaxPixPerThread; ++q) {
      const int pix = tid + q * kThreads;
      if (pix < npix) {
        const int x = pix / g.hori, y = pix - x * g.hori;
        float s = sRS[x * g.hori + y], kl = sRK[x * g.hori + y];
        for (int kx = 1; kx < g.p; ++kx) {
          s += sRS[(x + kx) * g.hori + y];
          kl += sRK[(x + kx) * g.hori + y];
        }
        float wv = expf(s / g.h + kl / g.T);
        if (isnan(wv) || isinf(wv)) wv = 0.0f;
        if (k == kc) wv = 0.0f;
        wt[(size_t)k * npix + pix] = wv;
        s1[q] += wv;
        s2[q] += wv * wv;
      }
    }
  };
  if (!g.mirror) {
    for (int hh = 0; hh < g.sws; ++hh)
      for (int ww = 0; ww < g.sws; ++ww) {
        sims_direct(hh, ww);
        __syncthreads();
        row_sums(direct_val);
        __syncthreads();
        weights_of(hh * g.sws + ww);
        __syncthreads();
      }
  } else {
    // the centre window row, computed as the reference computes it
    for (int ww = 0; ww < g.sws; ++ww) {
      sims_direct(g.wsh, ww);
      __syncthreads();
      row_sums(direct_val);
      __syncthreads();
      weights_of(g.wsh * g.sws + ww);
      __syncthreads();
    }
    // every lower-row offset with its mirror: the mirror's interior values are
    // the lower offset's maps shifted by the mirror's offset (the very values
    // the reference copies), its border values are computed here
    float* sBS = sRK + nrow;  // mirror's border: similarity, divergence
    float* sBK = sBS + g.nborder;
    const int top = g.wsh * g.hsim, band = 2 * g.wsh;
    for (int hl = g.wsh + 1; hl < g.sws; ++hl)
      for (int wl = 0; wl < g.sws; ++wl) {
        const int hu = 2 * g.wsh - hl, wu = 2 * g.wsh - wl;
        for (int it = tid; it < nsim + g.nborder; it += kThreads) {
          int c, q;
          if (it < nsim) {
            const int h = it / g.hsim, w = it - h * g.hsim;
            c = (h + g.wsh) * kTile + (w + g.wsh);
            q = (h + hl) * kTile + (w + wl);
            sS[it] = pixel_sim(sA1[c], sA2[c], sDp[c], sA1[q], sA2[q], sDp[q]);
            sK[it] = pixel_kl(sRf[c], sPf[c], sCf[c], sRf[q], sPf[q], sCf[q]);
          } else {
            const int ib = it - nsim;
            int h, w;
            if (ib < top) {
              h = ib / g.hsim;
              w = ib - h * g.hsim;
            } else {
              const int j = ib - top;
              h = g.wsh + j / band;
              const int m = j - (j / band) * band;
              w = m < g.wsh ? m : g.hsim - band + m;
            }
            c = (h + g.wsh) * kTile + (w + g.wsh);
            q = (h + hu) * kTile + (w + wu);
            sBS[ib] = pixel_sim(sA1[c], sA2[c], sDp[c], sA1[q], sA2[q], sDp[q]);
            sBK[ib] = pixel_kl(sRf[c], sPf[c], sCf[c], sRf[q], sPf[q], sCf[q]);
          }
        }
        __syncthreads();
        row_sums(direct_val);
        __syncthreads();
        weights_of(hl * g.sws + wl);
        __syncthreads();
        const int dh = hu - g.wsh, dw = wu - g.wsh;
        row_sums([&](int h, int w) {
          if (h >= g.wsh && w >= g.wsh && w < g.hsim - g.wsh) {
            const int i = (h + dh) * g.hsim + (w + dw);
            return make_float2(sS[i], sK[i]);
          }
          const int ib = h < g.wsh ? h * g.hsim + w : top + (h - g.wsh) * band + (w < g.wsh ? w : w - g.hsim + band);
          return make_float2(sBS[ib], sBK[ib]);
        });
        __syncthreads();
        weights_of(hu * g.sws + wu);
        __syncthreads();
      }
  }
#pragma unroll
  for (int q = 0; q < kMaxPixPerThread; ++q) {
    const int pix = tid + q * kThreads;
    if (pix < npix) nols[(size_t)blockIdx.x * npix + pix] = s1[q] * s1[q] / s2[q];
  }
}

// std::priority_queue<weight_el> of smoothing.cpp: a binary heap whose top is
// the smallest weight; push sifts up, pop moves the last element into the hole
// left by sifting the top down to a leaf and sifts it up again.
struct DevHeap {
  float w[kMaxLmin];
  int idx[kMaxLmin];
  int n = 0;
  __device__ static bool before(float aw, float bw) { return aw > bw; }
  __device__ void sift_up(int hole, float vw, int vi) {
    int parent = (hole - 1) / 2;
    while (hole > 0 && before(w[parent], vw)) {
      w[hole] = w[parent];
      idx[hole] = idx[parent];
      hole = parent;
      parent = (hole - 1) / 2;
    }
    w[hole] = vw;
    idx[hole] = vi;
  }
  __device__ void push(float vw, int vi) {
    ++n;
    sift_up(n - 1, vw, vi);
  }
  __device__ void pop() {
    const int len = n - 1;
    const float vw = w[len];
    const int vi = idx[len];
    int hole = 0, child = 0;
    while (child < (len - 1) / 2) {
      child = 2 * (child + 1);
      if (before(w[child], w[child - 1])) --child;
      w[hole] = w[child];
      idx[hole] = idx[child];
      hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
      child = 2 * (child + 1);
      w[hole] = w[child - 1];
      idx[hole] = idx[child - 1];
      hole = child - 1;
    }
    sift_up(hole, vw, vi);
    n = len;
  }
};

__global__ void __launch_bounds__(kEstThreads)
    nlinsar_estimate_kernel(const float* __restrict__ a1, const float* __restrict__ fa, const float* __restrict__ fr,
                            const float* __restrict__ fi, const float* __restrict__ prf,
                            const float* __restrict__ ppf, const float* __restrict__ pcf, float* __restrict__ orf,
                            float* __restrict__ opf, float* __restrict__ ocf, NlGeom g, int tile0,
                            const float* __restrict__ wts, const float* __restrict__ nols) {
  const int npix = g.hori * g.hori;
  const int pix = blockIdx.x * kEstThreads + threadIdx.x;
  if (pix >= npix) return;
  const int tile = tile0 + blockIdx.y;
  const int ti = tile / g.ntx, tj = tile - ti * g.ntx;
  const int h0 = -g.ov + ti * g.step, w0 = -g.ov + tj * g.step;
  const int x = pix / g.hori, y = pix - x * g.hori;
  // the output pixel this tile position writes last, if any
  const int ry = ti * g.step + x, rx = tj * g.step + y;  // = h0 + ov + x, w0 + ov + y
  int oy, ox;
  if (ry < g.H - 1) oy = ry;
  else if (ti == g.nty - 1 && x == g.hori - 1) oy = g.H - 1;
  else return;
  if (rx < g.W - 1) ox = rx;
  else if (tj == g.ntx - 1 && y == g.hori - 1) ox = g.W - 1;
  else return;
  const int no = g.sws * g.sws;
  const float* wp = wts + (size_t)blockIdx.y * no * npix + pix;
  // smoothing (smoothing.cpp:65-117)
  int sel[kMaxLmin];
  int nsel = 0;
  float wmean = 0.0f;
  if (nols[(size_t)blockIdx.y * npix + pix] < (float)g.lmin) {
    DevHeap hp;
    const double as = a1[(size_t)clampn(h0 + x + g.ov, 0, g.H - 1) * g.W + clampn(w0 + y + g.ov, 0, g.W - 1)];
    for (int hh = 0; hh < g.sws; ++hh) {
      const int iy = clampn(h0 + x + g.ov + hh - g.wsh, 0, g.H - 1);
      for (int ww = 0; ww < g.sws; ++ww) {
        const float at = a1[(size_t)iy * g.W + clampn(w0 + y + g.ov + ww - g.wsh, 0, g.W - 1)];
        if (at < 2.0 * as) {
          const int k = hh * g.sws + ww;
          const float wk = wp[(size_t)k * npix];
          if (hp.n < g.lmin)
            hp.push(wk, k);
          else if (hp.w[0] < wk) {
            hp.pop();
            hp.push(wk, k);
          }
        }
      }
    }
    while (hp.n > 0) {
      wmean += hp.w[0];
      sel[nsel++] = hp.idx[0];
      hp.pop();
    }
    wmean /= (float)nsel;
    // ascending offsets for the merge below
    for (int i = 1; i < nsel; ++i) {
      const int v = sel[i];
      int j = i - 1;
      while (j >= 0 && sel[j] > v) {
        sel[j + 1] = sel[j];
        --j;
      }
      sel[j + 1] = v;
    }
  }
  // weighted means (compute_insar.cl:68-102)
  float N = 0.0f, A = 0.0f, Xr = 0.0f, Xi = 0.0f;
  int si = 0;
  for (int i = 0; i < g.sws; ++i) {
    const int iy = clampn(h0 + x + i + g.psh, 0, g.H - 1);
    for (int j = 0; j < g.sws; ++j) {
      const int k = i * g.sws + j;
      float wk = wp[(size_t)k * npix];
      if (si < nsel && sel[si] == k) {
        wk = wmean;
        ++si;
      }
      const size_t f = (size_t)iy * g.W + clampn(w0 + y + j + g.psh, 0, g.W - 1);
      N += wk;
      A += wk * fa[f];
      Xr += wk * fr[f];
      Xi += wk * fi[f];
    }
  }
  const float refl = A / N, phi = atan2f(Xi, Xr), coh = sqrtf(Xr * Xr + Xi * Xi) / A;
  const size_t o = (size_t)oy * g.W + ox;
  auto valid = [](float v) { return !(isnan(v) || isinf(v) || v == 0.0f); };
  orf[o] = valid(refl) ? refl : prf[o];
  if (valid(phi)) {
    float ph = phi;
    if (ph > 3.14159274101257324f) ph -= 2.0f * 3.14159274101257324f;
    if (ph < -3.14159274101257324f) ph += 2.0f * 3.14159274101257324f;
    opf[o] = ph;
  } else {
    opf[o] = ppf[o];
  }
  ocf[o] = valid(coh) ? fminf(1.0f, fmaxf(0.0f, coh)) : pcf[o];
}

size_t weights_smem(const NlGeom& g) {
  return ((size_t)6 * kTile * kTile + 2 * (size_t)g.hsim * g.hsim + 2 * (size_t)g.hsim * g.hori +
          (g.mirror ? 2 * (size_t)g.nborder : 0)) *
         sizeof(float);
}

int nlinsar_geom(int H, int W, int sws, int p, int lmin, NlGeom& g) {
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  if (sws < 1 || sws % 2 == 0 || p < 1 || p % 2 == 0)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "search window and patch sizes must be odd");
  if (p != 3 && p != 7)
    return set_error(DCL_ERR_UNSUPPORTED,
                     "patch size %d: the reference's h is tabulated for 3 and 7 only (other sizes draw it from an "
                     "unseeded simulation, nlinsar.cpp:60-69)",
                     p);
  if (lmin < 1 || lmin > kMaxLmin) return set_error(DCL_ERR_UNSUPPORTED, "lmin must be in [1, %d]", kMaxLmin);
  g.H = H;
  g.W = W;
  g.sws = sws;
  g.wsh = (sws - 1) / 2;
  g.p = p;
  g.psh = (p - 1) / 2;
  g.ov = g.wsh + g.psh;
  g.hsim = kTile - sws + 1;
  g.hori = kTile - 2 * g.ov;
  // mirrored maps need an interior (rows from wsh, columns wsh .. hsim-wsh-1)
  // and room for the mirror's border values
  g.nborder = g.wsh * g.hsim + (g.hsim - g.wsh) * 2 * g.wsh;
  g.mirror = 2 * g.wsh < g.hsim ? 1 : 0;
  if (g.mirror && weights_smem(g) > 227 * 1024) g.mirror = 0;
  if (g.hori < 1) return set_error(DCL_ERR_UNSUPPORTED, "search window and patch too large for the 80 x 80 tiles");
  if ((g.hori * g.hori + kThreads - 1) / kThreads > kMaxPixPerThread || weights_smem(g) > 227 * 1024)
    return set_error(DCL_ERR_UNSUPPORTED, "search window %d with patch %d: tile state exceeds shared memory", sws, p);
  g.step = kTile - 2 * g.ov;
  g.nty = 0;
  for (int h0 = -g.ov; h0 < H; h0 += g.step) ++g.nty;
  g.ntx = 0;
  for (int w0 = -g.ov; w0 < W; w0 += g.step) ++g.ntx;
  g.lmin = lmin;
  const int area = p * p;
  const float h_theo = p == 3 ? 0.58f : 0.244f;
  g.h = h_theo * area;
  g.T = (float)(2.0 / g.h * M_PI / 4 * area);
  return DCL_OK;
}

}  // namespace

int nlinsar_check(int H, int W, int sws, int p, int lmin) {
  NlGeom g;
  return nlinsar_geom(H, W, sws, p, lmin, g);
}

// ref / phase / coh: initial estimates on entry, results on exit (device).
int nlinsar_device(const float* a1, const float* a2, const float* dp, float* ref, float* phase, float* coh, int H,
                   int W, int sws, int p, int niter, int lmin, cudaStream_t st) {
  if (!a1 || !a2 || !dp || !ref || !phase || !coh) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (niter < 0) return set_error(DCL_ERR_INVALID_ARGUMENT, "niter must be >= 0");
  {
    int dev = 0;
    const int rc0 = ensure_device_ready(dev);
    if (rc0) return rc0;
  }
  NlGeom g;
  int rc = nlinsar_geom(H, W, sws, p, lmin, g);
  if (rc) return rc;
  if (niter == 0) return DCL_OK;
  const size_t n = (size_t)H * W;
  const int ntiles = g.ntx * g.nty;
  const size_t npix = (size_t)g.hori * g.hori, no = (size_t)sws * sws;
  const size_t per_tile = (no * npix + npix) * sizeof(float);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(ntiles, ((size_t)4 << 30) / per_tile));
  float* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, (6 * n) * sizeof(float) + (size_t)chunk * per_tile, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(NL-InSAR)");
  float *fa = buf, *fr = fa + n, *fi = fr + n, *tr = fi + n, *tp = tr + n, *tc = tp + n;
  float* wts = tc + n;
  float* nols = wts + (size_t)chunk * no * npix;
  const size_t smem = weights_smem(g);
  e = cudaFuncSetAttribute(nlinsar_weights_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    nlinsar_filter_values_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a1, a2, dp, fa, fr, fi, n);
    profile_count(1);
    // estimates ping-pong between the caller's planes and tr/tp/tc; an odd
    // number of passes ends in tr/tp/tc and is copied back
    float* cur[3] = {ref, phase, coh};
    float* nxt[3] = {tr, tp, tc};
    for (int it = 0; it < niter; ++it) {
      for (int t0 = 0; t0 < ntiles; t0 += chunk) {
        const int nt = std::min(chunk, ntiles - t0);
        nlinsar_weights_kernel<<<nt, kThreads, smem, st>>>(a1, a2, dp, cur[0], cur[1], cur[2], g, t0, wts, nols);
        dim3 grid((unsigned)((npix + kEstThreads - 1) / kEstThreads), nt);
        nlinsar_estimate_kernel<<<grid, kEstThreads, 0, st>>>(a1, fa, fr, fi, cur[0], cur[1], cur[2], nxt[0], nxt[1],
                                                              nxt[2], g, t0, wts, nols);
        profile_count(2);
      }
      std::swap(cur, nxt);
    }
    if (cur[0] != ref)
      for (int d = 0; d < 3 && e == cudaSuccess; ++d)
        e = cudaMemcpyAsync(d == 0 ? ref : (d == 1 ? phase : coh), cur[d], n * sizeof(float),
                            cudaMemcpyDeviceToDevice, st);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_error(e, "NL-InSAR");
  return DCL_OK;
}

}  // namespace dcl

extern "C" int dcl_nlinsar_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                                  float* coh, int H, int W, int search_window_size, int patch_size, int niter, int lmin,
                                  void* stream) {
  return dcl::nlinsar_device(a1, a2, phi, ref, phase, coh, H, W, search_window_size, patch_size, niter, lmin,
                             (cudaStream_t)stream);
}

extern "C" int dcl_nlinsar(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                           int H, int W, int search_window_size, int patch_size, int niter, int lmin) {
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  const int vr = dcl::nlinsar_check(H, W, search_window_size, patch_size, lmin);
  if (vr) return vr;
  if (niter < 0) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "niter must be >= 0");
  cudaStream_t st = cudaStreamPerThread;
  const size_t n = (size_t)H * W, b = n * sizeof(float);
  float* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, 6 * b, st);
  if (e != cudaSuccess) return dcl::cuda_error(e, "cudaMallocAsync(NL-InSAR)");
  const float* hin[6] = {a1, a2, phi, ref, phase, coh};
  for (int d = 0; d < 6 && e == cudaSuccess; ++d)
    e = cudaMemcpyAsync(buf + d * n, hin[d], b, cudaMemcpyHostToDevice, st);
  int rc = DCL_OK;
  if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(H2D)");
  if (rc == DCL_OK)
    rc = dcl::nlinsar_device(buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, buf + 5 * n, H, W,
                             search_window_size, patch_size, niter, lmin, st);
  if (rc == DCL_OK) {
    float* hout[3] = {ref, phase, coh};
    for (int d = 0; d < 3 && e == cudaSuccess; ++d)
      e = cudaMemcpyAsync(hout[d], buf + (3 + d) * n, b, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(D2H)");
  }
  cudaFreeAsync(buf, st);
  e = cudaStreamSynchronize(st);
  if (rc == DCL_OK && e != cudaSuccess) rc = dcl::cuda_error(e, "NL-InSAR");
  return rc;
}

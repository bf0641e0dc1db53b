// NL-SAR on 3x3 (PolSAR) covariance images: despeckcl::nlsar with dim = 3
// (src/compute/nlsar/nlsar.cpp:171-194 in the reference, the same per-tile
// pipeline as the 2x2 case, nlsar_filter_sub_image.cpp:146-390) and
// despeckcl::nlsar_training on such images (training/get_dissims.cpp,
// training/patches.cpp:43-136).
//
// Differences from the 2x2 path, all following the reference (paths relative
// to src/compute/nlsar/):
//  * the covariance has 18 planes, plane 2(r*3+c) the real and 2(r*3+c)+1
//    the imaginary part of element (r, c);
//  * the rescale factor is (1/3)^0.33333 (cl_kernels/covmat_rescale.cl:25-26);
//  * the pixel similarity is the 3x3 GLR of
//    cl_kernels/compute_pixel_similarities_3x3.cl.in with
//    sim_measures.h:66-160 (Leibniz determinant of a Hermitian matrix from its
//    diagonal and upper triangle);
//  * statistics and alpha run over the three diagonal intensities
//    (cl_kernels/compute_nl_statistics.cl, compute_alphas.cl);
//  * the weighted means cover all 18 planes (cl_kernels/weighted_means.cl).
//
// Layout: the padded frame of the 2x2 engine (virtual plane, clamp padding),
// stored planar: c18 [18][Hp][pitch] (un-rescaled covariance) and, per scale,
// s9 [9][Hp][pitch] (the nine similarity reals of the rescaled, Gaussian-
// averaged covariance: a00, a11, a22, Re/Im a01, Re/Im a02, Re/Im a12) plus
// ld [Hp][pitch] (their ln det).  The fused kernel keeps one 32 x 8 output tile
// per CTA (one pixel per thread): per offset batch it computes the
// similarities of the tile plus patch halo from the staged s9 region, the
// horizontal sums of every patch size of the pass, then per pixel the
// vertical sums, the composite LUT weight and 23 accumulators per patch size
// (sum w, w^2, w I_d^2 for d = 0..2, and w times each of the 18 planes, read
// through the L1 cache); the epilogue derives ENL, alpha and ENL', selects and
// blends with the centre pixel.  Search 21 with patches {3,5,7} (or one of
// them) runs nlsar3_fast_kernel instead, which splits each pixel's
// accumulators over two threads.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_common.cuh"
#include "nlsar_plan.h"
#include "stats_internal.h"

namespace dcl {

std::vector<float> gauss_weights(int s);

namespace {

constexpr int kT3W = 32;        // output columns per tile (one lane per column)
constexpr int kT3Warps = 8;     // warps per CTA, one output row each
constexpr int kT3H = kT3Warps;  // output rows per tile
constexpr int kT3Threads = 32 * kT3Warps;
constexpr int kNA3 = 23;        // accumulators per patch size

// planes of the nine similarity reals within the 18 covariance planes
__host__ __device__ constexpr int sim_plane(int k) {
  return k == 0 ? 0 : k == 1 ? 8 : k == 2 ? 16 : k == 3 ? 2 : k == 4 ? 3 : k == 5 ? 4 : k == 6 ? 5 : k == 7 ? 10 : 11;
}
// planes of the diagonal intensities
__host__ __device__ constexpr int diag_plane(int d) { return 8 * d; }

__device__ __forceinline__ int clamp3(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sim_measures.h:78-97 with a = {a00, a11, a22, Re a01, Im a01, Re a02, Im a02, Re a12, Im a12}
__host__ __device__ __forceinline__ float det3f(const float* a) {
  return a[0] * a[1] * a[2] - a[0] * (a[7] * a[7] + a[8] * a[8]) - a[1] * (a[5] * a[5] + a[6] * a[6]) -
         a[2] * (a[3] * a[3] + a[4] * a[4]) +
         2.0f * (a[3] * a[7] * a[5] - a[4] * a[8] * a[5] + a[3] * a[8] * a[6] + a[4] * a[7] * a[6]);
}

struct Scene3 {
  const float* c18;             // [18][Hp][pitch]
  const float* s9[kMaxScales];  // [9][Hp][pitch] per scale slot
  const float* ld[kMaxScales];  // [Hp][pitch] per scale slot
  float* out;                   // [18][H][W]
  int H, W, vH, vW, pitch, tiles_x;
  int tile_skip;                // scene tiles before block 0 of the launch (row bands)
  size_t plane;                 // Hp * pitch
};

struct Smem3 {
  int rs_w, rs_h, sim_w, sim_h;
  int off_ld, off_sim, off_h, off_w, total;  // in 4-byte words; s9 planes start at 0
};

__host__ __device__ inline Smem3 smem3_layout(int wsh, int phm, int K) {
  Smem3 L;
  L.rs_w = kT3W + 2 * (phm + wsh);
  L.rs_h = kT3H + 2 * (phm + wsh);
  L.sim_w = kT3W + 2 * phm;
  L.sim_h = kT3H + 2 * phm;
  int o = 9 * L.rs_w * L.rs_h;
  L.off_ld = o;
  o += L.rs_w * L.rs_h;
  L.off_sim = o;
  o += K * L.sim_w * L.sim_h;
  L.off_h = o;
  o += K * kPatchPerPass * L.sim_h * kT3W;
  L.off_w = o;
  o += kPatchPerPass * kMaxLut;
  L.total = o;
  return L;
}

// 18 planes of the clamp-padded frame (sub_images.cpp:37-38 clamping)
__global__ void prep3_cov_kernel(const float* __restrict__ cin, int H, int W, float* __restrict__ c18, int Hp, int Wp,
                                 int pitch, size_t plane, int G, int row0, int row1) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= Wp || py >= row1) return;
  const int y = clamp3(py - G, 0, H - 1), x = clamp3(px - G, 0, W - 1);
  const size_t n = (size_t)H * W, i = (size_t)y * W + x, o = (size_t)py * pitch + px;
#pragma unroll
  for (int p = 0; p < 18; ++p) c18[p * plane + o] = cin[p * n + i];
}

// rescaled (off-diagonals x gamma, covmat_rescale.cl:31-39) and Gaussian
// averaged (covmat_spatial_avg.cl:50-57) similarity planes of one scale, and
// their ln det
__global__ void prep3_scale_kernel(const float* __restrict__ c18, int Hp, int Wp, int pitch, size_t plane, int s,
                                   GaussArg ga, float gamma, float* __restrict__ s9, float* __restrict__ ld, int row0,
                                   int row1) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= Wp || py >= row1) return;
  const int ssh = (s - 1) / 2;
  float a[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) a[k] = 0.0f;
  for (int kx = 0; kx < s; ++kx) {
    const int yy = clamp3(py - ssh + kx, 0, Hp - 1);
    for (int ky = 0; ky < s; ++ky) {
      const int xx = clamp3(px - ssh + ky, 0, Wp - 1);
      const size_t q = (size_t)yy * pitch + xx;
      const float g = ga.g[kx * s + ky];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const float v = c18[sim_plane(k) * plane + q];
        a[k] = fmaf(g, k >= 3 ? v * gamma : v, a[k]);
      }
    }
  }
  const size_t o = (size_t)py * pitch + px;
#pragma unroll
  for (int k = 0; k < 9; ++k) s9[k * plane + o] = a[k];
  ld[o] = logf(det3f(a));
}

__device__ __forceinline__ void offset3_of(int t, int sws, int wsh, int& dy, int& dx, bool& lower) {
  // pairs: upper-half slot u of the reference's half-window volume
  // (compute_pixel_similarities_3x3: quadrants as the 2x2 wrapper), then its
  // mirror -u (copy_symm_weights.cl:56-76)
  const int u = t >> 1;
  const int hh = u / sws, ww = u - hh * sws;
  dy = hh - wsh;
  dx = ww - wsh;
  lower = (t & 1) != 0;
  if (lower) {
    dy = -dy;
    dx = -dx;
  }
}

__global__ void __launch_bounds__(kT3Threads, 1) nlsar3_kernel(const FilterParams P, const Scene3 S) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int tid = threadIdx.x, lane = tid & 31, y = tid >> 5;
  const int wsh = P.wsh, phm = P.phm, sws = P.sws, G = P.G;
  const Smem3 L = smem3_layout(wsh, phm, P.K);
  const int rsn = L.rs_w * L.rs_h;
  float* sS = smem;
  float* sLd = smem + L.off_ld;
  float* sSim = smem + L.off_sim;
  float* sH = smem + L.off_h;
  float* sW = smem + L.off_w;
  const int lt = blockIdx.x + S.tile_skip;
  const int ty = lt / S.tiles_x, tx = lt - ty * S.tiles_x;
  const int vy0 = ty * kT3H, vx0 = tx * kT3W;
  // frame index of this thread's output pixel
  const size_t cfi = (size_t)(vy0 + y + G) * S.pitch + (vx0 + lane + G);

  float acc[kPatchPerPass][kNA3];
  float best_e = -1.0f, best_a = 0.0f, best_s0 = 1.0f, best_m[18];
  int best_rank = 0x7fffffff, best_combo = -1;
#pragma unroll
  for (int p = 0; p < 18; ++p) best_m[p] = 0.0f;

  int loaded_slot = -1;
  for (int ps = 0; ps < P.npass; ++ps) {
    const PassParams& pp = P.pass[ps];
    const int np = pp.np;
    __syncthreads();
    if (pp.scale_slot != loaded_slot) {
      const float* s9 = S.s9[pp.scale_slot];
      const float* ldp = S.ld[pp.scale_slot];
      const int by = vy0 - phm - wsh + G, bx = vx0 - phm - wsh + G;
      for (int i = tid; i < rsn; i += kT3Threads) {
        const int r = i / L.rs_w, c = i - r * L.rs_w;
        const size_t g = (size_t)(by + r) * S.pitch + (bx + c);
#pragma unroll
        for (int k = 0; k < 9; ++k) sS[k * rsn + i] = s9[k * S.plane + g];
        sLd[i] = ldp[g];
      }
      loaded_slot = pp.scale_slot;
    }
    for (int i = tid; i < np * kMaxLut; i += kT3Threads) {
      const int j = i / kMaxLut;
      sW[i] = P.wtab[pp.combo[j] * kMaxLut + (i - j * kMaxLut)];
    }
#pragma unroll
    for (int j = 0; j < kPatchPerPass; ++j)
#pragma unroll
      for (int a = 0; a < kNA3; ++a) acc[j][a] = 0.0f;
    __syncthreads();

    const int K = P.K;
    for (int t0 = 0; t0 < P.n_off; t0 += K) {
      const int kb = min(K, P.n_off - t0);
      // ---- A: 3x3 similarities of the batch on the tile + patch halo
      const int nsim = L.sim_w * L.sim_h;
      for (int i = tid; i < kb * nsim; i += kT3Threads) {
        const int k = i / nsim;
        const int rem = i - k * nsim;
        const int r = rem / L.sim_w, c = rem - r * L.sim_w;
        int dy, dx;
        bool lower;
        offset3_of(t0 + k, sws, wsh, dy, dx, lower);
        const int ci = (r + wsh) * L.rs_w + (c + wsh);
        const int ni = ci + dy * L.rs_w + dx;
        float sum[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) sum[q] = sS[q * rsn + ci] + sS[q * rsn + ni];
        const float det = det3f(sum);
        const float la = sLd[ci], lb = sLd[ni];
        // the mirrored half takes the neighbour as the first argument
        // (copy_symm_weights.cl:66-74)
        const float t = lower ? (P.c2d + lb) + la : (P.c2d + la) + lb;
        float sim = -(t - 2.0f * logf(det));
        if (sim != sim) sim = 0.0f;
        sSim[i] = sim;
      }
      __syncthreads();
      // ---- B: horizontal sums for every patch size of the pass (nested rings)
      const int nh = L.sim_h * kT3W;
      for (int i = tid; i < kb * nh; i += kT3Threads) {
        const int k = i / nh;
        const int rem = i - k * nh;
        const int r = rem / kT3W, c = rem - r * kT3W;
        const float* row = sSim + k * nsim + r * L.sim_w + c + phm;
        float sacc = row[0];
        int b = 0;
#pragma unroll
        for (int j = 0; j < kPatchPerPass; ++j) {
          if (j < np) {
            const int ph = pp.ph[j];
            for (; b < ph;) {
              ++b;
              sacc += row[-b] + row[b];
            }
            sH[((k * kPatchPerPass + j) * L.sim_h + r) * kT3W + c] = sacc;
          }
        }
      }
      __syncthreads();
      // ---- C: vertical sums, weights, accumulation
      for (int k = 0; k < kb; ++k) {
        int dy, dx;
        bool lower;
        offset3_of(t0 + k, sws, wsh, dy, dx, lower);
        const size_t nfi = cfi + (ptrdiff_t)dy * S.pitch + dx;
        float v[18];
#pragma unroll
        for (int p = 0; p < 18; ++p) v[p] = __ldg(S.c18 + p * S.plane + nfi);
        float i2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) i2[d] = v[diag_plane(d)] * v[diag_plane(d)];
#pragma unroll
        for (int j = 0; j < kPatchPerPass; ++j) {
          if (j < np) {
            const int ph = pp.ph[j];
            const ComboParams& cp = P.combo[pp.combo[j]];
            const float* col = sH + ((k * kPatchPerPass + j) * L.sim_h) * kT3W + lane;
            float d = 0.0f;
            for (int a = -ph; a <= ph; ++a) d += col[(y + phm + a) * kT3W];
            // compute_weights.cl:40-51 through the composite weight table
            float w;
            if (d > cp.dmax) {
              w = 0.0f;
            } else {
              float dc = fmaxf(d, cp.dmin);
              dc = fminf(dc, cp.dmax);
              const float mapped = __fdiv_rn(dc - cp.dmin, cp.span) * cp.lm1;
              w = sW[j * kMaxLut + (unsigned)mapped];
            }
            float* A = acc[j];
            A[0] += w;
            A[1] = fmaf(w, w, A[1]);
#pragma unroll
            for (int q = 0; q < 3; ++q) A[2 + q] = fmaf(w, i2[q], A[2 + q]);
#pragma unroll
            for (int p = 0; p < 18; ++p) A[5 + p] = fmaf(w, v[p], A[5 + p]);
          }
        }
      }
      __syncthreads();
    }

    // ---- centre weight 1 (routines.cpp:151-157), statistics, alpha, ENL', selection
    float c[18];
#pragma unroll
    for (int p = 0; p < 18; ++p) c[p] = __ldg(S.c18 + p * S.plane + cfi);
#pragma unroll
    for (int j = 0; j < kPatchPerPass; ++j) {
      if (j < np) {
        const float* A = acc[j];
        const float s0 = A[0] + 1.0f, s1 = A[1] + 1.0f;
        // compute_nl_statistics.cl:92-101 over the three diagonal intensities
        const float enl = s0 * s0 / s1;
        float alpha = 0.0f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float cd = c[diag_plane(d)];
          const float in = (A[5 + diag_plane(d)] + cd) / s0;
          const float var = (A[2 + d] + cd * cd) / s0 - in * in;
          // compute_alphas.cl:30-41 (nlooks = 1)
          alpha = fmaxf(alpha, fmaxf(0.0f, (var - in * in) / var));
        }
        if (P.alpha_zero) alpha = 0.0f;
        // compute_enls_nobias.cl:19-22
        const float oma = 1.0f - alpha;
        const float enb = enl / (oma * oma + (alpha * alpha + 2.0f * alpha * (1.0f - alpha) / s0) * enl);
        const int combo = pp.combo[j];
        const int rank = P.combo[combo].rank;
        const bool take = (P.select_mode == 0) || (enb > best_e) || (enb == best_e && rank < best_rank);
        const bool take_fb = !take && best_combo < 0 && combo == P.fallback_combo;
        if (take) {
          best_e = enb;
          best_rank = rank;
        }
        if (take || take_fb) {
          best_combo = combo;
          best_a = alpha;
          best_s0 = s0;
#pragma unroll
          for (int p = 0; p < 18; ++p) best_m[p] = A[5 + p] + c[p];
        }
      }
    }
  }

  // ---- blend with the centre (weighted_means.cl:79), store the 18 planes
  const int vy = vy0 + y, vx = vx0 + lane;
  const int oy = (vy < S.H - 1) ? vy : (vy == S.vH ? S.H - 1 : -1);
  const int ox = (vx < S.W - 1) ? vx : (vx == S.vW ? S.W - 1 : -1);
  if (oy < 0 || ox < 0) return;
  const size_t n = (size_t)S.H * S.W, o = (size_t)oy * S.W + ox;
  const float oma = 1.0f - best_a;
#pragma unroll
  for (int p = 0; p < 18; ++p) {
    const float cp = __ldg(S.c18 + p * S.plane + cfi);
    S.out[p * n + o] = oma * best_m[p] / best_s0 + best_a * cp;
  }
}

// ---- specialised kernel: search window 21, patches {3,5,7} or one of them,
// or {3,5,7} and {9,11} per scale ---------------------------------------------
//
// Same tile (32 x 8 outputs) and the same phases as nlsar3_kernel, with the
// window and patch sizes fixed at compile time and two threads per output
// pixel: warps 0-7 (group 0) and 8-15 (group 1) own the same 8 rows.  The
// two groups share the weights of each offset batch through shared memory,
// each computing half of them; group 0 keeps sum w, sum w^2, sum w I_d^2 and
// the weighted sums of the diagonal and upper-triangle planes (14
// accumulators per patch size), group 1 those of the other nine planes, so a
// thread holds at most 42 accumulators and the CTA runs 16 warps.  Group 0
// selects; its choice reaches group 1 through shared memory once per pass.
// Offsets run in window rows seven (with patches up to 11: three) at a time
// as in the 2x2 specialised kernel; the tile is staged for the call's largest
// patch, a pass with smaller patches reading its region further in; the measure is evaluated symmetrically in its two pixels
// ((ln det A + ln det B) first), the index of the composite weight by a
// saturating FMA and a round-toward-zero add (the reference's `(unsigned)`
// truncation), and the centre offset has weight 1 inside the sweep.

// planes accumulated by each group: group 0 the diagonal (0, 8, 16) and the
// upper triangle, group 1 the rest
__host__ __device__ constexpr int group_plane(int g, int q) {
  return g == 0 ? (q == 0 ? 0 : q == 1 ? 2 : q == 2 ? 3 : q == 3 ? 4 : q == 4 ? 5 : q == 5 ? 8 : q == 6 ? 10
                                                                                                        : q == 7 ? 11
                                                                                                                 : 16)
                : (q == 0 ? 1 : q == 1 ? 6 : q == 2 ? 7 : q == 3 ? 9 : q == 4 ? 12 : q == 5 ? 13 : q == 6 ? 14
                                                                                                        : q == 7 ? 15
                                                                                                                 : 17);
}
// position of diagonal d within group 0's planes
__host__ __device__ constexpr int diag_slot(int d) { return d == 0 ? 0 : d == 1 ? 5 : 8; }

// Shared-memory layout of the specialised 3x3 kernel: staging halo PHX_ (the
// call's largest patch half), at most NPX_ patch sizes per pass.
template <int PHX_, int NPX_>
struct Fast3 {
  static constexpr int WSH = 10, PHX = PHX_, NPX = NPX_;
  static constexpr int TH = kT3H, TW = kT3W;
  static constexpr int THREADS = 2 * 32 * TH;  // two groups of one warp per row
  // offsets per batch along a window row: seven with the small halo, three
  // with the large one, which keeps L1 room for the neighbour planes
  static constexpr int K = PHX <= 3 ? 7 : 3;
  static constexpr int NA = 14;                // accumulators per patch size (group 1 uses 9)
  static constexpr int RS = TW + 2 * (PHX + WSH), RSH = TH + 2 * (PHX + WSH);
  static constexpr int RN = RS * RSH;
  static constexpr int SIMWX = TW + 2 * PHX, SIMHX = TH + 2 * PHX;
  static constexpr int SIMPX = (SIMWX + 7) / 8 * 8;
  static constexpr int HPL = K * SIMHX * TW;  // one patch size's horizontal-sum plane
  static constexpr int LUTREP = 8;            // interleaved LUT copies (four lanes per copy)
  static constexpr int OFF_S9 = 0;            // [9][RSH][RS]
  static constexpr int OFF_LD = OFF_S9 + 9 * RN;
  static constexpr int OFF_SIM = OFF_LD + RN;  // [K][SIMH][SIMP]
  static constexpr int OFF_H = OFF_SIM + K * SIMHX * SIMPX;
  static constexpr int OFF_LUT = OFF_H + NPX * HPL;
  static constexpr int OFF_W = OFF_LUT + NPX * kMaxLut * LUTREP;  // [K][NPX][32 TH] weights of a batch
  static constexpr int OFF_X = OFF_W + K * NPX * 32 * TH;          // group 0 -> group 1: take, alpha, s0
  static constexpr int WORDS = OFF_X + 3 * 32 * TH;
  static_assert((2 * WSH + 1) % K == 0, "offset batches must tile a window row");
  static_assert(WORDS * 4 <= 227 * 1024, "shared memory");
};

template <int PH0, int PH1, int PH2>
__device__ __forceinline__ constexpr int ph3_of(int j) {
  return j == 0 ? PH0 : (j == 1 ? PH1 : PH2);
}

template <int PH0, int PH1, int PH2>
__host__ __device__ constexpr int np3_of() {
  return (PH0 >= 0) + (PH1 >= 0) + (PH2 >= 0);
}

__host__ __device__ constexpr int cmax3(int a, int b) { return a > b ? a : b; }

// Selection state of one thread's pixel: group 0 keeps the weighted sums of
// its nine planes and decides; group 1 keeps its nine planes' sums.
struct Best3 {
  float m[9];
  float e, a, s0;
  int rank, combo;
};

// One pass (one scale, patch halves PH0 < PH1 < PH2, -1 unused) of the 3x3
// kernel over all offsets on the staged tile; a pass with smaller patches
// than the call's largest reads its region CO pixels further in.
template <class L, int PH0, int PH1, int PH2>
__device__ __forceinline__ void fast3_pass(const FilterParams& P, const PassParams& pp, float* smem, const Scene3& S,
                                           size_t cfi, Best3& best) {
  constexpr int WSH = L::WSH, K = L::K, NA = L::NA, RS = L::RS, RN = L::RN, TW = L::TW, NT = L::THREADS;
  constexpr int NP = np3_of<PH0, PH1, PH2>();
  constexpr int PHM = cmax3(PH0, cmax3(PH1, PH2));
  constexpr int CO = L::PHX - PHM;
  constexpr int SIMW = TW + 2 * PHM, SIMH = L::TH + 2 * PHM;
  constexpr int SIMP = (SIMW + 7) / 8 * 8;
  constexpr int NQ4 = (4 + 2 * PHM + 3) / 4;
  static_assert(PH0 >= 1 && NP <= L::NPX && CO >= 0, "pass shape");
  static_assert(SIMP >= 4 * 7 + 4 * NQ4 && SIMP <= L::SIMPX, "phase-B segments must stay inside a row");
  const float* sS9 = smem + L::OFF_S9;
  const float* sLd = smem + L::OFF_LD;
  float* sSim = smem + L::OFF_SIM;
  float* sH = smem + L::OFF_H;
  float* sLut = smem + L::OFF_LUT;
  float* sW = smem + L::OFF_W;
  int* sTake = reinterpret_cast<int*>(smem + L::OFF_X);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp / L::TH, y = warp - grp * L::TH;  // warp-uniform group, output row
  const int px = y * 32 + lane;
  const float c2d = P.c2d;

  for (int i = tid; i < NP * kMaxLut * L::LUTREP; i += NT) {
    const int j = i / (kMaxLut * L::LUTREP);
    const int e = (i - j * kMaxLut * L::LUTREP) / L::LUTREP;
    sLut[i] = P.wtab[pp.combo[j] * kMaxLut + e];
  }
  float inv_span[NP], nbias[NP], lm1[NP], dmax[NP];
  const float* lut_j[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const ComboParams& cp = P.combo[pp.combo[j]];
    inv_span[j] = 1.0f / cp.span;
    nbias[j] = -cp.dmin * inv_span[j];
    lm1[j] = cp.lm1;
    dmax[j] = cp.dmax;
    lut_j[j] = sLut + j * kMaxLut * L::LUTREP + (lane & (L::LUTREP - 1));
  }
  static_assert(NA % 2 == 0, "accumulators in pairs");
  float2 acc[NP][NA / 2];  // accumulator a of patch j: component a % 2 of acc[j][a / 2]
#pragma unroll
  for (int j = 0; j < NP; ++j)
#pragma unroll
    for (int a = 0; a < NA / 2; ++a) acc[j][a] = make_float2(0.0f, 0.0f);
  __syncthreads();

  for (int dy = -WSH; dy <= WSH; ++dy) {
    for (int dx0 = -WSH; dx0 <= WSH; dx0 += K) {
      // ---- A: 3x3 similarities of offsets (dy, dx0..dx0+K-1) on the tile
      // plus patch halo (sim_measures.h:66-160), one pixel per item
      for (int it = tid; it < SIMH * SIMP; it += NT) {
        const int r = it / SIMP;
        const int c = it - r * SIMP;
        if (c >= SIMW) continue;
        const int ci = (r + WSH + CO) * RS + (c + WSH + CO);
        float a[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) a[q] = sS9[q * RN + ci];
        const float la = sLd[ci];
        const int ni = ci + dy * RS + dx0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          float sum[9];
#pragma unroll
          for (int q = 0; q < 9; ++q) sum[q] = a[q] + sS9[q * RN + ni + k];
          const float t = (la + sLd[ni + k]) + c2d;
          float sim = fmaf(2.0f * 0.69314718f, __log2f(det3f(sum)), -t);
          if (sim != sim) sim = 0.0f;
          sSim[k * SIMH * SIMP + it] = sim;
        }
      }
      __syncthreads();
      // ---- B: horizontal sums of every patch size (nested rings), 4 output
      // columns per item, a quarter warp per row
      {
        constexpr int QUADS = (SIMH + 3) / 4;
        const int r_off = lane >> 3, seg = lane & 7;
        for (int q = warp; q < K * QUADS; q += NT / 32) {
          const int k = q / QUADS;
          const int r = (q - k * QUADS) * 4 + r_off;
          if (r < SIMH) {
            const float4* row = reinterpret_cast<const float4*>(sSim + (k * SIMH + r) * SIMP + 4 * seg);
            float s[4 * NQ4];
#pragma unroll
            for (int q4 = 0; q4 < NQ4; ++q4) {
              const float4 v = row[q4];
              s[4 * q4] = v.x;
              s[4 * q4 + 1] = v.y;
              s[4 * q4 + 2] = v.z;
              s[4 * q4 + 3] = v.w;
            }
            float hs[NP][4];
#pragma unroll
            for (int o = 0; o < 4; ++o) {
              float h[3] = {0.f, 0.f, 0.f};
              float ring = s[o + PHM];
#pragma unroll
              for (int b = 1; b <= PHM; ++b) {
                ring += s[o + PHM - b] + s[o + PHM + b];
#pragma unroll
                for (int j = 0; j < 3; ++j)
                  if (ph3_of<PH0, PH1, PH2>(j) == b) h[j] = ring;
              }
#pragma unroll
              for (int j = 0; j < NP; ++j) hs[j][o] = h[j];
            }
#pragma unroll
            for (int j = 0; j < NP; ++j)
              *reinterpret_cast<float4*>(sH + j * L::HPL + (k * SIMH + r) * TW + 4 * seg) =
                  make_float4(hs[j][0], hs[j][1], hs[j][2], hs[j][3]);
          }
        }
      }
      __syncthreads();
      // ---- C1: vertical sums and weights, each computed once: group g
      // takes the offsets k = g, g + 2, ... of the batch for its row and
      // leaves them in shared memory for both groups
#pragma unroll
      for (int k = 0; k < K; ++k) {
        if ((k & 1) != grp) continue;
        const int dx = dx0 + k;
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const int ph = ph3_of<PH0, PH1, PH2>(j);
          const float* col = sH + j * L::HPL + (k * SIMH + y + PHM - ph) * TW + lane;
          float d = col[0];
#pragma unroll
          for (int a = 1; a <= 2 * ph3_of<PH0, PH1, PH2>(j); ++a) d += col[a * TW];
          // compute_weights.cl:40-51 through the composite weight table
          const float u = __saturatef(fmaf(d, inv_span[j], nbias[j]));
          const float t = __fmaf_rz(u, lm1[j], 8388608.0f);
          const int idx = __float_as_int(t) - 0x4B000000;
          const float lw = lut_j[j][idx * L::LUTREP];
          float w = (d > dmax[j]) ? 0.0f : lw;
          if (dy == 0 && dx == 0) w = 1.0f;
          sW[(k * NP + j) * (32 * L::TH) + px] = w;
        }
      }
      __syncthreads();
      // ---- C2: this group's accumulators, offsets in order
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int dx = dx0 + k;
        float w[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) w[j] = sW[(k * NP + j) * (32 * L::TH) + px];
        const size_t nfi = cfi + (ptrdiff_t)dy * S.pitch + dx;
        float v[9];
#pragma unroll
        for (int q = 0; q < 9; ++q)
          v[q] = __ldg(S.c18 + (grp == 0 ? group_plane(0, q) : group_plane(1, q)) * S.plane + nfi);
        if (grp == 0) {
          float i2[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) i2[d] = v[diag_slot(d)] * v[diag_slot(d)];
          // accumulators that share the weight, two per packed (f32x2) FMA,
          // each lane rounded like the scalar FMA; sum w as fma(w, 1, sum),
          // which equals sum + w
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            const float2 ww = make_float2(w[j], w[j]);
            float2* A = acc[j];
            A[0] = __ffma2_rn(ww, make_float2(1.0f, w[j]), A[0]);  // sum w, sum w^2
            A[1] = __ffma2_rn(ww, make_float2(i2[0], i2[1]), A[1]);
            A[2] = __ffma2_rn(ww, make_float2(i2[2], v[0]), A[2]);
            A[3] = __ffma2_rn(ww, make_float2(v[1], v[2]), A[3]);
            A[4] = __ffma2_rn(ww, make_float2(v[3], v[4]), A[4]);
            A[5] = __ffma2_rn(ww, make_float2(v[5], v[6]), A[5]);
            A[6] = __ffma2_rn(ww, make_float2(v[7], v[8]), A[6]);
          }
        } else {
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            const float2 ww = make_float2(w[j], w[j]);
            float2* A = acc[j];
            A[0] = __ffma2_rn(ww, make_float2(v[0], v[1]), A[0]);
            A[1] = __ffma2_rn(ww, make_float2(v[2], v[3]), A[1]);
            A[2] = __ffma2_rn(ww, make_float2(v[4], v[5]), A[2]);
            A[3] = __ffma2_rn(ww, make_float2(v[6], v[7]), A[3]);
            A[4].x = fmaf(w[j], v[8], A[4].x);
          }
        }
      }
    }
  }

  // ---- statistics over the three diagonal intensities, alpha, ENL',
  // selection (compute_nl_statistics.cl:92-101, compute_alphas.cl:30-41,
  // compute_enls_nobias.cl:19-22, best_params.cpp); group 0 decides
  if (grp == 0) {
    int taken = -1;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      float A[NA];
#pragma unroll
      for (int a = 0; a < NA; ++a) A[a] = (a & 1) ? acc[j][a / 2].y : acc[j][a / 2].x;
      const float s0 = A[0], s1 = A[1];
      const float enl = s0 * s0 / s1;
      float alpha = 0.0f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float in = A[5 + diag_slot(d)] / s0;
        const float var = A[2 + d] / s0 - in * in;
        alpha = fmaxf(alpha, fmaxf(0.0f, (var - in * in) / var));
      }
      if (P.alpha_zero) alpha = 0.0f;
      const float oma = 1.0f - alpha;
      const float enb = enl / (oma * oma + (alpha * alpha + 2.0f * alpha * (1.0f - alpha) / s0) * enl);
      const int combo = pp.combo[j];
      const int rank = P.combo[combo].rank;
      const bool take = (P.select_mode == 0) || (enb > best.e) || (enb == best.e && rank < best.rank);
      const bool take_fb = !take && best.combo < 0 && combo == P.fallback_combo;
      if (take) {
        best.e = enb;
        best.rank = rank;
      }
      if (take || take_fb) {
        best.combo = combo;
        best.a = alpha;
        best.s0 = s0;
        taken = j;
#pragma unroll
        for (int q = 0; q < 9; ++q) best.m[q] = A[5 + q];
      }
    }
    sTake[px] = taken;
  }
  __syncthreads();
  if (grp == 1) {
    const int taken = sTake[px];
#pragma unroll
    for (int j = 0; j < NP; ++j)
      if (taken == j) {
#pragma unroll
        for (int q = 0; q < 9; ++q) best.m[q] = (q & 1) ? acc[j][q / 2].y : acc[j][q / 2].x;
      }
  }
}

template <int PH0, int PH1, int PH2>
__device__ __forceinline__ bool pass3_is(const PassParams& pp) {
  constexpr int NP = np3_of<PH0, PH1, PH2>();
  return pp.np == NP && pp.ph[0] == PH0 && (NP < 2 || pp.ph[1] == PH1) && (NP < 3 || pp.ph[2] == PH2);
}

template <int PHX, int A0, int A1, int A2, int B0, int B1, int B2>
struct Fast3K {
  using L = Fast3<PHX, cmax3(np3_of<A0, A1, A2>(), np3_of<B0, B1, B2>())>;
};

// passes of shape A and, where B0 >= 0, of shape B, staged for patch half PHX
template <int PHX, int A0, int A1, int A2, int B0, int B1, int B2>
__global__ void __launch_bounds__(Fast3K<PHX, A0, A1, A2, B0, B1, B2>::L::THREADS, 1)
    nlsar3_fast_kernel(const FilterParams P, const Scene3 S) {
  using L = typename Fast3K<PHX, A0, A1, A2, B0, B1, B2>::L;
  constexpr int WSH = L::WSH, RS = L::RS, RN = L::RN, TW = L::TW, NT = L::THREADS;
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  float* sS9 = smem + L::OFF_S9;
  float* sLd = smem + L::OFF_LD;
  float* sAlpha = smem + L::OFF_X + 32 * L::TH;
  float* sS0 = smem + L::OFF_X + 64 * L::TH;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int grp = warp / L::TH, y = warp - grp * L::TH;  // warp-uniform group, output row
  const int px = y * 32 + lane;
  const int lt = blockIdx.x + S.tile_skip;
  const int ty = lt / S.tiles_x, tx = lt - ty * S.tiles_x;
  const int vy0 = ty * L::TH, vx0 = tx * TW;
  const int G = P.G;
  const size_t cfi = (size_t)(vy0 + y + G) * S.pitch + (vx0 + lane + G);

  Best3 best;
  best.e = -1.0f;
  best.a = 0.0f;
  best.s0 = 1.0f;
  best.rank = 0x7fffffff;
  best.combo = -1;
#pragma unroll
  for (int q = 0; q < 9; ++q) best.m[q] = 0.0f;

  int loaded_slot = -1;
  for (int ps = 0; ps < P.npass; ++ps) {
    const PassParams& pp = P.pass[ps];
    __syncthreads();
    if (pp.scale_slot != loaded_slot) {
      const float* s9 = S.s9[pp.scale_slot];
      const float* ldp = S.ld[pp.scale_slot];
      const int by = vy0 - PHX - WSH + G, bx = vx0 - PHX - WSH + G;
      for (int i = tid; i < RN; i += NT) {
        const int r = i / RS, c = i - r * RS;
        const size_t g = (size_t)(by + r) * S.pitch + (bx + c);
#pragma unroll
        for (int q = 0; q < 9; ++q) sS9[q * RN + i] = s9[q * S.plane + g];
        sLd[i] = ldp[g];
      }
      loaded_slot = pp.scale_slot;
    }
    if constexpr (B0 < 0) {
      fast3_pass<L, A0, A1, A2>(P, pp, smem, S, cfi, best);
    } else {
      if (pass3_is<A0, A1, A2>(pp))
        fast3_pass<L, A0, A1, A2>(P, pp, smem, S, cfi, best);
      else
        fast3_pass<L, B0, B1, B2>(P, pp, smem, S, cfi, best);
    }
  }

  // ---- blend with the centre (weighted_means.cl:79), nine planes per group
  if (grp == 0) {
    sAlpha[px] = best.a;
    sS0[px] = best.s0;
  }
  __syncthreads();
  const int vy = vy0 + y, vx = vx0 + lane;
  const int oy = (vy < S.H - 1) ? vy : (vy == S.vH ? S.H - 1 : -1);
  const int ox = (vx < S.W - 1) ? vx : (vx == S.vW ? S.W - 1 : -1);
  if (oy < 0 || ox < 0) return;
  const float alpha = sAlpha[px], s0 = sS0[px];
  const float oma = 1.0f - alpha;
  const size_t n = (size_t)S.H * S.W, o = (size_t)oy * S.W + ox;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int p = grp == 0 ? group_plane(0, q) : group_plane(1, q);
    const float cp = __ldg(S.c18 + p * S.plane + cfi);
    S.out[p * n + o] = oma * best.m[q] / s0 + alpha * cp;
  }
}

template <int PHX, int A0, int A1, int A2, int B0, int B1, int B2>
cudaError_t launch3_fast_t(const FilterParams& F, const Scene3& S, unsigned tiles, cudaStream_t st) {
  using L = typename Fast3K<PHX, A0, A1, A2, B0, B1, B2>::L;
  const size_t smem = (size_t)L::WORDS * 4;
  static size_t allowed[kMaxDevices];
  const void* fn = (const void*)nlsar3_fast_kernel<PHX, A0, A1, A2, B0, B1, B2>;
  const cudaError_t e = allow_dynamic_smem(fn, smem, allowed);
  if (e != cudaSuccess) return e;
  nlsar3_fast_kernel<PHX, A0, A1, A2, B0, B1, B2><<<tiles, L::THREADS, smem, st>>>(F, S);
  return cudaGetLastError();
}

// pass shapes of the specialised 3x3 kernel: 1 every pass {1,2,3}; 2..4 every
// pass the single half 1..3; 5 every pass {1,2,3} or {4,5} with at least one
// {4,5} (patches 3..11 at each scale); 0 none of these
int fast3_shape(const FilterParams& F) {
  if (F.wsh != 10 || F.npass < 1) return 0;
  auto is = [](const PassParams& p, int n, int a0, int a1, int a2) {
    return p.np == n && p.ph[0] == a0 && (n < 2 || p.ph[1] == a1) && (n < 3 || p.ph[2] == a2);
  };
  bool all123 = true, mix = true, any45 = false, single = true;
  const int h0 = F.pass[0].ph[0];
  for (int i = 0; i < F.npass; ++i) {
    const PassParams& p = F.pass[i];
    const bool s123 = is(p, 3, 1, 2, 3), s45 = is(p, 2, 4, 5, -1);
    all123 = all123 && s123;
    mix = mix && (s123 || s45);
    any45 = any45 || s45;
    single = single && p.np == 1 && p.ph[0] == h0;
  }
  if (all123) return 1;
  if (single && h0 >= 1 && h0 <= 3) return 1 + h0;
  if (mix && any45) return 5;
  return 0;
}

// whether the specialised 3x3 kernel has the call's pass shapes
bool fast3_supported(const FilterParams& F) { return fast3_shape(F) != 0; }

// the specialised 3x3 kernel, for the plans fast3_supported() accepts
cudaError_t launch3_fast(const FilterParams& F, const Scene3& S, unsigned tiles, cudaStream_t st) {
  switch (fast3_shape(F)) {
    case 1: return launch3_fast_t<3, 1, 2, 3, -1, -1, -1>(F, S, tiles, st);
    case 2: return launch3_fast_t<1, 1, -1, -1, -1, -1, -1>(F, S, tiles, st);
    case 3: return launch3_fast_t<2, 2, -1, -1, -1, -1, -1>(F, S, tiles, st);
    case 5: return launch3_fast_t<5, 1, 2, 3, 4, 5, -1>(F, S, tiles, st);
    default: return launch3_fast_t<3, 3, -1, -1, -1, -1, -1>(F, S, tiles, st);
  }
}


// ---- training ---------------------------------------------------------------

// rescaled and averaged similarity reals on the valid region (H-s+1) x (W-s+1),
// [pixel][9] (get_dissims.cpp:84-100 with scale_size_max = s)
__global__ void train3_avg_kernel(const float* __restrict__ cov, int H, int W, int s, GaussArg ga, float gamma,
                                  float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int yy = blockIdx.y * blockDim.y + threadIdx.y;
  const int Ho = H - s + 1, Wo = W - s + 1;
  if (x >= Wo || yy >= Ho) return;
  const size_t n = (size_t)H * W;
  float a[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) a[k] = 0.0f;
  for (int kx = 0; kx < s; ++kx)
    for (int ky = 0; ky < s; ++ky) {
      const size_t q = (size_t)(yy + kx) * W + x + ky;
      const float g = ga.g[kx * s + ky];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const float v = cov[sim_plane(k) * n + q];
        a[k] = fmaf(g, k >= 3 ? v * gamma : v, a[k]);
      }
    }
#pragma unroll
  for (int k = 0; k < 9; ++k) out[((size_t)yy * Wo + x) * 9 + k] = a[k];
}

// patches [n][p*p][9], patch k at ((k / nw) * p, (k % nw) * p), clamp padding
__global__ void train3_gather_kernel(const float* __restrict__ avg, int Ho, int Wo, int p, int nw, int n,
                                     float* __restrict__ patches) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int pp = p * p;
  if (i >= n * pp) return;
  const int k = i / pp, r = i - k * pp;
  const int yy = min(Ho - 1, (k / nw) * p + r / p);
  const int x = min(Wo - 1, (k % nw) * p + r % p);
#pragma unroll
  for (int q = 0; q < 9; ++q) patches[(size_t)i * 9 + q] = avg[((size_t)yy * Wo + x) * 9 + q];
}

// one thread per unordered pair (hi, j), hi > j: the later patch first
// (combinations.cpp:26-41, patches.cpp:43-69)
__global__ void train3_pairs_kernel(const float* __restrict__ patches, int pp, long long npairs, float c2d,
                                    float* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npairs) return;
  long long hi = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)t)) * 0.5);
  while (hi * (hi - 1) / 2 > t) --hi;
  while ((hi + 1) * hi / 2 <= t) ++hi;
  const long long j = t - hi * (hi - 1) / 2;
  const float* A = patches + (size_t)hi * pp * 9;
  const float* B = patches + (size_t)j * pp * 9;
  float sum = 0.0f;
  for (int i = 0; i < pp; ++i) {
    float a[9], b[9], s[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      a[q] = A[i * 9 + q];
      b[q] = B[i * 9 + q];
      s[q] = a[q] + b[q];
    }
    // sim_measures.h:100-160, nlooks 1
    float r = -(c2d + logf(det3f(a)) + logf(det3f(b)) - 2.0f * logf(det3f(s)));
    if (r != r) r = 0.0f;
    sum += r;
  }
  out[t] = sum;
}

float rescale_gamma_3x3() {
  // covmat_rescale.cl:25-26 with nlooks = 1, dimension = 3
  return std::pow(std::min(1.0f / 3.0f, 1.0f), 0.33333f);
}

}  // namespace

// A planned 3x3 call: kernel parameters, frame geometry and scratch (frames
// and the weight table, allocated on the call's stream).
struct Run3 {
  Plan pl;
  Scene3 S;
  size_t smem = 0;
  int tiles_y = 0, Hp = 0, Wp = 0, used = 0;
  char* scratch = nullptr;
};

static int plan3(const Plan& pl0, int H, int W, float* cout, Run3& r, cudaStream_t st) {
  int dev = 0;
  int rc = ensure_device_ready(dev);
  if (rc) return rc;
  r.pl = pl0;
  FilterParams& F = r.pl.P;
  F.c2d = 2 * 3 * std::log(2.0f);
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || optin <= 0)
    optin = 227 * 1024;
  int K = 0;
  for (int k = 8; k >= 1 && K == 0; --k) {
    const size_t b = (size_t)smem3_layout(F.wsh, F.phm, k).total * 4;
    if (b <= (size_t)optin) {
      K = k;
      r.smem = b;
    }
  }
  if (K < 1) return set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
  F.K = K;
  F.tile_h = kT3H;
  Scene3& S = r.S;
  std::memset(&S, 0, sizeof S);
  S.H = H;
  S.W = W;
  S.vH = H - 1 + r.pl.overlap;
  S.vW = W - 1 + r.pl.overlap;
  r.tiles_y = (S.vH + 1 + kT3H - 1) / kT3H;
  S.tiles_x = (S.vW + 1 + kT3W - 1) / kT3W;
  r.Hp = r.tiles_y * kT3H + 2 * F.G;
  r.Wp = S.tiles_x * kT3W + 2 * F.G;
  S.pitch = (r.Wp + 7) / 8 * 8;
  S.plane = (size_t)r.Hp * S.pitch;
  if ((long long)r.tiles_y * S.tiles_x > 0x7fffffff) return set_error(DCL_ERR_INVALID_ARGUMENT, "scene too large");
  r.used = 0;
  for (char u : r.pl.slot_used) r.used += u ? 1 : 0;
  const size_t frame_bytes = S.plane * sizeof(float) * (18 + 10 * (size_t)r.used);
  const size_t wtab_bytes = r.pl.wtab.size() * sizeof(float);
  cudaError_t e = cudaMallocAsync(&r.scratch, frame_bytes + wtab_bytes + 256, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(3x3 scratch)");
  float* p = reinterpret_cast<float*>(r.scratch);
  S.c18 = p;
  p += 18 * S.plane;
  for (size_t si = 0; si < r.pl.scales.size(); ++si)
    if (r.pl.slot_used[si]) {
      S.s9[si] = p;
      p += 9 * S.plane;
      S.ld[si] = p;
      p += S.plane;
    }
  float* d_wtab = reinterpret_cast<float*>(r.scratch + (frame_bytes + 255) / 256 * 256);
  S.out = cout;
  e = cudaMemcpyAsync(d_wtab, r.pl.wtab.data(), wtab_bytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync(3x3 weights)");
  F.wtab = d_wtab;
  F.n_scenes = 1;
  return DCL_OK;
}

// frame rows [co0, co1) of the covariance planes and [cs0, cs1) of every
// scale's similarity planes (the rows those read must be filled already)
static int prep3_rows(const Run3& r, const float* cin, int co0, int co1, int cs0, int cs1, cudaStream_t st) {
  const FilterParams& F = r.pl.P;
  const Scene3& S = r.S;
  const dim3 blk(32, 8);
  const unsigned gx = (unsigned)(r.Wp + 31) / 32;
  if (co1 > co0) {
    prep3_cov_kernel<<<dim3(gx, (unsigned)(co1 - co0 + 7) / 8), blk, 0, st>>>(
        cin, S.H, S.W, const_cast<float*>(S.c18), r.Hp, r.Wp, S.pitch, S.plane, F.G, co0, co1);
    profile_count(1);
  }
  if (cs1 > cs0) {
    const float gamma = rescale_gamma_3x3();
    for (size_t si = 0; si < r.pl.scales.size(); ++si) {
      if (!r.pl.slot_used[si]) continue;
      GaussArg ga;
      std::memset(&ga, 0, sizeof ga);
      const std::vector<float> gw = gauss_weights(r.pl.scales[si]);
      std::copy(gw.begin(), gw.end(), ga.g);
      prep3_scale_kernel<<<dim3(gx, (unsigned)(cs1 - cs0 + 7) / 8), blk, 0, st>>>(
          S.c18, r.Hp, r.Wp, S.pitch, S.plane, r.pl.scales[si], ga, gamma, const_cast<float*>(S.s9[si]),
          const_cast<float*>(S.ld[si]), cs0, cs1);
      profile_count(1);
    }
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DCL_OK : cuda_error(e, "NL-SAR 3x3 prep");
}

// the fused kernel on tile rows [t0, t1)
static int launch3_rows(const Run3& r, int t0, int t1, cudaStream_t st) {
  if (t1 <= t0) return DCL_OK;
  Scene3 S = r.S;
  S.tile_skip = t0 * S.tiles_x;
  FilterParams F = r.pl.P;
  const unsigned tiles = (unsigned)((t1 - t0) * S.tiles_x);
  F.total_tiles = (int)tiles;
  cudaError_t e;
  if (r.pl.fast && fast3_supported(F)) {
    e = launch3_fast(F, S, tiles, st);
  } else {
    static size_t allowed[kMaxDevices];
    e = allow_dynamic_smem((const void*)nlsar3_kernel, r.smem, allowed);
    if (e == cudaSuccess) {
      nlsar3_kernel<<<tiles, kT3Threads, r.smem, st>>>(F, S);
      e = cudaGetLastError();
    }
  }
  profile_count(1);
  return e == cudaSuccess ? DCL_OK : cuda_error(e, "NL-SAR 3x3");
}

// NL-SAR of one 3x3 covariance scene on device pointers (planes [18][H][W]).
int nlsar_covmat3_device(const Plan& pl, const float* cin, float* cout, int H, int W, cudaStream_t st) {
  if (!cin || !cout) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  Run3 r;
  int rc = plan3(pl, H, W, cout, r, st);
  if (rc == DCL_OK) rc = prep3_rows(r, cin, 0, r.Hp, 0, r.Hp, st);
  if (rc == DCL_OK) rc = launch3_rows(r, 0, r.tiles_y, st);
  if (r.scratch) cudaFreeAsync(r.scratch, st);
  return rc;
}

// Host pointers, in row bands as the 2x2 host calls: band b's input rows go
// up on a copy stream while band b-1 is filtered, its results come down on a
// second one; frame rows are filled only where their inputs have arrived, so
// the results equal the device entry point's.
int nlsar_covmat3_host(const Plan& pl, const float* cin, float* cout, int H, int W) {
  if (!cin || !cout) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  int dev = 0;
  int rc = ensure_device_ready(dev);
  if (rc) return rc;
  cudaStream_t st = cudaStreamPerThread;
  const size_t n = (size_t)H * W;
  float* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, 2 * 18 * n * sizeof(float), st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(io)");
  float* dout = buf + 18 * n;
  Run3 r;
  rc = plan3(pl, H, W, dout, r, st);
  const int nb = rc == DCL_OK ? band_count(dev, (long long)r.tiles_y * r.S.tiles_x, r.tiles_y) : 1;
  HostPipe* hp = nullptr;
  if (rc == DCL_OK) rc = host_pipe(dev, 2 * (size_t)nb + 2, hp);
  if (rc == DCL_OK) {
    cudaEvent_t* ev_in = hp->ev.data();
    cudaEvent_t* ev_out = hp->ev.data() + nb;
    cudaEvent_t ev_alloc = hp->ev[2 * nb];
    e = cudaEventRecord(ev_alloc, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp->h2d, ev_alloc, 0);
    if (e != cudaSuccess) rc = cuda_error(e, "event");
    std::vector<int> tb(nb + 1);
    for (int i = 0; i <= nb; ++i) tb[i] = (int)((long long)r.tiles_y * i / nb);
    const FilterParams& F = r.pl.P;
    int in_done = 0, co_done = 0, cs_done = 0;
    for (int i = 0; i < nb && rc == DCL_OK; ++i) {
      const bool last = i == nb - 1;
      const int cs_need = last ? r.Hp : std::min(r.Hp, tb[i + 1] * kT3H + F.phm + F.wsh + F.G);
      const int co_need = last ? r.Hp : std::min(r.Hp, cs_need + r.pl.shm);
      const int in_need = last ? H : std::max(1, std::min(H, co_need - F.G));
      if (in_need > in_done) {
        const size_t off = (size_t)in_done * W, cnt = (size_t)(in_need - in_done) * W * sizeof(float);
        for (int p = 0; p < 18 && e == cudaSuccess; ++p)
          e = cudaMemcpyAsync(buf + p * n + off, cin + p * n + off, cnt, cudaMemcpyHostToDevice, hp->h2d);
        in_done = in_need;
      }
      if (e == cudaSuccess) e = cudaEventRecord(ev_in[i], hp->h2d);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev_in[i], 0);
      if (e != cudaSuccess) {
        rc = cuda_error(e, "cudaMemcpyAsync(H2D)");
        break;
      }
      rc = prep3_rows(r, buf, co_done, co_need, cs_done, cs_need, st);
      co_done = co_need;
      cs_done = cs_need;
      if (rc == DCL_OK) rc = launch3_rows(r, tb[i], tb[i + 1], st);
      if (rc == DCL_OK && (e = cudaEventRecord(ev_out[i], st)) != cudaSuccess) rc = cuda_error(e, "event");
    }
    // band b holds output rows [tb[b] * 8, tb[b+1] * 8) below row H-1; row
    // H-1 comes from the last tile row
    for (int i = 0; i < nb && rc == DCL_OK; ++i) {
      const int r0 = std::min(tb[i] * kT3H, H - 1);
      const int r1 = i == nb - 1 ? H : std::min(tb[i + 1] * kT3H, H - 1);
      e = cudaStreamWaitEvent(hp->d2h, ev_out[i], 0);
      if (r1 > r0) {
        const size_t off = (size_t)r0 * W, cnt = (size_t)(r1 - r0) * W * sizeof(float);
        for (int p = 0; p < 18 && e == cudaSuccess; ++p)
          e = cudaMemcpyAsync(cout + p * n + off, dout + p * n + off, cnt, cudaMemcpyDeviceToHost, hp->d2h);
      }
      if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(D2H)");
    }
    // free in stream order after every copy
    cudaEvent_t ev_done = hp->ev[2 * nb + 1];
    cudaError_t e2 = cudaEventRecord(ev_done, hp->d2h);
    if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(st, ev_done, 0);
    cudaError_t e3 = cudaEventRecord(ev_done, hp->h2d);
    if (e3 == cudaSuccess) e3 = cudaStreamWaitEvent(st, ev_done, 0);
    if (e2 != cudaSuccess || e3 != cudaSuccess) {
      cudaStreamSynchronize(hp->h2d);
      cudaStreamSynchronize(hp->d2h);
    }
  }
  if (r.scratch) cudaFreeAsync(r.scratch, st);
  cudaFreeAsync(buf, st);
  const cudaError_t e4 = cudaStreamSynchronize(st);
  if (rc == DCL_OK && e4 != cudaSuccess) rc = cuda_error(e4, "NL-SAR 3x3");
  return rc;
}

namespace {

struct DevMem {
  void* p = nullptr;
  ~DevMem() {
    if (p) cudaFree(p);
  }
};

int train3_one(const float* d_cov, int H, int W, int p, int s, std::vector<float>& sorted) {
  const int Ho = H - s + 1, Wo = W - s + 1;
  if (Ho < 1 || Wo < 1)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "training area %dx%d smaller than scale %d", H, W, s);
  const int nh = (Ho + p - 1) / p, nw = (Wo + p - 1) / p;
  const long long n = (long long)nh * nw;
  if (n < 2) return set_error(DCL_ERR_INVALID_ARGUMENT, "training area holds fewer than two %dx%d patches", p, p);
  const long long npairs = n * (n - 1) / 2;
  const int pp = p * p;
  DevMem avg, pat, dis, dis2;
  cudaError_t e = cudaMalloc(&avg.p, (size_t)Ho * Wo * 9 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&pat.p, (size_t)n * pp * 9 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dis.p, (size_t)npairs * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dis2.p, (size_t)npairs * sizeof(float));
  if (e != cudaSuccess) return cuda_error(e, "training buffers");
  GaussArg ga;
  std::memset(&ga, 0, sizeof ga);
  const std::vector<float> g = gauss_weights(s);
  std::copy(g.begin(), g.end(), ga.g);
  dim3 blk(32, 8), grd((Wo + 31) / 32, (Ho + 7) / 8);
  train3_avg_kernel<<<grd, blk>>>(d_cov, H, W, s, ga, rescale_gamma_3x3(), (float*)avg.p);
  train3_gather_kernel<<<(unsigned)((n * pp + 255) / 256), 256>>>((const float*)avg.p, Ho, Wo, p, nw, (int)n,
                                                                  (float*)pat.p);
  train3_pairs_kernel<<<(unsigned)((npairs + 255) / 256), 256>>>((const float*)pat.p, pp, npairs,
                                                                2 * 3 * std::log(2.0f), (float*)dis.p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "training kernels");
  return sort_dissims((float*)dis.p, (float*)dis2.p, npairs, sorted);
}

}  // namespace

dcl_stats_collection* training_covmat3(const float* cov18, int H, int W, const int* patches, int np,
                                       const int* scales, int ns) {
  if (!cov18 || H < 1 || W < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "null input or empty training area");
    return nullptr;
  }
  if (!patches || !scales || np < 1 || ns < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "patch_sizes and scale_sizes must not be empty");
    return nullptr;
  }
  const size_t n = (size_t)18 * H * W;
  DevMem d_cov;
  cudaError_t e = cudaMalloc(&d_cov.p, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(d_cov.p, cov18, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cuda_error(e, "training setup");
    return nullptr;
  }
  dcl_stats_collection* c = dcl_collection_new();
  // get_stats.cpp:33-37: patch outer, scale inner; lut_size 256 (:31)
  for (int pi = 0; pi < np; ++pi)
    for (int si = 0; si < ns; ++si) {
      const int p = patches[pi], s = scales[si];
      if (p < 1 || p % 2 == 0 || s < 1 || s % 2 == 0 || s * s > kMaxGauss) {
        set_error(DCL_ERR_INVALID_ARGUMENT, "patch and scale sizes must be odd (scale <= 9)");
        dcl_stats_collection_free(c);
        return nullptr;
      }
      std::vector<float> sorted;
      if (train3_one((const float*)d_cov.p, H, W, p, s, sorted) != DCL_OK) {
        dcl_stats_collection_free(c);
        return nullptr;
      }
      dcl_collection_put(c, p, s, stats_from_sorted(sorted, 256));
    }
  return c;
}

}  // namespace dcl

// NL-SAR device kernels for sm_100a.
//
// Data flow (per scene):
//   prep kernels   (a1, a2, phi) or an 8-plane covariance  ->  clamp-padded
//                  "virtual plane" arrays in HBM: the un-rescaled covariance
//                  and, per scale, the rescaled Gaussian-averaged covariance
//                  plus its log-determinant.
//   fused kernel   one CTA per 32-column output tile: stages the tile and its
//                  halo in shared memory, loops over every search-window
//                  offset computing GLR pixel similarities, box sums for up to
//                  three patch sizes, LUT weights and register accumulators,
//                  then derives ENL, alpha and the bias-reduced ENL per
//                  (patch, scale), selects per pixel, blends with the centre
//                  pixel and decomposes.  No similarity or weight volume ever
//                  reaches HBM.
//
// Semantics follow the reference kernels (paths relative to the despeckCL
// project root): covmat_create.cl:19-56, covmat_rescale.cl:19-41,
// covmat_spatial_avg.cl:19-63, compute_pixel_similarities_2x2.cl.in:21-75 with
// sim_measures.h:31-65, patch_similarities_{row,col}_pass.cl, compute_weights.cl:19-56,
// copy_symm_weights.cl:19-78, compute_nl_statistics.cl:23-104,
// compute_alphas.cl:19-44, compute_enls_nobias.cl:19-39, weighted_means.cl:19-83,
// covmat_decompose.cl:19-39, all under src/compute/nlsar/cl_kernels/.
//
// Virtual plane: the reference filters overlapping tiles of a clamp-padded
// image and writes each tile's core back with clamped coordinates
// (src/compute/common/map_filter_tiles.h:91-96, src/data/sub_images.cpp:47-69).
// Its last tile always reaches at least `overlap` rows past the last image
// row, so output row H-1 holds the result computed at virtual row
// H-1+overlap of the clamp-extended image (likewise for column W-1).  The
// kernels compute on that virtual plane directly: vH = H-1+overlap.

#include <cuda_runtime.h>

#include "dcl_internal.h"
#include "nlsar_common.cuh"

namespace dcl {

// ---------------------------------------------------------------------------
// prep kernels (HBM-bound, run once per scene)
// ---------------------------------------------------------------------------

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Un-rescaled covariance of an InSAR pair on the padded frame
// (covmat_create.cl:32-42; clamp padding as src/data/sub_images.cpp:37-38).
__global__ void prep_cov_insar_kernel(const float* __restrict__ a1, const float* __restrict__ a2,
                                      const float* __restrict__ phi, int H, int W, float4* __restrict__ cori,
                                      int Hp, int Wp, int pitch, int G, int row0, int row1) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= Wp || py >= row1) return;
  const int y = clampi(py - G, 0, H - 1), x = clampi(px - G, 0, W - 1);
  const size_t i = (size_t)y * W + x;
  const float am = a1[i], as = a2[i];
  float sn, cs;
  sincosf(phi[i], &sn, &cs);
  const float m = am * as;
  cori[(size_t)py * pitch + px] = make_float4(am * am, as * as, m * cs, m * sn);
}

// Un-rescaled covariance from an 8-plane covariance image.
__global__ void prep_cov_planes_kernel(const float* __restrict__ cin, int H, int W, float4* __restrict__ cori,
                                       float4* __restrict__ cori2, int Hp, int Wp, int pitch, int G, int row0,
                                       int row1) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= Wp || py >= row1) return;
  const int y = clampi(py - G, 0, H - 1), x = clampi(px - G, 0, W - 1);
  const size_t n = (size_t)H * W, i = (size_t)y * W + x;
  cori[(size_t)py * pitch + px] = make_float4(cin[i], cin[6 * n + i], cin[2 * n + i], cin[3 * n + i]);
  cori2[(size_t)py * pitch + px] = make_float4(cin[n + i], cin[4 * n + i], cin[5 * n + i], cin[7 * n + i]);
}


// Rescaled (off-diagonals x gamma, covmat_rescale.cl:25-39) and Gaussian
// averaged (covmat_spatial_avg.cl:50-57, weights of
// cl_wrappers/covmat_spatial_avg.cpp:35-50) covariance of one scale, plus ln det.
__global__ void prep_scale_kernel(const float4* __restrict__ cori, int Hp, int Wp, int pitch, int s, GaussArg ga,
                                  float gamma, float4* __restrict__ cs, float* __restrict__ ld, int row0, int row1) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = row0 + blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= Wp || py >= row1) return;
  const int ssh = (s - 1) / 2;
  float c00 = 0.f, c11 = 0.f, re = 0.f, im = 0.f;
  for (int kx = 0; kx < s; ++kx) {
    const int yy = clampi(py - ssh + kx, 0, Hp - 1);
    for (int ky = 0; ky < s; ++ky) {
      const int xx = clampi(px - ssh + ky, 0, Wp - 1);
      const float4 v = cori[(size_t)yy * pitch + xx];
      const float g = ga.g[kx * s + ky];
      c00 = fmaf(g, v.x, c00);
      c11 = fmaf(g, v.y, c11);
      re = fmaf(g, v.z * gamma, re);
      im = fmaf(g, v.w * gamma, im);
    }
  }
  const size_t o = (size_t)py * pitch + px;
  cs[o] = make_float4(c00, c11, re, im);
  // sim_measures.h:31-34, each product and sum rounded separately (the
  // specialised kernel recomputes it the same way from its staged copy)
  const float det = __fsub_rn(__fmul_rn(c00, c11), __fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)));
  ld[o] = logf(det);
}

// ---------------------------------------------------------------------------
// fused per-tile kernel
// ---------------------------------------------------------------------------

__device__ __forceinline__ void offset_of(int t, int sws, int wsh, int& dy, int& dx, bool& lower) {
  // offsets come in pairs: the upper-half slot u of the reference's
  // half-window volume (compute_pixel_similarities_2x2.cpp:65-79), then its
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

template <int PX, bool FULL8>
__global__ void __launch_bounds__(kThreads, 1)
    nlsar_fused_kernel(const FilterParams P, const SceneDesc* __restrict__ scenes) {
  extern __shared__ float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int TH = P.tile_h;
  const int wsh = P.wsh, phm = P.phm, sws = P.sws;
  const SmemLayout L = smem_layout(TH, wsh, phm, P.K, FULL8);
  float4* sCs = reinterpret_cast<float4*>(smem + L.off_cs);
  float4* sCo = reinterpret_cast<float4*>(smem + L.off_co);
  float4* sCo2 = reinterpret_cast<float4*>(smem + L.off_co2);
  float* sLd = smem + L.off_ld;
  float* sSim = smem + L.off_sim;
  float* sH = smem + L.off_h;
  float* sW = smem + L.off_w;

  for (int tile = blockIdx.x; tile < P.total_tiles; tile += gridDim.x) {
    // scene lookup (scenes sorted by tile_begin)
    int lo = 0, hi = P.n_scenes - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (scenes[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    const SceneDesc& S = scenes[lo];
    const int lt = tile - S.tile_begin + S.tile_skip;
    const int ty = lt / S.tiles_x, tx = lt - ty * S.tiles_x;
    const int vy0 = ty * TH, vx0 = tx * kTileW;
    const int G = P.G, pitch = S.pitch;

    __syncthreads();  // previous tile done with shared memory
    // original covariance region: virtual [vy0-wsh, vy0+TH+wsh) x [vx0-wsh, vx0+TW+wsh)
    for (int i = tid; i < L.ro_w * L.ro_h; i += kThreads) {
      const int r = i / L.ro_w, c = i - r * L.ro_w;
      const size_t g = (size_t)(vy0 - wsh + r + G) * pitch + (vx0 - wsh + c + G);
      sCo[i] = S.cori[g];
      if (FULL8) sCo2[i] = S.cori2[g];
    }

    // accumulators: [PX][patch j][8 or 12]
    constexpr int NA = FULL8 ? 12 : 8;
    float acc[PX][kPatchPerPass][NA];
    // selection state per pixel
    float best_e[PX], best_a[PX], best_s0[PX];
    int best_rank[PX], best_combo[PX];
    float best_m[PX][FULL8 ? 8 : 4];
#pragma unroll
    for (int i = 0; i < PX; ++i) {
      best_e[i] = -1.0f;
      best_rank[i] = 0x7fffffff;
      best_combo[i] = -1;
      best_a[i] = 0.f;
      best_s0[i] = 1.f;
#pragma unroll
      for (int d = 0; d < (FULL8 ? 8 : 4); ++d) best_m[i][d] = 0.f;
    }

    int loaded_slot = -1;
    for (int ps = 0; ps < P.npass; ++ps) {
      const PassParams& pp = P.pass[ps];
      const int np = pp.np;
      if (pp.scale_slot != loaded_slot) {
        __syncthreads();
        const float4* cs = S.cs[pp.scale_slot];
        const float* ldp = S.ld[pp.scale_slot];
        const int base_y = vy0 - phm - wsh + G, base_x = vx0 - phm - wsh + G;
        for (int i = tid; i < L.rs_w * L.rs_h; i += kThreads) {
          const int r = i / L.rs_w, c = i - r * L.rs_w;
          const size_t g = (size_t)(base_y + r) * pitch + (base_x + c);
          sCs[i] = cs[g];
          sLd[i] = ldp[g];
        }
        loaded_slot = pp.scale_slot;
      }
      // composite weight tables of this pass's combinations
      for (int i = tid; i < np * kMaxLut; i += kThreads) {
        const int j = i / kMaxLut;
        sW[i] = P.wtab[pp.combo[j] * kMaxLut + (i - j * kMaxLut)];
      }
#pragma unroll
      for (int i = 0; i < PX; ++i)
#pragma unroll
        for (int j = 0; j < kPatchPerPass; ++j)
#pragma unroll
          for (int a = 0; a < NA; ++a) acc[i][j][a] = 0.f;
      __syncthreads();

      const int K = P.K;
      for (int t0 = 0; t0 < P.n_off; t0 += K) {
        const int kb = min(K, P.n_off - t0);
        // ---- phase A: pixel similarities of the batch on the tile + patch halo
        const int nsim = L.sim_w * L.sim_h;
        for (int i = tid; i < kb * nsim; i += kThreads) {
          const int k = i / nsim;
          const int rem = i - k * nsim;
          const int r = rem / L.sim_w, c = rem - r * L.sim_w;
          int dy, dx;
          bool lower;
          offset_of(t0 + k, sws, wsh, dy, dx, lower);
          const int ci = (r + wsh) * L.rs_w + (c + wsh);
          const int ni = ci + dy * L.rs_w + dx;
          const float4 a = sCs[ci];
          const float4 b = sCs[ni];
          const float la = sLd[ci], lb = sLd[ni];
          const float s00 = a.x + b.x, s11 = a.y + b.y, sre = a.z + b.z, sim_ = a.w + b.w;
          const float det = (s00 * s11) - (sre * sre + sim_ * sim_);
          // the reference evaluates the mirrored half with the neighbour as
          // the first argument (copy_symm_weights.cl:66-74)
          const float t = lower ? (P.c2d + lb) + la : (P.c2d + la) + lb;
          float sim = -(t - 2.0f * logf(det));
          if (sim != sim) sim = 0.0f;
          sSim[i] = sim;
        }
        __syncthreads();
        // ---- phase B: horizontal sums for every patch of the pass
        const int nh = L.sim_h * kTileW;
        for (int i = tid; i < kb * nh; i += kThreads) {
          const int k = i / nh;
          const int rem = i - k * nh;
          const int r = rem / kTileW, c = rem - r * kTileW;
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
              sH[((k * kPatchPerPass + j) * L.sim_h + r) * kTileW + c] = sacc;
            }
          }
        }
        __syncthreads();
        // ---- phase C: vertical sums, weights, accumulation
        for (int k = 0; k < kb; ++k) {
          int dy, dx;
          bool lower;
          offset_of(t0 + k, sws, wsh, dy, dx, lower);
          (void)lower;
#pragma unroll
          for (int j = 0; j < kPatchPerPass; ++j) {
            if (j < np) {
              const int ph = pp.ph[j];
              const ComboParams& cp = P.combo[pp.combo[j]];
              const float* col = sH + ((k * kPatchPerPass + j) * L.sim_h) * kTileW + lane;
#pragma unroll
              for (int i = 0; i < PX; ++i) {
                const int y = warp * PX + i;
                float d = 0.f;
                for (int a = -ph; a <= ph; ++a) d += col[(y + phm + a) * kTileW];
                // compute_weights.cl:40-51 through the composite weight table
                float w;
                if (d > cp.dmax) {
                  w = 0.0f;
                } else {
                  float dc = fmaxf(d, cp.dmin);
                  dc = fminf(dc, cp.dmax);
                  const float mapped = __fdiv_rn(dc - cp.dmin, cp.span) * cp.lm1;
                  const unsigned idx = (unsigned)mapped;
                  w = sW[j * kMaxLut + idx];
                }
                const int oi = (y + wsh + dy) * L.ro_w + (lane + wsh + dx);
                const float4 v = sCo[oi];
                float* A = acc[i][j];
                A[0] += w;
                A[1] = fmaf(w, w, A[1]);
                A[2] = fmaf(w, v.x, A[2]);
                A[3] = fmaf(w, v.y, A[3]);
                A[4] = fmaf(w, v.x * v.x, A[4]);
                A[5] = fmaf(w, v.y * v.y, A[5]);
                A[6] = fmaf(w, v.z, A[6]);
                A[7] = fmaf(w, v.w, A[7]);
                if (FULL8) {
                  const float4 v2 = sCo2[oi];
                  A[8 % NA] = fmaf(w, v2.x, A[8 % NA]);
                  A[9 % NA] = fmaf(w, v2.y, A[9 % NA]);
                  A[10 % NA] = fmaf(w, v2.z, A[10 % NA]);
                  A[11 % NA] = fmaf(w, v2.w, A[11 % NA]);
                }
              }
            }
          }
        }
        __syncthreads();
      }

      // ---- centre weight 1 (routines.cpp:151-157), statistics, alpha, ENL', selection
#pragma unroll
      for (int i = 0; i < PX; ++i) {
        const int y = warp * PX + i;
        const int oi = (y + wsh) * L.ro_w + (lane + wsh);
        const float4 c = sCo[oi];
        float4 c2 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (FULL8) c2 = sCo2[oi];
#pragma unroll
        for (int j = 0; j < kPatchPerPass; ++j) {
          if (j < np) {
            float* A = acc[i][j];
            const float s0 = A[0] + 1.0f, s1 = A[1] + 1.0f;
            const float s2 = A[2] + c.x, s3 = A[3] + c.y;
            const float s4 = A[4] + c.x * c.x, s5 = A[5] + c.y * c.y;
            const float s6 = A[6] + c.z, s7 = A[7] + c.w;
            // compute_nl_statistics.cl:92-101
            const float enl = s0 * s0 / s1;
            const float i0 = s2 / s0, i1 = s3 / s0;
            const float v0 = s4 / s0 - i0 * i0, v1 = s5 / s0 - i1 * i1;
            // compute_alphas.cl:30-41 (nlooks = 1)
            float alpha = 0.0f;
            alpha = fmaxf(alpha, fmaxf(0.0f, (v0 - i0 * i0) / v0));
            alpha = fmaxf(alpha, fmaxf(0.0f, (v1 - i1 * i1) / v1));
            if (P.alpha_zero) alpha = 0.0f;
            // compute_enls_nobias.cl:19-22
            const float oma = 1.0f - alpha;
            const float enb = enl / (oma * oma + (alpha * alpha + 2.0f * alpha * (1.0f - alpha) / s0) * enl);
            const int combo = pp.combo[j];
            const int rank = P.combo[combo].rank;
            bool take;
            if (P.select_mode == 0)
              take = true;
            else
              take = (enb > best_e[i]) || (enb == best_e[i] && rank < best_rank[i]);
            // no combination selected (every ENL' NaN): the reference's intended
            // rule leaves params{0,0}, i.e. index 0 of the loop order
            // (nlsar_filter_sub_image.cpp:537-541); keep it without raising the bar
            const bool take_fb = !take && best_combo[i] < 0 && combo == P.fallback_combo;
            if (take) {
              best_e[i] = enb;
              best_rank[i] = rank;
            }
            if (take || take_fb) {
              best_combo[i] = combo;
              best_a[i] = alpha;
              best_s0[i] = s0;
              best_m[i][0] = s2;
              best_m[i][1] = s3;
              best_m[i][2] = s6;
              best_m[i][3] = s7;
              if (FULL8) {
                best_m[i][4 % (FULL8 ? 8 : 4)] = A[8 % NA] + c2.x;
                best_m[i][5 % (FULL8 ? 8 : 4)] = A[9 % NA] + c2.y;
                best_m[i][6 % (FULL8 ? 8 : 4)] = A[10 % NA] + c2.z;
                best_m[i][7 % (FULL8 ? 8 : 4)] = A[11 % NA] + c2.w;
              }
            }
          }
        }
      }
    }

    // ---- blend with the centre (weighted_means.cl:79), decompose, store
#pragma unroll
    for (int i = 0; i < PX; ++i) {
      const int y = warp * PX + i;
      const int vy = vy0 + y, vx = vx0 + lane;
      const int oy = (vy < S.H - 1) ? vy : (vy == S.vH ? S.H - 1 : -1);
      const int ox = (vx < S.W - 1) ? vx : (vx == S.vW ? S.W - 1 : -1);
      if (oy < 0 || ox < 0) continue;
      const int oi = (y + wsh) * L.ro_w + (lane + wsh);
      const float4 c = sCo[oi];
      const int combo = best_combo[i];
      const float alpha = best_a[i], s0 = best_s0[i];
      float m[FULL8 ? 8 : 4];
#pragma unroll
      for (int d = 0; d < (FULL8 ? 8 : 4); ++d) m[d] = best_m[i][d];
      const float oma = 1.0f - alpha;
      const float c00 = oma * m[0] / s0 + alpha * c.x;
      const float c11 = oma * m[1] / s0 + alpha * c.y;
      const float cre = oma * m[2] / s0 + alpha * c.z;
      const float cim = oma * m[3] / s0 + alpha * c.w;
      const size_t o = (size_t)oy * S.W + ox;
      if (FULL8) {
        const float4 c2 = sCo2[oi];
        const size_t n = (size_t)S.H * S.W;
        S.cov_out[o] = c00;
        S.cov_out[n + o] = oma * m[4 % (FULL8 ? 8 : 4)] / s0 + alpha * c2.x;
        S.cov_out[2 * n + o] = cre;
        S.cov_out[3 * n + o] = cim;
        S.cov_out[4 * n + o] = oma * m[5 % (FULL8 ? 8 : 4)] / s0 + alpha * c2.y;
        S.cov_out[5 * n + o] = oma * m[6 % (FULL8 ? 8 : 4)] / s0 + alpha * c2.z;
        S.cov_out[6 * n + o] = c11;
        S.cov_out[7 * n + o] = oma * m[7 % (FULL8 ? 8 : 4)] / s0 + alpha * c2.w;
      } else {
        // covmat_decompose.cl:32-37
        const float am = sqrtf(c00), as = sqrtf(c11);
        const float r = 0.5f * (am + as);
        S.ref[o] = r * r;
        S.phase[o] = atan2f(cim, cre);
        S.coh[o] = sqrtf(cim * cim + cre * cre) / (am * as);
      }
      if (S.sel_out) S.sel_out[o] = combo;
    }
  }
}

// Launch of the fused kernel (kept in this translation unit with the template).
cudaError_t launch_nlsar_fused(bool full8, const FilterParams& F, const SceneDesc* d_scenes, size_t smem, int grid,
                               cudaStream_t st) {
  static size_t allowed8[kMaxDevices], allowed4[kMaxDevices];
  cudaError_t e = cudaSuccess;
  if (full8) {
    e = allow_dynamic_smem((const void*)nlsar_fused_kernel<2, true>, smem, allowed8);
    if (e != cudaSuccess) return e;
    nlsar_fused_kernel<2, true><<<grid, kThreads, smem, st>>>(F, d_scenes);
  } else {
    e = allow_dynamic_smem((const void*)nlsar_fused_kernel<4, false>, smem, allowed4);
    if (e != cudaSuccess) return e;
    nlsar_fused_kernel<4, false><<<grid, kThreads, smem, st>>>(F, d_scenes);
  }
  return cudaGetLastError();
}

}  // namespace dcl

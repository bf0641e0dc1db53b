// Boxcar InSAR filter: w x w window means of the intensity and of the complex
// interferogram (src/compute/boxcar/cl_kernels/boxcar_kernel.cl:19-69 in the
// reference, driven by src/compute/boxcar/boxcar.cpp:30-100 over 512x512 tiles
// with overlap (w-1)/2).
//
// One pass over HBM: each CTA stages its output tile plus a (w-1)/2 halo of
// (I, Re, Im) = ((a1^2+a2^2)/2, a1 a2 cos phi, a1 a2 sin phi) in shared memory,
// forms horizontal window sums, then vertical sums, and writes
// ref = mean I, phase = atan2(Im, Re), coh = |sum Re + j Im| / sum I.
//
// Like NL-SAR, the reference's clamped tile write-back puts the result of
// virtual row H-1+(w-1)/2 of the clamp-extended image into output row H-1
// (and likewise for the last column); the kernel computes on that virtual
// plane.

#include <cuda_runtime.h>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "fast_math.cuh"

namespace dcl {
namespace {

constexpr int kBoxTW = 64;
constexpr int kBoxTH = 32;
constexpr int kBoxThreads = 256;
constexpr int kBoxMaxR = 15;

__device__ __forceinline__ int clampi_b(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__global__ void __launch_bounds__(kBoxThreads)
    boxcar_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ phi,
                  float* __restrict__ ref, float* __restrict__ phase, float* __restrict__ coh, int H, int W, int r) {
  extern __shared__ float sm[];
  const int SW = kBoxTW + 2 * r, SH = kBoxTH + 2 * r;
  float* sI = sm;                 // [SH][SW]
  float* sR = sI + SH * SW;
  float* sJ = sR + SH * SW;
  float* hI = sJ + SH * SW;       // [SH][kBoxTW] horizontal sums
  float* hR = hI + SH * kBoxTW;
  float* hJ = hR + SH * kBoxTW;
  const int vy0 = blockIdx.y * kBoxTH, vx0 = blockIdx.x * kBoxTW;
  const int tid = threadIdx.x;
  for (int i = tid; i < SH * SW; i += kBoxThreads) {
    const int rr = i / SW, cc = i - rr * SW;
    const int y = clampi_b(vy0 - r + rr, 0, H - 1), x = clampi_b(vx0 - r + cc, 0, W - 1);
    const size_t g = (size_t)y * W + x;
    const float am = a1[g], as = a2[g];
    float sn, cs;
    __sincosf(phi[g], &sn, &cs);
    const float aa = am * as;
    sI[i] = (am * am + as * as) / 2;
    sR[i] = aa * cs;
    sJ[i] = aa * sn;
  }
  __syncthreads();
  for (int i = tid; i < SH * kBoxTW; i += kBoxThreads) {
    const int rr = i / kBoxTW, cc = i - rr * kBoxTW;
    const float* pI = sI + rr * SW + cc;
    const float* pR = sR + rr * SW + cc;
    const float* pJ = sJ + rr * SW + cc;
    float si = 0.f, sr = 0.f, sj = 0.f;
    for (int k = 0; k <= 2 * r; ++k) {
      si += pI[k];
      sr += pR[k];
      sj += pJ[k];
    }
    hI[i] = si;
    hR[i] = sr;
    hJ[i] = sj;
  }
  __syncthreads();
  const float inv_n = 1.0f / (float)((2 * r + 1) * (2 * r + 1));
  for (int i = tid; i < kBoxTH * kBoxTW; i += kBoxThreads) {
    const int rr = i / kBoxTW, cc = i - rr * kBoxTW;
    const int vy = vy0 + rr, vx = vx0 + cc;
    const int oy = (vy < H - 1) ? vy : (vy == H - 1 + r ? H - 1 : -1);
    const int ox = (vx < W - 1) ? vx : (vx == W - 1 + r ? W - 1 : -1);
    if (oy < 0 || ox < 0) continue;
    float si = 0.f, sr = 0.f, sj = 0.f;
    for (int k = 0; k <= 2 * r; ++k) {
      si += hI[(rr + k) * kBoxTW + cc];
      sr += hR[(rr + k) * kBoxTW + cc];
      sj += hJ[(rr + k) * kBoxTW + cc];
    }
    const size_t o = (size_t)oy * W + ox;
    ref[o] = si * inv_n;
    phase[o] = atan2_fast(sj, sr);
    coh[o] = sqrtf(sr * sr + sj * sj) / si;
  }
}

// Window sums of 4 consecutive outputs o[q] = v[q] + ... + v[q + w - 1],
// q = 0..3, from the 4 + w - 1 values v: the part v[3 .. w-1] that all four
// windows share is added once, then each window adds its own ends (w + 6 adds
// instead of 4 w).  No term is subtracted, so no sum cancels.
template <int R>
__device__ __forceinline__ void window4(const float* v, float* o) {
  constexpr int w = 2 * R + 1;
  if (w < 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float acc = v[q];
#pragma unroll
      for (int k = 1; k < w; ++k) acc += v[q + k];
      o[q] = acc;
    }
    return;
  }
  float c = v[3];
#pragma unroll
  for (int k = 4; k < w; ++k) c += v[k];
  const float l1 = v[1] + v[2];
  const float l0 = v[0] + l1;
  const float r2 = v[w] + v[w + 1];
  const float r3 = r2 + v[w + 2];
  o[0] = l0 + c;
  o[1] = (l1 + c) + v[w];
  o[2] = (v[2] + c) + r2;
  o[3] = c + r3;
}

// Compile-time window radius R (w = 2R+1 <= 15): a 64 x 32 tile per CTA,
// window sums from registers, each thread producing 4 consecutive outputs
// (columns in the horizontal pass, rows in the vertical one) from 4 + 2R
// loaded values per plane, with the shared part of their windows summed once
// (window4).
template <int R>
__global__ void __launch_bounds__(kBoxThreads)
    boxcar_r_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ phi,
                    float* __restrict__ ref, float* __restrict__ phase, float* __restrict__ coh, int H, int W) {
  // staged rows of SW values, pitch SWP (a multiple of 4: the horizontal
  // pass reads its windows as aligned 16-byte vectors, conflict free)
  constexpr int SW = kBoxTW + 2 * R, SH = kBoxTH + 2 * R, N = 4 + 2 * R;
  constexpr int SWP = (SW + 3) / 4 * 4, NQ = (N + 3) / 4;
  static_assert(4 * (kBoxTW / 4 - 1) + 4 * NQ <= SWP, "window vectors stay inside a staged row");
  extern __shared__ __align__(16) float sm[];
  float* sIn = sm;                   // [3][SH][SWP]: I, Re, Im
  float* sHs = sm + 3 * SH * SWP;    // [3][SH][kBoxTW] horizontal sums
  const int vy0 = blockIdx.y * kBoxTH, vx0 = blockIdx.x * kBoxTW;
  const int tid = threadIdx.x;
  // staging: each thread issues the loads of U pixels (all of its share, up
  // to 12) before using any of them, so up to 3U loads per thread are in
  // flight (the staging is bound by memory latency, not bandwidth, at one
  // load in flight per plane).  A thread's staged pixels are i = tid + u T
  // (T threads); their (row, column) advance by (T / SW, T % SW) with one
  // carry, with no division.  Tiles whose staged region lies inside the
  // scene (all but the edge tiles) read without clamping, at 32-bit offsets
  // from the tile's first staged pixel.
  constexpr int U = (SH * SW + kBoxThreads - 1) / kBoxThreads < 12 ? (SH * SW + kBoxThreads - 1) / kBoxThreads : 12;
  constexpr int DR = (U * kBoxThreads) / SW, DC = (U * kBoxThreads) % SW;
  constexpr int dr = kBoxThreads / SW, dc = kBoxThreads % SW;
  const bool interior = vy0 >= R && vy0 + kBoxTH + R <= H && vx0 >= R && vx0 + kBoxTW + R <= W;
  const size_t base = interior ? (size_t)(vy0 - R) * W + (vx0 - R) : 0;
  const float* b1 = a1 + base;
  const float* b2 = a2 + base;
  const float* bp = phi + base;
  int rr0 = tid / SW, cc0 = tid - (tid / SW) * SW;
  for (int i0 = tid; i0 < SH * SW; i0 += U * kBoxThreads) {
    float am[U], as[U], ph[U];
    int sidx[U];
    {
      int rr = rr0, cc = cc0;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int i = i0 + u * kBoxThreads;
        if (i < SH * SW) {
          int off;
          if (interior) {
            off = rr * W + cc;
          } else {
            const int y = clampi_b(vy0 - R + rr, 0, H - 1), x = clampi_b(vx0 - R + cc, 0, W - 1);
            off = 0;
            am[u] = __ldg(a1 + (size_t)y * W + x);
            as[u] = __ldg(a2 + (size_t)y * W + x);
            ph[u] = __ldg(phi + (size_t)y * W + x);
          }
          if (interior) {
            am[u] = __ldg(b1 + off);
            as[u] = __ldg(b2 + off);
            ph[u] = __ldg(bp + off);
          }
          sidx[u] = rr * SWP + cc;
        }
        rr += dr;
        cc += dc;
        if (cc >= SW) {
          cc -= SW;
          ++rr;
        }
      }
    }
    rr0 += DR;
    cc0 += DC;
    if (cc0 >= SW) {
      cc0 -= SW;
      ++rr0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * kBoxThreads;
      if (i < SH * SW) {
        const int si = sidx[u];
        float sn, cs;
        __sincosf(ph[u], &sn, &cs);
        const float aa = am[u] * as[u];
        sIn[si] = (am[u] * am[u] + as[u] * as[u]) / 2;
        sIn[SH * SWP + si] = aa * cs;
        sIn[2 * SH * SWP + si] = aa * sn;
      }
    }
  }
  __syncthreads();
  // horizontal: item = (plane, row, group of 4 columns)
  constexpr int HG = kBoxTW / 4;
  for (int it = tid; it < 3 * SH * HG; it += kBoxThreads) {
    const int pl = it / (SH * HG);
    const int rem = it - pl * SH * HG;
    const int rr = rem / HG, c0 = (rem - rr * HG) * 4;
    const float4* src = reinterpret_cast<const float4*>(sIn + pl * SH * SWP + rr * SWP + c0);
    float v[4 * NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const float4 t = src[q];
      v[4 * q] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
    float o[4];
    window4<R>(v, o);
    *reinterpret_cast<float4*>(sHs + pl * SH * kBoxTW + rr * kBoxTW + c0) = make_float4(o[0], o[1], o[2], o[3]);
  }
  __syncthreads();
  // vertical: item = (group of 4 rows, column); all three planes
  const float inv_n = 1.0f / (float)((2 * R + 1) * (2 * R + 1));
  for (int it = tid; it < (kBoxTH / 4) * kBoxTW; it += kBoxThreads) {
    const int r0 = (it / kBoxTW) * 4, cc = it - (it / kBoxTW) * kBoxTW;
    float sum[3][4];
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) {
      const float* src = sHs + pl * SH * kBoxTW + r0 * kBoxTW + cc;
      float v[N];
#pragma unroll
      for (int k = 0; k < N; ++k) v[k] = src[k * kBoxTW];
      window4<R>(v, sum[pl]);
    }
    const int vx = vx0 + cc;
    const int ox = (vx < W - 1) ? vx : (vx == W - 1 + R ? W - 1 : -1);
    if (ox < 0) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int vy = vy0 + r0 + q;
      const int oy = (vy < H - 1) ? vy : (vy == H - 1 + R ? H - 1 : -1);
      if (oy < 0) continue;
      const float si = sum[0][q], sr = sum[1][q], sj = sum[2][q];
      const size_t o = (size_t)oy * W + ox;
      ref[o] = si * inv_n;
      phase[o] = atan2_fast(sj, sr);
      // |sum| / sum I with the hardware square root and the fast division
      // (a few ulps, against the 1e-4 relative tolerance of the coherence):
      // 6 % of the kernel's time at w 7 against the correctly rounded pair
      float m;
      asm("sqrt.approx.f32 %0, %1;" : "=f"(m) : "f"(sr * sr + sj * sj));
      coh[o] = __fdividef(m, si);
    }
  }
}

template <int R>
cudaError_t launch_boxcar_r(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                            int H, int W, dim3 grid, cudaStream_t st) {
  constexpr size_t smem = (size_t)3 * ((kBoxTH + 2 * R) * ((kBoxTW + 2 * R + 3) / 4 * 4) + (kBoxTH + 2 * R) * kBoxTW) * 4;
  static size_t allowed[kMaxDevices];
  const cudaError_t e = allow_dynamic_smem((const void*)boxcar_r_kernel<R>, smem, allowed);
  if (e != cudaSuccess) return e;
  boxcar_r_kernel<R><<<grid, kBoxThreads, smem, st>>>(a1, a2, phi, ref, phase, coh, H, W);
  return cudaGetLastError();
}

}  // namespace

int boxcar_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh, int H,
                  int W, int w, cudaStream_t st) {
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  if (w < 1 || w % 2 == 0 || (w - 1) / 2 > kBoxMaxR)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "window width must be odd and in [1, %d], got %d", 2 * kBoxMaxR + 1, w);
  const int r = (w - 1) / 2;
  const int vH = H - 1 + r, vW = W - 1 + r;
  dim3 grid((vW + kBoxTW) / kBoxTW, (vH + kBoxTH) / kBoxTH);
  const size_t smem = (size_t)3 * ((kBoxTH + 2 * r) * (kBoxTW + 2 * r) + (kBoxTH + 2 * r) * kBoxTW) * sizeof(float);
  static size_t allowed[kMaxDevices];
  if (r > 7) {
    const cudaError_t e = allow_dynamic_smem((const void*)boxcar_kernel, smem, allowed);
    if (e != cudaSuccess) return cuda_error(e, "boxcar shared-memory limit");
  }
  cudaError_t e = cudaSuccess;
  switch (r) {
    case 0: e = launch_boxcar_r<0>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 1: e = launch_boxcar_r<1>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 2: e = launch_boxcar_r<2>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 3: e = launch_boxcar_r<3>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 4: e = launch_boxcar_r<4>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 5: e = launch_boxcar_r<5>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 6: e = launch_boxcar_r<6>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    case 7: e = launch_boxcar_r<7>(a1, a2, phi, ref, phase, coh, H, W, grid, st); break;
    default:
      boxcar_kernel<<<grid, kBoxThreads, smem, st>>>(a1, a2, phi, ref, phase, coh, H, W, r);
      e = cudaGetLastError();
  }
  profile_count(1);
  if (e != cudaSuccess) return cuda_error(e, "boxcar launch");
  return DCL_OK;
}

}  // namespace dcl

extern "C" int dcl_boxcar_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                                 float* coh, int H, int W, int window_width, void* stream) {
  return dcl::boxcar_device(a1, a2, phi, ref, phase, coh, H, W, window_width, (cudaStream_t)stream);
}

extern "C" int dcl_boxcar(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                          int H, int W, int window_width) {
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  cudaStream_t st = cudaStreamPerThread;
  const size_t n = (size_t)H * W, b = n * sizeof(float);
  float* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, 6 * b, st);
  if (e != cudaSuccess) return dcl::cuda_error(e, "cudaMallocAsync(boxcar)");
  e = cudaMemcpyAsync(buf, a1, b, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf + n, a2, b, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf + 2 * n, phi, b, cudaMemcpyHostToDevice, st);
  int rc = DCL_OK;
  if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(H2D)");
  if (rc == DCL_OK) rc = dcl::boxcar_device(buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, buf + 5 * n, H, W,
                                            window_width, st);
  if (rc == DCL_OK) {
    e = cudaMemcpyAsync(ref, buf + 3 * n, b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(phase, buf + 4 * n, b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(coh, buf + 5 * n, b, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(D2H)");
  }
  cudaFreeAsync(buf, st);
  e = cudaStreamSynchronize(st);
  if (rc == DCL_OK && e != cudaSuccess) rc = dcl::cuda_error(e, "boxcar");
  return rc;
}

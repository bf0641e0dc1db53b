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

#include <cstdint>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "fast_math.cuh"

namespace dcl {
namespace {

constexpr int kBoxTW = 64;
constexpr int kBoxTH = 32;  // 40- and 48-row tiles (2 CTAs per SM) measured slower
constexpr int kBoxThreads = kBoxTH * 8;  // one vertical item (4 rows x 2 columns) per thread
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

// Packed and scalar adds for the window sums: (Re, Im) pairs are summed two
// lanes at a time with the f32x2 add (each component rounded like a scalar
// add).
__device__ __forceinline__ float wadd(float a, float b) { return a + b; }
__device__ __forceinline__ float2 wadd(float2 a, float2 b) { return __fadd2_rn(a, b); }

// Window sums of 4 consecutive outputs o[q] = v[q] + ... + v[q + w - 1],
// q = 0..3, from the 4 + w - 1 values v: the part v[3 .. w-1] that all four
// windows share is added once, then each window adds its own ends (w + 6 adds
// instead of 4 w).  No term is subtracted, so no sum cancels.
template <int R, class T>
__device__ __forceinline__ void window4(const T* v, T* o) {
  constexpr int w = 2 * R + 1;
  if (w < 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      T acc = v[q];
#pragma unroll
      for (int k = 1; k < w; ++k) acc = wadd(acc, v[q + k]);
      o[q] = acc;
    }
    return;
  }
  T c = v[3];
#pragma unroll
  for (int k = 4; k < w; ++k) c = wadd(c, v[k]);
  const T l1 = wadd(v[1], v[2]);
  const T l0 = wadd(v[0], l1);
  const T r2 = wadd(v[w], v[w + 1]);
  const T r3 = wadd(r2, v[w + 2]);
  o[0] = wadd(l0, c);
  o[1] = wadd(wadd(l1, c), v[w]);
  o[2] = wadd(wadd(v[2], c), r2);
  o[3] = wadd(c, r3);
}

// Window sums of 2 consecutive outputs from the w + 1 values v: the middle
// v[1 .. w-1] is summed once (w + 1 adds instead of 2 (w - 1)).
template <int R, class T>
__device__ __forceinline__ void window2(const T* v, T& o0, T& o1) {
  constexpr int w = 2 * R + 1;
  if (w == 1) {
    o0 = v[0];
    o1 = v[1];
    return;
  }
  T m = v[1];
#pragma unroll
  for (int k = 2; k < w; ++k) m = wadd(m, v[k]);
  o0 = wadd(v[0], m);
  o1 = wadd(m, v[w]);
}

// Compile-time window radius R (w = 2R+1 <= 15): a 64 x 32 tile per CTA of
// 256 threads.  The staged tile holds the intensity I as one plane and the
// interferogram (Re, Im) as interleaved pairs, so both complex window sums
// run as packed f32x2 adds:
//   horizontal pass: window4 over one row x 4 columns of I and window2 over
//     one row x 2 columns of (Re, Im), from 16-byte loads;
//   vertical pass, 4 rows x 2 columns per thread (the 256 items of a tile):
//     window4 down the column pair of I and down each column's (Re, Im),
//     all as packed adds, from 8- and 16-byte loads;
//   output: ref = mean I, phase = atan2(Im, Re), coh = |sum| / sum I, written
//     as 8-byte vectors where both columns are interior and the planes allow
//     it.
template <int R>
__global__ void __launch_bounds__(kBoxThreads)
    boxcar_r_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ phi,
                    float* __restrict__ ref, float* __restrict__ phase, float* __restrict__ coh, int H, int W,
                    int vec_out) {
  // staged rows of SW values, pitch SWP (a multiple of 4: the horizontal
  // pass reads its windows as aligned 16-byte vectors, conflict free)
  constexpr int SW = kBoxTW + 2 * R, SH = kBoxTH + 2 * R, N = 4 + 2 * R;
  constexpr int SWP = (SW + 3) / 4 * 4, NQ = (N + 3) / 4;
  constexpr int HG = kBoxTW / 4;
  static_assert(4 * (HG - 1) + 4 * NQ <= SWP && (kBoxTW - 2) + 2 * (R + 1) <= SWP,
                "window vectors stay inside a staged row");
  static_assert((kBoxTH / 4) * (kBoxTW / 2) == kBoxThreads, "one vertical item per thread");
  extern __shared__ __align__(16) float sm[];
  float* sI = sm;                                              // [SH][SWP]: 2 I = a1^2 + a2^2
  float2* sZ = reinterpret_cast<float2*>(sm + SH * SWP);        // [SH][SWP] (Re, Im)
  float* hI = sm + 3 * SH * SWP;                               // [SH][kBoxTW] horizontal sums
  float2* hZ = reinterpret_cast<float2*>(hI + SH * kBoxTW);     // [SH][kBoxTW]
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
        // twice the intensity (I1 + I2): the halving is folded into the
        // output stage (exact: a power of two)
        sI[si] = am[u] * am[u] + as[u] * as[u];
        sZ[si] = make_float2(aa * cs, aa * sn);
      }
    }
  }
  __syncthreads();
  // horizontal: items of I (row, 4 columns: window4 from 16-byte loads) and
  // of (Re, Im) (row, 2 columns: window2 from 16-byte loads of 2 pairs);
  // consecutive lanes read consecutive 16-byte vectors of one row
  constexpr int NI = SH * HG, NZ = SH * (kBoxTW / 2);
  for (int it = tid; it < NI + NZ; it += kBoxThreads) {
    if (it < NI) {
      const int rr = it / HG, c0 = (it - rr * HG) * 4;
      const float4* src = reinterpret_cast<const float4*>(sI + rr * SWP + c0);
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
      *reinterpret_cast<float4*>(hI + rr * kBoxTW + c0) = make_float4(o[0], o[1], o[2], o[3]);
    } else {
      const int j = it - NI;
      const int rr = j / (kBoxTW / 2), c0 = (j - rr * (kBoxTW / 2)) * 2;
      const float4* src = reinterpret_cast<const float4*>(sZ + rr * SWP + c0);
      float2 v[2 + 2 * R + 1];
#pragma unroll
      for (int q = 0; q < R + 1; ++q) {
        const float4 t = src[q];
        v[2 * q] = make_float2(t.x, t.y);
        v[2 * q + 1] = make_float2(t.z, t.w);
      }
      float2 o0, o1;
      window2<R>(v, o0, o1);
      *reinterpret_cast<float4*>(hZ + rr * kBoxTW + c0) = make_float4(o0.x, o0.y, o1.x, o1.y);
    }
  }
  __syncthreads();
  // vertical: this thread's 4 rows x 2 columns (a warp covers 4 rows of the
  // tile's 64 columns): window4 down the column pair of I and down each
  // column's (Re, Im), all as packed adds
  const int c0 = (tid % (kBoxTW / 2)) * 2, r0 = (tid / (kBoxTW / 2)) * 4;
  float2 sIp[4];     // [row]: (I of column c0, I of column c0 + 1)
  float2 sZc[2][4];  // [column][row]: (Re, Im)
  {
    float2 vi[N], vz0[N], vz1[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      vi[k] = *reinterpret_cast<const float2*>(hI + (r0 + k) * kBoxTW + c0);
      const float4 t = *reinterpret_cast<const float4*>(hZ + (r0 + k) * kBoxTW + c0);
      vz0[k] = make_float2(t.x, t.y);
      vz1[k] = make_float2(t.z, t.w);
    }
    window4<R>(vi, sIp);
    window4<R>(vz0, sZc[0]);
    window4<R>(vz1, sZc[1]);
  }
  // outputs on the virtual plane: row H-1 holds virtual row H-1+R (likewise
  // column W-1); a column pair wholly left of column W-1 maps to itself
  // the staged plane holds 2 I: ref = (2 I sum) / (2 n), coh = 2 |sum| / (2 I sum)
  const float inv_2n = 0.5f / (float)((2 * R + 1) * (2 * R + 1));
  const int vx = vx0 + c0;
  const bool cols_plain = vx + 1 < W - 1;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int vy = vy0 + r0 + q;
    const int oy = (vy < H - 1) ? vy : (vy == H - 1 + R ? H - 1 : -1);
    if (oy < 0) continue;
    float o_r[2], o_p[2], o_c[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const float si = e == 0 ? sIp[q].x : sIp[q].y;
      const float sr = sZc[e][q].x, sj = sZc[e][q].y;
      o_r[e] = si * inv_2n;
      o_p[e] = atan2_fast(sj, sr);
      // |sum| / sum I with the hardware square root and the fast division
      // (a few ulps, against the 1e-4 relative tolerance of the coherence)
      float m;
      asm("sqrt.approx.f32 %0, %1;" : "=f"(m) : "f"(sr * sr + sj * sj));
      o_c[e] = __fdividef(2.0f * m, si);
    }
    const size_t rowo = (size_t)oy * W;
    if (cols_plain && vec_out) {
      *reinterpret_cast<float2*>(ref + rowo + vx) = make_float2(o_r[0], o_r[1]);
      *reinterpret_cast<float2*>(phase + rowo + vx) = make_float2(o_p[0], o_p[1]);
      *reinterpret_cast<float2*>(coh + rowo + vx) = make_float2(o_c[0], o_c[1]);
    } else {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int x = vx + e;
        const int ox = (x < W - 1) ? x : (x == W - 1 + R ? W - 1 : -1);
        if (ox < 0) continue;
        ref[rowo + ox] = o_r[e];
        phase[rowo + ox] = o_p[e];
        coh[rowo + ox] = o_c[e];
      }
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
  // 8-byte output vectors need an even row length and 8-byte aligned planes
  const int vec_out = (W % 2 == 0) && ((reinterpret_cast<uintptr_t>(ref) | reinterpret_cast<uintptr_t>(phase) |
                                         reinterpret_cast<uintptr_t>(coh)) % 8 == 0);
  boxcar_r_kernel<R><<<grid, kBoxThreads, smem, st>>>(a1, a2, phi, ref, phase, coh, H, W, vec_out);
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

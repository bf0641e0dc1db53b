// NL-SAR training on the GPU: dissimilarities of every pair of patches of a
// homogeneous area, sorted on the device, then the quantile / chi-squared LUTs.
//
// Follows (paths relative to the despeckCL project root):
//   src/compute/nlsar/training/get_stats.cpp:25-59      one entry per (patch, scale), lut_size 256
//   src/compute/nlsar/training/get_dissims.cpp:32-117   rescale, Gaussian average with s_max = s
//   src/compute/nlsar/training/patches.cpp:32-94        non-overlapping p x p patches from (0,0),
//                                                       clamp-padded at the far edges; dissimilarity
//                                                       = sum over the p*p pixels of the GLR measure,
//                                                       later patch first
//   src/compute/nlsar/training/combinations.cpp:26-41   every unordered pair
//   src/compute/nlsar/stats.cpp:28-80                   LUTs

#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_common.cuh"
#include "stats_internal.h"

namespace dcl {

std::vector<float> gauss_weights(int s);
float rescale_gamma_2x2();

namespace {

__global__ void train_cov_insar_kernel(const float* __restrict__ a1, const float* __restrict__ a2,
                                       const float* __restrict__ phi, size_t n, float4* __restrict__ cov) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // src/data/data.cpp:70-88
  const float am = a1[i], as = a2[i];
  float sn, cs;
  sincosf(phi[i], &sn, &cs);
  cov[i] = make_float4(am * am, as * as, am * as * cs, am * as * sn);
}

__global__ void train_cov_planes_kernel(const float* __restrict__ cin, size_t n, float4* __restrict__ cov) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cov[i] = make_float4(cin[i], cin[6 * n + i], cin[2 * n + i], cin[3 * n + i]);
}

// rescaled (covmat_rescale.cl:31-39) and averaged (covmat_spatial_avg.cl:50-57,
// s_max = s) covariance, valid region only: (H-s+1) x (W-s+1)
__global__ void train_avg_kernel(const float4* __restrict__ cov, int H, int W, int s, GaussArg ga, float gamma,
                                 float4* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int Ho = H - s + 1, Wo = W - s + 1;
  if (x >= Wo || y >= Ho) return;
  float c00 = 0.f, c11 = 0.f, re = 0.f, im = 0.f;
  for (int kx = 0; kx < s; ++kx)
    for (int ky = 0; ky < s; ++ky) {
      const float4 v = cov[(size_t)(y + kx) * W + x + ky];
      const float g = ga.g[kx * s + ky];
      c00 = fmaf(g, v.x, c00);
      c11 = fmaf(g, v.y, c11);
      re = fmaf(g, v.z * gamma, re);
      im = fmaf(g, v.w * gamma, im);
    }
  out[(size_t)y * Wo + x] = make_float4(c00, c11, re, im);
}

// patches [n][p*p], patch k at ((k / nw) * p, (k % nw) * p), clamp padding
// (src/data/sub_images.cpp:37-38)
__global__ void train_gather_kernel(const float4* __restrict__ avg, int Ho, int Wo, int p, int nw, int n,
                                    float4* __restrict__ patches) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int pp = p * p;
  if (i >= n * pp) return;
  const int k = i / pp, r = i - k * pp;
  const int y = min(Ho - 1, (k / nw) * p + r / p);
  const int x = min(Wo - 1, (k % nw) * p + r % p);
  patches[i] = avg[(size_t)y * Wo + x];
}

__device__ __forceinline__ float glr(const float4 a, const float4 b, float c2d) {
  // sim_measures.h:37-65 with nlooks 1: first argument a, second b
  const float n1 = (a.x * a.y) - (a.z * a.z + a.w * a.w);
  const float n2 = (b.x * b.y) - (b.z * b.z + b.w * b.w);
  const float s00 = a.x + b.x, s11 = a.y + b.y, sre = a.z + b.z, sim = a.w + b.w;
  const float d = (s00 * s11) - (sre * sre + sim * sim);
  float r = -(c2d + logf(n1) + logf(n2) - 2.0f * logf(d));
  if (r != r) r = 0.0f;
  return r;
}

// one thread per unordered pair (hi, j), hi > j: t = hi*(hi-1)/2 + j
__global__ void train_pairs_kernel(const float4* __restrict__ patches, int pp, long long npairs, float c2d,
                                   float* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npairs) return;
  long long hi = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)t)) * 0.5);
  while (hi * (hi - 1) / 2 > t) --hi;
  while ((hi + 1) * hi / 2 <= t) ++hi;
  const long long j = t - hi * (hi - 1) / 2;
  const float4* A = patches + hi * pp;
  const float4* B = patches + j * pp;
  float sum = 0.0f;
  for (int i = 0; i < pp; ++i) sum += glr(A[i], B[i], c2d);
  out[t] = sum;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

// Sorts the npairs device dissimilarities in `dis` (into `dis2`) and returns the
// finite ones on the host, ascending (stats.cpp:28-38 drops NaN and inf).
int sort_dissims(float* dis, float* dis2, long long npairs, std::vector<float>& sorted) {
  DevBuf tmp;
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, (const float*)dis, dis2, (int)npairs);
  cudaError_t e = cudaMalloc(&tmp.p, tmp_bytes);
  if (e != cudaSuccess) return cuda_error(e, "training sort buffer");
  e = cub::DeviceRadixSort::SortKeys(tmp.p, tmp_bytes, (const float*)dis, dis2, (int)npairs);
  if (e != cudaSuccess) return cuda_error(e, "training sort");
  std::vector<float> all((size_t)npairs);
  e = cudaMemcpy(all.data(), dis2, all.size() * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_error(e, "training copy");
  sorted.clear();
  sorted.reserve(all.size());
  for (float v : all)
    if (std::isfinite(v)) sorted.push_back(v);
  if (sorted.empty()) return set_error(DCL_ERR_INVALID_ARGUMENT, "no finite dissimilarity in the training area");
  return DCL_OK;
}

// dissimilarities of one (patch, scale) on a device covariance image; returns
// them sorted ascending, finite values only
static int train_one(const float4* d_cov, int H, int W, int p, int s, std::vector<float>& sorted) {
  const int Ho = H - s + 1, Wo = W - s + 1;
  if (Ho < 1 || Wo < 1)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "training area %dx%d smaller than scale %d", H, W, s);
  const int nh = (Ho + p - 1) / p, nw = (Wo + p - 1) / p;
  const long long n = (long long)nh * nw;
  if (n < 2) return set_error(DCL_ERR_INVALID_ARGUMENT, "training area holds fewer than two %dx%d patches", p, p);
  const long long npairs = n * (n - 1) / 2;
  const int pp = p * p;
  DevBuf avg, pat, dis, dis2;
  cudaError_t e = cudaMalloc(&avg.p, (size_t)Ho * Wo * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&pat.p, (size_t)n * pp * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&dis.p, (size_t)npairs * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dis2.p, (size_t)npairs * sizeof(float));
  if (e != cudaSuccess) return cuda_error(e, "training buffers");
  GaussArg ga;
  std::memset(&ga, 0, sizeof ga);
  const std::vector<float> g = gauss_weights(s);
  std::copy(g.begin(), g.end(), ga.g);
  dim3 blk(32, 8), grd((Wo + 31) / 32, (Ho + 7) / 8);
  train_avg_kernel<<<grd, blk>>>(d_cov, H, W, s, ga, rescale_gamma_2x2(), (float4*)avg.p);
  train_gather_kernel<<<(unsigned)((n * pp + 255) / 256), 256>>>((const float4*)avg.p, Ho, Wo, p, nw, (int)n,
                                                                 (float4*)pat.p);
  train_pairs_kernel<<<(unsigned)((npairs + 255) / 256), 256>>>((const float4*)pat.p, pp, npairs,
                                                               2 * 2 * std::log(2.0f), (float*)dis.p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "training kernels");
  return sort_dissims((float*)dis.p, (float*)dis2.p, npairs, sorted);
}

static dcl_stats_collection* train_common(const float4* d_cov, int H, int W, const int* patches, int np,
                                          const int* scales, int ns) {
  if (!patches || !scales || np < 1 || ns < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "patch_sizes and scale_sizes must not be empty");
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
      if (train_one(d_cov, H, W, p, s, sorted) != DCL_OK) {
        dcl_stats_collection_free(c);
        return nullptr;
      }
      dcl_collection_put(c, p, s, stats_from_sorted(sorted, 256));
    }
  return c;
}

}  // namespace dcl

using namespace dcl;

extern "C" dcl_stats_collection* dcl_nlsar_training_insar(const float* a1, const float* a2, const float* phi, int H,
                                                          int W, const int* patches, int np, const int* scales,
                                                          int ns) {
  if (!a1 || !a2 || !phi || H < 1 || W < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "null input or empty training area");
    return nullptr;
  }
  const size_t n = (size_t)H * W;
  float* d_in = nullptr;
  float4* d_cov = nullptr;
  cudaError_t e = cudaMalloc(&d_in, 3 * n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_cov, n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMemcpy(d_in, a1, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_in + n, a2, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_in + 2 * n, phi, n * sizeof(float), cudaMemcpyHostToDevice);
  dcl_stats_collection* c = nullptr;
  if (e == cudaSuccess) {
    train_cov_insar_kernel<<<(unsigned)((n + 255) / 256), 256>>>(d_in, d_in + n, d_in + 2 * n, n, d_cov);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    c = train_common(d_cov, H, W, patches, np, scales, ns);
  else
    cuda_error(e, "training setup");
  if (d_in) cudaFree(d_in);
  if (d_cov) cudaFree(d_cov);
  return c;
}

extern "C" dcl_stats_collection* dcl_nlsar_training_covmat(const float* cov8, int H, int W, int dim,
                                                           const int* patches, int np, const int* scales, int ns) {
  if (dim == 3) return training_covmat3(cov8, H, W, patches, np, scales, ns);
  if (dim != 2) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "covariance dimension %d: 2x2 and 3x3 covariances are supported", dim);
    return nullptr;
  }
  if (!cov8 || H < 1 || W < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "null input or empty training area");
    return nullptr;
  }
  const size_t n = (size_t)H * W;
  float* d_in = nullptr;
  float4* d_cov = nullptr;
  cudaError_t e = cudaMalloc(&d_in, 8 * n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_cov, n * sizeof(float4));
  if (e == cudaSuccess) e = cudaMemcpy(d_in, cov8, 8 * n * sizeof(float), cudaMemcpyHostToDevice);
  dcl_stats_collection* c = nullptr;
  if (e == cudaSuccess) {
    train_cov_planes_kernel<<<(unsigned)((n + 255) / 256), 256>>>(d_in, n, d_cov);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    c = train_common(d_cov, H, W, patches, np, scales, ns);
  else
    cuda_error(e, "training setup");
  if (d_in) cudaFree(d_in);
  if (d_cov) cudaFree(d_cov);
  return c;
}

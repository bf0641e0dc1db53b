// FP32 FMA throughput probe: the denominator of the fused kernel's roofline.
//
// Every thread runs 8 independent FMA chains for `iters` iterations; with
// enough resident warps the FMA pipes saturate.  The result is
// 2 * 8 * iters * threads / elapsed flop/s.  (No reference counterpart.)

#include <cuda_runtime.h>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"

namespace {

__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
  float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b);
      x1 = fmaf(x1, a, b);
      x2 = fmaf(x2, a, b);
      x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b);
      x5 = fmaf(x5, a, b);
      x6 = fmaf(x6, a, b);
      x7 = fmaf(x7, a, b);
    }
  }
  const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keep the chains alive
}

}  // namespace

extern "C" int dcl_measure_fp32_tflops(double* tflops) {
  if (!tflops) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null output");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  float* out = nullptr;
  cudaError_t e = cudaMalloc(&out, (size_t)blocks * threads * sizeof(float));
  if (e != cudaSuccess) return dcl::cuda_error(e, "probe buffer");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fma_probe_kernel<<<blocks, threads>>>(out, iters / 8, 0.999f, 1e-3f);  // warm-up
  cudaEventRecord(a);
  for (int r = 0; r < 3; ++r) fma_probe_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
  cudaEventRecord(b);
  e = cudaEventSynchronize(b);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return dcl::cuda_error(e, "probe");
  const double flops = 3.0 * 2.0 * 8.0 * 16.0 * iters * (double)blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return DCL_OK;
}

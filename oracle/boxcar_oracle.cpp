// BOXCAR ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of despeckCL's boxcar filter (paths relative to the
// reference project root): the kernel src/compute/boxcar/cl_kernels/boxcar_kernel.cl:19-69
// run over 512x512 tiles with overlap (w-1)/2 (src/compute/boxcar/boxcar.cpp:60-80)
// through map_filter_tiles (src/compute/common/map_filter_tiles.h:69-96):
// clamp-padded tile reads, crop of the overlap, clamped write-back in tile
// order.
#include <algorithm>
#include <cmath>
#include <vector>

extern "C" int oracle_boxcar(const float* a1, const float* a2, const float* ph, float* ref, float* phase,
                             float* coh, int H, int W, int w, int tile) {
  if (w < 1 || w % 2 == 0 || H < 1 || W < 1) return -1;
  const int r = (w - 1) / 2;
  if (tile <= 2 * r) return -1;
  const int N = w * w;
  std::vector<float> tr(tile * tile), tp(tile * tile), tc(tile * tile);
  int h0 = -r, w0 = -r;
  while (h0 < H) {
    // tile input (sub_images.cpp:23-45)
    std::vector<float> A(tile * tile), B(tile * tile), P(tile * tile);
    for (int y = 0; y < tile; ++y)
      for (int x = 0; x < tile; ++x) {
        const int yy = std::min(H - 1, std::max(0, y + h0)), xx = std::min(W - 1, std::max(0, x + w0));
        A[y * tile + x] = a1[(size_t)yy * W + xx];
        B[y * tile + x] = a2[(size_t)yy * W + xx];
        P[y * tile + x] = ph[(size_t)yy * W + xx];
      }
    // kernel on the valid region: output at in + r (boxcar_kernel.cl:27-68)
    for (int oy = r; oy < tile - r; ++oy)
      for (int ox = r; ox < tile - r; ++ox) {
        float a = 0, xr = 0, xi = 0;
        for (int kx = 0; kx < w; ++kx)
          for (int ky = 0; ky < w; ++ky) {
            const int i = (oy - r + kx) * tile + (ox - r + ky);
            a += (A[i] * A[i] + B[i] * B[i]) / 2;
            const float aa = A[i] * B[i];
            xr += aa * std::cos(P[i]);
            xi += aa * std::sin(P[i]);
          }
        tr[oy * tile + ox] = a / N;
        tp[oy * tile + ox] = std::atan2(xi, xr);
        tc[oy * tile + ox] = std::sqrt(xr * xr + xi * xi) / a;
      }
    // crop and clamped write-back
    for (int y = r; y < tile - r; ++y)
      for (int x = r; x < tile - r; ++x) {
        const int yy = std::min(H - 1, std::max(0, h0 + y)), xx = std::min(W - 1, std::max(0, w0 + x));
        ref[(size_t)yy * W + xx] = tr[y * tile + x];
        phase[(size_t)yy * W + xx] = tp[y * tile + x];
        coh[(size_t)yy * W + xx] = tc[y * tile + x];
      }
    w0 += tile - 2 * r;
    if (w0 >= W) {
      w0 = -r;
      h0 += tile - 2 * r;
    }
  }
  return 0;
}

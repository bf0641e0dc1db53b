// TEST INFRASTRUCTURE ONLY: a CPU restatement of despeckCL's Goldstein filter
// used as the checker of the GPU path (tests, smoke and the CPU baseline of
// the benchmark); never linked into the product library.
//
// Tiles of side
//   sub = round_up(max(H, W) + 2 ov, p - 2 ov),  goldstein.cpp:62-65,
//   round_up(n, m) = n - n % m + m,                tile_size.cpp:27-36
// (the reference's side whenever it fits its device allocation bound), laid
// out by tile_iterator.cpp (origins -ov + k (sub - 2 ov) while below H / W: a
// second tile row or column appears when the round-up adds less than ov) and
// written back in iterator order with clamping (map_filter_tiles.h:64-96,
// sub_images.cpp:47-69).  Per tile, goldstein_filter_sub_image.cpp:120-186:
//   raw interferogram  Z = 0.5 (a1 + a2) e^{j phi}          raw_interferogram.cl:29-35
//   patches of p x p at stride p - 2 ov, clamped             patches_unpack.cl:29-45
//   forward 2-D DFT, unnormalised                           goldstein_patch_ft_test.cpp:38-130
//   Z <- |Z|^alpha Z                                        weighted_multiply.cl:29-34
//   backward 2-D DFT scaled by 1 / p^2                      goldstein_patch_ft_test.cpp:132-229
//   overlap-add in four parity launches onto the buffer that still holds the
//   raw interferogram (nothing clears it between raw_interferogram and
//   patches_pack), x 0.5 per overlap band, x 2 per image edge  patches_pack.cl:29-71,
//                                                           patches_pack.cpp:48-77
//   ref = |Z|, phase = arg Z; coherence untouched           slc2real.cl:29-34
//
// T = double is the truth; T = float follows the reference's FP32 arithmetic
// (the FFT itself is a textbook radix-2 transform: clFFT is not available).
#include <cmath>
#include <complex>
#include <vector>

#include "oracle.h"

namespace {

template <typename T>
void fft_radix2(std::complex<T>* a, int n, int stride, bool inverse) {
  // bit reversal
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i * stride], a[j * stride]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    for (int k = 0; k < len / 2; ++k) {
      const double ang = 2.0 * M_PI * k / len * (inverse ? 1.0 : -1.0);
      const std::complex<T> w((T)std::cos(ang), (T)std::sin(ang));
      for (int i = 0; i < n; i += len) {
        const std::complex<T> u = a[(i + k) * stride];
        const std::complex<T> v = a[(i + k + len / 2) * stride] * w;
        a[(i + k) * stride] = u + v;
        a[(i + k + len / 2) * stride] = u - v;
      }
    }
  }
}

template <typename T>
void fft2(std::complex<T>* patch, int p, bool inverse) {
  for (int r = 0; r < p; ++r) fft_radix2(patch + r * p, p, 1, inverse);
  for (int c = 0; c < p; ++c) fft_radix2(patch + c, p, p, inverse);
  if (inverse) {
    const T sc = T(1) / T(p * p);
    for (int i = 0; i < p * p; ++i) patch[i] *= sc;
  }
}

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// One tile of side `sub` at image origin (h0, w0); writes its centre back
// into ref / phase with clamping, like sub_images.cpp:47-69.
template <typename T>
void goldstein_tile(const float* a1, const float* a2, const float* phi, float* ref, float* phase, int H, int W,
                    int p, int ov, float alpha, int sub, int h0, int w0) {
  const int s = p - 2 * ov;
  const int n = sub / s;
  std::vector<std::complex<T>> Z((size_t)sub * sub);
  for (int y = 0; y < sub; ++y)
    for (int x = 0; x < sub; ++x) {
      const size_t i = (size_t)clampi(y + h0, 0, H - 1) * W + clampi(x + w0, 0, W - 1);
      const T amp = T(0.5) * (T(a1[i]) + T(a2[i]));
      Z[(size_t)y * sub + x] = std::complex<T>(amp * (T)std::cos((T)phi[i]), amp * (T)std::sin((T)phi[i]));
    }
  std::vector<std::complex<T>> out = Z;
  std::vector<std::complex<T>> P((size_t)n * n * p * p);
  for (int py = 0; py < n; ++py)
    for (int px = 0; px < n; ++px) {
      std::complex<T>* q = &P[((size_t)py * n + px) * p * p];
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c)
          q[r * p + c] = Z[(size_t)clampi(py * s + r - ov, 0, sub - 1) * sub + clampi(px * s + c - ov, 0, sub - 1)];
      fft2(q, p, false);
      for (int i = 0; i < p * p; ++i) {
        const T psd = std::sqrt(q[i].real() * q[i].real() + q[i].imag() * q[i].imag());
        q[i] *= (T)std::pow(psd, (T)alpha);
      }
      fft2(q, p, true);
    }
  // launches (x offset, y offset) = (0,0), (0,p), (p,0), (p,p)
  for (int xpar = 0; xpar < 2; ++xpar)
    for (int ypar = 0; ypar < 2; ++ypar)
      for (int py = ypar; py < n; py += 2)
        for (int px = xpar; px < n; px += 2) {
          const std::complex<T>* q = &P[((size_t)py * n + px) * p * p];
          for (int r = 0; r < p; ++r)
            for (int c = 0; c < p; ++c) {
              const int ox = px * s + c - ov, oy = py * s + r - ov;
              if (ox < 0 || ox >= sub || oy < 0 || oy >= sub) continue;
              T f = 1;
              if (c < 2 * ov || c >= p - 2 * ov) f *= T(0.5);
              if (r < 2 * ov || r >= p - 2 * ov) f *= T(0.5);
              if (ox < ov || ox >= sub - ov) f *= T(2);
              if (oy < ov || oy >= sub - ov) f *= T(2);
              out[(size_t)oy * sub + ox] += f * q[r * p + c];
            }
        }
  for (int ty = ov; ty < sub - ov; ++ty)
    for (int tx = ov; tx < sub - ov; ++tx) {
      const int y = std::min(H - 1, ty + h0), x = std::min(W - 1, tx + w0);
      const std::complex<T> v = out[(size_t)ty * sub + tx];
      ref[(size_t)y * W + x] = (float)std::fabs(std::sqrt(v.real() * v.real() + v.imag() * v.imag()));
      phase[(size_t)y * W + x] = (float)std::atan2(v.imag(), v.real());
    }
}

template <typename T>
void goldstein_t(const float* a1, const float* a2, const float* phi, float* ref, float* phase, int H, int W, int p,
                 int ov, float alpha) {
  const int s = p - 2 * ov;
  const int m = std::max(H, W) + 2 * ov;
  const int sub = m - m % s + s;
  const int step = sub - 2 * ov;
  for (int h0 = -ov; h0 < H; h0 += step)
    for (int w0 = -ov; w0 < W; w0 += step) goldstein_tile<T>(a1, a2, phi, ref, phase, H, W, p, ov, alpha, sub, h0, w0);
}

}  // namespace

extern "C" int oracle_goldstein(const float* a1, const float* a2, const float* phi, float* ref, float* phase, int H,
                                int W, int patch_size, int overlap, float alpha, int use_double) {
  const int p = patch_size;
  if (H < 1 || W < 1 || p < 2 || (p & (p - 1)) || overlap < 0 || p - 2 * overlap <= 2 * overlap) return -1;
  if (use_double)
    goldstein_t<double>(a1, a2, phi, ref, phase, H, W, p, overlap, alpha);
  else
    goldstein_t<float>(a1, a2, phi, ref, phase, H, W, p, overlap, alpha);
  return 0;
}

// The padded tile side the reference picks for a scene (goldstein.cpp:62-65).
extern "C" int oracle_goldstein_tile_side(int H, int W, int patch_size, int overlap) {
  const int s = patch_size - 2 * overlap;
  const int m = std::max(H, W) + 2 * overlap;
  return m - m % s + s;
}

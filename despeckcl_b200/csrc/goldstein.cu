// Goldstein phase filter of an InSAR pair (despeckcl::goldstein,
// src/compute/goldstein/goldstein.cpp:39-106 and
// goldstein_filter_sub_image.cpp:27-187 in the reference), for 32 x 32
// patches.
//
// The reference cuts the scene into tiles of side
//   sub = round_up(max(H, W) + 2 ov, s),  s = p - 2 ov,  round_up(n, m) = n - n % m + m
// (goldstein.cpp:62-65, tile_size.cpp:27-36; that side whenever it fits its
// device allocation bound, i.e. every scene up to tens of thousands of pixels
// a side), at origins -ov + k (sub - 2 ov) while below H / W
// (tile_iterator.cpp), and writes each tile's centre back with clamping, later
// tiles over earlier ones (map_filter_tiles.h:64-96, sub_images.cpp:47-69).
// The result at (y, x) is therefore tile row y / (sub - 2 ov) at tile row
// y - origin for y < H-1, and the last tile row at tile row sub - ov - 1 for
// y = H-1 (columns alike).  Per tile, only the patches behind those final
// positions are filtered.  Two kernels per tile:
//
//  goldstein_patch_kernel  one warp per patch: gathers the 32 x 32 patch of the
//     clamp-extended raw interferogram Z = 0.5 (a1 + a2) e^{j phi}
//     (raw_interferogram.cl, patches_unpack.cl, sub_images.cpp), transforms it
//     with a 2-D FFT (rows then columns, each a 32-point radix-2 FFT held in a
//     lane's registers, shared memory for the transposes), multiplies by
//     |Z|^alpha (weighted_multiply.cl), transforms back with the 1/p^2 scale
//     of the reference's clFFT plan (goldstein_patch_ft_test.cpp) and stores the
//     patch;
//  goldstein_pack_kernel   one thread per 4 output pixels of a row: the raw interferogram
//     plus the weighted contributions of the (up to four) patches covering the
//     pixel, added in the order of the reference's four parity launches, which
//     accumulate onto the buffer that still holds the raw interferogram
//     (patches_pack.cl:29-71, patches_pack.cpp:48-77); then |Z| and arg Z
//     (slc2real.cl).  Output row H-1 (column W-1) takes the last tile row
//     (column) of the clamped write-back (sub_images.cpp:47-69).
//
// DESPECKCL_B200_GOLDSTEIN_FUSED=1 selects goldstein_fused_kernel instead, the
// same arithmetic in one warp-specialised launch per tile with the patches
// kept in shared memory (described above the kernel).  Both give the same
// bits.  On B200 the two kernels are faster at every measured size (8192^2:
// 1.09 ms against 1.56 ms): the fused kernel's ring of patch rows (205 KB)
// leaves one CTA of 16 warps per SM, half of them FFTs and half latency-bound
// overlap-add, while the patch kernel runs 24 warps per SM and the pack kernel
// up to 64, and the patches' round trip through HBM (~28 B per output pixel)
// hides behind their compute.
// The coherence output is not written, as in the reference.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "fast_math.cuh"

namespace dcl {
namespace {

// DESPECKCL_B200_GOLDSTEIN_FUSED=1: the fused kernel instead of the two
// kernels per tile (same bits; slower on B200)
const bool g_goldstein_fused = [] {
  const char* v = std::getenv("DESPECKCL_B200_GOLDSTEIN_FUSED");
  return v && v[0] == '1';
}();

constexpr int kP = 32;           // patch side (the FFT length)
constexpr int kWarps = 4;        // patches per CTA (34 KB of transpose buffers)
constexpr int kPitch = kP + 1;   // float2 row pitch of a warp's transpose buffer

// W_32^m = exp(-2 pi i m / 32), m = 0..15
__constant__ float2 c_tw32[16] = {
    {1.000000000e+00f, -0.000000000e+00f}, {9.807852804e-01f, -1.950903220e-01f},
    {9.238795325e-01f, -3.826834324e-01f}, {8.314696123e-01f, -5.555702330e-01f},
    {7.071067812e-01f, -7.071067812e-01f}, {5.555702330e-01f, -8.314696123e-01f},
    {3.826834324e-01f, -9.238795325e-01f}, {1.950903220e-01f, -9.807852804e-01f},
    {0.000000000e+00f, -1.000000000e+00f}, {-1.950903220e-01f, -9.807852804e-01f},
    {-3.826834324e-01f, -9.238795325e-01f}, {-5.555702330e-01f, -8.314696123e-01f},
    {-7.071067812e-01f, -7.071067812e-01f}, {-8.314696123e-01f, -5.555702330e-01f},
    {-9.238795325e-01f, -3.826834324e-01f}, {-9.807852804e-01f, -1.950903220e-01f},
};

__host__ __device__ constexpr int rev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// a - b on both lanes of a float pair in one packed (f32x2) instruction,
// each lane rounded like the scalar subtraction
__device__ __forceinline__ float2 fsub2_rn(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
  return *reinterpret_cast<const float2*>(&r);
}

// In-register 32-point radix-2 decimation-in-time FFT (forward: e^{-i}, no
// scaling; inverse: e^{+i}, no scaling).  Every product and sum below is an
// explicitly rounded intrinsic, so the two Goldstein paths of this file, which
// share these functions, give the same bits whatever the compiler contracts.
// The butterflies' complex additions are packed (f32x2) adds and subtractions,
// rounded per lane exactly like the scalar ones; the twiddle products stay
// scalar (their factors are constant operands).
template <bool INV>
__device__ __forceinline__ void fft32(float2 (&x)[kP]) {
#pragma unroll
  for (int i = 0; i < kP; ++i) {
    const int j = rev5(i);
    if (j > i) {
      const float2 t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
#pragma unroll
  for (int half = 1; half < kP; half <<= 1) {
#pragma unroll
    for (int i = 0; i < kP; i += 2 * half) {
#pragma unroll
      for (int k = 0; k < half; ++k) {
        const int m = k * (kP / (2 * half));  // twiddle index into W_32
        const float2 a = x[i + k];
        const float2 b = x[i + k + half];
        float2 t;
        if (m == 0) {
          t = b;
        } else if (m == 8) {  // W = -i (forward), +i (inverse)
          t = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
        } else {
          const float2 w = c_tw32[m];
          const float wy = INV ? -w.y : w.y;
          t = make_float2(__fmaf_rn(b.x, w.x, -__fmul_rn(b.y, wy)), __fmaf_rn(b.x, wy, __fmul_rn(b.y, w.x)));
        }
        if (m == 8) {
          // the pair (+-b.y, -+b.x) would need moves: scalar adds
          x[i + k] = make_float2(__fadd_rn(a.x, t.x), __fadd_rn(a.y, t.y));
          x[i + k + half] = make_float2(__fsub_rn(a.x, t.x), __fsub_rn(a.y, t.y));
        } else {
          x[i + k] = __fadd2_rn(a, t);
          x[i + k + half] = fsub2_rn(a, t);
        }
      }
    }
  }
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ int clampg(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct GoldsteinGeom {
  int H, W, ov, s, sub, n;
  float inv_s;  // 1 / s
};

// n / s for 0 <= n < 2^24: a float estimate corrected to the exact quotient
__device__ __forceinline__ int div_s(int n, const GoldsteinGeom& g) {
  int q = __float2int_rz((float)n * g.inv_s);
  if (q * g.s > n) --q;
  if ((q + 1) * g.s <= n) ++q;
  return q;
}

// One tile of the reference's tiling and the part of it this call computes.
struct GoldsteinTile {
  int h0, w0;          // image position of tile pixel (0, 0)
  int py_lo, px_lo;    // first patch row / column filtered
  int n_py, n_px;      // patches filtered per column / row
  int y_lo, y_hi;      // output rows whose final value comes from this tile (inclusive)
  int x_lo, x_hi;      // output columns likewise
};

// Z = 0.5 (a1 + a2) e^{j phi} at flat index i (raw_interferogram.cl)
__device__ __forceinline__ float2 raw_z(const float* __restrict__ a1, const float* __restrict__ a2,
                                        const float* __restrict__ phi, size_t i) {
  const float amp = __fmul_rn(0.5f, __fadd_rn(a1[i], a2[i]));
  float sn, cs;
  __sincosf(phi[i], &sn, &cs);
  return make_float2(__fmul_rn(amp, cs), __fmul_rn(amp, sn));
}

// Filters patch (py, px) of the tile whose position (0, 0) is image pixel
// (o0y, o0x) into buf[r * kPitch + c] (row r, column c), one warp: gathers the
// patch of the clamp-extended raw interferogram (lane = column), 2-D FFT (rows
// then columns), |Z|^alpha weight, inverse 2-D FFT with the 1/p^2 scale.  The
// caller synchronises the warp before other lanes read buf.
__device__ __forceinline__ void filter_patch(const float* __restrict__ a1, const float* __restrict__ a2,
                                             const float* __restrict__ phi, float2* buf, const GoldsteinGeom& g,
                                             int o0y, int o0x, int py, int px, float alpha, int lane) {
  {
    const int tx = clampg(px * g.s + lane - g.ov, 0, g.sub - 1);
    const int ix = clampg(o0x + tx, 0, g.W - 1);
#pragma unroll 4
    for (int r = 0; r < kP; ++r) {
      const int ty = clampg(py * g.s + r - g.ov, 0, g.sub - 1);
      const int iy = clampg(o0y + ty, 0, g.H - 1);
      buf[r * kPitch + lane] = raw_z(a1, a2, phi, (size_t)iy * g.W + ix);
    }
  }
  __syncwarp();
  float2 x[kP];
  // rows (lane = row), forward
#pragma unroll
  for (int k = 0; k < kP; ++k) x[k] = buf[lane * kPitch + k];
  fft32<false>(x);
#pragma unroll
  for (int k = 0; k < kP; ++k) buf[lane * kPitch + k] = x[k];
  __syncwarp();
  // columns (lane = column): forward, |Z|^alpha weight, inverse
#pragma unroll
  for (int r = 0; r < kP; ++r) x[r] = buf[r * kPitch + lane];
  fft32<false>(x);
  // |Z|^alpha = 2^(alpha/2 log2 |Z|^2) (pow(0, 0) = 1 kept for alpha = 0)
  const float half_alpha = 0.5f * alpha;
#pragma unroll
  for (int r = 0; r < kP; ++r) {
    const float m2 = __fmaf_rn(x[r].x, x[r].x, __fmul_rn(x[r].y, x[r].y));
    const float w = (alpha == 0.0f) ? 1.0f : ex2_approx(__fmul_rn(half_alpha, __log2f(m2)));
    x[r] = make_float2(__fmul_rn(w, x[r].x), __fmul_rn(w, x[r].y));
  }
  fft32<true>(x);
#pragma unroll
  for (int r = 0; r < kP; ++r) buf[r * kPitch + lane] = x[r];
  __syncwarp();
  // rows, inverse, scaled by 1/p^2 (a power of two: exact)
#pragma unroll
  for (int k = 0; k < kP; ++k) x[k] = buf[lane * kPitch + k];
  fft32<true>(x);
  constexpr float kScale = 1.0f / (kP * kP);
#pragma unroll
  for (int k = 0; k < kP; ++k) buf[lane * kPitch + k] = make_float2(__fmul_rn(x[k].x, kScale), __fmul_rn(x[k].y, kScale));
}

__global__ void __launch_bounds__(32 * kWarps)
    goldstein_patch_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ phi,
                           float2* __restrict__ patches, GoldsteinGeom g, GoldsteinTile t, float alpha) {
  __shared__ float2 sbuf[kWarps][kP * kPitch];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pid = blockIdx.x * kWarps + warp;
  if (pid >= t.n_py * t.n_px) return;  // whole warp leaves together
  float2* buf = sbuf[warp];
  filter_patch(a1, a2, phi, buf, g, t.h0, t.w0, t.py_lo + pid / t.n_px, t.px_lo + pid % t.n_px, alpha, lane);
  __syncwarp();
  float2* out = patches + (size_t)pid * kP * kP;
#pragma unroll 4
  for (int r = 0; r < kP; ++r) out[r * kP + lane] = buf[r * kPitch + lane];
}

// weight of a patch sample in the overlap-add (patches_pack.cl:50-63)
__device__ __forceinline__ float pack_factor(int rel, int o, int ov, int sub) {
  float f = 1.0f;
  if (rel < 2 * ov || rel >= kP - 2 * ov) f *= 0.5f;
  if (o < ov || o >= sub - ov) f *= 2.0f;
  return f;
}

// v += fx fy q (fx fy is a power of two: exact)
__device__ __forceinline__ void add_sample(float2& v, float fx, float fy, float2 q) {
  const float f = __fmul_rn(fx, fy);
  v.x = __fmaf_rn(f, q.x, v.x);
  v.y = __fmaf_rn(f, q.y, v.y);
}

// |Z| and arg Z (slc2real.cl): the magnitude by the hardware square root
// (a few parts in 1e7), the angle within 6e-7 rad (atan2_fast)
__device__ __forceinline__ void write_polar(float* __restrict__ ref, float* __restrict__ phase, size_t o, float2 v) {
  float m;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(m) : "f"(__fmaf_rn(v.x, v.x, __fmul_rn(v.y, v.y))));
  ref[o] = m;
  phase[o] = atan2_fast(v.y, v.x);
}

constexpr int kPackX = 4;  // output columns per thread (32 apart: coalesced per warp); 2 and 8 measured slower

__global__ void __launch_bounds__(256)
    goldstein_pack_kernel(const float* __restrict__ a1, const float* __restrict__ a2, const float* __restrict__ phi,
                          const float2* __restrict__ patches, float* __restrict__ ref, float* __restrict__ phase,
                          GoldsteinGeom g, GoldsteinTile t) {
  const int y = t.y_lo + blockIdx.y * 8 + (threadIdx.x >> 5);
  if (y > t.y_hi) return;
  // tile position whose result lands here (the clamped write-back keeps the
  // last one; only the last tile row / column reaches row H-1 / column W-1)
  const int ty = (y == g.H - 1) ? g.sub - g.ov - 1 : y - t.h0;
  const size_t irow = (size_t)clampg(t.h0 + ty, 0, g.H - 1) * g.W;
  // covering patches per axis: q = (t + ov) / s at offset t + ov - q s, and
  // q - 1 at offset + s when that is still inside the patch (one of each
  // parity); index 0 of the arrays below is the even patch, 1 the odd one
  const int qy = div_s(ty + g.ov, g), ry = ty + g.ov - qy * g.s;
  const bool vy0 = qy >= t.py_lo && qy < t.py_lo + t.n_py;
  const bool vy1 = qy - 1 >= t.py_lo && qy - 1 < t.py_lo + t.n_py && ry + g.s < kP;
  const bool ye1 = qy & 1;
  int py_[2], ry_[2];
  bool vy_[2];
  float fy_[2];
  py_[0] = ye1 ? qy - 1 : qy;
  py_[1] = ye1 ? qy : qy - 1;
  ry_[0] = ye1 ? ry + g.s : ry;
  ry_[1] = ye1 ? ry : ry + g.s;
  vy_[0] = ye1 ? vy1 : vy0;
  vy_[1] = ye1 ? vy0 : vy1;
#pragma unroll
  for (int b = 0; b < 2; ++b) fy_[b] = pack_factor(ry_[b], ty, g.ov, g.sub);
  const int x0 = t.x_lo + blockIdx.x * (32 * kPackX) + (threadIdx.x & 31);
#pragma unroll
  for (int m = 0; m < kPackX; ++m) {
    const int x = x0 + 32 * m;
    if (x > t.x_hi) break;
    const int tx = (x == g.W - 1) ? g.sub - g.ov - 1 : x - t.w0;
    float2 v = raw_z(a1, a2, phi, irow + clampg(t.w0 + tx, 0, g.W - 1));
    const int qx = div_s(tx + g.ov, g), cx = tx + g.ov - qx * g.s;
    const bool vx0 = qx >= t.px_lo && qx < t.px_lo + t.n_px;
    const bool vx1 = qx - 1 >= t.px_lo && qx - 1 < t.px_lo + t.n_px && cx + g.s < kP;
    const bool xe1 = qx & 1;
    int px_[2], cx_[2];
    bool vx_[2];
    float fx_[2];
    px_[0] = xe1 ? qx - 1 : qx;
    px_[1] = xe1 ? qx : qx - 1;
    cx_[0] = xe1 ? cx + g.s : cx;
    cx_[1] = xe1 ? cx : cx + g.s;
    vx_[0] = xe1 ? vx1 : vx0;
    vx_[1] = xe1 ? vx0 : vx1;
#pragma unroll
    for (int a = 0; a < 2; ++a) fx_[a] = pack_factor(cx_[a], tx, g.ov, g.sub);
    // the reference's four parity launches in order: (x, y) parity (0,0), (0,1), (1,0), (1,1)
#pragma unroll
    for (int xpar = 0; xpar < 2; ++xpar)
#pragma unroll
      for (int ypar = 0; ypar < 2; ++ypar) {
        if (!vx_[xpar] || !vy_[ypar]) continue;
        add_sample(v, fx_[xpar], fy_[ypar],
                   patches[((size_t)(py_[ypar] - t.py_lo) * t.n_px + (px_[xpar] - t.px_lo)) * kP * kP +
                           ry_[ypar] * kP + cx_[xpar]]);
      }
    write_polar(ref, phase, (size_t)y * g.W + x, v);
  }
}

// ---------------------------------------------------------------------------
// Fused kernel: patch FFTs and the overlap-add in one launch per tile, no
// patch scratch in HBM, warp-specialised.  A CTA works on a strip of kStripX
// patch columns of one tile at a time, patch row by patch row.  Its
// kStripX + 1 producer warps filter one patch each per patch row (the extra
// warp the column left of the strip, whose right edge overlaps it) into a
// ring of three patch-row buffers in shared memory; its consumer warps take
// the tile rows of patch row q - one warp a row, one lane a column - while
// the producers filter row q + 1: raw interferogram plus the weighted samples
// of patch rows q and q - 1 (both still in the ring) in the reference's parity
// order, then |Z| and arg Z.  Each patch is filtered once per strip and run of
// rows (plus one row per run and one column per strip of overlap).  Per tile
// column, the output column, the image column, the covering patches' buffer
// offsets and weights are tabulated in shared memory once per strip.
//
// Hand-offs use named barriers, each bar.arrive by one side matched by a
// bar.sync of the other (256 + 256 threads): step k of a run filters patch row
// q_start + k into ring slot k % 3; the consumers finalise it after FULL(k);
// the producers write slot k % 3 again (step k + 3 ... as step k') only after
// EMPTY(k' - 2), the consumers' release of step k' - 2, the last reader of that
// slot as the previous row.  FULL and EMPTY alternate between two hardware
// barriers by the parity of k, so one side can never arrive twice on a
// barrier generation the other side has not passed.
// ---------------------------------------------------------------------------

constexpr int kStripX = 7;                   // patch columns finalised per CTA
constexpr int kProducers = kStripX + 1;      // producer warps
constexpr int kConsumers = 8;                // consumer warps
constexpr int kFusedThreads = 32 * (kProducers + kConsumers);
constexpr int kRing = 3;                     // patch-row buffers
constexpr int kSlot = kProducers * kP * kPitch;  // float2 per patch-row buffer
constexpr int kMaxNx = kStripX * kP;         // tile columns finalised per CTA, at most
constexpr int kBarFull = 1, kBarEmpty = 3;   // named barriers 1-2 and 3-4 (0 is __syncthreads)

__device__ __forceinline__ void bar_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(kFusedThreads) : "memory");
}
__device__ __forceinline__ void bar_arrive(int id) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "n"(kFusedThreads) : "memory");
}

// One axis (rows or columns) of a tile, for the fused kernel.
struct GoldsteinAxis {
  int o0;      // image index of tile position 0
  int lo, hi;  // outputs o <= N - 2 taken at tile position o - o0 (none when lo > hi)
  int last;    // output N - 1 taken at tile position sub - ov - 1
  int q_lo;    // first patch holding positions [lo - o0, hi - o0]
  int n_main;  // patches q_lo .. q_lo + n_main - 1
  int q_far;   // patch n - 1 (position sub - ov - 1) when it lies past them, else -1
  int groups;  // groups of `group` patches along the axis (strips of columns)
};

// output index of tile position t, or -1 when no output takes its value
__device__ __forceinline__ int axis_out(const GoldsteinAxis& a, int t, int n_out, const GoldsteinGeom& g) {
  if (a.last && t == g.sub - g.ov - 1) return n_out - 1;
  const int o = t + a.o0;
  return (o >= a.lo && o <= a.hi) ? o : -1;
}

// patches [r0, r1) of group b along an axis cut into groups of G
__device__ __forceinline__ void axis_range(const GoldsteinAxis& a, int b, int G, int& r0, int& r1) {
  const int main_groups = (a.n_main + G - 1) / G;
  if (b < main_groups) {
    r0 = a.q_lo + b * G;
    r1 = min(r0 + G, a.q_lo + a.n_main);
  } else {
    r0 = a.q_far;
    r1 = r0 + 1;
  }
}

// Shared-memory layout of the fused kernel.
struct FusedSmem {
  float2* ring;  // [kRing][producer warp][kP][kPitch]: filtered patch rows
  int* t_xo;     // per tile column of the strip: output column (-1: none)
  int* t_icol;   // image column of the raw interferogram
  int* t_cb;     // [2]: offset in a ring slot of the even / odd covering patch column's sample
  float* t_fx;   // [2]: column weight (0: the patch does not cover the column)
};

// Column tables of the strip of patch columns [c0, c1).
__device__ __forceinline__ void fused_tables(const FusedSmem& S, const GoldsteinGeom& g, const GoldsteinAxis& ax,
                                             int c0, int c1) {
  const int ov2 = 2 * g.ov, nx = (c1 - c0) * g.s, tx_lo = c0 * g.s - g.ov;
  for (int cxr = threadIdx.x; cxr < nx; cxr += blockDim.x) {
    // tile column tx: patch column qx = c0 + k at offset cx, and qx - 1 at
    // cx + s for cx < 2 ov; the producer warp of patch column c0 - 1 + w is w
    const int tx = tx_lo + cxr;
    const int k = div_s(cxr, g);
    const int qx = c0 + k, cx = cxr - k * g.s;
    S.t_xo[cxr] = axis_out(ax, tx, g.W, g);
    S.t_icol[cxr] = clampg(ax.o0 + tx, 0, g.W - 1);
    const int own = qx & 1, oth = own ^ 1;
    S.t_cb[own * kMaxNx + cxr] = (k + 1) * kP * kPitch + cx;
    S.t_fx[own * kMaxNx + cxr] = pack_factor(cx, tx, g.ov, g.sub);
    const bool v1 = qx >= 1 && cx < ov2;
    S.t_cb[oth * kMaxNx + cxr] = v1 ? k * kP * kPitch + cx + g.s : 0;
    S.t_fx[oth * kMaxNx + cxr] = v1 ? pack_factor(cx + g.s, tx, g.ov, g.sub) : 0.0f;
  }
}

// One run: patch rows [qa, qb) of the strip [c0, c1) finalised, patch row
// qa - 1 filtered first (for the first 2 ov tile rows of qa).  Block-uniform
// arguments; every thread of the block calls it.
__device__ __forceinline__ void fused_run(const float* __restrict__ a1, const float* __restrict__ a2,
                                          const float* __restrict__ phi, float* __restrict__ ref,
                                          float* __restrict__ phase, const FusedSmem& S, const GoldsteinGeom& g,
                                          const GoldsteinAxis& ay, const GoldsteinAxis& ax, float alpha, int c0,
                                          int c1, int qa, int qb) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q_start = max(qa - 1, 0);
  const int K = qb - q_start;  // steps; step k handles patch row q_start + k
  if (warp < kProducers) {
    const int pxw = c0 - 1 + warp;  // this warp's patch column
    const bool col_ok = pxw >= 0 && pxw < c1;
    for (int k = 0; k < K; ++k) {
      if (k >= 2) bar_sync(kBarEmpty + (k & 1));  // slot k % 3 released by step k - 2
      if (col_ok)
        filter_patch(a1, a2, phi, S.ring + (k % kRing) * kSlot + warp * kP * kPitch, g, ay.o0, ax.o0, q_start + k,
                     pxw, alpha, lane);
      bar_arrive(kBarFull + (k & 1));
    }
    return;
  }
  const int ov2 = 2 * g.ov, nx = (c1 - c0) * g.s;
  const int cw = warp - kProducers;
  for (int k = 0; k < K; ++k) {
    bar_sync(kBarFull + (k & 1));  // patch row q_start + k filtered
    const int q = q_start + k;
    if (q >= qa) {
      // tile rows [q s - ov, (q + 1) s - ov): patch row q at offset ry (slot
      // k % 3) and q - 1 at ry + s for ry < 2 ov (slot (k - 1) % 3); slot 0 of
      // the parity order is the even row
      const float2* cur = S.ring + (k % kRing) * kSlot;
      const float2* prv = S.ring + ((k + kRing - 1) % kRing) * kSlot;
      const bool odd = q & 1;
      for (int ry = cw; ry < g.s; ry += kConsumers) {
        const int ty = q * g.s - g.ov + ry;
        const int y = axis_out(ay, ty, g.H, g);
        if (y < 0) continue;
        const size_t irow = (size_t)clampg(ay.o0 + ty, 0, g.H - 1) * g.W;
        const float f_own = pack_factor(ry, ty, g.ov, g.sub);
        const float f_oth = (q >= 1 && ry < ov2) ? pack_factor(ry + g.s, ty, g.ov, g.sub) : 0.0f;
        const float fy0 = odd ? f_oth : f_own, fy1 = odd ? f_own : f_oth;
        const float2* row0 = odd ? prv + (ry + g.s) * kPitch : cur + ry * kPitch;
        const float2* row1 = odd ? cur + ry * kPitch : prv + (ry + g.s) * kPitch;
        for (int cxr = lane; cxr < nx; cxr += 32) {
          const int x = S.t_xo[cxr];
          if (x < 0) continue;
          float2 v = raw_z(a1, a2, phi, irow + S.t_icol[cxr]);
#pragma unroll
          for (int xpar = 0; xpar < 2; ++xpar) {
            const float fx = S.t_fx[xpar * kMaxNx + cxr];
            if (fx == 0.0f) continue;
            const int cb = S.t_cb[xpar * kMaxNx + cxr];
            if (fy0 != 0.0f) add_sample(v, fx, fy0, row0[cb]);
            if (fy1 != 0.0f) add_sample(v, fx, fy1, row1[cb]);
          }
          write_polar(ref, phase, (size_t)y * g.W + x, v);
        }
      }
    }
    if (k + 2 < K) bar_arrive(kBarEmpty + (k & 1));  // done with slots k % 3 and (k - 1) % 3
  }
}

// The work of a tile is strips x rows patch-row steps (rows = the main patch
// rows plus the far one), strip-major; CTA b of G resident ones takes steps
// [b T / G, (b + 1) T / G), so every CTA gets the same work in one wave.
__global__ void __launch_bounds__(kFusedThreads, 1)
    goldstein_fused_kernel(const float* __restrict__ a1, const float* __restrict__ a2,
                           const float* __restrict__ phi, float* __restrict__ ref, float* __restrict__ phase,
                           GoldsteinGeom g, GoldsteinAxis ay, GoldsteinAxis ax, float alpha) {
  extern __shared__ float2 gsm[];
  FusedSmem S;
  S.ring = gsm;
  S.t_xo = reinterpret_cast<int*>(gsm + kRing * kSlot);
  S.t_icol = S.t_xo + kMaxNx;
  S.t_cb = S.t_icol + kMaxNx;
  S.t_fx = reinterpret_cast<float*>(S.t_cb + 2 * kMaxNx);
  const int rows = ay.n_main + (ay.q_far >= 0 ? 1 : 0);
  const long long T = (long long)ax.groups * rows;
  const long long u0 = T * blockIdx.x / gridDim.x, u1 = T * (blockIdx.x + 1) / gridDim.x;
  for (long long u = u0; u < u1;) {
    const int strip = (int)(u / rows);
    const int j0 = (int)(u - (long long)strip * rows);
    const int j1 = (int)min((long long)rows, u1 - (long long)strip * rows);
    u = (long long)strip * rows + j1;
    int c0, c1;
    axis_range(ax, strip, kStripX, c0, c1);
    __syncthreads();  // the previous run's ring and tables are no longer read
    fused_tables(S, g, ax, c0, c1);
    __syncthreads();
    // steps j < n_main are patch rows q_lo + j, step n_main the far one
    const int jm = min(j1, ay.n_main);
    if (j0 < jm) fused_run(a1, a2, phi, ref, phase, S, g, ay, ax, alpha, c0, c1, ay.q_lo + j0, ay.q_lo + jm);
    if (j1 > ay.n_main) {
      __syncthreads();
      fused_run(a1, a2, phi, ref, phase, S, g, ay, ax, alpha, c0, c1, ay.q_far, ay.q_far + 1);
    }
  }
}

size_t goldstein_fused_smem() {
  return (size_t)kRing * kSlot * sizeof(float2) + (size_t)6 * kMaxNx * sizeof(int);
}

// patches (of the n per side) covering tile positions [lo, hi]
void patch_span(const GoldsteinGeom& g, int lo, int hi, int& first, int& count) {
  // patch q covers [q s - ov, q s - ov + p)
  int a = lo + g.ov - kP + 1;
  a = a <= 0 ? 0 : (a + g.s - 1) / g.s;
  int b = (hi + g.ov) / g.s;
  if (b > g.n - 1) b = g.n - 1;
  first = a;
  count = b - a + 1;
}

}  // namespace

int goldstein_geom(int H, int W, int p, int ov, GoldsteinGeom& g) {
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  if (p != kP) return set_error(DCL_ERR_UNSUPPORTED, "patch size %d: the GPU Goldstein filter supports 32", p);
  if (ov < 0 || kP - 2 * ov <= 2 * ov)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "overlap must satisfy 0 <= overlap < patch_size / 4, got %d", ov);
  g.H = H;
  g.W = W;
  g.ov = ov;
  g.s = kP - 2 * ov;
  g.inv_s = 1.0f / (float)g.s;
  const long long m = (long long)std::max(H, W) + 2 * ov;
  const long long sub = m - m % g.s + g.s;
  if (sub > (1 << 20)) return set_error(DCL_ERR_INVALID_ARGUMENT, "scene too large");
  g.sub = (int)sub;
  g.n = g.sub / g.s;
  return DCL_OK;
}

// The reference's tiles (tile_iterator.cpp with tile side g.sub and overlap
// ov) and, per tile, the output rectangle it finally owns and the patches
// behind it.  A scene has one tile per axis unless sub - 3 ov < H (W), i.e.
// (max(H, W) + 2 ov) mod s > s - ov: then a second tile holds the last
// outputs, read from its own clamp-extended neighbourhood.
std::vector<GoldsteinTile> goldstein_tiles(const GoldsteinGeom& g) {
  const int step = g.sub - 2 * g.ov;
  std::vector<int> h0s, w0s;
  for (int h0 = -g.ov; h0 < g.H; h0 += step) h0s.push_back(h0);
  for (int w0 = -g.ov; w0 < g.W; w0 += step) w0s.push_back(w0);
  std::vector<GoldsteinTile> tiles;
  for (size_t i = 0; i < h0s.size(); ++i)
    for (size_t j = 0; j < w0s.size(); ++j) {
      GoldsteinTile t;
      t.h0 = h0s[i];
      t.w0 = w0s[j];
      const bool last_r = i + 1 == h0s.size(), last_c = j + 1 == w0s.size();
      // rows [i step, (i+1) step) below H-1, plus row H-1 for the last tile row
      t.y_lo = std::min((int)i * step, g.H - 1);
      t.y_hi = last_r ? g.H - 1 : std::min(((int)i + 1) * step, g.H - 1) - 1;
      t.x_lo = std::min((int)j * step, g.W - 1);
      t.x_hi = last_c ? g.W - 1 : std::min(((int)j + 1) * step, g.W - 1) - 1;
      // tile positions read: y - h0 for y < H-1, sub - ov - 1 for y = H-1
      const int ty_lo = (t.y_lo < g.H - 1) ? t.y_lo - t.h0 : g.sub - g.ov - 1;
      const int ty_hi = last_r ? g.sub - g.ov - 1 : t.y_hi - t.h0;
      const int tx_lo = (t.x_lo < g.W - 1) ? t.x_lo - t.w0 : g.sub - g.ov - 1;
      const int tx_hi = last_c ? g.sub - g.ov - 1 : t.x_hi - t.w0;
      patch_span(g, ty_lo, ty_hi, t.py_lo, t.n_py);
      patch_span(g, tx_lo, tx_hi, t.px_lo, t.n_px);
      tiles.push_back(t);
    }
  return tiles;
}

// One axis of a tile for the fused kernel: outputs [lo, hi_incl] of n_out,
// patches grouped by `group` per CTA.
GoldsteinAxis goldstein_axis(const GoldsteinGeom& g, int o0, int lo, int hi_incl, int n_out, int group) {
  GoldsteinAxis a;
  a.o0 = o0;
  a.lo = lo;
  a.hi = std::min(hi_incl, n_out - 2);
  a.last = hi_incl == n_out - 1;
  a.q_lo = 0;
  a.n_main = 0;
  int q_hi = -1;
  if (a.lo <= a.hi) {
    // tile positions [lo - o0, hi - o0] (>= 0: o0 >= -ov) in patches (t + ov) / s
    a.q_lo = (a.lo - o0 + g.ov) / g.s;
    q_hi = (a.hi - o0 + g.ov) / g.s;
    a.n_main = q_hi - a.q_lo + 1;
  }
  const int q_last = g.n - 1;  // (sub - ov - 1 + ov) / s
  a.q_far = (a.last && !(a.n_main > 0 && q_last >= a.q_lo && q_last <= q_hi)) ? q_last : -1;
  a.groups = (a.n_main + group - 1) / group + (a.q_far >= 0 ? 1 : 0);
  return a;
}

int goldstein_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase, int H, int W, int p,
                     int ov, float alpha, cudaStream_t st) {
  if (!a1 || !a2 || !phi || !ref || !phase) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  GoldsteinGeom g;
  int rc = goldstein_geom(H, W, p, ov, g);
  if (rc) return rc;
  int dev = 0;
  rc = ensure_device_ready(dev);
  if (rc) return rc;
  const std::vector<GoldsteinTile> tiles = goldstein_tiles(g);
  if (g_goldstein_fused) {
    const size_t smem = goldstein_fused_smem();
    static size_t allowed[kMaxDevices];
    cudaError_t e = allow_dynamic_smem((const void*)goldstein_fused_kernel, smem, allowed);
    if (e != cudaSuccess) return cuda_error(e, "Goldstein shared memory");
    int sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, goldstein_fused_kernel, kFusedThreads, smem);
    if (e != cudaSuccess) return cuda_error(e, "Goldstein occupancy");
    const long long resident = (long long)std::max(per_sm, 1) * sms;
    // tiles own disjoint outputs: one launch each (one for most scenes)
    for (const GoldsteinTile& t : tiles) {
      const GoldsteinAxis ay = goldstein_axis(g, t.h0, t.y_lo, t.y_hi, H, 1);
      const GoldsteinAxis ax = goldstein_axis(g, t.w0, t.x_lo, t.x_hi, W, kStripX);
      const long long steps = (long long)ax.groups * (ay.n_main + (ay.q_far >= 0 ? 1 : 0));
      if (steps == 0) continue;
      const unsigned grid = (unsigned)std::min(steps, resident);
      goldstein_fused_kernel<<<grid, kFusedThreads, smem, st>>>(a1, a2, phi, ref, phase, g, ay, ax, alpha);
      profile_count(1);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "Goldstein launch");
    return DCL_OK;
  }
  size_t np = 0;
  for (const GoldsteinTile& t : tiles) np = std::max(np, (size_t)t.n_py * t.n_px);
  float2* patches = nullptr;
  cudaError_t e = cudaMallocAsync(&patches, np * kP * kP * sizeof(float2), st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(Goldstein patches)");
  // tiles in the reference's order; each pack writes only the pixels its tile
  // owns, so one patch buffer serves the tiles in turn
  for (const GoldsteinTile& t : tiles) {
    const size_t n = (size_t)t.n_py * t.n_px;
    goldstein_patch_kernel<<<(unsigned)((n + kWarps - 1) / kWarps), 32 * kWarps, 0, st>>>(a1, a2, phi, patches, g, t,
                                                                                         alpha);
    dim3 grid((t.x_hi - t.x_lo + 32 * kPackX) / (32 * kPackX), (t.y_hi - t.y_lo + 8) / 8);
    goldstein_pack_kernel<<<grid, 256, 0, st>>>(a1, a2, phi, patches, ref, phase, g, t);
    profile_count(2);
  }
  e = cudaGetLastError();
  cudaFreeAsync(patches, st);
  if (e != cudaSuccess) return cuda_error(e, "Goldstein launch");
  return DCL_OK;
}

}  // namespace dcl

extern "C" int dcl_goldstein_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                                    float* coh, int H, int W, int patch_size, int overlap, float alpha, void* stream) {
  (void)coh;  // not written (slc2real.cl writes amplitude and phase only)
  return dcl::goldstein_device(a1, a2, phi, ref, phase, H, W, patch_size, overlap, alpha, (cudaStream_t)stream);
}

extern "C" int dcl_goldstein(const float* a1, const float* a2, const float* phi, float* ref, float* phase, float* coh,
                             int H, int W, int patch_size, int overlap, float alpha) {
  (void)coh;
  if (!a1 || !a2 || !phi || !ref || !phase) return dcl::set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  dcl::GoldsteinGeom g;
  const int vr = dcl::goldstein_geom(H, W, patch_size, overlap, g);
  if (vr) return vr;
  cudaStream_t st = cudaStreamPerThread;
  const size_t n = (size_t)H * W, b = n * sizeof(float);
  float* buf = nullptr;
  cudaError_t e = cudaMallocAsync(&buf, 5 * b, st);
  if (e != cudaSuccess) return dcl::cuda_error(e, "cudaMallocAsync(Goldstein)");
  e = cudaMemcpyAsync(buf, a1, b, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf + n, a2, b, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(buf + 2 * n, phi, b, cudaMemcpyHostToDevice, st);
  int rc = DCL_OK;
  if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(H2D)");
  if (rc == DCL_OK)
    rc = dcl::goldstein_device(buf, buf + n, buf + 2 * n, buf + 3 * n, buf + 4 * n, H, W, patch_size, overlap, alpha,
                               st);
  if (rc == DCL_OK) {
    e = cudaMemcpyAsync(ref, buf + 3 * n, b, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(phase, buf + 4 * n, b, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = dcl::cuda_error(e, "cudaMemcpyAsync(D2H)");
  }
  cudaFreeAsync(buf, st);
  e = cudaStreamSynchronize(st);
  if (rc == DCL_OK && e != cudaSuccess) rc = dcl::cuda_error(e, "Goldstein");
  return rc;
}

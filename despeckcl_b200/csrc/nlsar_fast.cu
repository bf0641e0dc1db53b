// Fused NL-SAR tile kernel specialised at compile time on the search-window
// half size and the patch half sizes of the passes (the common
// configurations: one pass shape, or two such as {3,5,7} and {9,11} with the
// tile staged for the largest patch), for sm_100a.  Same semantics as the
// generic kernel in nlsar_kernels.cu.
//
// Per CTA: a 32 x 32 output tile (32 x 24 for 8-plane covariance input), each
// thread owning 2 (16 warps) or 4 (8 warps) vertically consecutive pixels of
// one column.  For every scale the search-window offsets are taken three at a
// time (seven when every pass has one patch size of at most 7) along a row of
// the window (same dy, consecutive dx), in the reference's summation order
// (row-major over the window, compute_nl_statistics.cl:77-78):
//   A  GLR similarities of the batch on the tile plus the patch halo (each
//      thread three adjacent columns of one row, the neighbour of column j at
//      offset k being neighbour column j + k, so K + 2 neighbour loads serve
//      3 K pairs); the measure is evaluated in
//      an order symmetric in its two pixels, so the mirrored half window gets
//      exactly the values of the reference's copy
//      (center first in the upper half, neighbour first in the mirrored half,
//      compute_pixel_similarities_2x2.cl.in:54-71, copy_symm_weights.cl:56-76)
//   B  horizontal sums for all patch sizes of the pass at once (nested
//      rings), one plane per patch size
//   C  vertical sums, composite LUT weight (compute_weights.cl:40-51), and
//      register accumulation of sum w, sum w^2, sum w I_d, sum w I_d^2,
//      sum w Re C01, sum w Im C01 per patch size; the centre offset has weight
//      1 (routines.cpp:151-157)
// then ENL, alpha, bias-reduced ENL and the selection (compute_nl_statistics.cl,
// compute_alphas.cl, compute_enls_nobias.cl, best_params.cpp) and the blended
// weighted mean (weighted_means.cl:79), decomposed (covmat_decompose.cl:32-37).
// Every sum is evaluated in a fixed order relative to its output pixel, so a
// pixel's result does not depend on where tiles fall (shift invariant).

#include <cuda_runtime.h>

#include <cuda_fp16.h>

#include <cstdint>
#include <mutex>

#include "dcl_internal.h"
#include "nlsar_common.cuh"

namespace dcl {

namespace {

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Shared-memory layout and launch shape of one instantiation: staging halo
// PHX_ (the call's largest patch half), at most NPX_ patch sizes per pass,
// PX_ vertically adjacent pixels per thread, TH_ tile rows.
template <int WSH_, int PHX_, int NPX_, int PX_, int TH_, bool FULL8_>
struct FastL {
  static constexpr int WSH = WSH_, PHX = PHX_, NPX = NPX_;
  static constexpr int SWS = 2 * WSH + 1;
  static constexpr bool FULL8 = FULL8_;              // 8-plane covariance input and output
  static constexpr int TH = TH_, TW = 32, PX = PX_;  // tile rows; vertically adjacent pixels per thread
  static constexpr int WARPS = TH / PX, THREADS = 32 * WARPS;
  // offsets per batch (SWS % K == 0): single-patch passes with a small halo
  // leave shared memory for seven, which amortises phase A's centre loads and
  // the barriers
  static constexpr int K = (NPX == 1 && PHX <= 3) ? 7 : 3;
  static constexpr int NA = FULL8 ? 12 : 8;          // accumulators per (pixel, patch size)
  static constexpr int NM = FULL8 ? 8 : 4;           // weighted sums kept for the selected combination
  // scaled covariance region: RS x RSH, with one unused pixel more per row,
  // which makes the row pitch odd (phase A reads it down columns; fast_stage)
  static constexpr int RS = TW + 2 * (PHX + WSH) + 1;
  static constexpr int RSH = TH + 2 * (PHX + WSH);
  static constexpr int RO = TW + 2 * WSH;            // original covariance region: RO x ROH
  static constexpr int ROH = TH + 2 * WSH;
  // similarity region of the widest pass, SIMWX x SIMHX, at an odd row pitch
  // (phase A's lanes write down a column; phase B's quarter warps, one row
  // each, then read words of four rows that fall in different banks)
  static constexpr int SIMWX = TW + 2 * PHX, SIMHX = TH + 2 * PHX;
  static constexpr int SIMPX = SIMWX + 1;
  static constexpr int HP = TW;                      // horizontal-sum row pitch (words), unpadded
  static constexpr int HPL = K * SIMHX * HP;         // one patch size's horizontal-sum plane
  // shared memory, in 4-byte words; the TMA destinations start on 128-byte
  // boundaries
  static constexpr int OFF_CS = 0;
  static constexpr int OFF_CO = (OFF_CS + 4 * RS * RSH + 31) / 32 * 32;
  static constexpr int OFF_CO2 = (OFF_CO + 4 * RO * ROH + 31) / 32 * 32;  // 8-plane input only
  static constexpr int OFF_H = OFF_CO2 + (FULL8 ? 4 * RO * ROH : 0);
  static constexpr int OFF_LD = OFF_H + NPX * HPL;
  // the similarity map starts on a 128-byte boundary: the ln det plane before
  // it has an odd row pitch for InSAR input, and phase B may read the map in
  // 16-byte vectors
  static constexpr int OFF_SIM = (OFF_LD + RS * RSH + 31) / 32 * 32;
  static constexpr int OFF_LUT = OFF_SIM + K * SIMHX * SIMPX;
  // interleaved copies of the composite weight tables: 16 (two lanes per
  // copy) where they fit, else 8 (four lanes per copy)
  static constexpr int LUTREP = (OFF_LUT + NPX * kMaxLut * 16 + 4) * 4 <= 227 * 1024 ? 16 : 8;
  static constexpr int OFF_BAR = (OFF_LUT + NPX * kMaxLut * LUTREP + 1) / 2 * 2;  // the mbarrier (8 bytes)
  static constexpr int WORDS = OFF_BAR + 2;
  static constexpr uint32_t CO_BYTES = 16u * RO * ROH;  // one TMA box each
  static constexpr uint32_t CS_BYTES = 16u * RS * RSH;
  static_assert(SWS % K == 0, "offset batches must tile a window row");
  // every region read or written in 16-byte vectors (or by TMA) starts on a
  // 16-byte boundary; the mbarrier on an 8-byte one
  static_assert(OFF_CS % 32 == 0 && OFF_CO % 32 == 0 && OFF_CO2 % 4 == 0 && OFF_H % 4 == 0 && OFF_SIM % 4 == 0 &&
                    OFF_BAR % 2 == 0,
                "shared-memory region alignment");
  static_assert(PX % 2 == 0, "pixels are accumulated in pairs");
  static_assert(HP >= TW && HP % 4 == 0, "horizontal-sum pitch");
  static_assert(WORDS * 4 <= 227 * 1024, "shared memory");
  static_assert(4 * RS <= 256 && 4 * RO <= 256 && RSH <= 256, "TMA box sides are at most 256 elements");
  static_assert(TH % PX == 0 && TH % 4 == 0, "tile rows");
};

template <int PH0, int PH1, int PH2>
__host__ __device__ constexpr int np_of() {
  return (PH0 >= 0) + (PH1 >= 0) + (PH2 >= 0);
}

// ---- TMA staging through one mbarrier --------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  // make the initialised barrier visible to the asynchronous (TMA) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 2-D tiled copy of one box of `map` at (x, y) (in elements; x a multiple of
// 4 floats) into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Staging waits are bounded: a copy that has not landed after this many
// polls (each a hardware-bounded suspension) is reported, not waited for.
// The thread block then returns: its remaining tiles stay unwritten, and a
// copy that never landed may still be pending towards its shared memory (the
// wait ran out only because that copy did not complete).
constexpr int kStageWaitPolls = 1 << 22;
__device__ int g_stage_timeouts;  // thread blocks that gave up waiting for a staging copy (device ledger)
__device__ int g_stage_taken;     // the ledger's value at the last take

// Waits for phase `parity` of `bar` on every thread; false (for every thread
// of the CTA) when any thread gave up, which is then counted in the device
// ledger and in the launch's own word (P.timeouts) where it has one.
__device__ __forceinline__ bool stage_wait(const FilterParams& P, uint64_t* bar, uint32_t parity) {
  const int polls = P.stage_polls > 0 ? P.stage_polls : kStageWaitPolls;
  bool ok = false;
  for (int i = 0; i < polls && !ok; ++i) ok = mbar_try_wait(bar, parity);
  const bool failed = __syncthreads_or(!ok) != 0;
  if (failed && threadIdx.x == 0) {
    atomicAdd(&g_stage_timeouts, 1);
    if (P.timeouts) atomicAdd(P.timeouts, 1);
  }
  return !failed;
}

__global__ void take_stage_timeouts_kernel() { g_stage_taken = atomicExch(&g_stage_timeouts, 0); }

// Arithmetic variants of the similarity and the sums (the precision study;
// kPrecRatio is the default):
//   kPrecRatio  the GLR as one base-2 log of the ratio
//               det(A+B)^2 / (2^4 det A det B) (sim_measures.h:52-64 is the
//               natural log of that ratio), with 1/(4 det) of every staged
//               pixel precomputed; the similarities and patch sums are in
//               log2 units and the weight lookup scales by ln 2.  No large
//               logs cancel, so the similarity keeps about 1e-7 absolute
//               accuracy where the log form loses the ulps of ln det (~1e-6)
//   kPrecLog2   the log form 2 ln det(A+B) - ln det A - ln det B - 4 ln 2 with
//               the per-pixel ln det staged and an approximate base-2 log
//   kPrecLogf   the log form with the correctly rounded logf, the reference's
//               arithmetic
//   kPrecKahan  kPrecRatio with Kahan-compensated patch sums and accumulators
//   kPrecHalf   kPrecRatio with every similarity rounded to FP16, as FP16
//               staging of the similarity map would store it
enum { kPrecRatio = 0, kPrecLog2 = 1, kPrecLogf = 2, kPrecKahan = 3, kPrecHalf = 4 };

template <int PV>
__host__ __device__ constexpr bool ratio_form() {
  return PV == kPrecRatio || PV == kPrecKahan || PV == kPrecHalf;
}

// det of a staged scaled covariance, rounded like the prep kernel's
// (sim_measures.h:31-34)
__device__ __forceinline__ float det_of(const float4 c) {
  return __fsub_rn(__fmul_rn(c.x, c.y), __fadd_rn(__fmul_rn(c.z, c.z), __fmul_rn(c.w, c.w)));
}

// The per-pixel term of a staged pixel: ln det (log forms) or 1/(4 det)
// (ratio form; NaN for a negative det, whose log is NaN, +inf for det 0).
template <int PV>
__device__ __forceinline__ float pixel_term(const float4 c) {
  const float d = det_of(c);
  if (!ratio_form<PV>()) return logf(d);
  return d >= 0.0f ? __fdiv_rn(0.25f, fabsf(d)) : __int_as_float(0x7fffffff);
}

// load of one float from a 32-bit shared-memory address, for tables that
// stay unchanged while they are read (the compiler may schedule it freely)
__device__ __forceinline__ float lds_f32(uint32_t addr) {
  float v;
  asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}

__device__ __forceinline__ float lg2_ftz(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float kahan_add(float s, float x, float& c) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  return t;
}

template <int PV>
__device__ __forceinline__ float glr_sim(const float4 a, float la, const float4 b, float lb, float c2d) {
  // sim_measures.h:52-64 with nlooks 1 and the per-pixel terms precomputed;
  // NaN -> 0.  Each form is exactly symmetric in (A, B), which gives the
  // mirrored half window the reference's values (copy_symm_weights.cl:56-76).
  const float2 d01 = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  const float2 d23 = __fadd2_rn(make_float2(a.z, a.w), make_float2(b.z, b.w));
  const float s00 = d01.x, s11 = d01.y, sre = d23.x, sim = d23.y;
  const float det = (s00 * s11) - (sre * sre + sim * sim);
  float r;
  if (ratio_form<PV>()) {
    // log2 of det |det| / (16 det A det B): negative (NaN log) when det < 0
    r = lg2_ftz((det * fabsf(det)) * (la * lb));
    if (PV == kPrecHalf) r = __half2float(__float2half_rn(r));
  } else {
    const float t = (la + lb) + c2d;
    r = (PV == kPrecLogf) ? 2.0f * logf(det) - t : fmaf(2.0f * 0.69314718f, __log2f(det), -t);
  }
  if (r != r) r = 0.0f;
  return r;
}

// patch half size of pass component j (compile time)
template <int PH0, int PH1, int PH2>
__device__ __forceinline__ constexpr int ph_of(int j) {
  return j == 0 ? PH0 : (j == 1 ? PH1 : PH2);
}

// Selection state of a thread's PX pixels, kept across the passes.
template <int PX, int NM>
struct Best {
  float e[PX], a[PX], s0[PX], m[PX][NM];
  int rank[PX], combo[PX];
};

// One pass (one scale, the patch halves PH0 < PH1 < PH2 of this pass, -1
// where unused) over all search-window offsets, on the staged tile; its
// combinations update the selection state.  The staged scaled covariance
// carries the halo of the call's largest patch; a pass with smaller patches
// reads its region CO pixels further in.
template <class L, int PH0, int PH1, int PH2, int PV>
__device__ __forceinline__ void fast_pass(const FilterParams& P, const PassParams& pp, float* smem,
                                          Best<L::PX, L::NM>& best) {
  constexpr int WSH = L::WSH, K = L::K, RS = L::RS, RO = L::RO, TW = L::TW, PX = L::PX;
  constexpr int NT = L::THREADS, NW = L::WARPS, NA = L::NA, NM = L::NM;
  constexpr bool FULL8 = L::FULL8;
  constexpr int NP = np_of<PH0, PH1, PH2>();
  constexpr int PHM = cmax(PH0, cmax(PH1, PH2));
  constexpr int CO = L::PHX - PHM;
  constexpr int SIMW = TW + 2 * PHM, SIMH = L::TH + 2 * PHM;  // this pass's similarity region
  constexpr int SIMP = SIMW + 1;  // odd row pitch (FastL::SIMPX)
  static_assert(PH0 >= 0 && NP <= L::NPX && CO >= 0, "pass shape");
  static_assert(SIMP <= L::SIMPX && SIMP % 2 == 1 && 4 * 7 + 4 + 2 * PHM <= SIMW,
                "phase-B segments must stay inside a row");
  const float4* sCs = reinterpret_cast<const float4*>(smem + L::OFF_CS);
  const float4* sCo = reinterpret_cast<const float4*>(smem + L::OFF_CO);
  const float4* sCo2 = reinterpret_cast<const float4*>(smem + L::OFF_CO2);  // 8-plane input only
  float* sH = smem + L::OFF_H;  // [NP][K][SIMH][HP]
  const float* sLd = smem + L::OFF_LD;
  float* sSim = smem + L::OFF_SIM;
  float* sLut = smem + L::OFF_LUT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int y0 = warp * PX;
  const float c2d = P.c2d;

  // composite weight tables, LUTREP interleaved copies
  for (int i = tid; i < NP * kMaxLut * L::LUTREP; i += NT) {
    const int j = i / (kMaxLut * L::LUTREP);
    const int e = (i - j * kMaxLut * L::LUTREP) / L::LUTREP;
    sLut[i] = P.wtab[pp.combo[j] * kMaxLut + e];
  }
  // patch sums in log2 units (ratio form) are scaled by ln 2 in the lookup
  float inv_span[NP], nbias[NP], lm1[NP], dmax[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const ComboParams& cp = P.combo[pp.combo[j]];
    inv_span[j] = 1.0f / cp.span;
    nbias[j] = -cp.dmin * inv_span[j];
    lm1[j] = cp.lm1;
    dmax[j] = cp.dmax;
    if (ratio_form<PV>()) {
      inv_span[j] *= 0.69314718f;
      dmax[j] *= 1.44269504f;
    }
  }
  // shared-memory address of this lane's copy of the table of component j,
  // less the 2^23 bias of the index float's bits times the entry stride:
  // adding those bits times the stride gives the entry's address (32-bit
  // shared addresses wrap modulo 2^32), one instruction fewer per lookup
  // (the 8-plane instantiations, at their register limit, index this lane's
  // copy as an array instead)
  uint32_t lut_a[NP];
  const float* lut_j[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    lut_j[j] = sLut + j * kMaxLut * L::LUTREP + (lane & (L::LUTREP - 1));
    lut_a[j] = smem_u32(lut_j[j]) - 0x4B000000u * (4u * L::LUTREP);
  }
  float2 acc[PX / 2][NP][NA];  // .x: pixel 2i, .y: pixel 2i+1
  constexpr int NKC = PV == kPrecKahan ? NA : 1;  // Kahan compensation terms
  float2 kc[PX / 2][NP][NKC];
#pragma unroll
  for (int i = 0; i < PX / 2; ++i)
#pragma unroll
    for (int j = 0; j < NP; ++j) {
#pragma unroll
      for (int a = 0; a < NA; ++a) acc[i][j][a] = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < NKC; ++a) kc[i][j][a] = make_float2(0.f, 0.f);
    }
  __syncthreads();

  for (int dy = -WSH; dy <= WSH; ++dy) {
    for (int dx0 = -WSH; dx0 <= WSH; dx0 += K) {
      {
        // ---- A, column triples: a thread takes three adjacent columns of
        // one row of the similarity region for the K offsets; the neighbour
        // of column j at offset k is neighbour column j + k, so three centre
        // and K + 2 neighbour loads serve the 3 K pairs.
        // Consecutive lanes take consecutive rows of one triple of columns:
        // the staged rows (RS float4) and the similarity rows (SIMP words)
        // have odd pitches, so their 16-byte loads (8 lanes at a time) and
        // 4-byte loads and stores (32 lanes) fall in distinct banks.  The
        // last triple holds the region's last one or two columns where its
        // width is not a multiple of three; loads for its missing columns
        // repeat its last needed one, so every index stays inside the staged
        // region.
        constexpr int NTC = (SIMW + 2) / 3;
        static_assert(RS % 2 == 1, "odd staged pitch");
        for (int it = tid; it < SIMH * NTC; it += NT) {
          const int tc = it / SIMH;
          const int r = it - tc * SIMH;
          const int c0 = 3 * tc;
          const int nc = SIMW - c0 < 3 ? SIMW - c0 : 3;
          const int ci = (r + WSH + CO) * RS + (c0 + WSH + CO);
          const int ni = ci + dy * RS + dx0;
          float4 b[K + 2];
          float lb[K + 2];
#pragma unroll
          for (int j = 0; j < K + 2; ++j) {
            const int nj = ni + (j < nc + K - 1 ? j : nc + K - 2);
            b[j] = sCs[nj];
            lb[j] = sLd[nj];
          }
          float* out = sSim + r * SIMP + c0;
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            if (j >= nc) break;
            const float4 a = sCs[ci + j];
            const float la = sLd[ci + j];
#pragma unroll
            for (int k = 0; k < K; ++k) out[k * SIMH * SIMP + j] = glr_sim<PV>(a, la, b[j + k], lb[j + k], c2d);
          }
        }
      }
      __syncthreads();
      // ---- B: horizontal sums, 4 output columns per item.  A warp takes a
      // quad of rows x 8 column segments, each quarter warp one row: word
      // loads (the odd similarity pitch puts the four rows in different
      // banks) and contiguous 16-byte stores.
      {
        constexpr int QUADS = (SIMH + 3) / 4;
        const int r_off = lane >> 3;
        const int seg = lane & 7;
        for (int q = warp; q < K * QUADS; q += NW) {
          const int k = q / QUADS;
          const int r = (q - k * QUADS) * 4 + r_off;
          if (r < SIMH) {
            // odd row pitch: word loads of the 4 + 2 PHM values
            float s[4 + 2 * PHM];
            const float* row = sSim + (k * SIMH + r) * SIMP + 4 * seg;
#pragma unroll
            for (int e = 0; e < 4 + 2 * PHM; ++e) s[e] = row[e];
            float hs[NP][4];
#pragma unroll
            for (int o = 0; o < 4; ++o) {
              float h[3] = {0.f, 0.f, 0.f};
              float ring = s[o + PHM], rc = 0.0f;
#pragma unroll
              for (int j = 0; j < 3; ++j)
                if (ph_of<PH0, PH1, PH2>(j) == 0) h[j] = ring;
#pragma unroll
              for (int b = 1; b <= PHM; ++b) {
                if (PV == kPrecKahan) {
                  ring = kahan_add(ring, s[o + PHM - b], rc);
                  ring = kahan_add(ring, s[o + PHM + b], rc);
                } else {
                  ring += s[o + PHM - b] + s[o + PHM + b];
                }
#pragma unroll
                for (int j = 0; j < 3; ++j)
                  if (ph_of<PH0, PH1, PH2>(j) == b) h[j] = PV == kPrecKahan ? ring - rc : ring;
              }
#pragma unroll
              for (int j = 0; j < NP; ++j) hs[j][o] = h[j];
            }
#pragma unroll
            for (int j = 0; j < NP; ++j)
              *reinterpret_cast<float4*>(sH + j * L::HPL + (k * SIMH + r) * L::HP + 4 * seg) =
                  make_float4(hs[j][0], hs[j][1], hs[j][2], hs[j][3]);
          }
        }
      }
      __syncthreads();
      // ---- C: vertical sums, weights, accumulation
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int dx = dx0 + k;
        float w[PX][NP];
        // vertical windows: patch j needs rows y0+PHM-ph_j .. y0+PHM+PX-1+ph_j
        float hv[NP][PX + 2 * PHM];
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const float* col = sH + j * L::HPL + (k * SIMH + y0 + PHM - ph_of<PH0, PH1, PH2>(j)) * L::HP + lane;
#pragma unroll
          for (int r = 0; r < PX + 2 * ph_of<PH0, PH1, PH2>(j); ++r) hv[j][r] = col[r * L::HP];
        }
        if (dy == 0 && dx == 0) {
#pragma unroll
          for (int i = 0; i < PX; ++i)
#pragma unroll
            for (int j = 0; j < NP; ++j) w[i][j] = 1.0f;
        } else {
#pragma unroll
          for (int i = 0; i < PX; ++i) {
#pragma unroll
            for (int j = 0; j < NP; ++j) {
              // top-down sum of the 2ph+1 rows (the first term starts the sum:
              // no similarity sum is -0, so this equals 0 + ... bit for bit)
              float d = hv[j][i], dc = 0.0f;
#pragma unroll
              for (int a = 1; a <= 2 * ph_of<PH0, PH1, PH2>(j); ++a) {
                if (PV == kPrecKahan)
                  d = kahan_add(d, hv[j][i + a], dc);
                else
                  d += hv[j][i + a];
              }
              if (PV == kPrecKahan) d -= dc;
              // index = (unsigned)((clamp(d) - dmin) / (dmax - dmin) * (L - 1)):
              // a saturating FMA clamps (and maps NaN to 0), a round-toward-zero
              // add of 2^23 truncates, and the float's low mantissa bits are the
              // index; d > dmax has weight 0
              const float u = __saturatef(fmaf(d, inv_span[j], nbias[j]));
              const float t = __fmaf_rz(u, lm1[j], 8388608.0f);
              float lw;
              if constexpr (FULL8) {
                lw = lut_j[j][(__float_as_int(t) - 0x4B000000) * L::LUTREP];
              } else {
                lw = lds_f32(lut_a[j] + static_cast<uint32_t>(__float_as_int(t)) * (4u * L::LUTREP));
              }
              w[i][j] = (d > dmax[j]) ? 0.0f : lw;
            }
          }
        }
        // two pixels per packed (f32x2) operation; each component is
        // rounded exactly like the scalar add / multiply / fma
#pragma unroll
        for (int i = 0; i < PX; i += 2) {
          const int oa = (y0 + i + WSH + dy) * RO + (lane + WSH + dx);
          const float4 va = sCo[oa];
          const float4 vb = sCo[oa + RO];
          const float2 vx = make_float2(va.x, vb.x), vy = make_float2(va.y, vb.y);
          const float2 vz = make_float2(va.z, vb.z), vw = make_float2(va.w, vb.w);
          const float2 x2 = __fmul2_rn(vx, vx), y2 = __fmul2_rn(vy, vy);
          float2 ex[4];
          if (FULL8) {
            const float4 ea = sCo2[oa];
            const float4 eb = sCo2[oa + RO];
            ex[0] = make_float2(ea.x, eb.x);
            ex[1] = make_float2(ea.y, eb.y);
            ex[2] = make_float2(ea.z, eb.z);
            ex[3] = make_float2(ea.w, eb.w);
          }
#pragma unroll
          for (int j = 0; j < NP; ++j) {
            float2* A = acc[i / 2][j];
            const float2 ww = make_float2(w[i][j], w[i + 1][j]);
            if (PV == kPrecKahan) {
              // compensated: y = w v - c, t = A + y, c = (t - A) - y
              float2* C = kc[i / 2][j];
              const float2 one = make_float2(1.0f, 1.0f);
              const float2 terms[8] = {one, ww, vx, vy, x2, y2, vz, vw};
#pragma unroll
              for (int e = 0; e < 8; ++e) {
                const float2 y = __ffma2_rn(ww, terms[e], make_float2(-C[e % NKC].x, -C[e % NKC].y));
                const float2 t = __fadd2_rn(A[e], y);
                const float2 u = __fadd2_rn(t, make_float2(-A[e].x, -A[e].y));
                C[e % NKC] = __fadd2_rn(u, make_float2(-y.x, -y.y));
                A[e] = t;
              }
            } else {
              A[0] = __fadd2_rn(A[0], ww);
              A[1] = __ffma2_rn(ww, ww, A[1]);
              A[2] = __ffma2_rn(ww, vx, A[2]);
              A[3] = __ffma2_rn(ww, vy, A[3]);
              A[4] = __ffma2_rn(ww, x2, A[4]);
              A[5] = __ffma2_rn(ww, y2, A[5]);
              A[6] = __ffma2_rn(ww, vz, A[6]);
              A[7] = __ffma2_rn(ww, vw, A[7]);
            }
            if (FULL8) {
#pragma unroll
              for (int e = 0; e < 4; ++e) A[(8 + e) % NA] = __ffma2_rn(ww, ex[e], A[(8 + e) % NA]);
            }
          }
        }
      }
      // no barrier here: the next batch's phase A writes only the
      // similarity map, which every warp finished reading (phase B)
      // before the barrier above; its barrier after phase A orders this
      // phase C's reads of the horizontal sums before they are rewritten
    }
  }

  // ---- statistics, alpha, ENL', selection
#pragma unroll
  for (int i = 0; i < PX; ++i) {
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      float A[NA];
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        A[a] = (i & 1) ? acc[i / 2][j][a].y : acc[i / 2][j][a].x;
        if (PV == kPrecKahan && a < NKC) A[a] -= (i & 1) ? kc[i / 2][j][a].y : kc[i / 2][j][a].x;
      }
      const float s0 = A[0], s1 = A[1], s2 = A[2], s3 = A[3], s4 = A[4], s5 = A[5], s6 = A[6], s7 = A[7];
      const float enl = s0 * s0 / s1;
      const float i0 = s2 / s0, i1 = s3 / s0;
      const float v0 = s4 / s0 - i0 * i0, v1 = s5 / s0 - i1 * i1;
      float alpha = 0.0f;
      alpha = fmaxf(alpha, fmaxf(0.0f, (v0 - i0 * i0) / v0));
      alpha = fmaxf(alpha, fmaxf(0.0f, (v1 - i1 * i1) / v1));
      if (P.alpha_zero) alpha = 0.0f;
      const float oma = 1.0f - alpha;
      const float enb = enl / (oma * oma + (alpha * alpha + 2.0f * alpha * (1.0f - alpha) / s0) * enl);
      const int combo = pp.combo[j];
      const int rank = P.combo[combo].rank;
      const bool take = (P.select_mode == 0) || (enb > best.e[i]) || (enb == best.e[i] && rank < best.rank[i]);
      const bool take_fb = !take && best.combo[i] < 0 && combo == P.fallback_combo;
      if (take) {
        best.e[i] = enb;
        best.rank[i] = rank;
      }
      if (take || take_fb) {
        best.combo[i] = combo;
        best.a[i] = alpha;
        best.s0[i] = s0;
        best.m[i][0] = s2;
        best.m[i][1] = s3;
        best.m[i][2] = s6;
        best.m[i][3] = s7;
#pragma unroll
        for (int e = 4; e < NM; ++e) best.m[i][e] = A[(e + 4) % NA];
      }
    }
  }
}

template <int PH0, int PH1, int PH2>
__device__ __forceinline__ bool pass_is(const PassParams& pp) {
  constexpr int NP = np_of<PH0, PH1, PH2>();
  return pp.np == NP && pp.ph[0] == PH0 && (NP < 2 || pp.ph[1] == PH1) && (NP < 3 || pp.ph[2] == PH2);
}

// The kernel: passes of shape A (patch halves A0 < A1 < A2) and, where B0 >=
// 0, of shape B, staged for the largest patch half PHX.
template <int WSH, int PHX, int A0, int A1, int A2, int B0, int B1, int B2, int PX_, int TH_, bool FULL8_>
struct FastK {
  using L = FastL<WSH, PHX, cmax(np_of<A0, A1, A2>(), np_of<B0, B1, B2>()), PX_, TH_, FULL8_>;
};

template <int WSH, int PHX, int A0, int A1, int A2, int B0, int B1, int B2, int PX_, int TH_, bool FULL8_, int PV>
__global__ void __launch_bounds__(FastK<WSH, PHX, A0, A1, A2, B0, B1, B2, PX_, TH_, FULL8_>::L::THREADS, 1)
    nlsar_fast_kernel(const FilterParams P, const SceneDesc* __restrict__ scenes) {
  using L = typename FastK<WSH, PHX, A0, A1, A2, B0, B1, B2, PX_, TH_, FULL8_>::L;
  constexpr int RS = L::RS, RSH = L::RSH, RO = L::RO, TW = L::TW, PX = L::PX;
  constexpr int NT = L::THREADS, NM = L::NM;
  constexpr bool FULL8 = L::FULL8;
  extern __shared__ __align__(128) float4 smem4[];
  float* smem = reinterpret_cast<float*>(smem4);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::OFF_BAR);
  float4* sCs = reinterpret_cast<float4*>(smem + L::OFF_CS);
  float4* sCo = reinterpret_cast<float4*>(smem + L::OFF_CO);
  float4* sCo2 = reinterpret_cast<float4*>(smem + L::OFF_CO2);  // 8-plane input only
  float* sLd = smem + L::OFF_LD;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int y0 = warp * PX;
  if (tid == 0) mbar_init(bar, 1);
  __syncthreads();
  uint32_t parity = 0;

  for (int tile = blockIdx.x; tile < P.total_tiles; tile += gridDim.x) {
    int lo = 0, hi = P.n_scenes - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (scenes[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    const SceneDesc& S = scenes[lo];
    const int lt = tile - S.tile_begin + S.tile_skip;
    const int ty = lt / S.tiles_x, tx = lt - ty * S.tiles_x;
    const int vy0 = ty * L::TH, vx0 = tx * TW;
    const int G = P.G;

    // stage the original covariance (tile + search halo; both of its float4
    // planes for 8-plane input) and the first pass's scaled covariance (tile
    // + largest patch and search halo) with TMA; the barrier orders every
    // thread's reads of the previous tile before the copies overwrite shared
    // memory
    __syncthreads();
    if (tid == 0) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bar, (FULL8 ? 2 : 1) * L::CO_BYTES + L::CS_BYTES);
      if (!P.withhold_staging) {
        tma_load_2d(sCo, &S.tm_co, 4 * (vx0 - WSH + G), vy0 - WSH + G, bar);
        if (FULL8) tma_load_2d(sCo2, &S.tm_co2, 4 * (vx0 - WSH + G), vy0 - WSH + G, bar);
        tma_load_2d(sCs, &S.tm_cs[P.pass[0].scale_slot], 4 * (vx0 - PHX - WSH + G), vy0 - PHX - WSH + G, bar);
      }
    }
    if (!stage_wait(P, bar, parity)) return;
    parity ^= 1u;
    for (int i = tid; i < RS * RSH; i += NT) sLd[i] = pixel_term<PV>(sCs[i]);

    Best<PX, NM> best;
#pragma unroll
    for (int i = 0; i < PX; ++i) {
      best.e[i] = -1.0f;
      best.rank[i] = 0x7fffffff;
      best.combo[i] = -1;
      best.a[i] = 0.f;
      best.s0[i] = 1.f;
#pragma unroll
      for (int d = 0; d < NM; ++d) best.m[i][d] = 0.f;
    }

    int loaded_slot = P.pass[0].scale_slot;
    for (int ps = 0; ps < P.npass; ++ps) {
      const PassParams& pp = P.pass[ps];
      __syncthreads();
      if (pp.scale_slot != loaded_slot) {
        if (tid == 0) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_expect_tx(bar, L::CS_BYTES);
          tma_load_2d(sCs, &S.tm_cs[pp.scale_slot], 4 * (vx0 - PHX - WSH + G), vy0 - PHX - WSH + G, bar);
        }
        if (!stage_wait(P, bar, parity)) return;
        parity ^= 1u;
        for (int i = tid; i < RS * RSH; i += NT) sLd[i] = pixel_term<PV>(sCs[i]);
        loaded_slot = pp.scale_slot;
      }
      if constexpr (B0 < 0) {
        fast_pass<L, A0, A1, A2, PV>(P, pp, smem, best);
      } else {
        if (pass_is<A0, A1, A2>(pp))
          fast_pass<L, A0, A1, A2, PV>(P, pp, smem, best);
        else
          fast_pass<L, B0, B1, B2, PV>(P, pp, smem, best);
      }
    }

    // ---- blend with the centre (weighted_means.cl:79); InSAR input:
    // decompose (covmat_decompose.cl:32-37), 8-plane input: the 8 planes
#pragma unroll
    for (int i = 0; i < PX; ++i) {
      const int y = y0 + i;
      const int vy = vy0 + y, vx = vx0 + lane;
      const int oy = (vy < S.H - 1) ? vy : (vy == S.vH ? S.H - 1 : -1);
      const int ox = (vx < S.W - 1) ? vx : (vx == S.vW ? S.W - 1 : -1);
      if (oy < 0 || ox < 0) continue;
      const int ci = (y + WSH) * RO + (lane + WSH);
      const float4 c = sCo[ci];
      const float alpha = best.a[i], s0 = best.s0[i];
      const float oma = 1.0f - alpha;
      const float c00 = oma * best.m[i][0] / s0 + alpha * c.x;
      const float c11 = oma * best.m[i][1] / s0 + alpha * c.y;
      const float cre = oma * best.m[i][2] / s0 + alpha * c.z;
      const float cim = oma * best.m[i][3] / s0 + alpha * c.w;
      const size_t o = (size_t)oy * S.W + ox;
      if (FULL8) {
        // planes {Re, Im} of C00, C01, C10, C11; the second staged float4 is
        // {Im C00, Re C10, Im C10, Im C11}
        const float4 c2 = sCo2[ci];
        const size_t n = (size_t)S.H * S.W;
        S.cov_out[o] = c00;
        S.cov_out[n + o] = oma * best.m[i][4 % NM] / s0 + alpha * c2.x;
        S.cov_out[2 * n + o] = cre;
        S.cov_out[3 * n + o] = cim;
        S.cov_out[4 * n + o] = oma * best.m[i][5 % NM] / s0 + alpha * c2.y;
        S.cov_out[5 * n + o] = oma * best.m[i][6 % NM] / s0 + alpha * c2.z;
        S.cov_out[6 * n + o] = c11;
        S.cov_out[7 * n + o] = oma * best.m[i][7 % NM] / s0 + alpha * c2.w;
      } else {
        const float am = sqrtf(c00), as = sqrtf(c11);
        const float r = 0.5f * (am + as);
        S.ref[o] = r * r;
        S.phase[o] = atan2f(cim, cre);
        S.coh[o] = sqrtf(cim * cim + cre * cre) / (am * as);
      }
      if (S.sel_out) S.sel_out[o] = best.combo[i];
    }
  }
}

template <int WSH, int PHX, int A0, int A1, int A2, int B0, int B1, int B2, int PX_, int TH_, bool FULL8_,
          int PV = kPrecRatio>
cudaError_t launch_fast_t(const FilterParams& F, const SceneDesc* d_scenes, int grid, cudaStream_t st) {
  using L = typename FastK<WSH, PHX, A0, A1, A2, B0, B1, B2, PX_, TH_, FULL8_>::L;
  const size_t smem = (size_t)L::WORDS * 4;
  static size_t allowed[kMaxDevices];
  const void* fn = (const void*)nlsar_fast_kernel<WSH, PHX, A0, A1, A2, B0, B1, B2, PX_, TH_, FULL8_, PV>;
  const cudaError_t e = allow_dynamic_smem(fn, smem, allowed);
  if (e != cudaSuccess) return e;
  nlsar_fast_kernel<WSH, PHX, A0, A1, A2, B0, B1, B2, PX_, TH_, FULL8_, PV><<<grid, L::THREADS, smem, st>>>(F,
                                                                                                        d_scenes);
  return cudaGetLastError();
}

// pass shapes of a call: 1 every pass {1,2,3}; 2..6 every pass the single
// half 1..5; 7 every pass {1,2,3} or {4,5} with at least one {4,5} (patches
// 3..11 at each scale, InSAR and 8-plane input); 0 none of these
int fast_shape(const FilterParams& F, bool full8) {
  if (F.wsh != 10 || F.npass < 1) return 0;
  auto is = [](const PassParams& p, int n, int a0, int a1, int a2) {
    return p.np == n && p.ph[0] == a0 && (n < 2 || p.ph[1] == a1) && (n < 3 || p.ph[2] == a2);
  };
  bool all123 = true, all45_or_123 = true, any45 = false, single = true;
  const int h0 = F.pass[0].ph[0];
  for (int i = 0; i < F.npass; ++i) {
    const PassParams& p = F.pass[i];
    const bool s123 = is(p, 3, 1, 2, 3), s45 = is(p, 2, 4, 5, -1);
    all123 = all123 && s123;
    all45_or_123 = all45_or_123 && (s123 || s45);
    any45 = any45 || s45;
    single = single && p.np == 1 && p.ph[0] == h0;
  }
  if (all123) return 1;
  if (single && h0 >= 1 && h0 <= (full8 ? 3 : 5)) return 1 + h0;
  if (all45_or_123 && any45) return 7;
  return 0;
}

template <int PX_>
cudaError_t launch_fast_insar(int shape, const FilterParams& F, const SceneDesc* d_scenes, int grid,
                              cudaStream_t st) {
  constexpr int T = kFastTileH;
  if (shape == 1 && PX_ == 2) {
    // the arithmetic variants of the precision study (headline shape only)
    switch (F.prec) {
      case kPrecLog2: return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, T, false, kPrecLog2>(F, d_scenes, grid, st);
      case kPrecLogf: return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, T, false, kPrecLogf>(F, d_scenes, grid, st);
      case kPrecKahan:
        return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, T, false, kPrecKahan>(F, d_scenes, grid, st);
      case kPrecHalf: return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, T, false, kPrecHalf>(F, d_scenes, grid, st);
      default: break;
    }
  }
  switch (shape) {
    case 1: return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, PX_, T, false>(F, d_scenes, grid, st);
    case 2: return launch_fast_t<10, 1, 1, -1, -1, -1, -1, -1, PX_, T, false>(F, d_scenes, grid, st);
    case 3: return launch_fast_t<10, 2, 2, -1, -1, -1, -1, -1, PX_, T, false>(F, d_scenes, grid, st);
    default: return launch_fast_t<10, 3, 3, -1, -1, -1, -1, -1, PX_, T, false>(F, d_scenes, grid, st);
  }
}

}  // namespace

// Number of thread blocks that gave up waiting for a TMA staging copy on the
// current device since the last take; the ledger is read and reset by one
// atomic exchange on the device, so no increment is lost, and takes from
// several host threads are serialised.  Their tiles were left unwritten.
int take_stage_timeouts(int* count) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  int n = 0;
  take_stage_timeouts_kernel<<<1, 1, 0, cudaStreamPerThread>>>();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyFromSymbolAsync(&n, g_stage_taken, sizeof n, 0, cudaMemcpyDeviceToHost, cudaStreamPerThread);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
  *count = e == cudaSuccess ? n : 0;
  return e == cudaSuccess ? 0 : -1;
}

// Specialisations available: the search window 21 (half 10) with every pass
// holding the patch halves {1,2,3} (patches 3,5,7), or every pass one and the
// same patch half (reference selection; halves 1..5 for InSAR input, 1..3 for
// 8-plane input), or every pass {1,2,3} or {4,5} (patches 3..11 at each
// scale, the reference example's settings).
bool fast_kernel_supported(const FilterParams& F, bool full8) { return fast_shape(F, full8) != 0; }

// Instantiations the batch autotuner may time: 0 and 1 (2 or 4 pixels per
// thread on 32 x 32 tiles) for InSAR input with patches up to 7, and 2 (32 x 16
// tiles, 2 pixels per thread, 256-thread CTAs) for the patches {3,5,7} shape;
// 1 otherwise.  Variant 2 needs the scene geometry of 16-row tiles.
int fast_variants(const FilterParams& F, bool full8) {
  const int shape = fast_shape(F, full8);
  if (full8 || shape == 0 || shape >= 5) return 1;
  return shape == 1 ? 3 : 2;
}

// InSAR input (32 x 32 tiles): variant 0 has 2 pixels per thread in
// 512-thread CTAs (the default), variant 1 4 pixels per thread in 256-thread
// CTAs (the patch sizes up to 7), variant 2 32 x 16 tiles with 2 pixels per
// thread in 256-thread CTAs (patches {3,5,7}; F.tile_h must be 16); the batch
// autotuner times them (fast_variants).  8-plane
// covariance input: 32 x 24 tiles, 2 pixels per thread, 384-thread CTAs (the
// second staged covariance plane and its four accumulators per patch size
// need the room).
cudaError_t launch_nlsar_fast(const FilterParams& F, const SceneDesc* d_scenes, int grid, cudaStream_t st,
                              int variant, bool full8) {
  const int shape = fast_shape(F, full8);
  constexpr int T8 = kFastTileH8, T = kFastTileH;
  if (full8) {
    switch (shape) {
      case 1: return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, T8, true>(F, d_scenes, grid, st);
      case 2: return launch_fast_t<10, 1, 1, -1, -1, -1, -1, -1, 2, T8, true>(F, d_scenes, grid, st);
      case 3: return launch_fast_t<10, 2, 2, -1, -1, -1, -1, -1, 2, T8, true>(F, d_scenes, grid, st);
      case 7: return launch_fast_t<10, 5, 1, 2, 3, 4, 5, -1, 2, T8, true>(F, d_scenes, grid, st);
      default: return launch_fast_t<10, 3, 3, -1, -1, -1, -1, -1, 2, T8, true>(F, d_scenes, grid, st);
    }
  }
  switch (shape) {
    case 5: return launch_fast_t<10, 4, 4, -1, -1, -1, -1, -1, 2, T, false>(F, d_scenes, grid, st);
    case 6: return launch_fast_t<10, 5, 5, -1, -1, -1, -1, -1, 2, T, false>(F, d_scenes, grid, st);
    case 7: return launch_fast_t<10, 5, 1, 2, 3, 4, 5, -1, 2, T, false>(F, d_scenes, grid, st);
    default:
      if (variant == 2 && shape == 1 && F.tile_h == kFastTileHHalf)
        return launch_fast_t<10, 3, 1, 2, 3, -1, -1, -1, 2, kFastTileHHalf, false>(F, d_scenes, grid, st);
      if (variant == 1) return launch_fast_insar<4>(shape, F, d_scenes, grid, st);
      return launch_fast_insar<2>(shape, F, d_scenes, grid, st);
  }
}

}  // namespace dcl

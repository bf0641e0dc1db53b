// Shared host/device definitions of the fused NL-SAR engine.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace dcl {

constexpr int kMaxScales = 8;        // distinct scale sizes per call
constexpr int kMaxCombos = 48;       // (patch, scale) combinations per call
constexpr int kMaxPasses = 24;       // (scale, patch group) passes per call
constexpr int kPatchPerPass = 3;     // patch sizes accumulated together
constexpr int kMaxLut = 256;         // LUT entries per combination
constexpr int kMaxGauss = 81;        // scale sizes up to 9
constexpr int kTileW = 32;           // output columns per CTA tile (one lane per column)
constexpr int kWarps = 8;            // warps per CTA
constexpr int kThreads = kWarps * 32;
constexpr int kMaxSws = 41;          // search windows up to 41x41
constexpr int kMaxPatchHalf = 7;     // patches up to 15x15

// One (patch, scale) combination.
struct ComboParams {
  float dmin, dmax;  // dissimilarity range of the training LUT
  float span;        // dmax - dmin
  float lm1;         // lut_size - 1
  int rank;          // position of the key in the (patch, scale)-ordered statistics map
};

// One pass over all search-window offsets: one scale, up to three patch sizes.
struct PassParams {
  int scale_slot;            // index of the scale's padded arrays in SceneDesc
  int np;                    // patches in this pass
  int ph[kPatchPerPass];     // patch half sizes, ascending
  int combo[kPatchPerPass];  // combination index (reference loop order: scale outer, patch inner)
};

// One scene of a (possibly batched) launch.  All padded arrays share one
// frame: frame index = virtual coordinate + G, row pitch `pitch` elements.
struct SceneDesc {
  // TMA descriptors for the specialised kernel's staging: 2-D float views
  // [Hp][4 pitch] of the cori and cs[s] frames with the boxes of one tile's
  // staged regions; zero when that kernel is not used
  CUtensorMap tm_co;
  CUtensorMap tm_co2;  // cori2 (8-plane covariance input)
  CUtensorMap tm_cs[kMaxScales];
  const float4* cori;   // un-rescaled covariance {C00, C11, Re C01, Im C01}
  const float4* cori2;  // covariance path only: {Im C00, Re C10, Im C10, Im C11}
  const float4* cs[kMaxScales];  // rescaled + Gaussian-averaged {C00, C11, Re C01, Im C01}
  const float* ld[kMaxScales];   // ln det of cs
  float* ref;
  float* phase;
  float* coh;
  float* cov_out;  // covariance path: [8][H][W]
  int* sel_out;    // optional selected combination per pixel
  int H, W;
  int vH, vW;      // virtual coordinate whose result lands in row H-1 / column W-1
  int pitch;
  int tiles_x, tiles_y;
  int tile_begin;  // first launch-wide tile index of this scene
  int tile_skip;   // scene tiles before the first one this launch covers (chunked scenes)
};

struct FilterParams {
  int sws, wsh;
  int phm;         // largest patch half (similarity halo of a tile)
  int G;           // guard of the padded frame (wsh + phm + largest scale half)
  int n_off;       // non-centre offsets of the search window (sws*sws - 1)
  int npass;
  int ncombo;
  int select_mode;  // 0: the single combination of the only pass; 1: ENL argmax
  int alpha_zero;   // reference mode with a key that was not computed: alpha 0
  int fallback_combo;
  int K;            // offsets per batch
  int tile_h;       // output rows per tile
  float c2d;        // 2 * dim * ln 2
  int n_scenes;
  int total_tiles;
  PassParams pass[kMaxPasses];
  ComboParams combo[kMaxCombos];
  const float* wtab;  // [ncombo][kMaxLut] composite weights (device)
  // Staging timeouts of the specialised kernel: a thread block that gives up
  // waiting for a TMA staging copy leaves its remaining tiles unwritten and is
  // counted in the device-wide ledger (dcl_take_stage_timeouts) and, where
  // `timeouts` is set, in that per-launch device word too.
  int* timeouts;
  int stage_polls;     // poll limit of a staging wait; 0: the default
  int withhold_staging;  // tests only: arm the staging barrier without issuing the copies
  // arithmetic of the specialised kernel's similarities and sums: 0 the ratio
  // form (default), 1..4 the alternatives of the precision study (nlsar_fast.cu)
  int prec;
};

struct GaussArg {
  float g[kMaxGauss];
};

// Shared-memory carve-up of the fused kernel, in 4-byte words.
struct SmemLayout {
  int rs_w, rs_h;    // region of the scaled covariance: tile + 2*(phm+wsh)
  int ro_w, ro_h;    // region of the original covariance: tile + 2*wsh
  int sim_w, sim_h;  // similarity map: tile + 2*phm
  int off_cs, off_ld, off_co, off_co2, off_sim, off_h, off_w, total;
};

__host__ __device__ inline SmemLayout smem_layout(int tile_h, int wsh, int phm, int K, bool full8) {
  SmemLayout L;
  L.rs_w = kTileW + 2 * (phm + wsh);
  L.rs_h = tile_h + 2 * (phm + wsh);
  L.ro_w = kTileW + 2 * wsh;
  L.ro_h = tile_h + 2 * wsh;
  L.sim_w = kTileW + 2 * phm;
  L.sim_h = tile_h + 2 * phm;
  int o = 0;
  L.off_cs = o;
  o += 4 * L.rs_w * L.rs_h;
  L.off_co = o;
  o += 4 * L.ro_w * L.ro_h;
  L.off_co2 = o;
  if (full8) o += 4 * L.ro_w * L.ro_h;
  L.off_ld = o;
  o += L.rs_w * L.rs_h;
  L.off_sim = o;
  o += K * L.sim_w * L.sim_h;
  L.off_h = o;
  o += K * kPatchPerPass * L.sim_h * kTileW;
  L.off_w = o;
  o += kPatchPerPass * kMaxLut;
  L.total = o;
  return L;
}

// The prep kernels fill frame rows [row0, row1) of their outputs (the grid
// covers those rows); reads are clamped to the whole frame.
__global__ void prep_cov_insar_kernel(const float* a1, const float* a2, const float* phi, int H, int W,
                                      float4* cori, int Hp, int Wp, int pitch, int G, int row0, int row1);
__global__ void prep_cov_planes_kernel(const float* cin, int H, int W, float4* cori, float4* cori2, int Hp, int Wp,
                                       int pitch, int G, int row0, int row1);
__global__ void prep_scale_kernel(const float4* cori, int Hp, int Wp, int pitch, int s, GaussArg ga, float gamma,
                                  float4* cs, float* ld, int row0, int row1);
// Launches the fused kernel: one CTA per tile (grid = tiles), `smem` bytes of
// dynamic shared memory; full8 selects the 8-plane covariance variant.
cudaError_t launch_nlsar_fused(bool full8, const FilterParams& F, const SceneDesc* d_scenes, size_t smem, int grid,
                               cudaStream_t st);

// Tile rows of the specialised kernel: InSAR input, 8-plane covariance input,
// and the half-height InSAR tiles the batch autotuner may choose.
constexpr int kFastTileH = 32;
constexpr int kFastTileH8 = 24;
constexpr int kFastTileHHalf = 16;

// Staged regions of the specialised kernel's tile (32 x tile_h outputs), in
// pixels (width x height): scaled covariance RS x RSH, original covariance
// RO x ROH.  The scaled covariance box is one pixel wider than the tile and
// its halo, so that its rows in shared memory have an odd pitch (the
// kernel's phase A reads it down columns, one row per lane, free of bank
// conflicts only at an odd pitch); the extra pixel is not used.
struct FastStage {
  int RS, RSH, RO, ROH;
};
__host__ __device__ inline FastStage fast_stage(int wsh, int phm, int tile_h) {
  FastStage f;
  f.RS = 32 + 2 * (phm + wsh) + 1;
  f.RSH = tile_h + 2 * (phm + wsh);
  f.RO = 32 + 2 * wsh;
  f.ROH = tile_h + 2 * wsh;
  return f;
}

// The compile-time specialised kernel (nlsar_fast.cu) for the common
// configurations; fast_kernel_supported() tells whether `F` has one (for
// 8-plane covariance input when `full8`).
bool fast_kernel_supported(const FilterParams& F, bool full8);
// number of instantiations (launch_nlsar_fast variants) the autotuner may time
int fast_variants(const FilterParams& F, bool full8);
// Thread blocks of the specialised kernel that gave up waiting for a staging
// copy on the current device since the last take (read and reset in one
// atomic exchange); 0 on success, -1 on a CUDA error
int take_stage_timeouts(int* count);
cudaError_t launch_nlsar_fast(const FilterParams& F, const SceneDesc* d_scenes, int grid, cudaStream_t st,
                              int variant = 0, bool full8 = false);

}  // namespace dcl

// Host orchestration of the fused NL-SAR engine and its C ABI.
//
// Mirrors the reference's driver (src/compute/nlsar/nlsar.cpp:81-194) and
// per-tile pipeline (src/compute/nlsar/nlsar_filter_sub_image.cpp:146-390)
// without tiles on the host: arguments are validated, the (patch, scale)
// combinations are ordered as the reference orders them, the LUTs are folded
// into one composite weight table per combination, the scene is expanded once
// into its clamp-padded virtual plane, and one fused launch filters every tile.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_common.cuh"
#include "nlsar_plan.h"

namespace dcl {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_error(cudaError_t e, const char* where) {
  if (e == cudaErrorMemoryAllocation) return set_error(DCL_ERR_OUT_OF_MEMORY, "%s: %s", where, cudaGetErrorString(e));
  return set_error(DCL_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

const char* last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// plan: validated parameters -> FilterParams
// ---------------------------------------------------------------------------

std::vector<float> gauss_weights(int s) {
  // cl_wrappers/covmat_spatial_avg.cpp:35-50 (exponent in double, float storage,
  // float normalisation sum)
  std::vector<float> g;
  const int ssh = (s - 1) / 2;
  for (int x = -ssh; x <= ssh; ++x)
    for (int y = -ssh; y <= ssh; ++y) {
      const double den = std::pow((double)((float)ssh + 0.5f), 2.0);
      g.push_back((float)std::exp(-M_PI * (x * x + y * y) / den));
    }
  float K = 0.0f;
  for (float e : g) K += e;
  for (float& e : g) e = e / K;
  return g;
}

float rescale_gamma_2x2() {
  // covmat_rescale.cl:25-26 with nlooks = 1, dimension = 2
  return std::pow(std::min(1.0f / 2.0f, 1.0f), 0.33333f);
}

static int validate_sizes(int sws, const int* patches, int np, const int* scales, int ns, std::vector<int>& P,
                          std::vector<int>& S) {
  if (sws < 1 || sws % 2 == 0 || sws > kMaxSws)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "search_window_size must be odd and in [1, %d], got %d", kMaxSws, sws);
  if (!patches || np < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "patch_sizes must not be empty");
  if (!scales || ns < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "scale_sizes must not be empty");
  P.clear();
  S.clear();
  for (int i = 0; i < np; ++i) {
    const int p = patches[i];
    if (p < 1 || p % 2 == 0 || p > 2 * kMaxPatchHalf + 1)
      return set_error(DCL_ERR_INVALID_ARGUMENT, "patch sizes must be odd and in [1, %d], got %d",
                       2 * kMaxPatchHalf + 1, p);
    if (std::find(P.begin(), P.end(), p) == P.end()) P.push_back(p);
  }
  for (int i = 0; i < ns; ++i) {
    const int s = scales[i];
    if (s < 1 || s % 2 == 0 || s * s > kMaxGauss)
      return set_error(DCL_ERR_INVALID_ARGUMENT, "scale sizes must be odd and in [1, 9], got %d", s);
    if (std::find(S.begin(), S.end(), s) == S.end()) S.push_back(s);
  }
  if ((int)S.size() > kMaxScales) return set_error(DCL_ERR_INVALID_ARGUMENT, "at most %d scale sizes", kMaxScales);
  if ((int)(P.size() * S.size()) > kMaxCombos)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "at most %d (patch, scale) combinations", kMaxCombos);
  return DCL_OK;
}

// DESPECKCL_B200_GENERIC=1 routes every call to the generic kernel (used by
// the tests to check both kernels against each other)
static const bool g_force_generic = [] {
  const char* s = std::getenv("DESPECKCL_B200_GENERIC");
  return s && s[0] == '1';
}();

int make_plan(int sws, const int* patches, int np, const int* scales, int ns, const dcl_stats_entry* stats,
              int nstats, float h, float c, int select_mode, bool full8, Plan& pl) {
  std::vector<int> Pv, Sv;
  int rc = validate_sizes(sws, patches, np, scales, ns, Pv, Sv);
  if (rc) return rc;
  if (!stats || nstats < 1) return set_error(DCL_ERR_MISSING_STATS, "no NL-SAR statistics given");
  if (select_mode != DCL_SELECT_REFERENCE && select_mode != DCL_SELECT_ARGMAX_ENL)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "unknown select_mode %d", select_mode);
  if (!(h > 0.0f) || !std::isfinite(h)) return set_error(DCL_ERR_INVALID_ARGUMENT, "h_param must be > 0");
  if (!std::isfinite(c)) return set_error(DCL_ERR_INVALID_ARGUMENT, "c_param must be finite");
  // the statistics map, keyed and ordered like std::map<nlsar::params, ...>
  // (parameters.h:37-40: lexicographic (patch, scale))
  std::map<std::pair<int, int>, const dcl_stats_entry*> smap;
  for (int i = 0; i < nstats; ++i) {
    const dcl_stats_entry& e = stats[i];
    if (e.lut_size < 2 || e.lut_size > (unsigned)kMaxLut || !e.quantilles || !e.chi2cdf_inv)
      return set_error(DCL_ERR_INVALID_ARGUMENT, "stats (%d,%d): lut_size must be in [2, %d] with both tables",
                       e.patch_size, e.scale_size, kMaxLut);
    if (!(e.dissims_max > e.dissims_min))
      return set_error(DCL_ERR_INVALID_ARGUMENT, "stats (%d,%d): dissims_max must exceed dissims_min", e.patch_size,
                       e.scale_size);
    smap[{e.patch_size, e.scale_size}] = &e;
  }
  std::map<std::pair<int, int>, int> rank;
  {
    int r = 0;
    for (auto& kv : smap) rank[kv.first] = r++;
  }
  for (int s : Sv)
    for (int p : Pv)
      if (!smap.count({p, s}))
        return set_error(DCL_ERR_MISSING_STATS, "no statistics for patch size %d, scale size %d", p, s);

  FilterParams& F = pl.P;
  std::memset(&F, 0, sizeof F);
  // tests only: DESPECKCL_B200_TEST_WITHHOLD_STAGING=1 arms the specialised
  // kernel's staging barrier without issuing the copies, with a short poll
  // limit, so that every staging wait runs out and the reporting path runs (no
  // copy is then pending when a thread block gives up)
  // precision study: DESPECKCL_B200_PRECISION=n selects the specialised
  // kernel's arithmetic variant n (0 default; see nlsar_fast.cu)
  if (const char* pv = std::getenv("DESPECKCL_B200_PRECISION")) {
    const int v = std::atoi(pv);
    if (v >= 0 && v <= 4) F.prec = v;
  }
  if (const char* w = std::getenv("DESPECKCL_B200_TEST_WITHHOLD_STAGING")) {
    if (std::strcmp(w, "1") == 0) {
      F.withhold_staging = 1;
      F.stage_polls = 256;
    }
  }
  pl.full8 = full8;
  pl.px = full8 ? 2 : 4;
  pl.scales = Sv;
  pl.slot_used.assign(Sv.size(), 0);
  F.sws = sws;
  F.wsh = (sws - 1) / 2;
  F.n_off = sws * sws - 1;
  F.select_mode = select_mode == DCL_SELECT_ARGMAX_ENL ? 1 : 0;
  F.c2d = 2 * 2 * std::log(2.0f);
  F.fallback_combo = 0;
  F.tile_h = kWarps * pl.px;
  const int pmax = *std::max_element(Pv.begin(), Pv.end());
  const int smax = *std::max_element(Sv.begin(), Sv.end());
  pl.overlap = (pmax - 1) / 2 + F.wsh + (smax - 1) / 2;  // nlsar.cpp:41-51

  // combinations in the reference loop order (nlsar_filter_sub_image.cpp:449-470)
  struct C { int p, s, slot; };
  std::vector<C> combos;
  for (size_t si = 0; si < Sv.size(); ++si)
    for (int p : Pv) combos.push_back({p, Sv[si], (int)si});
  F.ncombo = (int)combos.size();
  pl.wtab.assign((size_t)F.ncombo * kMaxLut, 0.0f);
  for (int ci = 0; ci < F.ncombo; ++ci) {
    const dcl_stats_entry& e = *smap[{combos[ci].p, combos[ci].s}];
    ComboParams& cp = F.combo[ci];
    cp.dmin = e.dissims_min;
    cp.dmax = e.dissims_max;
    cp.span = e.dissims_max - e.dissims_min;
    cp.lm1 = (float)(int)(e.lut_size - 1);
    cp.rank = rank[{combos[ci].p, combos[ci].s}];
    // compute_weights.cl:49-51 folded into one table indexed by the first LUT index
    for (unsigned k = 0; k < e.lut_size; ++k) {
      const float q = e.quantilles[k];
      float qi = q * (float)(int)(e.lut_size - 1);
      unsigned i2 = (qi > 0.0f) ? (unsigned)qi : 0u;
      if (i2 >= e.lut_size) i2 = e.lut_size - 1;
      const float x = e.chi2cdf_inv[i2];
      pl.wtab[(size_t)ci * kMaxLut + k] = std::exp(-std::fabs(x - c) / h);
    }
  }

  // passes
  auto add_pass = [&](int slot, std::vector<int> ps) {
    std::sort(ps.begin(), ps.end());
    for (size_t g = 0; g < ps.size(); g += kPatchPerPass) {
      if (F.npass >= kMaxPasses) return false;
      PassParams& pp = F.pass[F.npass++];
      pp.scale_slot = slot;
      pp.np = (int)std::min<size_t>(kPatchPerPass, ps.size() - g);
      for (int j = 0; j < pp.np; ++j) {
        const int p = ps[g + j];
        pp.ph[j] = (p - 1) / 2;
        for (int ci = 0; ci < F.ncombo; ++ci)
          if (combos[ci].p == p && combos[ci].slot == slot) pp.combo[j] = ci;
      }
      pl.slot_used[slot] = 1;
    }
    return true;
  };
  if (F.select_mode == 1) {
    for (size_t si = 0; si < Sv.size(); ++si)
      if (!add_pass((int)si, Pv)) return set_error(DCL_ERR_INVALID_ARGUMENT, "too many (scale, patch) passes");
  } else {
    // best_params.cpp:27-54: every pixel takes the last key of the map.  A key
    // outside patch_sizes x scale_sizes maps to index 0 of the loop order
    // (params2idx default) with the zero-initialised alpha
    // (nlsar_filter_sub_image.cpp:418-422, 541, 545)
    const std::pair<int, int> last = smap.rbegin()->first;
    int ci_last = -1;
    for (int ci = 0; ci < F.ncombo; ++ci)
      if (combos[ci].p == last.first && combos[ci].s == last.second) ci_last = ci;
    if (ci_last < 0) {
      ci_last = 0;
      F.alpha_zero = 1;
    }
    add_pass(combos[ci_last].slot, {combos[ci_last].p});
  }
  F.phm = 0;
  for (int i = 0; i < F.npass; ++i)
    for (int j = 0; j < F.pass[i].np; ++j) F.phm = std::max(F.phm, F.pass[i].ph[j]);
  pl.shm = 0;
  for (size_t si = 0; si < Sv.size(); ++si)
    if (pl.slot_used[si]) pl.shm = std::max(pl.shm, (Sv[si] - 1) / 2);
  F.G = F.wsh + F.phm + pl.shm;
  // the specialised kernel serves the common settings, in 32 x 32 tiles for
  // InSAR input and 32 x 24 tiles for 8-plane covariance input
  pl.fast = !g_force_generic && fast_kernel_supported(F, full8);
  if (pl.fast && full8) F.tile_h = kFastTileH8;
  return DCL_OK;
}

// ---------------------------------------------------------------------------
// device state
// ---------------------------------------------------------------------------

static std::mutex g_init_mu;
static bool g_pool_ready[64];

int ensure_device_ready(int& dev) {
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (dev >= 0 && dev < 64 && !g_pool_ready[dev]) {
    // keep freed scratch in the stream-ordered pool between calls
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    g_pool_ready[dev] = true;
  }
  return DCL_OK;
}

int choose_k(const Plan& pl, size_t& smem_bytes) {
  int optin = 0, dev = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || optin <= 0)
    optin = 227 * 1024;
  for (int K = 8; K >= 1; --K) {
    const SmemLayout L = smem_layout(pl.P.tile_h, pl.P.wsh, pl.P.phm, K, pl.full8);
    const size_t b = (size_t)L.total * 4;
    if (b <= (size_t)optin) {
      smem_bytes = b;
      return K;
    }
  }
  return 0;
}

SceneGeom scene_geom(const Plan& pl, int H, int W) {
  SceneGeom g;
  g.H = H;
  g.W = W;
  g.vH = H - 1 + pl.overlap;
  g.vW = W - 1 + pl.overlap;
  g.tiles_y = (g.vH + 1 + pl.P.tile_h - 1) / pl.P.tile_h;
  g.tiles_x = (g.vW + 1 + kTileW - 1) / kTileW;
  g.Hp = g.tiles_y * pl.P.tile_h + 2 * pl.P.G;
  g.Wp = g.tiles_x * kTileW + 2 * pl.P.G;
  g.pitch = (g.Wp + 7) / 8 * 8;
  return g;
}

size_t scratch_bytes(const Plan& pl, const SceneGeom& g) {
  const size_t plane = (size_t)g.Hp * g.pitch;
  size_t b = plane * sizeof(float4) * (pl.full8 ? 2 : 1);
  for (size_t si = 0; si < pl.scales.size(); ++si)
    if (pl.slot_used[si]) b += plane * (sizeof(float4) + sizeof(float));
  return b;
}

// cuTensorMapEncodeTiled, fetched from the driver through the runtime (no
// link against libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// A 2-D float tensor map: `inner` floats per row, `rows` rows, row stride
// `stride` bytes, box `box_inner` x `box_rows`.  The constraints of the TMA
// unit are checked here: base 16-byte aligned, stride a multiple of 16
// bytes, box inner extent a multiple of 16 bytes, box sides at most 256.
static int encode_map_2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t rows, uint64_t stride,
                         uint32_t box_inner, uint32_t box_rows) {
  EncodeTiledFn fn = encode_tiled_fn();
  if (!fn) return set_error(DCL_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (stride & 15) || ((box_inner * 4) & 15) || box_inner > 256 ||
      box_rows > 256 || box_inner > inner || box_rows > rows)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "TMA map: misaligned frame or box");
  const cuuint64_t dims[2] = {inner, rows};
  const cuuint64_t strides[1] = {stride};
  const cuuint32_t box[2] = {box_inner, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(DCL_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DCL_OK;
}

// Carve the scratch of one scene and fill its descriptor (pointers into
// `base`, and the TMA maps of the specialised kernel when the plan uses it).
int carve_scene(const Plan& pl, const SceneGeom& g, char* base, SceneDesc& d) {
  const size_t plane = (size_t)g.Hp * g.pitch;
  char* p = base;
  d.cori = reinterpret_cast<float4*>(p);
  p += plane * sizeof(float4);
  d.cori2 = nullptr;
  if (pl.full8) {
    d.cori2 = reinterpret_cast<float4*>(p);
    p += plane * sizeof(float4);
  }
  for (int si = 0; si < kMaxScales; ++si) {
    d.cs[si] = nullptr;
    d.ld[si] = nullptr;
  }
  for (size_t si = 0; si < pl.scales.size(); ++si)
    if (pl.slot_used[si]) {
      d.cs[si] = reinterpret_cast<float4*>(p);
      p += plane * sizeof(float4);
      d.ld[si] = reinterpret_cast<float*>(p);
      p += plane * sizeof(float);
    }
  d.H = g.H;
  d.W = g.W;
  d.vH = g.vH;
  d.vW = g.vW;
  d.pitch = g.pitch;
  d.tiles_x = g.tiles_x;
  d.tiles_y = g.tiles_y;
  std::memset(&d.tm_co, 0, sizeof d.tm_co);
  std::memset(&d.tm_co2, 0, sizeof d.tm_co2);
  std::memset(d.tm_cs, 0, sizeof d.tm_cs);
  if (!uses_specialised_kernel(pl)) return DCL_OK;
  // the specialised kernel stages, per tile, the original covariance box at
  // (vx0 - wsh + G, vy0 - wsh + G) and the scaled covariance box at
  // (vx0 - phm - wsh + G, vy0 - phm - wsh + G), in float4 pixels: x origins
  // in floats are multiples of 4 (16 bytes), as the TMA unit requires
  const FastStage fs = fast_stage(pl.P.wsh, pl.P.phm, pl.P.tile_h);
  const uint64_t Hp = (uint64_t)g.Hp, pitch = (uint64_t)g.pitch;
  int rc = encode_map_2d(&d.tm_co, d.cori, 4 * pitch, Hp, pitch * 16, 4 * fs.RO, fs.ROH);
  if (rc == DCL_OK && pl.full8) rc = encode_map_2d(&d.tm_co2, d.cori2, 4 * pitch, Hp, pitch * 16, 4 * fs.RO, fs.ROH);
  for (size_t si = 0; si < pl.scales.size() && rc == DCL_OK; ++si)
    if (pl.slot_used[si])
      rc = encode_map_2d(&d.tm_cs[si], d.cs[si], 4 * pitch, Hp, pitch * 16, 4 * fs.RS, fs.RSH);
  return rc;
}

// Optional timing of the fused kernel (dcl_profile_begin / dcl_profile_end):
// CUDA events recorded on the launching stream around every fused launch of
// the calling thread.
struct ProfileState {
  bool on = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  long launches = 0;  // all kernels launched by the library while profiling
};
static thread_local ProfileState g_prof;

cudaError_t allow_dynamic_smem(const void* func, size_t bytes, size_t* cache) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (bytes <= cache[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cache[dev] = bytes;
  return e;
}

void profile_count(int n) {
  if (g_prof.on) g_prof.launches += n;
}

bool uses_specialised_kernel(const Plan& pl) { return pl.fast; }

int launch_prep_rows(const Plan& pl, const SceneGeom& g, const SceneDesc& d, const float* a1, const float* a2,
                     const float* phi, const float* cov_in, int co0, int co1, int cs0, int cs1, cudaStream_t st) {
  const dim3 blk(32, 8);
  const unsigned gx = (unsigned)(g.Wp + 31) / 32;
  if (co1 > co0) {
    profile_count(1);
    const dim3 grd(gx, (unsigned)(co1 - co0 + 7) / 8);
    if (pl.full8)
      prep_cov_planes_kernel<<<grd, blk, 0, st>>>(cov_in, g.H, g.W, const_cast<float4*>(d.cori),
                                                  const_cast<float4*>(d.cori2), g.Hp, g.Wp, g.pitch, pl.P.G, co0, co1);
    else
      prep_cov_insar_kernel<<<grd, blk, 0, st>>>(a1, a2, phi, g.H, g.W, const_cast<float4*>(d.cori), g.Hp, g.Wp,
                                                 g.pitch, pl.P.G, co0, co1);
  }
  if (cs1 <= cs0) return DCL_OK;
  const float gamma = rescale_gamma_2x2();
  const dim3 grd(gx, (unsigned)(cs1 - cs0 + 7) / 8);
  for (size_t si = 0; si < pl.scales.size(); ++si) {
    if (!pl.slot_used[si]) continue;
    GaussArg ga;
    std::memset(&ga, 0, sizeof ga);
    const std::vector<float> gw = gauss_weights(pl.scales[si]);
    std::copy(gw.begin(), gw.end(), ga.g);
    profile_count(1);
    prep_scale_kernel<<<grd, blk, 0, st>>>(d.cori, g.Hp, g.Wp, g.pitch, pl.scales[si], ga, gamma,
                                           const_cast<float4*>(d.cs[si]), const_cast<float*>(d.ld[si]), cs0, cs1);
  }
  return DCL_OK;
}

int launch_prep(const Plan& pl, const SceneGeom& g, const SceneDesc& d, const float* a1, const float* a2,
                const float* phi, const float* cov_in, cudaStream_t st) {
  return launch_prep_rows(pl, g, d, a1, a2, phi, cov_in, 0, g.Hp, 0, g.Hp, st);
}

int launch_fused(const Plan& pl, const FilterParams& F, const SceneDesc* d_scenes, size_t smem, cudaStream_t st,
                 int variant) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (g_prof.on) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
  }
  const bool fast = pl.fast && fast_kernel_supported(F, pl.full8);
  const cudaError_t e = fast ? launch_nlsar_fast(F, d_scenes, F.total_tiles, st, variant, pl.full8)
                             : launch_nlsar_fused(pl.full8, F, d_scenes, smem, F.total_tiles, st);
  if (g_prof.on) {
    cudaEventRecord(b, st);
    g_prof.ev.push_back({a, b});
    g_prof.launches += 1;
  }
  if (e != cudaSuccess) return cuda_error(e, "NL-SAR fused launch");
  return DCL_OK;
}

// ---------------------------------------------------------------------------
// one call on device pointers (single scene or batch)
// ---------------------------------------------------------------------------

struct SceneIO {
  const float *a1, *a2, *phi, *cov_in;
  float *ref, *phase, *coh, *cov_out;
  int* sel;
  int H, W;
};

int run_device(const Plan& pl0, const std::vector<SceneIO>& io, cudaStream_t st) {
  int dev;
  int rc = ensure_device_ready(dev);
  if (rc) return rc;
  Plan pl = pl0;
  size_t smem = 0;
  const int K = choose_k(pl, smem);
  if (K < 1) return set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
  pl.P.K = K;

  std::vector<SceneGeom> geo;
  std::vector<size_t> offs;
  size_t total = 0;
  int tiles = 0;
  for (const SceneIO& s : io) {
    if (s.H < 1 || s.W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
    geo.push_back(scene_geom(pl, s.H, s.W));
    offs.push_back(total);
    total += (scratch_bytes(pl, geo.back()) + 255) / 256 * 256;
    const long long t = (long long)geo.back().tiles_x * geo.back().tiles_y;
    if (t + tiles > 0x7fffffff) return set_error(DCL_ERR_INVALID_ARGUMENT, "scene too large");
    tiles += (int)t;
  }
  const size_t desc_bytes = io.size() * sizeof(SceneDesc);
  const size_t wtab_bytes = pl.wtab.size() * sizeof(float);
  char* scratch = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, total + desc_bytes + wtab_bytes + 512, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(scratch)");
  SceneDesc* d_desc = reinterpret_cast<SceneDesc*>(scratch + (total + 255) / 256 * 256);
  float* d_wtab = reinterpret_cast<float*>(reinterpret_cast<char*>(d_desc) + (desc_bytes + 255) / 256 * 256);

  std::vector<SceneDesc> desc(io.size());
  int tb = 0;
  for (size_t i = 0; i < io.size(); ++i) {
    std::memset(&desc[i], 0, sizeof(SceneDesc));
    rc = carve_scene(pl, geo[i], scratch + offs[i], desc[i]);
    if (rc) {
      cudaFreeAsync(scratch, st);
      return rc;
    }
    desc[i].ref = io[i].ref;
    desc[i].phase = io[i].phase;
    desc[i].coh = io[i].coh;
    desc[i].cov_out = io[i].cov_out;
    desc[i].sel_out = io[i].sel;
    desc[i].tile_begin = tb;
    tb += geo[i].tiles_x * geo[i].tiles_y;
    launch_prep(pl, geo[i], desc[i], io[i].a1, io[i].a2, io[i].phi, io[i].cov_in, st);
  }
  e = cudaMemcpyAsync(d_desc, desc.data(), desc_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_wtab, pl.wtab.data(), wtab_bytes, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    cudaFreeAsync(scratch, st);
    return cuda_error(e, "cudaMemcpyAsync(params)");
  }
  pl.P.wtab = d_wtab;
  pl.P.n_scenes = (int)io.size();
  pl.P.total_tiles = tiles;
  rc = launch_fused(pl, pl.P, d_desc, smem, st);
  e = cudaGetLastError();
  cudaFreeAsync(scratch, st);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_error(e, "NL-SAR launch");
  // the host vectors above were staged by cudaMemcpyAsync (pageable source),
  // so they may go out of scope now
  return DCL_OK;
}

// Copy streams and events of the calling thread's host-pointer calls, one
// set per device, created on first use and kept for the thread's lifetime.
static thread_local HostPipe g_pipes[kMaxDevices];

int host_pipe(int dev, size_t nev, HostPipe*& out) {
  if (dev < 0 || dev >= kMaxDevices) return set_error(DCL_ERR_CUDA, "device %d out of range", dev);
  HostPipe& p = g_pipes[dev];
  cudaError_t e = cudaSuccess;
  if (!p.h2d) e = cudaStreamCreateWithFlags(&p.h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess && !p.d2h) e = cudaStreamCreateWithFlags(&p.d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess && !p.h_timeouts)
    e = cudaHostAlloc(reinterpret_cast<void**>(&p.h_timeouts), sizeof(int), cudaHostAllocDefault);
  while (e == cudaSuccess && p.ev.size() < nev) {
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) p.ev.push_back(ev);
  }
  if (e != cudaSuccess) return cuda_error(e, "host copy streams");
  out = &p;
  return DCL_OK;
}

constexpr int kMaxBands = 8;   // row bands of a host-pointer call
constexpr int kBandWaves = 8;  // fewest waves of tiles (one CTA per SM) per band: each band's launch
                               // ends in a partly filled wave, so small scenes stay in one band

int band_count(int dev, long long tiles, int tile_rows) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  int nb = (int)std::max(1LL, std::min<long long>(std::min(kMaxBands, tile_rows),
                                                  tiles / ((long long)kBandWaves * sms)));
  // DESPECKCL_B200_BANDS=n forces n bands (at most one per tile row): the
  // tests use it to cut small scenes
  if (const char* fb = std::getenv("DESPECKCL_B200_BANDS")) {
    const int n = std::atoi(fb);
    if (n > 0) nb = std::min(n, tile_rows);
  }
  return std::max(1, nb);
}

// Host pointers: the reference's filter_sub_image uploads the inputs and
// downloads the results around its kernels (nlsar/conversion.cpp:22-142).
// Here the scene is cut into bands of tile rows and the copies overlap the
// filtering: band b's input rows go up on their own stream while band b-1 is
// filtered, and every band's results come down on a third stream as soon as
// its tiles are done.  The frames are filled band by band (each prep kernel
// only on rows whose inputs have arrived), so every tile reads exactly the
// values of the single-launch path and the results are identical.
// The downloads are issued after all bands are queued, so a pageable
// destination (a synchronous copy) still lets the later bands run meanwhile.
// `hin` / `hout` are the caller's H x W planes: a1, a2, phi and ref, phase,
// coh for InSAR inputs (nin = nout = 3), the 8 covariance planes in and out
// for the covariance path (pl.full8, nin = nout = 8).
static int run_host_banded(const Plan& pl0, const float* const* hin, int nin, float* const* hout, int nout, int H,
                           int W) {
  for (int i = 0; i < nin; ++i)
    if (!hin[i]) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  for (int i = 0; i < nout; ++i)
    if (!hout[i]) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  int dev;
  int rc = ensure_device_ready(dev);
  if (rc) return rc;
  Plan pl = pl0;
  size_t smem = 0;
  const int K = choose_k(pl, smem);
  if (K < 1) return set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
  pl.P.K = K;
  const SceneGeom g = scene_geom(pl, H, W);
  if ((long long)g.tiles_x * g.tiles_y > 0x7fffffff) return set_error(DCL_ERR_INVALID_ARGUMENT, "scene too large");
  const int nb = band_count(dev, (long long)g.tiles_x * g.tiles_y, g.tiles_y);
  HostPipe* hp = nullptr;
  rc = host_pipe(dev, 2 * (size_t)nb + 2, hp);
  if (rc) return rc;
  cudaEvent_t* ev_in = hp->ev.data();       // band inputs uploaded
  cudaEvent_t* ev_out = hp->ev.data() + nb;  // band results written
  cudaEvent_t ev_alloc = hp->ev[2 * nb], ev_done = hp->ev[2 * nb + 1];

  cudaStream_t st = cudaStreamPerThread;
  const size_t n = (size_t)H * W, b = n * sizeof(float);
  const size_t scratch = (scratch_bytes(pl, g) + 255) / 256 * 256;
  const size_t desc_bytes = (nb * sizeof(SceneDesc) + 255) / 256 * 256;
  const size_t wtab_bytes = pl.wtab.size() * sizeof(float);
  const size_t io_bytes = ((size_t)(nin + nout) * b + 255) / 256 * 256;
  const size_t wtab_pad = (wtab_bytes + 255) / 256 * 256;
  char* mem = nullptr;
  // ... + one word: this call's count of thread blocks whose staging wait ran out
  cudaError_t e = cudaMallocAsync(&mem, io_bytes + scratch + desc_bytes + wtab_pad + 256, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(io + scratch)");
  float* buf = reinterpret_cast<float*>(mem);  // [nin][H][W] inputs, then [nout][H][W] outputs
  float* dout = buf + (size_t)nin * n;
  SceneDesc* d_desc = reinterpret_cast<SceneDesc*>(mem + io_bytes + scratch);
  float* d_wtab = reinterpret_cast<float*>(mem + io_bytes + scratch + desc_bytes);
  int* d_timeouts = reinterpret_cast<int*>(mem + io_bytes + scratch + desc_bytes + wtab_pad);
  *hp->h_timeouts = 0;

  // band b covers tile rows [tb[b], tb[b+1])
  std::vector<int> tb(nb + 1);
  for (int i = 0; i <= nb; ++i) tb[i] = (int)((long long)g.tiles_y * i / nb);
  std::vector<SceneDesc> desc(nb);
  std::memset(desc.data(), 0, nb * sizeof(SceneDesc));
  rc = carve_scene(pl, g, mem + io_bytes, desc[0]);
  for (int i = 0; i < nb && rc == DCL_OK; ++i) {
    if (i) desc[i] = desc[0];
    if (pl.full8) {
      desc[i].cov_out = dout;
    } else {
      desc[i].ref = dout;
      desc[i].phase = dout + n;
      desc[i].coh = dout + 2 * n;
    }
    desc[i].tile_begin = 0;
    desc[i].tile_skip = tb[i] * g.tiles_x;
  }
  if (rc == DCL_OK) {
    e = cudaMemcpyAsync(d_desc, desc.data(), nb * sizeof(SceneDesc), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_wtab, pl.wtab.data(), wtab_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_timeouts, 0, sizeof(int), st);
    if (e == cudaSuccess) e = cudaEventRecord(ev_alloc, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(hp->h2d, ev_alloc, 0);
    if (e != cudaSuccess) rc = cuda_error(e, "NL-SAR parameters");
  }
  pl.P.wtab = d_wtab;
  pl.P.n_scenes = 1;
  pl.P.timeouts = d_timeouts;

  const int TH = pl.P.tile_h, G = pl.P.G;
  int in_done = 0, co_done = 0, cs_done = 0;
  for (int i = 0; i < nb && rc == DCL_OK; ++i) {
    const bool last = i == nb - 1;
    // frame rows the band's tiles read (scaled covariance: tile + patch and
    // search halo), the original-covariance rows those average over, and the
    // input rows behind them (frame row r holds input row r - G, clamped)
    const int cs_need = last ? g.Hp : std::min(g.Hp, tb[i + 1] * TH + pl.P.phm + pl.P.wsh + G);
    const int co_need = last ? g.Hp : std::min(g.Hp, cs_need + pl.shm);
    const int in_need = last ? H : std::max(1, std::min(H, co_need - G));
    if (in_need > in_done) {
      const size_t off = (size_t)in_done * W, cnt = (size_t)(in_need - in_done) * W * sizeof(float);
      for (int p = 0; p < nin && e == cudaSuccess; ++p)
        e = cudaMemcpyAsync(buf + p * n + off, hin[p] + off, cnt, cudaMemcpyHostToDevice, hp->h2d);
      in_done = in_need;
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev_in[i], hp->h2d);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev_in[i], 0);
    if (e != cudaSuccess) {
      rc = cuda_error(e, "cudaMemcpyAsync(H2D)");
      break;
    }
    if (pl.full8)
      launch_prep_rows(pl, g, desc[i], nullptr, nullptr, nullptr, buf, co_done, co_need, cs_done, cs_need, st);
    else
      launch_prep_rows(pl, g, desc[i], buf, buf + n, buf + 2 * n, nullptr, co_done, co_need, cs_done, cs_need, st);
    co_done = co_need;
    cs_done = cs_need;
    FilterParams F = pl.P;
    F.total_tiles = (tb[i + 1] - tb[i]) * g.tiles_x;
    if (F.total_tiles > 0) rc = launch_fused(pl, F, d_desc + i, smem, st);
    e = cudaGetLastError();
    if (rc == DCL_OK && e != cudaSuccess) rc = cuda_error(e, "NL-SAR launch");
    if (rc == DCL_OK && (e = cudaEventRecord(ev_out[i], st)) != cudaSuccess) rc = cuda_error(e, "event");
  }
  // results: band b holds output rows [tb[b] * TH, tb[b+1] * TH) below row
  // H-1; row H-1 comes from the last tile row (virtual row H-1+overlap)
  for (int i = 0; i < nb && rc == DCL_OK; ++i) {
    const int r0 = std::min(tb[i] * TH, H - 1);
    const int r1 = i == nb - 1 ? H : std::min(tb[i + 1] * TH, H - 1);
    e = cudaStreamWaitEvent(hp->d2h, ev_out[i], 0);
    if (r1 > r0) {
      const size_t off = (size_t)r0 * W, cnt = (size_t)(r1 - r0) * W * sizeof(float);
      for (int p = 0; p < nout && e == cudaSuccess; ++p)
        e = cudaMemcpyAsync(hout[p] + off, dout + p * n + off, cnt, cudaMemcpyDeviceToHost, hp->d2h);
    }
    if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpyAsync(D2H)");
  }
  // the buffers are freed in stream order after every copy that uses them
  cudaError_t e2 = cudaEventRecord(ev_done, hp->d2h);
  if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(st, ev_done, 0);
  cudaError_t e3 = cudaEventRecord(ev_done, hp->h2d);
  if (e3 == cudaSuccess) e3 = cudaStreamWaitEvent(st, ev_done, 0);
  if (e2 != cudaSuccess || e3 != cudaSuccess) {
    // ordering could not be expressed: wait for the copy streams on the host
    cudaStreamSynchronize(hp->h2d);
    cudaStreamSynchronize(hp->d2h);
  }
  if (rc == DCL_OK) {
    e2 = cudaMemcpyAsync(hp->h_timeouts, d_timeouts, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e2 != cudaSuccess) rc = cuda_error(e2, "NL-SAR timeout count");
  }
  cudaFreeAsync(mem, st);
  e2 = cudaStreamSynchronize(st);
  if (rc == DCL_OK && e2 != cudaSuccess) rc = cuda_error(e2, "NL-SAR");
  if (rc == DCL_OK && *hp->h_timeouts != 0)
    rc = set_error(DCL_ERR_TIMEOUT,
                   "NL-SAR: %d thread blocks gave up waiting for their TMA staging copies; their tiles are unwritten",
                   *hp->h_timeouts);
  return rc;
}

int run_host_insar(const Plan& pl, const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                   float* coh, int H, int W) {
  const float* in[3] = {a1, a2, phi};
  float* out[3] = {ref, phase, coh};
  return run_host_banded(pl, in, 3, out, 3, H, W);
}

int run_host_covmat(const Plan& pl, const float* cin, float* cout, int H, int W) {
  if (!cin || !cout) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  const size_t n = (size_t)H * W;
  const float* in[8];
  float* out[8];
  for (int p = 0; p < 8; ++p) {
    in[p] = cin + p * n;
    out[p] = cout + p * n;
  }
  return run_host_banded(pl, in, 8, out, 8, H, W);
}

}  // namespace dcl

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using namespace dcl;

extern "C" const char* dcl_last_error(void) { return last_error(); }

extern "C" const char* dcl_version(void) { return "despeckcl_b200 0.1 (sm_100a)"; }

extern "C" int dcl_take_stage_timeouts(int* count) {
  if (!count) return set_error(DCL_ERR_INVALID_ARGUMENT, "null count");
  *count = 0;
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "no CUDA device");
  if (take_stage_timeouts(count) != 0) return set_error(DCL_ERR_CUDA, "reading the staging-timeout ledger failed");
  return DCL_OK;
}

extern "C" void dcl_profile_begin(void) {
  for (auto& p : g_prof.ev) {
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  g_prof.ev.clear();
  g_prof.launches = 0;
  g_prof.on = true;
}

extern "C" int dcl_profile_end(double* fused_ms, long* fused_launches, long* all_launches) {
  double total = 0.0;
  int rc = DCL_OK;
  for (auto& p : g_prof.ev) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(p.second);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, p.first, p.second);
    if (e != cudaSuccess && rc == DCL_OK) rc = cuda_error(e, "profile events");
    total += ms;
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  if (fused_ms) *fused_ms = total;
  if (fused_launches) *fused_launches = (long)g_prof.ev.size();
  if (all_launches) *all_launches = g_prof.launches;
  g_prof.ev.clear();
  g_prof.launches = 0;
  g_prof.on = false;
  return rc;
}

extern "C" int dcl_nlsar_insar(const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                               float* coh, int H, int W, int sws, const int* patches, int np, const int* scales,
                               int ns, const dcl_stats_entry* stats, int nstats, float h, float c, int select_mode) {
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, pl);
  if (rc) return rc;
  return run_host_insar(pl, a1, a2, phi, ref, phase, coh, H, W);
}

extern "C" int dcl_nlsar_insar_device(const float* a1, const float* a2, const float* phi, float* ref, float* phase,
                                      float* coh, int H, int W, int sws, const int* patches, int np,
                                      const int* scales, int ns, const dcl_stats_entry* stats, int nstats, float h,
                                      float c, int select_mode, int* selection_out, void* stream) {
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, pl);
  if (rc) return rc;
  SceneIO s{a1, a2, phi, nullptr, ref, phase, coh, nullptr, selection_out, H, W};
  return run_device(pl, {s}, (cudaStream_t)stream);
}

extern "C" int dcl_nlsar_covmat(const float* cin, float* cout, int H, int W, int dim, int sws, const int* patches,
                                int np, const int* scales, int ns, const dcl_stats_entry* stats, int nstats, float h,
                                float c, int select_mode) {
  if (dim != 2 && dim != 3)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "covariance dimension %d: 2x2 and 3x3 covariances are supported", dim);
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, true, pl);
  if (rc) return rc;
  if (dim == 3) return nlsar_covmat3_host(pl, cin, cout, H, W);
  return run_host_covmat(pl, cin, cout, H, W);
}

extern "C" int dcl_nlsar_covmat_device(const float* cin, float* cout, int H, int W, int dim, int sws,
                                       const int* patches, int np, const int* scales, int ns,
                                       const dcl_stats_entry* stats, int nstats, float h, float c, int select_mode,
                                       void* stream) {
  if (dim != 2 && dim != 3)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "covariance dimension %d: 2x2 and 3x3 covariances are supported", dim);
  if (!cin || !cout) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, true, pl);
  if (rc) return rc;
  if (dim == 3) return nlsar_covmat3_device(pl, cin, cout, H, W, (cudaStream_t)stream);
  SceneIO s{nullptr, nullptr, nullptr, cin, nullptr, nullptr, nullptr, cout, nullptr, H, W};
  return run_device(pl, {s}, (cudaStream_t)stream);
}

extern "C" int dcl_nlsar_insar_batch_device(int n, const float* const* a1, const float* const* a2,
                                            const float* const* phi, float* const* ref, float* const* phase,
                                            float* const* coh, const int* heights, const int* widths, int sws,
                                            const int* patches, int np, const int* scales, int ns,
                                            const dcl_stats_entry* stats, int nstats, float h, float c,
                                            int select_mode, void* stream) {
  if (n < 1 || !a1 || !a2 || !phi || !ref || !phase || !coh || !heights || !widths)
    return set_error(DCL_ERR_INVALID_ARGUMENT, "empty batch or null pointer");
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, pl);
  if (rc) return rc;
  std::vector<SceneIO> io;
  for (int i = 0; i < n; ++i) {
    if (!a1[i] || !a2[i] || !phi[i] || !ref[i] || !phase[i] || !coh[i])
      return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer in scene %d", i);
    io.push_back(SceneIO{a1[i], a2[i], phi[i], nullptr, ref[i], phase[i], coh[i], nullptr, nullptr, heights[i],
                         widths[i]});
  }
  return run_device(pl, io, (cudaStream_t)stream);
}

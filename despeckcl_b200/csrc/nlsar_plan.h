// Host-side plan of an NL-SAR call and the helpers that stage and launch it
// (defined in nlsar_host.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/despeckcl_b200.h"
#include "nlsar_common.cuh"

namespace dcl {

// Validated parameters of one call, ready for the kernels.
struct Plan {
  FilterParams P;
  std::vector<float> wtab;
  std::vector<int> scales;       // distinct scale sizes, caller order (scale slots)
  std::vector<char> slot_used;   // slots referenced by the passes
  int overlap = 0;
  int shm = 0;                   // largest scale half among used slots
  bool full8 = false;
  bool fast = false;  // served by the specialised kernel (nlsar_fast.cu)
  int px = 4;
};

// Geometry of one scene on the virtual plane.
struct SceneGeom {
  int H, W, vH, vW, tiles_x, tiles_y, Hp, Wp, pitch;
};

int make_plan(int sws, const int* patches, int np, const int* scales, int ns, const dcl_stats_entry* stats,
              int nstats, float h, float c, int select_mode, bool full8, Plan& pl);
int choose_k(const Plan& pl, size_t& smem_bytes);
SceneGeom scene_geom(const Plan& pl, int H, int W);
size_t scratch_bytes(const Plan& pl, const SceneGeom& g);
int carve_scene(const Plan& pl, const SceneGeom& g, char* base, SceneDesc& d);
int launch_prep(const Plan& pl, const SceneGeom& g, const SceneDesc& d, const float* a1, const float* a2,
                const float* phi, const float* cov_in, cudaStream_t st);
// the same for frame rows [co0, co1) of the original covariance and [cs0, cs1)
// of every scaled covariance (the rows those read must be filled already)
int launch_prep_rows(const Plan& pl, const SceneGeom& g, const SceneDesc& d, const float* a1, const float* a2,
                     const float* phi, const float* cov_in, int co0, int co1, int cs0, int cs1, cudaStream_t st);
// variant selects the specialised kernel's instantiation (see launch_nlsar_fast)
int launch_fused(const Plan& pl, const FilterParams& F, const SceneDesc* d_scenes, size_t smem, cudaStream_t st,
                 int variant = 0);
// whether the call is served by the specialised kernel (variants apply)
bool uses_specialised_kernel(const Plan& pl);
// Copy streams and events of host-pointer calls (per thread and device):
// `ev` holds at least the number of events asked for.
struct HostPipe {
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> ev;
  int* h_timeouts = nullptr;  // pinned: the last call's staging-timeout count
};
int host_pipe(int dev, size_t nev, HostPipe*& out);
// Row bands of a host-pointer call over `tiles` tiles in `tile_rows` rows
// (DESPECKCL_B200_BANDS overrides).
int band_count(int dev, long long tiles, int tile_rows);
// NL-SAR of a 3x3 covariance scene [18][H][W] (nlsar_dim3.cu): device
// pointers on `st`, or host pointers (copied in and out, synchronous)
int nlsar_covmat3_device(const Plan& pl, const float* cin, float* cout, int H, int W, cudaStream_t st);
int nlsar_covmat3_host(const Plan& pl, const float* cin, float* cout, int H, int W);

}  // namespace dcl

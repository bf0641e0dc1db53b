// NL-SAR on device pointers without any device allocation.
//
// Some callers cannot allocate GPU memory while they filter: code that runs
// inside a memory budget fixed at start-up, callers whose allocator is owned
// by a host framework that forbids allocations on its hot path, or programs
// that must not trigger a device-wide synchronisation or allocator growth
// mid-stream.  dcl_nlsar_insar_device_noalloc serves them: the caller still
// passes its own input and output buffers, and the scratch the filter needs
// (the clamp-padded covariance frame, the scene descriptor and the weight
// tables) lives in one statically sized device array of this file instead of
// coming from cudaMalloc / cudaMallocAsync.
//
// Limits and rules:
//  * the array holds kNoAllocScratchBytes (64 MiB) on every GPU that loads
//    the library, for the life of the process;
//  * a scene whose padded frame does not fit is rejected with
//    DCL_ERR_INVALID_ARGUMENT (with the search window 21, patches {3,5,7} and
//    scales {1,3}, scenes up to about 1000 x 1000 pixels fit);
//  * every call rewrites all of the scratch it reads, so nothing has to start
//    at zero, but all calls on one device share the array: calls that overlap
//    on the GPU (different streams or threads at the same time) race;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress); make that first call before any stream capture;
//  * the scene descriptor and weight tables are copied from pageable host
//    memory, so a call may wait for the stream's earlier work before it
//    returns.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_plan.h"

namespace dcl {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (the host-side
// name of the array is only a stand-in, never a device pointer).
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_error(DCL_ERR_UNSUPPORTED, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(scratch)");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return DCL_OK;
}

}  // namespace
}  // namespace dcl

using namespace dcl;

extern "C" int dcl_nlsar_insar_device_noalloc(const float* a1, const float* a2, const float* phi, float* ref,
                                              float* phase, float* coh, int H, int W, int sws, const int* patches,
                                              int np, const int* scales, int ns, const dcl_stats_entry* stats,
                                              int nstats, float h, float c, int select_mode, int* selection_out,
                                              void* stream) {
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  Plan pl;
  int rc = make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, pl);
  if (rc) return rc;
  size_t smem = 0;
  const int K = choose_k(pl, smem);
  if (K < 1) return set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
  pl.P.K = K;

  const SceneGeom g = scene_geom(pl, H, W);
  const size_t frame = (scratch_bytes(pl, g) + 255) / 256 * 256;
  const size_t desc = (sizeof(SceneDesc) + 255) / 256 * 256;
  const size_t wtab = pl.wtab.size() * sizeof(float);
  if (frame + desc + wtab > kNoAllocScratchBytes)
    return set_error(DCL_ERR_INVALID_ARGUMENT,
                     "scene %dx%d needs %zu bytes of scratch; the allocation-free entry point holds %zu "
                     "(use dcl_nlsar_insar_device for larger scenes)",
                     H, W, frame + desc + wtab, kNoAllocScratchBytes);
  void* base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc) return rc;
  char* scratch = static_cast<char*>(base);
  cudaStream_t st = (cudaStream_t)stream;

  SceneDesc d;
  std::memset(&d, 0, sizeof d);
  rc = carve_scene(pl, g, scratch, d);
  if (rc) return rc;
  d.ref = ref;
  d.phase = phase;
  d.coh = coh;
  d.sel_out = selection_out;
  d.tile_begin = 0;
  SceneDesc* d_desc = reinterpret_cast<SceneDesc*>(scratch + frame);
  float* d_wtab = reinterpret_cast<float*>(scratch + frame + desc);
  cudaError_t e = cudaMemcpyAsync(d_desc, &d, sizeof d, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_wtab, pl.wtab.data(), wtab, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync(params)");
  rc = launch_prep(pl, g, d, a1, a2, phi, nullptr, st);
  if (rc) return rc;
  pl.P.wtab = d_wtab;
  pl.P.n_scenes = 1;
  pl.P.total_tiles = g.tiles_x * g.tiles_y;
  rc = launch_fused(pl, pl.P, d_desc, smem, st);
  if (rc) return rc;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "NL-SAR launch");
  return DCL_OK;
}

// Prepared NL-SAR batches: many scenes of uneven size filtered by one fused
// launch, with the scratch, the scene descriptors and the weight tables set up
// once, the launch sequence optionally captured in a CUDA graph, and the
// specialised kernel's instantiation picked by timing it on the batch.
//
// The reference filters one scene per call and one tile per OpenMP task
// (src/compute/common/map_filter_tiles.h:64-101); a batch here is the list of
// every tile of every scene, walked by one persistent grid.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_plan.h"

struct dcl_nlsar_batch {
  dcl::Plan pl;
  std::vector<dcl::SceneGeom> geo;
  std::vector<dcl::SceneDesc> desc;
  std::vector<const float*> a1, a2, phi;
  std::vector<float*> ref, phase, coh;
  std::vector<int> H, W;
  char* scratch = nullptr;
  dcl::SceneDesc* d_desc = nullptr;
  size_t smem = 0;
  int variant = 0;
  bool tuned = false;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace dcl {
namespace {

// Geometry, frames and descriptors of every scene for tiles of `tile_h` rows,
// carved from the batch's scratch (sized for the tallest tiles; a frame of
// shorter tiles is never larger), descriptors uploaded synchronously.
int prepare(dcl_nlsar_batch* b, int tile_h, size_t* scratch_total) {
  b->pl.P.tile_h = tile_h;
  const int n = (int)b->H.size();
  b->geo.clear();
  std::vector<size_t> offs;
  size_t total = 0;
  long long tiles = 0;
  for (int i = 0; i < n; ++i) {
    b->geo.push_back(scene_geom(b->pl, b->H[i], b->W[i]));
    offs.push_back(total);
    total += (scratch_bytes(b->pl, b->geo.back()) + 255) / 256 * 256;
    tiles += (long long)b->geo.back().tiles_x * b->geo.back().tiles_y;
  }
  if (tiles > 0x7fffffff) return set_error(DCL_ERR_INVALID_ARGUMENT, "batch too large");
  if (scratch_total) {  // sizing only
    *scratch_total = total;
    return DCL_OK;
  }
  b->desc.assign(n, SceneDesc{});
  int tb = 0;
  for (int i = 0; i < n; ++i) {
    SceneDesc& d = b->desc[i];
    std::memset(&d, 0, sizeof d);
    const int rc = carve_scene(b->pl, b->geo[i], b->scratch + offs[i], d);
    if (rc != DCL_OK) return rc;
    d.ref = b->ref[i];
    d.phase = b->phase[i];
    d.coh = b->coh[i];
    d.tile_begin = tb;
    tb += b->geo[i].tiles_x * b->geo[i].tiles_y;
  }
  const cudaError_t e = cudaMemcpy(b->d_desc, b->desc.data(), n * sizeof(SceneDesc), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemcpy(batch descriptors)");
  b->pl.P.total_tiles = (int)tiles;
  return DCL_OK;
}

// tile rows of a kernel instantiation (launch_nlsar_fast variants)
int variant_tile_h(int v) { return v == 2 ? kFastTileHHalf : kFastTileH; }

int enqueue(dcl_nlsar_batch* b, cudaStream_t st) {
  for (size_t i = 0; i < b->desc.size(); ++i) {
    const int rc = launch_prep(b->pl, b->geo[i], b->desc[i], b->a1[i], b->a2[i], b->phi[i], nullptr, st);
    if (rc) return rc;
  }
  return launch_fused(b->pl, b->pl.P, b->d_desc, b->smem, st, b->variant);
}

// Autotuner cache: (device, search window, patch halves, passes, selection,
// log2 of the tile count) -> fastest variant, kept for the process and, with
// DESPECKCL_B200_TUNE_CACHE=<file>, in a small text file.
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

std::string tune_key(const dcl_nlsar_batch* b) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  const FilterParams& F = b->pl.P;
  std::string k = prop.name;
  for (char& ch : k)
    if (ch == ' ') ch = '_';
  char buf[160];
  std::snprintf(buf, sizeof buf, "/sws%d/np%d/ph%d-%d-%d/pass%d/sel%d/t%d", F.sws, F.pass[0].np, F.pass[0].ph[0],
                F.pass[0].np > 1 ? F.pass[0].ph[1] : -1, F.pass[0].np > 2 ? F.pass[0].ph[2] : -1, F.npass,
                F.select_mode, (int)std::log2((double)F.total_tiles + 1));
  return k + buf;
}

void tune_load_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char* path = std::getenv("DESPECKCL_B200_TUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char key[512];
  int v;
  while (std::fscanf(f, "%511s %d", key, &v) == 2) g_tune[key] = v;
  std::fclose(f);
}

void tune_store_locked() {
  const char* path = std::getenv("DESPECKCL_B200_TUNE_CACHE");
  if (!path) return;
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  for (auto& kv : g_tune) std::fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
  std::fclose(f);
}

int autotune(dcl_nlsar_batch* b, cudaStream_t st) {
  if (!uses_specialised_kernel(b->pl)) return DCL_OK;
  const std::string key = tune_key(b);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_load_locked();
    auto it = g_tune.find(key);
    if (it != g_tune.end() && it->second < fast_variants(b->pl.P, false)) {
      b->variant = it->second;
      return b->pl.P.tile_h == variant_tile_h(b->variant) ? DCL_OK : prepare(b, variant_tile_h(b->variant), nullptr);
    }
  }
  float best = 0.f;
  int best_v = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int nv = fast_variants(b->pl.P, false);
  for (int v = 0; v < nv; ++v) {
    b->variant = v;
    int rc = DCL_OK;
    if (b->pl.P.tile_h != variant_tile_h(v)) {
      rc = cudaStreamSynchronize(st) == cudaSuccess ? prepare(b, variant_tile_h(v), nullptr) : DCL_ERR_CUDA;
      if (rc) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
      }
    }
    rc = enqueue(b, st);  // warm-up (also sets the kernel's shared-memory attribute)
    if (rc == DCL_OK) {
      cudaEventRecord(e0, st);
      rc = enqueue(b, st);
      cudaEventRecord(e1, st);
    }
    if (rc) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
    const cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return cuda_error(e, "autotune");
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (v == 0 || ms < best) {
      best = ms;
      best_v = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->variant = best_v;
  if (b->pl.P.tile_h != variant_tile_h(best_v)) {
    if (cudaStreamSynchronize(st) != cudaSuccess) return set_error(DCL_ERR_CUDA, "autotune");
    const int rc = prepare(b, variant_tile_h(best_v), nullptr);
    if (rc) return rc;
  }
  b->tuned = true;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best_v;
  tune_store_locked();
  return DCL_OK;
}

void release(dcl_nlsar_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->scratch) cudaFree(b->scratch);
  delete b;
}

}  // namespace
}  // namespace dcl

using namespace dcl;

extern "C" dcl_nlsar_batch* dcl_nlsar_batch_create(int n, const float* const* a1, const float* const* a2,
                                                   const float* const* phi, float* const* ref, float* const* phase,
                                                   float* const* coh, const int* heights, const int* widths, int sws,
                                                   const int* patches, int np, const int* scales, int ns,
                                                   const dcl_stats_entry* stats, int nstats, float h, float c,
                                                   int select_mode, int flags, void* stream) {
  if (n < 1 || !a1 || !a2 || !phi || !ref || !phase || !coh || !heights || !widths) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "empty batch or null pointer");
    return nullptr;
  }
  dcl_nlsar_batch* b = new dcl_nlsar_batch();
  if (make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, b->pl)) {
    delete b;
    return nullptr;
  }
  const int K = choose_k(b->pl, b->smem);
  if (K < 1) {
    set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
    delete b;
    return nullptr;
  }
  b->pl.P.K = K;
  for (int i = 0; i < n; ++i) {
    if (heights[i] < 1 || widths[i] < 1 || !a1[i] || !a2[i] || !phi[i] || !ref[i] || !phase[i] || !coh[i]) {
      set_error(DCL_ERR_INVALID_ARGUMENT, "scene %d: empty or null", i);
      delete b;
      return nullptr;
    }
    b->H.push_back(heights[i]);
    b->W.push_back(widths[i]);
    b->a1.push_back(a1[i]);
    b->a2.push_back(a2[i]);
    b->phi.push_back(phi[i]);
    b->ref.push_back(ref[i]);
    b->phase.push_back(phase[i]);
    b->coh.push_back(coh[i]);
  }
  // scratch for the tallest tiles the autotuner may try
  size_t total = 0;
  if (prepare(b, kFastTileH, &total) != DCL_OK) {
    delete b;
    return nullptr;
  }
  const size_t desc_bytes = (n * sizeof(SceneDesc) + 255) / 256 * 256;
  const size_t wtab_bytes = b->pl.wtab.size() * sizeof(float);
  cudaError_t e = cudaMalloc(&b->scratch, total + desc_bytes + wtab_bytes);
  if (e != cudaSuccess) {
    cuda_error(e, "cudaMalloc(batch scratch)");
    release(b);
    return nullptr;
  }
  b->d_desc = reinterpret_cast<SceneDesc*>(b->scratch + total);
  float* d_wtab = reinterpret_cast<float*>(b->scratch + total + desc_bytes);
  if (prepare(b, b->pl.P.tile_h, nullptr) != DCL_OK) {
    release(b);
    return nullptr;
  }
  e = cudaMemcpy(d_wtab, b->pl.wtab.data(), wtab_bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cuda_error(e, "cudaMemcpy(batch weight tables)");
    release(b);
    return nullptr;
  }
  b->pl.P.wtab = d_wtab;
  b->pl.P.n_scenes = n;
  cudaStream_t st = (cudaStream_t)stream;
  if (flags & DCL_BATCH_VARIANT1) b->variant = 1;
  if ((flags & DCL_BATCH_VARIANT2) && fast_variants(b->pl.P, false) > 2) {
    b->variant = 2;
    if (prepare(b, variant_tile_h(2), nullptr) != DCL_OK) {
      release(b);
      return nullptr;
    }
  }
  if ((flags & DCL_BATCH_AUTOTUNE) && autotune(b, st) != DCL_OK) {
    release(b);
    return nullptr;
  }
  if (flags & DCL_BATCH_GRAPH) {
    // one eager run sets every kernel attribute before the capture
    int rc = enqueue(b, st);
    if (rc == DCL_OK) {
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) rc = cuda_error(e, "batch warm-up");
    }
    if (rc == DCL_OK) {
      e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        rc = enqueue(b, b->cap);
        const cudaError_t e2 = cudaStreamEndCapture(b->cap, &b->graph);
        if (rc == DCL_OK && e2 != cudaSuccess) rc = cuda_error(e2, "cudaStreamEndCapture");
      } else {
        rc = cuda_error(e, "batch graph capture");
      }
      if (rc == DCL_OK) {
        e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphInstantiate");
      }
    }
    if (rc != DCL_OK) {
      release(b);
      return nullptr;
    }
  }
  return b;
}

extern "C" int dcl_nlsar_batch_run(dcl_nlsar_batch* b, void* stream) {
  if (!b) return set_error(DCL_ERR_INVALID_ARGUMENT, "null batch");
  cudaStream_t st = (cudaStream_t)stream;
  if (b->exec) {
    const cudaError_t e = cudaGraphLaunch(b->exec, st);
    return e == cudaSuccess ? DCL_OK : cuda_error(e, "cudaGraphLaunch");
  }
  return enqueue(b, st);
}

extern "C" int dcl_nlsar_batch_variant(const dcl_nlsar_batch* b) { return b ? b->variant : -1; }

extern "C" int dcl_nlsar_batch_launches(const dcl_nlsar_batch* b) {
  if (!b) return 0;
  int used = 0;
  for (char u : b->pl.slot_used) used += u ? 1 : 0;
  return (int)b->desc.size() * (1 + used) + 1;
}

extern "C" void dcl_nlsar_batch_destroy(dcl_nlsar_batch* b) { release(b); }

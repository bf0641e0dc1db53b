// NL-SAR request server: continuous batching of interferograms on one GPU.
//
// Requests (one scene each, on device or host buffers) queue in arrival
// order.  A worker thread
//  * admits them, oldest first, while their device memory fits a fixed HBM
//    budget (one arena allocated at start-up and carved first-fit);
//  * cuts the admitted work into launches of at most max_batch_tiles tiles: a
//    large scene is split over several launches (each launch covers a range
//    of its tiles), and scenes that arrive while it runs join the next launch
//    instead of waiting for the whole scene;
//  * keeps up to max_inflight launches queued on separate streams, so that
//    the tail of one launch overlaps the head of the next and host copies of
//    one batch overlap the kernels of another;
//  * retires launches as their events complete and frees the memory of every
//    request whose last tile has been filtered.
// The plan, the weight tables and the kernel configuration stay resident for
// the server's life.  Each tile is computed exactly as in a one-scene call
// (the scene's frame, descriptor and tile coordinates do not depend on the
// batch), so a request's result does not depend on what it was batched with.
//
// The reference filters one scene per blocking call
// (src/compute/nlsar/nlsar.cpp:139-167); serving has no counterpart there.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/despeckcl_b200.h"
#include "dcl_internal.h"
#include "nlsar_plan.h"

namespace dcl {
namespace {

constexpr size_t kAlign = 256;
constexpr int kMaxScenesPerLaunch = 1024;

size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over one device allocation (offsets only).
class Arena {
 public:
  void init(size_t cap) {
    cap_ = cap;
    used_ = 0;
    free_.clear();
    if (cap) free_[0] = cap;
  }
  bool alloc(size_t n, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const size_t o = it->first, rest = it->second - n;
      free_.erase(it);
      if (rest) free_[o + n] = rest;
      used_ += n;
      *off = o;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    used_ -= n;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + n == next->first) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += n;
        return;
      }
    }
    free_[off] = n;
  }
  size_t used() const { return used_; }
  size_t capacity() const { return cap_; }

 private:
  std::map<size_t, size_t> free_;
  size_t cap_ = 0, used_ = 0;
};

struct Batch;

struct Request {
  long long id = 0;
  const float *a1 = nullptr, *a2 = nullptr, *phi = nullptr;
  float *ref = nullptr, *phase = nullptr, *coh = nullptr;
  int H = 0, W = 0;
  bool host = false;
  cudaEvent_t ready = nullptr;  // caller's event guarding device inputs
  SceneGeom g{};
  size_t scratch = 0, plane = 0, bytes = 0, off = 0;
  int tiles = 0, next_tile = 0;
  SceneDesc desc{};         // frame pointers; tile fields are set per launch
  Batch* prep_batch = nullptr;  // in-flight launch that staged the frame
  std::vector<Batch*> open;     // in-flight launches that hold some of its tiles
  float *s_a1 = nullptr, *s_a2 = nullptr, *s_phi = nullptr;  // host requests: device staging
  float *s_ref = nullptr, *s_phase = nullptr, *s_coh = nullptr;
  bool finished = false;
  bool released = false;  // arena memory returned (finished and no launch holds it)
  dcl_request_info info{};
  std::string message;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t prep_done = nullptr, done = nullptr;
  SceneDesc* h_desc = nullptr;  // pinned
  SceneDesc* d_desc = nullptr;
  int* d_timeouts = nullptr;    // the launch's count of thread blocks whose staging wait ran out
  int* h_timeouts = nullptr;    // pinned copy, read when the launch has completed
  bool busy = false;
};

struct Batch {
  long long id = 0;
  int slot = 0;
  std::vector<std::shared_ptr<Request>> reqs;
};

}  // namespace
}  // namespace dcl

using namespace dcl;

struct dcl_server {
  Plan pl;
  size_t smem = 0;
  int variant = 0;
  int device = 0;
  int max_inflight = 2;
  int max_batch_tiles = 0;
  char* arena_base = nullptr;
  Arena arena;
  float* d_wtab = nullptr;
  std::vector<Slot> slots;
  std::chrono::steady_clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queued;    // submitted, not admitted
  std::deque<Request*> admitted;  // admitted, tiles left to launch
  std::vector<std::unique_ptr<Batch>> inflight;
  std::unordered_map<long long, std::shared_ptr<Request>> reqs;
  long long next_id = 0, next_batch = 0;
  bool stop = false;
  dcl_server_stats st{};
  std::thread worker;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void loop();
  bool retire_locked();
  bool admit_locked();
  bool launch_locked();
  int enqueue(Batch& b, const std::vector<std::pair<Request*, int>>& parts);
  void finish_locked(Request* r, int status, const std::string& msg, double t);
  void release_locked(Request* r);
};

// A request's memory goes back to the arena once it has finished and no
// in-flight launch still reads or writes it.
void dcl_server::release_locked(Request* r) {
  if (!r->finished || !r->open.empty() || r->released) return;
  r->released = true;
  if (r->bytes) arena.release(r->off, r->bytes);
  st.admitted_bytes = arena.used();
}

void dcl_server::finish_locked(Request* r, int status, const std::string& msg, double t) {
  if (r->finished) return;
  r->finished = true;
  r->info.status = status;
  r->info.done_s = t;
  r->message = msg;
  // a failed request leaves the launch queue for good
  auto it = std::find(admitted.begin(), admitted.end(), r);
  if (it != admitted.end()) admitted.erase(it);
  r->next_tile = r->tiles;
  release_locked(r);
  if (status == DCL_OK)
    st.completed++;
  else
    st.failed++;
  cv_done.notify_all();
}

bool dcl_server::retire_locked() {
  bool any = false;
  for (size_t i = 0; i < inflight.size();) {
    Batch* b = inflight[i].get();
    Slot& s = slots[b->slot];
    const cudaError_t q = cudaEventQuery(s.done);
    if (q == cudaErrorNotReady) {
      ++i;
      continue;
    }
    const double t = now();
    std::string msg;
    if (q != cudaSuccess) msg = std::string("NL-SAR launch failed: ") + cudaGetErrorString(q);
    const int timeouts = q == cudaSuccess ? *s.h_timeouts : 0;
    if (timeouts)
      msg = "NL-SAR: " + std::to_string(timeouts) +
            " thread blocks gave up waiting for their TMA staging copies; their tiles are unwritten";
    for (auto& rp : b->reqs) {
      Request* r = rp.get();
      r->open.erase(std::remove(r->open.begin(), r->open.end(), b), r->open.end());
      if (r->prep_batch == b) r->prep_batch = nullptr;
      if (q != cudaSuccess)
        finish_locked(r, DCL_ERR_CUDA, msg, t);
      else if (timeouts)
        finish_locked(r, DCL_ERR_TIMEOUT, msg, t);
      else if (r->open.empty() && r->next_tile == r->tiles)
        finish_locked(r, DCL_OK, "", t);
      release_locked(r);
    }
    s.busy = false;
    inflight.erase(inflight.begin() + i);
    any = true;
  }
  return any;
}

bool dcl_server::admit_locked() {
  bool any = false;
  while (!queued.empty()) {
    Request* r = queued.front();
    size_t off = 0;
    if (!arena.alloc(r->bytes, &off)) break;
    r->off = off;
    char* base = arena_base + off;
    const int crc = carve_scene(pl, r->g, base, r->desc);
    if (crc != DCL_OK) {
      // the request holds its arena block until finish_locked releases it
      queued.pop_front();
      finish_locked(r, crc, dcl_last_error(), now());
      any = true;
      continue;
    }
    r->desc.ref = r->ref;
    r->desc.phase = r->phase;
    r->desc.coh = r->coh;
    if (r->host) {
      float* p = reinterpret_cast<float*>(base + align_up(r->scratch));
      const size_t n = r->plane / sizeof(float);
      r->s_a1 = p;
      r->s_a2 = p + n;
      r->s_phi = p + 2 * n;
      r->s_ref = p + 3 * n;
      r->s_phase = p + 4 * n;
      r->s_coh = p + 5 * n;
      r->desc.ref = r->s_ref;
      r->desc.phase = r->s_phase;
      r->desc.coh = r->s_coh;
    }
    r->info.admit_s = now();
    st.admitted_bytes = arena.used();
    st.peak_admitted_bytes = std::max<unsigned long long>(st.peak_admitted_bytes, arena.used());
    queued.pop_front();
    admitted.push_back(r);
    any = true;
  }
  return any;
}

// Stage and launch one batch on its slot's stream.  parts: (request, tiles of
// it in this launch, starting at request->next_tile before the call).
int dcl_server::enqueue(Batch& b, const std::vector<std::pair<Request*, int>>& parts) {
  Slot& s = slots[b.slot];
  cudaStream_t str = s.stream;
  cudaError_t e = cudaSuccess;
  int launches = 0;
  // inputs: caller events, host copies, frame staging of requests new here
  for (auto& pr : parts) {
    Request* r = pr.first;
    if (r->next_tile != 0) continue;
    if (r->ready) e = cudaStreamWaitEvent(str, r->ready, 0);
    if (e == cudaSuccess && r->host) {
      const size_t n = (size_t)r->H * r->W * sizeof(float);
      e = cudaMemcpyAsync(r->s_a1, r->a1, n, cudaMemcpyHostToDevice, str);
      if (e == cudaSuccess) e = cudaMemcpyAsync(r->s_a2, r->a2, n, cudaMemcpyHostToDevice, str);
      if (e == cudaSuccess) e = cudaMemcpyAsync(r->s_phi, r->phi, n, cudaMemcpyHostToDevice, str);
    }
    if (e != cudaSuccess) return cuda_error(e, "server input staging");
    const int rc = launch_prep(pl, r->g, r->desc, r->host ? r->s_a1 : r->a1, r->host ? r->s_a2 : r->a2,
                               r->host ? r->s_phi : r->phi, nullptr, str);
    if (rc) return rc;
    for (char u : pl.slot_used) launches += u ? 1 : 0;
    launches += 1;
    r->prep_batch = &b;
  }
  // frames staged by launches still in flight on other streams
  for (auto& pr : parts) {
    Request* r = pr.first;
    if (r->prep_batch && r->prep_batch != &b) {
      e = cudaStreamWaitEvent(str, slots[r->prep_batch->slot].prep_done, 0);
      if (e != cudaSuccess) return cuda_error(e, "server frame dependency");
    }
  }
  e = cudaEventRecord(s.prep_done, str);
  if (e != cudaSuccess) return cuda_error(e, "server event");
  // descriptors of this launch
  int tb = 0;
  for (size_t i = 0; i < parts.size(); ++i) {
    Request* r = parts[i].first;
    SceneDesc d = r->desc;
    d.tile_begin = tb;
    d.tile_skip = r->next_tile;
    s.h_desc[i] = d;
    tb += parts[i].second;
  }
  e = cudaMemcpyAsync(s.d_desc, s.h_desc, parts.size() * sizeof(SceneDesc), cudaMemcpyHostToDevice, str);
  if (e != cudaSuccess) return cuda_error(e, "server descriptors");
  FilterParams F = pl.P;
  F.wtab = d_wtab;
  F.n_scenes = (int)parts.size();
  F.total_tiles = tb;
  F.timeouts = s.d_timeouts;
  e = cudaMemsetAsync(s.d_timeouts, 0, sizeof(int), str);
  if (e != cudaSuccess) return cuda_error(e, "server timeout word");
  int rc = launch_fused(pl, F, s.d_desc, smem, str, variant);
  if (rc) return rc;
  launches += 1;
  e = cudaMemcpyAsync(s.h_timeouts, s.d_timeouts, sizeof(int), cudaMemcpyDeviceToHost, str);
  if (e != cudaSuccess) return cuda_error(e, "server timeout word");
  // results of host requests whose last tiles run here
  for (auto& pr : parts) {
    Request* r = pr.first;
    if (!r->host || r->next_tile + pr.second != r->tiles) continue;
    for (Batch* o : r->open)
      if (o != &b) {
        e = cudaStreamWaitEvent(str, slots[o->slot].done, 0);
        if (e != cudaSuccess) return cuda_error(e, "server result dependency");
      }
    const size_t n = (size_t)r->H * r->W * sizeof(float);
    e = cudaMemcpyAsync(r->ref, r->s_ref, n, cudaMemcpyDeviceToHost, str);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->phase, r->s_phase, n, cudaMemcpyDeviceToHost, str);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->coh, r->s_coh, n, cudaMemcpyDeviceToHost, str);
    if (e != cudaSuccess) return cuda_error(e, "server result copies");
  }
  e = cudaEventRecord(s.done, str);
  if (e != cudaSuccess) return cuda_error(e, "server event");
  st.kernel_launches += launches;
  st.tiles += tb;
  return DCL_OK;
}

bool dcl_server::launch_locked() {
  if (admitted.empty() || (int)inflight.size() >= max_inflight) return false;
  int slot = -1;
  for (int i = 0; i < (int)slots.size(); ++i)
    if (!slots[i].busy) {
      slot = i;
      break;
    }
  if (slot < 0) return false;
  std::unique_ptr<Batch> b(new Batch());
  b->id = next_batch++;
  b->slot = slot;
  std::vector<std::pair<Request*, int>> parts;
  int budget = max_batch_tiles;
  for (Request* r : admitted) {
    if (budget <= 0 || (int)parts.size() == kMaxScenesPerLaunch) break;
    const int take = std::min(budget, r->tiles - r->next_tile);
    parts.push_back({r, take});
    budget -= take;
  }
  const double t = now();
  const int rc = enqueue(*b, parts);
  if (rc != DCL_OK) {
    // nothing of a failed enqueue is trusted: fail its requests
    const std::string msg = dcl_last_error();
    cudaStreamSynchronize(slots[slot].stream);
    for (auto& pr : parts) finish_locked(pr.first, rc, msg, t);
    return true;
  }
  slots[slot].busy = true;
  for (auto& pr : parts) {
    Request* r = pr.first;
    if (r->next_tile == 0) {
      r->info.launch_s = t;
      r->info.first_batch = b->id;
    }
    r->info.last_batch = b->id;
    r->info.chunks += 1;
    r->next_tile += pr.second;
    r->open.push_back(b.get());
    b->reqs.push_back(reqs.at(r->id));
  }
  while (!admitted.empty() && admitted.front()->next_tile == admitted.front()->tiles) admitted.pop_front();
  st.batches++;
  inflight.push_back(std::move(b));
  st.peak_inflight = std::max<int>(st.peak_inflight, (int)inflight.size());
  return true;
}

void dcl_server::loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    bool progress = retire_locked();
    progress |= admit_locked();
    progress |= launch_locked();
    if (stop && queued.empty() && admitted.empty() && inflight.empty()) break;
    if (progress) continue;
    if (inflight.empty() && admitted.empty() && !stop) {
      // idle until a submission (queued requests that do not fit yet wait
      // for memory that only in-flight launches can free)
      // (nothing in flight or admitted means the arena is empty, and every
      // request fits an empty arena, so a queued request is admitted at once)
      cv_work.wait(lk, [&] { return stop || !queued.empty(); });
      continue;
    }
    lk.unlock();
    std::this_thread::sleep_for(std::chrono::microseconds(10));
    lk.lock();
  }
}

namespace {

void destroy_server(dcl_server* s) {
  if (!s) return;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
    }
    s->cv_work.notify_all();
    s->worker.join();
  }
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.prep_done) cudaEventDestroy(sl.prep_done);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.h_desc) cudaFreeHost(sl.h_desc);
    if (sl.h_timeouts) cudaFreeHost(sl.h_timeouts);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  if (s->arena_base) cudaFree(s->arena_base);
  delete s;
}

}  // namespace

extern "C" dcl_server* dcl_server_create(int sws, const int* patches, int np, const int* scales, int ns,
                                         const dcl_stats_entry* stats, int nstats, float h, float c,
                                         int select_mode, unsigned long long hbm_budget_bytes, int max_inflight,
                                         int max_batch_tiles, int flags) {
  if (max_inflight < 1 || max_inflight > 16 || max_batch_tiles < 1) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "max_inflight must be in [1, 16] and max_batch_tiles >= 1");
    return nullptr;
  }
  std::unique_ptr<dcl_server> s(new dcl_server());
  if (make_plan(sws, patches, np, scales, ns, stats, nstats, h, c, select_mode, false, s->pl)) return nullptr;
  const int K = choose_k(s->pl, s->smem);
  if (K < 1) {
    set_error(DCL_ERR_UNSUPPORTED, "search window / patch sizes too large for shared memory");
    return nullptr;
  }
  s->pl.P.K = K;
  s->variant = (flags & DCL_BATCH_VARIANT1) ? 1 : 0;
  s->max_inflight = max_inflight;
  s->max_batch_tiles = max_batch_tiles;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e != cudaSuccess) {
    cuda_error(e, "cudaGetDevice");
    return nullptr;
  }
  const size_t wtab_bytes = align_up(s->pl.wtab.size() * sizeof(float));
  const size_t budget = hbm_budget_bytes / kAlign * kAlign;
  if (budget < kAlign) {
    set_error(DCL_ERR_INVALID_ARGUMENT, "HBM budget too small");
    return nullptr;
  }
  e = cudaMalloc(&s->arena_base, budget + wtab_bytes +
                                      max_inflight * (align_up(kMaxScenesPerLaunch * sizeof(SceneDesc)) + kAlign));
  if (e != cudaSuccess) {
    cuda_error(e, "cudaMalloc(server arena)");
    return nullptr;
  }
  s->arena.init(budget);
  s->d_wtab = reinterpret_cast<float*>(s->arena_base + budget);
  e = cudaMemcpy(s->d_wtab, s->pl.wtab.data(), s->pl.wtab.size() * sizeof(float), cudaMemcpyHostToDevice);
  s->slots.resize(max_inflight);
  char* dp = s->arena_base + budget + wtab_bytes;
  for (int i = 0; i < max_inflight && e == cudaSuccess; ++i) {
    Slot& sl = s->slots[i];
    sl.d_desc = reinterpret_cast<SceneDesc*>(dp);
    dp += align_up(kMaxScenesPerLaunch * sizeof(SceneDesc));
    sl.d_timeouts = reinterpret_cast<int*>(dp);
    dp += kAlign;
    e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.prep_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc(&sl.h_desc, kMaxScenesPerLaunch * sizeof(SceneDesc), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&sl.h_timeouts), sizeof(int), cudaHostAllocDefault);
    if (e == cudaSuccess) *sl.h_timeouts = 0;
  }
  if (e != cudaSuccess) {
    cuda_error(e, "server set-up");
    destroy_server(s.release());
    return nullptr;
  }
  s->st.budget_bytes = budget;
  s->t0 = std::chrono::steady_clock::now();
  dcl_server* raw = s.release();
  raw->worker = std::thread([raw] { raw->loop(); });
  return raw;
}

extern "C" long long dcl_server_submit(dcl_server* s, const float* a1, const float* a2, const float* phi,
                                       float* ref, float* phase, float* coh, int H, int W, int host_buffers,
                                       void* ready_event) {
  if (!s) return set_error(DCL_ERR_INVALID_ARGUMENT, "null server");
  if (!a1 || !a2 || !phi || !ref || !phase || !coh) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  if (H < 1 || W < 1) return set_error(DCL_ERR_INVALID_ARGUMENT, "height and width must be >= 1");
  std::shared_ptr<Request> r(new Request());
  r->a1 = a1;
  r->a2 = a2;
  r->phi = phi;
  r->ref = ref;
  r->phase = phase;
  r->coh = coh;
  r->H = H;
  r->W = W;
  r->host = host_buffers != 0;
  r->ready = (cudaEvent_t)ready_event;
  r->g = scene_geom(s->pl, H, W);
  const long long tiles = (long long)r->g.tiles_x * r->g.tiles_y;
  if (tiles > 0x7fffffff) return set_error(DCL_ERR_INVALID_ARGUMENT, "scene too large");
  r->tiles = (int)tiles;
  r->scratch = scratch_bytes(s->pl, r->g);
  r->plane = align_up((size_t)H * W * sizeof(float));
  r->bytes = align_up(r->scratch) + (r->host ? 6 * r->plane : 0);
  if (r->bytes > s->arena.capacity())
    return set_error(DCL_ERR_OUT_OF_MEMORY, "request %dx%d needs %zu bytes; the server's HBM budget is %zu", H, W,
                     r->bytes, s->arena.capacity());
  long long id;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return set_error(DCL_ERR_INVALID_ARGUMENT, "server is shutting down");
    id = s->next_id++;
    r->id = id;
    r->info.submit_s = s->now();
    r->info.first_batch = r->info.last_batch = -1;
    s->queued.push_back(r.get());
    s->reqs[id] = std::move(r);
    s->st.submitted++;
  }
  s->cv_work.notify_one();
  return id;
}

namespace {

int take_result(dcl_server* s, long long id, dcl_request_info* info) {
  auto it = s->reqs.find(id);
  Request* r = it->second.get();
  if (info) *info = r->info;
  const int status = r->info.status;
  if (status != DCL_OK) set_error(status, "request %lld: %s", id, r->message.c_str());
  s->reqs.erase(it);
  return status;
}

}  // namespace

extern "C" int dcl_server_wait(dcl_server* s, long long id, double timeout_s, dcl_request_info* info) {
  if (!s) return set_error(DCL_ERR_INVALID_ARGUMENT, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(DCL_ERR_INVALID_ARGUMENT, "unknown request %lld", id);
  Request* r = it->second.get();
  auto pred = [r] { return r->finished; };
  if (timeout_s < 0)
    s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
    return set_error(DCL_ERR_TIMEOUT, "request %lld not finished after %.3f s", id, timeout_s);
  take_result(s, id, info);
  return DCL_OK;
}

extern "C" int dcl_server_poll(dcl_server* s, long long id, dcl_request_info* info) {
  if (!s) return set_error(DCL_ERR_INVALID_ARGUMENT, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return set_error(DCL_ERR_INVALID_ARGUMENT, "unknown request %lld", id);
  if (!it->second->finished) return 0;
  take_result(s, id, info);
  return 1;
}

extern "C" double dcl_server_now(const dcl_server* s) { return s ? s->now() : 0.0; }

extern "C" int dcl_server_get_stats(dcl_server* s, dcl_server_stats* out) {
  if (!s || !out) return set_error(DCL_ERR_INVALID_ARGUMENT, "null pointer");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->queued = (int)s->queued.size();
  out->admitted = (int)s->admitted.size();
  out->inflight = (int)s->inflight.size();
  return DCL_OK;
}

extern "C" void dcl_server_destroy(dcl_server* s) { destroy_server(s); }

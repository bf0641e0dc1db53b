// TEST INFRASTRUCTURE ONLY.  The reference's NL-SAR device kernels
// (src/compute/nlsar/cl_kernels/*.cl) are OpenCL C that is also valid C++
// once the address-space qualifiers and the work-item functions are supplied.
// oracle/Makefile compiles them here, in place from the reference tree (the
// pixel-similarity template configured like CMake's configure_file, and the
// two kernels that declare __local arrays in their bodies rewritten so those
// arrays are shared by a work group), and this file runs them:
//
//   * an NDRange emulator: every work group runs its work items in turn.  In
//     the kernels that call barrier() every work item reaches a barrier
//     before any work item passes it:
//       - covmat_spatial_avg and weighted_means (barriers inside loops): each
//         work item is a fiber (ucontext) and barrier() switches to the next
//         work item of the group.  Work items resume in ascending order of
//         local id (dimension 0 slowest): covmat_spatial_avg.cl:36-60 reads,
//         after its barrier, only __local elements at or after the reader's
//         own position and then overwrites its own element for the next plane
//         without a second barrier, which this order keeps race free;
//       - the row and column passes of the patch sums and
//         compute_nl_statistics (one barrier, and before it only __local
//         stores of values read from global memory): every work item runs up
//         to the barrier, then every work item runs again from the start
//         through the barrier to the end.  Repeating the part before the
//         barrier stores the same values again and writes no global memory,
//         so this is the same as one run, at a fraction of the fibers' cost;
//   * the host steps of one tile, restated from
//     src/compute/nlsar/nlsar_filter_sub_image.cpp:146-390 and
//     src/compute/nlsar/routines/routines.cpp:20-250, with the NDRange sizes of
//     the wrappers in src/compute/nlsar/cl_wrappers/*.cpp (the two quadrant
//     launches of compute_pixel_similarities_2x2.cpp:61-79, the row / column
//     passes of compute_patch_similarities.cpp:62-118, work-group sizes of
//     cl_wrappers.h:60-78) and the conversions of conversion.cpp:22-142;
//   * the reference's own host code where it compiles without OpenCL:
//     get_best_params (best_params.cpp), best_alpha_copy (best_alpha_copy.cpp),
//     tile_iterator (tile_iterator.cpp), get_sub_image / write_sub_image
//     (sub_images.cpp), driven as map_filter_tiles.h:69-96 does (tiles in
//     iteration order, so a later tile's write wins).
//
// Arithmetic: the kernels run with IEEE single precision and glibc's float
// math functions (-ffp-contract=off: no multiply-add contraction), one valid
// OpenCL implementation among those the reference targets.  OpenCL's float
// min/max on a NaN operand return the other operand here (fmin / fmax).  The
// ENL-argmax selection (the documented NL-SAR rule; the reference's
// get_best_params keeps the last key) is the one restated step: largest
// bias-reduced ENL over the computed (patch, scale) keys in map order, first on
// ties, as in oracle/nlsar_oracle.cpp.  The search-window size and the work
// group sizes are compile-time constants of the two kernels with in-body
// __local arrays (SEARCH_WINDOW_SIZE, set by the Makefile).
#include <setjmp.h>
#include <ucontext.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <vector>

#include "best_alpha_copy.h"
#include "best_params.h"
#include "sub_images.h"
#include "tile.h"
#include "tile_iterator.h"

namespace refnl {

// ---------------------------------------------------------------------------
// NDRange emulation
// ---------------------------------------------------------------------------

int g_lid[3], g_grp[3], g_lsz[3] = {1, 1, 1}, g_off[3];

inline size_t get_global_id(int d) { return (size_t)g_grp[d] * g_lsz[d] + g_lid[d] + g_off[d]; }
inline size_t get_local_id(int d) { return (size_t)g_lid[d]; }
inline size_t get_group_id(int d) { return (size_t)g_grp[d]; }
inline size_t get_local_size(int d) { return (size_t)g_lsz[d]; }

struct Fiber {
  ucontext_t ctx;
  int lid[3];
  int barriers;
  bool done;
};

ucontext_t g_main;
std::vector<Fiber> g_fibers;
std::vector<std::unique_ptr<char[]>> g_stacks;
constexpr size_t kStack = 1 << 16;
int g_cur = -1;
const std::function<void()>* g_body = nullptr;

void fiber_main() {
  (*g_body)();
  g_fibers[g_cur].done = true;
}

// barrier handling of the running launch
enum Sync { kNone = 0, kReplay = 1, kFibers = 2 };
int g_sync = kNone;
int g_replay_phase = 0;  // kReplay: 0 = up to the barrier, 1 = the whole kernel
jmp_buf g_replay_jmp;

#define CLK_LOCAL_MEM_FENCE 1
void barrier(int) {
  if (g_sync == kReplay) {
    if (g_replay_phase == 0) _longjmp(g_replay_jmp, 1);
    return;
  }
  if (g_sync != kFibers || g_cur < 0) throw std::logic_error("barrier() in a launch without barrier support");
  Fiber& f = g_fibers[g_cur];
  ++f.barriers;
  swapcontext(&f.ctx, &g_main);
}

// One launch: global sizes g[], local sizes l[], global offsets o[]; the
// global sizes are multiples of the local sizes, as the wrappers make them.
// sync: kNone (no barrier in the kernel), kReplay or kFibers (see the header).
void ndrange(int dims, const size_t* g, const size_t* l, const size_t* o, int sync,
             const std::function<void()>& body) {
  const bool barriers = sync == kFibers;
  g_sync = sync;
  int ng[3] = {1, 1, 1}, ls[3] = {1, 1, 1};
  for (int d = 0; d < dims; ++d) {
    if (l[d] == 0 || g[d] % l[d] != 0) throw std::logic_error("global size not a multiple of the local size");
    ls[d] = (int)l[d];
    ng[d] = (int)(g[d] / l[d]);
  }
  for (int d = 0; d < 3; ++d) {
    g_lsz[d] = ls[d];
    g_off[d] = (d < dims && o) ? (int)o[d] : 0;
  }
  const int items = ls[0] * ls[1] * ls[2];
  if (barriers) {
    g_fibers.resize(items);
    while ((int)g_stacks.size() < items) g_stacks.emplace_back(new char[kStack]);
  }
  g_body = &body;
  for (int z = 0; z < ng[2]; ++z)
    for (int y = 0; y < ng[1]; ++y)
      for (int x = 0; x < ng[0]; ++x) {
        g_grp[0] = x;
        g_grp[1] = y;
        g_grp[2] = z;
        if (!barriers) {
          for (int phase = (sync == kReplay ? 0 : 1); phase < 2; ++phase) {
            g_replay_phase = phase;
            for (int a = 0; a < ls[0]; ++a)
              for (int b = 0; b < ls[1]; ++b)
                for (int c = 0; c < ls[2]; ++c) {
                  g_lid[0] = a;
                  g_lid[1] = b;
                  g_lid[2] = c;
                  if (phase == 0) {
                    if (_setjmp(g_replay_jmp) == 0) {
                      body();
                      throw std::logic_error("a work item finished without reaching the barrier");
                    }
                  } else {
                    body();
                  }
                }
          }
          continue;
        }
        // fibers in ascending local-id order, dimension 0 slowest
        int i = 0;
        for (int a = 0; a < ls[0]; ++a)
          for (int b = 0; b < ls[1]; ++b)
            for (int c = 0; c < ls[2]; ++c, ++i) {
              Fiber& f = g_fibers[i];
              f.lid[0] = a;
              f.lid[1] = b;
              f.lid[2] = c;
              f.barriers = 0;
              f.done = false;
              getcontext(&f.ctx);
              f.ctx.uc_stack.ss_sp = g_stacks[i].get();
              f.ctx.uc_stack.ss_size = kStack;
              f.ctx.uc_link = &g_main;
              makecontext(&f.ctx, fiber_main, 0);
            }
        for (bool pending = true; pending;) {
          pending = false;
          for (int k = 0; k < items; ++k) {
            Fiber& f = g_fibers[k];
            if (f.done) continue;
            g_cur = k;
            g_lid[0] = f.lid[0];
            g_lid[1] = f.lid[1];
            g_lid[2] = f.lid[2];
            swapcontext(&g_main, &f.ctx);
            pending = pending || !f.done;
          }
          g_cur = -1;
        }
        for (int k = 1; k < items; ++k)
          if (g_fibers[k].barriers != g_fibers[0].barriers)
            throw std::logic_error("work items of a group reached different numbers of barriers");
      }
}

void nd1(size_t g0, size_t l0, int bar, const std::function<void()>& f) {
  const size_t g[1] = {g0}, l[1] = {l0};
  ndrange(1, g, l, nullptr, bar, f);
}
void nd2(size_t g0, size_t g1, size_t l0, size_t l1, size_t o0, size_t o1, int bar,
         const std::function<void()>& f) {
  const size_t g[2] = {g0, g1}, l[2] = {l0, l1}, o[2] = {o0, o1};
  ndrange(2, g, l, o, bar, f);
}
void nd3(size_t g0, size_t g1, size_t g2, size_t l0, size_t l1, size_t l2, int bar,
         const std::function<void()>& f) {
  const size_t g[3] = {g0, g1, g2}, l[3] = {l0, l1, l2};
  ndrange(3, g, l, nullptr, bar, f);
}

// ---------------------------------------------------------------------------
// The reference's kernels
// ---------------------------------------------------------------------------

using std::atan2;
using std::cos;
using std::exp;
using std::fabs;
using std::isnan;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
inline float max(float a, float b) { return std::fmax(a, b); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }

#define __kernel static
#define __global
#define __constant const
#define __local
#define __private

#include "covmat_create.cl"
#include "covmat_rescale.cl"
#include "covmat_spatial_avg.cl"
#include "compute_pixel_similarities_2x2.cl"  // configured copy (_ref/)

#define BLOCK_SIZE_X 16
#define BLOCK_SIZE_Y 4
#define STEPS_ROW 4
#define STEPS_COL 4
#include "patch_similarities_row_pass.cl"
#include "patch_similarities_col_pass.cl"

#include "compute_weights.cl"
#include "copy_symm_weights.cl"

#define BLOCK_SIZE 16
#define DIMENSION 2
#include "nlsar_compute_nl_statistics.cl"  // in-body __local arrays made static (_ref/)
#include "compute_alphas.cl"
#include "compute_enls_nobias.cl"
#include "copy_best_weights.cl"
#include "nlsar_weighted_means.cl"  // in-body __local array made static (_ref/)
#include "covmat_decompose.cl"

#undef __kernel
#undef __global
#undef __constant
#undef __local
#undef __private

// ---------------------------------------------------------------------------
// Host steps of one tile
// ---------------------------------------------------------------------------

constexpr int kBlock = 16;      // kernel_params::block_size (nlsar.cpp:114)
constexpr int kBlock1d = 64;    // compute_weights / copy_best_weights (cl_wrappers.h:66,73)
constexpr size_t kGuard = 1 << 16;  // zeroed floats after every buffer (see filter_tile)

inline size_t rup(int n, int b) { return (size_t)b * ((n - 1) / b + 1); }

struct Lut {
  int lut_size;
  float dmin, dmax;
  std::vector<float> quant, chi2;
};

using Buf = std::vector<float>;
inline Buf buf(size_t n) { return Buf(n + kGuard, 0.0f); }

// covmat_spatial_avg.cpp:35-50
std::vector<float> gen_gauss(const int scale_size) {
  std::vector<float> gauss;
  const int ssh = (scale_size - 1) / 2;
  for (int x = -ssh; x <= ssh; x++)
    for (int y = -ssh; y <= ssh; y++)
      gauss.push_back(std::exp(-M_PI * (x * x + y * y) / std::pow(ssh + 0.5f, 2.0f)));
  float K = 0.0f;
  for (float g : gauss) K += g;
  for (float& g : gauss) g = g / K;
  return gauss;
}

// One tile's covariance (8 planes of height x width) through the pipeline of
// nlsar_filter_sub_image.cpp:146-390; returns the filtered covariance (its
// interior, `overlap` pixels in from every side, is the tile's result).  The
// guard of zeros after every buffer keeps the first-quadrant similarity
// launch's reads past the row ends of its last rows inside memory, as device
// memory does; what they read lands only in similarity slots no weight uses.
Buf filter_tile(const Buf& covmat_ori, int height, int width, int sws, const std::vector<int>& patch_sizes,
                const std::vector<int>& scale_sizes, std::map<nlsar::params, Lut>& dissim_stats, float h_param,
                float c_param, int select_mode, std::vector<int>* sel_out) {
  const int dimensions = 2, nlooks = 1;
  const int patch_size_max = *std::max_element(patch_sizes.begin(), patch_sizes.end());
  const int scale_size_max = *std::max_element(scale_sizes.begin(), scale_sizes.end());
  const int psh = (patch_size_max - 1) / 2;
  const int wsh = (sws - 1) / 2;
  const int overlap = wsh + psh;
  const int hoa = height, woa = width;
  const int n_oa = hoa * woa;
  const int ho = hoa - scale_size_max + 1, wo = woa - scale_size_max + 1;
  const int hori = ho - 2 * overlap, wori = wo - 2 * overlap;
  const int n_ori = hori * wori;
  const size_t n_w = (size_t)sws * sws * n_ori;  // buffer_sizes::weights()
  const int n_combo = (int)(patch_sizes.size() * scale_sizes.size());

  Buf covmat_filt = buf((size_t)2 * dimensions * dimensions * n_oa);
  Buf rescaled(covmat_ori);
  {
    float* cv = rescaled.data();
    nd2(rup(hoa, kBlock), rup(woa, kBlock), kBlock, kBlock, 0, 0, kNone,
        [&] { covmat_rescale(cv, dimensions, nlooks, hoa, woa); });
  }
  std::map<nlsar::params, int> params2idx;
  std::map<nlsar::params, std::vector<float>> enls_nobias, alphas;
  for (auto& ps : dissim_stats) {
    enls_nobias[ps.first] = std::vector<float>(n_ori);
    alphas[ps.first] = std::vector<float>(n_ori);
  }
  Buf all_weights = buf((size_t)n_combo * n_w);
  std::vector<nlsar::params> computed;
  int idx = 0;
  for (int scale_size : scale_sizes) {
    // routines.cpp:20-68
    const int hs = ho - wsh, ws = wo;  // height_symm / width_symm of the similarity kernel
    Buf pix = buf((size_t)(wsh + 1) * sws * hs * ws);
    Buf avg = buf((size_t)2 * dimensions * dimensions * ho * wo);
    {
      const int obs = kBlock - scale_size + 1;
      std::vector<float> gauss = gen_gauss(scale_size);
      std::vector<float> local((size_t)kBlock * kBlock);
      float *in = rescaled.data(), *out = avg.data(), *lm = local.data();
      const float* gs = gauss.data();
      nd2((size_t)kBlock * ((ho - 1) / obs + 1), (size_t)kBlock * ((wo - 1) / obs + 1), kBlock, kBlock, 0, 0, kFibers,
          [&] { covmat_spatial_avg(in, out, dimensions, ho, wo, scale_size, scale_size_max, lm, gs); });
    }
    {
      float *cv = avg.data(), *ps = pix.data();
      const size_t g0 = rup(ho - wsh, kBlock), g1 = rup(wo - wsh, kBlock);
      nd2(g0, g1, kBlock, kBlock, 0, 0, kNone, [&] {
        compute_pixel_similarities_2x2(cv, ps, ho, wo, dimensions, nlooks, sws, 0, wsh, wsh, sws);
      });
      nd2(g0, g1, kBlock, kBlock, 0, wsh, kNone, [&] {
        compute_pixel_similarities_2x2(cv, ps, ho, wo, dimensions, nlooks, sws, 0, wsh + 1, 0, wsh);
      });
    }
    for (int patch_size : patch_sizes) {
      const nlsar::params parameter{patch_size, scale_size};
      params2idx[parameter] = idx;
      idx++;
      computed.push_back(parameter);
      Lut& st = dissim_stats.at(parameter);
      // routines.cpp:70-160
      Buf weights = buf(n_w);
      const int hps = ho - wsh, wps = wo;
      const int hpat = hps - patch_size_max + 1, wpat = wps - patch_size_max + 1;
      const int n_half = sws * wsh + wsh;
      Buf patsim = buf((size_t)n_half * hpat * wpat);
      Buf wsymm = buf((size_t)n_half * hpat * wpat);
      {
        // compute_patch_similarities.cpp:62-118
        const int offset = (patch_size_max - patch_size) / 2;
        const int hi = hps - 2 * offset, wi = wps - 2 * offset - patch_size + 1;
        const int hp = hi - patch_size + 1, wp = wi;
        Buf inter = buf((size_t)sws * sws * hi * wi);
        std::vector<float> lrow((size_t)BLOCK_SIZE_X * (STEPS_ROW + 2) * BLOCK_SIZE_Y);
        std::vector<float> lcol((size_t)BLOCK_SIZE_Y * (STEPS_COL + 4) * BLOCK_SIZE_X);
        float *ps = pix.data(), *it = inter.data(), *pt = patsim.data(), *lr = lrow.data(), *lc = lcol.data();
        nd3((size_t)BLOCK_SIZE_X * ((wi - 1) / (BLOCK_SIZE_X * STEPS_ROW) + 1),
            (size_t)BLOCK_SIZE_Y * ((hi - 1) / BLOCK_SIZE_Y + 1), (size_t)n_half, BLOCK_SIZE_X, BLOCK_SIZE_Y, 1, kReplay,
            [&] { patch_similarities_row_pass(ps, it, hps, wps, patch_size, patch_size_max, lr); });
        nd3((size_t)BLOCK_SIZE_X * ((wp - 1) / BLOCK_SIZE_X + 1),
            (size_t)BLOCK_SIZE_Y * ((hp - 1) / (BLOCK_SIZE_Y * STEPS_COL) + 1), (size_t)n_half, BLOCK_SIZE_X,
            BLOCK_SIZE_Y, 1, kReplay,
            [&] { patch_similarities_col_pass(it, pt, hps, wps, patch_size, patch_size_max, lc); });
      }
      {
        float *pt = patsim.data(), *wsy = wsymm.data();
        const float *q = st.quant.data(), *c2 = st.chi2.data();
        nd1((size_t)kBlock1d * (((size_t)n_half * hpat * wpat - 1) / kBlock1d + 1), kBlock1d, kNone, [&] {
          compute_weights(pt, wsy, hpat, wpat, sws, patch_size, h_param, c_param, q, c2, st.lut_size, st.dmin, st.dmax);
        });
      }
      {
        float *wsy = wsymm.data(), *wf = weights.data();
        // NullRange work groups: any size; no barrier in this kernel
        nd2((size_t)wori, (size_t)hori, 1, 1, 0, 0, kNone, [&] { copy_symm_weights(wsy, wf, hori, wori, sws); });
      }
      // self weight (routines.cpp:151-157)
      std::fill(weights.begin() + (size_t)n_ori * n_half, weights.begin() + (size_t)n_ori * (n_half + 1), 1.0f);
      std::copy(weights.begin(), weights.begin() + n_w, all_weights.begin() + (size_t)(idx - 1) * n_w);
      // routines.cpp:162-240
      Buf enl = buf(n_ori), int_nl = buf((size_t)dimensions * n_ori), wvar = buf((size_t)dimensions * n_ori);
      Buf wsums = buf(n_ori), alph = buf(n_ori), enb = buf(n_ori);
      {
        const float* co = covmat_ori.data();
        float *wf = weights.data(), *in = int_nl.data(), *wv = wvar.data(), *wsm = wsums.data(), *en = enl.data();
        float *al = alph.data(), *eb = enb.data();
        const size_t g0 = rup(hori, kBlock), g1 = rup(wori, kBlock);
        nd2(g0, g1, kBlock, kBlock, 0, 0, kReplay, [&] {
          compute_nl_statistics(const_cast<float*>(co), wf, in, wv, wsm, en, hori, wori, sws, patch_size_max,
                                scale_size_max);
        });
        nd2(g0, g1, kBlock, kBlock, 0, 0, kNone,
            [&] { compute_alphas(in, wv, al, hori, wori, dimensions, nlooks); });
        nd2(g0, g1, kBlock, kBlock, 0, 0, kNone, [&] { compute_enls_nobias(en, al, wsm, eb, hori, wori); });
      }
      std::copy(enb.begin(), enb.begin() + n_ori, enls_nobias[parameter].begin());
      std::copy(alph.begin(), alph.begin() + n_ori, alphas[parameter].begin());
    }
  }

  std::vector<nlsar::params> best_parameters;
  if (select_mode == 0) {
    best_parameters = nlsar::get_best_params(enls_nobias);  // the reference's own selection
  } else {
    std::vector<nlsar::params> order;  // computed keys in map order
    for (auto& kv : enls_nobias)
      if (std::find(computed.begin(), computed.end(), kv.first) != computed.end()) order.push_back(kv.first);
    best_parameters.resize(n_ori, computed.front());
    for (int o = 0; o < n_ori; ++o) {
      float best = -1.0f;
      for (const auto& k : order) {
        const float e = enls_nobias[k][o];
        if (e > best) {
          best = e;
          best_parameters[o] = k;
        }
      }
    }
  }
  std::vector<int> best_idxs(best_parameters.size());
  std::transform(best_parameters.begin(), best_parameters.end(), best_idxs.begin(),
                 [&params2idx](nlsar::params p) { return params2idx[p]; });
  if (sel_out) *sel_out = best_idxs;
  std::vector<float> best_alphas = nlsar::best_alpha_copy(alphas, best_parameters, hori, wori);
  Buf best_weights = buf(n_w);
  {
    float *aw = all_weights.data(), *bw = best_weights.data();
    int* bi = best_idxs.data();
    nd1(rup(n_ori, kBlock1d), kBlock1d, kNone, [&] { copy_best_weights(aw, bi, bw, hori, wori, sws); });
  }
  {
    float *co = const_cast<float*>(covmat_ori.data()), *cf = covmat_filt.data(), *bw = best_weights.data();
    float* ba = best_alphas.data();
    nd2(rup(hori, kBlock), rup(wori, kBlock), kBlock, kBlock, 0, 0, kFibers,
        [&] { weighted_means(co, cf, bw, ba, hori, wori, sws, patch_size_max, scale_size_max); });
  }
  return covmat_filt;
}

int get_overlap(int sws, const std::vector<int>& patch_sizes, const std::vector<int>& scale_sizes) {
  // nlsar.cpp:41-51
  const int pmax = *std::max_element(patch_sizes.begin(), patch_sizes.end());
  const int smax = *std::max_element(scale_sizes.begin(), scale_sizes.end());
  return (pmax - 1) / 2 + (sws - 1) / 2 + (smax - 1) / 2;
}

// map_filter_tiles.h:69-96 over an image of `nin` input planes; `to_cov`
// turns a tile's input planes into the 8-plane covariance (conversion.cpp),
// `from_cov` writes the filtered tile's output planes (nout of them).
int filter_image(const float* in, int nin, float* out, int nout, int H, int W, int sws, const std::vector<int>& patches,
                 const std::vector<int>& scales, std::map<nlsar::params, Lut>& stats, float h, float c,
                 int select_mode, int tile_h, int tile_w, int* sel,
                 const std::function<Buf(const float*, int, int)>& to_cov,
                 const std::function<void(const Buf&, int, int, float*)>& from_cov) {
  const int overlap = get_overlap(sws, patches, scales);
  if (tile_h <= 2 * overlap || tile_w <= 2 * overlap) return -1;
  for (auto t : tile_iterator(H, W, tile_h, tile_w, overlap, overlap)) {
    const int th = t[0].stop - t[0].start, tw = t[1].stop - t[1].start;
    std::unique_ptr<float[]> sub = get_sub_image(in, H, W, nin, t[0].start, t[1].start, th, tw);
    const Buf cov = to_cov(sub.get(), th, tw);
    std::vector<int> tsel;
    const Buf filt = filter_tile(cov, th, tw, sws, patches, scales, stats, h, c, select_mode, sel ? &tsel : nullptr);
    std::vector<float> res((size_t)nout * th * tw);
    from_cov(filt, th, tw, res.data());
    // crop the overlap and write back with clamped coordinates
    const tile<2> rel_sub{t[0].get_sub(overlap, -overlap), t[1].get_sub(overlap, -overlap)};
    const int sh = th - 2 * overlap, sw = tw - 2 * overlap;
    std::vector<float> crop((size_t)nout * sh * sw);
    for (int p = 0; p < nout; ++p)
      for (int y = 0; y < sh; ++y)
        for (int x = 0; x < sw; ++x)
          crop[((size_t)p * sh + y) * sw + x] = res[((size_t)p * th + y + overlap) * tw + x + overlap];
    write_sub_image(out, H, W, nout, crop.data(), rel_sub[0].start, rel_sub[1].start, sh, sw, 0);
    if (sel)  // the filtered core (hori x wori) is the crop: 2 * overlap = smax - 1 + 2 * (wsh + psh)
      for (int y = 0; y < sh; ++y)
        for (int x = 0; x < sw; ++x) {
          const int yy = std::min(H - 1, std::max(0, rel_sub[0].start + y));
          const int xx = std::min(W - 1, std::max(0, rel_sub[1].start + x));
          sel[(size_t)yy * W + xx] = tsel[(size_t)y * sw + x];
        }
  }
  return 0;
}

std::map<nlsar::params, Lut> make_stats(const int* keys, int nkeys, const int* lut_sizes, const float* dmin,
                                        const float* dmax, const float* quant, const float* chi2) {
  std::map<nlsar::params, Lut> m;
  size_t off = 0;
  for (int i = 0; i < nkeys; ++i) {
    Lut l;
    l.lut_size = lut_sizes[i];
    l.dmin = dmin[i];
    l.dmax = dmax[i];
    l.quant.assign(quant + off, quant + off + lut_sizes[i]);
    l.chi2.assign(chi2 + off, chi2 + off + lut_sizes[i]);
    off += lut_sizes[i];
    m[nlsar::params{keys[2 * i], keys[2 * i + 1]}] = l;
  }
  return m;
}

}  // namespace refnl

// ---------------------------------------------------------------------------
// C ABI for the tests and the fixture script
// ---------------------------------------------------------------------------

// InSAR input (despeckcl::nlsar, nlsar.cpp:139-167): a1, a2, phi -> ref,
// phase, coh.  Statistics: keys[2i] = patch, keys[2i+1] = scale; LUT i holds
// lut_sizes[i] entries of quantilles and chi2cdf_inv, concatenated.  sel
// (optional, H x W): the selected combination index per pixel (params2idx).
extern "C" int ref_nlsar_insar(const float* a1, const float* a2, const float* ph, float* ref, float* phase,
                               float* coh, int H, int W, int sws, const int* patches, int np, const int* scales,
                               int ns, const int* keys, int nkeys, const int* lut_sizes, const float* dmin,
                               const float* dmax, const float* quant, const float* chi2, float h, float c,
                               int select_mode, int tile_h, int tile_w, int* sel) {
  using namespace refnl;
  try {
#ifdef SEARCH_WINDOW_SIZE
    if (sws != SEARCH_WINDOW_SIZE) return -3;
#endif
    std::vector<int> P(patches, patches + np), S(scales, scales + ns);
    auto stats = make_stats(keys, nkeys, lut_sizes, dmin, dmax, quant, chi2);
    for (int p : P)
      for (int s : S)
        if (!stats.count(nlsar::params{p, s})) return -2;
    const size_t n = (size_t)H * W;
    std::vector<float> in(3 * n), out(3 * n, 0.0f);
    std::copy(a1, a1 + n, in.begin());
    std::copy(a2, a2 + n, in.begin() + n);
    std::copy(ph, ph + n, in.begin() + 2 * n);
    auto to_cov = [](const float* sub, int th, int tw) {
      // conversion.cpp:22-62 with covmat_create.cl
      const size_t m = (size_t)th * tw;
      Buf am(sub, sub + m), as(sub + m, sub + 2 * m), phs(sub + 2 * m, sub + 3 * m);
      am.resize(m + kGuard);
      as.resize(m + kGuard);
      phs.resize(m + kGuard);
      Buf cov = buf(8 * m);
      float *pa = am.data(), *pb = as.data(), *pp = phs.data(), *pc = cov.data();
      nd2(rup(th, kBlock), rup(tw, kBlock), kBlock, kBlock, 0, 0, kNone,
          [&] { covmat_create(pa, pb, pp, pc, th, tw); });
      return cov;
    };
    auto from_cov = [](const Buf& filt, int th, int tw, float* res) {
      // conversion.cpp:88-142 with covmat_decompose.cl
      const size_t m = (size_t)th * tw;
      Buf cf(filt);
      Buf r = buf(m), p = buf(m), ch = buf(m);
      float *pc = cf.data(), *pr = r.data(), *pp = p.data(), *pk = ch.data();
      nd2(rup(th, kBlock), rup(tw, kBlock), kBlock, kBlock, 0, 0, kNone,
          [&] { covmat_decompose(pc, pr, pp, pk, th, tw); });
      std::copy(r.begin(), r.begin() + m, res);
      std::copy(p.begin(), p.begin() + m, res + m);
      std::copy(ch.begin(), ch.begin() + m, res + 2 * m);
    };
    const int rc = filter_image(in.data(), 3, out.data(), 3, H, W, sws, P, S, stats, h, c, select_mode, tile_h,
                                tile_w, sel, to_cov, from_cov);
    if (rc) return rc;
    std::copy(out.begin(), out.begin() + n, ref);
    std::copy(out.begin() + n, out.begin() + 2 * n, phase);
    std::copy(out.begin() + 2 * n, out.begin() + 3 * n, coh);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_nlsar_insar: %s\n", e.what());
    return -1;
  }
}

// Covariance input (nlsar.cpp:171-194, dim 2): cin / cout [8][H][W].
extern "C" int ref_nlsar_covmat(const float* cin, float* cout, int H, int W, int sws, const int* patches, int np,
                                const int* scales, int ns, const int* keys, int nkeys, const int* lut_sizes,
                                const float* dmin, const float* dmax, const float* quant, const float* chi2, float h,
                                float c, int select_mode, int tile_h, int tile_w) {
  using namespace refnl;
  try {
#ifdef SEARCH_WINDOW_SIZE
    if (sws != SEARCH_WINDOW_SIZE) return -3;
#endif
    std::vector<int> P(patches, patches + np), S(scales, scales + ns);
    auto stats = make_stats(keys, nkeys, lut_sizes, dmin, dmax, quant, chi2);
    for (int p : P)
      for (int s : S)
        if (!stats.count(nlsar::params{p, s})) return -2;
    auto to_cov = [](const float* sub, int th, int tw) {
      Buf cov = buf((size_t)8 * th * tw);
      std::copy(sub, sub + (size_t)8 * th * tw, cov.begin());
      return cov;
    };
    auto from_cov = [](const Buf& filt, int th, int tw, float* res) {
      std::copy(filt.begin(), filt.begin() + (size_t)8 * th * tw, res);
    };
    return filter_image(cin, 8, cout, 8, H, W, sws, P, S, stats, h, c, select_mode, tile_h, tile_w, nullptr, to_cov,
                        from_cov);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_nlsar_covmat: %s\n", e.what());
    return -1;
  }
}

// compute_patch_similarities_test.cpp:31-81 setup: the row and column passes
// over `n_half` planes of height_sim x width_sim pixel similarities `pix`,
// patch sums into `out` (n_half planes of (height_sim - pmax + 1) x
// (width_sim - pmax + 1)).
extern "C" int ref_patch_similarities(const float* pix, float* out, int height_sim, int width_sim, int sws,
                                      int patch_size, int patch_size_max) {
  using namespace refnl;
  try {
    const int wsh = (sws - 1) / 2, n_half = sws * wsh + wsh;
    const int offset = (patch_size_max - patch_size) / 2;
    const int hi = height_sim - 2 * offset, wi = width_sim - 2 * offset - patch_size + 1;
    const int hp = hi - patch_size + 1, wp = wi;
    const int hpat = height_sim - patch_size_max + 1, wpat = width_sim - patch_size_max + 1;
    Buf ps(pix, pix + (size_t)n_half * height_sim * width_sim);
    ps.resize(ps.size() + kGuard);
    Buf inter = buf((size_t)sws * sws * hi * wi), pt = buf((size_t)n_half * hpat * wpat);
    std::vector<float> lrow((size_t)BLOCK_SIZE_X * (STEPS_ROW + 2) * BLOCK_SIZE_Y);
    std::vector<float> lcol((size_t)BLOCK_SIZE_Y * (STEPS_COL + 4) * BLOCK_SIZE_X);
    float *p = ps.data(), *it = inter.data(), *o = pt.data(), *lr = lrow.data(), *lc = lcol.data();
    nd3((size_t)BLOCK_SIZE_X * ((wi - 1) / (BLOCK_SIZE_X * STEPS_ROW) + 1),
        (size_t)BLOCK_SIZE_Y * ((hi - 1) / BLOCK_SIZE_Y + 1), (size_t)n_half, BLOCK_SIZE_X, BLOCK_SIZE_Y, 1, kReplay,
        [&] { patch_similarities_row_pass(p, it, height_sim, width_sim, patch_size, patch_size_max, lr); });
    nd3((size_t)BLOCK_SIZE_X * ((wp - 1) / BLOCK_SIZE_X + 1),
        (size_t)BLOCK_SIZE_Y * ((hp - 1) / (BLOCK_SIZE_Y * STEPS_COL) + 1), (size_t)n_half, BLOCK_SIZE_X,
        BLOCK_SIZE_Y, 1, kReplay,
        [&] { patch_similarities_col_pass(it, o, height_sim, width_sim, patch_size, patch_size_max, lc); });
    std::copy(pt.begin(), pt.begin() + (size_t)n_half * hpat * wpat, out);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_patch_similarities: %s\n", e.what());
    return -1;
  }
}

// copy_symm_weights_test.cpp:33-128 setup: the upper half window of weights
// (n_half planes of (height_ori + wsh) x (width_ori + 2 wsh)) to the full
// window (sws^2 planes of height_ori x width_ori).
extern "C" int ref_copy_symm_weights(const float* wsymm, float* wfull, int height_ori, int width_ori, int sws) {
  using namespace refnl;
  try {
    const int wsh = (sws - 1) / 2, n_half = sws * wsh + wsh;
    Buf ws(wsymm, wsymm + (size_t)n_half * (height_ori + wsh) * (width_ori + 2 * wsh));
    ws.resize(ws.size() + kGuard);
    Buf wf = buf((size_t)sws * sws * height_ori * width_ori);
    float *a = ws.data(), *b = wf.data();
    nd2((size_t)width_ori, (size_t)height_ori, 1, 1, 0, 0, kNone,
        [&] { copy_symm_weights(a, b, height_ori, width_ori, sws); });
    std::copy(wf.begin(), wf.begin() + (size_t)sws * sws * height_ori * width_ori, wfull);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_copy_symm_weights: %s\n", e.what());
    return -1;
  }
}

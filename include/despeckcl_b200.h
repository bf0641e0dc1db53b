/* despeckcl_b200: C ABI of the B200-native NL-SAR engine.
 *
 * Plain pointers and sizes only.  Every entry point returns 0 on success and a
 * negative dcl_status on failure; dcl_last_error() describes the last failure
 * of the calling thread.  Host-pointer entry points copy inputs to the GPU and
 * results back, like the reference's filter drivers; *_device entry points
 * take device pointers and a cudaStream_t (passed as void*) and do not
 * synchronise.
 *
 * Reference interfaces replaced (paths relative to the despeckCL project root):
 *   dcl_nlsar_insar*         despeckcl::nlsar(float* ampl_master, ...)   include/despeckcl.h:45-59,
 *                                                                          src/compute/nlsar/nlsar.cpp:139-167
 *   dcl_nlsar_covmat*        despeckcl::nlsar(float* covmat_raw, ...)    include/despeckcl.h:62-73,
 *                                                                          src/compute/nlsar/nlsar.cpp:171-194
 *   dcl_nlsar_training_*     despeckcl::nlsar_training(...)              include/despeckcl.h:75-92,
 *                                                                          src/compute/nlsar/training/nlsar_training.cpp:57-96
 *   dcl_stats_save, _load    despeckcl::store/load_nlsar_stats_collection include/despeckcl.h:94-95,
 *                                                                          src/compute/nlsar/training/nlsar_training.cpp:99-113
 *   dcl_boxcar*              despeckcl::boxcar(...)                      include/despeckcl.h:34-43,
 *                                                                          src/compute/boxcar/boxcar.cpp:30-100
 *   dcl_goldstein*           despeckcl::goldstein(...)                   include/despeckcl.h:111-122,
 *                                                                          src/compute/goldstein/goldstein.cpp:39-106
 *   dcl_nlinsar*             despeckcl::nlinsar(...)                     include/despeckcl.h:97-109,
 *                                                                          src/compute/nlinsar/nlinsar.cpp:42-130
 *   dcl_stats_entry          nlsar::params + nlsar::stats                include/compute/nlsar/parameters.h:26-57,
 *                                                                          include/compute/nlsar/stats.h:28-55
 *
 * Staging timeouts.  The specialised NL-SAR kernel stages each tile with TMA
 * copies and waits for them with a bounded wait.  A thread block whose wait
 * runs out stops and leaves its remaining tiles unwritten (the reference has no
 * such case: it terminates the process on any OpenCL error,
 * src/compute/nlsar/nlsar_filter_sub_image.cpp:74-78).  It is reported:
 *   - by the host-pointer entry points (dcl_nlsar_insar, dcl_nlsar_covmat):
 *     DCL_ERR_TIMEOUT for that call;
 *   - by the request server: the requests of the affected launch finish with
 *     info.status DCL_ERR_TIMEOUT;
 *   - for every launch, whichever entry point made it: in the device's ledger,
 *     which dcl_take_stage_timeouts reads and resets.  The device, batched,
 *     prepared-batch and allocation-free entry points return once their work is
 *     queued, so their callers read the ledger after synchronising.
 */
#ifndef DESPECKCL_B200_H
#define DESPECKCL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum dcl_status {
  DCL_OK = 0,
  DCL_ERR_INVALID_ARGUMENT = -1,
  DCL_ERR_MISSING_STATS = -2,
  DCL_ERR_OUT_OF_MEMORY = -3,
  DCL_ERR_CUDA = -4,
  DCL_ERR_UNSUPPORTED = -5,
  DCL_ERR_TIMEOUT = -6,
  DCL_ERR_IO = -7
};

/* Per-pixel (patch, scale) selection.
 * DCL_SELECT_REFERENCE reproduces nlsar::get_best_params
 * (src/compute/nlsar/best_params.cpp:27-54): every pixel takes the last key of
 * the statistics map in (patch, scale) order.
 * DCL_SELECT_ARGMAX_ENL takes, per pixel, the combination with the largest
 * bias-reduced ENL (first in map order on ties), the documented NL-SAR rule. */
enum dcl_select_mode { DCL_SELECT_REFERENCE = 0, DCL_SELECT_ARGMAX_ENL = 1 };

/* One entry of an NL-SAR statistics collection: the key nlsar::params and the
 * fields of nlsar::stats.  quantilles and chi2cdf_inv hold lut_size floats. */
typedef struct dcl_stats_entry {
  int patch_size;
  int scale_size;
  unsigned int lut_size;
  float dissims_min;
  float dissims_max;
  const float* quantilles;
  const float* chi2cdf_inv;
} dcl_stats_entry;

/* Opaque statistics collection owned by the library (training and loading). */
typedef struct dcl_stats_collection dcl_stats_collection;

const char* dcl_last_error(void);
const char* dcl_version(void);

/* Thread blocks of this library's NL-SAR kernels on the current device that
 * gave up waiting for a TMA staging copy since the last call (see "Staging
 * timeouts" above); the ledger is read and reset atomically.  Call it after
 * synchronising the streams whose launches it should cover.  No reference
 * counterpart. */
int dcl_take_stage_timeouts(int* count);

/* Timing of this library's kernels on the calling thread (no reference
 * counterpart; the reference's timed_run, src/clcfg/clcfg.h:97-119, measures
 * host wall clock).  Between begin and end, CUDA events are recorded on the
 * launching stream around every fused NL-SAR launch; end waits for them and
 * returns the summed fused-kernel time, the number of fused launches and the
 * number of all kernels the library launched. */
void dcl_profile_begin(void);
/* Measured FP32 FMA throughput of the current device in TFLOP/s (FMA = 2
 * flops): the roofline denominator for the fused NL-SAR kernel.  No
 * reference counterpart. */
int dcl_measure_fp32_tflops(double* tflops);
int dcl_profile_end(double* fused_ms, long* fused_launches, long* all_launches);

/* NL-SAR on an InSAR pair; host pointers, row-major height x width float32.
 * Replaces despeckcl::nlsar (include/despeckcl.h:45-59). */
int dcl_nlsar_insar(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                    float* phase_filt, float* coh_filt, int height, int width, int search_window_size,
                    const int* patch_sizes, int n_patch_sizes, const int* scale_sizes, int n_scale_sizes,
                    const dcl_stats_entry* stats, int n_stats, float h_param, float c_param, int select_mode);

/* Same on device pointers, asynchronous on `stream`.  selection_out (device,
 * height x width int32, may be NULL) receives the selected combination's index
 * in the reference loop order (scale outer, patch inner).  A staging timeout
 * is counted in the device ledger (dcl_take_stage_timeouts).  Replaces
 * despeckcl::nlsar (include/despeckcl.h:45-59). */
int dcl_nlsar_insar_device(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                           float* phase_filt, float* coh_filt, int height, int width, int search_window_size,
                           const int* patch_sizes, int n_patch_sizes, const int* scale_sizes, int n_scale_sizes,
                           const dcl_stats_entry* stats, int n_stats, float h_param, float c_param,
                           int select_mode, int* selection_out, void* stream);

/* NL-SAR on device pointers without allocating device memory.  No
 * counterpart in the reference: it exists for callers that cannot allocate
 * GPU memory while they filter (a fixed memory budget, a host framework that
 * owns the allocator, or code that must not grow the pool mid-stream).  Same
 * arguments and results as dcl_nlsar_insar_device; the scratch is a 64 MiB
 * static device array shared by all calls on a device, so scenes whose padded
 * frame does not fit are rejected with DCL_ERR_INVALID_ARGUMENT (about
 * 1000 x 1000 pixels with search 21, patches {3,5,7}, scales {1,3}), and calls
 * that overlap on the GPU race.  The first call on a device resolves the
 * array's address: make it before any stream capture.  The call copies its
 * scene descriptor and weight tables from pageable host memory, so it may wait
 * for the stream's earlier work before returning.  A staging timeout is counted
 * in the device ledger (dcl_take_stage_timeouts). */
int dcl_nlsar_insar_device_noalloc(const float* ampl_master, const float* ampl_slave, const float* phase,
                                   float* ref_filt, float* phase_filt, float* coh_filt, int height, int width,
                                   int search_window_size, const int* patch_sizes, int n_patch_sizes,
                                   const int* scale_sizes, int n_scale_sizes, const dcl_stats_entry* stats,
                                   int n_stats, float h_param, float c_param, int select_mode, int* selection_out,
                                   void* stream);

/* NL-SAR on a covariance image [2*dim*dim][height][width] (even planes real,
 * odd planes imaginary), host pointers.  dim 2 (InSAR) or 3 (PolSAR); any
 * other dim is DCL_ERR_INVALID_ARGUMENT.  Replaces despeckcl::nlsar
 * (include/despeckcl.h:62-73). */
int dcl_nlsar_covmat(const float* covmat_raw, float* covmat_filt, int height, int width, int dim,
                     int search_window_size, const int* patch_sizes, int n_patch_sizes, const int* scale_sizes,
                     int n_scale_sizes, const dcl_stats_entry* stats, int n_stats, float h_param, float c_param,
                     int select_mode);

/* Same on device pointers, asynchronous on `stream`; a staging timeout is
 * counted in the device ledger (dcl_take_stage_timeouts).  Replaces
 * despeckcl::nlsar (include/despeckcl.h:62-73). */
int dcl_nlsar_covmat_device(const float* covmat_raw, float* covmat_filt, int height, int width, int dim,
                            int search_window_size, const int* patch_sizes, int n_patch_sizes,
                            const int* scale_sizes, int n_scale_sizes, const dcl_stats_entry* stats, int n_stats,
                            float h_param, float c_param, int select_mode, void* stream);

/* Batched NL-SAR: n_scenes InSAR pairs of possibly different sizes, all
 * filtered with the same parameters in one persistent launch.  Each array
 * holds n_scenes device pointers / sizes; a staging timeout is counted in the
 * device ledger (dcl_take_stage_timeouts).  The batched counterpart of
 * despeckcl::nlsar (include/despeckcl.h:45-59). */
int dcl_nlsar_insar_batch_device(int n_scenes, const float* const* ampl_master, const float* const* ampl_slave,
                                 const float* const* phase, float* const* ref_filt, float* const* phase_filt,
                                 float* const* coh_filt, const int* heights, const int* widths,
                                 int search_window_size, const int* patch_sizes, int n_patch_sizes,
                                 const int* scale_sizes, int n_scale_sizes, const dcl_stats_entry* stats,
                                 int n_stats, float h_param, float c_param, int select_mode, void* stream);

/* Prepared batches.  A batch binds n_scenes device input/output pointer sets
 * and the filter parameters once: the scratch, the scene descriptors and the
 * weight tables are set up at creation, every run filters all scenes with one
 * fused launch.  Flags: DCL_BATCH_GRAPH captures the launch sequence in a CUDA
 * graph (each run is one graph launch); DCL_BATCH_AUTOTUNE times the
 * specialised kernel's instantiations on the batch at creation and keeps the
 * fastest (cached per device and configuration; DESPECKCL_B200_TUNE_CACHE names
 * a file that keeps the choices across processes).  The autotuner times up to
 * three tile shapes: 32 x 32 tiles with 2 or 4 pixels per thread (variants 0
 * and 1) and, for patches {3,5,7}, 32 x 16 tiles with 2 pixels per thread
 * (variant 2, the batch's frames re-carved for 16-row tiles); every shape
 * gives the same bits.  DCL_BATCH_VARIANT1 / DCL_BATCH_VARIANT2 select
 * variant 1 / 2 without timing (variant 2 where the shape has it).  A run's staging
 * timeouts are counted in the device ledger (dcl_take_stage_timeouts).  The batched counterpart of
 * despeckcl::nlsar (include/despeckcl.h:45-59); the reference filters one scene
 * per call. */
enum dcl_batch_flags { DCL_BATCH_GRAPH = 1, DCL_BATCH_AUTOTUNE = 2, DCL_BATCH_VARIANT1 = 4, DCL_BATCH_VARIANT2 = 8 };
typedef struct dcl_nlsar_batch dcl_nlsar_batch;
dcl_nlsar_batch* dcl_nlsar_batch_create(int n_scenes, const float* const* ampl_master,
                                        const float* const* ampl_slave, const float* const* phase,
                                        float* const* ref_filt, float* const* phase_filt, float* const* coh_filt,
                                        const int* heights, const int* widths, int search_window_size,
                                        const int* patch_sizes, int n_patch_sizes, const int* scale_sizes,
                                        int n_scale_sizes, const dcl_stats_entry* stats, int n_stats,
                                        float h_param, float c_param, int select_mode, int flags, void* stream);
int dcl_nlsar_batch_run(dcl_nlsar_batch* batch, void* stream);
/* The kernel instantiation in use (0: 32 x 32 tiles, 2 pixels per thread;
 * 1: 32 x 32, 4 pixels per thread; 2: 32 x 16, 2 pixels per thread). */
int dcl_nlsar_batch_variant(const dcl_nlsar_batch* batch);
/* Kernels one run launches (prep kernels per scene plus the fused launch). */
int dcl_nlsar_batch_launches(const dcl_nlsar_batch* batch);
void dcl_nlsar_batch_destroy(dcl_nlsar_batch* batch);

/* Request server (no counterpart in the reference, which filters one scene per
 * blocking call, src/compute/nlsar/nlsar.cpp:139-167).  A server binds the
 * filter parameters and a device-memory budget on the current device; a worker
 * thread admits submitted scenes oldest-first while their memory fits the
 * budget, filters the admitted tiles in launches of at most max_batch_tiles
 * tiles (large scenes are split over several launches, scenes that arrive while
 * one runs join the next), and keeps up to max_inflight launches queued on
 * separate streams.  Results are bitwise those of dcl_nlsar_insar_device on the
 * same scene.  A launch with a staging timeout fails its requests with
 * DCL_ERR_TIMEOUT.  flags: DCL_BATCH_VARIANT1 as for prepared batches. */
typedef struct dcl_server dcl_server;
typedef struct {
  int status;                  /* DCL_OK, or the error that failed the request */
  int chunks;                  /* launches the request's tiles were spread over */
  long long first_batch, last_batch;
  double submit_s, admit_s, launch_s, done_s; /* seconds since dcl_server_create */
} dcl_request_info;
typedef struct {
  long long submitted, completed, failed, batches, kernel_launches, tiles;
  unsigned long long budget_bytes, admitted_bytes, peak_admitted_bytes;
  int queued, admitted, inflight; /* now */
  int peak_inflight;              /* launches in flight at once, highest seen */
} dcl_server_stats;
dcl_server* dcl_server_create(int search_window_size, const int* patch_sizes, int n_patch_sizes,
                              const int* scale_sizes, int n_scale_sizes, const dcl_stats_entry* stats, int n_stats,
                              float h_param, float c_param, int select_mode, unsigned long long hbm_budget_bytes,
                              int max_inflight, int max_batch_tiles, int flags);
/* Queue one scene.  host_buffers = 0: device pointers, read after
 * `ready_event` (a cudaEvent_t, or NULL) completes; 1: host pointers (pinned
 * for overlap), staged through the budget.  Returns the request id (>= 0) or a
 * negative status (DCL_ERR_OUT_OF_MEMORY when the scene alone exceeds the
 * budget).  The buffers must stay valid until the request is waited for. */
long long dcl_server_submit(dcl_server* server, const float* ampl_master, const float* ampl_slave,
                            const float* phase, float* ref_filt, float* phase_filt, float* coh_filt, int height,
                            int width, int host_buffers, void* ready_event);
/* Block until the request has finished (timeout_s < 0: no limit), fill `info`
 * and forget the request.  Returns DCL_OK when it finished (info->status tells
 * how), DCL_ERR_TIMEOUT otherwise. */
int dcl_server_wait(dcl_server* server, long long request, double timeout_s, dcl_request_info* info);
/* 1 (and `info`, request forgotten) if finished, 0 if not, negative on error. */
int dcl_server_poll(dcl_server* server, long long request, dcl_request_info* info);
double dcl_server_now(const dcl_server* server);
int dcl_server_get_stats(dcl_server* server, dcl_server_stats* out);
/* Finishes every submitted request, then frees the server. */
void dcl_server_destroy(dcl_server* server);

/* Boxcar filter with a window_width x window_width window; host pointers.
 * Replaces despeckcl::boxcar (include/despeckcl.h:34-43). */
int dcl_boxcar(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
               float* phase_filt, float* coh_filt, int height, int width, int window_width);

/* Same on device pointers, asynchronous on `stream`.  Replaces
 * despeckcl::boxcar (include/despeckcl.h:34-43). */
int dcl_boxcar_device(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                      float* phase_filt, float* coh_filt, int height, int width, int window_width, void* stream);

/* Goldstein phase filter with patch_size x patch_size FFT patches (32 on the
 * GPU), overlap `overlap` and exponent `alpha`; host pointers.  ref_filt gets
 * the filtered interferogram's amplitude and phase_filt its phase; coh_filt is
 * not written (the reference leaves it as passed).  Scenes are one tile of the
 * reference's tiling, which holds for every scene whose padded side fits the
 * reference's device allocation bound.  Replaces despeckcl::goldstein
 * (include/despeckcl.h:111-122). */
int dcl_goldstein(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                  float* phase_filt, float* coh_filt, int height, int width, int patch_size, int overlap,
                  float alpha);

/* Same on device pointers, asynchronous on `stream`.  Replaces
 * despeckcl::goldstein (include/despeckcl.h:111-122). */
int dcl_goldstein_device(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                         float* phase_filt, float* coh_filt, int height, int width, int patch_size, int overlap,
                         float alpha, void* stream);

/* NL-InSAR with a search window search_window_size^2, patch_size^2 patches
 * (3 or 7: the sizes for which the reference tabulates its h), niter passes
 * and at least lmin looks (1..64); host pointers.  ref_filt, phase_filt and
 * coh_filt hold the initial estimates on entry (the Python binding passes
 * zeros) and the results on exit.  Replaces despeckcl::nlinsar
 * (include/despeckcl.h:97-109). */
int dcl_nlinsar(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                float* phase_filt, float* coh_filt, int height, int width, int search_window_size, int patch_size,
                int niter, int lmin);

/* Same on device pointers, asynchronous on `stream`.  Replaces
 * despeckcl::nlinsar (include/despeckcl.h:97-109). */
int dcl_nlinsar_device(const float* ampl_master, const float* ampl_slave, const float* phase, float* ref_filt,
                       float* phase_filt, float* coh_filt, int height, int width, int search_window_size,
                       int patch_size, int niter, int lmin, void* stream);

/* Training on a homogeneous area; host pointers.  Returns NULL on failure.
 * Replaces despeckcl::nlsar_training (include/despeckcl.h:75-83). */
dcl_stats_collection* dcl_nlsar_training_insar(const float* ampl_master, const float* ampl_slave,
                                               const float* phase, int height, int width, const int* patch_sizes,
                                               int n_patch_sizes, const int* scale_sizes, int n_scale_sizes);

/* Training on a covariance image [2*dim*dim][height][width]; dim 2 or 3.
 * Replaces despeckcl::nlsar_training (include/despeckcl.h:85-92). */
dcl_stats_collection* dcl_nlsar_training_covmat(const float* covmat, int height, int width, int dim,
                                                const int* patch_sizes, int n_patch_sizes, const int* scale_sizes,
                                                int n_scale_sizes);

/* A one-entry collection with the LUTs of `n` dissimilarities, as the
 * reference's nlsar::stats::stats(std::vector<float> dissims, unsigned lut_size)
 * constructor builds them (src/compute/nlsar/stats.cpp:28-80). */
dcl_stats_collection* dcl_stats_from_dissims(int patch_size, int scale_size, const float* dissims, long n,
                                             unsigned int lut_size);

int dcl_stats_collection_size(const dcl_stats_collection* c);
/* Entry i in (patch, scale) order; the pointers stay valid until the collection is freed. */
int dcl_stats_collection_get(const dcl_stats_collection* c, int i, dcl_stats_entry* out);
/* A collection holding copies of the given entries. */
dcl_stats_collection* dcl_stats_collection_from_entries(const dcl_stats_entry* entries, int n);
void dcl_stats_collection_free(dcl_stats_collection* c);

/* Store / load a statistics collection (despeckcl::store/load_nlsar_stats_collection,
 * include/despeckcl.h:94-95).
 * dcl_stats_save writes this library's versioned text format.
 * dcl_stats_save_boost_text writes the file the reference's
 * store_nlsar_stats_collection writes (src/compute/nlsar/training/nlsar_training.cpp:99-104):
 * a Boost text archive of std::map<nlsar::params, nlsar::stats>, produced
 * without Boost; the reference's load_nlsar_stats_collection reads it.
 * dcl_stats_load reads either, telling them apart by their first words; a
 * Boost archive is parsed strictly (class-info, count and item-version words
 * where Boost writes them) and a malformed one fails with DCL_ERR_IO. */
int dcl_stats_save(const dcl_stats_collection* c, const char* filename);
int dcl_stats_save_boost_text(const dcl_stats_collection* c, const char* filename);
dcl_stats_collection* dcl_stats_load(const char* filename);

#ifdef __cplusplus
}
#endif
#endif

/* apg-sgm B200 engine: extended C-ABI.
 *
 * The reference-compatible session API lives in apg_sgm/c_api.h and is implemented by the same
 * library (libapg_sgm_b200.so).  This header adds the entry points a host needs beyond that API:
 * an engine over an explicit configuration record, device-pointer processing on a caller stream,
 * stage dumps for parity checking, the batched form and the served form.
 *
 * Every function is extern "C" with plain pointers and sizes; no exception crosses the ABI.
 * Status codes are the reference's apg_status_code_t values (0 = OK).
 */
#ifndef APG_SGM_CUDA_H
#define APG_SGM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "apg_sgm/c_api.h"
#include "apg_sgm/metrics.h"
#include "apg_sgm/pipeline_config.h"
#include "apg_sgm/telemetry.h"

#if defined(__GNUC__) && __GNUC__ >= 4
#define APGCU_API __attribute__((visibility("default")))
#else
#define APGCU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct apgcu_engine_s* apgcu_engine_t;

/* Intermediates that apgcu_engine_dump can copy out after a process call. */
enum {
    APGCU_DUMP_LEFT_GRAY = 0, APGCU_DUMP_LEFT_GX, APGCU_DUMP_LEFT_GY,
    APGCU_DUMP_RIGHT_GRAY, APGCU_DUMP_RIGHT_GX, APGCU_DUMP_RIGHT_GY,  /* u8  W*H */
    APGCU_DUMP_CENSUS_LEFT, APGCU_DUMP_CENSUS_RIGHT,                  /* u32 W*H (u64 for 9x7) */
    APGCU_DUMP_RANGE_MIN, APGCU_DUMP_RANGE_MAX,                        /* i16 W*H */
    APGCU_DUMP_COST_RAW,        /* u16 W*H*D  (needs APGCU_DEBUG_RAW_COST) */
    APGCU_DUMP_COST_AGG,        /* u16 W*H*D  (cross-aggregated volume; Balanced/HQ) */
    APGCU_DUMP_SGM_SUM,         /* u16 W*H*D  (needs APGCU_DEBUG_KEEP_SUM) */
    APGCU_DUMP_DISP_WTA, APGCU_DUMP_BEST, APGCU_DUMP_SECOND, APGCU_DUMP_DISP_RIGHT,
    APGCU_DUMP_CONFIDENCE, APGCU_DUMP_RELIABLE, APGCU_DUMP_REASON_CONF,
    APGCU_DUMP_DISP_REFINED, APGCU_DUMP_DISP_LR, APGCU_DUMP_REASON, APGCU_DUMP_DISP_FILL,
    APGCU_DUMP_DISPARITY, APGCU_DUMP_D_PRIOR,
    APGCU_DUMP_COUNT
};

/* Debug flags (apgcu_engine_set_debug). */
#define APGCU_DEBUG_RAW_COST 1   /* also materialise the raw cost volume */
#define APGCU_DEBUG_KEEP_SUM 2   /* also store the final path sum */
#define APGCU_DEBUG_NO_FUSION 4  /* Fast mode: read a stored volume instead of recomputing costs */
#define APGCU_DEBUG_PROFILE 8    /* record a CUDA event after every launch (apgcu_engine_launch_profile) */

/* Engine on CUDA device `device`.  stream may be NULL (the engine creates its own) or a
 * cudaStream_t the caller keeps alive for the engine's lifetime.  Returns NULL on failure. */
APGCU_API apgcu_engine_t apgcu_engine_create(const apg_pipeline_config_t* cfg, int device, void* stream);
APGCU_API void apgcu_engine_destroy(apgcu_engine_t e);
APGCU_API const char* apgcu_engine_last_error(apgcu_engine_t e);
APGCU_API int apgcu_engine_set_debug(apgcu_engine_t e, int flags);

/* Kernel tuning knobs (results never change, only speed):
 *   "sgm_lanes": lanes per SGM scanline chain, 8 / 16 / 32 (0 = default, 32);
 *   "sgm_split": the volume-fed last sweep with its recurrence and its sums / WTA on two warps per
 *                chain: 0 = for 64 padded disparities (default), 1 = never, 2 = always;
 *   "cost_tile": columns per block of the cost kernel, 64 / 128 / 256 (0 = default for the range);
 *   "fast_fused": 1 = census-only Fast mode recomputes its costs inside the SGM sweeps and stores no
 *                 cost volume (less memory, slower); 0 = store the volume once (default);
 *   "cost_kernel": 0 = pixel-run cost kernel where it applies (default), 1 = column-tile kernel;
 *   "cost8": the volume the SGM sweeps read (the census-only Fast volume, or the aggregated
 *            volume of one aggregation pass) at one byte per voxel (0xFF invalid; exact while
 *            every quantised cost is below 255): 0 = at 256 padded disparities (default),
 *            1 = never, 2 = at 128 and 256;
 *   "refine_window": 0 = HighQuality refiner reads the right-image window from shared memory where
 *                 every band fits on the device at once (default), 1 = always through L1;
 *   "host_bands": frames whose outputs go to host memory (apgcu_engine_process, the session) run
 *                 the last SGM sweep in this many row bands, 2..16, and each band's finished map
 *                 rows are post-processed and copied to the host while the next band runs:
 *                 0 = 6 bands where the path allows it (default; Path4, 128..256 padded
 *                 disparities, one warp per chain, no refiner, 3x3 or no median, no telemetry
 *                 scope, at least 256 rows), 1 = never (one sweep, then the copies);
 *   "device_bands": the same for apgcu_engine_process_device (the copies go to the caller's
 *                 device buffers): 0 = never (default), 2..16 = that many bands.  The post kernels
 *                 then run beside the sweep's bands; measured on one B200 that was slower at
 *                 1280x720 (0.735 -> 0.786 ms Fast) and faster at 1920x1080 D256 Fast (2.570 ->
 *                 2.400 ms with 6 bands).
 * And one key that bounds a wait rather than tuning speed:
 *   "refine_spin_limit": polls (each ~128 ns) before a refiner band stops waiting for the band above
 *                 (0 = default, about a second).  A wait that runs out sets the frame's error flag,
 *                 every band returns, and the frame fails with APG_STATUS_INTERNAL_ERROR ("refine: a
 *                 wavefront wait timed out"); the next frame starts clean.
 * Returns 0, or APG_STATUS_INVALID_CONFIG for an unknown key or value. */
APGCU_API int apgcu_engine_set_tuning(apgcu_engine_t e, const char* key, int value);

/* One pair from HOST memory (strided, 1 or 3 channels); outputs are host arrays of W*H.
 * Copies in and out are part of the call.  Any output pointer may be NULL. */
APGCU_API int apgcu_engine_process(apgcu_engine_t e, const uint8_t* left, const uint8_t* right, int width,
                                   int height, int stride, int channels, float* disparity, float* confidence,
                                   uint8_t* invalid_reason, uint8_t* reliable_mask);

/* One pair already resident in DEVICE memory; outputs are device arrays.  Enqueued on the
 * engine stream; returns after enqueueing (call apgcu_engine_sync to wait). */
APGCU_API int apgcu_engine_process_device(apgcu_engine_t e, const uint8_t* d_left, const uint8_t* d_right,
                                          int width, int height, int stride, int channels, float* d_disparity,
                                          float* d_confidence, uint8_t* d_invalid_reason,
                                          uint8_t* d_reliable_mask);
APGCU_API int apgcu_engine_sync(apgcu_engine_t e);

/* Copy intermediate `what` (APGCU_DUMP_*) of the last processed pair to host memory. */
APGCU_API int apgcu_engine_dump(apgcu_engine_t e, int what, void* host_dst, size_t bytes);

/* Per-stage device times of the last pair (ms): aux, prior, cost, cross, right_wta, sgm, wta,
 * confidence, refine, post, total -- the reference StageTiming fields in declaration order. */
APGCU_API int apgcu_engine_stage_times(apgcu_engine_t e, double* ms11);

/* Per-launch device times of the last pair (needs APGCU_DEBUG_PROFILE): up to max entries of
 * (static kernel name, ms); returns the number written. */
APGCU_API int apgcu_engine_launch_profile(apgcu_engine_t e, int max, const char** names, float* ms);

/* Bytes of device workspace the engine holds now, and would need for a W x H pair. */
APGCU_API size_t apgcu_engine_allocated_bytes(apgcu_engine_t e);
APGCU_API size_t apgcu_workspace_bytes(const apg_pipeline_config_t* cfg, int width, int height);
APGCU_API void apgcu_engine_release(apgcu_engine_t e);

/* Stream the engine enqueues on (a cudaStream_t). */
APGCU_API void* apgcu_engine_stream(apgcu_engine_t e);

/* HierarchicalTelemetry of the engine's last pair (src/hierarchical_stereo.hpp:36-42), computed
 * from device counters: out6 = {avg_states_per_pixel, coarse_valid_ratio, fallback_pixel_ratio,
 * full_range_pixel_ratio, coarse pass device time in ms, 1 if the coarse pass ran (0 for frames
 * under 32 x 32 or with hierarchical mode off)}.  Waits for the engine stream. */
APGCU_API int apgcu_engine_hier_telemetry(apgcu_engine_t e, double* out6);

/* Experimental scopes of the CALLING THREAD (ExperimentalSubpixelScope, src/subpixel_estimator.hpp;
 * ExperimentalInpaintScope, src/inpaint_internal.hpp), read by every engine, session and batch call
 * made on that thread when it starts a frame: subpixel_method 0 Legacy, 1 CurvGate, 2 ConfGate,
 * 3 Stabilized with its parameter (<= 0: the method's default); inpaint_method 0 Legacy,
 * 1 ShadowReclass with its gap (Legacy at 32 keeps the configuration's max_fill_gap).  Defaults
 * (0, 0, 0, 32) reproduce the reference without scopes.  The allocation-free right-image WTA
 * always uses Legacy.  Returns 0 or APG_STATUS_INVALID_CONFIG for an unknown method. */
APGCU_API int apgcu_set_experimental(int subpixel_method, float subpixel_param, int inpaint_method, int inpaint_gap);
APGCU_API void apgcu_get_experimental(int* subpixel_method, float* subpixel_param, int* inpaint_method,
                                      int* inpaint_gap);
/* The scopes' telemetry (collect_telemetry): while on for the calling thread, every frame it runs
 * adds the WTA's sub-pixel counters and the hole fill's counters (SubpixelTelemetry,
 * InpaintTelemetry; the hierarchical coarse pass included, as in the reference) to the thread's
 * totals when the frame completes (apgcu_engine_process, apg_session_process, a batch call, or
 * apgcu_engine_sync after apgcu_engine_process_device).  get copies the totals, reset clears them. */
APGCU_API int apgcu_set_experimental_telemetry(int subpixel, int inpaint);
APGCU_API void apgcu_get_experimental_telemetry(int* subpixel, int* inpaint);
APGCU_API void apgcu_get_telemetry(apg_subpixel_telemetry_t* subpixel, apg_inpaint_telemetry_t* inpaint);
APGCU_API void apgcu_reset_telemetry(int subpixel, int inpaint);

/* The prior's selected supports of the engine's last pair, in the reference's order
 * (PipelineBuffers::supports): up to cap entries written; returns the total count (0 without a
 * prior, -1 on error).  Waits for the engine stream. */
APGCU_API int apgcu_engine_supports(apgcu_engine_t e, int* x, int* y, float* disparity, float* confidence, int cap);

/* PipelineConfig::from_mode (src/config.cpp:5-45) into *out. */
APGCU_API void apgcu_config_from_mode(int mode, int max_disparity, apg_pipeline_config_t* out);

/* Session over a full configuration record (the reference's C++ StereoSession(PipelineConfig,
 * ExecutionOptions) constructor, include/apg_sgm/session.hpp:19-23); processed with
 * apg_session_process like any other session. */
APGCU_API apg_session_t apgcu_session_create_config(const apg_pipeline_config_t* cfg, int memory_policy,
                                                    size_t max_retained_bytes);
/* PipelineStats of the last frame: stage_ms11 as apgcu_engine_stage_times; counters4 =
 * {frame_allocation_count, frame_reuse_count, peak_workspace_bytes, retained_workspace_bytes}. */
APGCU_API int apgcu_session_get_stats(apg_session_t s, double* stage_ms11, size_t* counters4);
/* The engine tuning keys of apgcu_engine_set_tuning for a session's engine (kept across
 * ReleasePerFrame and the lazily created engine).  Returns 0 or APG_STATUS_INVALID_CONFIG. */
APGCU_API int apgcu_session_set_tuning(apg_session_t s, const char* key, int value);
/* Frame counters of the last frame (PipelineStats, src/pipeline.cpp:650-707), computed on the device:
 * counts8 = {valid_pixels, reliable_pixels, unreliable_pixels, refine_changed_pixels, lr_fail_pixels,
 * prior_support_count, sum of search-range widths, sum of geometric range widths}. */
APGCU_API int apgcu_session_get_frame_counts(apg_session_t s, unsigned long long* counts8);
/* HierarchicalTelemetry of the session's last frame, as apgcu_engine_hier_telemetry. */
APGCU_API int apgcu_session_hier_telemetry(apg_session_t s, double* out6);
/* Workspace bytes the budget gate compares against max_retained_bytes for a W x H x C frame. */
APGCU_API size_t apgcu_session_estimate_bytes(apg_session_t s, int width, int height, int channels);

/* ---- Accuracy metrics (evaluate_stereo, src/metrics.cpp:119-502; the support block is not part
 * of it).  est / gt: W*H disparity maps; range_min / range_max (int16 W*H, half-open per-pixel
 * intervals), d_before_refine / d_after_refine, vis_mask (W*H, >= 200 = visible) and left_image
 * (left_stride bytes per row, 1 or 3 channels: the low-texture split) may each be NULL, as the
 * reference's optional arguments.  thresholds NULL means QualityThresholds{}.  device_buffers != 0:
 * every array is device memory on the current device and the call enqueues on `stream` (a
 * cudaStream_t, NULL = the legacy default stream); otherwise they are host arrays copied in.
 * Returns when *out is written: counts exact, ratios formed with the reference's float
 * expressions, sums of errors in double (equal to the reference's whenever its sequential double
 * sum is exact).  Scratch (and the device copies of host inputs) comes from a stream-ordered pool the
 * library owns per device, which keeps its high-water mark between calls. */
APGCU_API int apgcu_evaluate_stereo(const float* est, const float* gt, int width, int height,
                                    const int16_t* range_min, const int16_t* range_max,
                                    const float* d_before_refine, const float* d_after_refine,
                                    const uint8_t* vis_mask, float max_valid_gt, const uint8_t* left_image,
                                    int left_stride, int left_channels, const apg_quality_thresholds_t* thresholds,
                                    int device_buffers, void* stream, apg_stereo_metrics_t* out);

/* evaluate_supports (src/metrics.cpp:8-124): n_supports support matches (x, y, disparity; e.g.
 * apgcu_engine_supports) against the W x H ground truth gt, vis_mask (nullable, >= 200 = visible),
 * cells of cell_size pixels (16 in the reference).  Buffers as apgcu_evaluate_stereo's. */
APGCU_API int apgcu_evaluate_supports(const int* x, const int* y, const float* disparity, int n_supports,
                                      const float* gt, int width, int height, const uint8_t* vis_mask,
                                      float max_valid_gt, int cell_size, int device_buffers, void* stream,
                                      apg_support_metrics_t* out);

/* Device time (ms) of the two kernels of this thread's last apgcu_evaluate_stereo, from events on
 * its stream around them. */
APGCU_API float apgcu_metrics_last_kernel_ms(void);

/* ---- On-disk formats (src/image.cpp:62-206), byte-compatible with the reference's readers and
 * writers.  Status: 0, APG_STATUS_EMPTY_INPUT (no such file / null argument),
 * APG_STATUS_INVALID_CONFIG (malformed or short file, unsupported magic, maxval outside 1..255),
 * APG_STATUS_SIZE_MISMATCH (dst too small: the dimensions are still written). */
APGCU_API int apgcu_image_info(const char* path, int* width, int* height, int* channels);   /* P5 / P6 */
APGCU_API int apgcu_load_image(const char* path, uint8_t* dst, size_t dst_bytes, int* width, int* height,
                               int* channels);                                             /* load_image */
APGCU_API int apgcu_save_pgm(const char* path, const uint8_t* img, int width, int height); /* save_pgm */
APGCU_API int apgcu_save_pgm16(const char* path, const int16_t* disp, int width, int height); /* save_pgm16 */
APGCU_API int apgcu_save_disparity_preview(const char* path, const float* disp, int width, int height,
                                           float dmax);                                    /* save_disparity_preview */
APGCU_API int apgcu_pfm_info(const char* path, int* width, int* height, int* channels);
APGCU_API int apgcu_load_pfm(const char* path, float* dst, size_t dst_floats, int* width, int* height); /* load_pfm */
APGCU_API int apgcu_save_pfm(const char* path, const float* img, int width, int height);  /* save_pfm */

/* Pair loader (no reference counterpart): `threads` workers read (left, right) image files into
 * page-locked buffers that the loader recycles, so engines and the server take them by DMA.
 * submit returns at once with a ticket; wait blocks until that pair is read and lends its two
 * images (valid until release). */
typedef struct apgcu_loader_s* apgcu_loader_t;
typedef struct {
    int status;                 /* as apgcu_load_image; SIZE_MISMATCH if the two images differ */
    int width, height, channels;
    const uint8_t* left;        /* page-locked, width*height*channels bytes, rows contiguous */
    const uint8_t* right;
} apgcu_loaded_pair_t;
APGCU_API apgcu_loader_t apgcu_loader_create(int threads);
APGCU_API void apgcu_loader_destroy(apgcu_loader_t l);
APGCU_API int apgcu_loader_submit(apgcu_loader_t l, const char* left_path, const char* right_path,
                                  unsigned long long* ticket);
APGCU_API int apgcu_loader_wait(apgcu_loader_t l, unsigned long long ticket, apgcu_loaded_pair_t* out);
APGCU_API int apgcu_loader_release(apgcu_loader_t l, unsigned long long ticket);
APGCU_API size_t apgcu_loader_pinned_bytes(apgcu_loader_t l);

/* Number of kernels the library has launched in this process (all engines). */
APGCU_API unsigned long long apgcu_kernel_launch_count(void);

/* ---- Batched form: many pairs of uneven sizes per call.
 *
 * No counterpart in the reference (which processes one pair per call): pairs are grouped into
 * buckets of equal size and disparity range; every pair runs its per-pixel stages on its own
 * stream, and the pairs of ALL buckets share one persistent SGM launch per phase (a work queue of
 * (pair, direction, scanline) units over pairs of any size and padded range); the whole call is a
 * cached CUDA graph per composition (buckets and pair counts); the cost kernel's tile width is
 * autotuned per bucket.  With the option "unified_sgm" 0 each bucket runs on its own stream with
 * its own SGM launches, and the tuner also chooses lanes per scanline and the persistent-grid cap.
 * Every pair's outputs equal what apgcu_engine_process gives for it alone. */
typedef struct apgcu_batch_s* apgcu_batch_t;
typedef struct {
    const uint8_t* left;        /* host or device memory, as the call's device_buffers says */
    const uint8_t* right;
    int width, height, stride, channels;
    int max_disparity;          /* this pair's range end (0: the batch configuration's) */
    float* disparity;           /* outputs, W*H each; any may be NULL */
    float* confidence;
    uint8_t* invalid_reason;
    uint8_t* reliable_mask;
} apgcu_pair_t;

/* Batch over a configuration record (its max_disparity is the default range end). NULL if the
 * configuration is invalid. */
APGCU_API apgcu_batch_t apgcu_batch_create(const apg_pipeline_config_t* cfg, int device);
APGCU_API void apgcu_batch_destroy(apgcu_batch_t b);
APGCU_API const char* apgcu_batch_last_error(apgcu_batch_t b);
/* Processes npairs pairs and returns when every output is written.  device_buffers != 0: inputs
 * and outputs are device pointers on the batch's device. */
APGCU_API int apgcu_batch_process(apgcu_batch_t b, int npairs, const apgcu_pair_t* pairs, int device_buffers);
/* Options (results never change): "graphs" 0/1, "batched_sgm" 0/1, "unified_sgm" 0/1 (one SGM
 * launch per phase over all buckets, default 1), "autotune" 0/1, "sgm_lanes" 0/16/32 (0 =
 * autotuned; 16 runs per bucket), "max_blocks_per_sm" -1 (autotuned) / 0 (occupancy) / N,
 * "cost_tile" 0 (autotuned) / 64 / 128 / 256. */
APGCU_API int apgcu_batch_set_option(apgcu_batch_t b, const char* key, int value);
APGCU_API size_t apgcu_batch_allocated_bytes(apgcu_batch_t b);
/* Device time of the last apgcu_batch_process (ms): from one start event every bucket waits on to
 * the latest bucket end, copies included. */
APGCU_API float apgcu_batch_last_time_ms(apgcu_batch_t b);
APGCU_API void apgcu_batch_release(apgcu_batch_t b);

/* ---- Served form: a request loop with continuous batching.
 *
 * No counterpart in the reference.  `slots` worker threads take requests in arrival order; each
 * borrows a device-resident engine of the request's (mode, size, range) from a pool (or creates
 * one), runs it on the engine's own stream and returns it, so requests that arrive while others
 * are on the GPU are admitted as slots and memory free up and overlap on the device.  Engine
 * workspaces are admitted against an HBM budget (min of hbm_budget_bytes and the device's free
 * memory less 2 GiB); idle engines of other buckets are released to make room.  Each result
 * equals the single-pair engine's output for that pair. */
typedef struct apgcu_server_s* apgcu_server_t;
typedef struct {
    int mode;                   /* APG_QUALITY_FAST / BALANCED / HIGH_QUALITY */
    int min_disparity, max_disparity;
    const uint8_t* left;        /* host memory, valid until the request completes */
    const uint8_t* right;
    int width, height, stride, channels;
    float* disparity;           /* host outputs, W*H each; any may be NULL */
    float* confidence;
    uint8_t* invalid_reason;
    uint8_t* reliable_mask;
} apgcu_request_t;

APGCU_API apgcu_server_t apgcu_server_create(int device, size_t hbm_budget_bytes, int slots);
/* Finishes queued requests' in-flight work, then stops the workers. */
APGCU_API void apgcu_server_destroy(apgcu_server_t s);
/* Queues a request (returns at once); *ticket identifies it. */
APGCU_API int apgcu_server_submit(apgcu_server_t s, const apgcu_request_t* r, unsigned long long* ticket);
/* Blocks until the request completes; returns its status; *latency_ms = submission to completion. */
APGCU_API int apgcu_server_wait(apgcu_server_t s, unsigned long long ticket, double* latency_ms);
/* counts4 = {completed, failed, engine evictions, peak requests in flight};
 * bytes2 = {reserved workspace bytes now, peak reserved}. */
APGCU_API int apgcu_server_stats(apgcu_server_t s, unsigned long long* counts4, size_t* bytes2);
APGCU_API size_t apgcu_server_budget(apgcu_server_t s);
/* Warm pool: creates `count` idle engines for requests like *like (its mode, size and range; the
 * image pointers are not read), each run once on a blank pair, so that later requests of that
 * bucket find device-resident workspaces.  Counts against the HBM budget. */
APGCU_API int apgcu_server_reserve(apgcu_server_t s, const apgcu_request_t* like, int count);
APGCU_API const char* apgcu_server_last_error(apgcu_server_t s);

/* Right-image winner-take-all over a caller's cost volume, allocating nothing.
 *
 * No counterpart in the reference: it exposes as one call the right-image WTA that the reference
 * runs inside its pipeline (wta_right_from_left_volume, src/pipeline.cpp:24-84, internal) and that
 * the engine fuses into its cost kernel.  It is for callers that must not allocate device memory
 * on their hot path -- a host that runs under a fixed device-memory budget it accounts itself, or
 * whose allocator would synchronise the device -- and so cannot hold an engine workspace.  The
 * call makes no cudaMalloc, cudaFree or other allocating call: its per-pixel keys live in a
 * static device array of APGCU_NOALLOC_MAX_PIXELS u32 (8 MiB), cleared by the call itself.
 *
 * d_cost: u16 volume on the current device, C(x, y, d) at d_cost[(y*width + x)*pitch + d -
 * min_disparity] for d in [min_disparity, min_disparity + num_disparities), 0xFFFF = invalid.
 * d_disparity_right: float width*height on the same device; -1 where no valid disparity.
 * subpixel: nonzero applies the legacy parabola.  stream: a cudaStream_t, or NULL.
 * Enqueued only; synchronise the stream before reading the result.
 *
 * The first call on each device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current, and under CUDA's default lazy module loading that first call also loads the
 * library's noalloc module into the context, which creates the 8 MiB array and the kernels there.
 * So make one warm-up call per device at start-up, before any stream capture and before the hot
 * path begins; with eager loading (CUDA_MODULE_LOADING=EAGER) every context that loads the library
 * holds the array from the start.  The address is remembered per device together with the context
 * it belongs to and looked up again if the device's current context changes.  All calls on one
 * device share the array and it keeps the last call's keys (each call clears the pixels it uses):
 * calls that overlap in time on one device race and must be serialised by the caller.
 *
 * Returns APG_STATUS_OK; APG_STATUS_EMPTY_INPUT for a NULL pointer or a non-positive size;
 * APG_STATUS_INVALID_DISPARITY_RANGE for num_disparities outside [1,
 * APGCU_NOALLOC_MAX_DISPARITIES] or |min_disparity| > APGCU_NOALLOC_MAX_ABS_DISPARITY;
 * APG_STATUS_SIZE_MISMATCH for pitch < num_disparities;
 * APG_STATUS_RESOURCE_LIMIT_EXCEEDED when width*height > APGCU_NOALLOC_MAX_PIXELS or height > 65535
 * (nothing is launched); APG_STATUS_UNSUPPORTED_BACKEND / APG_STATUS_INTERNAL_ERROR for CUDA failures. */
#define APGCU_NOALLOC_MAX_PIXELS (1 << 21)
#define APGCU_NOALLOC_MAX_DISPARITIES 1024
#define APGCU_NOALLOC_MAX_ABS_DISPARITY (1 << 20)
APGCU_API int apgcu_right_wta_noalloc(const uint16_t* d_cost, int width, int height, int min_disparity,
                                      int num_disparities, int pitch, int subpixel, float* d_disparity_right,
                                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* APG_SGM_CUDA_H */

// Device pipeline for one stereo pair at a time: workspace arena, stage orchestration, timing.
//
// Mirrors StereoMatcher::compute_impl (src/pipeline.cpp:435-719): aux -> search range / prior ->
// cost (+cross-H, +right argmin) -> right-WTA -> cross-V -> SGM sweeps (+WTA) -> confidence ->
// refine -> LR -> fill -> median.  Everything between the input upload and the output download
// runs on one CUDA stream with no host synchronisation, except the HighQuality refiner, which
// needs one device->host read of the per-pass draw count (the draws come from the C++ standard
// library's mt19937 / uniform_int_distribution, exactly like the reference).
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/apg_sgm/pipeline_config.h"
#include "kernels.h"

namespace apgcu {

enum Status : int {
    kOk = 0, kEmptyInput = 1, kSizeMismatch = 2, kInvalidDisparityRange = 3, kInvalidConfig = 4,
    kUnsupportedBackend = 5, kResourceLimitExceeded = 6, kAllocationFailure = 7, kInternalError = 8
};

// Layout request bit beside the debug flags: Fast census-only sweeps recompute their costs.
constexpr int kLayoutFastFused = 1 << 16;
constexpr int kLayoutCost16 = 1 << 17;  // keep a Fast volume at two bytes per voxel
constexpr int kLayoutCost8 = 1 << 18;   // one byte per voxel at a padded range of 128 too

// Frame-size-dependent layout of the device arena.
struct Layout {
    int w = 0, h = 0, ch = 0, D = 0, Dp = 0;
    bool fused_fast = false;  // Fast path: costs recomputed inside the SGM sweeps, no volume
    bool cross = false;
    bool raw_cost = false;    // debug: materialise the raw volume
    bool cost8 = false;       // Fast path: the volume the sweeps read holds one byte per voxel (0xFF invalid)
    size_t total = 0;
    // offsets
    size_t in_left, in_right;
    size_t lgray, lgx, lgy, rgray, rgx, rgy;
    size_t cl, cr;
    size_t rmin, rmax, rkey;
    size_t disp_right, disp_wta, best, second, confidence, disp_ref, disp_lr, disp_fill, disp_out, d_prior;
    size_t reliable, reason_conf, reason;
    size_t volA, volB, volRaw;
    size_t sbuf[7] = {};
    int nsbuf = 0;
    size_t lut, qlut, magic;
    // HighQuality prior / refine
    size_t pr_cand, pr_ncand, pr_taken, pr_grid, pr_maps, pr_scratch, pr_count;
    size_t rf_prefix, rf_scan_tmp, rf_state, rf_pack, rf_steps;  // refine: draw-index prefix, scan scratch,
                                                                   // pass state, packed images, pixel records
    size_t stats = 0;  // u64 frame counters (launch_frame_stats) + prior support count
    // hierarchical search range: half-size grays of both images, telemetry counters (4 x u64)
    size_t hc_left = 0, hc_right = 0, hstats = 0;
    size_t tel = 0;  // scope telemetry of the frame: apg_subpixel_telemetry_t then apg_inpaint_telemetry_t
    size_t rf_scan_tmp_bytes = 0;
    int n_cells = 0, gw = 0, gh = 0, max_cand = 0;
};

// The experimental scopes of the calling thread (ExperimentalSubpixelScope,
// src/subpixel_estimator.cpp:7-57; ExperimentalInpaintScope, src/postprocess.cpp:42-53): the
// sub-pixel method (0 Legacy, 1 CurvGate, 2 ConfGate, 3 Stabilized) with its parameter, and the
// inpaint method (0 Legacy, 1 ShadowReclass) with its gap.  An engine reads them once per frame.
struct ExperimentalScope {
    int sp_method = 0;
    float sp_param = 0.0f;
    int ip_method = 0;
    int ip_gap = 32;
    int sp_telem = 0, ip_telem = 0;  // collect the scopes' telemetry
};
ExperimentalScope& experimental_scope();
inline bool same_scope(const ExperimentalScope& a, const ExperimentalScope& b) {
    return a.sp_method == b.sp_method && a.sp_param == b.sp_param && a.ip_method == b.ip_method &&
           a.ip_gap == b.ip_gap && a.sp_telem == b.sp_telem && a.ip_telem == b.ip_telem;
}
// The calling thread's accumulated scope telemetry (the reference's thread-local
// ExperimentalSubpixelScope / ExperimentalInpaintScope::current_telemetry()).
struct TelemetryTotals {
    apg_subpixel_telemetry_t sp{};
    apg_inpaint_telemetry_t ip{};
};
TelemetryTotals& telemetry_totals();

// Refine pass state (u32 words at Layout::rf_state): pass start positions, error flag, progress.
constexpr int kRefineMaxIter = 63;
constexpr int kRefineErrWord = 64;
constexpr int kRefineProgWord = 80;

// Per-engine device copies of the refiner's draw tables (see refine.cu).
struct RefineTables {
    void* dev = nullptr;
    size_t bytes = 0;
    int iters = 0, n_built = 0, radius_built = 0;
    int16_t* value[kRefineMaxIter] = {};
    unsigned* rejected[kRefineMaxIter] = {};
    int nrej[kRefineMaxIter] = {};
    int build(int iterations, int base_radius, int n);  // 0 on success
    void release();
};
int refine_band_count(int h);
// Refiner tuning (Engine::set_refine_*): the poll budget of each cross-band wait before it gives up
// and flags the frame (0: the default, about a second) and the right-image window form (0: shared
// memory where every band fits on the device at once, 1: always the L1-read form).
struct RefineTuning {
    int spin_limit = 0;
    int window = 0;
};

class Engine {
public:
    Engine(const apg_pipeline_config_t& cfg, int device, cudaStream_t stream);
    ~Engine();

    // outputs_pinned: the four host outputs are page-locked, so the device copies land in them
    // directly (otherwise they go through the engine's pinned staging)
    int process_host(const uint8_t* left, const uint8_t* right, int w, int h, int stride, int ch,
                     float* disp, float* conf, uint8_t* reason, uint8_t* reliable, bool outputs_pinned = false);
    // Batch hooks.  upload: copy a pair (host or device memory) into the engine's input buffers on
    // stream s; enqueue_pre / enqueue_post: the phases before and after the SGM on the engine's own
    // stream; sgm_launch: the SGM arguments and path-sum buffers (returns their count); download:
    // outputs to device pointers, or to the pinned staging that finish_download copies out.
    int upload(const uint8_t* left, const uint8_t* right, int w, int h, int stride, int ch, bool device,
               cudaStream_t s);
    int enqueue_pre();
    int sgm_launch(SgmLaunch* out, uint32_t** sbufs) const;
    int enqueue_post();
    int enqueue_sgm() { return run_sgm(); }
    int download(float* disp, float* conf, uint8_t* reason, uint8_t* reliable, bool device, cudaStream_t s);
    void finish_download(float* disp, float* conf, uint8_t* reason, uint8_t* reliable) const;
    bool refine_enabled() const { return cfg_.refine_enable && cfg_.refine_iterations > 0; }
    // Frame counters of the last pair: valid, reliable, lr_fail, refine_changed, sum of range
    // widths, prior support count.  Waits for the engine stream.
    int frame_counts(unsigned long long* out6);
    int process_device(const uint8_t* dl, const uint8_t* dr, int w, int h, int stride, int ch,
                       float* d_disp, float* d_conf, uint8_t* d_reason, uint8_t* d_reliable);
    int sync();
    int dump(int what, void* dst, size_t bytes);
    void stage_times(double* ms11) const;
    size_t allocated_bytes() const {
        return arena_bytes_ + pinned_bytes_ + rtab_.bytes + (coarse_ ? coarse_->allocated_bytes() : 0);
    }
    // HierarchicalTelemetry of the last frame (src/hierarchical_stereo.hpp:36-42) from the device
    // counters: avg_states_per_pixel, coarse_valid_ratio, fallback_pixel_ratio,
    // full_range_pixel_ratio, coarse pass device time (ms), 1 if the coarse pass ran.  Waits for
    // the engine stream.
    int hier_telemetry(double* out6);
    // The prior's selected supports of the last frame in the reference's order
    // (PipelineBuffers::supports, src/prior_estimator.cpp:112-165): x, y, disparity, confidence.
    // Waits for the engine stream; empty without a prior.
    struct SupportOut { int x, y; float d, conf; };
    int supports(std::vector<SupportOut>& out);
    void release();
    cudaStream_t stream() const { return stream_; }
    const std::string& last_error() const { return err_; }
    void set_debug(int f) { debug_ = f; }
    void set_sgm_lanes(int t) { sgm_lanes_ = t; }
    void set_sgm_split(int v) { sgm_split_ = v; }
    void set_cost8(int mode) { cost8_ = mode; }
    void set_fast_fused(bool on) { fast_fused_ = on; }
    void set_cost_tile(int t) { cost_tile_ = t; }
    void set_cost_kernel(int k) { cost_kernel_ = k; }
    // refiner waits: polls before a cross-band wait gives up (0: about a second); shared-memory
    // right-image window (0: where it fits, 1: never, the L1 form)
    void set_refine_spin_limit(int n) { refine_.spin_limit = n; }
    void set_refine_window(int mode) { refine_.window = mode; }
    // the last sweep in this many row bands, each band's rows post-processed and copied to the
    // outputs while the next band runs (0: kBands where the path allows it, 1: never)
    void set_host_bands(int n) { host_bands_ = n; }
    // device-output frames (process_device) in that many bands: 0 = never (default)
    void set_device_bands(int n) { device_bands_ = n; }
    static constexpr int kBands = 6;
    static constexpr int kMaxBands = 16;
    // takes the calling thread's experimental scopes now (run_pre does so for every frame; the
    // batched form needs them before it builds SGM plans from sgm_launch)
    void capture_scope() { scope_ = experimental_scope(); }
    // adds the last frame's scope telemetry (and the coarse pass's) to the calling thread's totals
    // once the frame has completed; process_host and sync() call it
    int collect_telemetry();
    int debug() const { return debug_; }
    const apg_pipeline_config_t& config() const { return cfg_; }
    int device() const { return device_; }

    // Validation shared with the session layer (src/pipeline.cpp:171-232 + device limits).
    static int validate_config(const apg_pipeline_config_t& c, std::string& msg);
    static Layout make_layout(const apg_pipeline_config_t& c, int w, int h, int ch, int debug);
    // Device bytes for a W x H frame: the arena plus, in hierarchical mode, the half-size engine's.
    static size_t workspace_bytes(const apg_pipeline_config_t& c, int w, int h, int ch, int debug);
    // The half-size pass's configuration (src/hierarchical_stereo.cpp:172-182).
    static apg_pipeline_config_t coarse_config(const apg_pipeline_config_t& c);
    // Hierarchical mode runs its coarse pass for frames of at least 32 x 32 pixels.
    static bool hier_runs(const apg_pipeline_config_t& c, int w, int h) {
        return c.hier_enable && w >= 32 && h >= 32;
    }

private:
    int prepare(int w, int h, int ch);
    int prepare_arena(int w, int h, int ch);
    int run(const uint8_t* dl, int lstride, const uint8_t* dr, int rstride, int ch, float* d_disp, float* d_conf,
            uint8_t* d_reason, uint8_t* d_reliable);
    // the three phases of run(): aux .. cross-V, the SGM sweeps + WTA, confidence .. frame counters
    int run_pre(const uint8_t* dl, int lstride, const uint8_t* dr, int rstride, int ch);
    int run_sgm();
    int run_post(float* d_disp, float* d_conf, uint8_t* d_reason, uint8_t* d_reliable);
    // run_sgm + run_post with the last sweep in row bands (host_band_count() > 1): every map row
    // goes to the output pointers (host, or device when !to_host) on copy_stream_ as soon as it is
    // final; ev_copied_ follows the last copy
    int host_band_count(bool device = false) const;
    int run_banded(int nb, float* odisp, float* oconf, uint8_t* oreason, uint8_t* orel, bool to_host);
    int ensure_streams();  // copy_stream_, post_stream_ and their events, created on first use
    int run_prior();
    int run_hier();
    // per-pixel ranges: from the prior or from the hierarchical pass (every other frame has the
    // default range of each pixel); the prior does not run in hierarchical mode
    bool ranged() const { return cfg_.prior_enable || cfg_.hier_enable; }
    bool prior_runs() const { return cfg_.prior_enable && !cfg_.hier_enable; }
    int run_refine(float* work);
    int check_refine();  // after a synchronisation: the refine error flag of the last frame
    int fail(int code, const std::string& m) { err_ = m; return code; }
    int ensure_pinned(size_t need);
    int cuda_fail(cudaError_t e, const char* where);
    template <typename T> T* ptr(size_t off) const { return reinterpret_cast<T*>(arena_ + off); }
    CostCtx cost_ctx() const;
    bool range_planes_needed() const;
    unsigned long long default_range_width_sum() const;

    apg_pipeline_config_t cfg_;
    int device_ = 0;
    int debug_ = 0;
    int sgm_lanes_ = 0;
    int sgm_split_ = 0;  // last sweep over two warps per chain: 0 auto, 1 never, 2 always
    int cost8_ = 0;  // Fast volume at one byte per voxel: 0 = padded range 256, 1 = never, 2 = 128 and 256
    bool fast_fused_ = false;
    int cost_tile_ = 0;
    int cost_kernel_ = 0;  // 0: pixel-run cost kernel where it applies, 1: column-tile kernel
    int host_bands_ = 0;   // see set_host_bands
    int device_bands_ = 0;  // see set_device_bands
    RefineTuning refine_;
    cudaStream_t stream_ = nullptr;
    bool own_stream_ = false;
    unsigned char* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    Layout lay_;
    // host staging (pinned)
    unsigned char* pin_ = nullptr;
    size_t pinned_bytes_ = 0;
    bool direct_out_ = false;
    bool ranges_written_ = false;  // the last frame wrote the range planes (else: default ranges)  // the last download() wrote the caller's page-locked (or device) outputs
    std::vector<float> lut_host_;
    std::vector<uint16_t> qlut_host_;
    cudaEvent_t ev_[12] = {};
    bool have_times_ = false;
    // per-launch profile (APGCU_DEBUG_PROFILE): event after every launch, on the engine stream
    static constexpr int kMaxProf = 64;
    cudaEvent_t pev_[kMaxProf + 1] = {};
    const char* pname_[kMaxProf] = {};
    int nprof_ = 0;
    void prof_mark(const char* name);

public:
    int launch_profile(int max, const char** names, float* ms) const;

private:
    int support_count_ = 0;
    std::unique_ptr<Engine> coarse_;  // hierarchical mode: the half-size engine (same stream)
    ExperimentalScope scope_;         // the calling thread's experimental scopes, read per frame
    bool tel_pending_ = false;        // the last frame counted telemetry not yet collected
    bool skip_fill_ = false;          // coarse engine without coarse_fill_holes: no fill stage
    bool hier_ran_ = false;           // the last frame ran the coarse pass
    unsigned long long counts_[8] = {};  // frame counters copied with the host outputs
    const uint32_t* sgm_src_ = nullptr;  // volume the SGM sweeps read (set by run_pre)
    RefineTables rtab_;                   // refine draw tables (HighQuality)
    // host path: confidence / reliability (and reason, without refine) are final after the
    // confidence kernel; their device-to-host copies run on copy_stream_ while the rest finishes
    cudaStream_t copy_stream_ = nullptr;
    cudaStream_t side_stream_ = nullptr;  // the right-image WTA finalize, beside aggregation and SGM
    bool rwta_forked_ = false;            // the last frame finalized it there (join before confidence)
    cudaEvent_t ev_maps_ = nullptr, ev_copied_ = nullptr;
    // banded host path: the post-processing stream and the per-band events (sweep done, rows done)
    cudaStream_t post_stream_ = nullptr;
    // the sweep's bands run on a stream of the highest priority, so that the block scheduler
    // places their blocks before those of the post-processing kernels beside them
    cudaStream_t sweep_stream_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr;
    // host path with page-locked inputs: the right image goes up on copy_stream_ (ev_right_ after
    // it) while the left image's aux kernel runs; run_pre then waits for it before the right's
    cudaEvent_t ev_right_ = nullptr;
    bool right_on_copy_ = false;
    cudaEvent_t band_ev_[2 * kMaxBands] = {};
    float* early_conf_ = nullptr;
    uint8_t* early_reason_ = nullptr;
    uint8_t* early_rel_ = nullptr;
    bool early_issued_ = false, early_reason_done_ = false;
    int* refine_err_host_ = nullptr;      // pinned copy of the refine error flag
    bool refine_pending_ = false;
    bool counts_fresh_ = false;
    std::string err_;
};

// The tuning keys of apgcu_engine_set_tuning for engines and sessions; kInvalidConfig for an
// unknown key or a value out of range.  A null engine only validates the key and value.
int set_tuning(Engine* e, const char* key, int value);

// Process-wide launch counter (reported by bench.py as gpu_launches).
void count_launches(unsigned n);
unsigned long long launch_count();


// prior.cu / refine.cu
cudaError_t launch_prior(const apg_pipeline_config_t& cfg, const CostCtx& c, const Layout& L, unsigned char* arena,
                         cudaStream_t s, unsigned* launches);
cudaError_t launch_refine_count(const Layout& L, unsigned char* arena, const float* work, int fwd,
                                cudaStream_t s, unsigned* launches);
cudaError_t launch_refine_pack(const CostCtx& c, const Layout& L, unsigned char* arena, cudaStream_t s,
                               unsigned* launches);
size_t refine_pack_bytes(int n, bool c64);
size_t refine_steps_bytes(int n);
cudaError_t launch_refine_pass(const CostCtx& c, const Layout& L, unsigned char* arena, const RefineTables& tab,
                               int it, float* work, const RefineTuning& tune, cudaStream_t s, unsigned* launches);
size_t refine_scan_temp_bytes(int n);

}  // namespace apgcu

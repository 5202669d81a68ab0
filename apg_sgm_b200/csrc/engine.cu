// Device pipeline orchestration (see engine.h).
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

namespace apgcu {

namespace {
std::atomic<unsigned long long> g_launches{0};

inline size_t a256(size_t v) { return (v + 255) & ~size_t(255); }

// Default per-pixel search range (PriorEstimator::estimate, src/prior_estimator.cpp:414-424 with
// SearchRange::set_pixel clamping, include/apg_sgm/search_range.hpp:29-35).
__global__ void default_range_kernel(int w, int h, int d0, int dmax, int16_t* rmin, int16_t* rmax) {
    const int n = w * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int x = i % w;
        int lo = d0, hi = min(dmax, x + 1);
        lo = max(lo, d0);
        hi = min(hi, dmax);
        if (hi < lo) hi = lo;
        rmin[i] = (int16_t)lo;
        rmax[i] = (int16_t)hi;
    }
}

__global__ void fill_u32_kernel(uint32_t* p, size_t n, uint32_t v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

bool u16_path_ok(const apg_pipeline_config_t& c) {
    // can_use_u16_sgm_accumulator (include/apg_sgm/sgm_optimizer.hpp:9-18) plus headroom for
    // the saturating path arithmetic: m' + P2 and every path value stay below 0xFFFF.
    const long long p2max = std::max<long long>(c.P2_base, (long long)c.P1 + 1);
    const long long path_max = (long long)c.cost_max + p2max;
    const int npath = c.paths == 8 ? 8 : 4;
    // Path values use 0x7FFF as "invalid": valid sums must stay below it and an invalid value
    // plus P2 and P1 must not wrap 16 bits.
    if ((long long)npath * path_max >= 0x7FFF) return false;
    if (p2max + c.P1 >= 0x7FFF) return false;
    if (!c.piecewise_p2 && c.adaptive_penalties && c.p2_alpha < 0.f) return false;
    return true;
}
}  // namespace

void count_launches(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

ExperimentalScope& experimental_scope() {
    static thread_local ExperimentalScope s;
    return s;
}

TelemetryTotals& telemetry_totals() {
    static thread_local TelemetryTotals t;
    return t;
}
unsigned long long launch_count() { return g_launches.load(); }

cudaError_t launch_default_range(int w, int h, int d0, int dmax, int16_t* rmin, int16_t* rmax, cudaStream_t s) {
    const int n = w * h;
    const int blocks = std::min((n + 255) / 256, 148 * 8);
    default_range_kernel<<<blocks, 256, 0, s>>>(w, h, d0, dmax, rmin, rmax);
    return cudaGetLastError();
}

int Engine::validate_config(const apg_pipeline_config_t& c, std::string& msg) {
    // validate_config, src/pipeline.cpp:171-213
    if (c.max_disparity <= c.min_disparity) {
        msg = "max_disparity must be strictly greater than min_disparity";
        return kInvalidDisparityRange;
    }
    if (c.cost_max < 0 || c.cost_max > 65535) {
        msg = "cost_max out of valid uint16 representation range [0, 65535]";
        return kInvalidConfig;
    }
    if (c.P1 < 0) { msg = "SGM P1 penalty must be non-negative"; return kInvalidConfig; }
    if (c.P2_base <= c.P1) { msg = "SGM P2_base must be strictly greater than P1"; return kInvalidConfig; }
    if (c.grad_t1 < 0 || c.grad_t2 < c.grad_t1) {
        msg = "SGM gradient thresholds must satisfy 0 <= grad_t1 <= grad_t2";
        return kInvalidConfig;
    }
    if (c.prior_enable && c.prior_search_radius < 0) { msg = "prior search_radius must be non-negative"; return kInvalidConfig; }
    if (c.refine_enable && c.refine_iterations < 0) { msg = "refine iterations must be non-negative"; return kInvalidConfig; }
    if (c.hier_enable) {
        // src/pipeline.cpp:193-210
        if (c.volume_backend == 1) { msg = "hierarchical mode requires Auto or Packed backend"; return kInvalidConfig; }
        if (c.hier_radius <= 0) { msg = "hierarchical radius must be strictly positive"; return kInvalidConfig; }
        if (c.hier_scale != 2) { msg = "hierarchical scale currently supports only 2"; return kInvalidConfig; }
        if (c.hier_adaptive_radius) {
            if (c.hier_expanded_radius < c.hier_radius) {
                msg = "hierarchical expanded_radius cannot be less than radius";
                return kInvalidConfig;
            }
            if (!(c.hier_confidence_threshold >= 0.f && c.hier_confidence_threshold <= 1.f)) {
                msg = "hierarchical confidence_threshold must be between 0.0 and 1.0";
                return kInvalidConfig;
            }
        }
    }
    if (c.refine_enable && c.refine_iterations > kRefineMaxIter) {
        msg = "refine iterations above 63 are not supported by the CUDA backend";
        return kUnsupportedBackend;
    }
    // Limits of the device kernels (documented in the library header).
    const int D = c.max_disparity - c.min_disparity;
    if (D > 512) { msg = "disparity range above 512 is not supported by the CUDA backend"; return kUnsupportedBackend; }
    if (c.min_disparity < -32768 || c.max_disparity > 32767) { msg = "disparity bounds must fit int16"; return kInvalidConfig; }
    if (!u16_path_ok(c)) {
        msg = "SGM penalties/cost_max exceed the 16-bit path range of the CUDA backend";
        return kUnsupportedBackend;
    }
    if (c.agg_enable) {
        const int lmax = std::max(1, c.max_arm_length);
        if (lmax > 127 || (long long)(2 * lmax + 1) * c.cost_max >= 65536) {
            msg = "cross arm length x cost_max exceeds the 16-bit window range of the CUDA backend";
            return kUnsupportedBackend;
        }
        if (cost_kernel_smem_bytes(D, round_up(D, 64), lmax, true, c.census_type == APG_CENSUS_9X7) > 227 * 1024 ||
            cross_v_smem_bytes(round_up(D, 64), lmax) > 227 * 1024) {
            msg = "cross arm length too large for on-chip staging";
            return kUnsupportedBackend;
        }
    }
    if (c.median_radius > 15) { msg = "median radius above 15 is not supported"; return kUnsupportedBackend; }
    if (c.hier_enable) {
        // the half-size pass runs on the same kernels: its configuration must fit them too
        std::string m;
        const int rc = validate_config(coarse_config(c), m);
        if (rc != kOk) { msg = "hierarchical coarse pass: " + m; return rc; }
    }
    return kOk;
}

apg_pipeline_config_t Engine::coarse_config(const apg_pipeline_config_t& c) {
    apg_pipeline_config_t k = c;
    k.min_disparity = std::max(0, c.min_disparity / 2);
    k.max_disparity = std::max(k.min_disparity + 1, (c.max_disparity + 1) / 2);
    k.prior_enable = 0;
    k.refine_enable = 0;
    k.agg_enable = c.hier_coarse_cross_agg;
    k.volume_backend = 2;
    k.subpixel = 1;
    k.lr_check = 1;
    k.median_radius = 1;
    k.max_fill_gap = c.hier_coarse_fill_holes ? 16 : 0;
    k.hier_enable = 0;
    return k;
}

size_t Engine::workspace_bytes(const apg_pipeline_config_t& c, int w, int h, int ch, int debug) {
    size_t t = make_layout(c, w, h, ch, debug).total;
    if (hier_runs(c, w, h)) t += make_layout(coarse_config(c), w / 2, h / 2, 1, 0).total;
    return t;
}

// The largest census-only quantised cost (the table of the constructor, same float steps).
static int max_census_cost(const apg_pipeline_config_t& c) {
    const float lc = std::max(c.lambda_census, 1e-3f);
    const float norm = 1.f + (c.use_ad ? c.eta_ad : 0.f) + (c.use_grad ? c.mu_grad : 0.f);
    const float scale = static_cast<float>(c.cost_max) / std::max(norm, 1e-6f);
    int m = 0;
    for (int i = 0; i <= 64; ++i) {
        const int q = static_cast<int>((1.f - std::exp(-static_cast<float>(i) / lc)) * scale + 0.5f);
        m = std::max(m, std::min(std::max(q, 0), c.cost_max));
    }
    return m;
}

// An upper bound of every quantised cost with AD and gradient terms: the cost kernels add the
// census, AD and gradient tables (each non-decreasing in its index) at most at their largest
// entries, then scale and round; computed in double with a margin over the kernels' float steps.
static int max_full_cost(const apg_pipeline_config_t& c) {
    if (!c.use_ad && !c.use_grad) return max_census_cost(c);
    if (c.eta_ad < 0.f || c.mu_grad < 0.f) return c.cost_max;
    const double lc = std::max(c.lambda_census, 1e-3f), la = std::max(c.lambda_ad, 1e-3f),
                 lg = std::max(c.lambda_grad, 1e-3f);
    double v = 1.0 - std::exp(-64.0 / lc);
    if (c.use_ad) v += c.eta_ad * (1.0 - std::exp(-255.0 / la));
    if (c.use_grad) v += c.mu_grad * (1.0 - std::exp(-510.0 / lg));
    const float norm = 1.f + (c.use_ad ? c.eta_ad : 0.f) + (c.use_grad ? c.mu_grad : 0.f);
    const double scale = (double)c.cost_max / std::max(norm, 1e-6f);
    return std::min((int)(v * scale + 0.5 + 1e-3), c.cost_max);
}

Layout Engine::make_layout(const apg_pipeline_config_t& c, int w, int h, int ch, int debug) {
    Layout L;
    L.w = w; L.h = h; L.ch = ch;
    L.D = c.max_disparity - c.min_disparity;
    L.Dp = round_up(L.D, 64);
    L.cross = c.agg_enable != 0;
    // Fast census-only path: by default the raw volume is stored once and the sweeps read it (the
    // volume-fed sweeps are the faster ones); on request the sweeps recompute the census costs
    // instead and no volume is allocated (kLayoutFastFused)
    L.fused_fast = !L.cross && c.census_type == APG_CENSUS_SYMMETRIC_9X7 && !c.use_ad && !c.use_grad &&
                   !c.prior_enable && !c.hier_enable && (debug & kLayoutFastFused) && !(debug & 4);
    L.raw_cost = (debug & 1) != 0;
    // Fast census-only path with its volume stored: one byte per voxel when every quantised cost is
    // below 255, so 0xFF marks the invalid voxels exactly (the sweeps' 32-lane form, the pixel-run
    // cost kernel).  At a padded range of 256 it is the default: one B200, Fast 1920x1080 D256, 2.64
    // vs 2.83 ms per frame (first phase 0.96 vs 1.20 ms).  At 128 only on request (kLayoutCost8):
    // Fast 1280x720 D128 0.757 vs 0.749 ms, the first phase's chains there wait on the latency of
    // each step (widening the bytes) more than on the volume's bytes.  kLayoutCost16 keeps two bytes.
    // The same holds for the aggregated volume of Balanced / HighQuality (one aggregation pass),
    // written by the vertical aggregation: aggregated costs are window averages of quantised costs,
    // so below 255 when every quantised cost is.
    const bool fast8 = !L.cross && !L.fused_fast && c.census_type == APG_CENSUS_SYMMETRIC_9X7 && !c.use_ad &&
                       !c.use_grad && !c.prior_enable && !c.hier_enable && max_census_cost(c) < 255;
    const bool cross8 = L.cross && c.agg_iterations <= 1 && max_full_cost(c) < 255;
    L.cost8 = (fast8 || cross8) && (L.Dp == 256 || (L.Dp == 128 && (debug & kLayoutCost8))) &&
              !(debug & kLayoutCost16);
    const size_t n = (size_t)w * h;
    const size_t csz = c.census_type == APG_CENSUS_9X7 ? 8 : 4;
    const size_t vol = n * (size_t)L.Dp * 2;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t r = o; o = a256(o + bytes); return r; };
    L.in_left = take(n * ch);
    L.in_right = take(n * ch);
    L.lgray = take(n); L.lgx = take(n); L.lgy = take(n);
    L.rgray = take(n); L.rgx = take(n); L.rgy = take(n);
    L.cl = take(n * csz); L.cr = take(n * csz);
    L.rmin = take(n * 2); L.rmax = take(n * 2);
    L.rkey = take(n * 4);
    L.disp_right = take(n * 4); L.disp_wta = take(n * 4); L.best = take(n * 4); L.second = take(n * 4);
    L.confidence = take(n * 4); L.disp_ref = take(n * 4); L.disp_lr = take(n * 4); L.disp_fill = take(n * 4);
    L.disp_out = take(n * 4); L.d_prior = take(n * 4);
    L.reliable = take(n); L.reason_conf = take(n); L.reason = take(n);
    // volA: cross-H output T (Balanced/HQ), raw cost (Fast without fusion) or the first path-sum
    // buffer (fused Fast); volB: aggregated cost.  The first SGM phase writes one buffer per
    // direction (3 for Path4, 7 for Path8); buffer 0 reuses volA whenever volA is dead by then.
    L.volA = take(L.cost8 && !L.cross ? vol / 2 : vol);
    L.volB = L.cross ? take(L.cost8 ? vol / 2 : vol) : 0;
    L.nsbuf = (c.paths == 8 ? 8 : 4) - 1;
    for (int i = 0; i < L.nsbuf; ++i) L.sbuf[i] = (i == 0 && (L.cross || L.fused_fast)) ? L.volA : take(vol);
    L.volRaw = L.raw_cost ? take(vol) : 0;
    L.tel = take(sizeof(apg_subpixel_telemetry_t) + sizeof(apg_inpaint_telemetry_t));
    L.lut = take(kLutSize * 4);
    L.qlut = take(65 * 2);
    L.magic = take(256 * 4);
    L.stats = take(64);
    if (hier_runs(c, w, h)) {
        const size_t nc = (size_t)(w / 2) * (h / 2);
        L.hc_left = take(nc);
        L.hc_right = take(nc);
    }
    if (c.hier_enable) L.hstats = take(64);
    if (c.prior_enable && !c.hier_enable) {
        const int cell = 16;
        L.gw = (w + cell - 1) / cell; L.gh = (h + cell - 1) / cell; L.n_cells = L.gw * L.gh;
        const int hard_max = std::max(0, c.prior_max_supports);
        L.max_cand = std::max(8, (hard_max * 2 + L.n_cells - 1) / std::max(1, L.n_cells));
        L.pr_cand = take((size_t)L.n_cells * L.max_cand * 16);
        L.pr_ncand = take((size_t)L.n_cells * 4);
        L.pr_taken = take((size_t)L.n_cells * 4 * 4);
        L.pr_grid = take((size_t)L.n_cells * 4 * 10);
        L.pr_maps = take(n * 4 * 4);
        L.pr_scratch = take((size_t)L.n_cells * L.max_cand * 8 * 2);
        L.pr_count = take(64);
    }
    if (c.refine_enable) {
        L.rf_prefix = take(n * 4 + 4);
        L.rf_scan_tmp_bytes = refine_scan_temp_bytes((int)n);
        L.rf_scan_tmp = take(L.rf_scan_tmp_bytes);
        L.rf_state = take((size_t)(kRefineProgWord + refine_band_count(h)) * 4);
        L.rf_pack = take(refine_pack_bytes((int)n, c.census_type == APG_CENSUS_9X7));
        L.rf_steps = take(refine_steps_bytes((int)n));
    }
    L.total = o;
    return L;
}

Engine::Engine(const apg_pipeline_config_t& cfg, int device, cudaStream_t stream) : cfg_(cfg), device_(device) {
    cudaSetDevice(device_);
    if (stream) {
        stream_ = stream;
    } else {
        cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
        own_stream_ = true;
    }
    for (auto& e : ev_) cudaEventCreate(&e);
    for (auto& e : pev_) cudaEventCreate(&e);
    // the right-image WTA's finalize runs here beside the aggregation and the sweeps
    if (cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        side_stream_ = nullptr;
    }
    // Cost LUTs on the host with std::exp, exactly as DiscreteCostLut (src/discrete_cost_lut.hpp:20-35).
    lut_host_.assign(kLutSize, 0.f);
    const float lc = std::max(cfg_.lambda_census, 1e-3f);
    const float la = std::max(cfg_.lambda_ad, 1e-3f);
    const float lg = std::max(cfg_.lambda_grad, 1e-3f);
    for (int i = 0; i <= 64; ++i) lut_host_[kLutCensus + i] = 1.f - std::exp(-static_cast<float>(i) / lc);
    if (cfg_.use_ad)
        for (int i = 0; i < 256; ++i) lut_host_[kLutAd + i] = cfg_.eta_ad * (1.f - std::exp(-static_cast<float>(i) / la));
    if (cfg_.use_grad)
        for (int i = 0; i < 511; ++i) lut_host_[kLutGrad + i] = cfg_.mu_grad * (1.f - std::exp(-static_cast<float>(i) / lg));
    const float norm = 1.f + (cfg_.use_ad ? cfg_.eta_ad : 0.f) + (cfg_.use_grad ? cfg_.mu_grad : 0.f);
    const float scale = static_cast<float>(cfg_.cost_max) / std::max(norm, 1e-6f);
    qlut_host_.assign(65, 0);
    for (int i = 0; i <= 64; ++i) {
        const int q = static_cast<int>(lut_host_[kLutCensus + i] * scale + 0.5f);
        qlut_host_[i] = static_cast<uint16_t>(std::min(std::max(q, 0), cfg_.cost_max));
    }
}

Engine::~Engine() {
    release();
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
    if (post_stream_) cudaStreamDestroy(post_stream_);
    if (sweep_stream_) cudaStreamDestroy(sweep_stream_);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_right_) cudaEventDestroy(ev_right_);
    for (auto& ev : band_ev_) if (ev) cudaEventDestroy(ev);
    if (side_stream_) cudaStreamDestroy(side_stream_);
    if (ev_maps_) cudaEventDestroy(ev_maps_);
    if (ev_copied_) cudaEventDestroy(ev_copied_);
    if (refine_err_host_) cudaFreeHost(refine_err_host_);
    for (auto& e : ev_) if (e) cudaEventDestroy(e);
    for (auto& e : pev_) if (e) cudaEventDestroy(e);
    if (own_stream_ && stream_) cudaStreamDestroy(stream_);
}

void Engine::release() {
    if (arena_) {
        cudaStreamSynchronize(stream_);
        cudaFree(arena_);
        arena_ = nullptr;
        arena_bytes_ = 0;
    }
    if (pin_) {
        cudaFreeHost(pin_);
        pin_ = nullptr;
        pinned_bytes_ = 0;
    }
    rtab_.release();
    coarse_.reset();
    lay_ = Layout();
}

int Engine::cuda_fail(cudaError_t e, const char* where) {
    err_ = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? kAllocationFailure : kInternalError;
}

// The per-pixel range planes are read by the prior and the refiner, the stage dumps, the general
// vertical aggregation (negative minimum disparity or more than 256 padded disparities) and the
// aggregation iterations after the first.  Every other consumer -- the cost kernels, the
// right-image sub-pixel step and the frame counters -- uses the default range
// [d0, max(min(dmax, x + 1), d0)) in closed form, so without those readers the planes are not
// written at all.
bool Engine::range_planes_needed() const {
    // the stage-dump debug flags keep every intermediate; the launch profile alone changes no work
    if (ranged() || cfg_.refine_enable || (debug_ & ~8)) return true;
    return cfg_.agg_enable && (cfg_.agg_iterations > 1 || cfg_.min_disparity < 0 || lay_.Dp > 256);
}

// Sum over the frame of the default range widths max(min(dmax, x + 1) - d0, 0)
// (PipelineStats' search-width total for frames without a prior).
unsigned long long Engine::default_range_width_sum() const {
    unsigned long long row = 0;
    for (int x = 0; x < lay_.w; ++x) {
        const int wd = std::min(cfg_.max_disparity, x + 1) - cfg_.min_disparity;
        row += wd > 0 ? (unsigned long long)wd : 0ull;
    }
    return row * (unsigned long long)lay_.h;
}

CostCtx Engine::cost_ctx() const {
    CostCtx c;
    c.w = lay_.w; c.h = lay_.h; c.d0 = cfg_.min_disparity; c.D = lay_.D; c.Dp = lay_.Dp;
    c.census64 = cfg_.census_type == APG_CENSUS_9X7;
    c.use_ad = cfg_.use_ad; c.use_grad = cfg_.use_grad; c.cost_max = cfg_.cost_max;
    const float norm = 1.f + (cfg_.use_ad ? cfg_.eta_ad : 0.f) + (cfg_.use_grad ? cfg_.mu_grad : 0.f);
    c.scale = static_cast<float>(cfg_.cost_max) / std::max(norm, 1e-6f);
    c.lut = ptr<float>(lay_.lut);
    c.qlut = ptr<uint16_t>(lay_.qlut);
    c.lgray = ptr<uint8_t>(lay_.lgray); c.lgx = ptr<uint8_t>(lay_.lgx); c.lgy = ptr<uint8_t>(lay_.lgy);
    c.rgray = ptr<uint8_t>(lay_.rgray); c.rgx = ptr<uint8_t>(lay_.rgx); c.rgy = ptr<uint8_t>(lay_.rgy);
    c.cl = ptr<uint32_t>(lay_.cl); c.cr = ptr<uint32_t>(lay_.cr);
    c.cl64 = ptr<unsigned long long>(lay_.cl); c.cr64 = ptr<unsigned long long>(lay_.cr);
    c.rmin = ptr<int16_t>(lay_.rmin); c.rmax = ptr<int16_t>(lay_.rmax);
    c.prior_ranges = ranged() ? 1 : 0;
    c.sp_method = scope_.sp_method;
    c.sp_param = scope_.sp_param;
    c.tile = cost_tile_;
    c.kernel = cost_kernel_;
    return c;
}

int Engine::prepare(int w, int h, int ch) {
    const int rc = prepare_arena(w, h, ch);
    if (rc != kOk || !hier_runs(cfg_, w, h)) return rc;
    // hierarchical mode: the half-size engine enqueues on this engine's stream
    if (!coarse_) {
        coarse_ = std::make_unique<Engine>(coarse_config(cfg_), device_, stream_);
        coarse_->skip_fill_ = !cfg_.hier_coarse_fill_holes;
    }
    coarse_->cost_kernel_ = cost_kernel_;
    const int r2 = coarse_->prepare(w / 2, h / 2, 1);
    if (r2 != kOk) return fail(r2, "hierarchical coarse pass: " + coarse_->last_error());
    return kOk;
}

int Engine::prepare_arena(int w, int h, int ch) {
    // the byte volume needs 32-lane sweeps, and in Fast mode the pixel-run cost kernel (which
    // writes it; the vertical aggregation writes it otherwise)
    const bool cost16 =
        cost8_ == 1 || (!cfg_.agg_enable && cost_kernel_ == 1) || (sgm_lanes_ != 0 && sgm_lanes_ != 32);
    const Layout L = make_layout(cfg_, w, h, ch,
                                 debug_ | (fast_fused_ ? kLayoutFastFused : 0) | (cost16 ? kLayoutCost16 : 0) |
                                     (cost8_ == 2 ? kLayoutCost8 : 0));
    if (arena_ && arena_bytes_ >= L.total && lay_.w == w && lay_.h == h && lay_.ch == ch &&
        lay_.raw_cost == L.raw_cost && lay_.fused_fast == L.fused_fast && lay_.cost8 == L.cost8) {
        return kOk;
    }
    if (arena_ && arena_bytes_ >= L.total) {
        lay_ = L;  // capacity retained (BoundedReuse large -> small)
    } else {
        if (arena_) {
            cudaStreamSynchronize(stream_);
            cudaFree(arena_);
            arena_ = nullptr;
            arena_bytes_ = 0;
        }
        cudaError_t e = cudaMalloc(&arena_, L.total);
        if (e != cudaSuccess) {
            cudaGetLastError();
            arena_ = nullptr;
            return fail(kAllocationFailure, "device workspace allocation failed (" + std::to_string(L.total) + " bytes)");
        }
        arena_bytes_ = L.total;
        lay_ = L;
    }
    // constant tables
    cudaError_t e = cudaMemcpyAsync(ptr<float>(lay_.lut), lut_host_.data(), kLutSize * 4, cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ptr<uint16_t>(lay_.qlut), qlut_host_.data(), 65 * 2, cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess) {
        uint32_t magic[256];
        for (int d = 0; d < 256; ++d) magic[d] = div_magic(d);
        e = cudaMemcpyAsync(ptr<uint32_t>(lay_.magic), magic, sizeof(magic), cudaMemcpyHostToDevice, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);  // magic[] lives on the stack
    }
    if (e != cudaSuccess) return cuda_fail(e, "table upload");
    return kOk;
}

// True when p lies in page-locked host memory (cudaMallocHost / cudaHostAlloc / cudaHostRegister),
// which the copy engines read and write directly.
static bool host_pinned(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int Engine::process_host(const uint8_t* left, const uint8_t* right, int w, int h, int stride, int ch, float* disp,
                         float* conf, uint8_t* reason, uint8_t* reliable, bool outputs_pinned) {
    cudaSetDevice(device_);
    int rc = prepare(w, h, ch);
    if (rc) return rc;
    const size_t n = (size_t)w * h;
    const size_t in_bytes = n * ch;
    // page-locked caller buffers skip the staging copies: inputs go up by DMA from where they lie,
    // results come down into the caller's arrays
    const bool inputs_pinned = host_pinned(left) && host_pinned(right);
    if (!outputs_pinned)
        outputs_pinned = host_pinned(disp) && host_pinned(conf) && host_pinned(reason) && host_pinned(reliable);
    const size_t out_bytes = outputs_pinned ? 0 : n * 4 * 2 + n * 2;
    const size_t need = (inputs_pinned ? 0 : 2 * in_bytes) + out_bytes;
    if (need && (!pin_ || pinned_bytes_ < need)) {
        if (pin_) cudaFreeHost(pin_);
        pin_ = nullptr;
        pinned_bytes_ = 0;
        if (cudaMallocHost(&pin_, need) != cudaSuccess) {
            cudaGetLastError();
            return fail(kAllocationFailure, "pinned host staging allocation failed");
        }
        pinned_bytes_ = need;
    }
    unsigned char* pl = inputs_pinned ? nullptr : pin_;
    unsigned char* pr = inputs_pinned ? nullptr : pin_ + in_bytes;
    unsigned char* pout = inputs_pinned ? pin_ : pin_ + 2 * in_bytes;
    float* pdisp = outputs_pinned ? disp : reinterpret_cast<float*>(pout);
    float* pconf = outputs_pinned ? conf : pdisp + n;
    uint8_t* preason = outputs_pinned ? reason : reinterpret_cast<uint8_t*>(pconf + n);
    uint8_t* prel = outputs_pinned ? reliable : preason + n;
    const size_t row = (size_t)w * ch;
    rc = ensure_streams();
    if (rc) return rc;
    cudaError_t e;
    if (inputs_pinned) {
        e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_left), row, left, stride, row, h, cudaMemcpyHostToDevice, stream_);
        // the right image on the copy stream, beside the left image's aux kernel (the previous
        // frame's work on every stream ended before this call)
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_right), row, right, stride, row, h, cudaMemcpyHostToDevice,
                                  copy_stream_);
        if (e == cudaSuccess) e = cudaEventRecord(ev_right_, copy_stream_);
        right_on_copy_ = e == cudaSuccess && !(debug_ & 8);
        if (e == cudaSuccess && (debug_ & 8)) e = cudaStreamWaitEvent(stream_, ev_right_, 0);
    } else {
        // the left image goes up while the right one is staged
        for (int y = 0; y < h; ++y) std::memcpy(pl + y * row, left + (size_t)y * stride, row);
        e = cudaMemcpyAsync(ptr<uint8_t>(lay_.in_left), pl, in_bytes, cudaMemcpyHostToDevice, stream_);
        for (int y = 0; y < h; ++y) std::memcpy(pr + y * row, right + (size_t)y * stride, row);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ptr<uint8_t>(lay_.in_right), pr, in_bytes, cudaMemcpyHostToDevice, stream_);
    }
    if (e != cudaSuccess) return cuda_fail(e, "input upload");
    early_conf_ = pconf;
    early_rel_ = prel;
    early_reason_ = preason;
    early_issued_ = early_reason_done_ = false;
    // as run(), with the last sweep in row bands where the path allows it (run_banded issues every
    // output copy itself, the last one followed by ev_copied_)
    nprof_ = 0;
    if (debug_ & 8) cudaEventRecord(pev_[0], stream_);
    bool banded = false;
    rc = run_pre(ptr<uint8_t>(lay_.in_left), (int)row, ptr<uint8_t>(lay_.in_right), (int)row, ch);
    if (rc == kOk) {
        const int nb = host_band_count();
        banded = nb > 1;
        rc = banded ? run_banded(nb, pdisp, pconf, preason, prel, true) : run_sgm();
        if (rc == kOk && !banded) rc = run_post(nullptr, nullptr, nullptr, nullptr);
    }
    early_conf_ = nullptr;
    early_rel_ = nullptr;
    early_reason_ = nullptr;
    if (rc) {
        cudaStreamSynchronize(sweep_stream_);
        cudaStreamSynchronize(post_stream_);
        cudaStreamSynchronize(copy_stream_);
        return rc;
    }
    e = cudaSuccess;
    if (!banded) {
        if (pdisp) e = cudaMemcpyAsync(pdisp, ptr<float>(lay_.disp_out), n * 4, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess && pconf && !early_issued_)
            e = cudaMemcpyAsync(pconf, ptr<float>(lay_.confidence), n * 4, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess && preason && !early_reason_done_)
            e = cudaMemcpyAsync(preason, ptr<uint8_t>(lay_.reason), n, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess && prel && !early_issued_)
            e = cudaMemcpyAsync(prel, ptr<uint8_t>(lay_.reliable), n, cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess) e = cudaMemcpyAsync(counts_, ptr<unsigned long long>(lay_.stats), sizeof(counts_),
                                                  cudaMemcpyDeviceToHost, stream_);
    }
    if (e == cudaSuccess && (early_issued_ || banded)) e = cudaStreamWaitEvent(stream_, ev_copied_, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "output download");
    rc = check_refine();
    if (rc) return rc;
    rc = collect_telemetry();
    if (rc) return rc;
    counts_fresh_ = true;
    if (!outputs_pinned) {
        if (disp) std::memcpy(disp, pdisp, n * 4);
        if (conf) std::memcpy(conf, pconf, n * 4);
        if (reason) std::memcpy(reason, preason, n);
        if (reliable) std::memcpy(reliable, prel, n);
    }
    return kOk;
}

int Engine::frame_counts(unsigned long long* out6) {
    if (!arena_) return fail(kInternalError, "no frame has been processed");
    if (!counts_fresh_) {
        cudaSetDevice(device_);
        cudaError_t e = cudaMemcpyAsync(counts_, ptr<unsigned long long>(lay_.stats), sizeof(counts_),
                                        cudaMemcpyDeviceToHost, stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) return cuda_fail(e, "frame counters");
        counts_fresh_ = true;
    }
    std::memcpy(out6, counts_, 6 * sizeof(unsigned long long));
    return kOk;
}

int Engine::process_device(const uint8_t* dl, const uint8_t* dr, int w, int h, int stride, int ch, float* d_disp,
                           float* d_conf, uint8_t* d_reason, uint8_t* d_reliable) {
    cudaSetDevice(device_);
    int rc = prepare(w, h, ch);
    if (rc) return rc;
    counts_fresh_ = false;
    // one launch of the last sweep by default: with its post-processing in row bands beside it
    // (the host path's form) the post kernels took SM slots from the sweep's bands, and
    // device-only frames were slower (Fast 1280x720 D128 0.733 -> 0.790 ms, Balanced 1.090 ->
    // 1.170 ms); tuning device_bands asks for it
    if (device_bands_ > 1 && !debug_) {
        rc = ensure_streams();
        if (rc) return rc;
        nprof_ = 0;
        rc = run_pre(dl, stride, dr, stride, ch);
        if (rc) return rc;
        const int nb = host_band_count(true);
        if (nb > 1) {
            rc = run_banded(nb, d_disp, d_conf, d_reason, d_reliable, false);
            if (rc == kOk) {
                const cudaError_t e = cudaStreamWaitEvent(stream_, ev_copied_, 0);
                if (e != cudaSuccess) return cuda_fail(e, "join");
            }
            return rc;
        }
        rc = run_sgm();
        return rc == kOk ? run_post(d_disp, d_conf, d_reason, d_reliable) : rc;
    }
    return run(dl, stride, dr, stride, ch, d_disp, d_conf, d_reason, d_reliable);
}

int Engine::ensure_streams() {
    if (!copy_stream_) {
        if (cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_maps_, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev_copied_, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, "copy stream creation failed");
        }
    }
    if (!post_stream_) {
        int least = 0, greatest = 0;
        bool ok = cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess;
        ok = ok && cudaStreamCreateWithPriority(&sweep_stream_, cudaStreamNonBlocking, greatest) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&ev_right_, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaStreamCreateWithFlags(&post_stream_, cudaStreamNonBlocking) == cudaSuccess;
        for (auto& ev : band_ev_) ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return fail(kInternalError, "post stream creation failed");
        }
    }
    return kOk;
}

int Engine::sync() {
    cudaError_t e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
    const int rc = check_refine();
    return rc ? rc : collect_telemetry();
}

int Engine::collect_telemetry() {
    if (coarse_) {
        const int rc = coarse_->collect_telemetry();
        if (rc) return fail(rc, coarse_->last_error());
    }
    if (!tel_pending_) return kOk;
    tel_pending_ = false;
    apg_subpixel_telemetry_t sp;
    apg_inpaint_telemetry_t ip;
    cudaError_t e = cudaMemcpyAsync(&sp, arena_ + lay_.tel, sizeof(sp), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&ip, arena_ + lay_.tel + sizeof(sp), sizeof(ip), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "telemetry");
    TelemetryTotals& t = telemetry_totals();
    if (scope_.sp_telem) {
        t.sp.candidate_pixels += sp.candidate_pixels;
        t.sp.applied_pixels += sp.applied_pixels;
        t.sp.degenerate_count += sp.degenerate_count;
        t.sp.clamped_count += sp.clamped_count;
        t.sp.negative_curvature_count += sp.negative_curvature_count;
        t.sp.sum_abs_delta += sp.sum_abs_delta;
        for (int i = 0; i < 50; ++i) t.sp.delta_buckets[i] += sp.delta_buckets[i];
    }
    if (scope_.ip_telem) {
        t.ip.total_invalid_pixels += ip.total_invalid_pixels;
        t.ip.classified_occ_pixels += ip.classified_occ_pixels;
        t.ip.classified_mismatch_pixels += ip.classified_mismatch_pixels;
        t.ip.hit_max_gap_pixels += ip.hit_max_gap_pixels;
        t.ip.reclassified_shadow_pixels += ip.reclassified_shadow_pixels;
        for (int i = 0; i < 11; ++i) t.ip.route_counts[i] += ip.route_counts[i];
        t.ip.invalid_runs_count += ip.invalid_runs_count;
        t.ip.invalid_runs_truncated += ip.invalid_runs_truncated;
        for (int i = 0; i < 10; ++i) t.ip.run_length_buckets[i] += ip.run_length_buckets[i];
    }
    return kOk;
}

#define RUN(expr, what)                                  \
    do {                                                 \
        e = (expr);                                      \
        if (e != cudaSuccess) return cuda_fail(e, what); \
        ++launches;                                      \
        if (prof) prof_mark(what);                       \
    } while (0)
#define RUNC(expr, what)                                 \
    do {                                                 \
        e = (expr);                                      \
        if (e != cudaSuccess) return cuda_fail(e, what); \
        if (prof) prof_mark("copy");                     \
    } while (0)

int Engine::run(const uint8_t* dl, int lstride, const uint8_t* dr, int rstride, int ch, float* d_disp, float* d_conf,
                uint8_t* d_reason, uint8_t* d_reliable) {
    nprof_ = 0;
    if (debug_ & 8) cudaEventRecord(pev_[0], stream_);
    int rc = run_pre(dl, lstride, dr, rstride, ch);
    if (rc == kOk) rc = run_sgm();
    if (rc == kOk) rc = run_post(d_disp, d_conf, d_reason, d_reliable);
    return rc;
}

int Engine::run_pre(const uint8_t* dl, int lstride, const uint8_t* dr, int rstride, int ch) {
    const Layout& L = lay_;
    const int w = L.w, h = L.h, D = L.D, Dp = L.Dp, d0 = cfg_.min_disparity;
    const size_t n = (size_t)w * h;
    cudaStream_t s = stream_;
    unsigned launches = 0;
    cudaError_t e = cudaSuccess;
    const bool prof = (debug_ & 8) != 0;
    (void)D; (void)Dp; (void)d0; (void)n; (void)w; (void)h;
    const int c64 = cfg_.census_type == APG_CENSUS_9X7;
    scope_ = experimental_scope();
    cudaEventRecord(ev_[0], s);
    if (scope_.sp_telem || scope_.ip_telem) {
        RUNC(cudaMemsetAsync(arena_ + L.tel, 0, sizeof(apg_subpixel_telemetry_t) + sizeof(apg_inpaint_telemetry_t), s),
             "telemetry init");
        tel_pending_ = true;
    }
    {
        const AuxImage li{dl, lstride, ptr<uint8_t>(L.lgray), ptr<uint8_t>(L.lgx), ptr<uint8_t>(L.lgy),
                          ptr<uint32_t>(L.cl), ptr<unsigned long long>(L.cl)};
        const AuxImage ri{dr, rstride, ptr<uint8_t>(L.rgray), ptr<uint8_t>(L.rgx), ptr<uint8_t>(L.rgy),
                          ptr<uint32_t>(L.cr), ptr<unsigned long long>(L.cr)};
        if (right_on_copy_) {
            right_on_copy_ = false;
            RUN(launch_aux_one(li, ch, w, h, c64, s), "aux");
            RUNC(cudaStreamWaitEvent(s, ev_right_, 0), "right image");
            RUN(launch_aux_one(ri, ch, w, h, c64, s), "aux");
        } else {
            RUN(launch_aux(li, ri, ch, w, h, c64, s), "aux");
        }
    }
    cudaEventRecord(ev_[1], s);
    // search ranges: the hierarchical pass (frames of 32 x 32 and more) writes every pixel's
    // range itself; otherwise the default ranges, narrowed by the prior where it runs
    hier_ran_ = hier_runs(cfg_, w, h);
    ranges_written_ = range_planes_needed();
    if (ranges_written_ && !hier_ran_)
        RUN(launch_default_range(w, h, d0, cfg_.max_disparity, ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax), s),
            "range");
    const CostCtx cc = cost_ctx();
    support_count_ = 0;
    if (hier_ran_) {
        count_launches(launches);
        launches = 0;
        const int rc = run_hier();
        if (rc != kOk) return rc;
    } else if (prior_runs()) {
        e = launch_prior(cfg_, cc, L, arena_, s, &launches);
        if (e != cudaSuccess) return cuda_fail(e, "prior");
        if (prof) prof_mark("prior");
    } else if (debug_ || ranged()) {
        // no guiding disparity: d_prior is -1 everywhere (read by the fill in hierarchical mode,
        // otherwise only by the stage dump)
        fill_u32_kernel<<<std::min((int)((n + 255) / 256), 148 * 8), 256, 0, s>>>(ptr<uint32_t>(L.d_prior), n, 0xBF800000u);
        ++launches;
    }
    if (cfg_.hier_enable && !hier_ran_) RUNC(cudaMemsetAsync(arena_ + L.hstats, 0, 32, s), "hier stats init");
    cudaEventRecord(ev_[2], s);
    // cost (+ cross-H, + right argmin)
    RUNC(cudaMemsetAsync(ptr<uint32_t>(L.rkey), 0xFF, n * 4, s), "rkey init");
    const int lmax = std::max(1, cfg_.max_arm_length);
    const uint32_t* magic = ptr<uint32_t>(L.magic);
    if (L.raw_cost) RUN(launch_cost(cc, 0, lmax, cfg_.color_threshold, ptr<uint32_t>(L.volRaw), ptr<uint32_t>(L.rkey), magic, s), "cost(raw)");
    const uint32_t* sgm_src = nullptr;
    if (L.cross) {
        RUN(launch_cost(cc, 1, lmax, cfg_.color_threshold, ptr<uint32_t>(L.volA), ptr<uint32_t>(L.rkey), magic, s), "cost+crossH");
    } else if (L.fused_fast) {
        if (!L.raw_cost) RUN(launch_cost(cc, 2, lmax, 0, nullptr, ptr<uint32_t>(L.rkey), magic, s), "right argmin");
    } else {
        CostCtx cv = cc;
        cv.vol8 = L.cost8 ? 1 : 0;
        RUN(launch_cost(cv, 0, lmax, 0, ptr<uint32_t>(L.volA), ptr<uint32_t>(L.rkey), magic, s), "cost");
        sgm_src = ptr<uint32_t>(L.volA);
    }
    cudaEventRecord(ev_[3], s);
    // the right-image disparity needs only the argmin keys: it is finalized on the side stream while
    // the vertical aggregation and the sweeps run, and the confidence stage waits for it (serial
    // when every launch is profiled)
    rwta_forked_ = side_stream_ && !prof;
    if (rwta_forked_) {
        cudaEventRecord(ev_[10], s);
        RUNC(cudaStreamWaitEvent(side_stream_, ev_[10], 0), "fork");
        RUN(launch_right_wta_finalize(cc, ptr<uint32_t>(L.rkey), cfg_.subpixel, ptr<float>(L.disp_right), side_stream_),
            "right wta");
        cudaEventRecord(ev_[11], side_stream_);
    } else {
        RUN(launch_right_wta_finalize(cc, ptr<uint32_t>(L.rkey), cfg_.subpixel, ptr<float>(L.disp_right), s), "right wta");
    }
    cudaEventRecord(ev_[4], s);
    if (L.cross) {
        const int tau = cfg_.color_threshold;
        RUN(launch_cross_v(w, h, d0, D, Dp, lmax, tau, ptr<uint8_t>(L.lgray), ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax),
                           ptr<uint32_t>(L.volA), ptr<uint32_t>(L.volB), magic, !ranged(), L.cost8, s), "crossV");
        const int iters = std::max(1, cfg_.agg_iterations);
        for (int it = 1; it < iters; ++it) {
            RUN(launch_cross_h(w, h, d0, D, Dp, lmax, tau, ptr<uint8_t>(L.lgray), ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax),
                               ptr<uint32_t>(L.volB), ptr<uint32_t>(L.volA), magic, s), "crossH");
            RUN(launch_cross_v(w, h, d0, D, Dp, lmax, tau, ptr<uint8_t>(L.lgray), ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax),
                               ptr<uint32_t>(L.volA), ptr<uint32_t>(L.volB), magic, !ranged(), false, s), "crossV");
        }
        sgm_src = ptr<uint32_t>(L.volB);
    }
    cudaEventRecord(ev_[5], s);
    sgm_src_ = sgm_src;
    count_launches(launches);
    return kOk;
}

int Engine::sgm_launch(SgmLaunch* out, uint32_t** sbufs) const {
    const Layout& L = lay_;
    SgmLaunch& pl = *out;
    pl.w = L.w; pl.h = L.h; pl.d0 = cfg_.min_disparity; pl.D = L.D; pl.Dp = L.Dp;
    pl.pen = SgmPen{cfg_.P1, cfg_.P2_base, cfg_.adaptive_penalties, cfg_.piecewise_p2, cfg_.grad_t1, cfg_.grad_t2,
                    cfg_.p2_alpha};
    pl.gray = ptr<uint8_t>(L.lgray);
    // the volume run_pre leaves for the sweeps: cross-aggregated (volB), raw (volA), or none when
    // the Fast sweeps recompute their census costs
    pl.cvol = L.cross ? ptr<uint32_t>(L.volB) : (L.fused_fast ? nullptr : ptr<uint32_t>(L.volA));
    pl.cl = ptr<uint32_t>(L.cl); pl.cr = ptr<uint32_t>(L.cr); pl.qlut = ptr<uint16_t>(L.qlut);
    pl.disp = ptr<float>(L.disp_wta); pl.best = ptr<float>(L.best); pl.second = ptr<float>(L.second);
    pl.subpixel = cfg_.subpixel;
    pl.sp_method = scope_.sp_method;
    pl.sp_param = scope_.sp_param;
    pl.sp_tel = scope_.sp_telem ? ptr<apg_subpixel_telemetry_t>(L.tel) : nullptr;
    pl.store_final = (debug_ & 2) != 0;
    pl.lanes = sgm_lanes_;
    pl.split = sgm_split_;
    pl.cost8 = (!L.fused_fast && L.cost8) ? 1 : 0;
    for (int i = 0; i < L.nsbuf; ++i) sbufs[i] = ptr<uint32_t>(L.sbuf[i]);
    return L.nsbuf;
}

int Engine::ensure_pinned(size_t need) {
    if (pin_ && pinned_bytes_ >= need) return kOk;
    if (pin_) {
        cudaStreamSynchronize(stream_);
        cudaFreeHost(pin_);
    }
    pin_ = nullptr;
    pinned_bytes_ = 0;
    if (cudaMallocHost(&pin_, need) != cudaSuccess) {
        cudaGetLastError();
        return fail(kAllocationFailure, "pinned host staging allocation failed");
    }
    pinned_bytes_ = need;
    return kOk;
}

int Engine::upload(const uint8_t* left, const uint8_t* right, int w, int h, int stride, int ch, bool device,
                   cudaStream_t s) {
    cudaSetDevice(device_);
    int rc = prepare(w, h, ch);
    if (rc) return rc;
    const size_t n = (size_t)w * h, row = (size_t)w * ch, in_bytes = n * ch;
    cudaError_t e;
    if (device) {
        e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_left), row, left, stride, row, h, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_right), row, right, stride, row, h, cudaMemcpyDeviceToDevice, s);
    } else if (host_pinned(left) && host_pinned(right)) {
        e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_left), row, left, stride, row, h, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(ptr<uint8_t>(lay_.in_right), row, right, stride, row, h, cudaMemcpyHostToDevice, s);
    } else {
        rc = ensure_pinned(2 * in_bytes + n * 10 + 64);
        if (rc) return rc;
        for (int y = 0; y < h; ++y) {
            std::memcpy(pin_ + y * row, left + (size_t)y * stride, row);
            std::memcpy(pin_ + in_bytes + y * row, right + (size_t)y * stride, row);
        }
        e = cudaMemcpyAsync(ptr<uint8_t>(lay_.in_left), pin_, in_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ptr<uint8_t>(lay_.in_right), pin_ + in_bytes, in_bytes, cudaMemcpyHostToDevice, s);
    }
    return e == cudaSuccess ? kOk : cuda_fail(e, "input upload");
}

int Engine::enqueue_pre() {
    counts_fresh_ = false;
    const int row = lay_.w * lay_.ch;
    return run_pre(ptr<uint8_t>(lay_.in_left), row, ptr<uint8_t>(lay_.in_right), row, lay_.ch);
}

int Engine::enqueue_post() { return run_post(nullptr, nullptr, nullptr, nullptr); }

int Engine::download(float* disp, float* conf, uint8_t* reason, uint8_t* reliable, bool device, cudaStream_t s) {
    const size_t n = (size_t)lay_.w * lay_.h;
    const size_t in_bytes = n * lay_.ch;
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    // page-locked host outputs take the copies directly (finish_download then has nothing to do)
    direct_out_ = device || (host_pinned(disp) && host_pinned(conf) && host_pinned(reason) && host_pinned(reliable));
    if (!direct_out_) {
        int rc = ensure_pinned(2 * in_bytes + n * 10 + 64);
        if (rc) return rc;
    }
    unsigned char* st = direct_out_ ? nullptr : pin_ + 2 * in_bytes;  // host staging: disparity, confidence, reason, reliable
    float* pd = direct_out_ ? disp : reinterpret_cast<float*>(st);
    float* pc = direct_out_ ? conf : reinterpret_cast<float*>(st + n * 4);
    uint8_t* pr = direct_out_ ? reason : st + n * 8;
    uint8_t* pm = direct_out_ ? reliable : st + n * 9;
    cudaError_t e = cudaSuccess;
    if (disp) e = cudaMemcpyAsync(pd, ptr<float>(lay_.disp_out), n * 4, kind, s);
    if (e == cudaSuccess && conf) e = cudaMemcpyAsync(pc, ptr<float>(lay_.confidence), n * 4, kind, s);
    if (e == cudaSuccess && reason) e = cudaMemcpyAsync(pr, ptr<uint8_t>(lay_.reason), n, kind, s);
    if (e == cudaSuccess && reliable) e = cudaMemcpyAsync(pm, ptr<uint8_t>(lay_.reliable), n, kind, s);
    return e == cudaSuccess ? kOk : cuda_fail(e, "output download");
}

void Engine::finish_download(float* disp, float* conf, uint8_t* reason, uint8_t* reliable) const {
    if (direct_out_) return;
    const size_t n = (size_t)lay_.w * lay_.h;
    const unsigned char* st = pin_ + 2 * n * lay_.ch;
    if (disp) std::memcpy(disp, st, n * 4);
    if (conf) std::memcpy(conf, st + n * 4, n * 4);
    if (reason) std::memcpy(reason, st + n * 8, n);
    if (reliable) std::memcpy(reliable, st + n * 9, n);
}

int Engine::run_sgm() {
    const Layout& L = lay_;
    const int w = L.w, h = L.h, D = L.D, Dp = L.Dp, d0 = cfg_.min_disparity;
    const size_t n = (size_t)w * h;
    cudaStream_t s = stream_;
    unsigned launches = 0;
    cudaError_t e = cudaSuccess;
    const bool prof = (debug_ & 8) != 0;
    (void)D; (void)Dp; (void)d0; (void)n; (void)w; (void)h;
    // SGM: every sweep but the last in one launch (each direction into its own buffer), then the
    // last sweep adds three of them and runs the WTA (Path8: five buffers folded into the first
    // one before, 12 bytes per voxel, where folding all seven took 16 and the last sweep read one;
    // HighQuality 1920x1080 D256: fold + last sweep 2.02 -> 1.82 ms).  The sum over directions is
    // order-free (saturating adds of non-negative terms), so this changes no value.
    static const int first4[3][2] = {{1, 0}, {-1, 0}, {0, 1}};
    static const int first8[7][2] = {{1, 0}, {-1, 0}, {0, 1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    SgmLaunch pl;
    uint32_t* sb[7];
    sgm_launch(&pl, sb);
    RUN(launch_sgm_first(pl, L.nsbuf, L.nsbuf == 7 ? first8 : first4, sb, s), "sgm_first");
    if (L.nsbuf == 7) {
        RUN(launch_sgm_fold(sb, 5, n * (size_t)(Dp / 2), s), "sgm_fold5");
        sb[1] = sb[5];
        sb[2] = sb[6];
    }
    RUN(launch_sgm_last(pl, 0, -1, 3, sb, s), "sgm_last_wta");
    cudaEventRecord(ev_[6], s);
    count_launches(launches);
    return kOk;
}

int Engine::run_post(float* d_disp, float* d_conf, uint8_t* d_reason, uint8_t* d_reliable) {
    const Layout& L = lay_;
    const int w = L.w, h = L.h, D = L.D, Dp = L.Dp, d0 = cfg_.min_disparity;
    const size_t n = (size_t)w * h;
    cudaStream_t s = stream_;
    unsigned launches = 0;
    cudaError_t e = cudaSuccess;
    const bool prof = (debug_ & 8) != 0;
    (void)D; (void)Dp; (void)d0; (void)n; (void)w; (void)h;
    // confidence (+ LR when nothing runs between them)
    const bool refine = cfg_.refine_enable && cfg_.refine_iterations > 0;
    ConfLrArgs ca;
    ca.w = w; ca.h = h;
    ca.disp = ptr<float>(L.disp_wta); ca.disp_right = ptr<float>(L.disp_right);
    ca.best = ptr<float>(L.best); ca.second = ptr<float>(L.second);
    ca.lgx = ptr<uint8_t>(L.lgx); ca.lgy = ptr<uint8_t>(L.lgy);
    ca.uniqueness_ratio = cfg_.conf_uniqueness_ratio; ca.min_texture = cfg_.conf_min_texture;
    ca.reliable_threshold = cfg_.conf_reliable_threshold; ca.conf_lr_max_diff = cfg_.conf_lr_max_diff;
    ca.confidence = ptr<float>(L.confidence);
    ca.reliable = ptr<uint8_t>(L.reliable);
    ca.reason = ptr<uint8_t>(L.reason);
    ca.fuse_lr = refine ? 0 : 1;
    ca.lr_check = cfg_.lr_check;
    ca.post_lr_max_diff = cfg_.post_lr_max_diff;
    ca.disp_out = ptr<float>(L.disp_lr);
    if (rwta_forked_) RUNC(cudaStreamWaitEvent(s, ev_[11], 0), "join");  // the right-image disparity
    RUN(launch_conf_lr(ca, s), "confidence");
    if (debug_) RUNC(cudaMemcpyAsync(ptr<uint8_t>(L.reason_conf), ptr<uint8_t>(L.reason), n, cudaMemcpyDeviceToDevice, s), "dbg");
    if (early_conf_ || early_rel_ || early_reason_) {
        // maps that no later stage writes go to the host now, beside fill / median / counters
        RUNC(cudaEventRecord(ev_maps_, s), "event");
        RUNC(cudaStreamWaitEvent(copy_stream_, ev_maps_, 0), "event");
        if (early_conf_)
            RUNC(cudaMemcpyAsync(early_conf_, ptr<float>(L.confidence), n * 4, cudaMemcpyDeviceToHost, copy_stream_), "conf out");
        if (early_rel_)
            RUNC(cudaMemcpyAsync(early_rel_, ptr<uint8_t>(L.reliable), n, cudaMemcpyDeviceToHost, copy_stream_), "rel out");
        if (early_reason_ && !refine) {
            RUNC(cudaMemcpyAsync(early_reason_, ptr<uint8_t>(L.reason), n, cudaMemcpyDeviceToHost, copy_stream_), "reason out");
            early_reason_done_ = true;
        }
        RUNC(cudaEventRecord(ev_copied_, copy_stream_), "event");
        early_issued_ = true;
    }
    cudaEventRecord(ev_[7], s);
    const float* post_in = ptr<float>(L.disp_lr);
    if (refine) {
        RUNC(cudaMemcpyAsync(ptr<float>(L.disp_ref), ptr<float>(L.disp_wta), n * 4, cudaMemcpyDeviceToDevice, s), "refine copy");
        const int rc = run_refine(ptr<float>(L.disp_ref));
        if (rc) return rc;
        if (prof) prof_mark("refine");
        cudaEventRecord(ev_[8], s);
        if (cfg_.lr_check) {
            RUN(launch_lr(w, h, cfg_.post_lr_max_diff, ptr<float>(L.disp_right), ptr<float>(L.disp_ref), ptr<float>(L.disp_lr),
                          ptr<uint8_t>(L.reason), s), "lr");
        } else {
            post_in = ptr<float>(L.disp_ref);
        }
    } else {
        cudaEventRecord(ev_[8], s);
    }
    // the hierarchical coarse pass without coarse_fill_holes calls no fill at all
    // (src/hierarchical_stereo.cpp:262-265); a zero gap would still fill from the neighbours
    const float* med_in = post_in;
    if (!skip_fill_) {
        // the inpaint scope's gap replaces max_fill_gap unless it is Legacy at its default 32
        // (src/postprocess.cpp:45-48)
        const int gap = (scope_.ip_method == 0 && scope_.ip_gap == 32) ? cfg_.max_fill_gap : scope_.ip_gap;
        apg_inpaint_telemetry_t* ipt =
            scope_.ip_telem ? reinterpret_cast<apg_inpaint_telemetry_t*>(arena_ + L.tel + sizeof(apg_subpixel_telemetry_t))
                            : nullptr;
        RUN(launch_fill(w, h, gap, scope_.ip_method == 1, ipt, post_in, ptr<uint8_t>(L.reason), ptr<uint8_t>(L.lgray),
                        ranged() ? ptr<float>(L.d_prior) : nullptr, ptr<float>(L.disp_fill), s), "fill");
        med_in = ptr<float>(L.disp_fill);
    }
    float* final_out = d_disp ? d_disp : ptr<float>(L.disp_out);
    if (cfg_.median_radius > 0) {
        RUN(launch_median(w, h, cfg_.median_radius, med_in, final_out, s), "median");
    } else {
        RUNC(cudaMemcpyAsync(final_out, med_in, n * 4, cudaMemcpyDeviceToDevice, s), "copy");
    }
    if (d_reason) RUNC(cudaMemcpyAsync(d_reason, ptr<uint8_t>(L.reason), n, cudaMemcpyDeviceToDevice, s), "reason out");
    if (d_conf) RUNC(cudaMemcpyAsync(d_conf, ptr<float>(L.confidence), n * 4, cudaMemcpyDeviceToDevice, s), "conf out");
    if (d_reliable) RUNC(cudaMemcpyAsync(d_reliable, ptr<uint8_t>(L.reliable), n, cudaMemcpyDeviceToDevice, s), "rel out");
    if (d_disp && d_disp != ptr<float>(L.disp_out) && debug_)
        RUNC(cudaMemcpyAsync(ptr<float>(L.disp_out), d_disp, n * 4, cudaMemcpyDeviceToDevice, s), "dbg");
    // PipelineStats counters (src/pipeline.cpp:650-707); refine_changed compares the WTA map with
    // the refined one, prior_support_count is the prior's selected-support count
    unsigned long long* st = ptr<unsigned long long>(L.stats);
    RUNC(cudaMemsetAsync(st, 0, 64, s), "stats init");
    const bool planes = range_planes_needed();
    RUN(launch_frame_stats((int)n, final_out, ptr<uint8_t>(L.reliable), ptr<uint8_t>(L.reason),
                           refine ? ptr<float>(L.disp_wta) : nullptr, refine ? ptr<float>(L.disp_ref) : nullptr,
                           planes ? ptr<int16_t>(L.rmin) : nullptr, planes ? ptr<int16_t>(L.rmax) : nullptr,
                           planes ? 0ull : default_range_width_sum(), st, s),
        "frame stats");
    if (prior_runs()) RUNC(cudaMemcpyAsync(st + 5, arena_ + L.pr_count, 4, cudaMemcpyDeviceToDevice, s), "support count");
    cudaEventRecord(ev_[9], s);
    have_times_ = true;
    count_launches(launches);
    return kOk;
}

// Banded host path.  The last sweep runs bottom-up, so its rows finish from the bottom of the
// frame: it runs as nb launches over bands of rows (the chains' L and m carried between launches),
// and after each band, on post_stream_, the confidence / LR of the band's rows, then the fill and
// the median of the rows whose neighbourhoods are final (each stage reads one row above and below
// its own), then on copy_stream_ the device-to-host copies of every map row that is final.  The
// copies of all but the top band overlap the sweep.  Same kernels, same maps as run_sgm +
// run_post; frame counters over the whole map at the end.
int Engine::host_band_count(bool device) const {
    const Layout& L = lay_;
    const int req = device ? device_bands_ : host_bands_;
    if (req == 1 || (device && req == 0) || debug_ || !post_stream_ || !copy_stream_) return 0;
    if (refine_enabled() || L.nsbuf != 3 || L.h < 256 || cfg_.median_radius > 1) return 0;
    if (scope_.sp_telem || scope_.ip_telem) return 0;
    const int gap = (scope_.ip_method == 0 && scope_.ip_gap == 32) ? cfg_.max_fill_gap : scope_.ip_gap;
    if (!skip_fill_ && gap < 0) return 0;
    SgmLaunch pl;
    uint32_t* sb[7];
    sgm_launch(&pl, sb);
    if (!sgm_last_band_supported(pl, 3)) return 0;
    // the chains' state between bands lives in the refiner's map, unused without the refiner
    if ((size_t)32 * (L.Dp / 64 + 1) * 4 > (size_t)L.h * 4) return 0;
    return req > 1 ? std::min(req, (int)kMaxBands) : (int)kBands;
}

int Engine::run_banded(int nb, float* hdisp, float* hconf, uint8_t* hreason, uint8_t* hrel, bool to_host) {
    const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const Layout& L = lay_;
    const int w = L.w, h = L.h;
    const size_t n = (size_t)w * h;
    cudaStream_t s = stream_, ps = post_stream_, cs = copy_stream_, ss = sweep_stream_;
    unsigned launches = 0;
    cudaError_t e = cudaSuccess;
    const bool prof = false;
    static const int first4[3][2] = {{1, 0}, {-1, 0}, {0, 1}};
    SgmLaunch pl;
    uint32_t* sb[7];
    sgm_launch(&pl, sb);
    RUN(launch_sgm_first(pl, 3, first4, sb, s), "sgm_first");
    RUNC(cudaEventRecord(ev_fork_, s), "event");
    RUNC(cudaStreamWaitEvent(ss, ev_fork_, 0), "event");
    // the confidence stage reads the right-image disparity
    if (rwta_forked_) RUNC(cudaStreamWaitEvent(ps, ev_[11], 0), "join");
    ConfLrArgs ca;
    ca.w = w; ca.h = h;
    ca.disp = ptr<float>(L.disp_wta); ca.disp_right = ptr<float>(L.disp_right);
    ca.best = ptr<float>(L.best); ca.second = ptr<float>(L.second);
    ca.lgx = ptr<uint8_t>(L.lgx); ca.lgy = ptr<uint8_t>(L.lgy);
    ca.uniqueness_ratio = cfg_.conf_uniqueness_ratio; ca.min_texture = cfg_.conf_min_texture;
    ca.reliable_threshold = cfg_.conf_reliable_threshold; ca.conf_lr_max_diff = cfg_.conf_lr_max_diff;
    ca.confidence = ptr<float>(L.confidence);
    ca.reliable = ptr<uint8_t>(L.reliable);
    ca.reason = ptr<uint8_t>(L.reason);
    ca.fuse_lr = 1;
    ca.lr_check = cfg_.lr_check;
    ca.post_lr_max_diff = cfg_.post_lr_max_diff;
    ca.disp_out = ptr<float>(L.disp_lr);
    const bool fill = !skip_fill_;
    const bool med = cfg_.median_radius == 1;
    const int gap = (scope_.ip_method == 0 && scope_.ip_gap == 32) ? cfg_.max_fill_gap : scope_.ip_gap;
    const float* lr_map = ptr<float>(L.disp_lr);
    float* fill_map = ptr<float>(L.disp_fill);
    const float* med_in = fill ? fill_map : lr_map;
    const float* final_map = med ? ptr<float>(L.disp_out) : med_in;
    const int dfinal = (fill ? 1 : 0) + (med ? 1 : 0);  // rows a final row needs below the LR rows
    // band boundaries in steps from the bottom row, multiples of the WTA's 32-step blocks: sizes
    // shrink by about 0.7 a band (a row's copies take about 0.7 of its sweep time or less, so each
    // band's copies end while the next band sweeps), and the top band, whose post-processing and
    // copies follow the sweep, is small
    int tb[kMaxBands + 1];
    int nband = 0;
    {
        double wsum = 0.0, wk = 1.0;
        for (int k = 0; k < nb; ++k, wk *= 0.7) wsum += wk;
        double acc = 0.0;
        wk = 1.0;
        tb[0] = 0;
        for (int k = 0; k < nb; ++k, wk *= 0.7) {
            acc += wk;
            const int t = k == nb - 1 ? h : std::min(h, round_up((int)(h * acc / wsum + 0.5), 32));
            if (t > tb[nband]) tb[++nband] = t;
        }
    }
    uint32_t* carry = ptr<uint32_t>(L.disp_ref);
    int fill_hi = h, fin_hi = h;  // rows [fill_hi, h) of the fill map, [fin_hi, h) of the final map are done
    for (int band = 0; band < nband; ++band) {
        const int t0 = tb[band], t1 = tb[band + 1];
        RUN(launch_sgm_last_band(pl, 0, -1, 3, sb, t0, t1, carry, ss), "sgm_last_band");
        RUNC(cudaEventRecord(band_ev_[2 * band], ss), "event");
        RUNC(cudaStreamWaitEvent(ps, band_ev_[2 * band], 0), "event");
        const int ylo = h - t1, yhi = h - t0;
        const bool top = ylo == 0;
        // confidence + LR of the band's rows (each reads only its own row of the right-image map)
        const size_t o = (size_t)ylo * w, rows = (size_t)(yhi - ylo) * w;
        ConfLrArgs cb = ca;
        cb.h = yhi - ylo;
        cb.disp += o; cb.disp_right += o; cb.best += o; cb.second += o; cb.lgx += o; cb.lgy += o;
        cb.confidence += o; cb.reliable += o; cb.reason += o; cb.disp_out += o;
        RUN(launch_conf_lr(cb, ps), "confidence");
        if (fill) {
            const int flo = top ? 0 : ylo + 1;
            if (flo < fill_hi)
                RUN(launch_fill_rows(w, h, flo, fill_hi, gap, scope_.ip_method == 1, lr_map, ptr<uint8_t>(L.reason),
                                     ptr<uint8_t>(L.lgray), ranged() ? ptr<float>(L.d_prior) : nullptr, fill_map, ps),
                    "fill");
            fill_hi = flo;
        }
        const int mlo = top ? 0 : ylo + dfinal;
        if (med && mlo < fin_hi) RUN(launch_median3_rows(w, h, mlo, fin_hi, med_in, ptr<float>(L.disp_out), ps), "median");
        RUNC(cudaEventRecord(band_ev_[2 * band + 1], ps), "event");
        RUNC(cudaStreamWaitEvent(cs, band_ev_[2 * band + 1], 0), "event");
        if (hconf) RUNC(cudaMemcpyAsync(hconf + o, ptr<float>(L.confidence) + o, rows * 4, kind, cs), "conf out");
        if (hrel) RUNC(cudaMemcpyAsync(hrel + o, ptr<uint8_t>(L.reliable) + o, rows, kind, cs), "rel out");
        if (hreason) RUNC(cudaMemcpyAsync(hreason + o, ptr<uint8_t>(L.reason) + o, rows, kind, cs), "reason out");
        if (hdisp && mlo < fin_hi) {
            const size_t fo = (size_t)mlo * w;
            RUNC(cudaMemcpyAsync(hdisp + fo, final_map + fo, (size_t)(fin_hi - mlo) * w * 4, kind, cs), "disp out");
        }
        fin_hi = mlo;
    }
    RUNC(cudaEventRecord(ev_[6], ss), "event");
    RUNC(cudaStreamWaitEvent(s, ev_[6], 0), "event");
    cudaEventRecord(ev_[7], ps);
    cudaEventRecord(ev_[8], ps);
    // PipelineStats counters over the whole map (src/pipeline.cpp:650-707)
    unsigned long long* st = ptr<unsigned long long>(L.stats);
    RUNC(cudaMemsetAsync(st, 0, 64, ps), "stats init");
    const bool planes = range_planes_needed();
    RUN(launch_frame_stats((int)n, final_map, ptr<uint8_t>(L.reliable), ptr<uint8_t>(L.reason), nullptr, nullptr,
                           planes ? ptr<int16_t>(L.rmin) : nullptr, planes ? ptr<int16_t>(L.rmax) : nullptr,
                           planes ? 0ull : default_range_width_sum(), st, ps),
        "frame stats");
    if (prior_runs()) RUNC(cudaMemcpyAsync(st + 5, arena_ + L.pr_count, 4, cudaMemcpyDeviceToDevice, ps), "support count");
    cudaEventRecord(ev_[9], ps);
    RUNC(cudaStreamWaitEvent(cs, ev_[9], 0), "event");
    if (to_host) RUNC(cudaMemcpyAsync(counts_, st, sizeof(counts_), cudaMemcpyDeviceToHost, cs), "counters out");
    RUNC(cudaEventRecord(ev_copied_, cs), "event");
    have_times_ = true;
    count_launches(launches);
    return kOk;
}

// HierarchicalStereo::estimate_search_range (src/hierarchical_stereo.cpp:113-431) after the
// full-size aux planes: the half-size grays, the whole pipeline over them on the coarse engine
// (same stream, its outputs stay in its arena), then every full-size pixel's range and guiding
// disparity from the coarse disparity and confidence.
int Engine::run_hier() {
    const Layout& L = lay_;
    const int w = L.w, h = L.h;
    cudaStream_t s = stream_;
    unsigned launches = 0;
    cudaError_t e = cudaSuccess;
    const bool prof = (debug_ & 8) != 0;
    RUN(launch_hier_downsample(ptr<uint8_t>(L.lgray), ptr<uint8_t>(L.rgray), w, h, ptr<uint8_t>(L.hc_left),
                               ptr<uint8_t>(L.hc_right), s), "hier downsample");
    count_launches(launches);
    launches = 0;
    const int rc = coarse_->run(ptr<uint8_t>(L.hc_left), w / 2, ptr<uint8_t>(L.hc_right), w / 2, 1, nullptr, nullptr,
                                nullptr, nullptr);
    if (rc != kOk) return fail(rc, "hierarchical coarse pass: " + coarse_->last_error());
    if (prof) prof_mark("hier coarse pass");
    RUNC(cudaMemsetAsync(arena_ + L.hstats, 0, 32, s), "hier stats init");
    const Layout& K = coarse_->lay_;
    RUN(launch_hier_range(cfg_, w, h, coarse_->ptr<float>(K.disp_out), coarse_->ptr<float>(K.confidence),
                          ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax), ptr<float>(L.d_prior),
                          ptr<unsigned long long>(L.hstats), s), "hier range");
    count_launches(launches);
    return kOk;
}

#undef RUN
#undef RUNC

int Engine::supports(std::vector<SupportOut>& out) {
    out.clear();
    if (!arena_ || !prior_runs() || lay_.n_cells == 0) return kOk;
    const int nc = lay_.n_cells, mc = lay_.max_cand;
    std::vector<int> ncand(nc), taken(nc);
    std::vector<SupportOut> cand((size_t)nc * mc);
    static_assert(sizeof(SupportOut) == 16, "device Support record: int x, y; float d, conf");
    cudaError_t e = cudaMemcpyAsync(ncand.data(), arena_ + lay_.pr_ncand, nc * 4, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaMemcpyAsync(taken.data(), arena_ + lay_.pr_taken, nc * 4, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cand.data(), arena_ + lay_.pr_cand, cand.size() * 16, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "supports");
    // the selection order of extract_supports: pass 1 (each non-empty cell's base quota), then
    // round-robin rounds; or, with more non-empty cells than the budget, one per sampled cell
    std::vector<int> ne;
    for (int ci = 0; ci < nc; ++ci)
        if (ncand[ci] > 0) ne.push_back(ci);
    const int hard_max = cfg_.prior_max_supports;
    auto emit = [&](int ci, int k) { out.push_back(cand[(size_t)ci * mc + k]); };
    if ((int)ne.size() <= hard_max) {
        const int bq = std::max(1, hard_max / std::max(1, (int)ne.size()));
        std::vector<int> q1(nc, 0);
        for (int ci : ne) {
            q1[ci] = std::min(std::min(bq, ncand[ci]), taken[ci]);
            for (int k = 0; k < q1[ci]; ++k) emit(ci, k);
        }
        for (int r = 0;; ++r) {
            bool any = false;
            for (int ci : ne)
                if (taken[ci] > q1[ci] + r) {
                    emit(ci, q1[ci] + r);
                    any = true;
                }
            if (!any) break;
        }
    } else {
        for (int ci : ne)
            if (taken[ci] > 0) emit(ci, 0);
    }
    return kOk;
}

int Engine::hier_telemetry(double* out6) {
    for (int i = 0; i < 6; ++i) out6[i] = 0.0;
    if (!arena_ || !cfg_.hier_enable) return kOk;
    unsigned long long c[4] = {};
    cudaError_t e = cudaMemcpyAsync(c, arena_ + lay_.hstats, sizeof(c), cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "hierarchical telemetry");
    if (!hier_ran_) return kOk;
    // src/hierarchical_stereo.cpp:413-420: double ratios, three of them stored as float
    const double n = (double)lay_.w * lay_.h, nc = (double)(lay_.w / 2) * (lay_.h / 2);
    out6[0] = n > 0 ? (double)(long long)c[3] / n : 0.0;
    out6[1] = nc > 0 ? (double)(float)((double)c[0] / nc) : 0.0;
    out6[2] = n > 0 ? (double)(float)((double)c[1] / n) : 0.0;
    out6[3] = n > 0 ? (double)(float)((double)c[2] / n) : 0.0;
    float ms = 0.f;
    if (have_times_ && cudaEventElapsedTime(&ms, ev_[1], ev_[2]) == cudaSuccess) out6[4] = ms;
    cudaGetLastError();
    out6[5] = 1.0;
    return kOk;
}

void Engine::prof_mark(const char* name) {
    if (nprof_ >= kMaxProf) return;
    pname_[nprof_] = name;
    cudaEventRecord(pev_[nprof_ + 1], stream_);
    ++nprof_;
}

int Engine::launch_profile(int max, const char** names, float* ms) const {
    if (nprof_ == 0) return 0;
    cudaEventSynchronize(pev_[nprof_]);
    const int n = nprof_ < max ? nprof_ : max;
    for (int i = 0; i < n; ++i) {
        float t = 0.f;
        cudaEventElapsedTime(&t, pev_[i], pev_[i + 1]);
        if (names) names[i] = pname_[i];
        if (ms) ms[i] = t;
    }
    return n;
}

int Engine::run_refine(float* work) {
    // detail::refine_scalar (src/refiner.cpp:42-100): one mt19937(12345) stream, a fresh
    // uniform_int_distribution(-r, r) per iteration, draws consumed in the pass's raster order
    // (the draw tables and the on-device stream positions of refine.cu); no host synchronisation.
    const Layout& L = lay_;
    const int n = L.w * L.h;
    const int iters = cfg_.refine_iterations;
    if (!rtab_.dev || rtab_.iters != iters || rtab_.n_built < n || rtab_.radius_built != cfg_.refine_random_radius) {
        cudaStreamSynchronize(stream_);
        if (rtab_.build(iters, cfg_.refine_random_radius, n) != 0) {
            rtab_.release();
            cudaGetLastError();
            return fail(kAllocationFailure, "refine draw tables could not be built");
        }
    }
    if (!refine_err_host_) {
        if (cudaMallocHost(&refine_err_host_, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            refine_err_host_ = nullptr;
            return fail(kAllocationFailure, "pinned refine flag allocation failed");
        }
        *refine_err_host_ = 0;
    }
    const CostCtx cc = cost_ctx();
    unsigned launches = 0;
    unsigned char* state = arena_ + L.rf_state;
    cudaError_t e = cudaMemsetAsync(state, 0, (size_t)(kRefineProgWord + refine_band_count(L.h)) * 4, stream_);
    if (e == cudaSuccess) e = launch_refine_pack(cc, L, arena_, stream_, &launches);
    for (int it = 0; it < iters && e == cudaSuccess; ++it) {
        e = launch_refine_count(L, arena_, work, (it % 2) == 0, stream_, &launches);
        if (e == cudaSuccess) e = launch_refine_pass(cc, L, arena_, rtab_, it, work, refine_, stream_, &launches);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(refine_err_host_, state + kRefineErrWord * 4, sizeof(int), cudaMemcpyDeviceToHost, stream_);
    if (e != cudaSuccess) return cuda_fail(e, "refine");
    refine_pending_ = true;
    count_launches(launches);
    return kOk;
}

int Engine::check_refine() {
    if (!refine_pending_) return kOk;
    refine_pending_ = false;
    if (refine_err_host_ && *refine_err_host_) {
        *refine_err_host_ = 0;
        return fail(kInternalError, "refine: a wavefront wait timed out");
    }
    return kOk;
}

void Engine::stage_times(double* ms) const {
    for (int i = 0; i < 11; ++i) ms[i] = 0.0;
    if (!have_times_) return;
    cudaEventSynchronize(ev_[9]);
    auto el = [&](int a, int b) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev_[a], ev_[b]);
        return (double)t;
    };
    ms[0] = el(0, 1);   // aux
    ms[1] = el(1, 2);   // prior / range
    ms[2] = el(2, 3);   // cost (+cross-H, +right argmin)
    ms[3] = el(4, 5);   // cross (vertical)
    ms[4] = rwta_forked_ ? el(10, 11) : el(3, 4);   // right WTA (on the side stream when forked)
    ms[5] = el(5, 6);   // sgm (WTA fused into the last sweep)
    ms[6] = 0.0;        // wta: fused into the last SGM sweep
    ms[7] = el(6, 7);   // confidence (+LR when fused)
    ms[8] = el(7, 8);   // refine
    ms[9] = el(8, 9);   // post
    ms[10] = el(0, 9);  // total device time
}

int Engine::dump(int what, void* dst, size_t bytes) {
    if (!arena_) return fail(kInternalError, "nothing processed yet");
    const Layout& L = lay_;
    const size_t n = (size_t)L.w * L.h;
    const size_t csz = cfg_.census_type == APG_CENSUS_9X7 ? 8 : 4;
    size_t off = 0, sz = 0;
    bool vol = false, vol8 = false;
    switch (what) {
        case 0: off = L.lgray; sz = n; break;
        case 1: off = L.lgx; sz = n; break;
        case 2: off = L.lgy; sz = n; break;
        case 3: off = L.rgray; sz = n; break;
        case 4: off = L.rgx; sz = n; break;
        case 5: off = L.rgy; sz = n; break;
        case 6: off = L.cl; sz = n * csz; break;
        case 7: off = L.cr; sz = n * csz; break;
        case 8:
        case 9:
            off = what == 8 ? L.rmin : L.rmax;
            sz = n * 2;
            if (!ranges_written_) {
                // the frame used the default ranges in closed form: write the planes now
                const cudaError_t e = launch_default_range(L.w, L.h, cfg_.min_disparity, cfg_.max_disparity,
                                                           ptr<int16_t>(L.rmin), ptr<int16_t>(L.rmax), stream_);
                if (e != cudaSuccess) return cuda_fail(e, "range planes");
                ranges_written_ = true;
            }
            break;
        case 10: if (!L.raw_cost) return fail(kInternalError, "raw cost not materialised"); off = L.volRaw; vol = true; break;
        case 11:
            if (!L.cross) return fail(kInternalError, "no aggregated volume");
            off = L.volB;
            vol = true;
            vol8 = L.cost8;
            break;
        case 12: if (!(debug_ & 2)) return fail(kInternalError, "path sum not kept"); off = L.sbuf[0]; vol = true; break;
        case 13: off = L.disp_wta; sz = n * 4; break;
        case 14: off = L.best; sz = n * 4; break;
        case 15: off = L.second; sz = n * 4; break;
        case 16: off = L.disp_right; sz = n * 4; break;
        case 17: off = L.confidence; sz = n * 4; break;
        case 18: off = L.reliable; sz = n; break;
        case 19: off = L.reason_conf; sz = n; break;
        case 20: off = L.disp_ref; sz = n * 4; break;
        case 21: off = L.disp_lr; sz = n * 4; break;
        case 22: off = L.reason; sz = n; break;
        case 23: off = L.disp_fill; sz = n * 4; break;
        case 24: off = L.disp_out; sz = n * 4; break;
        case 25: off = L.d_prior; sz = n * 4; break;
        default: return fail(kInternalError, "unknown dump id");
    }
    cudaError_t e;
    if (vol) {
        // strip the disparity padding: D u16 of every Dp-long pixel run
        if (bytes < n * L.D * 2) return fail(kInternalError, "dump buffer too small");
        if (vol8) {
            // the byte volume, widened on the host (0xFF -> the invalid 0xFFFF)
            std::vector<uint8_t> tmp(n * L.D);
            e = cudaMemcpy2DAsync(tmp.data(), L.D, arena_ + off, L.Dp, L.D, n, cudaMemcpyDeviceToHost, stream_);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
            uint16_t* o = static_cast<uint16_t*>(dst);
            if (e == cudaSuccess)
                for (size_t i = 0; i < tmp.size(); ++i) o[i] = tmp[i] == 0xFF ? 0xFFFF : tmp[i];
        } else {
            e = cudaMemcpy2DAsync(dst, L.D * 2, arena_ + off, L.Dp * 2, L.D * 2, n, cudaMemcpyDeviceToHost, stream_);
        }
    } else {
        if (bytes < sz) return fail(kInternalError, "dump buffer too small");
        e = cudaMemcpyAsync(dst, arena_ + off, sz, cudaMemcpyDeviceToHost, stream_);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    return e == cudaSuccess ? kOk : cuda_fail(e, "dump");
}

int set_tuning(Engine* e, const char* key, int value) {
    if (std::strcmp(key, "sgm_lanes") == 0) {
        if (value != 0 && value != 8 && value != 16 && value != 32) return kInvalidConfig;
        if (e) e->set_sgm_lanes(value);
        return kOk;
    }
    if (std::strcmp(key, "sgm_split") == 0) {
        if (value < 0 || value > 2) return kInvalidConfig;
        if (e) e->set_sgm_split(value);
        return kOk;
    }
    if (std::strcmp(key, "cost8") == 0) {
        if (value < 0 || value > 2) return kInvalidConfig;
        if (e) e->set_cost8(value);
        return kOk;
    }
    if (std::strcmp(key, "cost_tile") == 0) {
        if (value != 0 && value != 64 && value != 128 && value != 256) return kInvalidConfig;
        if (e) e->set_cost_tile(value);
        return kOk;
    }
    if (std::strcmp(key, "cost_kernel") == 0) {
        if (value != 0 && value != 1) return kInvalidConfig;
        if (e) e->set_cost_kernel(value);
        return kOk;
    }
    if (std::strcmp(key, "fast_fused") == 0) {
        if (value != 0 && value != 1) return kInvalidConfig;
        if (e) e->set_fast_fused(value != 0);
        return kOk;
    }
    if (std::strcmp(key, "refine_spin_limit") == 0) {
        if (value < 0) return kInvalidConfig;
        if (e) e->set_refine_spin_limit(value);
        return kOk;
    }
    if (std::strcmp(key, "host_bands") == 0) {
        if (value < 0 || value > Engine::kMaxBands) return kInvalidConfig;
        if (e) e->set_host_bands(value);
        return kOk;
    }
    if (std::strcmp(key, "device_bands") == 0) {
        if (value < 0 || value > Engine::kMaxBands) return kInvalidConfig;
        if (e) e->set_device_bands(value);
        return kOk;
    }
    if (std::strcmp(key, "refine_window") == 0) {
        if (value != 0 && value != 1) return kInvalidConfig;
        if (e) e->set_refine_window(value);
        return kOk;
    }
    return kInvalidConfig;
}

}  // namespace apgcu

// ------------------------------------------------------------------------------------------------
// Extended C-ABI (include/apg_sgm_cuda.h)
// ------------------------------------------------------------------------------------------------
#include "../../include/apg_sgm_cuda.h"

struct apgcu_engine_s {
    apgcu::Engine* eng;
    std::string err;
};

extern "C" {

apgcu_engine_t apgcu_engine_create(const apg_pipeline_config_t* cfg, int device, void* stream) {
    if (!cfg) return nullptr;
    try {
        std::string msg;
        if (apgcu::Engine::validate_config(*cfg, msg) != apgcu::kOk) return nullptr;
        auto* h = new apgcu_engine_s;
        h->eng = new apgcu::Engine(*cfg, device, static_cast<cudaStream_t>(stream));
        return h;
    } catch (...) {
        return nullptr;
    }
}

void apgcu_engine_destroy(apgcu_engine_t e) {
    if (!e) return;
    delete e->eng;
    delete e;
}

const char* apgcu_engine_last_error(apgcu_engine_t e) { return e ? e->eng->last_error().c_str() : "Invalid engine handle"; }

int apgcu_engine_set_tuning(apgcu_engine_t e, const char* key, int value) {
    if (!e || !key) return apgcu::kInternalError;
    return apgcu::set_tuning(e->eng, key, value);
}

int apgcu_engine_set_debug(apgcu_engine_t e, int flags) {
    if (!e) return apgcu::kInternalError;
    e->eng->set_debug(flags);
    return 0;
}

static int check_views(const uint8_t* l, const uint8_t* r, int w, int h, int stride, int ch) {
    if (!l || !r || w <= 0 || h <= 0) return apgcu::kEmptyInput;
    if (ch != 1 && ch != 3 && ch != 4) return apgcu::kSizeMismatch;
    if (stride < w * ch) return apgcu::kSizeMismatch;
    return 0;
}

int apgcu_engine_process(apgcu_engine_t e, const uint8_t* left, const uint8_t* right, int width, int height, int stride,
                         int channels, float* disparity, float* confidence, uint8_t* invalid_reason,
                         uint8_t* reliable_mask) {
    if (!e) return apgcu::kInternalError;
    if (int v = check_views(left, right, width, height, stride, channels)) return v;
    try {
        return e->eng->process_host(left, right, width, height, stride, channels, disparity, confidence, invalid_reason,
                                    reliable_mask);
    } catch (const std::bad_alloc&) {
        return apgcu::kAllocationFailure;
    } catch (...) {
        return apgcu::kInternalError;
    }
}

int apgcu_engine_process_device(apgcu_engine_t e, const uint8_t* d_left, const uint8_t* d_right, int width, int height,
                                int stride, int channels, float* d_disparity, float* d_confidence,
                                uint8_t* d_invalid_reason, uint8_t* d_reliable_mask) {
    if (!e) return apgcu::kInternalError;
    if (int v = check_views(d_left, d_right, width, height, stride, channels)) return v;
    try {
        return e->eng->process_device(d_left, d_right, width, height, stride, channels, d_disparity, d_confidence,
                                      d_invalid_reason, d_reliable_mask);
    } catch (...) {
        return apgcu::kInternalError;
    }
}

int apgcu_engine_sync(apgcu_engine_t e) { return e ? e->eng->sync() : apgcu::kInternalError; }

int apgcu_engine_dump(apgcu_engine_t e, int what, void* host_dst, size_t bytes) {
    if (!e || !host_dst) return apgcu::kInternalError;
    return e->eng->dump(what, host_dst, bytes);
}

int apgcu_engine_stage_times(apgcu_engine_t e, double* ms11) {
    if (!e || !ms11) return apgcu::kInternalError;
    e->eng->stage_times(ms11);
    return 0;
}

size_t apgcu_engine_allocated_bytes(apgcu_engine_t e) { return e ? e->eng->allocated_bytes() : 0; }

size_t apgcu_workspace_bytes(const apg_pipeline_config_t* cfg, int width, int height) {
    if (!cfg || width <= 0 || height <= 0) return 0;
    return apgcu::Engine::workspace_bytes(*cfg, width, height, 3, 0);
}

int apgcu_set_experimental(int subpixel_method, float subpixel_param, int inpaint_method, int inpaint_gap) {
    if (subpixel_method < 0 || subpixel_method > 3 || inpaint_method < 0 || inpaint_method > 1)
        return apgcu::kInvalidConfig;
    apgcu::ExperimentalScope& s = apgcu::experimental_scope();
    s.sp_method = subpixel_method;
    s.sp_param = subpixel_param;
    s.ip_method = inpaint_method;
    s.ip_gap = inpaint_gap;
    return 0;
}

int apgcu_set_experimental_telemetry(int subpixel, int inpaint) {
    apgcu::ExperimentalScope& s = apgcu::experimental_scope();
    s.sp_telem = subpixel != 0;
    s.ip_telem = inpaint != 0;
    return 0;
}

void apgcu_get_experimental_telemetry(int* subpixel, int* inpaint) {
    const apgcu::ExperimentalScope& s = apgcu::experimental_scope();
    if (subpixel) *subpixel = s.sp_telem;
    if (inpaint) *inpaint = s.ip_telem;
}

void apgcu_get_telemetry(apg_subpixel_telemetry_t* sp, apg_inpaint_telemetry_t* ip) {
    const apgcu::TelemetryTotals& t = apgcu::telemetry_totals();
    if (sp) *sp = t.sp;
    if (ip) *ip = t.ip;
}

void apgcu_reset_telemetry(int subpixel, int inpaint) {
    apgcu::TelemetryTotals& t = apgcu::telemetry_totals();
    if (subpixel) t.sp = apg_subpixel_telemetry_t{};
    if (inpaint) t.ip = apg_inpaint_telemetry_t{};
}

void apgcu_get_experimental(int* subpixel_method, float* subpixel_param, int* inpaint_method, int* inpaint_gap) {
    const apgcu::ExperimentalScope& s = apgcu::experimental_scope();
    if (subpixel_method) *subpixel_method = s.sp_method;
    if (subpixel_param) *subpixel_param = s.sp_param;
    if (inpaint_method) *inpaint_method = s.ip_method;
    if (inpaint_gap) *inpaint_gap = s.ip_gap;
}

int apgcu_engine_supports(apgcu_engine_t e, int* x, int* y, float* disparity, float* confidence, int cap) {
    if (!e) return -1;
    std::vector<apgcu::Engine::SupportOut> s;
    if (e->eng->supports(s) != apgcu::kOk) return -1;
    const int n = (int)s.size();
    for (int i = 0; i < n && i < cap; ++i) {
        if (x) x[i] = s[i].x;
        if (y) y[i] = s[i].y;
        if (disparity) disparity[i] = s[i].d;
        if (confidence) confidence[i] = s[i].conf;
    }
    return n;
}

int apgcu_engine_hier_telemetry(apgcu_engine_t e, double* out6) {
    if (!e || !out6) return apgcu::kInternalError;
    return e->eng->hier_telemetry(out6);
}

void apgcu_engine_release(apgcu_engine_t e) {
    if (e) e->eng->release();
}

void* apgcu_engine_stream(apgcu_engine_t e) { return e ? static_cast<void*>(e->eng->stream()) : nullptr; }

void apgcu_config_from_mode(int mode, int max_disparity, apg_pipeline_config_t* out) {
    if (out) *out = apg_config_from_mode(mode, max_disparity);
}

unsigned long long apgcu_kernel_launch_count(void) { return apgcu::launch_count(); }

int apgcu_engine_launch_profile(apgcu_engine_t e, int max, const char** names, float* ms) {
    return e ? e->eng->launch_profile(max, names, ms) : 0;
}

}  // extern "C"

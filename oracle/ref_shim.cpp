// Stage-dump shim over the REFERENCE library (test infrastructure; see oracle/Makefile).
//
// It is compiled together with the reference's own sources into oracle/_ref/libapg_ref.so and
// only calls the reference's public C++ API (include/apg_sgm/*.hpp of the reference).  It
// exists so that the tests can
//   * pin the C restatement in oracle/apg_oracle.c against the reference, stage by stage;
//   * time the reference's own CPU path (the AVX2/OpenMP Packed backend) in bench.py.
// Nothing in the shipped library links or loads it.
//
// The staged run below repeats StereoMatcher::compute_impl (src/pipeline.cpp:435-719) for the
// Dense backend one stage at a time so that every intermediate can be copied out; the final
// outputs of the staged run are checked against a full StereoMatcher::compute of the same
// inputs, so a staged dump can never drift from what the reference really computes.

#include "apg_sgm/confidence_estimator.hpp"
#include "apg_sgm/cost_aggregator.hpp"
#include "apg_sgm/cost_computer.hpp"
#include "apg_sgm/pipeline.hpp"
#include "apg_sgm/postprocess.hpp"
#include "apg_sgm/prior_estimator.hpp"
#include "apg_sgm/refiner.hpp"
#include "apg_sgm/session.hpp"
#include "apg_sgm/sgm_optimizer.hpp"
#include "apg_sgm/metrics.hpp"
#include "hierarchical_stereo.hpp"
#include "inpaint_internal.hpp"
#include "subpixel_estimator.hpp"

#include "../include/apg_sgm/metrics.h"
#include "../include/apg_sgm/telemetry.h"
#include "../include/apg_sgm/pipeline_config.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

#if defined(_OPENMP)
#include <omp.h>
#endif

using namespace apg;

namespace {

PipelineConfig to_ref(const apg_pipeline_config_t& c) {
    PipelineConfig p = PipelineConfig::from_mode(
        c.mode == APG_MODE_FAST ? QualityMode::Fast
                                : (c.mode == APG_MODE_HIGH_QUALITY ? QualityMode::HighQuality
                                                                   : QualityMode::Balanced),
        c.max_disparity);
    p.min_disparity = c.min_disparity;
    p.max_disparity = c.max_disparity;
    p.num_threads = c.num_threads;
    p.volume_backend = c.volume_backend == 1 ? VolumeBackend::Dense
                       : (c.volume_backend == 2 ? VolumeBackend::Packed : VolumeBackend::Auto);
    p.cost.census = c.census_type == APG_CENSUS_9X7 ? CensusType::Census9x7
                                                    : CensusType::SymmetricCensus9x7;
    p.cost.lambda_census = c.lambda_census;
    p.cost.lambda_ad = c.lambda_ad;
    p.cost.lambda_grad = c.lambda_grad;
    p.cost.eta_ad = c.eta_ad;
    p.cost.mu_grad = c.mu_grad;
    p.cost.use_ad = c.use_ad != 0;
    p.cost.use_grad = c.use_grad != 0;
    p.cost.cost_max = c.cost_max;
    p.aggregation.enable = c.agg_enable != 0;
    p.aggregation.max_arm_length = c.max_arm_length;
    p.aggregation.color_threshold = c.color_threshold;
    p.aggregation.iterations = c.agg_iterations;
    p.sgm.paths = c.paths == 8 ? PathType::Path8 : PathType::Path4;
    p.sgm.P1 = c.P1;
    p.sgm.P2_base = c.P2_base;
    p.sgm.adaptive_penalties = c.adaptive_penalties != 0;
    p.sgm.grad_t1 = c.grad_t1;
    p.sgm.grad_t2 = c.grad_t2;
    p.sgm.p2_alpha = c.p2_alpha;
    p.sgm.piecewise_p2 = c.piecewise_p2 != 0;
    p.prior.enable = c.prior_enable != 0;
    p.prior.uniqueness_ratio = c.prior_uniqueness_ratio;
    p.prior.texture_threshold = c.prior_texture_threshold;
    p.prior.lr_max_diff = c.prior_lr_max_diff;
    p.prior.search_radius = c.prior_search_radius;
    p.prior.min_supports = c.prior_min_supports;
    p.prior.max_supports = c.prior_max_supports;
    p.confidence.uniqueness_ratio = c.conf_uniqueness_ratio;
    p.confidence.lr_max_diff = c.conf_lr_max_diff;
    p.confidence.min_texture = c.conf_min_texture;
    p.confidence.reliable_threshold = c.conf_reliable_threshold;
    p.refine.enable = c.refine_enable != 0;
    p.refine.iterations = c.refine_iterations;
    p.refine.random_radius = c.refine_random_radius;
    p.post.subpixel = c.subpixel != 0;
    p.post.lr_check = c.lr_check != 0;
    p.post.lr_max_diff = c.post_lr_max_diff;
    p.post.median_radius = c.median_radius;
    p.post.max_fill_gap = c.max_fill_gap;
    p.hierarchical.enable = c.hier_enable != 0;
    p.hierarchical.radius = c.hier_radius;
    p.hierarchical.scale = c.hier_scale;
    p.hierarchical.fallback = c.hier_fallback == APG_HIER_FALLBACK_FULL_RANGE ? HierarchicalFallback::FullRange
                              : (c.hier_fallback == APG_HIER_FALLBACK_EXPANDED_RADIUS
                                     ? HierarchicalFallback::ExpandedRadius
                                     : HierarchicalFallback::NearestValid);
    p.hierarchical.coarse_cross_agg = c.hier_coarse_cross_agg != 0;
    p.hierarchical.coarse_fill_holes = c.hier_coarse_fill_holes != 0;
    p.hierarchical.adaptive_radius = c.hier_adaptive_radius != 0;
    p.hierarchical.confidence_threshold = c.hier_confidence_threshold;
    p.hierarchical.expanded_radius = c.hier_expanded_radius;
    return p;
}

Image8 to_image(const uint8_t* data, int w, int h, int stride, int ch) {
    return ImageView8(data, w, h, stride, ch).to_image();
}

template <typename T>
void put(T* dst, const T* src, size_t n) {
    if (dst && src && n) std::memcpy(dst, src, n * sizeof(T));
}

} // namespace

extern "C" {

typedef struct {
    uint8_t *left_gray, *left_gx, *left_gy, *right_gray, *right_gx, *right_gy;
    uint32_t *census_left, *census_right;
    uint64_t *census_left64, *census_right64;
    int16_t *range_min, *range_max;
    uint16_t *cost_raw;   /* W*H*D, after CostComputer::compute_volume */
    uint16_t *cost_agg;   /* W*H*D, after CostAggregator::aggregate (== cost_raw when off) */
    uint32_t *sgm_sum;    /* W*H*D, SgmOptimizer::optimize accumulator */
    float *disp_wta, *best, *second, *disp_right;
    float *conf_confidence; uint8_t *conf_reliable, *conf_reason;
    float *d_prior, *disp_refined;
    float *disp_lr; uint8_t *reason_lr;
    float *disp_fill;
    float *disparity, *confidence; uint8_t *invalid_reason, *reliable_mask;
    int support_count;
    float *prior_conf, *prior_spread, *prior_dmin, *prior_dmax;
} ref_dump_t;

// Full staged run of the Dense pipeline.  Returns 0 on success, a StatusCode on a rejected
// input, -100 if the staged run disagrees with StereoMatcher::compute.
int ref_dump(const apg_pipeline_config_t* ccfg, const uint8_t* left, const uint8_t* right,
             int w, int h, int stride, int ch, ref_dump_t* out) {
    PipelineConfig cfg = to_ref(*ccfg);
    cfg.volume_backend = VolumeBackend::Dense;
    const Image8 L = to_image(left, w, h, stride, ch);
    const Image8 R = to_image(right, w, h, stride, ch);
#if defined(_OPENMP)
    if (cfg.num_threads > 0) omp_set_num_threads(cfg.num_threads);
#endif

    StereoMatcher matcher(cfg);
    PipelineBuffers full;
    if (!matcher.compute(L, R, full)) {
        Status s = validate_inputs(L, R);
        if (!s.ok()) return static_cast<int>(s.code);
        s = validate_config(cfg);
        return s.ok() ? static_cast<int>(StatusCode::InternalError) : static_cast<int>(s.code);
    }

    PipelineBuffers b;
    CostComputer cost;
    PriorEstimator prior;
    CostAggregator agg;
    SgmOptimizer sgm;
    ConfidenceEstimator conf;
    Refiner refiner;
    PostProcessor post;
    const size_t n = static_cast<size_t>(w) * h;

    cost.compute_aux(L, R, cfg, b);
    put(out->left_gray, b.left_gray.data(), n);
    put(out->left_gx, b.left_gx.data(), n);
    put(out->left_gy, b.left_gy.data(), n);
    put(out->right_gray, b.right_gray.data(), n);
    put(out->right_gx, b.right_gx.data(), n);
    put(out->right_gy, b.right_gy.data(), n);
    put(out->census_left, b.census_left.data(), b.census_left.size());
    put(out->census_right, b.census_right.data(), b.census_right.size());
    put(out->census_left64, b.census_left64.data(), b.census_left64.size());
    put(out->census_right64, b.census_right64.data(), b.census_right64.size());

    prior.estimate(cfg, b);
    put(out->range_min, b.range.dmin.data(), n);
    put(out->range_max, b.range.dmax.data(), n);
    put(out->d_prior, b.d_prior.data(), n);
    put(out->prior_conf, b.prior_confidence.data(), b.prior_confidence.empty() ? 0 : n);
    put(out->prior_spread, b.prior_spread.data(), b.prior_spread.empty() ? 0 : n);
    put(out->prior_dmin, b.d_prior_min.data(), b.d_prior_min.empty() ? 0 : n);
    put(out->prior_dmax, b.d_prior_max.data(), b.d_prior_max.empty() ? 0 : n);
    out->support_count = static_cast<int>(b.support_count);

    cost.compute_volume(cfg, b);
    const size_t nv = b.cost.bytes() / sizeof(uint16_t);
    put(out->cost_raw, b.cost.data(), nv);

    agg.aggregate(cfg, b);
    put(out->cost_agg, b.cost.data(), nv);

    sgm.optimize(cfg, b);
    put(out->sgm_sum, b.cost32.data(), nv);

    Image32f best, second;
    sgm.winner_take_all(cfg, b.cost32, b.range, b.disparity, &best, &second);
    put(out->disp_wta, b.disparity.data(), n);
    put(out->best, best.data(), n);
    put(out->second, second.data(), n);

    // The right-image WTA lives in an internal helper of pipeline.cpp; take it from the full run.
    b.disparity_right = full.disparity_right;
    put(out->disp_right, b.disparity_right.data(), n);

    conf.estimate(cfg, b, best, second);
    put(out->conf_confidence, b.confidence.data(), n);
    put(out->conf_reliable, b.reliable_mask.data(), n);
    put(out->conf_reason, b.invalid_reason.data(), n);

    refiner.refine(cfg, b);
    put(out->disp_refined, b.disparity.data(), n);

    post.left_right_check(cfg, b);
    put(out->disp_lr, b.disparity.data(), n);
    put(out->reason_lr, b.invalid_reason.data(), n);
    post.fill_holes(cfg, b);
    put(out->disp_fill, b.disparity.data(), n);
    post.median(cfg, b);

    put(out->disparity, full.disparity.data(), n);
    put(out->confidence, full.confidence.data(), n);
    put(out->invalid_reason, full.invalid_reason.data(), n);
    put(out->reliable_mask, full.reliable_mask.data(), n);

    if (std::memcmp(b.disparity.data(), full.disparity.data(), n * sizeof(float)) != 0 ||
        std::memcmp(b.confidence.data(), full.confidence.data(), n * sizeof(float)) != 0 ||
        std::memcmp(b.invalid_reason.data(), full.invalid_reason.data(), n) != 0 ||
        std::memcmp(b.reliable_mask.data(), full.reliable_mask.data(), n) != 0) {
        return -100;
    }
    return 0;
}

// One SGM path direction over a caller-supplied dense volume (SgmOptimizer::aggregate_path,
// src/sgm_optimizer.cpp:186-259).  acc (u32, W*H*D) is accumulated in place.
void ref_aggregate_path(const apg_pipeline_config_t* ccfg, const uint8_t* gray, const uint16_t* base,
                        uint32_t* acc, int w, int h, int d0, int D, int dx, int dy) {
    PipelineConfig cfg = to_ref(*ccfg);
    Image8 g(w, h, 1);
    std::memcpy(g.data(), gray, static_cast<size_t>(w) * h);
    CostVolume vb(w, h, d0, d0 + D, 0);
    std::memcpy(vb.data(), base, vb.bytes());
    CostVolume32 va(w, h, d0, d0 + D, 0);
    std::memcpy(va.data(), acc, va.bytes());
    SgmOptimizer().aggregate_path(cfg, g, vb, va, dx, dy);
    std::memcpy(acc, va.data(), va.bytes());
}

// SgmOptimizer::winner_take_all over a u32 volume (src/sgm_optimizer.cpp:436-555).
void ref_winner_take_all(const apg_pipeline_config_t* ccfg, const uint32_t* vol, const int16_t* rmin,
                         const int16_t* rmax, int w, int h, int d0, int D, float* disp, float* best,
                         float* second) {
    PipelineConfig cfg = to_ref(*ccfg);
    CostVolume32 v(w, h, d0, d0 + D, 0);
    std::memcpy(v.data(), vol, v.bytes());
    SearchRange r;
    r.allocate(w, h, d0, d0 + D);
    std::memcpy(r.dmin.data(), rmin, static_cast<size_t>(w) * h * sizeof(int16_t));
    std::memcpy(r.dmax.data(), rmax, static_cast<size_t>(w) * h * sizeof(int16_t));
    Image32f d, b, s;
    SgmOptimizer().winner_take_all(cfg, v, r, d, &b, &s);
    const size_t n = static_cast<size_t>(w) * h;
    put(disp, d.data(), n);
    put(best, b.data(), n);
    put(second, s.data(), n);
}

// Hierarchical search range of one pair (HierarchicalStereo::estimate_search_range after
// CostComputer::compute_aux, src/hierarchical_stereo.cpp:113-431) and the final maps of a full
// StereoMatcher::compute with the same configuration (Packed backend).  telem5 (nullable):
// avg_states_per_pixel, coarse_valid_ratio, fallback_pixel_ratio, full_range_pixel_ratio and 1 if
// the coarse pass ran (0: the small-frame fallback).  d_prior is -1 where the reference leaves it
// unset.  Returns 0, or the StatusCode of a rejected configuration or input.
int ref_hier_dump(const apg_pipeline_config_t* ccfg, const uint8_t* left, const uint8_t* right, int w, int h,
                  int stride, int ch, int16_t* rmin, int16_t* rmax, float* d_prior, double* telem5,
                  float* disparity, float* confidence, uint8_t* invalid_reason, uint8_t* reliable_mask) {
    PipelineConfig cfg = to_ref(*ccfg);
    Status s = validate_config(cfg);
    if (!s.ok()) return static_cast<int>(s.code);
    const Image8 L = to_image(left, w, h, stride, ch);
    const Image8 R = to_image(right, w, h, stride, ch);
    const size_t n = static_cast<size_t>(w) * h;
    PipelineBuffers b;
    CostComputer().compute_aux(L, R, cfg, b);
    HierarchicalTelemetry t;
    const bool ran = HierarchicalStereo::estimate_search_range(cfg.hierarchical, cfg, b, &t, nullptr, cfg.num_threads);
    put(rmin, b.range.dmin.data(), n);
    put(rmax, b.range.dmax.data(), n);
    if (d_prior) {
        if (b.d_prior.empty()) std::fill(d_prior, d_prior + n, -1.f);
        else put(d_prior, b.d_prior.data(), n);
    }
    if (telem5) {
        const double v[5] = {t.avg_states_per_pixel, t.coarse_valid_ratio, t.fallback_pixel_ratio,
                             t.full_range_pixel_ratio, ran ? 1.0 : 0.0};
        std::memcpy(telem5, v, sizeof(v));
    }
    StereoMatcher matcher(cfg);
    PipelineBuffers full;
    if (!matcher.compute(L, R, full)) {
        s = validate_inputs(L, R);
        return s.ok() ? static_cast<int>(StatusCode::InternalError) : static_cast<int>(s.code);
    }
    put(disparity, full.disparity.data(), n);
    put(confidence, full.confidence.data(), n);
    put(invalid_reason, full.invalid_reason.data(), n);
    put(reliable_mask, full.reliable_mask.data(), n);
    return 0;
}

static void region_out(const RegionMetrics& r, apg_region_metrics_t* o) {
    o->total_pixels = r.total_pixels;
    o->valid_est_pixels = r.valid_est_pixels;
    o->valid_ratio = r.valid_ratio;
    o->epe = r.epe;
    o->bad_0_5 = r.bad_0_5;
    o->bad_1_0 = r.bad_1_0;
    o->bad_2_0 = r.bad_2_0;
    o->bad_3_0 = r.bad_3_0;
    o->d1 = r.d1;
}

// The reference's evaluate_stereo (src/metrics.cpp:119-502) on plain buffers; nullable inputs
// are passed as null pointers, thr NULL means QualityThresholds{}.
void ref_evaluate_stereo(const float* est, const float* gt, int w, int h, const int16_t* rmin, const int16_t* rmax,
                         const float* before, const float* after, const uint8_t* vis, float max_valid_gt,
                         const uint8_t* left, int left_stride, int left_ch, const apg_quality_thresholds_t* thr,
                         apg_stereo_metrics_t* out) {
    const size_t n = static_cast<size_t>(w) * h;
    auto img32 = [&](const float* p) {
        Image32f im(w, h);
        std::memcpy(im.data(), p, n * sizeof(float));
        return im;
    };
    const Image32f E = img32(est), G = img32(gt);
    SearchRange range;
    if (rmin && rmax) {
        range.allocate(w, h, 0, 1);
        std::memcpy(range.dmin.data(), rmin, n * sizeof(int16_t));
        std::memcpy(range.dmax.data(), rmax, n * sizeof(int16_t));
    }
    Image32f B, A;
    if (before && after) {
        B = img32(before);
        A = img32(after);
    }
    Image8 V;
    if (vis) V = to_image(vis, w, h, w, 1);
    Image8 Lf;
    if (left) Lf = to_image(left, w, h, left_stride, left_ch);
    QualityThresholds q;
    if (thr) {
        q.boundary_disparity_gradient = thr->boundary_disparity_gradient;
        q.low_texture_gradient = thr->low_texture_gradient;
        q.max_valid_gt = thr->max_valid_gt;
    }
    const StereoMetrics m = evaluate_stereo(E, G, (rmin && rmax) ? &range : nullptr, (before && after) ? &B : nullptr,
                                            (before && after) ? &A : nullptr, vis ? &V : nullptr, max_valid_gt,
                                            nullptr, left ? &Lf : nullptr, q);
    apg_stereo_metrics_t o;
    std::memset(&o, 0, sizeof(o));
    o.total_pixels = m.total_pixels;
    o.evaluated_pixels = m.evaluated_pixels;
    o.valid_pixels = m.valid_pixels;
    o.valid_ratio = m.valid_ratio;
    o.epe = m.epe;
    o.bad_0_5 = m.bad_0_5;
    o.bad_1_0 = m.bad_1_0;
    o.bad_2_0 = m.bad_2_0;
    o.bad_3_0 = m.bad_3_0;
    o.kitti_d1_all = m.kitti_d1_all;
    o.kitti_d1_noc = m.kitti_d1_noc;
    o.edge_pixels = m.edge_pixels;
    o.edge_epe = m.edge_epe;
    o.nonedge_pixels = m.nonedge_pixels;
    o.nonedge_epe = m.nonedge_epe;
    o.lr_fail_ratio = m.lr_fail_ratio;
    o.has_range = m.has_range ? 1 : 0;
    o.range_recall_all = m.range_recall_all;
    o.range_recall_matchable = m.range_recall_matchable;
    o.range_recall_visible = m.range_recall_visible;
    o.range_visible_eval_pixels = m.range_visible_eval_pixels;
    o.range_visible_in_pixels = m.range_visible_in_pixels;
    o.range_matchable_eval_pixels = m.range_matchable_eval_pixels;
    o.range_matchable_in_pixels = m.range_matchable_in_pixels;
    o.prior_miss_visible_count = m.prior_miss_visible_count;
    o.prior_miss_edge = m.prior_miss_edge;
    o.prior_miss_nonedge = m.prior_miss_nonedge;
    o.prior_miss_edge_ratio = m.prior_miss_edge_ratio;
    o.prior_miss_nonedge_ratio = m.prior_miss_nonedge_ratio;
    region_out(m.reg_all, &o.reg_all);
    region_out(m.reg_noc, &o.reg_noc);
    region_out(m.reg_occ, &o.reg_occ);
    region_out(m.reg_boundary, &o.reg_boundary);
    region_out(m.reg_non_boundary, &o.reg_non_boundary);
    region_out(m.reg_low_texture, &o.reg_low_texture);
    region_out(m.reg_high_texture, &o.reg_high_texture);
    o.has_refine_stats = m.has_refine_stats ? 1 : 0;
    o.refine_eval_pixels = m.refine_eval_pixels;
    o.refine_epe_delta = m.refine_epe_delta;
    o.post_epe_delta = m.post_epe_delta;
    o.total_epe_delta = m.total_epe_delta;
    o.refine_improved_ratio = m.refine_improved_ratio;
    o.refine_worsened_ratio = m.refine_worsened_ratio;
    o.refine_unchanged_ratio = m.refine_unchanged_ratio;
    o.refine_changed_ratio = m.refine_changed_ratio;
    *out = o;
}

// The reference's image I/O (src/image.cpp:62-206).  Loads return 1 on success, 0 on failure, -1
// where the reference throws (std::stoi / std::stof on a malformed header); dims are written on
// success only.
int ref_load_image(const char* path, uint8_t* dst, size_t cap, int* w, int* h, int* ch) {
    try {
        Image8 im;
        if (!load_image(path, im)) return 0;
        *w = im.width();
        *h = im.height();
        *ch = im.channels();
        const size_t n = static_cast<size_t>(im.width()) * im.height() * im.channels();
        if (dst && cap >= n) std::memcpy(dst, im.data(), n);
        return 1;
    } catch (...) {
        return -1;
    }
}

int ref_load_pfm(const char* path, float* dst, size_t cap, int* w, int* h) {
    try {
        Image32f im;
        if (!load_pfm(path, im)) return 0;
        *w = im.width();
        *h = im.height();
        const size_t n = static_cast<size_t>(im.width()) * im.height();
        if (dst && cap >= n) std::memcpy(dst, im.data(), n * sizeof(float));
        return 1;
    } catch (...) {
        return -1;
    }
}

int ref_save_pgm(const char* path, const uint8_t* img, int w, int h) {
    Image8 im(w, h, 1);
    std::memcpy(im.data(), img, static_cast<size_t>(w) * h);
    return save_pgm(path, im) ? 1 : 0;
}

int ref_save_pgm16(const char* path, const int16_t* d, int w, int h) {
    Image16s im(w, h);
    std::memcpy(im.data(), d, static_cast<size_t>(w) * h * sizeof(int16_t));
    return save_pgm16(path, im) ? 1 : 0;
}

int ref_save_disparity_preview(const char* path, const float* d, int w, int h, float dmax) {
    Image32f im(w, h);
    std::memcpy(im.data(), d, static_cast<size_t>(w) * h * sizeof(float));
    return save_disparity_preview(path, im, dmax) ? 1 : 0;
}

int ref_save_pfm(const char* path, const float* d, int w, int h) {
    Image32f im(w, h);
    std::memcpy(im.data(), d, static_cast<size_t>(w) * h * sizeof(float));
    return save_pfm(path, im) ? 1 : 0;
}

// The reference's experimental scopes on the calling thread, kept open until the next call
// (defaults 0, 0, 0, 32 restore the reference's production behaviour).
static std::unique_ptr<ExperimentalInpaintScope> g_ip_scope;
static std::unique_ptr<ExperimentalSubpixelScope> g_sp_scope;

void ref_set_experimental_tel(int sp_method, float sp_param, int sp_tel, int ip_method, int ip_gap, int ip_tel) {
    g_ip_scope.reset();
    g_sp_scope.reset();
    g_sp_scope.reset(new ExperimentalSubpixelScope(static_cast<SubpixelMethod>(sp_method), sp_param, sp_tel != 0));
    g_ip_scope.reset(new ExperimentalInpaintScope(static_cast<InpaintMethod>(ip_method), ip_gap, ip_tel != 0));
}

void ref_set_experimental(int sp_method, float sp_param, int ip_method, int ip_gap) {
    ref_set_experimental_tel(sp_method, sp_param, 0, ip_method, ip_gap, 0);
}

// The reference's telemetry totals of the calling thread (current_telemetry() of both scopes).
void ref_get_telemetry(apg_subpixel_telemetry_t* sp, apg_inpaint_telemetry_t* ip) {
    const SubpixelTelemetry& s = ExperimentalSubpixelScope::current_telemetry();
    sp->candidate_pixels = s.candidate_pixels;
    sp->applied_pixels = s.applied_pixels;
    sp->degenerate_count = s.degenerate_count;
    sp->clamped_count = s.clamped_count;
    sp->negative_curvature_count = s.negative_curvature_count;
    sp->sum_abs_delta = s.sum_abs_delta;
    for (int i = 0; i < 50; ++i) sp->delta_buckets[i] = s.delta_buckets[i];
    const InpaintTelemetry& t = ExperimentalInpaintScope::current_telemetry();
    ip->total_invalid_pixels = t.total_invalid_pixels;
    ip->classified_occ_pixels = t.classified_occ_pixels;
    ip->classified_mismatch_pixels = t.classified_mismatch_pixels;
    ip->hit_max_gap_pixels = t.hit_max_gap_pixels;
    ip->reclassified_shadow_pixels = t.reclassified_shadow_pixels;
    for (int i = 0; i < 11; ++i) ip->route_counts[i] = t.route_counts[i];
    ip->invalid_runs_count = t.invalid_runs_count;
    ip->invalid_runs_truncated = t.invalid_runs_truncated;
    for (int i = 0; i < 10; ++i) ip->run_length_buckets[i] = t.run_length_buckets[i];
}

// The reference's evaluate_supports (src/metrics.cpp:8-124) on plain arrays.
void ref_evaluate_supports(const int* x, const int* y, const float* d, int n, const float* gt, int w, int h,
                           const uint8_t* vis, float max_valid_gt, int cell_size, apg_support_metrics_t* out) {
    std::vector<SupportMatch> s(static_cast<size_t>(std::max(n, 0)));
    for (int i = 0; i < n; ++i) {
        s[i].x = x[i];
        s[i].y = y[i];
        s[i].disparity = d[i];
    }
    Image32f G(w, h);
    std::memcpy(G.data(), gt, static_cast<size_t>(w) * h * sizeof(float));
    Image8 V;
    if (vis) V = to_image(vis, w, h, w, 1);
    const SupportMetrics m = evaluate_supports(s, G, vis ? &V : nullptr, max_valid_gt, cell_size);
    apg_support_metrics_t o;
    std::memset(&o, 0, sizeof(o));
    o.total = m.total; o.gt_valid = m.gt_valid; o.visible = m.visible;
    o.correct_05 = m.correct_05; o.correct_1 = m.correct_1; o.correct_2 = m.correct_2;
    o.visible_correct_05 = m.visible_correct_05; o.visible_correct_1 = m.visible_correct_1;
    o.visible_correct_2 = m.visible_correct_2; o.visible_gt_cells = m.visible_gt_cells;
    o.correct_visible_cells = m.correct_visible_cells;
    o.precision_05 = m.precision_05; o.precision_1 = m.precision_1; o.precision_2 = m.precision_2;
    o.precision_all_05 = m.precision_all_05; o.precision_all_1 = m.precision_all_1; o.precision_all_2 = m.precision_all_2;
    o.precision_vis_05 = m.precision_vis_05; o.precision_vis_1 = m.precision_vis_1; o.precision_vis_2 = m.precision_vis_2;
    o.mean_abs_error = m.mean_abs_error; o.mae_all = m.mae_all; o.mae_visible = m.mae_visible;
    o.grid_recall_1 = m.grid_recall_1; o.grid_coverage = m.grid_coverage;
    o.support_grid_recall_vis_1 = m.support_grid_recall_vis_1;
    *out = o;
}

// Public-API session used for timing the reference CPU path.
void* ref_session_create(const apg_pipeline_config_t* ccfg, int bounded_reuse) {
    ExecutionOptions opt;
    opt.memory_policy = bounded_reuse ? MemoryPolicy::BoundedReuse : MemoryPolicy::ReleasePerFrame;
    opt.num_threads = ccfg->num_threads;
    return new StereoSession(to_ref(*ccfg), opt);
}

void ref_session_destroy(void* s) { delete static_cast<StereoSession*>(s); }

// StereoSession::process_status (include/apg_sgm/session.hpp:26-41) on a borrowed strided view.
// stage_ms (nullable) receives the 11 StageTiming fields in declaration order; stats13 (nullable)
// the PipelineStats frame counters: valid, reliable, unreliable, refine_changed and lr_fail pixels,
// prior_support_count, mean_search_width, mean_geometry_width, then the five ratios.
int ref_session_process(void* s, const uint8_t* left, const uint8_t* right, int w, int h, int stride,
                        int ch, float* disp, float* conf, uint8_t* reason, uint8_t* reliable,
                        double* stage_ms, double* stats13) {
    auto* ss = static_cast<StereoSession*>(s);
    StereoResult res;
    PipelineStats st;
    Status status = ss->process_status(ImageView8(left, w, h, stride, ch),
                                       ImageView8(right, w, h, stride, ch), res, &st);
    if (!status.ok()) return static_cast<int>(status.code);
    const size_t n = static_cast<size_t>(w) * h;
    put(disp, res.disparity.data(), n);
    put(conf, res.confidence.data(), n);
    put(reason, res.invalid_reason.data(), n);
    put(reliable, res.reliable_mask.data(), n);
    if (stage_ms) {
        const StageTiming& t = st.timing;
        const double v[11] = {t.aux_ms, t.prior_ms, t.cost_ms, t.cross_ms, t.right_wta_ms, t.sgm_ms,
                              t.wta_ms, t.confidence_ms, t.refine_ms, t.post_ms, t.total_ms};
        std::memcpy(stage_ms, v, sizeof(v));
    }
    if (stats13) {
        const double v[13] = {(double)st.valid_pixels, (double)st.reliable_pixels, (double)st.unreliable_pixels,
                              (double)st.refine_changed_pixels, (double)st.lr_fail_pixels,
                              (double)st.prior_support_count, st.mean_search_width, st.mean_geometry_width,
                              st.valid_disparity_ratio, st.reliable_ratio, st.unreliable_ratio,
                              st.refine_changed_ratio, st.lr_fail_ratio};
        std::memcpy(stats13, v, sizeof(v));
    }
    return 0;
}

int ref_max_threads(void) {
#if defined(_OPENMP)
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"

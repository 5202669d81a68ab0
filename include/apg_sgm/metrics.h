/* Plain-C mirror of the reference's accuracy metrics records (include/apg_sgm/metrics.hpp:11-125 of
 * the reference: SupportMetrics, RegionMetrics, QualityThresholds, and StereoMetrics, whose
 * support block is evaluated separately by evaluate_supports),
 * shared by the CUDA library's evaluate entry point (include/apg_sgm_cuda.h), the CPU oracle and
 * the reference shim under oracle/.  Field names and meanings are the reference's; counts of
 * pixels are int as there, the four range pixel counts size_t-wide (unsigned long long).
 */
#ifndef APG_METRICS_T_DEFINED
#define APG_METRICS_T_DEFINED

#ifdef __cplusplus
extern "C" {
#endif

/* RegionMetrics (metrics.hpp:46-56). */
typedef struct {
    int total_pixels;     /* valid GT pixels in the region */
    int valid_est_pixels; /* estimate finite and >= 0 */
    float valid_ratio;
    float epe;            /* mean |est - gt| over valid estimates */
    float bad_0_5, bad_1_0, bad_2_0, bad_3_0; /* % of valid estimates above the error */
    float d1;             /* KITTI D1 outlier rate, % of total_pixels */
} apg_region_metrics_t;

/* QualityThresholds (metrics.hpp:58-62). */
typedef struct {
    float boundary_disparity_gradient; /* 1.0: GT 4-neighbour difference >= this marks a boundary */
    float low_texture_gradient;        /* 4.0: luma gradient below this marks low texture */
    float max_valid_gt;                /* 1e5 (the struct member; evaluate_stereo takes its own bound) */
} apg_quality_thresholds_t;

/* StereoMetrics (metrics.hpp:64-125) without has_supports / support_metrics. */
typedef struct {
    int total_pixels, evaluated_pixels, valid_pixels;
    float valid_ratio;
    float epe, bad_0_5, bad_1_0, bad_2_0, bad_3_0;
    float kitti_d1_all, kitti_d1_noc;
    int edge_pixels;
    float edge_epe;
    int nonedge_pixels;
    float nonedge_epe;
    float lr_fail_ratio;
    int has_range;
    float range_recall_all, range_recall_matchable, range_recall_visible;
    unsigned long long range_visible_eval_pixels, range_visible_in_pixels;
    unsigned long long range_matchable_eval_pixels, range_matchable_in_pixels;
    int prior_miss_visible_count, prior_miss_edge, prior_miss_nonedge;
    float prior_miss_edge_ratio, prior_miss_nonedge_ratio;
    apg_region_metrics_t reg_all, reg_noc, reg_occ, reg_boundary, reg_non_boundary, reg_low_texture,
        reg_high_texture;
    int has_refine_stats, refine_eval_pixels;
    float refine_epe_delta, post_epe_delta, total_epe_delta;
    float refine_improved_ratio, refine_worsened_ratio, refine_unchanged_ratio, refine_changed_ratio;
} apg_stereo_metrics_t;

/* SupportMetrics (metrics.hpp:11-44): the prior's support matches against the ground truth. */
typedef struct {
    int total, gt_valid, visible, correct_05, correct_1, correct_2;
    int visible_correct_05, visible_correct_1, visible_correct_2, visible_gt_cells, correct_visible_cells;
    float precision_05, precision_1, precision_2;
    float precision_all_05, precision_all_1, precision_all_2;
    float precision_vis_05, precision_vis_1, precision_vis_2;
    float mean_abs_error, mae_all, mae_visible;
    float grid_recall_1, grid_coverage, support_grid_recall_vis_1;
} apg_support_metrics_t;

/* SupportMetrics from its tallies (src/metrics.cpp:92-124): c = {gt_valid, visible, correct_05,
 * correct_1, correct_2, visible_correct_05, visible_correct_1, visible_correct_2, visible_gt_cells,
 * correct_visible_cells}, s = {sum of errors, sum of visible errors}. */
static inline void apg_support_finalize(int total, const long long* c, const double* s, apg_support_metrics_t* m) {
    apg_support_metrics_t z = {0};
    *m = z;
    m->total = total;
    m->gt_valid = (int)c[0];
    m->visible = (int)c[1];
    m->correct_05 = (int)c[2];
    m->correct_1 = (int)c[3];
    m->correct_2 = (int)c[4];
    m->visible_correct_05 = (int)c[5];
    m->visible_correct_1 = (int)c[6];
    m->visible_correct_2 = (int)c[7];
    if (m->gt_valid > 0) {
        m->precision_all_05 = (float)m->correct_05 / (float)m->gt_valid;
        m->precision_all_1 = (float)m->correct_1 / (float)m->gt_valid;
        m->precision_all_2 = (float)m->correct_2 / (float)m->gt_valid;
        m->precision_05 = m->precision_all_05;
        m->precision_1 = m->precision_all_1;
        m->precision_2 = m->precision_all_2;
        m->mae_all = (float)(s[0] / m->gt_valid);
        m->mean_abs_error = m->mae_all;
    }
    if (m->visible > 0) {
        m->precision_vis_05 = (float)m->visible_correct_05 / (float)m->visible;
        m->precision_vis_1 = (float)m->visible_correct_1 / (float)m->visible;
        m->precision_vis_2 = (float)m->visible_correct_2 / (float)m->visible;
        m->mae_visible = (float)(s[1] / m->visible);
    }
    m->visible_gt_cells = (int)c[8];
    m->correct_visible_cells = (int)c[9];
    if (c[8] > 0) {
        m->grid_recall_1 = (float)(int)c[9] / (float)(int)c[8];
        m->grid_coverage = m->grid_recall_1;
        m->support_grid_recall_vis_1 = m->grid_recall_1;
    }
}

/* QualityThresholds{} defaults. */
static inline apg_quality_thresholds_t apg_quality_thresholds_default(void) {
    apg_quality_thresholds_t t;
    t.boundary_disparity_gradient = 1.0f;
    t.low_texture_gradient = 4.0f;
    t.max_valid_gt = 1e5f;
    return t;
}

/* The per-pixel tallies every evaluate_stereo implementation reduces (integer counts, then double
 * sums of float errors), in this order; apg_metrics_finalize turns them into the record with the
 * reference's float expressions (src/metrics.cpp:240-262, 430-499). */
enum {
    APG_MC_EVALUATED = 0, APG_MC_VALID, APG_MC_C05, APG_MC_C10, APG_MC_C20, APG_MC_C30,
    APG_MC_D1_ALL, APG_MC_D1_NOC, APG_MC_EVAL_NOC, APG_MC_LR_FAIL,
    APG_MC_EVAL_ALL, APG_MC_IN_ALL, APG_MC_EVAL_MATCH, APG_MC_IN_MATCH, APG_MC_EVAL_VIS, APG_MC_IN_VIS,
    APG_MC_MISS_VIS, APG_MC_MISS_EDGE, APG_MC_MISS_NONEDGE, APG_MC_EDGE, APG_MC_NONEDGE,
    APG_MC_REF_EVAL, APG_MC_REF_IMPROVED, APG_MC_REF_WORSENED, APG_MC_REF_UNCHANGED, APG_MC_REF_CHANGED,
    APG_MC_TOTAL_EVAL,
    APG_MC_REGION0, /* 7 regions (all, noc, occ, boundary, non-boundary, low texture, high texture) x
                       (total, valid, >0.5, >1, >2, >3, d1) */
    APG_MC_COUNT = APG_MC_REGION0 + 49
};
enum {
    APG_MS_EPE = 0, APG_MS_EDGE, APG_MS_NONEDGE, APG_MS_BEFORE, APG_MS_AFTER, APG_MS_TOT_BEFORE,
    APG_MS_TOT_AFTER, APG_MS_TOT_FINAL, APG_MS_REGION0, /* 7 region error sums */
    APG_MS_COUNT = APG_MS_REGION0 + 7
};

static inline void apg_region_finalize(const long long* c, double sum, apg_region_metrics_t* r) {
    const int total = (int)c[0], valid = (int)c[1];
    r->total_pixels = total;
    r->valid_est_pixels = valid;
    r->valid_ratio = r->d1 = 0.0f;
    r->epe = r->bad_0_5 = r->bad_1_0 = r->bad_2_0 = r->bad_3_0 = 0.0f;
    if (total > 0) {
        r->valid_ratio = (float)valid / (float)total;
        r->d1 = (float)(int)c[6] * 100.0f / (float)total;
    }
    if (valid > 0) {
        r->epe = (float)(sum / valid);
        r->bad_0_5 = (float)(int)c[2] * 100.0f / (float)valid;
        r->bad_1_0 = (float)(int)c[3] * 100.0f / (float)valid;
        r->bad_2_0 = (float)(int)c[4] * 100.0f / (float)valid;
        r->bad_3_0 = (float)(int)c[5] * 100.0f / (float)valid;
    }
}

/* StereoMetrics from the tallies (src/metrics.cpp:430-502); has_range / has_refine_data / w*h as
 * the call saw them. */
static inline void apg_metrics_finalize(const long long* c, const double* s, int total_pixels, int has_range,
                                        int has_refine_data, apg_stereo_metrics_t* m) {
    int i;
    (void)has_refine_data;
    apg_stereo_metrics_t z = {0};
    *m = z;
    m->total_pixels = total_pixels;
    m->evaluated_pixels = (int)c[APG_MC_EVALUATED];
    m->valid_pixels = (int)c[APG_MC_VALID];
    m->edge_pixels = (int)c[APG_MC_EDGE];
    m->nonedge_pixels = (int)c[APG_MC_NONEDGE];
    if (m->evaluated_pixels > 0) {
        m->valid_ratio = (float)m->valid_pixels / (float)m->evaluated_pixels;
        m->lr_fail_ratio = (float)(int)c[APG_MC_LR_FAIL] / (float)m->evaluated_pixels;
    }
    if (has_range) {
        const int ea = (int)c[APG_MC_EVAL_ALL], em = (int)c[APG_MC_EVAL_MATCH], ev = (int)c[APG_MC_EVAL_VIS];
        const int miss = (int)c[APG_MC_MISS_VIS];
        m->has_range = 1;
        m->range_recall_all = ea > 0 ? (float)(int)c[APG_MC_IN_ALL] / ea : 0.0f;
        m->range_recall_matchable = em > 0 ? (float)(int)c[APG_MC_IN_MATCH] / em : 0.0f;
        m->range_recall_visible = ev > 0 ? (float)(int)c[APG_MC_IN_VIS] / ev : 0.0f;
        m->range_visible_eval_pixels = (unsigned long long)ev;
        m->range_visible_in_pixels = (unsigned long long)c[APG_MC_IN_VIS];
        m->range_matchable_eval_pixels = (unsigned long long)em;
        m->range_matchable_in_pixels = (unsigned long long)c[APG_MC_IN_MATCH];
        m->prior_miss_visible_count = miss;
        m->prior_miss_edge = (int)c[APG_MC_MISS_EDGE];
        m->prior_miss_nonedge = (int)c[APG_MC_MISS_NONEDGE];
        if (miss > 0) {
            m->prior_miss_edge_ratio = (float)m->prior_miss_edge / miss;
            m->prior_miss_nonedge_ratio = (float)m->prior_miss_nonedge / miss;
        }
    }
    if (m->valid_pixels > 0) {
        const float v = (float)m->valid_pixels;
        m->epe = (float)(s[APG_MS_EPE] / m->valid_pixels);
        m->bad_0_5 = (float)(int)c[APG_MC_C05] / v * 100.0f;
        m->bad_1_0 = (float)(int)c[APG_MC_C10] / v * 100.0f;
        m->bad_2_0 = (float)(int)c[APG_MC_C20] / v * 100.0f;
        m->bad_3_0 = (float)(int)c[APG_MC_C30] / v * 100.0f;
    }
    if (m->evaluated_pixels > 0)
        m->kitti_d1_all = (float)(int)c[APG_MC_D1_ALL] / (float)m->evaluated_pixels * 100.0f;
    if (c[APG_MC_EVAL_NOC] > 0)
        m->kitti_d1_noc = (float)(int)c[APG_MC_D1_NOC] / (float)(int)c[APG_MC_EVAL_NOC] * 100.0f;
    if (m->edge_pixels > 0) m->edge_epe = (float)(s[APG_MS_EDGE] / m->edge_pixels);
    if (m->nonedge_pixels > 0) m->nonedge_epe = (float)(s[APG_MS_NONEDGE] / m->nonedge_pixels);
    {
        const int re = (int)c[APG_MC_REF_EVAL];
        if (re > 0) {
            m->has_refine_stats = 1;
            m->refine_eval_pixels = re;
            m->refine_epe_delta = (float)((s[APG_MS_AFTER] - s[APG_MS_BEFORE]) / re);
            m->refine_improved_ratio = (float)(int)c[APG_MC_REF_IMPROVED] / (float)re;
            m->refine_worsened_ratio = (float)(int)c[APG_MC_REF_WORSENED] / (float)re;
            m->refine_unchanged_ratio = (float)(int)c[APG_MC_REF_UNCHANGED] / (float)re;
            m->refine_changed_ratio = (float)(int)c[APG_MC_REF_CHANGED] / (float)re;
        }
    }
    {
        const int te = (int)c[APG_MC_TOTAL_EVAL];
        if (te > 0) {
            m->post_epe_delta = (float)((s[APG_MS_TOT_FINAL] - s[APG_MS_TOT_AFTER]) / te);
            m->total_epe_delta = (float)((s[APG_MS_TOT_FINAL] - s[APG_MS_TOT_BEFORE]) / te);
        }
    }
    {
        apg_region_metrics_t* regs[7] = {&m->reg_all, &m->reg_noc, &m->reg_occ, &m->reg_boundary,
                                         &m->reg_non_boundary, &m->reg_low_texture, &m->reg_high_texture};
        for (i = 0; i < 7; ++i) apg_region_finalize(c + APG_MC_REGION0 + 7 * i, s[APG_MS_REGION0 + i], regs[i]);
    }
}

#ifdef __cplusplus
}
#endif

#endif /* APG_METRICS_T_DEFINED */

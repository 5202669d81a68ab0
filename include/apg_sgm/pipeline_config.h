/* Plain-C mirror of the reference's apg::PipelineConfig (include/apg_sgm/config.hpp:7-112)
 * shared by the oracle, the reference shim and the CUDA library's extended C-ABI.
 *
 * Every numeric knob of PipelineConfig that the dense-matching path reads is a field here,
 * with the same meaning and units.  apg_config_from_mode() restates
 * PipelineConfig::from_mode (src/config.cpp:5-45) and the member defaults of
 * include/apg_sgm/config.hpp:7-84, including HierarchicalConfig (the opt-in coarse-to-fine
 * search range of src/hierarchical_stereo.cpp, which no quality preset enables).
 *
 * It is the configuration record of the CUDA library's extended C-ABI (include/apg_sgm_cuda.h)
 * and is also read by the CPU oracle and the reference shim under oracle/.
 */
#ifndef APG_PIPELINE_CONFIG_T_DEFINED
#define APG_PIPELINE_CONFIG_T_DEFINED

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Quality presets (include/apg_sgm/types.hpp:12-16). */
#define APG_MODE_FAST 0
#define APG_MODE_BALANCED 1
#define APG_MODE_HIGH_QUALITY 2

/* Census flavours (include/apg_sgm/types.hpp:24-27). */
#define APG_CENSUS_9X7 0           /* 62-bit plain census, uint64 descriptors */
#define APG_CENSUS_SYMMETRIC_9X7 1 /* 31-bit symmetric census, uint32 descriptors */

/* HierarchicalFallback (include/apg_sgm/config.hpp:68-72). */
#define APG_HIER_FALLBACK_NEAREST_VALID 0
#define APG_HIER_FALLBACK_FULL_RANGE 1
#define APG_HIER_FALLBACK_EXPANDED_RADIUS 2

typedef struct {
    int mode;          /* APG_MODE_* (informational once the fields below are set) */
    int min_disparity; /* d0, may be negative */
    int max_disparity; /* exclusive upper bound */
    int num_threads;   /* CPU reference only */
    int volume_backend;/* 0 Auto, 1 Dense, 2 Packed, 3 CUDA */

    /* CostParams (config.hpp:7-17) */
    int census_type;
    float lambda_census, lambda_ad, lambda_grad;
    float eta_ad, mu_grad;
    int use_ad, use_grad;
    int cost_max;

    /* AggregationParams (config.hpp:19-24) */
    int agg_enable, max_arm_length, color_threshold, agg_iterations;

    /* SgmParams (config.hpp:26-35) */
    int paths; /* 4 or 8 */
    int P1, P2_base, adaptive_penalties, grad_t1, grad_t2;
    float p2_alpha;
    int piecewise_p2;

    /* PriorParams (config.hpp:37-45) */
    int prior_enable;
    float prior_uniqueness_ratio;
    int prior_texture_threshold, prior_lr_max_diff, prior_search_radius;
    int prior_min_supports, prior_max_supports;

    /* ConfidenceParams (config.hpp:47-52) */
    float conf_uniqueness_ratio;
    int conf_lr_max_diff;
    float conf_min_texture, conf_reliable_threshold;

    /* RefineParams (config.hpp:54-58) */
    int refine_enable, refine_iterations, refine_random_radius;

    /* PostParams (config.hpp:60-66) */
    int subpixel, lr_check, post_lr_max_diff, median_radius, max_fill_gap;

    /* HierarchicalConfig (config.hpp:74-84); hier_fallback is APG_HIER_FALLBACK_* */
    int hier_enable, hier_radius, hier_scale, hier_fallback;
    int hier_coarse_cross_agg, hier_coarse_fill_holes, hier_adaptive_radius;
    float hier_confidence_threshold;
    int hier_expanded_radius;
} apg_pipeline_config_t;

/* PipelineConfig::from_mode(mode, max_disparity) with min_disparity 0 (src/config.cpp:5-45). */
static inline apg_pipeline_config_t apg_config_from_mode(int mode, int max_disparity) {
    apg_pipeline_config_t c;
    c.mode = mode;
    c.min_disparity = 0;
    c.max_disparity = max_disparity;
    c.num_threads = 0;
    c.volume_backend = 0;
    c.census_type = APG_CENSUS_SYMMETRIC_9X7;
    c.lambda_census = 16.f; c.lambda_ad = 30.f; c.lambda_grad = 20.f;
    c.eta_ad = 0.4f; c.mu_grad = 0.3f;
    c.use_ad = 1; c.use_grad = 1; c.cost_max = 255;
    c.agg_enable = 1; c.max_arm_length = 17; c.color_threshold = 12; c.agg_iterations = 1;
    c.paths = 4; c.P1 = 10; c.P2_base = 120; c.adaptive_penalties = 1;
    c.grad_t1 = 8; c.grad_t2 = 24; c.p2_alpha = 0.15f; c.piecewise_p2 = 1;
    c.prior_enable = 0; c.prior_uniqueness_ratio = 0.4f; c.prior_texture_threshold = 4;
    c.prior_lr_max_diff = 1; c.prior_search_radius = 16; c.prior_min_supports = 32;
    c.prior_max_supports = 4000;
    c.conf_uniqueness_ratio = 0.15f; c.conf_lr_max_diff = 1;
    c.conf_min_texture = 2.f; c.conf_reliable_threshold = 0.25f;
    c.refine_enable = 0; c.refine_iterations = 3; c.refine_random_radius = 4;
    c.subpixel = 1; c.lr_check = 1; c.post_lr_max_diff = 1; c.median_radius = 1; c.max_fill_gap = 32;
    c.hier_enable = 0; c.hier_radius = 4; c.hier_scale = 2; c.hier_fallback = APG_HIER_FALLBACK_NEAREST_VALID;
    c.hier_coarse_cross_agg = 1; c.hier_coarse_fill_holes = 1; c.hier_adaptive_radius = 0;
    c.hier_confidence_threshold = 0.5f; c.hier_expanded_radius = 8;
    if (mode == APG_MODE_FAST) {
        c.use_ad = 0; c.use_grad = 0; c.agg_enable = 0; c.paths = 4; c.adaptive_penalties = 0;
        c.prior_enable = 0; c.refine_enable = 0; c.subpixel = 1; c.lr_check = 1;
    } else if (mode == APG_MODE_HIGH_QUALITY) {
        c.paths = 8; c.prior_enable = 1; c.refine_enable = 1; c.refine_iterations = 3;
    } else {
        c.agg_iterations = 1;
    }
    return c;
}

#ifdef __cplusplus
}
#endif

#endif /* APG_PIPELINE_CONFIG_T_DEFINED */

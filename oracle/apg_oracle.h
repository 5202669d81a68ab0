/* CPU oracle: a plain-C99 restatement of the reference apg-sgm dense-matching path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load this library, and only as the checker.  The shipped CUDA library never links,
 * loads or calls it, and has no CPU fallback.
 *
 * Parity pin: every stage is compared byte-for-byte with the reference's own stage outputs
 * (oracle/_ref/libapg_ref.so, built from the reference sources by oracle/Makefile) and against
 * the reference's frozen FNV-1a fingerprints (tests/test_api_contract.cpp:243-257) and its 1-D
 * SGM known-answer test (tests/test_synthetic.cpp:26-71); see tests/test_oracle_pins.py.
 *
 * Layouts follow the reference Dense backend: images row-major W*H; volumes
 * vol[(y*W + x)*D + (d - d0)] (include/apg_sgm/buffers.hpp:45-55).
 */
#ifndef APG_ORACLE_H
#define APG_ORACLE_H

#include <stdint.h>
#include "../include/apg_sgm/pipeline_config.h"
#include "../include/apg_sgm/metrics.h"
#include "../include/apg_sgm/telemetry.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_INVALID_COST 65535u
#define ORC_INVALID_COST32 0xFFFFFFFFu
#define ORC_PATH_INF (1 << 28)

enum { ORC_VALID = 0, ORC_OCCLUSION = 1, ORC_MISMATCH = 2, ORC_LOW_CONFIDENCE = 3, ORC_OUT_OF_RANGE = 4 };

void orc_gray_grad(const uint8_t* src, int w, int h, int stride, int ch,
                   uint8_t* gray, uint8_t* gx, uint8_t* gy);
void orc_census_sym(const uint8_t* gray, int w, int h, uint32_t* out);
void orc_census64(const uint8_t* gray, int w, int h, uint64_t* out);
void orc_range_default(const apg_pipeline_config_t* cfg, int w, int h, int16_t* rmin, int16_t* rmax);
void orc_cost_lut(const apg_pipeline_config_t* cfg, float* lut_census65, float* lut_ad256, float* lut_grad511);
void orc_cost_volume(const apg_pipeline_config_t* cfg, int w, int h,
                     const uint8_t* lgray, const uint8_t* lgx, const uint8_t* lgy,
                     const uint8_t* rgray, const uint8_t* rgx, const uint8_t* rgy,
                     const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                     const int16_t* rmin, const int16_t* rmax, uint16_t* vol);
void orc_cross_arms(const uint8_t* gray, int w, int h, int max_arm, int tau,
                    int16_t* L, int16_t* R, int16_t* U, int16_t* Dn);
void orc_cross_aggregate(const apg_pipeline_config_t* cfg, const uint8_t* gray, int w, int h,
                         const int16_t* rmin, const int16_t* rmax, uint16_t* vol);
void orc_sgm_path(const apg_pipeline_config_t* cfg, const uint8_t* gray, const uint16_t* vol,
                  uint32_t* acc, int w, int h, int D, int dx, int dy);
void orc_sgm_optimize(const apg_pipeline_config_t* cfg, const uint8_t* gray, const uint16_t* vol,
                      uint32_t* acc, int w, int h);
void orc_wta(const apg_pipeline_config_t* cfg, const uint32_t* acc, const int16_t* rmin,
             const int16_t* rmax, int w, int h, float* disp, float* best, float* second);
void orc_wta_right(const apg_pipeline_config_t* cfg, const uint16_t* raw, int w, int h, float* disp_right);
void orc_confidence(const apg_pipeline_config_t* cfg, int w, int h, const float* disp,
                    const float* disp_right, const float* best, const float* second,
                    const uint8_t* lgx, const uint8_t* lgy,
                    float* conf, uint8_t* reliable, uint8_t* reason);
int  orc_refine_count(int w, int h, const uint8_t* reliable, const int16_t* rmin, const int16_t* rmax,
                      const float* work);
void orc_refine_pass(const apg_pipeline_config_t* cfg, int it, int w, int h,
                     const uint8_t* lgray, const uint8_t* lgx, const uint8_t* lgy,
                     const uint8_t* rgray, const uint8_t* rgx, const uint8_t* rgy,
                     const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                     const int16_t* rmin, const int16_t* rmax, const uint8_t* reliable,
                     const int* draws, float* work);
void orc_lr_check(const apg_pipeline_config_t* cfg, int w, int h, const float* disp_right,
                  float* disp, uint8_t* reason);
void orc_fill_holes(const apg_pipeline_config_t* cfg, int w, int h, const float* disp_in,
                    const uint8_t* reason, const uint8_t* lgray, const float* d_prior, float* disp_out);
void orc_median(const apg_pipeline_config_t* cfg, int w, int h, const float* disp_in, float* disp_out);

/* HighQuality sparse prior (src/prior_estimator.cpp). */
typedef struct { int x, y; float disparity, confidence; } orc_support_t;
int  orc_extract_supports(const apg_pipeline_config_t* cfg, int w, int h,
                          const uint8_t* lgx, const uint8_t* lgy,
                          const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                          orc_support_t* out, int out_cap);
void orc_interpolate_prior(int w, int h, const orc_support_t* s, int n,
                           float* d_prior, float* conf, float* spread, float* dmin, float* dmax);
void orc_apply_search_range(const apg_pipeline_config_t* cfg, int w, int h, const float* d_prior,
                            const float* conf, const float* spread, const float* dmin, const float* dmax,
                            int16_t* rmin, int16_t* rmax);

/* Draws of std::uniform_int_distribution<int>(-r, r) over one std::mt19937(seed) stream
 * (oracle/rng_draws.cpp calls the C++ standard library itself). */
void* orc_rng_create(uint32_t seed);
void  orc_rng_destroy(void* rng);
void  orc_rng_draws(void* rng, int radius, int n, int* out);

/* Whole pipeline, Dense semantics (src/pipeline.cpp:435-719).  Optional intermediate outputs
 * may be NULL.  Returns 0 or a reference StatusCode. */
typedef struct {
    float* disp_wta; float* best; float* second; float* disp_right;
    float* disp_refined; float* disp_lr; float* disp_fill;
    uint16_t* cost_raw; uint16_t* cost_agg; uint32_t* sgm_sum;
    int16_t* range_min; int16_t* range_max; float* d_prior;
    int support_count;
} orc_stages_t;
int orc_pipeline(const apg_pipeline_config_t* cfg, const uint8_t* left, const uint8_t* right,
                 int w, int h, int stride, int ch,
                 float* disparity, float* confidence, uint8_t* invalid_reason, uint8_t* reliable_mask,
                 orc_stages_t* stages);

/* Hierarchical coarse-to-fine search range (src/hierarchical_stereo.cpp:113-431).  lg / rg are
 * the full-size grays; coarse_disp / coarse_conf (nullable, (W/2)*(H/2)) receive the coarse pass's
 * final disparity and confidence.  Returns 0 for the small-frame fallback, 1 otherwise. */
void orc_hier_coarse_config(const apg_pipeline_config_t* cfg, apg_pipeline_config_t* coarse);
int  orc_hier_range(const apg_pipeline_config_t* cfg, int w, int h, const uint8_t* lg, const uint8_t* rg,
                    int16_t* rmin, int16_t* rmax, float* d_prior, int64_t* counts4,
                    float* coarse_disp, float* coarse_conf);

/* Accuracy metrics (src/metrics.cpp:119-502, without supports).  Any nullable input may be NULL. */
void orc_evaluate_stereo(const float* est, const float* gt, int w, int h, const int16_t* rmin, const int16_t* rmax,
                         const float* before, const float* after, const uint8_t* vis, float max_valid_gt,
                         const uint8_t* left, int left_stride, int left_ch, const apg_quality_thresholds_t* thr,
                         apg_stereo_metrics_t* out);

/* evaluate_supports (src/metrics.cpp:8-124). */
void orc_evaluate_supports(const orc_support_t* s, int n, const float* gt, int w, int h, const uint8_t* vis,
                           float max_valid_gt, int cell_size, apg_support_metrics_t* out);

/* Experimental scopes: sub-pixel method 0 Legacy, 1 CurvGate, 2 ConfGate, 3 Stabilized with its
 * parameter; inpaint method 0 Legacy, 1 ShadowReclass with its gap.  Defaults (0, 0, 0, 32). */
void orc_set_experimental(int sp_method, float sp_param, int ip_method, int ip_gap);
/* The scopes' telemetry: on/off, read, reset (the oracle's totals, over every pipeline run). */
void orc_set_telemetry(int subpixel, int inpaint);
void orc_get_telemetry(apg_subpixel_telemetry_t* sp, apg_inpaint_telemetry_t* ip);

uint64_t orc_fnv1a64(const uint8_t* data, uint64_t n);
void orc_config_from_mode(int mode, int max_disparity, apg_pipeline_config_t* out);

#ifdef __cplusplus
}
#endif
#endif

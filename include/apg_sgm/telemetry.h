/* Plain-C mirror of the experimental scopes' telemetry records: SubpixelTelemetry
 * (src/subpixel_estimator.hpp:50-118 of the reference) and InpaintTelemetry
 * (src/inpaint_internal.hpp:65-163), shared by the CUDA library (include/apg_sgm_cuda.h), the CPU
 * oracle and the reference shim under oracle/.  Every field is 8 bytes, so a device block of one
 * record of each is updated with 64-bit atomics.
 */
#ifndef APG_TELEMETRY_T_DEFINED
#define APG_TELEMETRY_T_DEFINED

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    unsigned long long candidate_pixels, applied_pixels, degenerate_count, clamped_count, negative_curvature_count;
    double sum_abs_delta;
    unsigned long long delta_buckets[50]; /* |delta| in [0.01 i, 0.01 (i + 1)), the last one up to 0.5 */
} apg_subpixel_telemetry_t;

/* FillRoute order (src/inpaint_internal.hpp:34-47): none, occ_both_min, occ_left_only,
 * occ_right_only, mismatch_color_horiz, mismatch_color_vert, mismatch_prior, mismatch_lerp,
 * mismatch_left_only, mismatch_right_only, remained_invalid. */
typedef struct {
    unsigned long long total_invalid_pixels, classified_occ_pixels, classified_mismatch_pixels, hit_max_gap_pixels,
        reclassified_shadow_pixels;
    unsigned long long route_counts[11];
    unsigned long long invalid_runs_count, invalid_runs_truncated;
    unsigned long long run_length_buckets[10]; /* [0,4) [4,8) [8,16) [16,24) [24,32) [32,48) [48,64) [64,96) [96,128) [128,) */
} apg_inpaint_telemetry_t;

#ifdef __cplusplus
}
#endif

#endif /* APG_TELEMETRY_T_DEFINED */

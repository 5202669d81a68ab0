/* CPU oracle for the apg-sgm dense-matching path: a plain-C99 restatement of the reference.
 *
 * TEST INFRASTRUCTURE ONLY (see apg_oracle.h).  Each function names the reference file:line it
 * restates.  Floating-point sites keep the reference's operation order; the library is built
 * with -ffp-contract=off (oracle/Makefile) so, like the reference's own -mavx2-only x86-64 build,
 * no multiply-add is ever contracted.  The cost LUT uses the host libm expf exactly as the
 * reference's std::exp(float) does (src/discrete_cost_lut.hpp:20-35).
 */
#include "apg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline float fmaxf_ref(float a, float b) { return (a < b) ? b : a; } /* std::max(a, b) */
static inline float fminf_ref(float a, float b) { return (b < a) ? b : a; } /* std::min(a, b) */

static inline uint8_t sample8(const uint8_t* img, int w, int h, int x, int y) {
    /* Image8::sample, src/image.cpp:15-19 */
    return img[clampi(y, 0, h - 1) * w + clampi(x, 0, w - 1)];
}

/* build_gray_and_grad, src/cost_computer.cpp:63-88, with ImageView8::gray
 * (include/apg_sgm/image_view.hpp:50-56). */
void orc_gray_grad(const uint8_t* src, int w, int h, int stride, int ch,
                   uint8_t* gray, uint8_t* gx, uint8_t* gy) {
    for (int y = 0; y < h; ++y) {
        const uint8_t* row = src + (size_t)y * stride;
        for (int x = 0; x < w; ++x) {
            if (ch == 1) {
                gray[y * w + x] = row[x];
            } else {
                const int r = row[x * ch + 0], g = row[x * ch + 1], b = row[x * ch + 2];
                gray[y * w + x] = (uint8_t)((77 * r + 150 * g + 29 * b) >> 8);
            }
        }
    }
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int gxv = (int)sample8(gray, w, h, x + 1, y) - (int)sample8(gray, w, h, x - 1, y);
            const int gyv = (int)sample8(gray, w, h, x, y + 1) - (int)sample8(gray, w, h, x, y - 1);
            gx[y * w + x] = (uint8_t)clampi(abs(gxv), 0, 255);
            gy[y * w + x] = (uint8_t)clampi(abs(gyv), 0, 255);
        }
    }
}

/* CostComputer::symmetric_census9x7, src/cost_computer.cpp:33-47. */
void orc_census_sym(const uint8_t* gray, int w, int h, uint32_t* out) {
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            uint32_t bits = 0;
            int b = 0;
            for (int dy = -3; dy <= 3; ++dy) {
                for (int dx = -4; dx <= 4; ++dx) {
                    if (dy < 0 || (dy == 0 && dx < 0)) {
                        const uint8_t a = sample8(gray, w, h, x + dx, y + dy);
                        const uint8_t c = sample8(gray, w, h, x - dx, y - dy);
                        if (a > c) bits |= (1u << b);
                        ++b;
                    }
                }
            }
            out[y * w + x] = bits;
        }
    }
}

/* CostComputer::census9x7, src/cost_computer.cpp:49-61. */
void orc_census64(const uint8_t* gray, int w, int h, uint64_t* out) {
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const uint8_t center = sample8(gray, w, h, x, y);
            uint64_t bits = 0;
            int b = 0;
            for (int dy = -3; dy <= 3; ++dy) {
                for (int dx = -4; dx <= 4; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    if (sample8(gray, w, h, x + dx, y + dy) > center) bits |= (1ull << b);
                    ++b;
                }
            }
            out[y * w + x] = bits;
        }
    }
}

/* SearchRange::set_pixel, include/apg_sgm/search_range.hpp:29-35. */
static inline void set_range(const apg_pipeline_config_t* cfg, int16_t* rmin, int16_t* rmax, int i,
                             int lo, int hi) {
    lo = imax(lo, cfg->min_disparity);
    hi = imin(hi, cfg->max_disparity);
    if (hi < lo) hi = lo;
    rmin[i] = (int16_t)lo;
    rmax[i] = (int16_t)hi;
}

/* PriorEstimator::estimate, range part, src/prior_estimator.cpp:414-424. */
void orc_range_default(const apg_pipeline_config_t* cfg, int w, int h, int16_t* rmin, int16_t* rmax) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
            set_range(cfg, rmin, rmax, y * w + x, cfg->min_disparity, imin(cfg->max_disparity, x + 1));
}

/* DiscreteCostLut, src/discrete_cost_lut.hpp:10-38. */
void orc_cost_lut(const apg_pipeline_config_t* cfg, float* census, float* ad, float* grad) {
    const float lc = fmaxf_ref(cfg->lambda_census, 1e-3f);
    const float la = fmaxf_ref(cfg->lambda_ad, 1e-3f);
    const float lg = fmaxf_ref(cfg->lambda_grad, 1e-3f);
    for (int i = 0; i <= 64; ++i) census[i] = 1.f - expf(-(float)i / lc);
    for (int i = 0; i < 256; ++i) ad[i] = cfg->use_ad ? cfg->eta_ad * (1.f - expf(-(float)i / la)) : 0.f;
    for (int i = 0; i < 511; ++i) grad[i] = cfg->use_grad ? cfg->mu_grad * (1.f - expf(-(float)i / lg)) : 0.f;
}

static float cost_scale(const apg_pipeline_config_t* cfg) {
    /* src/cost_computer.cpp:154-155 */
    const float norm = 1.f + (cfg->use_ad ? cfg->eta_ad : 0.f) + (cfg->use_grad ? cfg->mu_grad : 0.f);
    return (float)cfg->cost_max / fmaxf_ref(norm, 1e-6f);
}

static inline int popcount64(uint64_t v) { return __builtin_popcountll(v); }

/* Unquantised matching cost of (x, y) against (xr, y): LUT sum in the reference order
 * (src/cost_computer.cpp:176-197 dense, :247-262 packed, src/refiner.cpp:14-36). */
static inline float raw_cost(const apg_pipeline_config_t* cfg, const float* lc, const float* la,
                             const float* lg, int w, int x, int y, int xr,
                             const uint8_t* lgray, const uint8_t* lgx, const uint8_t* lgy,
                             const uint8_t* rgray, const uint8_t* rgx, const uint8_t* rgy,
                             const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64,
                             const uint64_t* cr64) {
    const int pop = cfg->census_type == APG_CENSUS_SYMMETRIC_9X7
                        ? __builtin_popcount(cl[y * w + x] ^ cr[y * w + xr])
                        : popcount64(cl64[y * w + x] ^ cr64[y * w + xr]);
    float c = lc[pop];
    if (cfg->use_ad) {
        const int ad = abs((int)lgray[y * w + x] - (int)rgray[y * w + xr]);
        c += la[ad];
    }
    if (cfg->use_grad) {
        const int g = abs((int)lgx[y * w + x] - (int)rgx[y * w + xr]) +
                      abs((int)lgy[y * w + x] - (int)rgy[y * w + xr]);
        c += lg[g];
    }
    return c;
}

/* CostComputer::compute_volume, src/cost_computer.cpp:139-203. */
void orc_cost_volume(const apg_pipeline_config_t* cfg, int w, int h,
                     const uint8_t* lgray, const uint8_t* lgx, const uint8_t* lgy,
                     const uint8_t* rgray, const uint8_t* rgx, const uint8_t* rgy,
                     const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                     const int16_t* rmin, const int16_t* rmax, uint16_t* vol) {
    float lc[65], la[256], lg[511];
    orc_cost_lut(cfg, lc, la, lg);
    const float scale = cost_scale(cfg);
    const int d0 = cfg->min_disparity, d1 = cfg->max_disparity, D = d1 - d0;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int lo = rmin[y * w + x], hi = rmax[y * w + x];
            uint16_t* s = vol + ((size_t)y * w + x) * D;
            for (int d = d0; d < d1; ++d) {
                const int di = d - d0;
                const int xr = x - d;
                if (d < lo || d >= hi || xr < 0 || xr >= w) {
                    s[di] = ORC_INVALID_COST;
                    continue;
                }
                const float c = raw_cost(cfg, lc, la, lg, w, x, y, xr, lgray, lgx, lgy, rgray, rgx, rgy,
                                         cl, cr, cl64, cr64);
                const int q = (int)(c * scale + 0.5f);
                s[di] = (uint16_t)clampi(q, 0, cfg->cost_max);
            }
        }
    }
}

/* CostAggregator::build_cross_arms, src/cost_aggregator.cpp:17-63. */
void orc_cross_arms(const uint8_t* gray, int w, int h, int max_arm, int tau,
                    int16_t* L, int16_t* R, int16_t* U, int16_t* Dn) {
    const int Lmax = imax(1, max_arm);
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int c0 = gray[y * w + x];
            int l = 0, r = 0, u = 0, v = 0;
            while (l < Lmax && x - l - 1 >= 0 && abs((int)gray[y * w + x - l - 1] - c0) <= tau) ++l;
            while (r < Lmax && x + r + 1 < w && abs((int)gray[y * w + x + r + 1] - c0) <= tau) ++r;
            while (u < Lmax && y - u - 1 >= 0 && abs((int)gray[(y - u - 1) * w + x] - c0) <= tau) ++u;
            while (v < Lmax && y + v + 1 < h && abs((int)gray[(y + v + 1) * w + x] - c0) <= tau) ++v;
            const int i = y * w + x;
            L[i] = (int16_t)l; R[i] = (int16_t)r; U[i] = (int16_t)u; Dn[i] = (int16_t)v;
        }
    }
}

/* CostAggregator::aggregate + aggregate_hv, src/cost_aggregator.cpp:65-149. */
void orc_cross_aggregate(const apg_pipeline_config_t* cfg, const uint8_t* gray, int w, int h,
                         const int16_t* rmin, const int16_t* rmax, uint16_t* vol) {
    if (!cfg->agg_enable) return;
    const int d0 = cfg->min_disparity, D = cfg->max_disparity - cfg->min_disparity;
    const size_t n = (size_t)w * h;
    int16_t* La = (int16_t*)malloc(n * 2); int16_t* Ra = (int16_t*)malloc(n * 2);
    int16_t* Ua = (int16_t*)malloc(n * 2); int16_t* Da = (int16_t*)malloc(n * 2);
    uint16_t* tmp = (uint16_t*)malloc(n * D * 2);
    orc_cross_arms(gray, w, h, cfg->max_arm_length, cfg->color_threshold, La, Ra, Ua, Da);
    const int iters = imax(1, cfg->agg_iterations);
    for (int it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                const int i = y * w + x;
                const int x0 = x - La[i], x1 = x + Ra[i];
                const int lo = rmin[i], hi = rmax[i];
                uint16_t* dst = tmp + (size_t)i * D;
                for (int di = 0; di < D; ++di) {
                    const int d = d0 + di;
                    if (d < lo || d >= hi) { dst[di] = ORC_INVALID_COST; continue; }
                    int acc = 0, cnt = 0;
                    for (int xx = x0; xx <= x1; ++xx) {
                        const int j = y * w + xx;
                        if (d < rmin[j] || d >= rmax[j]) continue;
                        const uint16_t c = vol[(size_t)j * D + di];
                        if (c == ORC_INVALID_COST) continue;
                        acc += c; ++cnt;
                    }
                    dst[di] = cnt > 0 ? (uint16_t)(acc / cnt) : ORC_INVALID_COST;
                }
            }
        }
#pragma omp parallel for schedule(static)
        for (int y = 0; y < h; ++y) {
            for (int x = 0; x < w; ++x) {
                const int i = y * w + x;
                const int y0 = y - Ua[i], y1 = y + Da[i];
                const int lo = rmin[i], hi = rmax[i];
                uint16_t* dst = vol + (size_t)i * D;
                for (int di = 0; di < D; ++di) {
                    const int d = d0 + di;
                    if (d < lo || d >= hi) { dst[di] = ORC_INVALID_COST; continue; }
                    int acc = 0, cnt = 0;
                    for (int yy = y0; yy <= y1; ++yy) {
                        const int j = yy * w + x;
                        if (d < rmin[j] || d >= rmax[j]) continue;
                        const uint16_t c = tmp[(size_t)j * D + di];
                        if (c == ORC_INVALID_COST) continue;
                        acc += c; ++cnt;
                    }
                    dst[di] = cnt > 0 ? (uint16_t)(acc / cnt) : ORC_INVALID_COST;
                }
            }
        }
    }
    free(La); free(Ra); free(Ua); free(Da); free(tmp);
}

/* detail::adaptive_p2, src/sgm_common.hpp:25-39. */
static int adaptive_p2(const apg_pipeline_config_t* p, int dI) {
    dI = abs(dI);
    int P2 = p->P2_base;
    if (!p->adaptive_penalties) return imax(P2, p->P1 + 1);
    if (p->piecewise_p2) {
        if (dI >= p->grad_t2) P2 = p->P2_base / 4;
        else if (dI >= p->grad_t1) P2 = p->P2_base / 2;
        else P2 = p->P2_base;
    } else {
        P2 = (int)((float)p->P2_base / (1.f + p->p2_alpha * (float)dI) + 0.5f);
    }
    return imax(P2, p->P1 + 1);
}

/* process_pixel (dense), src/sgm_optimizer.cpp:21-81. */
static void process_pixel(const apg_pipeline_config_t* cfg, const uint8_t* gray, const uint16_t* vol,
                          uint32_t* acc, int w, int D, int x, int y, int has_prev, int px, int py,
                          int* prev, int* cur) {
    const uint16_t* c = vol + ((size_t)y * w + x) * D;
    uint32_t* a = acc + ((size_t)y * w + x) * D;
    if (!has_prev) {
        for (int d = 0; d < D; ++d) {
            if (c[d] == ORC_INVALID_COST) {
                cur[d] = ORC_PATH_INF;
                a[d] = ORC_INVALID_COST32;
            } else {
                cur[d] = c[d];
                if (a[d] != ORC_INVALID_COST32) a[d] += (uint32_t)cur[d];
            }
        }
        memcpy(prev, cur, sizeof(int) * D);
        return;
    }
    const int dI = (int)gray[y * w + x] - (int)gray[py * w + px];
    const int P2 = adaptive_p2(cfg, dI);
    const int P1 = cfg->P1;
    int min_prev = ORC_PATH_INF;
    for (int d = 0; d < D; ++d) if (prev[d] < min_prev) min_prev = prev[d];
    for (int d = 0; d < D; ++d) {
        if (c[d] == ORC_INVALID_COST) {
            cur[d] = ORC_PATH_INF;
            a[d] = ORC_INVALID_COST32;
            continue;
        }
        int best = ORC_PATH_INF;
        if (prev[d] < ORC_PATH_INF) best = imin(best, prev[d]);
        if (d > 0 && prev[d - 1] < ORC_PATH_INF) best = imin(best, prev[d - 1] + P1);
        if (d + 1 < D && prev[d + 1] < ORC_PATH_INF) best = imin(best, prev[d + 1] + P1);
        if (min_prev < ORC_PATH_INF) best = imin(best, min_prev + P2);
        cur[d] = best >= ORC_PATH_INF ? (int)c[d] : (int)c[d] + best - min_prev;
        if (a[d] != ORC_INVALID_COST32) a[d] += (uint32_t)cur[d];
    }
    memcpy(prev, cur, sizeof(int) * D);
}

/* SgmOptimizer::aggregate_path, src/sgm_optimizer.cpp:186-259.  Each scanline (row, column or
 * diagonal ray) starts at the image border and walks in direction (dx, dy). */
void orc_sgm_path(const apg_pipeline_config_t* cfg, const uint8_t* gray, const uint16_t* vol,
                  uint32_t* acc, int w, int h, int D, int dx, int dy) {
    if (dy == 0) {
#pragma omp parallel for schedule(static)
        for (int y = 0; y < h; ++y) {
            int* prev = (int*)malloc(sizeof(int) * D); int* cur = (int*)malloc(sizeof(int) * D);
            if (dx == 1) for (int x = 0; x < w; ++x) process_pixel(cfg, gray, vol, acc, w, D, x, y, x > 0, x - 1, y, prev, cur);
            else for (int x = w - 1; x >= 0; --x) process_pixel(cfg, gray, vol, acc, w, D, x, y, x + 1 < w, x + 1, y, prev, cur);
            free(prev); free(cur);
        }
    } else if (dx == 0) {
#pragma omp parallel for schedule(static)
        for (int x = 0; x < w; ++x) {
            int* prev = (int*)malloc(sizeof(int) * D); int* cur = (int*)malloc(sizeof(int) * D);
            if (dy == 1) for (int y = 0; y < h; ++y) process_pixel(cfg, gray, vol, acc, w, D, x, y, y > 0, x, y - 1, prev, cur);
            else for (int y = h - 1; y >= 0; --y) process_pixel(cfg, gray, vol, acc, w, D, x, y, y + 1 < h, x, y + 1, prev, cur);
            free(prev); free(cur);
        }
    } else {
        /* Diagonal: every ray is entered at its first in-image pixel against (dx, dy).  Rays are
         * disjoint, so the per-ray order of the reference's serial raster discovery loop does not
         * change any value. */
        const int nrays = w + h - 1;
#pragma omp parallel for schedule(dynamic, 8)
        for (int r = 0; r < nrays; ++r) {
            int* prev = (int*)malloc(sizeof(int) * D); int* cur = (int*)malloc(sizeof(int) * D);
            int x, y;
            /* start pixel: the border pixel whose predecessor (x - dx, y - dy) is outside */
            if (r < w) { x = r; y = (dy == 1) ? 0 : h - 1; }
            else { x = (dx == 1) ? 0 : w - 1; y = (dy == 1) ? (r - w + 1) : (h - 1 - (r - w + 1)); }
            int hp = 0, px = x, py = y;
            while (x >= 0 && x < w && y >= 0 && y < h) {
                process_pixel(cfg, gray, vol, acc, w, D, x, y, hp, px, py, prev, cur);
                hp = 1; px = x; py = y; x += dx; y += dy;
            }
            free(prev); free(cur);
        }
    }
}

/* SgmOptimizer::optimize, src/sgm_optimizer.cpp:261-274. */
void orc_sgm_optimize(const apg_pipeline_config_t* cfg, const uint8_t* gray, const uint16_t* vol,
                      uint32_t* acc, int w, int h) {
    static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    const int D = cfg->max_disparity - cfg->min_disparity;
    memset(acc, 0, sizeof(uint32_t) * (size_t)w * h * D);
    const int npath = cfg->paths == 8 ? 8 : 4;
    for (int p = 0; p < npath; ++p) orc_sgm_path(cfg, gray, vol, acc, w, h, D, dirs[p][0], dirs[p][1]);
}

/* SubpixelEstimator::compute_legacy_delta, src/subpixel_estimator.hpp:115-124. */
static float legacy_delta(float cm, float c0, float cp) {
    const float denom = cm - 2.0f * c0 + cp;
    if (fabsf(denom) > 1e-6f) {
        const float delta = 0.5f * (cm - cp) / denom;
        if (delta < -0.5f) return -0.5f;
        if (delta > 0.5f) return 0.5f;
        return delta;
    }
    return 0.0f;
}

/* Experimental scopes (ExperimentalSubpixelScope, src/subpixel_estimator.cpp:7-57;
 * ExperimentalInpaintScope, src/postprocess.cpp:42-53), process-wide in the oracle. */
static int g_sp_method = 0, g_ip_method = 0, g_ip_gap = 32;
static float g_sp_param = 0.0f;

void orc_set_experimental(int sp_method, float sp_param, int ip_method, int ip_gap) {
    g_sp_method = sp_method;
    g_sp_param = sp_param;
    g_ip_method = ip_method;
    g_ip_gap = ip_gap;
}

static int g_sp_tel = 0, g_ip_tel = 0;
static apg_subpixel_telemetry_t g_spt;
static apg_inpaint_telemetry_t g_ipt;

/* Telemetry on/off; switching on clears the totals (the scopes' constructors reset them). */
void orc_set_telemetry(int subpixel, int inpaint) {
    g_sp_tel = subpixel;
    g_ip_tel = inpaint;
    if (subpixel) memset(&g_spt, 0, sizeof(g_spt));
    if (inpaint) memset(&g_ipt, 0, sizeof(g_ipt));
}

void orc_get_telemetry(apg_subpixel_telemetry_t* sp, apg_inpaint_telemetry_t* ip) {
    if (sp) *sp = g_spt;
    if (ip) *ip = g_ipt;
}

/* compute_delta with telemetry, src/subpixel_estimator.cpp:58-134. */
static float sp_delta_tel(float cm, float c0, float cp, float uniq) {
    apg_subpixel_telemetry_t* t = &g_spt;
    t->candidate_pixels++;
    const float denom = cm - 2.0f * c0 + cp;
    const int non_convex = c0 >= cm || c0 >= cp || denom <= 1e-6f;
    if (non_convex) {
        t->negative_curvature_count++;
        if (fabsf(denom) <= 1e-6f || (cm == c0 && c0 == cp)) t->degenerate_count++;
    }
    float raw = 0.0f, delta = 0.0f;
    int apply;
    float den = denom;
    if (g_sp_method == 0) apply = fabsf(denom) > 1e-6f;
    else if (g_sp_method == 1) apply = !non_convex && denom >= (g_sp_param > 0.0f ? g_sp_param : 4.0f);
    else if (g_sp_method == 2) apply = !non_convex && uniq >= (g_sp_param > 0.0f ? g_sp_param : 0.05f);
    else {
        apply = c0 <= cm && c0 <= cp && denom > 0.0f;
        den = denom + (g_sp_param > 0.0f ? g_sp_param : 4.0f);
    }
    if (apply) {
        raw = 0.5f * (cm - cp) / den;
        delta = raw < -0.5f ? -0.5f : (0.5f < raw ? 0.5f : raw);
    }
    if (fabsf(delta) > 1e-5f) {
        const float a = fabsf(delta);
        t->applied_pixels++;
        t->sum_abs_delta += a;
        t->delta_buckets[imin(49, (int)(a * 100.0f))]++;
    }
    if (fabsf(raw) >= 0.5f) t->clamped_count++;
    return delta;
}

/* SubpixelEstimator::compute_delta without telemetry, src/subpixel_estimator.cpp:58-119. */
static float sp_delta(float cm, float c0, float cp, float uniq) {
    if (g_sp_method == 0) return legacy_delta(cm, c0, cp);
    const float denom = cm - 2.0f * c0 + cp;
    const int non_convex = c0 >= cm || c0 >= cp || denom <= 1e-6f;
    float raw;
    if (g_sp_method == 1) {
        if (non_convex || !(denom >= (g_sp_param > 0.0f ? g_sp_param : 4.0f))) return 0.0f;
        raw = 0.5f * (cm - cp) / denom;
    } else if (g_sp_method == 2) {
        if (non_convex || !(uniq >= (g_sp_param > 0.0f ? g_sp_param : 0.05f))) return 0.0f;
        raw = 0.5f * (cm - cp) / denom;
    } else {
        if (!(c0 <= cm && c0 <= cp && denom > 0.0f)) return 0.0f;
        raw = 0.5f * (cm - cp) / (denom + (g_sp_param > 0.0f ? g_sp_param : 4.0f));
    }
    return raw < -0.5f ? -0.5f : (0.5f < raw ? 0.5f : raw);
}

/* wta_impl<uint32_t>, src/sgm_optimizer.cpp:436-555 (sub-pixel step as the scope selects, no
 * telemetry). */
void orc_wta(const apg_pipeline_config_t* cfg, const uint32_t* acc, const int16_t* rmin,
             const int16_t* rmax, int w, int h, float* disp, float* best_out, float* second_out) {
    const int d0 = cfg->min_disparity, D = cfg->max_disparity - cfg->min_disparity;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int i = y * w + x;
            const uint32_t* s = acc + (size_t)i * D;
            const int lo = rmin[i], hi = rmax[i];
            disp[i] = -1.f;
            if (best_out) best_out[i] = INFINITY;
            if (second_out) second_out[i] = INFINITY;
            if (hi <= lo) continue;
            int best_d = -1;
            uint64_t best = UINT64_MAX;
            for (int d = lo; d < hi; ++d) {
                const int di = d - d0;
                if (di < 0 || di >= D) continue;
                const uint32_t c = s[di];
                if (c == ORC_INVALID_COST32) continue;
                if ((uint64_t)c < best) { best = c; best_d = d; }
            }
            if (best_d < 0) continue;
            uint64_t second = UINT64_MAX;
            for (int d = lo; d < hi; ++d) {
                if (abs(d - best_d) <= 1) continue;
                const int di = d - d0;
                if (di < 0 || di >= D) continue;
                const uint32_t c = s[di];
                if (c == ORC_INVALID_COST32) continue;
                if ((uint64_t)c < second) second = c;
            }
            float dval = (float)best_d;
            if (cfg->subpixel && best_d - 1 >= lo && best_d + 1 < hi) {
                const int di = best_d - d0;
                if (di > 0 && di + 1 < D) {
                    const uint32_t cm = s[di - 1], c0 = s[di], cp = s[di + 1];
                    if (cm != ORC_INVALID_COST32 && cp != ORC_INVALID_COST32) {
                        float u = 1.0f;
                        if (second < UINT64_MAX) u = (float)(second - best) / (float)(best > 1 ? best : 1);
                        dval += g_sp_tel ? sp_delta_tel((float)cm, (float)c0, (float)cp, u)
                                         : sp_delta((float)cm, (float)c0, (float)cp, u);
                    }
                }
            }
            disp[i] = dval;
            if (best_out) best_out[i] = (float)best;
            if (second_out) second_out[i] = second < UINT64_MAX ? (float)second : INFINITY;
        }
    }
}

/* wta_right_from_left_volume, src/pipeline.cpp:24-85 (on the pre-Cross volume). */
void orc_wta_right(const apg_pipeline_config_t* cfg, const uint16_t* vol, int w, int h, float* dr) {
    const int d0 = cfg->min_disparity, D = cfg->max_disparity - cfg->min_disparity;
    for (int y = 0; y < h; ++y) {
        for (int xr = 0; xr < w; ++xr) {
            int best_d = -1;
            uint32_t best = UINT32_MAX;
            for (int d = d0; d < d0 + D; ++d) {
                const int xl = xr + d;
                if (xl < 0 || xl >= w) continue;
                const uint16_t c = vol[((size_t)y * w + xl) * D + (d - d0)];
                if (c == ORC_INVALID_COST) continue;
                if (c < best) { best = c; best_d = d; }
            }
            float dval = -1.f;
            if (best_d >= 0) {
                dval = (float)best_d;
                if (cfg->subpixel) {
                    const int di = best_d - d0;
                    const int xm = xr + best_d - 1, x0 = xr + best_d, xp = xr + best_d + 1;
                    if (xm >= 0 && xm < w && x0 >= 0 && x0 < w && xp >= 0 && xp < w && di > 0 && di + 1 < D) {
                        const uint16_t cm = vol[((size_t)y * w + xm) * D + di - 1];
                        const uint16_t c0 = vol[((size_t)y * w + x0) * D + di];
                        const uint16_t cp = vol[((size_t)y * w + xp) * D + di + 1];
                        if (cm != ORC_INVALID_COST && c0 != ORC_INVALID_COST && cp != ORC_INVALID_COST)
                            dval += sp_delta((float)cm, (float)c0, (float)cp, 1.0f);
                    }
                }
            }
            dr[y * w + xr] = dval;
        }
    }
}

/* ConfidenceEstimator::estimate, src/confidence_estimator.cpp:7-63. */
void orc_confidence(const apg_pipeline_config_t* cfg, int w, int h, const float* disp,
                    const float* disp_right, const float* best, const float* second,
                    const uint8_t* lgx, const uint8_t* lgy,
                    float* conf_out, uint8_t* reliable, uint8_t* reason) {
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int i = y * w + x;
            const float c1 = best[i], c2 = second[i];
            float uniq = 0.f;
            if (isfinite(c1) && isfinite(c2)) {
                uniq = (c2 - c1) / fmaxf_ref(c2, 1e-3f);
                uniq = clampf(uniq, 0.f, 1.f);
            }
            float lr = 1.f;
            if (disp_right) {
                const float d = disp[i];
                const int xr = (int)roundf((float)x - d);
                if (xr < 0 || xr >= w || d < 0.f) {
                    lr = 0.f;
                } else {
                    const float dr = disp_right[y * w + xr];
                    if (dr < 0.f || fabsf(d - dr) > (float)cfg->conf_lr_max_diff + 0.5f) lr = 0.f;
                }
            }
            const float tex = (float)(lgx[i] + lgy[i]);
            const float tex_term = clampf(tex / 16.f, 0.f, 1.f);
            float conf = clampf(uniq, 0.f, 4.f);
            conf = conf * (0.5f + 0.5f * tex_term);
            if (lr < 0.5f) conf *= 0.25f;
            conf_out[i] = conf;
            const int lr_ok = lr >= 0.5f;
            const int rel = lr_ok && conf >= cfg->conf_reliable_threshold &&
                            uniq >= cfg->conf_uniqueness_ratio && tex >= cfg->conf_min_texture &&
                            disp[i] >= 0.f;
            reliable[i] = rel ? 1 : 0;
            reason[i] = rel ? ORC_VALID : (lr_ok ? ORC_LOW_CONFIDENCE : ORC_MISMATCH);
        }
    }
}

/* Number of pixels that consume one random draw in a refine pass (src/refiner.cpp:62-84):
 * unreliable, non-empty range, current value >= 0.  The value tested is the one the pixel had
 * at the end of the previous pass, because a pass reads a pixel before writing it. */
int orc_refine_count(int w, int h, const uint8_t* reliable, const int16_t* rmin, const int16_t* rmax,
                     const float* work) {
    int n = 0;
    for (int i = 0; i < w * h; ++i)
        if (!reliable[i] && rmax[i] > rmin[i] && work[i] >= 0.f) ++n;
    return n;
}

/* One pass of detail::refine_scalar, src/refiner.cpp:42-100.  draws[k] is the k-th draw of this
 * pass in raster order of the pass (forward on even it, backward on odd it). */
void orc_refine_pass(const apg_pipeline_config_t* cfg, int it, int w, int h,
                     const uint8_t* lgray, const uint8_t* lgx, const uint8_t* lgy,
                     const uint8_t* rgray, const uint8_t* rgx, const uint8_t* rgy,
                     const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                     const int16_t* rmin, const int16_t* rmax, const uint8_t* reliable,
                     const int* draws, float* work) {
    float lc[65], la[256], lg[511];
    orc_cost_lut(cfg, lc, la, lg);
    const int fwd = (it % 2) == 0;
    const int y0 = fwd ? 0 : h - 1, y1 = fwd ? h : -1, ys = fwd ? 1 : -1;
    const int x0 = fwd ? 0 : w - 1, x1 = fwd ? w : -1, xs = fwd ? 1 : -1;
    int k = 0;
    for (int y = y0; y != y1; y += ys) {
        for (int x = x0; x != x1; x += xs) {
            const int i = y * w + x;
            if (reliable[i]) continue;
            const int lo = rmin[i], hi = rmax[i];
            if (hi <= lo) continue;
            const float cur = work[i];
            int cand[6], n = 0;
            float vals[4];
            int nv = 0;
            vals[nv++] = cur;
            if (fwd) {
                if (x > 0) vals[nv++] = work[i - 1];
                if (y > 0) vals[nv++] = work[i - w];
            } else {
                if (x + 1 < w) vals[nv++] = work[i + 1];
                if (y + 1 < h) vals[nv++] = work[i + w];
            }
            if (cur >= 0.f) vals[nv++] = cur + (float)draws[k++];
            for (int j = 0; j < nv; ++j)
                if (!(vals[j] < 0.f)) cand[n++] = clampi((int)roundf(vals[j]), lo, hi - 1);
            float best_c = 1e9f;
            int best_d = cur >= 0.f ? clampi((int)roundf(cur), lo, hi - 1) : lo;
            for (int j = 0; j < n; ++j) {
                const int d = cand[j];
                const int xr = x - d;
                float c;
                if (xr < 0 || xr >= w || d < lo || d >= hi) c = 1e6f;
                else c = raw_cost(cfg, lc, la, lg, w, x, y, xr, lgray, lgx, lgy, rgray, rgx, rgy, cl, cr, cl64, cr64);
                if (c < best_c) { best_c = c; best_d = d; }
            }
            work[i] = (float)best_d;
        }
    }
}

/* PostProcessor::left_right_check, src/postprocess.cpp:10-40. */
void orc_lr_check(const apg_pipeline_config_t* cfg, int w, int h, const float* dr_img, float* disp,
                  uint8_t* reason) {
    if (!cfg->lr_check || !dr_img) return;
    const float tol = (float)cfg->post_lr_max_diff + 0.5f;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int i = y * w + x;
            const float d = disp[i];
            if (d < 0.f) continue;
            const int xr = (int)roundf((float)x - d);
            if (xr < 0 || xr >= w) { disp[i] = -1.f; reason[i] = ORC_OCCLUSION; continue; }
            const float dr = dr_img[y * w + xr];
            if (dr < 0.f || fabsf(d - dr) > tol) {
                disp[i] = -1.f;
                reason[i] = (dr > d + tol) ? ORC_OCCLUSION : ORC_MISMATCH;
            }
        }
    }
}

/* PostProcessor::fill_holes, Legacy route, src/postprocess.cpp:42-168 and :252. */
void orc_fill_holes(const apg_pipeline_config_t* cfg, int w, int h, const float* in,
                    const uint8_t* reason, const uint8_t* lgray, const float* d_prior, float* out) {
    /* the inpaint scope's gap replaces max_fill_gap unless it is Legacy at 32 (postprocess.cpp:45-48) */
    const int gap = (g_ip_method == 0 && g_ip_gap == 32) ? cfg->max_fill_gap : g_ip_gap;
    apg_inpaint_telemetry_t* t = g_ip_tel ? &g_ipt : NULL;
    memcpy(out, in, sizeof(float) * (size_t)w * h);
    for (int y = 0; y < h; ++y) {
        if (t) { /* run statistics, postprocess.cpp:64-85 */
            int len = 0;
            for (int x = 0; x <= w; ++x) {
                if (x < w && in[y * w + x] < 0.f) { ++len; continue; }
                if (len > 0) {
                    t->invalid_runs_count++;
                    if (len > gap) t->invalid_runs_truncated++;
                    t->run_length_buckets[len < 4 ? 0 : len < 8 ? 1 : len < 16 ? 2 : len < 24 ? 3 : len < 32 ? 4
                                          : len < 48 ? 5 : len < 64 ? 6 : len < 96 ? 7 : len < 128 ? 8 : 9]++;
                    len = 0;
                }
            }
        }
        for (int x = 0; x < w; ++x) {
            const int i = y * w + x;
            if (in[i] >= 0.f) continue;
            int xl = x - 1;
            while (xl >= 0 && xl >= x - gap && in[y * w + xl] < 0.f) --xl;
            int xr = x + 1;
            while (xr < w && xr <= x + gap && in[y * w + xr] < 0.f) ++xr;
            const float dl = (xl >= 0 && in[y * w + xl] >= 0.f) ? in[y * w + xl] : -1.f;
            const float dr = (xr < w && in[y * w + xr] >= 0.f) ? in[y * w + xr] : -1.f;
            if (t) {
                t->total_invalid_pixels++;
                if (reason[i] == ORC_OCCLUSION) t->classified_occ_pixels++;
                else if (reason[i] == ORC_MISMATCH) t->classified_mismatch_pixels++;
                if (xl < 0 || x - xl > gap || xr >= w || xr - x > gap) t->hit_max_gap_pixels++;
            }
            int route;
            /* ShadowReclass (postprocess.cpp:170-192): a mismatch between valid neighbours >= 4 px
             * apart is filled like an occlusion */
            const int shadow = g_ip_method == 1 && reason[i] == ORC_MISMATCH && dl >= 0.f && dr >= 0.f &&
                               fabsf(dr - dl) >= 4.0f;
            if (reason[i] == ORC_OCCLUSION || shadow) {
                if (t && shadow) t->reclassified_shadow_pixels++;
                if (dl >= 0.f && dr >= 0.f) { out[i] = fminf_ref(dl, dr); route = 1; }
                else if (dl >= 0.f) { out[i] = dl; route = 2; }
                else if (dr >= 0.f) { out[i] = dr; route = 3; }
                else route = 10;
                if (t) t->route_counts[route]++;
                continue;
            }
            const int c0 = lgray[i];
            float best_d = -1.f;
            int best_abs = 999, best_vert = 0;
            const int cx[4] = {xl, xr, x, x};
            const int cy[4] = {y, y, y - 1, y + 1};
            const int en[4] = {1, 1, y > 0, y + 1 < h};
            for (int k = 0; k < 4; ++k) {
                if (!en[k]) continue;
                const int xx = cx[k], yy = cy[k];
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                const float d = in[yy * w + xx];
                if (d < 0.f) continue;
                const int ad = abs((int)lgray[yy * w + xx] - c0);
                if (ad < best_abs) { best_abs = ad; best_d = d; best_vert = k >= 2; }
            }
            if (best_d >= 0.f && best_abs <= 18) {
                out[i] = best_d;
                route = best_vert ? 5 : 4;
            } else if (d_prior && d_prior[i] >= 0.f) {
                out[i] = d_prior[i];
                route = 6;
            } else if (dl >= 0.f && dr >= 0.f) {
                const float tt = (float)(x - xl) / (float)(xr - xl);
                out[i] = dl * (1.f - tt) + dr * tt;
                route = 7;
            } else if (dl >= 0.f) {
                out[i] = dl;
                route = 8;
            } else if (dr >= 0.f) {
                out[i] = dr;
                route = 9;
            } else {
                route = 10;
            }
            if (t) t->route_counts[route]++;
        }
    }
}

static int cmp_float(const void* a, const void* b) {
    const float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

/* PostProcessor::median, src/postprocess.cpp:255-309: the size/2-th smallest valid value of the
 * (2r+1)^2 window; pixels without any valid neighbour keep their value. */
void orc_median(const apg_pipeline_config_t* cfg, int w, int h, const float* in, float* out) {
    const int r = cfg->median_radius;
    memcpy(out, in, sizeof(float) * (size_t)w * h);
    if (r <= 0) return;
    float* win = (float*)malloc(sizeof(float) * (2 * r + 1) * (2 * r + 1));
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            int n = 0;
            for (int oy = -r; oy <= r; ++oy)
                for (int ox = -r; ox <= r; ++ox) {
                    const int xx = x + ox, yy = y + oy;
                    if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                    const float d = in[yy * w + xx];
                    if (d >= 0.f) win[n++] = d;
                }
            if (n == 0) continue;
            qsort(win, n, sizeof(float), cmp_float);
            out[y * w + x] = win[n / 2];
        }
    }
    free(win);
}

/* ---------------------------------------------------------------------------------------------
 * HighQuality sparse prior, src/prior_estimator.cpp:13-412.
 * ------------------------------------------------------------------------------------------- */

/* PriorEstimator::extract_supports, src/prior_estimator.cpp:13-168. */
int orc_extract_supports(const apg_pipeline_config_t* cfg, int w, int h,
                         const uint8_t* lgx, const uint8_t* lgy,
                         const uint32_t* cl, const uint32_t* cr, const uint64_t* cl64, const uint64_t* cr64,
                         orc_support_t* out, int out_cap) {
    const int d0 = cfg->min_disparity, d1 = cfg->max_disparity;
    const int sym = cfg->census_type == APG_CENSUS_SYMMETRIC_9X7;
    const int cell = 16, step = 2;
    const int gw = (w + cell - 1) / cell, gh = (h + cell - 1) / cell, n_cells = gw * gh;
    const int hard_max = cfg->prior_max_supports;
    const int max_cand = imax(8, (hard_max * 2 + n_cells - 1) / imax(1, n_cells));
    orc_support_t* cand = (orc_support_t*)malloc(sizeof(orc_support_t) * (size_t)n_cells * max_cand);
    int* ncand = (int*)calloc(n_cells, sizeof(int));
    for (int ci = 0; ci < n_cells; ++ci) {
        const int gx = ci % gw, gy = ci / gw;
        const int y_min = imax(2, gy * cell), y_max = imin(h - 2, (gy + 1) * cell);
        const int y_start = (y_min % 2 != 0) ? y_min + 1 : y_min;
        const int x_min = imax(2, gx * cell), x_max = imin(w - 2, (gx + 1) * cell);
        const int x_start = (x_min % 2 != 0) ? x_min + 1 : x_min;
        for (int y = y_start; y < y_max; y += step) {
            for (int x = x_start; x < x_max; x += step) {
                if (ncand[ci] >= max_cand) continue;
                const int tex = (int)lgx[y * w + x] + (int)lgy[y * w + x];
                if (tex < cfg->prior_texture_threshold) continue;
                int best_d = d0, best = 255, second = 255;
                for (int d = d0; d < d1; ++d) {
                    const int xr = x - d;
                    if (xr < 0 || xr >= w) continue;
                    const int c = sym ? __builtin_popcount(cl[y * w + x] ^ cr[y * w + xr])
                                      : popcount64(cl64[y * w + x] ^ cr64[y * w + xr]);
                    if (c < best) { second = best; best = c; best_d = d; }
                    else if (c < second) second = c;
                }
                if (second <= 0) continue;
                const float uniq = (float)(second - best) / (float)second;
                if (uniq < cfg->prior_uniqueness_ratio) continue;
                const int xr = x - best_d;
                if (xr < 1 || xr >= w - 1) continue;
                int rbest = 255, rbest_d = 0;
                for (int d = d0; d < d1; ++d) {
                    const int xl = xr + d;
                    if (xl < 0 || xl >= w) continue;
                    const int c = sym ? __builtin_popcount(cl[y * w + xl] ^ cr[y * w + xr])
                                      : popcount64(cl64[y * w + xl] ^ cr64[y * w + xr]);
                    if (c < rbest) { rbest = c; rbest_d = d; }
                }
                if (abs(rbest_d - best_d) > cfg->prior_lr_max_diff) continue;
                orc_support_t m = {x, y, (float)best_d, uniq};
                cand[(size_t)ci * max_cand + ncand[ci]++] = m;
            }
        }
    }
    int n_out = 0;
    int* nonempty = (int*)malloc(sizeof(int) * n_cells);
    int nne = 0;
    for (int i = 0; i < n_cells; ++i) if (ncand[i] > 0) nonempty[nne++] = i;
    if (nne <= hard_max) {
        int* taken = (int*)calloc(n_cells, sizeof(int));
        const int base_quota = imax(1, hard_max / imax(1, nne));
        for (int k = 0; k < nne; ++k) {
            const int ci = nonempty[k];
            const int take = imin(base_quota, ncand[ci]);
            for (int j = 0; j < take && n_out < hard_max; ++j) {
                if (n_out < out_cap) out[n_out] = cand[(size_t)ci * max_cand + j];
                ++n_out; taken[ci]++;
            }
        }
        int added = 1;
        while (added && n_out < hard_max) {
            added = 0;
            for (int k = 0; k < nne; ++k) {
                if (n_out >= hard_max) break;
                const int ci = nonempty[k];
                if (taken[ci] < ncand[ci]) {
                    if (n_out < out_cap) out[n_out] = cand[(size_t)ci * max_cand + taken[ci]];
                    ++n_out; taken[ci]++; added = 1;
                }
            }
        }
        free(taken);
    } else {
        for (int k = 0; k < hard_max; ++k) {
            const size_t idx = ((uint64_t)k * (uint64_t)nne) / (uint64_t)hard_max;
            const int ci = nonempty[idx];
            if (n_out < out_cap) out[n_out] = cand[(size_t)ci * max_cand];
            ++n_out;
        }
    }
    free(nonempty); free(cand); free(ncand);
    return n_out;
}

typedef struct { float first, second; } pairf;

/* Stable insertion sort by .first ascending.  The reference calls std::sort; for up to 16
 * elements libstdc++'s std::sort is a plain insertion sort, so this order is the reference's
 * order whenever a 16x16 cell holds at most 16 supports (every image of 500+ cells). */
static void sort_pairs(pairf* a, int n) {
    for (int i = 1; i < n; ++i) {
        pairf v = a[i];
        int j = i - 1;
        while (j >= 0 && v.first < a[j].first) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
}

/* PriorEstimator::interpolate_prior, src/prior_estimator.cpp:170-365. */
void orc_interpolate_prior(int w, int h, const orc_support_t* s, int n,
                           float* d_prior, float* pconf, float* pspread, float* pmin, float* pmax) {
    const size_t np = (size_t)w * h;
    for (size_t i = 0; i < np; ++i) { d_prior[i] = -1.f; pconf[i] = 0.f; pspread[i] = 999.f; pmin[i] = -1.f; pmax[i] = -1.f; }
    if (n <= 0) return;
    const int cell = 16;
    const int gw = (w + cell - 1) / cell, gh = (h + cell - 1) / cell, n_cells = gw * gh;
    int* cnt = (int*)calloc(n_cells, sizeof(int));
    for (int k = 0; k < n; ++k) {
        const int gx = clampi(s[k].x / cell, 0, gw - 1), gy = clampi(s[k].y / cell, 0, gh - 1);
        cnt[gy * gw + gx]++;
    }
    int* off = (int*)malloc(sizeof(int) * (n_cells + 1));
    off[0] = 0;
    for (int i = 0; i < n_cells; ++i) off[i + 1] = off[i] + cnt[i];
    pairf* pts = (pairf*)malloc(sizeof(pairf) * n);
    pairf* devs = (pairf*)malloc(sizeof(pairf) * n);
    memset(cnt, 0, sizeof(int) * n_cells);
    for (int k = 0; k < n; ++k) {
        const int gx = clampi(s[k].x / cell, 0, gw - 1), gy = clampi(s[k].y / cell, 0, gh - 1);
        const int ci = gy * gw + gx;
        pts[off[ci] + cnt[ci]++] = (pairf){s[k].disparity, s[k].confidence};
    }
    float* gd = (float*)malloc(sizeof(float) * n_cells);
    float* gc = (float*)malloc(sizeof(float) * n_cells);
    float* gs = (float*)malloc(sizeof(float) * n_cells);
    float* gmn = (float*)malloc(sizeof(float) * n_cells);
    float* gmx = (float*)malloc(sizeof(float) * n_cells);
    for (int i = 0; i < n_cells; ++i) { gd[i] = -1.f; gc[i] = 0.f; gs[i] = -1.f; gmn[i] = -1.f; gmx[i] = -1.f; }
    for (int i = 0; i < n_cells; ++i) {
        const int m = off[i + 1] - off[i];
        if (m == 0) continue;
        pairf* p = pts + off[i];
        sort_pairs(p, m);
        gmn[i] = p[0].first;
        gmx[i] = p[m - 1].first;
        const float intra_span = gmx[i] - gmn[i];
        float total_w = 0.f;
        for (int k = 0; k < m; ++k) total_w += p[k].second;
        if (total_w <= 1e-6f) continue;
        const float half_w = total_w * 0.5f;
        float cur_w = 0.f;
        float d_med = p[0].first;
        for (int k = 0; k < m; ++k) { cur_w += p[k].second; if (cur_w >= half_w) { d_med = p[k].first; break; } }
        gd[i] = d_med;
        pairf* dv = devs + off[i];
        for (int k = 0; k < m; ++k) dv[k] = (pairf){fabsf(p[k].first - d_med), p[k].second};
        sort_pairs(dv, m);
        cur_w = 0.f;
        float dev_med = dv[0].first;
        for (int k = 0; k < m; ++k) { cur_w += dv[k].second; if (cur_w >= half_w) { dev_med = dv[k].first; break; } }
        gs[i] = fmaxf_ref(dev_med * 1.4826f, intra_span * 0.5f);
        const float mean_conf = total_w / (float)m;
        const float count_factor = clampf((float)m / 3.f, 0.3f, 1.f);
        gc[i] = clampf(mean_conf * count_factor, 0.f, 1.f);
    }
    /* fill_grids, :253-301 */
    float* nd = (float*)malloc(sizeof(float) * n_cells);
    float* nc = (float*)malloc(sizeof(float) * n_cells);
    float* ns = (float*)malloc(sizeof(float) * n_cells);
    float* nmn = (float*)malloc(sizeof(float) * n_cells);
    float* nmx = (float*)malloc(sizeof(float) * n_cells);
    const int max_iters = imax(gw, gh);
    for (int iter = 0; iter < max_iters; ++iter) {
        memcpy(nd, gd, sizeof(float) * n_cells); memcpy(nc, gc, sizeof(float) * n_cells);
        memcpy(ns, gs, sizeof(float) * n_cells); memcpy(nmn, gmn, sizeof(float) * n_cells);
        memcpy(nmx, gmx, sizeof(float) * n_cells);
        int changed = 0;
        for (int gy = 0; gy < gh; ++gy) {
            for (int gx = 0; gx < gw; ++gx) {
                const int i = gy * gw + gx;
                if (gd[i] >= 0.f) continue;
                float ad = 0.f, ac = 0.f, as = 0.f, ww = 0.f, cmin = 1e9f, cmax = -1e9f;
                for (int oy = -1; oy <= 1; ++oy)
                    for (int ox = -1; ox <= 1; ++ox) {
                        const int nx = gx + ox, ny = gy + oy;
                        if (nx < 0 || ny < 0 || nx >= gw || ny >= gh) continue;
                        const int ni = ny * gw + nx;
                        const float v = gd[ni];
                        if (v < 0.f) continue;
                        ad += v;
                        ac += gc[ni];
                        as += (gs[ni] >= 0.f ? gs[ni] : 8.f);
                        cmin = fminf_ref(cmin, gmn[ni] >= 0.f ? gmn[ni] : v);
                        cmax = fmaxf_ref(cmax, gmx[ni] >= 0.f ? gmx[ni] : v);
                        ww += 1.f;
                    }
                if (ww > 0.f) {
                    nd[i] = ad / ww;
                    nc[i] = (ac / ww) * 0.85f;
                    ns[i] = as / ww;
                    nmn[i] = cmin;
                    nmx[i] = cmax;
                    changed = 1;
                }
            }
        }
        float* t;
        t = gd; gd = nd; nd = t; t = gc; gc = nc; nc = t; t = gs; gs = ns; ns = t;
        t = gmn; gmn = nmn; nmn = t; t = gmx; gmx = nmx; nmx = t;
        if (!changed) break;
    }
    /* bilinear, :303-364 */
    for (int y = 0; y < h; ++y) {
        const float fy = ((float)y + 0.5f) / cell - 0.5f;
        const int gy = clampi((int)floorf(fy), 0, gh - 1);
        const int gy1 = imin(gy + 1, gh - 1);
        const float ty = clampf(fy - (float)gy, 0.f, 1.f);
        for (int x = 0; x < w; ++x) {
            const float fx = ((float)x + 0.5f) / cell - 0.5f;
            const int gx = clampi((int)floorf(fx), 0, gw - 1);
            const int gx1 = imin(gx + 1, gw - 1);
            const float tx = clampf(fx - (float)gx, 0.f, 1.f);
            const int i00 = gy * gw + gx, i10 = gy * gw + gx1, i01 = gy1 * gw + gx, i11 = gy1 * gw + gx1;
#define PICK(v) ((v) < 0.f ? 0.f : (v))
#define WGT(v) ((v) < 0.f ? 0.f : 1.f)
            const float w00 = (1.f - tx) * (1.f - ty) * WGT(gd[i00]);
            const float w10 = tx * (1.f - ty) * WGT(gd[i10]);
            const float w01 = (1.f - tx) * ty * WGT(gd[i01]);
            const float w11 = tx * ty * WGT(gd[i11]);
            const float ww = w00 + w10 + w01 + w11;
            const int p = y * w + x;
            if (ww > 1e-6f) {
                const float dp = (w00 * PICK(gd[i00]) + w10 * PICK(gd[i10]) + w01 * PICK(gd[i01]) +
                                  w11 * PICK(gd[i11])) / ww;
                d_prior[p] = dp;
                pconf[p] = (w00 * gc[i00] + w10 * gc[i10] + w01 * gc[i01] + w11 * gc[i11]) / ww;
                float cmin = 1e9f, cmax = -1e9f;
                const int idx[4] = {i00, i10, i01, i11};
                for (int k = 0; k < 4; ++k) {
                    const int q = idx[k];
                    if (gd[q] >= 0.f) {
                        const float mn = gmn[q] >= 0.f ? gmn[q] : gd[q];
                        const float mx = gmx[q] >= 0.f ? gmx[q] : gd[q];
                        cmin = fminf_ref(cmin, mn);
                        cmax = fmaxf_ref(cmax, mx);
                    }
                }
                pspread[p] = (w00 * PICK(gs[i00]) + w10 * PICK(gs[i10]) + w01 * PICK(gs[i01]) +
                              w11 * PICK(gs[i11])) / ww;
                pmin[p] = (cmin <= cmax) ? fminf_ref(cmin, dp) : dp;
                pmax[p] = (cmin <= cmax) ? fmaxf_ref(cmax, dp) : dp;
            }
#undef PICK
#undef WGT
        }
    }
    free(cnt); free(off); free(pts); free(devs);
    free(gd); free(gc); free(gs); free(gmn); free(gmx);
    free(nd); free(nc); free(ns); free(nmn); free(nmx);
}

/* PriorEstimator::apply_search_range, src/prior_estimator.cpp:367-412. */
void orc_apply_search_range(const apg_pipeline_config_t* cfg, int w, int h, const float* d_prior,
                            const float* pc, const float* ps, const float* pmn, const float* pmx,
                            int16_t* rmin, int16_t* rmax) {
    const int default_R = cfg->prior_search_radius;
    const int global_D = cfg->max_disparity - cfg->min_disparity;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const int i = y * w + x;
            const float dp = d_prior[i];
            if (dp < 0.f) continue;
            const float conf = pc[i], spread = ps[i];
            const float pmin = pmn[i] >= 0.f ? pmn[i] : dp;
            const float pmax = pmx[i] >= 0.f ? pmx[i] : dp;
            int R = default_R;
            if (conf < 0.25f) R = global_D;
            else if (conf > 0.85f && spread < 1.5f) R = 8;
            else if (conf > 0.60f && spread < 3.0f) R = (int)(12.f + 1.5f * spread + 0.5f);
            else if (conf > 0.40f && spread < 6.0f) R = (int)(18.f + 2.0f * spread + 0.5f);
            else R = imax(24, (int)(16.f + 2.0f * spread + 0.5f));
            R = imin(R, global_D);
            const int bound_lo = (int)floorf(pmin) - 4;
            const int bound_hi = (int)ceilf(pmax) + 4 + 1;
            const int lo = imin((int)floorf(dp) - R, bound_lo);
            int hi = imax((int)ceilf(dp) + R + 1, bound_hi);
            hi = imin(hi, x + 1);
            set_range(cfg, rmin, rmax, i, lo, hi);
        }
    }
}

uint64_t orc_fnv1a64(const uint8_t* data, uint64_t n) {
    uint64_t hsh = 14695981039346656037ULL;
    for (uint64_t i = 0; i < n; ++i) { hsh ^= data[i]; hsh *= 1099511628211ULL; }
    return hsh;
}

/* validate_inputs / validate_config, src/pipeline.cpp:171-232 (codes of include/apg_sgm/status.hpp). */
static int validate(const apg_pipeline_config_t* c, const uint8_t* l, const uint8_t* r, int w, int h,
                    int stride, int ch) {
    if (!l || !r || w <= 0 || h <= 0) return 1;
    if (stride < w * ch) return 2;
    if (c->max_disparity <= c->min_disparity) return 3;
    if (c->cost_max < 0 || c->cost_max > 65535) return 4;
    if (c->P1 < 0 || c->P2_base <= c->P1) return 4;
    if (c->grad_t1 < 0 || c->grad_t2 < c->grad_t1) return 4;
    if (c->prior_enable && c->prior_search_radius < 0) return 4;
    if (c->refine_enable && c->refine_iterations < 0) return 4;
    return 0;
}

/* The coarse configuration of HierarchicalStereo::estimate_search_range,
 * src/hierarchical_stereo.cpp:172-182: half the disparity bounds, no prior, no refine,
 * aggregation as coarse_cross_agg, sub-pixel and LR on, median radius 1, fill gap 16 or none. */
void orc_hier_coarse_config(const apg_pipeline_config_t* cfg, apg_pipeline_config_t* c) {
    *c = *cfg;
    c->min_disparity = imax(0, cfg->min_disparity / 2);
    c->max_disparity = imax(c->min_disparity + 1, (cfg->max_disparity + 1) / 2);
    c->prior_enable = 0;
    c->refine_enable = 0;
    c->agg_enable = cfg->hier_coarse_cross_agg;
    c->volume_backend = 2;
    c->subpixel = 1;
    c->lr_check = 1;
    c->median_radius = 1;
    c->max_fill_gap = cfg->hier_coarse_fill_holes ? 16 : 0;
    c->hier_enable = 0;
}

static int pipeline_run(const apg_pipeline_config_t* cfg, const uint8_t* left, const uint8_t* right,
                        int w, int h, int stride, int ch, float* disparity, float* confidence,
                        uint8_t* invalid_reason, uint8_t* reliable_mask, orc_stages_t* st, int skip_fill);

/* HierarchicalStereo::estimate_search_range, src/hierarchical_stereo.cpp:113-431: a half-size
 * pass of the whole pipeline (2x2 box-averaged grays, (sum + 2) / 4) and, per full-size pixel,
 * a range around twice the coarse disparities of its 2x2 coarse neighbourhood, with the
 * confidence-adaptive radius and the NearestValid / ExpandedRadius / FullRange fallbacks.
 * d_prior receives the guiding disparity (-1 where none).  counts4 (nullable) receives
 * {coarse pixels with a valid disparity, fallback pixels, full-range pixels, sum of widths}
 * (HierarchicalTelemetry's numerators, src/hierarchical_stereo.cpp:413-420).
 * Returns 0 for frames under 32 pixels in either dimension (default ranges), 1 otherwise. */
int orc_hier_range(const apg_pipeline_config_t* cfg, int W, int H, const uint8_t* lg, const uint8_t* rg,
                   int16_t* rmin, int16_t* rmax, float* d_prior, int64_t* counts4,
                   float* coarse_disp, float* coarse_conf) {
    if (counts4) counts4[0] = counts4[1] = counts4[2] = counts4[3] = 0;
    if (W < 32 || H < 32) {
        orc_range_default(cfg, W, H, rmin, rmax);
        for (size_t i = 0; i < (size_t)W * H; ++i) d_prior[i] = -1.f;
        return 0;
    }
    const int Wc = W / 2, Hc = H / 2;
    const size_t nc = (size_t)Wc * Hc;
    uint8_t* cimg = (uint8_t*)malloc(nc * 2);
    uint8_t *cl = cimg, *cr = cimg + nc;
    for (int yc = 0; yc < Hc; ++yc) {
        const int y0 = yc * 2, y1 = imin(y0 + 1, H - 1);
        for (int xc = 0; xc < Wc; ++xc) {
            const int x0 = xc * 2, x1 = imin(x0 + 1, W - 1);
            const int sl = lg[y0 * W + x0] + lg[y0 * W + x1] + lg[y1 * W + x0] + lg[y1 * W + x1];
            const int sr = rg[y0 * W + x0] + rg[y0 * W + x1] + rg[y1 * W + x0] + rg[y1 * W + x1];
            cl[yc * Wc + xc] = (uint8_t)((sl + 2) / 4);
            cr[yc * Wc + xc] = (uint8_t)((sr + 2) / 4);
        }
    }
    apg_pipeline_config_t cc;
    orc_hier_coarse_config(cfg, &cc);
    float* cd = (float*)malloc(nc * 8);
    float* cf = cd + nc;
    uint8_t* cm = (uint8_t*)malloc(nc * 2);
    pipeline_run(&cc, cl, cr, Wc, Hc, Wc, 1, cd, cf, cm, cm + nc, NULL, !cfg->hier_coarse_fill_holes);
    if (coarse_disp) memcpy(coarse_disp, cd, nc * 4);
    if (coarse_conf) memcpy(coarse_conf, cf, nc * 4);
    int64_t nvalid = 0, nfall = 0, nfull = 0, wsum = 0;
    for (size_t i = 0; i < nc; ++i) nvalid += cd[i] >= 0.f;
    const int R = cfg->hier_radius;
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const int i = y * W + x;
            const int xc = imax(0, imin(x / 2, Wc - 1)), yc = imax(0, imin(y / 2, Hc - 1));
            const int xc1 = imin(xc + 1, Wc - 1), yc1 = imin(yc + 1, Hc - 1);
            const float q[4] = {cd[yc * Wc + xc], cd[yc * Wc + xc1], cd[yc1 * Wc + xc], cd[yc1 * Wc + xc1]};
            float mn = 1e9f, mx = -1e9f;
            int nv = 0;
            for (int k = 0; k < 4; ++k)
                if (q[k] >= 0.f) {
                    mn = fminf_ref(mn, q[k]);
                    mx = fmaxf_ref(mx, q[k]);
                    ++nv;
                }
            const int glo = cfg->min_disparity, ghi = imin(cfg->max_disparity, x + 1);
            d_prior[i] = -1.f;
            int lo = glo, hi = ghi;
            if (nv > 0) {
                const float dc = q[0] >= 0.f ? q[0] : 0.5f * (mn + mx);
                const float Dc = 2.0f * dc, Dmn = 2.0f * mn, Dmx = 2.0f * mx;
                int er = R;
                if (cfg->hier_adaptive_radius && cf[yc * Wc + xc] < cfg->hier_confidence_threshold)
                    er = cfg->hier_expanded_radius;
                lo = imin((int)floorf(Dc) - er, (int)floorf(Dmn) - 1);
                hi = imax((int)ceilf(Dc) + er + 1, (int)ceilf(Dmx) + 2);
                lo = imax(lo, glo);
                hi = imin(hi, ghi);
                if (hi < lo) hi = lo;
                d_prior[i] = Dc;
            } else {
                ++nfall;
                if (cfg->hier_fallback != APG_HIER_FALLBACK_FULL_RANGE) {
                    const int K = 4;
                    float near = -1.f;
                    int best = 1000;
                    for (int sy = imax(0, yc - K); sy <= imin(Hc - 1, yc + K); ++sy)
                        for (int sx = imax(0, xc - K); sx <= imin(Wc - 1, xc + K); ++sx) {
                            const float v = cd[sy * Wc + sx];
                            const int d2 = (sx - xc) * (sx - xc) + (sy - yc) * (sy - yc);
                            if (v >= 0.f && d2 < best) { best = d2; near = v; }
                        }
                    if (near >= 0.f) {
                        const float Dn = 2.0f * near;
                        const int re = cfg->hier_fallback == APG_HIER_FALLBACK_EXPANDED_RADIUS ? 2 * R : R + 8;
                        lo = imax(glo, (int)floorf(Dn) - re);
                        hi = imin(ghi, (int)ceilf(Dn) + re + 1);
                        if (hi < lo) hi = lo;
                        d_prior[i] = Dn;
                    }
                }
            }
            set_range(cfg, rmin, rmax, i, lo, hi);
            wsum += hi - lo;  /* the full-range branches add ghi - glo unclamped, as the reference */
            if (hi - lo == ghi - glo) ++nfull;
        }
    }
    if (counts4) { counts4[0] = nvalid; counts4[1] = nfall; counts4[2] = nfull; counts4[3] = wsum; }
    free(cimg); free(cd); free(cm);
    return 1;
}

/* StereoMatcher::compute_impl, src/pipeline.cpp:435-719, Dense branch. */
int orc_pipeline(const apg_pipeline_config_t* cfg, const uint8_t* left, const uint8_t* right,
                 int w, int h, int stride, int ch,
                 float* disparity, float* confidence, uint8_t* invalid_reason, uint8_t* reliable_mask,
                 orc_stages_t* st) {
    return pipeline_run(cfg, left, right, w, h, stride, ch, disparity, confidence, invalid_reason,
                        reliable_mask, st, 0);
}

/* skip_fill: the coarse pass of the hierarchical mode calls fill_holes only with a positive gap
 * (src/hierarchical_stereo.cpp:262-265); a zero gap still fills from the direct neighbours. */
static int pipeline_run(const apg_pipeline_config_t* cfg, const uint8_t* left, const uint8_t* right,
                        int w, int h, int stride, int ch, float* disparity, float* confidence,
                        uint8_t* invalid_reason, uint8_t* reliable_mask, orc_stages_t* st, int skip_fill) {
    const int v = validate(cfg, left, right, w, h, stride, ch);
    if (v) return v;
    const size_t n = (size_t)w * h;
    const int D = cfg->max_disparity - cfg->min_disparity;
    const size_t nv = n * (size_t)D;
    const int sym = cfg->census_type == APG_CENSUS_SYMMETRIC_9X7;
    uint8_t* aux = (uint8_t*)malloc(n * 6);
    uint8_t *lg = aux, *lgx = aux + n, *lgy = aux + 2 * n, *rg = aux + 3 * n, *rgx = aux + 4 * n, *rgy = aux + 5 * n;
    uint32_t *cl = NULL, *cr = NULL;
    uint64_t *cl64 = NULL, *cr64 = NULL;
    orc_gray_grad(left, w, h, stride, ch, lg, lgx, lgy);
    orc_gray_grad(right, w, h, stride, ch, rg, rgx, rgy);
    if (sym) {
        cl = (uint32_t*)malloc(n * 4); cr = (uint32_t*)malloc(n * 4);
        orc_census_sym(lg, w, h, cl); orc_census_sym(rg, w, h, cr);
    } else {
        cl64 = (uint64_t*)malloc(n * 8); cr64 = (uint64_t*)malloc(n * 8);
        orc_census64(lg, w, h, cl64); orc_census64(rg, w, h, cr64);
    }
    int16_t* rmin = (int16_t*)malloc(n * 2);
    int16_t* rmax = (int16_t*)malloc(n * 2);
    float* d_prior = (float*)malloc(n * 4);
    orc_range_default(cfg, w, h, rmin, rmax);
    for (size_t i = 0; i < n; ++i) d_prior[i] = -1.f;
    int support_count = 0;
    if (cfg->hier_enable) {
        /* the hierarchical range replaces the prior (src/pipeline.cpp:483-499) */
        orc_hier_range(cfg, w, h, lg, rg, rmin, rmax, d_prior, NULL, NULL, NULL);
    } else if (cfg->prior_enable) {
        const int cap = cfg->prior_max_supports > 0 ? cfg->prior_max_supports : 1;
        orc_support_t* sup = (orc_support_t*)malloc(sizeof(orc_support_t) * cap);
        support_count = orc_extract_supports(cfg, w, h, lgx, lgy, cl, cr, cl64, cr64, sup, cap);
        if (support_count >= cfg->prior_min_supports) {
            float* pc = (float*)malloc(n * 4); float* ps = (float*)malloc(n * 4);
            float* pmn = (float*)malloc(n * 4); float* pmx = (float*)malloc(n * 4);
            orc_interpolate_prior(w, h, sup, support_count, d_prior, pc, ps, pmn, pmx);
            orc_apply_search_range(cfg, w, h, d_prior, pc, ps, pmn, pmx, rmin, rmax);
            free(pc); free(ps); free(pmn); free(pmx);
        }
        free(sup);
    }
    uint16_t* vol = (uint16_t*)malloc(nv * 2);
    orc_cost_volume(cfg, w, h, lg, lgx, lgy, rg, rgx, rgy, cl, cr, cl64, cr64, rmin, rmax, vol);
    if (st && st->cost_raw) memcpy(st->cost_raw, vol, nv * 2);
    float* dr = (float*)malloc(n * 4);
    orc_wta_right(cfg, vol, w, h, dr);
    orc_cross_aggregate(cfg, lg, w, h, rmin, rmax, vol);
    if (st && st->cost_agg) memcpy(st->cost_agg, vol, nv * 2);
    uint32_t* acc = (uint32_t*)malloc(nv * 4);
    orc_sgm_optimize(cfg, lg, vol, acc, w, h);
    if (st && st->sgm_sum) memcpy(st->sgm_sum, acc, nv * 4);
    free(vol);
    float* disp = (float*)malloc(n * 4);
    float* best = (float*)malloc(n * 4);
    float* second = (float*)malloc(n * 4);
    orc_wta(cfg, acc, rmin, rmax, w, h, disp, best, second);
    free(acc);
    if (st) {
        if (st->disp_wta) memcpy(st->disp_wta, disp, n * 4);
        if (st->best) memcpy(st->best, best, n * 4);
        if (st->second) memcpy(st->second, second, n * 4);
        if (st->disp_right) memcpy(st->disp_right, dr, n * 4);
        if (st->range_min) memcpy(st->range_min, rmin, n * 2);
        if (st->range_max) memcpy(st->range_max, rmax, n * 2);
        if (st->d_prior) memcpy(st->d_prior, d_prior, n * 4);
        st->support_count = support_count;
    }
    orc_confidence(cfg, w, h, disp, dr, best, second, lgx, lgy, confidence, reliable_mask, invalid_reason);
    if (cfg->refine_enable) {
        void* rng = orc_rng_create(12345u);
        int* draws = (int*)malloc(sizeof(int) * (n + 1));
        for (int it = 0; it < cfg->refine_iterations; ++it) {
            const int radius = imax(1, cfg->refine_random_radius >> it);
            const int cnt = orc_refine_count(w, h, reliable_mask, rmin, rmax, disp);
            orc_rng_draws(rng, radius, cnt, draws);
            orc_refine_pass(cfg, it, w, h, lg, lgx, lgy, rg, rgx, rgy, cl, cr, cl64, cr64, rmin, rmax,
                            reliable_mask, draws, disp);
        }
        free(draws);
        orc_rng_destroy(rng);
    }
    if (st && st->disp_refined) memcpy(st->disp_refined, disp, n * 4);
    orc_lr_check(cfg, w, h, dr, disp, invalid_reason);
    if (st && st->disp_lr) memcpy(st->disp_lr, disp, n * 4);
    float* filled = (float*)malloc(n * 4);
    if (skip_fill)
        memcpy(filled, disp, n * 4);
    else
        orc_fill_holes(cfg, w, h, disp, invalid_reason, lg, d_prior, filled);
    if (st && st->disp_fill) memcpy(st->disp_fill, filled, n * 4);
    orc_median(cfg, w, h, filled, disparity);
    free(filled); free(disp); free(best); free(second); free(dr); free(d_prior);
    free(rmin); free(rmax); free(aux); free(cl); free(cr); free(cl64); free(cr64);
    return 0;
}

/* Exported wrapper of the header's PipelineConfig::from_mode restatement. */
void orc_config_from_mode(int mode, int max_disparity, apg_pipeline_config_t* out) {
    *out = apg_config_from_mode(mode, max_disparity);
}

/* evaluate_stereo, src/metrics.cpp:119-502, without the support block: the per-pixel tallies in
 * raster order (so the double sums are the reference's, rounding included), then
 * apg_metrics_finalize (include/apg_sgm/metrics.h) for the float ratios.  left (nullable) is the
 * left image with its row stride and channel count; thr NULL means QualityThresholds{}. */
static int gt_valid(float g, float mx) { return isfinite(g) && g >= 0.0f && g < mx; }

static float orc_luma(const uint8_t* img, int stride, int ch, int x, int y) {
    const uint8_t* p = img + (size_t)y * stride + (size_t)x * ch;
    if (ch == 1) return (float)p[0];
    return 0.299f * (float)p[0] + 0.587f * (float)p[1] + 0.114f * (float)p[2];
}

static void region_add(long long* r, double* sum, float e, float g) {
    const int ok = isfinite(e) && e >= 0.0f;
    const float diff = ok ? fabsf(e - g) : 1e9f;
    const int d1 = !ok || (diff > 3.0f && (g > 1e-3f ? (diff / g > 0.05f) : 1));
    r[0]++;
    if (d1) r[6]++;
    if (ok) {
        r[1]++;
        *sum += diff;
        if (diff > 0.5f) r[2]++;
        if (diff > 1.0f) r[3]++;
        if (diff > 2.0f) r[4]++;
        if (diff > 3.0f) r[5]++;
    }
}

void orc_evaluate_stereo(const float* est, const float* gt, int w, int h, const int16_t* rmin, const int16_t* rmax,
                         const float* before, const float* after, const uint8_t* vis, float max_valid_gt,
                         const uint8_t* left, int left_stride, int left_ch, const apg_quality_thresholds_t* thr,
                         apg_stereo_metrics_t* out) {
    static const int dxs[4] = {1, -1, 0, 0}, dys[4] = {0, 0, 1, -1};
    const apg_quality_thresholds_t T = thr ? *thr : apg_quality_thresholds_default();
    long long c[APG_MC_COUNT];
    double sm[APG_MS_COUNT];
    memset(c, 0, sizeof(c));
    memset(sm, 0, sizeof(sm));
    if (w <= 0 || h <= 0) {
        apg_stereo_metrics_t z;
        memset(&z, 0, sizeof(z));
        *out = z;
        return;
    }
    const size_t n = (size_t)w * h;
    const int has_range = rmin && rmax, has_ref = before && after, has_left = left != NULL;
    uint8_t* edge = (uint8_t*)calloc(n, 1);
    uint8_t* low = has_left ? (uint8_t*)calloc(n, 1) : NULL;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float g = gt[(size_t)y * w + x];
            if (!gt_valid(g, max_valid_gt)) continue;
            float md = 0.0f;
            for (int k = 0; k < 4; ++k) {
                const int nx = x + dxs[k], ny = y + dys[k];
                if (nx >= 0 && nx < w && ny >= 0 && ny < h) {
                    const float ng = gt[(size_t)ny * w + nx];
                    if (isfinite(ng) && ng >= 0.0f && ng < max_valid_gt) md = fmaxf_ref(md, fabsf(g - ng));
                }
            }
            if (md >= T.boundary_disparity_gradient) edge[(size_t)y * w + x] = 1;
        }
    if (has_left)
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const int xp = imax(0, x - 1), xn = imin(w - 1, x + 1), yp = imax(0, y - 1), yn = imin(h - 1, y + 1);
                const float sx = (x == 0 || x == w - 1) ? 1.0f : 2.0f, sy = (y == 0 || y == h - 1) ? 1.0f : 2.0f;
                const float dx = (orc_luma(left, left_stride, left_ch, xn, y) - orc_luma(left, left_stride, left_ch, xp, y)) / sx;
                const float dy = (orc_luma(left, left_stride, left_ch, x, yn) - orc_luma(left, left_stride, left_ch, x, yp)) / sy;
                if (sqrtf(dx * dx + dy * dy) < T.low_texture_gradient) low[(size_t)y * w + x] = 1;
            }
    long long* reg = c + APG_MC_REGION0;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const size_t i = (size_t)y * w + x;
            const float g = gt[i];
            if (!gt_valid(g, max_valid_gt)) continue;
            c[APG_MC_EVALUATED]++;
            const int xr = x - (int)roundf(g);
            const int matchable = xr >= 0 && xr < w;
            const int visible = vis ? vis[i] >= 200 : matchable;
            const int ed = edge[i] != 0;
            if (has_range) {
                const int in = g >= (float)rmin[i] && g < (float)rmax[i];
                c[APG_MC_EVAL_ALL]++;
                if (in) c[APG_MC_IN_ALL]++;
                if (matchable) {
                    c[APG_MC_EVAL_MATCH]++;
                    if (in) c[APG_MC_IN_MATCH]++;
                }
                if (visible) {
                    c[APG_MC_EVAL_VIS]++;
                    if (in) c[APG_MC_IN_VIS]++;
                    else {
                        c[APG_MC_MISS_VIS]++;
                        if (ed) c[APG_MC_MISS_EDGE]++;
                        else c[APG_MC_MISS_NONEDGE]++;
                    }
                }
            }
            const float e = est[i];
            const int ok = isfinite(e) && e >= 0.0f;
            if (!ok) {
                c[APG_MC_LR_FAIL]++;
            } else {
                const float diff = fabsf(e - g);
                c[APG_MC_VALID]++;
                sm[APG_MS_EPE] += diff;
                if (diff > 0.5f) c[APG_MC_C05]++;
                if (diff > 1.0f) c[APG_MC_C10]++;
                if (diff > 2.0f) c[APG_MC_C20]++;
                if (diff > 3.0f) c[APG_MC_C30]++;
                if (ed) { c[APG_MC_EDGE]++; sm[APG_MS_EDGE] += diff; }
                else { c[APG_MC_NONEDGE]++; sm[APG_MS_NONEDGE] += diff; }
            }
            const int d1 = !ok || (fabsf(e - g) > 3.0f && (g > 1e-3f ? (fabsf(e - g) / g > 0.05f) : 1));
            if (d1) c[APG_MC_D1_ALL]++;
            if (visible) {
                c[APG_MC_EVAL_NOC]++;
                if (d1) c[APG_MC_D1_NOC]++;
            }
            region_add(reg + 0, sm + APG_MS_REGION0 + 0, e, g);
            if (visible) region_add(reg + 7, sm + APG_MS_REGION0 + 1, e, g);
            else region_add(reg + 14, sm + APG_MS_REGION0 + 2, e, g);
            if (ed) region_add(reg + 21, sm + APG_MS_REGION0 + 3, e, g);
            else region_add(reg + 28, sm + APG_MS_REGION0 + 4, e, g);
            if (has_left) {
                if (low[i]) region_add(reg + 35, sm + APG_MS_REGION0 + 5, e, g);
                else region_add(reg + 42, sm + APG_MS_REGION0 + 6, e, g);
            }
            if (has_ref) {
                const float eb = before[i], ea = after[i];
                if (isfinite(eb) && eb >= 0.0f && isfinite(ea) && ea >= 0.0f) {
                    const float db = fabsf(eb - g), da = fabsf(ea - g);
                    c[APG_MC_REF_EVAL]++;
                    sm[APG_MS_BEFORE] += db;
                    sm[APG_MS_AFTER] += da;
                    if (da < db - 1e-4f) c[APG_MC_REF_IMPROVED]++;
                    else if (da > db + 1e-4f) c[APG_MC_REF_WORSENED]++;
                    else c[APG_MC_REF_UNCHANGED]++;
                    if (fabsf(ea - eb) > 1e-4f) c[APG_MC_REF_CHANGED]++;
                    if (ok) {
                        c[APG_MC_TOTAL_EVAL]++;
                        sm[APG_MS_TOT_BEFORE] += db;
                        sm[APG_MS_TOT_AFTER] += da;
                        sm[APG_MS_TOT_FINAL] += fabsf(e - g);
                    }
                }
            }
        }
    free(edge);
    free(low);
    apg_metrics_finalize(c, sm, w * h, has_range, has_ref, out);
}

/* evaluate_supports, src/metrics.cpp:8-124: the supports in their order (so the double sums are the
 * reference's), cells of cell_size pixels. */
void orc_evaluate_supports(const orc_support_t* sp, int ns, const float* gt, int w, int h, const uint8_t* vis,
                           float max_valid_gt, int cell_size, apg_support_metrics_t* out) {
    long long c[10];
    double s[2] = {0.0, 0.0};
    memset(c, 0, sizeof(c));
    if (ns <= 0 || w <= 0 || h <= 0) {
        apg_support_metrics_t z;
        memset(&z, 0, sizeof(z));
        z.total = ns;
        *out = z;
        return;
    }
    const int gw = (w + cell_size - 1) / cell_size, gh = (h + cell_size - 1) / cell_size, nc = gw * gh;
    uint8_t* vc = (uint8_t*)calloc((size_t)nc * 2, 1);
    uint8_t* oc = vc + nc;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            const float g = gt[(size_t)y * w + x];
            if (!gt_valid(g, max_valid_gt)) continue;
            const int xr = x - (int)roundf(g);
            const int v = vis ? vis[(size_t)y * w + x] >= 200 : (xr >= 0 && xr < w);
            if (v && x / cell_size < gw && y / cell_size < gh) vc[(y / cell_size) * gw + x / cell_size] = 1;
        }
    for (int k = 0; k < ns; ++k) {
        const int x = sp[k].x, y = sp[k].y;
        if (x < 0 || x >= w || y < 0 || y >= h) continue;
        const float g = gt[(size_t)y * w + x];
        if (!gt_valid(g, max_valid_gt)) continue;
        c[0]++;
        const int xr = x - (int)roundf(g);
        const int v = vis ? vis[(size_t)y * w + x] >= 200 : (xr >= 0 && xr < w);
        if (v) c[1]++;
        const float err = fabsf(sp[k].disparity - g);
        s[0] += err;
        if (v) s[1] += err;
        if (err <= 0.5f) { c[2]++; if (v) c[5]++; }
        if (err <= 1.0f) {
            c[3]++;
            if (v) {
                c[6]++;
                if (x / cell_size < gw && y / cell_size < gh) oc[(y / cell_size) * gw + x / cell_size] = 1;
            }
        }
        if (err <= 2.0f) { c[4]++; if (v) c[7]++; }
    }
    for (int i = 0; i < nc; ++i) {
        c[8] += vc[i];
        c[9] += vc[i] && oc[i];
    }
    free(vc);
    apg_support_finalize(ns, c, s, out);
}


// Per-pixel back end: confidence, left-right check, hole fill, median.
//
// Restates ConfidenceEstimator::estimate (src/confidence_estimator.cpp:7-63),
// PostProcessor::left_right_check / fill_holes (Legacy route) / median
// (src/postprocess.cpp:10-40, 42-168, 255-309).  Every float expression keeps the reference's
// operation order with explicitly rounded intrinsics (no contraction), so outputs are bit-exact.
// These kernels touch O(W*H) bytes and are a few microseconds each at 720p.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace apgcu {

namespace {

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Confidence (+ optional fused LR check when no refinement sits between them).
__global__ void conf_lr_kernel(ConfLrArgs a) {
    const int n = a.w * a.h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / a.w, x = i - y * a.w;
        const float c1 = a.best[i], c2 = a.second[i];
        float uniq = 0.f;
        if (isfinite(c1) && isfinite(c2)) {
            uniq = __fdiv_rn(__fsub_rn(c2, c1), (c2 < 1e-3f) ? 1e-3f : c2);
            uniq = clampf(uniq, 0.f, 1.f);
        }
        const float d = a.disp[i];
        float lr = 1.f;
        {
            const int xr = (int)roundf(__fsub_rn((float)x, d));
            if (xr < 0 || xr >= a.w || d < 0.f) {
                lr = 0.f;
            } else {
                const float dr = a.disp_right[y * a.w + xr];
                if (dr < 0.f || fabsf(__fsub_rn(d, dr)) > __fadd_rn((float)a.conf_lr_max_diff, 0.5f)) lr = 0.f;
            }
        }
        const float tex = (float)((int)a.lgx[i] + (int)a.lgy[i]);
        const float tex_term = clampf(__fdiv_rn(tex, 16.f), 0.f, 1.f);
        float conf = clampf(uniq, 0.f, 4.f);
        conf = __fmul_rn(conf, __fadd_rn(0.5f, __fmul_rn(0.5f, tex_term)));
        if (lr < 0.5f) conf = __fmul_rn(conf, 0.25f);
        a.confidence[i] = conf;
        const bool lr_ok = lr >= 0.5f;
        const bool rel = lr_ok && conf >= a.reliable_threshold && uniq >= a.uniqueness_ratio &&
                         tex >= a.min_texture && d >= 0.f;
        a.reliable[i] = rel ? 1 : 0;
        uint8_t reason = rel ? kValid : (lr_ok ? kLowConfidence : kMismatch);
        if (a.fuse_lr) {
            float dout = d;
            if (a.lr_check && d >= 0.f) {
                const float tol = __fadd_rn((float)a.post_lr_max_diff, 0.5f);
                const int xr = (int)roundf(__fsub_rn((float)x, d));
                if (xr < 0 || xr >= a.w) {
                    dout = -1.f;
                    reason = kOcclusion;
                } else {
                    const float dr = a.disp_right[y * a.w + xr];
                    if (dr < 0.f || fabsf(__fsub_rn(d, dr)) > tol) {
                        dout = -1.f;
                        reason = (dr > __fadd_rn(d, tol)) ? kOcclusion : kMismatch;
                    }
                }
            }
            a.disp_out[i] = dout;
        }
        a.reason[i] = reason;
    }
}

// Stand-alone LR check (after refinement), src/postprocess.cpp:10-40.
__global__ void lr_kernel(int w, int h, int lr_max_diff, const float* __restrict__ dr_img,
                          const float* __restrict__ din, float* __restrict__ dout, uint8_t* __restrict__ reason) {
    const int n = w * h;
    const float tol = __fadd_rn((float)lr_max_diff, 0.5f);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / w, x = i - y * w;
        const float d = din[i];
        float o = d;
        if (d >= 0.f) {
            const int xr = (int)roundf(__fsub_rn((float)x, d));
            if (xr < 0 || xr >= w) {
                o = -1.f;
                reason[i] = kOcclusion;
            } else {
                const float dr = dr_img[y * w + xr];
                if (dr < 0.f || fabsf(__fsub_rn(d, dr)) > tol) {
                    o = -1.f;
                    reason[i] = (dr > __fadd_rn(d, tol)) ? kOcclusion : kMismatch;
                }
            }
        }
        dout[i] = o;
    }
}

// ShadowReclass (src/postprocess.cpp:170-192): a mismatch hole between two valid neighbours at least
// 4 px apart is a depth step's shadow and is filled like an occlusion.
__device__ __forceinline__ bool occlusion_like(uint8_t r, int shadow, float dl, float dr) {
    return r == kOcclusion ||
           (shadow && r == kMismatch && dl >= 0.f && dr >= 0.f && fabsf(__fsub_rn(dr, dl)) >= 4.0f);
}

// Legacy hole fill, src/postprocess.cpp:87-168 (shadow != 0: the ShadowReclass inpaint,
// :170-239).  Reads the pre-fill map, writes a copy.  tel (nullable): the InpaintTelemetry
// counters of every hole (classification, gap bound hit, fill route, shadow reclassification).
__global__ void fill_kernel(int w, int h, int gap, int shadow, apg_inpaint_telemetry_t* __restrict__ tel,
                            const float* __restrict__ in, const uint8_t* __restrict__ reason,
                            const uint8_t* __restrict__ gray, const float* __restrict__ d_prior,
                            float* __restrict__ out) {
    const int n = w * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = in[i];
        if (v >= 0.f) { out[i] = v; continue; }
        const int y = i / w, x = i - y * w;
        const float* row = in + (size_t)y * w;
        int xl = x - 1;
        while (xl >= 0 && xl >= x - gap && row[xl] < 0.f) --xl;
        int xr = x + 1;
        while (xr < w && xr <= x + gap && row[xr] < 0.f) ++xr;
        const float dl = (xl >= 0 && row[xl] >= 0.f) ? row[xl] : -1.f;
        const float dr = (xr < w && row[xr] >= 0.f) ? row[xr] : -1.f;
        const uint8_t r = reason[i];
        if (tel) {
            atomicAdd(&tel->total_invalid_pixels, 1ull);
            if (r == kOcclusion) atomicAdd(&tel->classified_occ_pixels, 1ull);
            else if (r == kMismatch) atomicAdd(&tel->classified_mismatch_pixels, 1ull);
            if (xl < 0 || x - xl > gap || xr >= w || xr - x > gap) atomicAdd(&tel->hit_max_gap_pixels, 1ull);
        }
        float o = v;
        int route;  // FillRoute (src/inpaint_internal.hpp:34-47)
        if (occlusion_like(r, shadow, dl, dr)) {
            if (tel && r != kOcclusion) atomicAdd(&tel->reclassified_shadow_pixels, 1ull);
            if (dl >= 0.f && dr >= 0.f) { o = (dr < dl) ? dr : dl; route = 1; }
            else if (dl >= 0.f) { o = dl; route = 2; }
            else if (dr >= 0.f) { o = dr; route = 3; }
            else route = 10;
        } else {
            const int c0 = gray[i];
            float best_d = -1.f;
            int best_abs = 999;
            bool best_vert = false;
            const int cx[4] = {xl, xr, x, x};
            const int cy[4] = {y, y, y - 1, y + 1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int xx = cx[k], yy = cy[k];
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                const float dv = in[(size_t)yy * w + xx];
                if (dv < 0.f) continue;
                const int ad = abs((int)gray[(size_t)yy * w + xx] - c0);
                if (ad < best_abs) { best_abs = ad; best_d = dv; best_vert = k >= 2; }
            }
            if (best_d >= 0.f && best_abs <= 18) {
                o = best_d;
                route = best_vert ? 5 : 4;
            } else if (d_prior && d_prior[i] >= 0.f) {
                o = d_prior[i];
                route = 6;
            } else if (dl >= 0.f && dr >= 0.f) {
                const float t = __fdiv_rn((float)(x - xl), (float)(xr - xl));
                o = __fadd_rn(__fmul_rn(dl, __fsub_rn(1.f, t)), __fmul_rn(dr, t));
                route = 7;
            } else if (dl >= 0.f) {
                o = dl;
                route = 8;
            } else if (dr >= 0.f) {
                o = dr;
                route = 9;
            } else {
                route = 10;
            }
        }
        if (tel) atomicAdd(&tel->route_counts[route], 1ull);
        out[i] = o;
    }
}

// InpaintTelemetry's run statistics (src/postprocess.cpp:64-85): each row's runs of invalid
// pixels, one thread per row.
__global__ void fill_runs_kernel(int w, int h, int gap, const float* __restrict__ in,
                                 apg_inpaint_telemetry_t* __restrict__ tel) {
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < h; y += gridDim.x * blockDim.x) {
        const float* row = in + (size_t)y * w;
        int len = 0;
        for (int x = 0; x <= w; ++x) {
            if (x < w && row[x] < 0.f) {
                ++len;
                continue;
            }
            if (len > 0) {
                atomicAdd(&tel->invalid_runs_count, 1ull);
                if (len > gap) atomicAdd(&tel->invalid_runs_truncated, 1ull);
                const int b = len < 4 ? 0 : len < 8 ? 1 : len < 16 ? 2 : len < 24 ? 3 : len < 32 ? 4 : len < 48 ? 5
                                                   : len < 64 ? 6 : len < 96 ? 7 : len < 128 ? 8 : 9;
                atomicAdd(&tel->run_length_buckets[b], 1ull);
                len = 0;
            }
        }
    }
}

// Median of the valid values of the (2r+1)^2 window (the size/2-th smallest, as
// std::nth_element at mid = size/2), src/postprocess.cpp:255-309.  The k-th smallest is found
// by rank counting, which needs no per-thread storage and gives the same value as any
// selection algorithm.
__global__ void median_kernel(int w, int h, int r, const float* __restrict__ in, float* __restrict__ out) {
    const int n = w * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int y = i / w, x = i - y * w;
        const int ya = max(0, y - r), yb = min(h - 1, y + r), xa = max(0, x - r), xb = min(w - 1, x + r);
        int cnt = 0;
        for (int yy = ya; yy <= yb; ++yy)
            for (int xx = xa; xx <= xb; ++xx) cnt += in[(size_t)yy * w + xx] >= 0.f;
        if (cnt == 0) { out[i] = in[i]; continue; }
        const int k = cnt / 2;
        float res = in[i];
        bool found = false;
        for (int yy = ya; yy <= yb && !found; ++yy)
            for (int xx = xa; xx <= xb && !found; ++xx) {
                const float v = in[(size_t)yy * w + xx];
                if (!(v >= 0.f)) continue;
                int lt = 0, le = 0;
                for (int y2 = ya; y2 <= yb; ++y2)
                    for (int x2 = xa; x2 <= xb; ++x2) {
                        const float u = in[(size_t)y2 * w + x2];
                        if (!(u >= 0.f)) continue;
                        lt += u < v;
                        le += u <= v;
                    }
                if (lt <= k && k < le) { res = v; found = true; }
            }
        out[i] = res;
    }
}


// The same fill with the neighbour search done by warp ballots: a warp owns 32 consecutive pixels
// of a row; the walk of the reference (xl = x - 1 down while xl >= max(x - gap, 0) and
// row[xl] < 0) stops at the nearest "stopper" q, a pixel with !(row[q] < 0), or ends one beyond the
// gap.  The nearest stopper on each side comes from the segments' stopper masks (this segment,
// then further ones while some lane's gap reaches them), so each pixel costs a few bit operations
// instead of a walk.  Everything after the two neighbours is the per-pixel rule above.
// Rows [y_begin, y_end) of the frame (the whole frame, or one band of the host-output path).
__global__ void fill_ballot_kernel(int w, int h, int y_begin, int y_end, int gap, int shadow,
                                   const float* __restrict__ in, const uint8_t* __restrict__ reason,
                                   const uint8_t* __restrict__ gray, const float* __restrict__ d_prior,
                                   float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int nseg = (w + 31) >> 5;
    const int total = nseg * (y_end - y_begin);  // segments of the rows (w * h / 32 + h, far below 2^31)
    const int wstride = (gridDim.x * blockDim.x) >> 5;
    for (int sg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sg < total; sg += wstride) {
        const int yb = sg / nseg, s = sg - yb * nseg;
        const int y = y_begin + yb;
        const int x = (s << 5) + lane;
        const float* row = in + (size_t)y * w;
        const bool inimg = x < w;
        const float v = inimg ? row[x] : 0.f;
        const bool hole = inimg && !(v >= 0.f);
        if (!__any_sync(0xFFFFFFFFu, hole)) {
            if (inimg) out[(size_t)y * w + x] = v;
            continue;
        }
        const unsigned stop = __ballot_sync(0xFFFFFFFFu, inimg && !(v < 0.f));
        // left: largest stopper in [max(x - gap, 0), x - 1]
        int ql = -1;
        {
            const unsigned below = stop & ((1u << lane) - 1u);
            if (below) ql = (s << 5) + 31 - __clz(below);
            bool need = hole && !below;
            for (int k = s - 1; __any_sync(0xFFFFFFFFu, need && (k << 5) + 31 >= x - gap && k >= 0); --k) {
                const unsigned mk = __ballot_sync(0xFFFFFFFFu, !(row[(k << 5) + lane] < 0.f));
                if (need && mk) {
                    ql = (k << 5) + 31 - __clz(mk);
                    need = false;
                }
            }
        }
        // right: smallest stopper in [x + 1, min(x + gap, w - 1)]
        int qr = w;
        {
            const unsigned above = lane < 31 ? (stop & ~((2u << lane) - 1u)) : 0u;
            if (above) qr = (s << 5) + __ffs(above) - 1;
            bool need = hole && !above;
            for (int k = s + 1; __any_sync(0xFFFFFFFFu, need && (k << 5) <= x + gap && k < nseg); ++k) {
                const int xx = (k << 5) + lane;
                const unsigned mk = __ballot_sync(0xFFFFFFFFu, xx < w && !(row[xx] < 0.f));
                if (need && mk) {
                    qr = (k << 5) + __ffs(mk) - 1;
                    need = false;
                }
            }
        }
        if (!hole) {
            if (inimg) out[(size_t)y * w + x] = v;
            continue;
        }
        const int xl = (ql >= 0 && ql >= x - gap) ? ql : max(x - gap - 1, -1);
        const int xr = (qr < w && qr <= x + gap) ? qr : min(x + gap + 1, w);
        const float dl = (xl >= 0 && row[xl] >= 0.f) ? row[xl] : -1.f;
        const float dr = (xr < w && row[xr] >= 0.f) ? row[xr] : -1.f;
        const size_t i = (size_t)y * w + x;
        float o = v;
        if (occlusion_like(reason[i], shadow, dl, dr)) {
            if (dl >= 0.f && dr >= 0.f) o = (dr < dl) ? dr : dl;
            else if (dl >= 0.f) o = dl;
            else if (dr >= 0.f) o = dr;
            out[i] = o;
            continue;
        }
        const int c0 = gray[i];
        float best_d = -1.f;
        int best_abs = 999;
        const int cx[4] = {xl, xr, x, x};
        const int cy[4] = {y, y, y - 1, y + 1};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int xx = cx[k], yy = cy[k];
            if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
            const float dv = in[(size_t)yy * w + xx];
            if (dv < 0.f) continue;
            const int ad = abs((int)gray[(size_t)yy * w + xx] - c0);
            if (ad < best_abs) { best_abs = ad; best_d = dv; }
        }
        if (best_d >= 0.f && best_abs <= 18) {
            o = best_d;
        } else if (d_prior && d_prior[i] >= 0.f) {
            o = d_prior[i];
        } else if (dl >= 0.f && dr >= 0.f) {
            const float t = __fdiv_rn((float)(x - xl), (float)(xr - xl));
            o = __fadd_rn(__fmul_rn(dl, __fsub_rn(1.f, t)), __fmul_rn(dr, t));
        } else if (dl >= 0.f) {
            o = dl;
        } else if (dr >= 0.f) {
            o = dr;
        }
        out[i] = o;
    }
}

// The 3x3 case (median_radius 1, the default) over a staged 34x10 tile: each thread sorts its nine
// window values in registers with a 25-exchange sorting network (invalid values, !(v >= 0), as
// +inf, so the cnt valid ones come first) and takes entry cnt/2 -- the cnt/2-th smallest, as the
// rank count above.  Equal values are interchangeable except +0 and -0; when the selected value is
// a zero, the first valid zero in raster order is returned, as the rank count does.
constexpr int kMedTX = 32, kMedTY = 8;

__device__ __forceinline__ void cswap(float& a, float& b) {
    const float lo = fminf(a, b), hi = fmaxf(a, b);
    a = lo;
    b = hi;
}

// Rows [y_begin, y_end) of the frame (the window reads rows y_begin - 1 .. y_end inside the frame).
__global__ void __launch_bounds__(kMedTX * kMedTY) median3_kernel(int w, int h, int y_begin, int y_end,
                                                                  const float* __restrict__ in,
                                                                  float* __restrict__ out) {
    __shared__ float t[kMedTY + 2][kMedTX + 2];
    const int x0 = blockIdx.x * kMedTX, y0 = y_begin + blockIdx.y * kMedTY;
    const int tid = threadIdx.y * kMedTX + threadIdx.x;
    for (int i = tid; i < (kMedTY + 2) * (kMedTX + 2); i += kMedTX * kMedTY) {
        const int sy = i / (kMedTX + 2), sx = i - sy * (kMedTX + 2);
        const int yy = y0 + sy - 1, xx = x0 + sx - 1;
        // outside the image: not part of the window (invalid)
        t[sy][sx] = (xx >= 0 && xx < w && yy >= 0 && yy < h) ? in[(size_t)yy * w + xx] : -1.f;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= y_end) return;
    float v[9];
    int cnt = 0;
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
            const float u = t[threadIdx.y + dy][threadIdx.x + dx];
            const bool ok = u >= 0.f;
            cnt += ok;
            v[dy * 3 + dx] = ok ? u : __int_as_float(0x7f800000);
        }
    const float center = t[threadIdx.y + 1][threadIdx.x + 1];
    if (cnt == 0) {
        out[(size_t)y * w + x] = center;
        return;
    }
    float s[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) s[i] = v[i];
    // 9-input sorting network (25 compare-exchanges)
    cswap(s[0], s[3]); cswap(s[1], s[7]); cswap(s[2], s[5]); cswap(s[4], s[8]);
    cswap(s[0], s[7]); cswap(s[2], s[4]); cswap(s[3], s[8]); cswap(s[5], s[6]);
    cswap(s[0], s[2]); cswap(s[1], s[3]); cswap(s[4], s[5]); cswap(s[7], s[8]);
    cswap(s[1], s[4]); cswap(s[3], s[6]); cswap(s[5], s[7]);
    cswap(s[0], s[1]); cswap(s[2], s[4]); cswap(s[3], s[5]); cswap(s[6], s[8]);
    cswap(s[2], s[3]); cswap(s[4], s[5]); cswap(s[6], s[7]);
    cswap(s[1], s[2]); cswap(s[3], s[4]); cswap(s[5], s[6]);
    const int k = cnt / 2;
    float res = s[0];
#pragma unroll
    for (int i = 1; i < 9; ++i)
        if (i == k) res = s[i];
    if (res == 0.f) {
        // the sign of the first valid zero in raster order
#pragma unroll
        for (int i = 8; i >= 0; --i)
            if (v[i] == 0.f) res = v[i];
    }
    out[(size_t)y * w + x] = res;
}

// Frame counters of PipelineStats (src/pipeline.cpp:650-707): out[0] valid (disparity >= 0),
// out[1] reliable (mask != 0), out[2] lr_fail (reason Occlusion or Mismatch), out[3] refine_changed
// (before and after both >= 0 and |after - before| > 1e-4), out[4] sum over pixels of the search
// range width max(hi - lo, 0) -- read from the range planes, or, for the default ranges (rmin
// null), the host's closed form `range_sum`.  Four pixels per thread and step when the buffers
// allow 16-byte and 4-byte loads (n4 = n / 4, the tail one pixel at a time), warp
// and block reductions, then one 64-bit atomic per block and counter (a few hundred blocks:
// same-address atomics serialise at L2); out[] starts at zero.
__device__ __forceinline__ void stats_pixel(unsigned long long (&c)[5], float d, uint8_t rel, uint8_t r,
                                            const float* before, const float* after, const int16_t* rmin,
                                            const int16_t* rmax, int p) {
    c[0] += d >= 0.f;
    c[1] += rel != 0;
    c[2] += (r == kOcclusion || r == kMismatch);
    if (before) {
        const float db = before[p], da = after[p];
        c[3] += (db >= 0.f && da >= 0.f && fabsf(__fsub_rn(da, db)) > 1e-4f);
    }
    if (rmin) {
        const int wd = (int)rmax[p] - (int)rmin[p];
        c[4] += wd > 0 ? (unsigned)wd : 0u;
    }
}

__global__ void __launch_bounds__(256) frame_stats_kernel(int n, const float* __restrict__ disp,
                                                          const uint8_t* __restrict__ reliable,
                                                          const uint8_t* __restrict__ reason,
                                                          const float* __restrict__ before,
                                                          const float* __restrict__ after,
                                                          const int16_t* __restrict__ rmin,
                                                          const int16_t* __restrict__ rmax,
                                                          unsigned long long range_sum, bool vec,
                                                          unsigned long long* __restrict__ out) {
    unsigned long long c[5] = {0, 0, 0, 0, 0};
    const int stride = gridDim.x * blockDim.x;
    int tail = 0;
    if (vec) {
        const int n4 = n / 4;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
            const float4 d = reinterpret_cast<const float4*>(disp)[q];
            const uchar4 rl = reinterpret_cast<const uchar4*>(reliable)[q];
            const uchar4 rs = reinterpret_cast<const uchar4*>(reason)[q];
            stats_pixel(c, d.x, rl.x, rs.x, before, after, rmin, rmax, 4 * q);
            stats_pixel(c, d.y, rl.y, rs.y, before, after, rmin, rmax, 4 * q + 1);
            stats_pixel(c, d.z, rl.z, rs.z, before, after, rmin, rmax, 4 * q + 2);
            stats_pixel(c, d.w, rl.w, rs.w, before, after, rmin, rmax, 4 * q + 3);
        }
        tail = 4 * n4;
    }
    for (int p = tail + blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride)
        stats_pixel(c, disp[p], reliable[p], reason[p], before, after, rmin, rmax, p);
    if (blockIdx.x == 0 && threadIdx.x == 0) c[4] += range_sum;
    __shared__ unsigned long long s_c[5][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        unsigned long long v = c[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_c[i][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        unsigned long long v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s_c[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, v);
    }
}

inline int grid_for(int n) {
    const int b = (n + 255) / 256;
    return b < 148 * 16 ? b : 148 * 16;
}

}  // namespace

cudaError_t launch_conf_lr(const ConfLrArgs& a, cudaStream_t s) {
    conf_lr_kernel<<<grid_for(a.w * a.h), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_lr(int w, int h, int lr_max_diff, const float* dr, const float* din, float* dout,
                      uint8_t* reason, cudaStream_t s) {
    lr_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, lr_max_diff, dr, din, dout, reason);
    return cudaGetLastError();
}

cudaError_t launch_fill(int w, int h, int gap, int shadow, apg_inpaint_telemetry_t* tel, const float* in,
                        const uint8_t* reason, const uint8_t* gray, const float* d_prior, float* out, cudaStream_t s) {
    if (tel) {
        // telemetry: the per-pixel form (same map) counts every hole, one thread per row the runs
        fill_runs_kernel<<<(h + 127) / 128, 128, 0, s>>>(w, h, gap, in, tel);
        fill_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, gap, shadow, tel, in, reason, gray, d_prior, out);
        return cudaGetLastError();
    }
    if (gap >= 0) {
        const long long warps = (long long)((w + 31) / 32) * h;
        const int blocks = (int)std::min<long long>((warps + 7) / 8, 148 * 16);
        fill_ballot_kernel<<<blocks, 256, 0, s>>>(w, h, 0, h, gap, shadow, in, reason, gray, d_prior, out);
    } else {
        fill_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, gap, shadow, nullptr, in, reason, gray, d_prior, out);
    }
    return cudaGetLastError();
}

cudaError_t launch_median(int w, int h, int r, const float* in, float* out, cudaStream_t s) {
    if (r == 1) {
        const dim3 grid((w + kMedTX - 1) / kMedTX, (h + kMedTY - 1) / kMedTY), block(kMedTX, kMedTY);
        median3_kernel<<<grid, block, 0, s>>>(w, h, 0, h, in, out);
    } else {
        median_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, r, in, out);
    }
    return cudaGetLastError();
}

cudaError_t launch_fill_rows(int w, int h, int y_begin, int y_end, int gap, int shadow, const float* in,
                             const uint8_t* reason, const uint8_t* gray, const float* d_prior, float* out,
                             cudaStream_t s) {
    if (gap < 0 || y_begin < 0 || y_end > h || y_end <= y_begin) return cudaErrorInvalidValue;
    const long long warps = (long long)((w + 31) / 32) * (y_end - y_begin);
    const int blocks = (int)std::min<long long>((warps + 7) / 8, 148 * 16);
    fill_ballot_kernel<<<blocks, 256, 0, s>>>(w, h, y_begin, y_end, gap, shadow, in, reason, gray, d_prior, out);
    return cudaGetLastError();
}

cudaError_t launch_median3_rows(int w, int h, int y_begin, int y_end, const float* in, float* out, cudaStream_t s) {
    if (y_begin < 0 || y_end > h || y_end <= y_begin) return cudaErrorInvalidValue;
    const dim3 grid((w + kMedTX - 1) / kMedTX, (y_end - y_begin + kMedTY - 1) / kMedTY), block(kMedTX, kMedTY);
    median3_kernel<<<grid, block, 0, s>>>(w, h, y_begin, y_end, in, out);
    return cudaGetLastError();
}

cudaError_t launch_frame_stats(int n, const float* disp, const uint8_t* reliable, const uint8_t* reason,
                               const float* before, const float* after, const int16_t* rmin, const int16_t* rmax,
                               unsigned long long range_sum, unsigned long long* out5, cudaStream_t s) {
    const int blocks = (n + 255) / 256 < 148 * 2 ? (n + 255) / 256 : 148 * 2;
    // 16-byte loads of the map and 4-byte loads of the byte planes need those alignments
    const bool vec = ((reinterpret_cast<uintptr_t>(disp) & 15) | (reinterpret_cast<uintptr_t>(reliable) & 3) |
                      (reinterpret_cast<uintptr_t>(reason) & 3)) == 0;
    frame_stats_kernel<<<blocks, 256, 0, s>>>(n, disp, reliable, reason, before, after, rmin, rmax, range_sum, vec,
                                              out5);
    return cudaGetLastError();
}

}  // namespace apgcu

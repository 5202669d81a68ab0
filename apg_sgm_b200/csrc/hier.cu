// Hierarchical coarse-to-fine search range (HierarchicalStereo::estimate_search_range,
// src/hierarchical_stereo.cpp:113-431): the two per-pixel steps around the half-size pipeline
// pass that Engine::run_hier enqueues on the engine stream.
//
//   hier_downsample_kernel  2x2 box average of both full-size grays, (sum + 2) / 4
//                           (hierarchical_stereo.cpp:148-170)
//   hier_range_kernel       per full-size pixel, the search range [lo, hi) and the guiding
//                           disparity from the coarse pass's final disparity and confidence
//                           (hierarchical_stereo.cpp:280-410), plus HierarchicalTelemetry's
//                           numerators (coarse valid pixels, fallback pixels, full-range pixels,
//                           sum of widths) as four 64-bit counters
//
// Both are HBM-bound byte work: the downsample reads 4 and writes 0.5 bytes per full-size pixel
// of each image; the range step reads the quarter-size coarse planes (L2-resident: 8 bytes per
// coarse pixel) and writes 8 bytes per full-size pixel (two int16 bounds, one float).
#include "kernels.h"

namespace apgcu {

namespace {

__global__ void __launch_bounds__(256) hier_downsample_kernel(const uint8_t* __restrict__ lg, const uint8_t* __restrict__ rg,
                                                              int W, int H, int Wc, int Hc, uint8_t* __restrict__ cl,
                                                              uint8_t* __restrict__ cr) {
    const int nc = Wc * Hc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nc; i += gridDim.x * blockDim.x) {
        const int yc = i / Wc, xc = i - yc * Wc;
        const int y0 = yc * 2, y1 = min(y0 + 1, H - 1);
        const int x0 = xc * 2, x1 = min(x0 + 1, W - 1);
        const size_t a = (size_t)y0 * W, b = (size_t)y1 * W;
        const int sl = lg[a + x0] + lg[a + x1] + lg[b + x0] + lg[b + x1];
        const int sr = rg[a + x0] + rg[a + x1] + rg[b + x0] + rg[b + x1];
        cl[i] = (uint8_t)((sl + 2) / 4);
        cr[i] = (uint8_t)((sr + 2) / 4);
    }
}

struct HierArgs {
    int W, H, Wc, Hc, d0, dmax;
    int radius, adaptive, expanded, fallback;
    float threshold;
    const float* cd;  // coarse final disparity, Wc*Hc
    const float* cf;  // coarse final confidence, Wc*Hc
    int16_t* rmin;
    int16_t* rmax;
    float* d_prior;
    unsigned long long* counts;  // coarse valid, fallback, full range, sum of widths (two's complement)
};

// std::min / std::max on floats, operand order as the reference's calls.
__device__ __forceinline__ float ref_min(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float ref_max(float a, float b) { return (a < b) ? b : a; }

__global__ void __launch_bounds__(256) hier_range_kernel(HierArgs a) {
    const int n = a.W * a.H, nc = a.Wc * a.Hc;
    long long cvalid = 0, nfall = 0, nfull = 0, wsum = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < nc) cvalid += __ldg(a.cd + i) >= 0.f;
        const int y = i / a.W, x = i - y * a.W;
        const int xc = max(0, min(x / 2, a.Wc - 1)), yc = max(0, min(y / 2, a.Hc - 1));
        const int xc1 = min(xc + 1, a.Wc - 1), yc1 = min(yc + 1, a.Hc - 1);
        const float q0 = __ldg(a.cd + yc * a.Wc + xc), q1 = __ldg(a.cd + yc * a.Wc + xc1);
        const float q2 = __ldg(a.cd + yc1 * a.Wc + xc), q3 = __ldg(a.cd + yc1 * a.Wc + xc1);
        float mn = 1e9f, mx = -1e9f;
        int nv = 0;
        if (q0 >= 0.f) { mn = ref_min(mn, q0); mx = ref_max(mx, q0); ++nv; }
        if (q1 >= 0.f) { mn = ref_min(mn, q1); mx = ref_max(mx, q1); ++nv; }
        if (q2 >= 0.f) { mn = ref_min(mn, q2); mx = ref_max(mx, q2); ++nv; }
        if (q3 >= 0.f) { mn = ref_min(mn, q3); mx = ref_max(mx, q3); ++nv; }
        const int glo = a.d0, ghi = min(a.dmax, x + 1);
        int lo = glo, hi = ghi;
        float dp = -1.f;
        bool guided = false;
        if (nv > 0) {
            const float dc = q0 >= 0.f ? q0 : __fmul_rn(0.5f, __fadd_rn(mn, mx));
            const float Dc = 2.0f * dc;
            int er = a.radius;
            if (a.adaptive && __ldg(a.cf + yc * a.Wc + xc) < a.threshold) er = a.expanded;
            lo = min((int)floorf(Dc) - er, (int)floorf(2.0f * mn) - 1);
            hi = max((int)ceilf(Dc) + er + 1, (int)ceilf(2.0f * mx) + 2);
            dp = Dc;
            guided = true;
        } else {
            ++nfall;
            if (a.fallback != APG_HIER_FALLBACK_FULL_RANGE) {
                // nearest valid coarse pixel within 4 coarse pixels, first in raster order on ties
                float near = -1.f;
                int best = 1000;
                const int sy1 = min(a.Hc - 1, yc + 4), sx0 = max(0, xc - 4), sx1 = min(a.Wc - 1, xc + 4);
                for (int sy = max(0, yc - 4); sy <= sy1; ++sy)
                    for (int sx = sx0; sx <= sx1; ++sx) {
                        const float v = __ldg(a.cd + sy * a.Wc + sx);
                        const int d2 = (sx - xc) * (sx - xc) + (sy - yc) * (sy - yc);
                        if (v >= 0.f && d2 < best) { best = d2; near = v; }
                    }
                if (near >= 0.f) {
                    const float Dn = 2.0f * near;
                    const int re = a.fallback == APG_HIER_FALLBACK_EXPANDED_RADIUS ? 2 * a.radius : a.radius + 8;
                    lo = (int)floorf(Dn) - re;
                    hi = (int)ceilf(Dn) + re + 1;
                    dp = Dn;
                    guided = true;
                }
            }
        }
        if (guided) {
            lo = max(lo, glo);
            hi = min(hi, ghi);
            if (hi < lo) hi = lo;
            wsum += hi - lo;
            nfull += (hi - lo == ghi - glo);
        } else {
            wsum += ghi - glo;  // the full-range branches count the unclamped width
            ++nfull;
        }
        // SearchRange::set_pixel (include/apg_sgm/search_range.hpp:29-35)
        int slo = max(lo, a.d0), shi = min(hi, a.dmax);
        if (shi < slo) shi = slo;
        a.rmin[i] = (int16_t)slo;
        a.rmax[i] = (int16_t)shi;
        a.d_prior[i] = dp;
    }
    // block sums, then one atomic per counter and block
    __shared__ long long part[4][8];
    long long v[4] = {cvalid, nfall, nfull, wsum};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        long long t = v[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) part[k][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[threadIdx.x][w];
        if (t) atomicAdd(a.counts + threadIdx.x, (unsigned long long)t);
    }
}

}  // namespace

cudaError_t launch_hier_downsample(const uint8_t* lg, const uint8_t* rg, int w, int h, uint8_t* cl, uint8_t* cr,
                                   cudaStream_t s) {
    const int wc = w / 2, hc = h / 2, nc = wc * hc;
    if (nc <= 0) return cudaSuccess;
    const int blocks = std::min((nc + 255) / 256, 148 * 8);
    hier_downsample_kernel<<<blocks, 256, 0, s>>>(lg, rg, w, h, wc, hc, cl, cr);
    return cudaGetLastError();
}

cudaError_t launch_hier_range(const apg_pipeline_config_t& c, int w, int h, const float* coarse_disp,
                              const float* coarse_conf, int16_t* rmin, int16_t* rmax, float* d_prior,
                              unsigned long long* counts, cudaStream_t s) {
    HierArgs a;
    a.W = w; a.H = h; a.Wc = w / 2; a.Hc = h / 2;
    a.d0 = c.min_disparity; a.dmax = c.max_disparity;
    a.radius = c.hier_radius; a.adaptive = c.hier_adaptive_radius; a.expanded = c.hier_expanded_radius;
    a.fallback = c.hier_fallback; a.threshold = c.hier_confidence_threshold;
    a.cd = coarse_disp; a.cf = coarse_conf;
    a.rmin = rmin; a.rmax = rmax; a.d_prior = d_prior; a.counts = counts;
    const int n = w * h;
    const int blocks = std::min((n + 255) / 256, 148 * 8);
    hier_range_kernel<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace apgcu

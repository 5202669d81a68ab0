// Per-pixel back end: confidence, left-right check, hole fill, median.
//
// Restates ConfidenceEstimator::estimate (src/confidence_estimator.cpp:7-63),
// PostProcessor::left_right_check / fill_holes (Legacy route) / median
// (src/postprocess.cpp:10-40, 42-168, 255-309).  Every float expression keeps the reference's
// operation order with explicitly rounded intrinsics (no contraction), so outputs are bit-exact.
// These kernels touch O(W*H) bytes and are a few microseconds each at 720p.
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

// Legacy hole fill, src/postprocess.cpp:87-168.  Reads the pre-fill map, writes a copy.
__global__ void fill_kernel(int w, int h, int gap, const float* __restrict__ in, const uint8_t* __restrict__ reason,
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
        float o = v;
        if (reason[i] == kOcclusion) {
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

// Frame counters of PipelineStats (src/pipeline.cpp:650-707): out[0] valid (disparity >= 0),
// out[1] reliable (mask != 0), out[2] lr_fail (reason Occlusion or Mismatch), out[3] refine_changed
// (before and after both >= 0 and |after - before| > 1e-4), out[4] sum over pixels of the search
// range width max(hi - lo, 0).  Warp and block reductions, then one 64-bit atomic per block and
// counter (a few hundred blocks: same-address atomics serialise at L2); out[] starts at zero.
__global__ void __launch_bounds__(256) frame_stats_kernel(int n, const float* __restrict__ disp,
                                                          const uint8_t* __restrict__ reliable,
                                                          const uint8_t* __restrict__ reason,
                                                          const float* __restrict__ before,
                                                          const float* __restrict__ after,
                                                          const int16_t* __restrict__ rmin,
                                                          const int16_t* __restrict__ rmax,
                                                          unsigned long long* __restrict__ out) {
    unsigned long long c[5] = {0, 0, 0, 0, 0};
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        c[0] += disp[p] >= 0.f;
        c[1] += reliable[p] != 0;
        const uint8_t r = reason[p];
        c[2] += (r == kOcclusion || r == kMismatch);
        if (before) {
            const float db = before[p], da = after[p];
            c[3] += (db >= 0.f && da >= 0.f && fabsf(__fsub_rn(da, db)) > 1e-4f);
        }
        const int wd = (int)rmax[p] - (int)rmin[p];
        c[4] += wd > 0 ? (unsigned)wd : 0u;
    }
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

cudaError_t launch_fill(int w, int h, int gap, const float* in, const uint8_t* reason, const uint8_t* gray,
                        const float* d_prior, float* out, cudaStream_t s) {
    fill_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, gap, in, reason, gray, d_prior, out);
    return cudaGetLastError();
}

cudaError_t launch_median(int w, int h, int r, const float* in, float* out, cudaStream_t s) {
    median_kernel<<<grid_for(w * h), 256, 0, s>>>(w, h, r, in, out);
    return cudaGetLastError();
}

cudaError_t launch_frame_stats(int n, const float* disp, const uint8_t* reliable, const uint8_t* reason,
                               const float* before, const float* after, const int16_t* rmin, const int16_t* rmax,
                               unsigned long long* out5, cudaStream_t s) {
    const int blocks = (n + 255) / 256 < 148 * 2 ? (n + 255) / 256 : 148 * 2;
    frame_stats_kernel<<<blocks, 256, 0, s>>>(n, disp, reliable, reason, before, after, rmin, rmax, out5);
    return cudaGetLastError();
}

}  // namespace apgcu

// Accuracy metrics on the device: evaluate_stereo (src/metrics.cpp:119-502) without the support
// block, for dataset-scale evaluation beside the matcher.
//
// One pass over the frame: each warp takes 32 consecutive pixels per step; every tally of the
// reference (include/apg_sgm/metrics.h: 76 integer counts, 15 double sums of float errors) is
// one warp ballot + popcount per step, added by the lane that owns it (counter k lives in lane
// k % 32), and the double sums stay in each lane's registers.  The disparity-boundary mask (GT
// 4-neighbour difference) and the low-texture mask (luma central difference) are computed on the
// fly from the neighbours, in the reference's float operation order.  Blocks write their tallies
// to a partial buffer in a fixed tree order and one block adds the partials in block order, so a
// frame's result does not depend on scheduling; the float ratios are then formed on the host with
// the reference's expressions (apg_metrics_finalize).
//
// Counts are exact.  Each double sum is the exact sum whenever the reference's own sequential
// double sum is exact (e.g. errors on a 2^-24 grid below 2^8 over up to 2^21 pixels); otherwise
// the two differ by the rounding of the reference's summation order, far below the float the
// sum is divided into.
//
// HBM-bound: 8 bytes per pixel (estimate, GT) plus the optional planes (ranges 4, refine maps 8,
// visibility 1, left image 1-3); the neighbour reads hit L1/L2.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/apg_sgm/metrics.h"
#include "common.cuh"

namespace apgcu {

namespace {

constexpr int kMetricBlocks = 296;  // fixed grid: the summation order depends on it, not on the device
constexpr int kMetricThreads = 256;
constexpr int kSlots = (APG_MC_COUNT + 31) / 32;

struct MetricArgs {
    const float* est;
    const float* gt;
    int w, h;
    const int16_t* rmin;
    const int16_t* rmax;
    const float* before;
    const float* after;
    const uint8_t* vis;
    float max_gt;
    const uint8_t* left;
    int lstride, lch;
    float boundary, lowtex;
    unsigned* part_c;  // kMetricBlocks x APG_MC_COUNT
    double* part_s;    // kMetricBlocks x APG_MS_COUNT
};

__device__ __forceinline__ bool gt_ok(float g, float mx) { return isfinite(g) && g >= 0.0f && g < mx; }

__device__ __forceinline__ float luma(const MetricArgs& a, int x, int y) {
    const uint8_t* p = a.left + (size_t)y * a.lstride + (size_t)x * a.lch;
    if (a.lch == 1) return (float)p[0];
    return __fadd_rn(__fadd_rn(__fmul_rn(0.299f, (float)p[0]), __fmul_rn(0.587f, (float)p[1])),
                     __fmul_rn(0.114f, (float)p[2]));
}

// Warp tally: counter K gets the number of lanes whose predicate holds, in its owner lane.
template <int K>
__device__ __forceinline__ void tally(unsigned (&acc)[kSlots], int lane, bool p) {
    const unsigned b = __ballot_sync(0xffffffffu, p);
    if (lane == (K & 31)) acc[K >> 5] += __popc(b);
}

template <int R>
__device__ __forceinline__ void region(unsigned (&acc)[kSlots], double (&sum)[APG_MS_COUNT], int lane, bool in,
                                       bool ok, float diff, bool d1) {
    constexpr int b = APG_MC_REGION0 + 7 * R;
    tally<b + 0>(acc, lane, in);
    tally<b + 1>(acc, lane, in && ok);
    tally<b + 2>(acc, lane, in && ok && diff > 0.5f);
    tally<b + 3>(acc, lane, in && ok && diff > 1.0f);
    tally<b + 4>(acc, lane, in && ok && diff > 2.0f);
    tally<b + 5>(acc, lane, in && ok && diff > 3.0f);
    tally<b + 6>(acc, lane, in && d1);
    if (in && ok) sum[APG_MS_REGION0 + R] += diff;
}

__global__ void __launch_bounds__(kMetricThreads) metrics_kernel(MetricArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned acc[kSlots] = {};
    double sum[APG_MS_COUNT] = {};
    const int n = a.w * a.h;
    const bool has_range = a.rmin && a.rmax, has_ref = a.before && a.after, has_left = a.left != nullptr;
    const int gwarp = blockIdx.x * (kMetricThreads / 32) + warp, nwarps = gridDim.x * (kMetricThreads / 32);
    for (int base = gwarp * 32; base < n; base += nwarps * 32) {
        const int i = base + lane;
        const bool inb = i < n;
        const int y = inb ? i / a.w : 0, x = inb ? i - y * a.w : 0;
        const float g = inb ? a.gt[i] : -1.0f;
        const bool ev = inb && gt_ok(g, a.max_gt);
        // disparity boundary: largest |g - neighbour| over the valid 4-neighbours (+x, -x, +y, -y)
        bool edge = false;
        bool visible = false, matchable = false;
        float e = -1.0f;
        if (ev) {
            float md = 0.0f;
            const int nx[4] = {x + 1, x - 1, x, x}, ny[4] = {y, y, y + 1, y - 1};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (nx[k] >= 0 && nx[k] < a.w && ny[k] >= 0 && ny[k] < a.h) {
                    const float ng = a.gt[ny[k] * a.w + nx[k]];
                    if (gt_ok(ng, a.max_gt)) {
                        const float d = fabsf(__fsub_rn(g, ng));
                        md = (md < d) ? d : md;
                    }
                }
            }
            edge = md >= a.boundary;
            const int xr = x - (int)roundf(g);
            matchable = xr >= 0 && xr < a.w;
            visible = a.vis ? a.vis[i] >= 200 : matchable;
            e = a.est[i];
        }
        const bool ok = ev && isfinite(e) && e >= 0.0f;
        const float adiff = fabsf(__fsub_rn(e, g));
        const float diff = ok ? adiff : 1e9f;
        const bool d1 = ev && (!ok || (adiff > 3.0f && (g > 1e-3f ? (__fdiv_rn(adiff, g) > 0.05f) : true)));

        tally<APG_MC_EVALUATED>(acc, lane, ev);
        tally<APG_MC_VALID>(acc, lane, ok);
        tally<APG_MC_C05>(acc, lane, ok && diff > 0.5f);
        tally<APG_MC_C10>(acc, lane, ok && diff > 1.0f);
        tally<APG_MC_C20>(acc, lane, ok && diff > 2.0f);
        tally<APG_MC_C30>(acc, lane, ok && diff > 3.0f);
        tally<APG_MC_D1_ALL>(acc, lane, d1);
        tally<APG_MC_D1_NOC>(acc, lane, d1 && visible);
        tally<APG_MC_EVAL_NOC>(acc, lane, ev && visible);
        tally<APG_MC_LR_FAIL>(acc, lane, ev && !ok);
        tally<APG_MC_EDGE>(acc, lane, ok && edge);
        tally<APG_MC_NONEDGE>(acc, lane, ok && !edge);
        if (ok) {
            sum[APG_MS_EPE] += diff;
            sum[edge ? APG_MS_EDGE : APG_MS_NONEDGE] += diff;
        }
        if (has_range) {
            bool in = false;
            if (ev) in = g >= (float)a.rmin[i] && g < (float)a.rmax[i];
            tally<APG_MC_EVAL_ALL>(acc, lane, ev);
            tally<APG_MC_IN_ALL>(acc, lane, ev && in);
            tally<APG_MC_EVAL_MATCH>(acc, lane, ev && matchable);
            tally<APG_MC_IN_MATCH>(acc, lane, ev && matchable && in);
            tally<APG_MC_EVAL_VIS>(acc, lane, ev && visible);
            tally<APG_MC_IN_VIS>(acc, lane, ev && visible && in);
            tally<APG_MC_MISS_VIS>(acc, lane, ev && visible && !in);
            tally<APG_MC_MISS_EDGE>(acc, lane, ev && visible && !in && edge);
            tally<APG_MC_MISS_NONEDGE>(acc, lane, ev && visible && !in && !edge);
        }
        region<0>(acc, sum, lane, ev, ok, diff, d1);
        region<1>(acc, sum, lane, ev && visible, ok, diff, d1);
        region<2>(acc, sum, lane, ev && !visible, ok, diff, d1);
        region<3>(acc, sum, lane, ev && edge, ok, diff, d1);
        region<4>(acc, sum, lane, ev && !edge, ok, diff, d1);
        if (has_left) {
            bool low = false;
            if (ev) {
                const int xp = max(0, x - 1), xn = min(a.w - 1, x + 1), yp = max(0, y - 1), yn = min(a.h - 1, y + 1);
                const float sx = (x == 0 || x == a.w - 1) ? 1.0f : 2.0f, sy = (y == 0 || y == a.h - 1) ? 1.0f : 2.0f;
                const float dx = __fdiv_rn(__fsub_rn(luma(a, xn, y), luma(a, xp, y)), sx);
                const float dy = __fdiv_rn(__fsub_rn(luma(a, x, yn), luma(a, x, yp)), sy);
                low = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))) < a.lowtex;
            }
            region<5>(acc, sum, lane, ev && low, ok, diff, d1);
            region<6>(acc, sum, lane, ev && !low, ok, diff, d1);
        }
        if (has_ref) {
            bool rv = false;
            float db = 0.0f, da = 0.0f, eb = 0.0f, ea = 0.0f;
            if (ev) {
                eb = a.before[i];
                ea = a.after[i];
                rv = isfinite(eb) && eb >= 0.0f && isfinite(ea) && ea >= 0.0f;
                db = fabsf(__fsub_rn(eb, g));
                da = fabsf(__fsub_rn(ea, g));
            }
            const bool improved = rv && da < __fsub_rn(db, 1e-4f);
            const bool worsened = rv && !improved && da > __fadd_rn(db, 1e-4f);
            tally<APG_MC_REF_EVAL>(acc, lane, rv);
            tally<APG_MC_REF_IMPROVED>(acc, lane, improved);
            tally<APG_MC_REF_WORSENED>(acc, lane, worsened);
            tally<APG_MC_REF_UNCHANGED>(acc, lane, rv && !improved && !worsened);
            tally<APG_MC_REF_CHANGED>(acc, lane, rv && fabsf(__fsub_rn(ea, eb)) > 1e-4f);
            tally<APG_MC_TOTAL_EVAL>(acc, lane, rv && ok);
            if (rv) {
                sum[APG_MS_BEFORE] += db;
                sum[APG_MS_AFTER] += da;
                if (ok) {
                    sum[APG_MS_TOT_BEFORE] += db;
                    sum[APG_MS_TOT_AFTER] += da;
                    sum[APG_MS_TOT_FINAL] += adiff;
                }
            }
        }
    }
    // block partials in a fixed order: doubles by a shuffle tree per warp, then warps in order
    __shared__ unsigned sc[kMetricThreads / 32][kSlots * 32];
    __shared__ double ss[kMetricThreads / 32][APG_MS_COUNT];
#pragma unroll
    for (int k = 0; k < kSlots; ++k) sc[warp][k * 32 + lane] = acc[k];
#pragma unroll
    for (int k = 0; k < APG_MS_COUNT; ++k) {
        double v = sum[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) ss[warp][k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < APG_MC_COUNT; k += blockDim.x) {
        unsigned t = 0;
        for (int wp = 0; wp < kMetricThreads / 32; ++wp) t += sc[wp][k];
        a.part_c[blockIdx.x * APG_MC_COUNT + k] = t;
    }
    for (int k = threadIdx.x; k < APG_MS_COUNT; k += blockDim.x) {
        double t = 0.0;
        for (int wp = 0; wp < kMetricThreads / 32; ++wp) t += ss[wp][k];
        a.part_s[blockIdx.x * APG_MS_COUNT + k] = t;
    }
}

__global__ void metrics_final_kernel(const unsigned* part_c, const double* part_s, long long* out_c, double* out_s) {
    for (int k = threadIdx.x; k < APG_MC_COUNT; k += blockDim.x) {
        long long t = 0;
        for (int b = 0; b < kMetricBlocks; ++b) t += part_c[b * APG_MC_COUNT + k];
        out_c[k] = t;
    }
    for (int k = threadIdx.x; k < APG_MS_COUNT; k += blockDim.x) {
        double t = 0.0;
        for (int b = 0; b < kMetricBlocks; ++b) t += part_s[b * APG_MS_COUNT + k];
        out_s[k] = t;
    }
}

}  // namespace

// Scratch bytes of one evaluation: block partials and the final tallies.
size_t metrics_scratch_bytes() {
    return (size_t)kMetricBlocks * (APG_MC_COUNT * 4 + APG_MS_COUNT * 8) + APG_MC_COUNT * 8 + APG_MS_COUNT * 8 + 512;
}

// Enqueues the two kernels; the tallies land in `scratch` (device, metrics_scratch_bytes()) at
// offsets returned through out_c / out_s.
cudaError_t launch_metrics(const float* est, const float* gt, int w, int h, const int16_t* rmin, const int16_t* rmax,
                           const float* before, const float* after, const uint8_t* vis, float max_valid_gt,
                           const uint8_t* left, int left_stride, int left_ch, const apg_quality_thresholds_t& thr,
                           unsigned char* scratch, long long** out_c, double** out_s, cudaStream_t s) {
    MetricArgs a;
    a.est = est; a.gt = gt; a.w = w; a.h = h; a.rmin = rmin; a.rmax = rmax; a.before = before; a.after = after;
    a.vis = vis; a.max_gt = max_valid_gt; a.left = left; a.lstride = left_stride; a.lch = left_ch;
    a.boundary = thr.boundary_disparity_gradient; a.lowtex = thr.low_texture_gradient;
    size_t o = 0;
    a.part_s = reinterpret_cast<double*>(scratch + o);
    o += (size_t)kMetricBlocks * APG_MS_COUNT * 8;
    double* fs = reinterpret_cast<double*>(scratch + o);
    o += APG_MS_COUNT * 8;
    long long* fc = reinterpret_cast<long long*>(scratch + o);
    o += APG_MC_COUNT * 8;
    a.part_c = reinterpret_cast<unsigned*>(scratch + o);
    metrics_kernel<<<kMetricBlocks, kMetricThreads, 0, s>>>(a);
    metrics_final_kernel<<<1, 128, 0, s>>>(a.part_c, a.part_s, fc, fs);
    *out_c = fc;
    *out_s = fs;
    return cudaGetLastError();
}

void count_launches(unsigned n);

}  // namespace apgcu

// ------------------------------------------------------------------------------------------------
// C entry (include/apg_sgm_cuda.h)
// ------------------------------------------------------------------------------------------------
#include "../../include/apg_sgm_cuda.h"

namespace {
thread_local float g_metrics_ms = 0.0f;  // device time of this thread's last evaluation's kernels
}

extern "C" APGCU_API float apgcu_metrics_last_kernel_ms(void) { return g_metrics_ms; }

extern "C" APGCU_API int apgcu_evaluate_stereo(const float* est, const float* gt, int w, int h, const int16_t* rmin,
                                               const int16_t* rmax, const float* before, const float* after,
                                               const uint8_t* vis, float max_valid_gt, const uint8_t* left,
                                               int left_stride, int left_ch, const apg_quality_thresholds_t* thr,
                                               int device_buffers, void* stream, apg_stereo_metrics_t* out) {
    if (!out) return APG_STATUS_INTERNAL_ERROR;
    std::memset(out, 0, sizeof(*out));
    if (w <= 0 || h <= 0) return APG_STATUS_OK;  // evaluate_stereo returns an empty record
    if (!est || !gt) return APG_STATUS_EMPTY_INPUT;
    if (left && (left_ch < 1 || left_ch == 2 || left_ch > 4 || left_stride < w * left_ch)) return APG_STATUS_SIZE_MISMATCH;
    const apg_quality_thresholds_t T = thr ? *thr : apg_quality_thresholds_default();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)w * h;
    const bool has_range = rmin && rmax, has_ref = before && after;
    // device copies of host inputs go into one stream-ordered block beside the scratch
    size_t in_bytes = 0;
    auto a256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
    if (!device_buffers) {
        in_bytes = 2 * a256(n * 4) + (has_range ? 2 * a256(n * 2) : 0) + (has_ref ? 2 * a256(n * 4) : 0) +
                   (vis ? a256(n) : 0) + (left ? a256((size_t)left_stride * h) : 0);
    }
    const size_t scratch = apgcu::metrics_scratch_bytes();
    unsigned char* blk = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&blk), in_bytes + scratch, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return APG_STATUS_ALLOCATION_FAILURE;
    }
    const float *dE = est, *dG = gt, *dB = before, *dA = after;
    const int16_t *dR0 = rmin, *dR1 = rmax;
    const uint8_t *dV = vis, *dL = left;
    if (!device_buffers) {
        size_t o = 0;
        auto up = [&](const void* src, size_t bytes) -> void* {
            void* d = blk + o;
            o += a256(bytes);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, s);
            return d;
        };
        dE = static_cast<const float*>(up(est, n * 4));
        dG = static_cast<const float*>(up(gt, n * 4));
        if (has_range) {
            dR0 = static_cast<const int16_t*>(up(rmin, n * 2));
            dR1 = static_cast<const int16_t*>(up(rmax, n * 2));
        }
        if (has_ref) {
            dB = static_cast<const float*>(up(before, n * 4));
            dA = static_cast<const float*>(up(after, n * 4));
        }
        if (vis) dV = static_cast<const uint8_t*>(up(vis, n));
        if (left) dL = static_cast<const uint8_t*>(up(left, (size_t)left_stride * h));
    }
    long long* dc = nullptr;
    double* ds = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const bool timed = cudaEventCreate(&ev[0]) == cudaSuccess && cudaEventCreate(&ev[1]) == cudaSuccess;
    if (timed && e == cudaSuccess) cudaEventRecord(ev[0], s);
    if (e == cudaSuccess)
        e = apgcu::launch_metrics(dE, dG, w, h, has_range ? dR0 : nullptr, has_range ? dR1 : nullptr,
                                  has_ref ? dB : nullptr, has_ref ? dA : nullptr, dV, max_valid_gt, dL, left_stride,
                                  left_ch, T, blk + in_bytes, &dc, &ds, s);
    long long c[APG_MC_COUNT];
    double sm[APG_MS_COUNT];
    if (timed && e == cudaSuccess) cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) {
        apgcu::count_launches(2);
        e = cudaMemcpyAsync(c, dc, sizeof(c), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(sm, ds, sizeof(sm), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(blk, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (timed) {
        if (e == cudaSuccess) cudaEventElapsedTime(&g_metrics_ms, ev[0], ev[1]);
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return APG_STATUS_INTERNAL_ERROR;
    }
    apg_metrics_finalize(c, sm, w * h, has_range, has_ref, out);
    return APG_STATUS_OK;
}

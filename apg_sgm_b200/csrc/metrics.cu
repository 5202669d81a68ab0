// Accuracy metrics on the device: evaluate_stereo (src/metrics.cpp:119-502) without the support
// block, for dataset-scale evaluation beside the matcher.
//
// One pass over the frame: each warp takes 32 consecutive pixels per step.  Of the reference's 76
// integer tallies (include/apg_sgm/metrics.h) 44 are independent -- the 7 counts of the all,
// visible, boundary and low-texture regions, 5 range and 5 refine counts; the others are exact
// differences (occluded = all - visible, LR failures = evaluated - valid, ...) formed on the host.
// Each lane keeps the 44 as byte counters packed four to a register and adds a pixel's counts with
// one select and add per register; every 255 steps (and at the end) a warp folds its bytes into
// shared counters with two 16-bit-lane reductions per register.  The 12 independent double sums
// of float errors stay in registers.  The disparity-boundary mask (GT 4-neighbour difference) and
// the low-texture mask (luma central difference) are computed on the fly from the neighbours, in
// the reference's float operation order.  Blocks write their tallies to a partial buffer in a fixed
// order and one block adds the partials in a fixed order, so a frame's result does not depend on
// scheduling; the float ratios are then formed on the host with the reference's expressions
// (apg_metrics_finalize).
//
// Counts are exact.  Each double sum is the exact sum whenever the reference's own sequential
// double sum is exact (e.g. errors on a 2^-24 grid below 2^8 over up to 2^21 pixels); otherwise
// the two differ by the rounding of the reference's summation order, far below the float the
// sum is divided into.
//
// HBM-bound: 8 bytes per pixel (estimate, GT) plus the optional planes (ranges 4, refine maps 8,
// visibility 1, left image 1-3); the neighbour reads hit L1/L2.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>

#include "../../include/apg_sgm/metrics.h"
#include "common.cuh"

namespace apgcu {

namespace {

constexpr int kMetricBlocks = 444;  // fixed grid (3 blocks per SM on 148 SMs): the summation order depends on it only
constexpr int kMetricThreads = 256;
constexpr int kWarps = kMetricThreads / 32;
// Independent tallies: 4 regions x 7 (all, visible, boundary, low texture), 5 range and 5 refine
// counts, as 11 registers of four byte counters each; the other tallies of the reference are
// differences of these (occluded = all - visible, ...), formed on the host.
constexpr int kPacked = 11;
constexpr int kCounts = kPacked * 4;
// Independent double sums: the 7 region error sums and the 5 refine sums (the frame's error sums are
// the "all", "boundary" and "non-boundary" region sums: the same pixels in the same order).
constexpr int kSums = 12;

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
    unsigned* part_c;  // kMetricBlocks x kCounts
    double* part_s;    // kMetricBlocks x kSums
};

__device__ __forceinline__ bool gt_ok(float g, float mx) { return isfinite(g) && g >= 0.0f && g < mx; }

__device__ __forceinline__ float luma(const MetricArgs& a, int x, int y) {
    const uint8_t* p = a.left + (size_t)y * a.lstride + (size_t)x * a.lch;
    if (a.lch == 1) return (float)p[0];
    return __fadd_rn(__fadd_rn(__fmul_rn(0.299f, (float)p[0]), __fmul_rn(0.587f, (float)p[1])),
                     __fmul_rn(0.114f, (float)p[2]));
}

__device__ __forceinline__ unsigned pack4(bool a, bool b, bool c, bool d) {
    return (unsigned)a | ((unsigned)b << 8) | ((unsigned)c << 16) | ((unsigned)d << 24);
}

// Adds every lane's byte counters of the packed registers into the warp's shared counters (lane 0)
// and clears them: even and odd bytes as two 16-bit halves each, which a warp sum cannot overflow
// (32 x 255 < 2^16).
__device__ __forceinline__ void flush(unsigned (&p)[kPacked], unsigned* wc, int lane) {
#pragma unroll
    for (int k = 0; k < kPacked; ++k) {
        const unsigned ev = __reduce_add_sync(0xffffffffu, p[k] & 0x00FF00FFu);
        const unsigned od = __reduce_add_sync(0xffffffffu, (p[k] >> 8) & 0x00FF00FFu);
        if (lane == 0) {
            wc[4 * k + 0] += ev & 0xFFFFu;
            wc[4 * k + 1] += od & 0xFFFFu;
            wc[4 * k + 2] += ev >> 16;
            wc[4 * k + 3] += od >> 16;
        }
        p[k] = 0;
    }
}

__global__ void __launch_bounds__(kMetricThreads, 3) metrics_kernel(MetricArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ unsigned wc[kWarps][kCounts];
    __shared__ double ss[kWarps][kSums];
    for (int k = lane; k < kCounts; k += 32) wc[warp][k] = 0;
    __syncwarp();
    unsigned p[kPacked] = {};
    double sum[kSums] = {};
    const int n = a.w * a.h;
    const bool has_range = a.rmin && a.rmax, has_ref = a.before && a.after, has_left = a.left != nullptr;
    const int gwarp = blockIdx.x * kWarps + warp, nwarps = gridDim.x * kWarps;
    int steps = 0;
    for (int base = gwarp * 32; base < n; base += nwarps * 32) {
        const int i = base + lane;
        const bool inb = i < n;
        const int y = inb ? i / a.w : 0, x = inb ? i - y * a.w : 0;
        // every load of the pixel first (none waits for another), then the predicates
        const bool hx1 = x + 1 < a.w, hx0 = x > 0, hy1 = y + 1 < a.h, hy0 = y > 0;
        const float g = inb ? __ldg(a.gt + i) : -1.0f;
        const float g1 = inb && hx1 ? __ldg(a.gt + i + 1) : -1.0f;
        const float g2 = inb && hx0 ? __ldg(a.gt + i - 1) : -1.0f;
        const float g3 = inb && hy1 ? __ldg(a.gt + i + a.w) : -1.0f;
        const float g4 = inb && hy0 ? __ldg(a.gt + i - a.w) : -1.0f;
        float e = inb ? __ldg(a.est + i) : -1.0f;
        const uint8_t vm = inb && a.vis ? __ldg(a.vis + i) : 0;
        int16_t r0 = 0, r1 = 0;
        if (inb && has_range) { r0 = __ldg(a.rmin + i); r1 = __ldg(a.rmax + i); }
        float eb = -1.0f, ea = -1.0f;
        if (inb && has_ref) { eb = __ldg(a.before + i); ea = __ldg(a.after + i); }
        float lx1 = 0.f, lx0 = 0.f, ly1 = 0.f, ly0 = 0.f;
        if (inb && has_left) {
            const int xp = max(0, x - 1), xn = min(a.w - 1, x + 1), yp = max(0, y - 1), yn = min(a.h - 1, y + 1);
            lx1 = luma(a, xn, y); lx0 = luma(a, xp, y); ly1 = luma(a, x, yn); ly0 = luma(a, x, yp);
        }
        const bool ev = inb && gt_ok(g, a.max_gt);
        if (!ev) e = -1.0f;
        // disparity boundary: largest |g - neighbour| over the valid 4-neighbours (+x, -x, +y, -y)
        float md = 0.0f;
        {
            const float ng[4] = {g1, g2, g3, g4};
            const bool has[4] = {hx1, hx0, hy1, hy0};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (has[k] && gt_ok(ng[k], a.max_gt)) {
                    const float d = fabsf(__fsub_rn(g, ng[k]));
                    md = (md < d) ? d : md;
                }
            }
        }
        const bool edge = ev && md >= a.boundary;
        const int xr = x - (int)roundf(ev ? g : 0.0f);
        const bool matchable = ev && xr >= 0 && xr < a.w;
        const bool visible = ev && (a.vis ? vm >= 200 : matchable);
        bool low = false;
        if (ev && has_left) {
            // (next - prev) / scale with scale 1 or 2: a multiplication by 1 or 0.5 is the same
            // correctly rounded quotient
            const float sx = (x == 0 || x == a.w - 1) ? 1.0f : 0.5f, sy = (y == 0 || y == a.h - 1) ? 1.0f : 0.5f;
            const float dx = __fmul_rn(__fsub_rn(lx1, lx0), sx);
            const float dy = __fmul_rn(__fsub_rn(ly1, ly0), sy);
            low = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))) < a.lowtex;
        }
        const bool ok = ev && isfinite(e) && e >= 0.0f;
        const float adiff = fabsf(__fsub_rn(e, g));
        const bool d1 = ev && (!ok || (adiff > 3.0f && (g > 1e-3f ? (__fdiv_rn(adiff, g) > 0.05f) : true)));
        // a region's 7 counts for this pixel: in, valid, > 0.5, > 1, > 2, > 3, D1
        const unsigned lo = pack4(ev, ok, ok && adiff > 0.5f, ok && adiff > 1.0f);
        const unsigned hi = pack4(ok && adiff > 2.0f, ok && adiff > 3.0f, d1, false);
        p[0] += lo;
        p[1] += hi;
        p[2] += visible ? lo : 0u;
        p[3] += visible ? hi : 0u;
        p[4] += edge ? lo : 0u;
        p[5] += edge ? hi : 0u;
        p[6] += low ? lo : 0u;
        p[7] += low ? hi : 0u;
        if (ok) {
            sum[0] += adiff;
            sum[visible ? 1 : 2] += adiff;
            sum[edge ? 3 : 4] += adiff;
            if (has_left) sum[low ? 5 : 6] += adiff;
        }
        const bool in = has_range && ev && g >= (float)r0 && g < (float)r1;
        p[8] += pack4(ev && in, ev && matchable, ev && matchable && in, ev && visible && in);
        bool rv = false, improved = false, worsened = false, changed = false;
        if (has_ref && ev) {
            rv = isfinite(eb) && eb >= 0.0f && isfinite(ea) && ea >= 0.0f;
            if (rv) {
                const float db = fabsf(__fsub_rn(eb, g)), da = fabsf(__fsub_rn(ea, g));
                improved = da < __fsub_rn(db, 1e-4f);
                worsened = !improved && da > __fadd_rn(db, 1e-4f);
                changed = fabsf(__fsub_rn(ea, eb)) > 1e-4f;
                sum[7] += db;
                sum[8] += da;
                if (ok) {
                    sum[9] += db;
                    sum[10] += da;
                    sum[11] += adiff;
                }
            }
        }
        p[9] += pack4(rv, improved, worsened, changed);
        p[10] += pack4(ev && visible && !in && edge && has_range, rv && ok, false, false);
        if (++steps == 255) {  // byte counters hold at most 255 steps
            flush(p, wc[warp], lane);
            steps = 0;
        }
    }
    flush(p, wc[warp], lane);
#pragma unroll
    for (int k = 0; k < kSums; ++k) {
        double v = sum[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) ss[warp][k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kCounts; k += blockDim.x) {
        unsigned t = 0;
        for (int wp = 0; wp < kWarps; ++wp) t += wc[wp][k];
        a.part_c[blockIdx.x * kCounts + k] = t;
    }
    for (int k = threadIdx.x; k < kSums; k += blockDim.x) {
        double t = 0.0;
        for (int wp = 0; wp < kWarps; ++wp) t += ss[wp][k];
        a.part_s[blockIdx.x * kSums + k] = t;
    }
}

// One warp per value: lanes take the blocks in a fixed stride, then a fixed shuffle tree.
__global__ void __launch_bounds__(256) metrics_final_kernel(const unsigned* part_c, const double* part_s,
                                                            long long* out_c, double* out_s) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = warp; k < kCounts + kSums; k += nw) {
        if (k < kCounts) {
            unsigned long long t = 0;
            for (int b = lane; b < kMetricBlocks; b += 32) t += part_c[b * kCounts + k];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) out_c[k] = (long long)t;
        } else {
            double t = 0.0;
            for (int b = lane; b < kMetricBlocks; b += 32) t += part_s[b * kSums + (k - kCounts)];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) out_s[k - kCounts] = t;
        }
    }
}

}  // namespace

// The reference's tallies (include/apg_sgm/metrics.h order) from the independent ones.
void metrics_expand(const long long* in, const double* ins, bool has_range, bool has_ref, bool has_left,
                    long long* c, double* s) {
    for (int k = 0; k < APG_MC_COUNT; ++k) c[k] = 0;
    for (int k = 0; k < APG_MS_COUNT; ++k) s[k] = 0.0;
    const long long* all = in + 0;  // bytes 0-6 of registers 0-1: in, valid, >0.5, >1, >2, >3, d1
    const long long* vis = in + 8;
    const long long* bnd = in + 16;
    const long long* low = in + 24;
    long long* reg = c + APG_MC_REGION0;
    for (int f = 0; f < 7; ++f) {
        reg[0 * 7 + f] = all[f];
        reg[1 * 7 + f] = vis[f];
        reg[2 * 7 + f] = all[f] - vis[f];
        reg[3 * 7 + f] = bnd[f];
        reg[4 * 7 + f] = all[f] - bnd[f];
        if (has_left) {
            reg[5 * 7 + f] = low[f];
            reg[6 * 7 + f] = all[f] - low[f];
        }
    }
    c[APG_MC_EVALUATED] = all[0];
    c[APG_MC_VALID] = all[1];
    c[APG_MC_C05] = all[2];
    c[APG_MC_C10] = all[3];
    c[APG_MC_C20] = all[4];
    c[APG_MC_C30] = all[5];
    c[APG_MC_D1_ALL] = all[6];
    c[APG_MC_EVAL_NOC] = vis[0];
    c[APG_MC_D1_NOC] = vis[6];
    c[APG_MC_LR_FAIL] = all[0] - all[1];
    c[APG_MC_EDGE] = bnd[1];
    c[APG_MC_NONEDGE] = all[1] - bnd[1];
    if (has_range) {
        c[APG_MC_EVAL_ALL] = all[0];
        c[APG_MC_IN_ALL] = in[32];
        c[APG_MC_EVAL_MATCH] = in[33];
        c[APG_MC_IN_MATCH] = in[34];
        c[APG_MC_EVAL_VIS] = vis[0];
        c[APG_MC_IN_VIS] = in[35];
        c[APG_MC_MISS_VIS] = vis[0] - in[35];
        c[APG_MC_MISS_EDGE] = in[40];
        c[APG_MC_MISS_NONEDGE] = vis[0] - in[35] - in[40];
    }
    if (has_ref) {
        c[APG_MC_REF_EVAL] = in[36];
        c[APG_MC_REF_IMPROVED] = in[37];
        c[APG_MC_REF_WORSENED] = in[38];
        c[APG_MC_REF_UNCHANGED] = in[36] - in[37] - in[38];
        c[APG_MC_REF_CHANGED] = in[39];
        c[APG_MC_TOTAL_EVAL] = in[41];
    }
    for (int r = 0; r < 7; ++r) s[APG_MS_REGION0 + r] = ins[r];
    s[APG_MS_EPE] = ins[0];
    s[APG_MS_EDGE] = ins[3];
    s[APG_MS_NONEDGE] = ins[4];
    s[APG_MS_BEFORE] = ins[7];
    s[APG_MS_AFTER] = ins[8];
    s[APG_MS_TOT_BEFORE] = ins[9];
    s[APG_MS_TOT_AFTER] = ins[10];
    s[APG_MS_TOT_FINAL] = ins[11];
}

// Scratch bytes of one evaluation: block partials and the final tallies.
size_t metrics_scratch_bytes() {
    return (size_t)kMetricBlocks * (kCounts * 4 + kSums * 8) + kCounts * 8 + kSums * 8 + 512;
}

int metrics_independent_counts() { return kCounts; }
int metrics_independent_sums() { return kSums; }

// Enqueues the two kernels; the independent tallies land in `scratch` (device,
// metrics_scratch_bytes()) at the offsets returned through out_c / out_s.
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
    o += (size_t)kMetricBlocks * kSums * 8;
    double* fs = reinterpret_cast<double*>(scratch + o);
    o += kSums * 8;
    long long* fc = reinterpret_cast<long long*>(scratch + o);
    o += kCounts * 8;
    a.part_c = reinterpret_cast<unsigned*>(scratch + o);
    metrics_kernel<<<kMetricBlocks, kMetricThreads, 0, s>>>(a);
    metrics_final_kernel<<<1, 256, 0, s>>>(a.part_c, a.part_s, fc, fs);
    *out_c = fc;
    *out_s = fs;
    return cudaGetLastError();
}

// ---- evaluate_supports (src/metrics.cpp:8-124) -------------------------------------------------

namespace {

__device__ __forceinline__ bool support_visible(const float* gt, const uint8_t* vis, int w, int i, int x, float g) {
    const int xr = x - (int)roundf(g);
    return vis ? vis[i] >= 200 : (xr >= 0 && xr < w);
}

// Cells holding a visible ground-truth pixel.
__global__ void support_cells_kernel(const float* __restrict__ gt, const uint8_t* __restrict__ vis, int w, int h,
                                     float max_gt, int cell, int gw, uint8_t* __restrict__ vis_cell) {
    const int n = w * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = gt[i];
        if (!gt_ok(g, max_gt)) continue;
        const int y = i / w, x = i - y * w;
        if (support_visible(gt, vis, w, i, x, g)) vis_cell[(y / cell) * gw + x / cell] = 1;
    }
}

// One block: the supports' tallies (thread-strided, then a fixed tree), cells with a correct
// visible support, then the cell counts.  out_c: 10 counts, out_s: 2 sums.
__global__ void __launch_bounds__(256) support_eval_kernel(const int* __restrict__ sx, const int* __restrict__ sy,
                                                           const float* __restrict__ sd, int ns,
                                                           const float* __restrict__ gt,
                                                           const uint8_t* __restrict__ vis, int w, int h,
                                                           float max_gt, int cell, int gw, int n_cells,
                                                           const uint8_t* __restrict__ vis_cell,
                                                           uint8_t* __restrict__ ok_cell, long long* out_c,
                                                           double* out_s) {
    unsigned c[8] = {};
    double s0 = 0.0, s1 = 0.0;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        const int x = sx[k], y = sy[k];
        if (x < 0 || x >= w || y < 0 || y >= h) continue;
        const int i = y * w + x;
        const float g = gt[i];
        if (!gt_ok(g, max_gt)) continue;
        const bool v = support_visible(gt, vis, w, i, x, g);
        const float err = fabsf(__fsub_rn(sd[k], g));
        c[0] += 1;
        c[1] += v;
        s0 += err;
        if (v) s1 += err;
        c[2] += err <= 0.5f;
        c[3] += err <= 1.0f;
        c[4] += err <= 2.0f;
        c[5] += v && err <= 0.5f;
        c[6] += v && err <= 1.0f;
        c[7] += v && err <= 2.0f;
        if (v && err <= 1.0f) {
            const int gx = x / cell, gy = y / cell;
            ok_cell[gy * gw + gx] = 1;
        }
    }
    __shared__ unsigned sc[8][8];
    __shared__ double ss[2][8];
    __shared__ unsigned cells[2][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const unsigned t = __reduce_add_sync(0xffffffffu, c[k]);
        if (lane == 0) sc[k][warp] = t;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
    }
    if (lane == 0) { ss[0][warp] = s0; ss[1][warp] = s1; }
    __syncthreads();  // every ok_cell store is done
    unsigned nv = 0, nok = 0;
    for (int ci = threadIdx.x; ci < n_cells; ci += blockDim.x) {
        nv += vis_cell[ci];
        nok += vis_cell[ci] && ok_cell[ci];
    }
    nv = __reduce_add_sync(0xffffffffu, nv);
    nok = __reduce_add_sync(0xffffffffu, nok);
    if (lane == 0) { cells[0][warp] = nv; cells[1][warp] = nok; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) {
            long long t = 0;
            for (int wp = 0; wp < 8; ++wp) t += sc[k][wp];
            out_c[k] = t;
        }
        long long a = 0, b = 0;
        double d0 = 0.0, d1 = 0.0;
        for (int wp = 0; wp < 8; ++wp) { a += cells[0][wp]; b += cells[1][wp]; d0 += ss[0][wp]; d1 += ss[1][wp]; }
        out_c[8] = a;
        out_c[9] = b;
        out_s[0] = d0;
        out_s[1] = d1;
    }
}

}  // namespace

void count_launches(unsigned n);

}  // namespace apgcu

// ------------------------------------------------------------------------------------------------
// C entry (include/apg_sgm_cuda.h)
// ------------------------------------------------------------------------------------------------
#include "../../include/apg_sgm_cuda.h"

namespace {
thread_local float g_metrics_ms = 0.0f;  // device time of this thread's last evaluation's kernels

// The evaluation scratch (and the device copies of host inputs) comes from a stream-ordered pool
// the library owns, one per device, that keeps its memory between calls (release threshold at the
// maximum): the default pool would hand it back at every synchronisation and each call would map
// its ~50 MB again.  The pool holds its high-water mark for the life of the process.
cudaError_t metrics_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
    *out = p;
    return cudaSuccess;
}
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
    cudaMemPool_t pool = nullptr;
    cudaError_t e = metrics_pool(&pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&blk), in_bytes + scratch, pool, s);
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
    long long ci[64];
    double si[16];
    const int nci = apgcu::metrics_independent_counts(), nsi = apgcu::metrics_independent_sums();
    if (timed && e == cudaSuccess) cudaEventRecord(ev[1], s);
    if (e == cudaSuccess) {
        apgcu::count_launches(2);
        e = cudaMemcpyAsync(ci, dc, nci * sizeof(long long), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(si, ds, nsi * sizeof(double), cudaMemcpyDeviceToHost, s);
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
    long long c[APG_MC_COUNT];
    double sm[APG_MS_COUNT];
    apgcu::metrics_expand(ci, si, has_range, has_ref, left != nullptr, c, sm);
    apg_metrics_finalize(c, sm, w * h, has_range, has_ref, out);
    return APG_STATUS_OK;
}

extern "C" APGCU_API int apgcu_evaluate_supports(const int* sx, const int* sy, const float* sd, int n_supports,
                                                 const float* gt, int w, int h, const uint8_t* vis, float max_valid_gt,
                                                 int cell_size, int device_buffers, void* stream,
                                                 apg_support_metrics_t* out) {
    if (!out) return APG_STATUS_INTERNAL_ERROR;
    std::memset(out, 0, sizeof(*out));
    out->total = n_supports;
    if (n_supports <= 0 || w <= 0 || h <= 0) return APG_STATUS_OK;  // no supports or no ground truth
    if (!sx || !sy || !sd || !gt) return APG_STATUS_EMPTY_INPUT;
    if (cell_size <= 0) return APG_STATUS_INVALID_CONFIG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)w * h;
    const int gw = (w + cell_size - 1) / cell_size, gh = (h + cell_size - 1) / cell_size, n_cells = gw * gh;
    auto a256 = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t in_bytes = device_buffers ? 0 : 3 * a256((size_t)n_supports * 4) + a256(n * 4) + (vis ? a256(n) : 0);
    const size_t scratch = 2 * a256((size_t)n_cells) + 256;
    unsigned char* blk = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = metrics_pool(&pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&blk), in_bytes + scratch, pool, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return APG_STATUS_ALLOCATION_FAILURE;
    }
    const int *dx = sx, *dy = sy;
    const float *dd = sd, *dg = gt;
    const uint8_t* dv = vis;
    size_t o = 0;
    auto up = [&](const void* src, size_t bytes) -> void* {
        void* d = blk + o;
        o += a256(bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, s);
        return d;
    };
    if (!device_buffers) {
        dx = static_cast<const int*>(up(sx, (size_t)n_supports * 4));
        dy = static_cast<const int*>(up(sy, (size_t)n_supports * 4));
        dd = static_cast<const float*>(up(sd, (size_t)n_supports * 4));
        dg = static_cast<const float*>(up(gt, n * 4));
        if (vis) dv = static_cast<const uint8_t*>(up(vis, n));
    }
    unsigned char* sc = blk + in_bytes;
    uint8_t* vis_cell = sc;
    uint8_t* ok_cell = sc + a256((size_t)n_cells);
    long long* dc = reinterpret_cast<long long*>(sc + 2 * a256((size_t)n_cells));
    double* ds = reinterpret_cast<double*>(dc + 10);
    if (e == cudaSuccess) e = cudaMemsetAsync(sc, 0, 2 * a256((size_t)n_cells), s);
    if (e == cudaSuccess) {
        const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 4);
        apgcu::support_cells_kernel<<<blocks, 256, 0, s>>>(dg, dv, w, h, max_valid_gt, cell_size, gw, vis_cell);
        apgcu::support_eval_kernel<<<1, 256, 0, s>>>(dx, dy, dd, n_supports, dg, dv, w, h, max_valid_gt, cell_size, gw,
                                                     n_cells, vis_cell, ok_cell, dc, ds);
        e = cudaGetLastError();
        if (e == cudaSuccess) apgcu::count_launches(2);
    }
    long long c[10];
    double sm[2];
    if (e == cudaSuccess) e = cudaMemcpyAsync(c, dc, sizeof(c), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sm, ds, sizeof(sm), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(blk, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return APG_STATUS_INTERNAL_ERROR;
    }
    apg_support_finalize(n_supports, c, sm, out);
    return APG_STATUS_OK;
}


// Shared device-side definitions of the apg-sgm B200 engine.
//
// Layouts in HBM (one stereo pair):
//   * 2-D planes: row-major W*H (gray/gx/gy u8, census u32 or u64, range i16, maps f32/u8).
//   * volumes: u16, pixel-major with the disparity axis innermost and padded to Dp, a multiple
//     of 64:  vol[(y*W + x)*Dp + (d - d0)].  This is the reference Dense layout
//     (include/apg_sgm/buffers.hpp:45-55) with a padded stride, so one pixel's costs are one
//     128-byte-aligned run that a warp reads with one vector load per lane.  Padding entries
//     hold the invalid marker 0xFFFF and behave as out-of-range disparities everywhere.
#pragma once

#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

#include "apg_sgm/telemetry.h"

namespace apgcu {

constexpr uint16_t kInvalidCost = 0xFFFFu;   // types.hpp:44 kInvalidCost
constexpr uint32_t kInvalidWord = 0xFFFFFFFFu;
constexpr int kLutCensus = 0;                 // offsets into the float LUT block
constexpr int kLutAd = 65;
constexpr int kLutGrad = 65 + 256;
constexpr int kLutSize = 65 + 256 + 511;      // src/discrete_cost_lut.hpp:10-38

enum InvalidReason : uint8_t { kValid = 0, kOcclusion = 1, kMismatch = 2, kLowConfidence = 3 };

__host__ __device__ inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Everything a kernel needs to evaluate one matching cost.
struct CostCtx {
    int w, h, d0, D, Dp;
    int census64;      // 1: plain 9x7 census (u64), 0: symmetric 9x7 (u32)
    int use_ad, use_grad, cost_max;
    float scale;       // cost_max / (1 + eta + mu), src/cost_computer.cpp:154-155
    const float* lut;  // kLutSize floats built on the host with std::exp
    const uint16_t* qlut;  // 65 quantised census-only costs (same float ops, done on the host)
    const uint8_t *lgray, *lgx, *lgy, *rgray, *rgx, *rgy;
    const uint32_t *cl, *cr;
    const unsigned long long *cl64, *cr64;
    const int16_t *rmin, *rmax;
    int prior_ranges;  // 0: every pixel has the default range [d0, min(dmax, x+1)); 1: rmin/rmax vary
    int sp_method = 0;     // sub-pixel method of the right-image WTA (subpixel_delta), 0 = Legacy
    float sp_param = 0.0f;
    int tile;          // cost kernel tile width (64, 128, 256; 0 = default for Dp)
    int kernel;        // cost kernel: 0 = pixel runs where they apply, 1 = column tiles always
    int vol8 = 0;      // raw volume at one byte per voxel, 0xFF invalid (Fast census-only, pixel runs)
};

// Unquantised (float) cost, used by the refiner's local cost (src/refiner.cpp:14-36).
template <bool C64>
__device__ __forceinline__ float raw_cost(const CostCtx& c, const float* lut, int x, int y, int xr) {
    const int row = y * c.w;
    int pop;
    if (C64) pop = __popcll(c.cl64[row + x] ^ c.cr64[row + xr]);
    else pop = __popc(c.cl[row + x] ^ c.cr[row + xr]);
    float v = lut[kLutCensus + pop];
    if (c.use_ad) v = __fadd_rn(v, lut[kLutAd + abs((int)c.lgray[row + x] - (int)c.rgray[row + xr])]);
    if (c.use_grad) {
        const int g = abs((int)c.lgx[row + x] - (int)c.rgx[row + xr]) +
                      abs((int)c.lgy[row + x] - (int)c.rgy[row + xr]);
        v = __fadd_rn(v, lut[kLutGrad + g]);
    }
    return v;
}

// Legacy parabolic sub-pixel offset, SubpixelEstimator::compute_legacy_delta
// (src/subpixel_estimator.hpp:115-124).  Inputs are integer-valued floats.
__device__ __forceinline__ float legacy_delta(float cm, float c0, float cp) {
    const float denom = __fadd_rn(__fsub_rn(cm, __fmul_rn(2.0f, c0)), cp);
    if (fabsf(denom) > 1e-6f) {
        const float delta = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(cm, cp)), denom);
        if (delta < -0.5f) return -0.5f;
        if (delta > 0.5f) return 0.5f;
        return delta;
    }
    return 0.0f;
}

// SubpixelEstimator::compute_delta without telemetry (src/subpixel_estimator.cpp:58-119), the
// method an ExperimentalSubpixelScope selects: 0 Legacy, 1 CurvGate (denominator >= param, 4 by
// default, on a convex triple), 2 ConfGate (uniqueness >= param, 0.05 by default, on a convex
// triple), 3 Stabilized (denominator + param, 4 by default, when the centre is a minimum).
// Inputs are integer-valued floats; uniq is the WTA's (second - best) / max(best, 1), 1 elsewhere.
__device__ __forceinline__ float subpixel_delta(float cm, float c0, float cp, int method, float param, float uniq) {
    if (method == 0) return legacy_delta(cm, c0, cp);
    const float denom = __fadd_rn(__fsub_rn(cm, __fmul_rn(2.0f, c0)), cp);
    const bool non_convex = c0 >= cm || c0 >= cp || denom <= 1e-6f;
    float den = denom;
    bool apply;
    if (method == 1) {
        apply = !non_convex && denom >= (param > 0.0f ? param : 4.0f);
    } else if (method == 2) {
        apply = !non_convex && uniq >= (param > 0.0f ? param : 0.05f);
    } else {
        apply = c0 <= cm && c0 <= cp && denom > 0.0f;
        den = __fadd_rn(denom, param > 0.0f ? param : 4.0f);
    }
    if (!apply) return 0.0f;
    const float raw = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(cm, cp)), den);
    return raw < -0.5f ? -0.5f : (0.5f < raw ? 0.5f : raw);
}

// compute_delta with telemetry (src/subpixel_estimator.cpp:58-134): the same delta, and the
// reference's counters (candidates, non-convex and degenerate triples, applied offsets with their
// |delta| histogram and sum, clamped raw offsets) added with 64-bit atomics.
__device__ __forceinline__ float subpixel_delta_tel(float cm, float c0, float cp, int method, float param, float uniq,
                                                    apg_subpixel_telemetry_t* t) {
    atomicAdd(&t->candidate_pixels, 1ull);
    const float denom = __fadd_rn(__fsub_rn(cm, __fmul_rn(2.0f, c0)), cp);
    const bool non_convex = c0 >= cm || c0 >= cp || denom <= 1e-6f;
    if (non_convex) {
        atomicAdd(&t->negative_curvature_count, 1ull);
        if (fabsf(denom) <= 1e-6f || (cm == c0 && c0 == cp)) atomicAdd(&t->degenerate_count, 1ull);
    }
    float den = denom;
    bool apply;
    if (method == 0) {
        apply = fabsf(denom) > 1e-6f;
    } else if (method == 1) {
        apply = !non_convex && denom >= (param > 0.0f ? param : 4.0f);
    } else if (method == 2) {
        apply = !non_convex && uniq >= (param > 0.0f ? param : 0.05f);
    } else {
        apply = c0 <= cm && c0 <= cp && denom > 0.0f;
        den = __fadd_rn(denom, param > 0.0f ? param : 4.0f);
    }
    float raw = 0.0f, delta = 0.0f;
    if (apply) {
        raw = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(cm, cp)), den);
        delta = raw < -0.5f ? -0.5f : (0.5f < raw ? 0.5f : raw);
    }
    if (fabsf(delta) > 1e-5f) {
        const float a = fabsf(delta);
        atomicAdd(&t->applied_pixels, 1ull);
        atomicAdd(&t->sum_abs_delta, (double)a);
        atomicAdd(&t->delta_buckets[min(49, (int)__fmul_rn(a, 100.0f))], 1ull);
    }
    if (fabsf(raw) >= 0.5f) atomicAdd(&t->clamped_count, 1ull);
    return delta;
}

// Exact q = n / d for n < 2^16 and 1 <= d < 2^16 with one high multiply:
// m = floor(2^32 / d) + 1 gives n*m/2^32 = n/d + e with 0 < e < 2^-16 <= 1/d, so the floor is
// exact (tests/test_host_logic.py checks every n, d used by the cross aggregation).
__host__ __device__ inline uint32_t div_magic(uint32_t d) {
    return d <= 1 ? 0u : (uint32_t)((0x100000000ull / d) + 1ull);
}
__device__ __forceinline__ uint32_t div_by_magic(uint32_t n, uint32_t d, uint32_t m) {
    return d == 1 ? n : __umulhi(n, m);
}

// adaptive P2, detail::adaptive_p2 (src/sgm_common.hpp:25-39).
struct SgmPen {
    int P1, P2_base, adaptive, piecewise, t1, t2;
    float alpha;
};
__device__ __forceinline__ int adaptive_p2(const SgmPen& p, int dI) {
    dI = abs(dI);
    int P2 = p.P2_base;
    const int floor_p2 = p.P1 + 1;
    if (!p.adaptive) return P2 > floor_p2 ? P2 : floor_p2;
    if (p.piecewise) {
        if (dI >= p.t2) P2 = p.P2_base / 4;
        else if (dI >= p.t1) P2 = p.P2_base / 2;
    } else {
        P2 = __float2int_rz(__fadd_rn(
            __fdiv_rn((float)p.P2_base, __fadd_rn(1.f, __fmul_rn(p.alpha, (float)dI))), 0.5f));
    }
    return P2 > floor_p2 ? P2 : floor_p2;
}

// Lets `kern` launch with as much dynamic shared memory as the device allows it (the opt-in
// maximum less the function's static shared memory), and refuses a larger request.  The attribute
// is per function and shared by every host thread, so it is always set to that same per-function
// maximum, never to one launch's size: a thread launching with more shared memory than another
// thread's last setting would otherwise be refused.  It is set once per (function, device) -- also
// for requests under 48 KB, whose sum with the static size may still exceed the default limit --
// and remembered.  Occupancy follows each launch's actual size.
template <typename F>
inline cudaError_t allow_dynamic_smem(F kern, size_t smem) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> limits;
    const std::pair<const void*, int> key(reinterpret_cast<const void*>(kern), dev);
    int limit = -1;
    {
        std::lock_guard<std::mutex> lk(mu);
        const auto it = limits.find(key);
        if (it != limits.end()) limit = it->second;
    }
    if (limit < 0) {
        int optin = 0;
        cudaFuncAttributes fa;
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
        if (e == cudaSuccess) {
            limit = optin - (int)fa.sharedSizeBytes;
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
        }
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lk(mu);
        limits[key] = limit;
    }
    return (long long)smem > limit ? cudaErrorInvalidValue : cudaSuccess;
}

#define APGCU_CHECK(expr)                                                    \
    do {                                                                     \
        cudaError_t _e = (expr);                                             \
        if (_e != cudaSuccess) return _e;                                    \
    } while (0)

}  // namespace apgcu

// HighQuality selective refinement, detail::refine_scalar (src/refiner.cpp:42-100).
//
// The reference walks the image in raster order (forward on even passes, backward on odd) and
// updates unreliable pixels in place, so a pixel sees the already-updated values of its causal
// neighbours (left/up forward, right/down backward).  On the GPU one pass is an anti-diagonal
// wavefront: 32x32 tiles are launched one tile-diagonal at a time, and inside a tile one warp
// sweeps the 63 pixel anti-diagonals (lane = tile column).  This preserves exactly the
// reference's read-after-write order.
//
// Random draws: the pixel that consumes a draw is unreliable, has a non-empty range and holds a
// non-negative value at the start of the pass (a pass reads a pixel before writing it), so the
// draw index of every pixel is an exclusive prefix count of those pixels in the pass's raster
// order, computed before the pass.  The draws themselves are produced on the host by
// std::mt19937 / std::uniform_int_distribution, the reference's own generator.
#include <cub/device/device_scan.cuh>

#include "engine.h"

namespace apgcu {

namespace {

constexpr int kTile = 32;

__global__ void refine_flags_kernel(int w, int h, const uint8_t* __restrict__ reliable, const int16_t* __restrict__ rmin,
                                    const int16_t* __restrict__ rmax, const float* __restrict__ work, int fwd,
                                    int* __restrict__ flags) {
    const int n = w * h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        if (i == n) { flags[n] = 0; continue; }
        const int f = (!reliable[i] && rmax[i] > rmin[i] && work[i] >= 0.f) ? 1 : 0;
        flags[fwd ? i : n - 1 - i] = f;
    }
}

__global__ void copy_total_kernel(const int* prefix, int n, int* out) { *out = prefix[n]; }

template <bool C64>
__global__ void __launch_bounds__(32) refine_tile_kernel(CostCtx c, int fwd, int diag, int ntv,
                                                         const uint8_t* __restrict__ reliable,
                                                         const int* __restrict__ prefix,
                                                         const int* __restrict__ draws, float* work) {
    __shared__ float s_lut[kLutSize];
    for (int i = threadIdx.x; i < kLutSize; i += 32) s_lut[i] = c.lut[i];
    __syncwarp();
    const int tu_min = max(0, diag - (ntv - 1));
    const int tu = tu_min + blockIdx.x, tv = diag - tu;
    const int w = c.w, h = c.h, n = w * h;
    const int lu = threadIdx.x;
    const int u = tu * kTile + lu;
    for (int s = 0; s < 2 * kTile - 1; ++s) {
        const int lv = s - lu;
        const int v = tv * kTile + lv;
        if (lv >= 0 && lv < kTile && u < w && v < h) {
            const int x = fwd ? u : w - 1 - u;
            const int y = fwd ? v : h - 1 - v;
            const int i = y * w + x;
            const int lo = c.rmin[i], hi = c.rmax[i];
            if (!reliable[i] && hi > lo) {
                const float cur = work[i];
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
                if (cur >= 0.f) vals[nv++] = __fadd_rn(cur, (float)draws[prefix[fwd ? i : n - 1 - i]]);
                float best_c = 1e9f;
                int best_d = cur >= 0.f ? min(max((int)roundf(cur), lo), hi - 1) : lo;
                for (int j = 0; j < nv; ++j) {
                    if (vals[j] < 0.f) continue;
                    const int d = min(max((int)roundf(vals[j]), lo), hi - 1);
                    const int xr = x - d;
                    float cc = 1e6f;
                    if (xr >= 0 && xr < w && d >= lo && d < hi) cc = raw_cost<C64>(c, s_lut, x, y, xr);
                    if (cc < best_c) { best_c = cc; best_d = d; }
                }
                work[i] = (float)best_d;
            }
        }
        __syncwarp();
    }
}

}  // namespace

size_t refine_scan_temp_bytes(int n) {
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int*)nullptr, (int*)nullptr, n + 1);
    return bytes;
}

cudaError_t launch_refine_count(const Layout& L, unsigned char* arena, const float* work, int fwd, int* d_count,
                                cudaStream_t s, unsigned* launches) {
    const int n = L.w * L.h;
    int* flags = reinterpret_cast<int*>(arena + L.rf_prefix);
    const int blocks = min((n + 256) / 256, 148 * 8);
    refine_flags_kernel<<<blocks, 256, 0, s>>>(L.w, L.h, reinterpret_cast<const uint8_t*>(arena + L.reliable),
                                                reinterpret_cast<const int16_t*>(arena + L.rmin),
                                                reinterpret_cast<const int16_t*>(arena + L.rmax), work, fwd, flags);
    size_t tmp = L.rf_scan_tmp_bytes;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(arena + L.rf_scan_tmp, tmp, flags, flags, n + 1, s);
    if (e != cudaSuccess) return e;
    copy_total_kernel<<<1, 1, 0, s>>>(flags, n, d_count);
    *launches += 3;
    return cudaGetLastError();
}

cudaError_t launch_refine_pass(const apg_pipeline_config_t& cfg, const CostCtx& c, const Layout& L,
                               unsigned char* arena, float* work, int fwd, cudaStream_t s, unsigned* launches) {
    (void)cfg;
    const int ntu = (L.w + kTile - 1) / kTile, ntv = (L.h + kTile - 1) / kTile;
    const uint8_t* rel = reinterpret_cast<const uint8_t*>(arena + L.reliable);
    const int* prefix = reinterpret_cast<const int*>(arena + L.rf_prefix);
    const int* draws = reinterpret_cast<const int*>(arena + L.rf_draws);
    for (int dg = 0; dg < ntu + ntv - 1; ++dg) {
        const int tu_min = max(0, dg - (ntv - 1)), tu_max = min(ntu - 1, dg);
        const int nb = tu_max - tu_min + 1;
        if (c.census64) refine_tile_kernel<true><<<nb, 32, 0, s>>>(c, fwd, dg, ntv, rel, prefix, draws, work);
        else refine_tile_kernel<false><<<nb, 32, 0, s>>>(c, fwd, dg, ntv, rel, prefix, draws, work);
        ++*launches;
    }
    return cudaGetLastError();
}

}  // namespace apgcu

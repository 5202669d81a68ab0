// Right-image winner-take-all over a caller's cost volume, with no device allocation.
//
// This is the allocation-free variant of the engine's right-image WTA (cost.cu: the argmin that
// the cost kernel folds into per-pixel atomicMin keys, then right_wta_finalize_kernel).  The
// engine keeps those keys in its arena; this entry point keeps them in a file-scope __device__
// array of fixed size instead, so a call makes no cudaMalloc / cudaFree and no allocating
// library call.  It serves callers that must not allocate device memory on their hot path: a
// host that runs under its own fixed device-memory budget (an allocator it accounts itself, a
// memory pool it has already carved), or one whose allocator would synchronise the device,
// where an engine arena of W*H*Dp*2 bytes per frame is not available.
//
// Semantics follow wta_right_from_left_volume (src/pipeline.cpp:24-84): for each right pixel
// xr the lowest-cost valid C(xr + d, y, d) over d in [d0, d0 + D), ties to the smaller d, the
// invalid marker 0xFFFF skipped; best_d < 0 reads as "none" (-1); the legacy parabola when
// subpixel is on and the three neighbours along the diagonal are inside the image and valid.
//
// The scratch is one array per device, shared by every call on that device: two calls that
// overlap in time on one device (different streams or host threads) race on it.  The array is part
// of this library's device code: with CUDA's default lazy module loading it is created in a
// context by the first call there (together with the kernels), so callers make one warm-up call at
// start-up; with eager loading every context that loads the library holds it from the start.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "apg_sgm_cuda.h"
#include "common.cuh"
#include "engine.h"

namespace apgcu {
namespace {

// 2^21 pixels: 8 MiB of u32 keys; 1920 x 1080 (2,073,600 pixels) fits.
constexpr int kMaxPixels = APGCU_NOALLOC_MAX_PIXELS;
static __device__ __align__(256) uint32_t g_rwta_keys[kMaxPixels];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_keys_ptr[kMaxDevices] = {};
void* g_keys_ctx[kMaxDevices] = {};  // the context the cached address belongs to

// cuCtxGetCurrent from the driver, found through the runtime (no link-time libcuda dependency)
using CtxGetCurrent = int (*)(void**);
CtxGetCurrent ctx_get_current() {
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    return fn;
}

// The keys start at all-ones ("no candidate"); every call clears the pixels it will use.
__global__ void noalloc_clear_kernel(uint32_t* __restrict__ keys, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) keys[p] = kInvalidWord;
}

// One block per (tile of TX left columns, row).  The tile's slices C(xl, y, .) are staged in
// shared memory with a row pitch of SP u16 (D rounded up to even, plus 2), then every right
// pixel xr whose diagonal xl = xr + d0 + di crosses the tile takes the minimum key (c << 16 | di)
// along its part of the diagonal and folds it into keys[y*W + xr] with atomicMin.  Consecutive
// xr read consecutive u16 at each step, so the reads are free of bank conflicts.
__global__ void noalloc_argmin_kernel(const uint16_t* __restrict__ vol, int w, int D, int pitch, int d0, int tx,
                                      int sp, uint32_t* __restrict__ keys) {
    extern __shared__ uint16_t s_tile[];
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * tx;
    const int ncols = min(tx, w - x0);
    // element i = j * D + di of the tile; each thread steps by blockDim.x = dq * D + dr elements
    const int dq = blockDim.x / D, dr = blockDim.x - dq * D;
    int j = threadIdx.x / D, di = threadIdx.x - j * D;
    for (; j < ncols; j += dq, di += dr) {
        if (di >= D) {
            di -= D;
            ++j;
            if (j >= ncols) break;
        }
        s_tile[j * sp + di] = vol[((size_t)y * w + x0 + j) * pitch + di];
    }
    __syncthreads();
    // xr = xl - d0 - di with xl in [x0, x0 + ncols), di in [0, D)
    const int xr_lo = max(0, x0 - d0 - D + 1);
    const int xr_hi = min(w - 1, x0 + ncols - 1 - d0);
    for (int xr = xr_lo + threadIdx.x; xr <= xr_hi; xr += blockDim.x) {
        uint32_t best = kInvalidWord;
        // j = xl - x0 ranges where di = j + x0 - d0 - xr is inside [0, D)
        const int c = x0 - d0 - xr;
        const int j_lo = max(0, -c);
        const int j_hi = min(ncols - 1, D - 1 - c);
        for (int j = j_lo; j <= j_hi; ++j) {
            const int di = j + c;
            const uint32_t v = s_tile[j * sp + di];
            if (v != kInvalidCost) best = min(best, (v << 16) | (uint32_t)di);
        }
        if (best != kInvalidWord) atomicMin(&keys[(size_t)y * w + xr], best);
    }
}

__global__ void noalloc_finalize_kernel(const uint16_t* __restrict__ vol, const uint32_t* __restrict__ keys, int w,
                                        int h, int D, int pitch, int d0, int subpixel, float* __restrict__ disp) {
    const int n = w * h;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t key = keys[p];
        float dv = -1.f;
        if (key != kInvalidWord && d0 + (int)(key & 0xFFFFu) >= 0) {
            const int di = (int)(key & 0xFFFFu);
            const int bd = d0 + di;
            dv = (float)bd;
            const int y = p / w, xr = p - y * w;
            const int xm = xr + bd - 1, x0 = xr + bd, xp = xr + bd + 1;
            if (subpixel && xm >= 0 && xm < w && x0 >= 0 && x0 < w && xp >= 0 && xp < w && di > 0 && di + 1 < D) {
                const size_t row = (size_t)y * w;
                const uint16_t cm = vol[(row + xm) * pitch + di - 1];
                const uint16_t c0 = vol[(row + x0) * pitch + di];
                const uint16_t cp = vol[(row + xp) * pitch + di + 1];
                if (cm != kInvalidCost && c0 != kInvalidCost && cp != kInvalidCost)
                    dv = __fadd_rn(dv, legacy_delta((float)cm, (float)c0, (float)cp));
            }
        }
        disp[p] = dv;
    }
}

// Device address of this device's key array: looked up once per device, with that device
// current, on the first call there (which also loads the module under lazy loading).  The address
// is remembered with the context it was found in and looked up again when the device's current
// context is another one (the primary context was reset and created anew).
int keys_for_device(uint32_t** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return APG_STATUS_UNSUPPORTED_BACKEND;
    }
    if (dev < 0 || dev >= kMaxDevices) return APG_STATUS_UNSUPPORTED_BACKEND;
    const CtxGetCurrent current = ctx_get_current();
    auto context = [&]() -> void* {
        void* c = nullptr;
        if (current && current(&c) != 0) c = nullptr;
        return c;
    };
    std::lock_guard<std::mutex> lock(g_mu);
    const void* ctx = context();  // null before the runtime has made a context current on this thread
    if (!g_keys_ptr[dev] || !ctx || g_keys_ctx[dev] != ctx) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_rwta_keys) != cudaSuccess || !p) {
            cudaGetLastError();
            g_keys_ptr[dev] = nullptr;
            return APG_STATUS_INTERNAL_ERROR;
        }
        g_keys_ptr[dev] = static_cast<uint32_t*>(p);
        g_keys_ctx[dev] = context();  // the lookup made the device's primary context current
    }
    *out = g_keys_ptr[dev];
    return APG_STATUS_OK;
}

}  // namespace
}  // namespace apgcu

extern "C" APGCU_API int apgcu_right_wta_noalloc(const uint16_t* d_cost, int width, int height, int min_disparity,
                                                 int num_disparities, int pitch, int subpixel, float* d_disparity_right,
                                                 void* stream) {
    using namespace apgcu;
    if (!d_cost || !d_disparity_right) return APG_STATUS_EMPTY_INPUT;
    if (width <= 0 || height <= 0) return APG_STATUS_EMPTY_INPUT;
    if (num_disparities <= 0 || num_disparities > APGCU_NOALLOC_MAX_DISPARITIES)
        return APG_STATUS_INVALID_DISPARITY_RANGE;
    // disparities, x + d and x - d stay far inside int for every accepted size
    if (min_disparity < -APGCU_NOALLOC_MAX_ABS_DISPARITY || min_disparity > APGCU_NOALLOC_MAX_ABS_DISPARITY)
        return APG_STATUS_INVALID_DISPARITY_RANGE;
    if (pitch < num_disparities) return APG_STATUS_SIZE_MISMATCH;
    if ((long long)width * height > kMaxPixels || height > 65535) return APG_STATUS_RESOURCE_LIMIT_EXCEEDED;
    uint32_t* keys = nullptr;
    int rc = keys_for_device(&keys);
    if (rc != APG_STATUS_OK) return rc;
    // an error left on this thread by earlier work must not be read as this call's
    cudaGetLastError();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = width * height;
    const int D = num_disparities;
    const int sp = ((D + 1) & ~1) + 2;
    // widest tile whose staged slices fit in 40 KB of shared memory (no opt-in attribute needed)
    int tx = 64;
    while (tx > 8 && (size_t)tx * sp * 2 > 40 * 1024) tx /= 2;
    const size_t smem = (size_t)tx * sp * 2;
    const int blocks = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
    noalloc_clear_kernel<<<blocks, 256, 0, s>>>(keys, n);
    if (cudaGetLastError() != cudaSuccess) return APG_STATUS_INTERNAL_ERROR;
    count_launches(1);
    noalloc_argmin_kernel<<<dim3((width + tx - 1) / tx, height), 256, smem, s>>>(d_cost, width, D, pitch,
                                                                                min_disparity, tx, sp, keys);
    if (cudaGetLastError() != cudaSuccess) return APG_STATUS_INTERNAL_ERROR;
    count_launches(1);
    noalloc_finalize_kernel<<<blocks, 256, 0, s>>>(d_cost, keys, width, height, D, pitch, min_disparity,
                                                   subpixel ? 1 : 0, d_disparity_right);
    if (cudaGetLastError() != cudaSuccess) return APG_STATUS_INTERNAL_ERROR;
    count_launches(1);
    return APG_STATUS_OK;
}

// Gray conversion, gradients and census of one image, fused in one pass.
//
// Restates CostComputer::compute_aux (src/cost_computer.cpp:124-130): gray via
// ImageView8::gray (include/apg_sgm/image_view.hpp:50-56), gx/gy as clamped absolute central
// differences (src/cost_computer.cpp:63-88) and the 9x7 census (symmetric 31-bit,
// :33-47, or plain 62-bit, :49-61), all with clamp-to-edge sampling (src/image.cpp:15-19).
//
// One CTA produces a 32x32 output tile.  It converts the (32+8)x(32+6) haloed input window to gray
// once into shared memory (each gray value is needed by up to 63 census comparisons) and then
// derives gradients and census from shared memory.  Bound: HBM, about ch + 7 (or 11) bytes per
// pixel; the census comparisons are cheap integer work on staged data.
#include "common.cuh"
#include "kernels.h"

namespace apgcu {

namespace {
// A CTA of TX x BY threads produces a TX x TY tile, each thread TY / BY rows of a column, so a
// CTA's staging latency is paid once for TY rows.
constexpr int TX = 32, TY = 32, BY = 8, HX = 4, HY = 3;
constexpr int SX = TX + 2 * HX, SY = TY + 2 * HY;

// blockIdx.z selects the image: both images of a pair go through one launch.
template <bool C64>
__global__ void __launch_bounds__(TX * BY) aux_kernel(AuxImage im0, AuxImage im1, int ch, int w, int h) {
    const AuxImage& im = blockIdx.z ? im1 : im0;
    const uint8_t* __restrict__ src = im.src;
    const int stride = im.stride;
    uint8_t* __restrict__ gray = im.gray;
    uint8_t* __restrict__ gx = im.gx;
    uint8_t* __restrict__ gy = im.gy;
    uint32_t* __restrict__ census = im.census;
    unsigned long long* __restrict__ census64 = im.census64;
    __shared__ __align__(16) uint8_t g[SY][SX];  // rows of SX bytes, a multiple of 4
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    for (int i = tid; i < SX * SY; i += TX * BY) {
        const int sy = i / SX, sx = i % SX;
        const int yy = min(max(y0 + sy - HY, 0), h - 1);
        const int xx = min(max(x0 + sx - HX, 0), w - 1);
        const uint8_t* row = src + (size_t)yy * stride;
        uint8_t v;
        if (ch == 1) {
            v = row[xx];
        } else {
            const int r = row[xx * ch], gg = row[xx * ch + 1], b = row[xx * ch + 2];
            v = (uint8_t)((77 * r + 150 * gg + 29 * b) >> 8);
        }
        g[sy][sx] = v;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x;
    if (x >= w) return;
    for (int j = 0; j < TY / BY; ++j) {
        const int ty = threadIdx.y + BY * j, y = y0 + ty;
        if (y >= h) break;
        const int cx = threadIdx.x + HX, cy = ty + HY;
        // Clamp-to-edge neighbours: outside the image the staged window already repeats the border
        // value, so x+-1 / y+-1 read the clamped sample directly.
        const int gxv = (int)g[cy][cx + 1] - (int)g[cy][cx - 1];
        const int gyv = (int)g[cy + 1][cx] - (int)g[cy - 1][cx];
        const size_t o = (size_t)y * w + x;
        gray[o] = g[cy][cx];
        gx[o] = (uint8_t)min(abs(gxv), 255);
        gy[o] = (uint8_t)min(abs(gyv), 255);
        if (C64) {
            const uint8_t center = g[cy][cx];
            unsigned long long bits = 0;
            int b = 0;
#pragma unroll
            for (int dy = -3; dy <= 3; ++dy)
#pragma unroll
                for (int dx = -4; dx <= 4; ++dx) {
                    if (dx == 0 && dy == 0) continue;
                    if (g[cy + dy][cx + dx] > center) bits |= (1ull << b);
                    ++b;
                }
            census64[o] = bits;
        } else {
            // The window's seven rows as nine bytes each (columns cx - 4 .. cx + 4): three aligned
            // 32-bit loads per row and funnel shifts, so a pixel costs 21 shared-memory loads instead
            // of 62.  Bit b of the symmetric census compares byte dx + 4 of row dy + 3 with byte
            // 4 - dx of the mirrored row 3 - dy (dy < 0, then dy == 0 with dx < 0), for four
            // consecutive bits at once: the mirrored row's bytes reversed by a permute, one
            // four-byte compare, and the four result bytes gathered into a nibble by a multiply.
            uint32_t ra[7], rb[7], rc[7];  // bytes 0-3, 4-7 and 8 of each window row
            const int sh = 8 * (threadIdx.x & 3);
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                const uint32_t* row = reinterpret_cast<const uint32_t*>(&g[cy - 3 + k][0]) + (threadIdx.x >> 2);
                const uint32_t w0 = row[0], w1 = row[1], w2 = row[2];
                ra[k] = __funnelshift_r(w0, w1, sh);
                rb[k] = __funnelshift_r(w1, w2, sh);
                rc[k] = (w2 >> sh) & 0xFFu;
            }
            auto nibble = [](uint32_t r) { return ((r & 0x01010101u) * 0x01020408u) >> 24; };
            uint32_t bits = 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {  // dy = k - 3: bits 9k .. 9k + 8
                const int m = 6 - k;       // the mirrored row
                const uint32_t rev0 = __byte_perm(rb[m], rc[m], 0x1234);  // bytes 8, 7, 6, 5
                const uint32_t rev1 = __byte_perm(ra[m], rb[m], 0x1234);  // bytes 4, 3, 2, 1
                bits |= nibble(__vcmpgtu4(ra[k], rev0)) << (9 * k);
                bits |= nibble(__vcmpgtu4(rb[k], rev1)) << (9 * k + 4);
                bits |= (rc[k] > (ra[m] & 0xFFu) ? 1u : 0u) << (9 * k + 8);  // byte 8 against byte 0
            }
            // dy = 0, dx = -4 .. -1: bytes 0-3 of the centre row against its bytes 8, 7, 6, 5
            bits |= nibble(__vcmpgtu4(ra[3], __byte_perm(rb[3], rc[3], 0x1234))) << 27;
            census[o] = bits;
        }
    }
}
}  // namespace

cudaError_t launch_aux(const AuxImage& left, const AuxImage& right, int ch, int w, int h, int census64,
                       cudaStream_t s) {
    dim3 grid((w + TX - 1) / TX, (h + TY - 1) / TY, 2), block(TX, BY);
    if (census64) aux_kernel<true><<<grid, block, 0, s>>>(left, right, ch, w, h);
    else aux_kernel<false><<<grid, block, 0, s>>>(left, right, ch, w, h);
    return cudaGetLastError();
}

cudaError_t launch_aux_one(const AuxImage& im, int ch, int w, int h, int census64, cudaStream_t s) {
    dim3 grid((w + TX - 1) / TX, (h + TY - 1) / TY, 1), block(TX, BY);
    if (census64) aux_kernel<true><<<grid, block, 0, s>>>(im, im, ch, w, h);
    else aux_kernel<false><<<grid, block, 0, s>>>(im, im, ch, w, h);
    return cudaGetLastError();
}

}  // namespace apgcu

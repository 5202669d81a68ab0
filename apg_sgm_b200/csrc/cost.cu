// Matching-cost volume, fused with the horizontal Cross-arm pass and the right-image WTA.
//
// Restates, in one kernel over (row y, 64- or 32-pixel column tile):
//   * CostComputer::compute_volume (src/cost_computer.cpp:139-203; LUT form :205-268):
//     census Hamming + AD + gradient terms from host-built LUTs, quantised to u16;
//   * the horizontal half of CostAggregator::aggregate_hv (src/cost_aggregator.cpp:65-105):
//     T(x,d) = floor(sum of valid C over [x-L(x), x+R(x)] / count), arms from
//     build_cross_arms (:17-63) computed on the fly from the staged gray row;
//   * the argmin half of wta_right_from_left_volume (src/pipeline.cpp:24-85): per right pixel
//     xr the first minimum over d of the RAW cost C(xr+d, d), reduced inside the CTA and then
//     merged across CTAs with one 32-bit atomicMin per right pixel (key = cost<<16 | d-d0, so
//     the minimum key is the lowest cost and, among equal costs, the lowest d).
//
// The raw volume therefore never goes to HBM: the kernel reads only the 2-D aux planes and
// writes the horizontally aggregated volume T (2 bytes per voxel).  With aggregation off
// (Fast mode) it either writes the raw volume or, in the fused Fast path, writes nothing and
// only produces the right-image argmin.
//
// Prefix sums over x run in 16-bit lanes (two disparities per 32-bit word, __vadd2, wrapping);
// a window difference is exact because a window sum is at most (2*Lmax+1)*cost_max < 2^16,
// which the host checks before choosing this kernel.
#include "common.cuh"
#include "kernels.h"

namespace apgcu {

namespace {

struct CostSmem {
    int nx;        // TXc + 2*HA staged left pixels
    int nr;        // staged right pixels
    size_t bytes;
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

template <bool C64>
__host__ __device__ inline void cost_smem_layout(int txc, int ha, int D, int Dp, bool cross,
                                                 size_t* off_lut, size_t* off_left, size_t* off_right,
                                                 size_t* off_cost, size_t* off_pre, size_t* total) {
    const int nx = txc + 2 * ha;
    const int nr = nx + D - 1;
    const size_t csz = C64 ? 8 : 4;
    size_t o = 0;
    *off_lut = o; o = align16(o + kLutSize * 4);
    *off_left = o; o = align16(o + (size_t)nx * (csz + 3 + 4));   // census, gray, gx, gy, rmin, rmax
    *off_right = o; o = align16(o + (size_t)nr * (csz + 3));      // census, gray, gx, gy
    *off_cost = o; o = align16(o + (size_t)nx * (Dp + 2) * 2);  // row stride Dp+2: conflict-free diagonals
    *off_pre = o;
    if (cross) o = align16(o + (size_t)(nx + 1) * (Dp / 2) * 8);
    *total = o;
}

template <bool C64, bool CROSS, bool STORE, bool RWTA>
__global__ void __launch_bounds__(256) cost_kernel(CostCtx c, int txc, int ha, int lmax, int tau,
                                                   uint32_t* __restrict__ out_vol,
                                                   uint32_t* __restrict__ rkey,
                                                   const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    size_t o_lut, o_left, o_right, o_cost, o_pre, total;
    cost_smem_layout<C64>(txc, ha, c.D, c.Dp, CROSS, &o_lut, &o_left, &o_right, &o_cost, &o_pre, &total);
    const int nx = txc + 2 * ha;
    const int nr = nx + c.D - 1;
    const int W2 = c.Dp / 2;  // 32-bit words per pixel
    const int CS = W2 + 1;    // staged cost row stride in words (odd: diagonal reads hit distinct banks)
    float* s_lut = reinterpret_cast<float*>(smem + o_lut);
    const size_t csz = C64 ? 8 : 4;
    unsigned char* L = smem + o_left;
    unsigned char* Rg = smem + o_right;
    uint32_t* s_cost = reinterpret_cast<uint32_t*>(smem + o_cost);

    const int y = blockIdx.y;
    const int x0 = blockIdx.x * txc;
    const int xbase = x0 - ha;                  // staged left pixel 0
    const int rbase = xbase - (c.d0 + c.D - 1); // staged right pixel 0
    const int row = y * c.w;
    const int tid = threadIdx.x, nt = blockDim.x;

    __shared__ uint16_t s_q[65];
    for (int i = tid; i < kLutSize; i += nt) s_lut[i] = c.lut[i];
    for (int i = tid; i < 65; i += nt) s_q[i] = c.qlut[i];
    // left aux (census, gray, gx, gy, rmin, rmax) for x in [xbase, xbase+nx)
    for (int i = tid; i < nx; i += nt) {
        const int x = xbase + i;
        const bool in = x >= 0 && x < c.w;
        if (C64) reinterpret_cast<unsigned long long*>(L)[i] = in ? c.cl64[row + x] : 0ull;
        else reinterpret_cast<uint32_t*>(L)[i] = in ? c.cl[row + x] : 0u;
        L[nx * csz + i] = in ? c.lgray[row + x] : 0;
        L[nx * (csz + 1) + i] = in ? c.lgx[row + x] : 0;
        L[nx * (csz + 2) + i] = in ? c.lgy[row + x] : 0;
        int16_t* rm = reinterpret_cast<int16_t*>(L + nx * (csz + 3));
        rm[i] = in ? c.rmin[row + x] : (int16_t)0;
        rm[nx + i] = in ? c.rmax[row + x] : (int16_t)0;  // empty range outside the image
    }
    for (int i = tid; i < nr; i += nt) {
        const int xr = rbase + i;
        const bool in = xr >= 0 && xr < c.w;
        if (C64) reinterpret_cast<unsigned long long*>(Rg)[i] = in ? c.cr64[row + xr] : 0ull;
        else reinterpret_cast<uint32_t*>(Rg)[i] = in ? c.cr[row + xr] : 0u;
        Rg[nr * csz + i] = in ? c.rgray[row + xr] : 0;
        Rg[nr * (csz + 1) + i] = in ? c.rgx[row + xr] : 0;
        Rg[nr * (csz + 2) + i] = in ? c.rgy[row + xr] : 0;
    }
    __syncthreads();

    const int16_t* s_rmin = reinterpret_cast<const int16_t*>(L + nx * (csz + 3));
    const int16_t* s_rmax = s_rmin + nx;
    // raw costs for every staged left pixel and disparity pair
    for (int i = tid; i < nx * W2; i += nt) {
        const int xi = i / W2, k = i - xi * W2;
        const int x = xbase + xi;
        uint32_t word = kInvalidWord;
        if (x >= 0 && x < c.w) {
            const int lo = s_rmin[xi], hi = s_rmax[xi];
            uint32_t clv = 0;
            unsigned long long clv64 = 0;
            if (C64) clv64 = reinterpret_cast<const unsigned long long*>(L)[xi];
            else clv = reinterpret_cast<const uint32_t*>(L)[xi];
            const int gl = L[nx * csz + xi], gxl = L[nx * (csz + 1) + xi], gyl = L[nx * (csz + 2) + xi];
#pragma unroll
            for (int hsel = 0; hsel < 2; ++hsel) {
                const int di = 2 * k + hsel;
                const int d = c.d0 + di;
                const int xr = x - d;
                uint32_t q = kInvalidCost;
                if (di < c.D && d >= lo && d < hi && xr >= 0 && xr < c.w) {
                    const int ri = xr - rbase;
                    int pop;
                    if (C64) pop = __popcll(clv64 ^ reinterpret_cast<const unsigned long long*>(Rg)[ri]);
                    else pop = __popc(clv ^ reinterpret_cast<const uint32_t*>(Rg)[ri]);
                    if (!c.use_ad && !c.use_grad) {
                        // census-only cost: the host pre-quantised LUT (same float ops)
                        q = s_q[pop];
                        word = hsel == 0 ? ((word & 0xFFFF0000u) | q) : ((word & 0x0000FFFFu) | (q << 16));
                        continue;
                    }
                    float v = s_lut[kLutCensus + pop];
                    if (c.use_ad) v = __fadd_rn(v, s_lut[kLutAd + abs(gl - (int)Rg[nr * csz + ri])]);
                    if (c.use_grad) {
                        const int g = abs(gxl - (int)Rg[nr * (csz + 1) + ri]) + abs(gyl - (int)Rg[nr * (csz + 2) + ri]);
                        v = __fadd_rn(v, s_lut[kLutGrad + g]);
                    }
                    int qi = __float2int_rz(__fadd_rn(__fmul_rn(v, c.scale), 0.5f));
                    qi = qi < 0 ? 0 : (qi > c.cost_max ? c.cost_max : qi);
                    q = (uint32_t)qi;
                }
                word = hsel == 0 ? ((word & 0xFFFF0000u) | q) : ((word & 0x0000FFFFu) | (q << 16));
            }
        }
        s_cost[xi * CS + k] = word;
    }
    __syncthreads();

    const uint16_t* s_c16 = reinterpret_cast<const uint16_t*>(s_cost);
    if (RWTA) {
        // right pixels receiving a contribution from this tile's own (non-halo) columns
        const int xe = min(x0 + txc, c.w);
        const int r_lo = x0 - c.d0 - c.D + 1, r_hi = xe - c.d0;
        for (int xr = r_lo + tid; xr < r_hi; xr += nt) {
            if (xr < 0 || xr >= c.w) continue;
            int di_lo = x0 - xr - c.d0, di_hi = xe - xr - c.d0;
            di_lo = max(di_lo, 0);
            di_hi = min(di_hi, c.D);
            uint32_t best = kInvalidWord;
            for (int di = di_lo; di < di_hi; ++di) {
                const int xi = xr + c.d0 + di - xbase;
                const uint32_t v = s_c16[xi * (c.Dp + 2) + di];
                if (v != kInvalidCost) {
                    const uint32_t key = (v << 16) | (uint32_t)di;
                    best = key < best ? key : best;
                }
            }
            if (best != kInvalidWord) atomicMin(rkey + row + xr, best);
        }
    }

    if (!CROSS) {
        if (STORE) {
            for (int i = tid; i < txc * W2; i += nt) {
                const int xi = i / W2, k = i - xi * W2;
                const int x = x0 + xi;
                if (x < c.w) out_vol[((size_t)row + x) * W2 + k] = s_cost[(xi + ha) * CS + k];
            }
        }
        return;
    }

    // prefix over staged x of (sum, count) in 16-bit lanes
    uint32_t* s_psum = reinterpret_cast<uint32_t*>(smem + o_pre);
    uint32_t* s_pcnt = s_psum + (size_t)(nx + 1) * W2;
    for (int k = tid; k < W2; k += nt) {
        uint32_t ps = 0, pc = 0;
        s_psum[k] = 0;
        s_pcnt[k] = 0;
        for (int xi = 0; xi < nx; ++xi) {
            const uint32_t v = s_cost[xi * CS + k];
            const uint32_t inval = __vcmpeq2(v, kInvalidWord);  // 0xFFFF per invalid half
            ps = __vadd2(ps, v & ~inval);
            pc = __vadd2(pc, 0x00010001u & ~inval);
            s_psum[(xi + 1) * W2 + k] = ps;
            s_pcnt[(xi + 1) * W2 + k] = pc;
        }
    }
    __syncthreads();

    // query: one (tile pixel, word) per thread-iteration
    for (int i = tid; i < txc * W2; i += nt) {
        const int xi = i / W2, k = i - xi * W2;
        const int x = x0 + xi;
        if (x >= c.w) continue;
        const int sxi = xi + ha;
        // arms L and R of build_cross_arms from the staged gray row
        const int c0 = L[nx * csz + sxi];
        int l = 0, r = 0;
        while (l < lmax && x - l - 1 >= 0 && abs((int)L[nx * csz + sxi - l - 1] - c0) <= tau) ++l;
        while (r < lmax && x + r + 1 < c.w && abs((int)L[nx * csz + sxi + r + 1] - c0) <= tau) ++r;
        const int a = sxi - l, b = sxi + r + 1;
        const uint32_t s = __vsub2(s_psum[b * W2 + k], s_psum[a * W2 + k]);
        const uint32_t n = __vsub2(s_pcnt[b * W2 + k], s_pcnt[a * W2 + k]);
        const int lo = s_rmin[sxi], hi = s_rmax[sxi];
        uint32_t word = 0;
#pragma unroll
        for (int hsel = 0; hsel < 2; ++hsel) {
            const int di = 2 * k + hsel;
            const int d = c.d0 + di;
            const uint32_t sh = (s >> (16 * hsel)) & 0xFFFFu, nh = (n >> (16 * hsel)) & 0xFFFFu;
            uint32_t q = kInvalidCost;
            if (di < c.D && d >= lo && d < hi && nh > 0) q = div_by_magic(sh, nh, magic[nh]);
            word |= q << (16 * hsel);
        }
        out_vol[((size_t)row + x) * W2 + k] = word;
    }
}

template <bool C64, bool CROSS, bool STORE, bool RWTA>
cudaError_t launch_cost_t(const CostCtx& c, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    const int txc = c.Dp <= 128 ? 64 : 32;
    const int ha = CROSS ? lmax : 0;
    size_t a, b, d, e, f, total;
    cost_smem_layout<C64>(txc, ha, c.D, c.Dp, CROSS, &a, &b, &d, &e, &f, &total);
    auto kern = cost_kernel<C64, CROSS, STORE, RWTA>;
    if (total > 48 * 1024) {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)total);
        if (err != cudaSuccess) return err;
    }
    dim3 grid((c.w + txc - 1) / txc, c.h);
    kern<<<grid, 256, total, s>>>(c, txc, ha, lmax, tau, vol, rkey, magic);
    return cudaGetLastError();
}

}  // namespace

size_t cost_kernel_smem_bytes(int D, int Dp, int lmax, bool cross, bool census64) {
    const int txc = Dp <= 128 ? 64 : 32;
    size_t a, b, d, e, f, total;
    if (census64) cost_smem_layout<true>(txc, cross ? lmax : 0, D, Dp, cross, &a, &b, &d, &e, &f, &total);
    else cost_smem_layout<false>(txc, cross ? lmax : 0, D, Dp, cross, &a, &b, &d, &e, &f, &total);
    return total;
}

cudaError_t launch_cost(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                        const uint32_t* magic, cudaStream_t s) {
    // mode: 0 = raw volume + right argmin, 1 = cross-H volume + right argmin,
    //       2 = right argmin only (fused Fast path)
    if (c.census64) {
        if (mode == 0) return launch_cost_t<true, false, true, true>(c, lmax, tau, vol, rkey, magic, s);
        if (mode == 1) return launch_cost_t<true, true, true, true>(c, lmax, tau, vol, rkey, magic, s);
        return launch_cost_t<true, false, false, true>(c, lmax, tau, vol, rkey, magic, s);
    }
    if (mode == 0) return launch_cost_t<false, false, true, true>(c, lmax, tau, vol, rkey, magic, s);
    if (mode == 1) return launch_cost_t<false, true, true, true>(c, lmax, tau, vol, rkey, magic, s);
    return launch_cost_t<false, false, false, true>(c, lmax, tau, vol, rkey, magic, s);
}

// disparity_right from the per-right-pixel argmin keys: legacy sub-pixel on the raw costs of the
// diagonal neighbours C(xr+d-1, d-1), C(xr+d, d), C(xr+d+1, d+1) (src/pipeline.cpp:53-82),
// recomputed from the aux planes.
template <bool C64>
__global__ void right_wta_finalize_kernel(CostCtx c, const uint32_t* __restrict__ rkey, int subpixel,
                                          float* __restrict__ disp_right) {
    __shared__ float s_lut[kLutSize];
    for (int i = threadIdx.x; i < kLutSize; i += blockDim.x) s_lut[i] = c.lut[i];
    __syncthreads();
    const int n = c.w * c.h;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t key = rkey[p];
        float dv = -1.f;
        // best_d = -1 is the reference's "none" marker, tested as best_d >= 0: a negative
        // winning disparity is reported as -1 too (src/pipeline.cpp:40-53).
        if (key != kInvalidWord && c.d0 + (int)(key & 0xFFFFu) >= 0) {
            const int di = (int)(key & 0xFFFFu);
            const int bd = c.d0 + di;
            dv = (float)bd;
            const int y = p / c.w, xr = p - y * c.w;
            const int xm = xr + bd - 1, x0 = xr + bd, xp = xr + bd + 1;
            if (subpixel && xm >= 0 && xm < c.w && x0 >= 0 && x0 < c.w && xp >= 0 && xp < c.w && di > 0 &&
                di + 1 < c.D) {
                const int row = y * c.w;
                // C(xl, d) is valid iff d is inside range(xl) and xl - d is inside the image;
                // here xl - d == xr for all three, so only the range test remains.
                auto cost_at = [&](int xl, int d, uint32_t& out) -> bool {
                    if (d < c.rmin[row + xl] || d >= c.rmax[row + xl]) return false;
                    if (C64) out = quantised_cost<true>(c, s_lut, 0u, c.cl64[row + xl], c.lgray[row + xl],
                                                        c.lgx[row + xl], c.lgy[row + xl], row, xr);
                    else out = quantised_cost<false>(c, s_lut, c.cl[row + xl], 0ull, c.lgray[row + xl],
                                                     c.lgx[row + xl], c.lgy[row + xl], row, xr);
                    return true;
                };
                uint32_t cm, c0v, cp;
                if (cost_at(xm, bd - 1, cm) && cost_at(x0, bd, c0v) && cost_at(xp, bd + 1, cp))
                    dv = __fadd_rn(dv, legacy_delta((float)cm, (float)c0v, (float)cp));
            }
        }
        disp_right[p] = dv;
    }
}

cudaError_t launch_right_wta_finalize(const CostCtx& c, const uint32_t* rkey, int subpixel, float* disp_right,
                                      cudaStream_t s) {
    const int n = c.w * c.h;
    const int blocks = min((n + 255) / 256, 148 * 8);
    if (c.census64) right_wta_finalize_kernel<true><<<blocks, 256, 0, s>>>(c, rkey, subpixel, disp_right);
    else right_wta_finalize_kernel<false><<<blocks, 256, 0, s>>>(c, rkey, subpixel, disp_right);
    return cudaGetLastError();
}

}  // namespace apgcu

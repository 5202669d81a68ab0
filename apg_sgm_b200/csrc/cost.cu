// Matching-cost volume, fused with the horizontal Cross-arm pass and the right-image WTA.
//
// Restates, in one kernel over (row y, 128- or 64-pixel column tile):
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

// Staged per-pixel descriptor: census bits and the three 8-bit planes packed as
// gray | gx << 8 | gy << 16, so one __vabsdiffu4 yields |dgray|, |dgx|, |dgy|.
template <bool C64> struct Aux;
template <> struct __align__(8) Aux<false> { uint32_t c; uint32_t g; };
template <> struct __align__(16) Aux<true> { unsigned long long c; uint32_t g; uint32_t pad; };

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// Threads per block: a multiple of the words per pixel W2 (up to 256), so a thread keeps one word
// index k for the whole kernel and walks pixels with a fixed stride.
__host__ __device__ inline int cost_threads(int W2) { return W2 <= 256 ? W2 * (256 / W2) : 256; }

struct CostLayout {
    int txc, ha, nx, nr, segs;
    size_t lut, magic, arm, left, right, rng, cost, cnt, seg, total;
};

__host__ __device__ inline CostLayout cost_layout(int txc, int ha, int D, int Dp, bool cross, bool prior, bool c64) {
    CostLayout l;
    const int W2 = Dp / 2, CS = W2 + 1;
    const int nt = cost_threads(W2);
    l.txc = txc; l.ha = ha;
    l.nx = txc + 2 * ha;
    l.nr = l.nx + D - 1;
    l.segs = W2 <= nt ? nt / W2 : 1;
    const size_t asz = c64 ? 16 : 8;
    size_t o = 0;
    l.lut = o; o = align16(o + kLutSize * 4);
    l.magic = o; o = align16(o + (cross ? (2 * ha + 2) * 4 : 0));
    l.arm = o; o = align16(o + (cross ? txc * 4 : 0));
    l.left = o; o = align16(o + l.nx * asz);
    l.right = o; o = align16(o + l.nr * asz);
    l.rng = o; o = align16(o + (prior ? l.nx * 4 : 0));
    l.cost = o; o = align16(o + (size_t)l.nx * CS * 4);  // odd word stride: diagonals hit distinct banks
    l.cnt = o; o = align16(o + (cross && prior ? (size_t)l.nx * W2 * 4 : 0));
    l.seg = o; o = align16(o + (cross ? (size_t)l.segs * W2 * 4 * 2 : 0));
    l.total = o;
    return l;
}

// Visit every (staged pixel xi < nrows, word k) pair of the block once.
template <typename F>
__device__ __forceinline__ void for_each_word(int nrows, int W2, int nt, F&& body) {
    const int tid = threadIdx.x;
    if (W2 <= nt) {
        const int k = tid % W2, rstep = nt / W2;
        for (int xi = tid / W2; xi < nrows; xi += rstep) body(xi, k);
    } else {
        for (int xi = 0; xi < nrows; ++xi)
            for (int k = tid; k < W2; k += nt) body(xi, k);
    }
}

// One block per (row y, tile of txc columns); the tile's raw costs over [x0 - ha, x0 + txc + ha)
// are built in shared memory, then (RWTA) folded into the right-image argmin keys, then (CROSS)
// turned into in-place prefix sums over x and queried over each pixel's horizontal arm.
template <bool C64, bool CROSS, bool STORE, bool RWTA, bool PRIOR, bool QLUT>
__global__ void __launch_bounds__(256) cost_kernel(CostCtx c, int txc, int ha, int lmax, int tau,
                                                   uint32_t* __restrict__ out_vol,
                                                   uint32_t* __restrict__ rkey,
                                                   const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    const CostLayout ly = cost_layout(txc, ha, c.D, c.Dp, CROSS, PRIOR, C64);
    const int nx = ly.nx, nr = ly.nr;
    const int W2 = c.Dp / 2;
    const int CS = W2 + 1;
    const int nt = blockDim.x, tid = threadIdx.x;
    float* s_lut = reinterpret_cast<float*>(smem + ly.lut);
    uint32_t* s_magic = reinterpret_cast<uint32_t*>(smem + ly.magic);
    uint32_t* s_arm = reinterpret_cast<uint32_t*>(smem + ly.arm);
    Aux<C64>* s_left = reinterpret_cast<Aux<C64>*>(smem + ly.left);
    Aux<C64>* s_right = reinterpret_cast<Aux<C64>*>(smem + ly.right);
    uint32_t* s_rng = reinterpret_cast<uint32_t*>(smem + ly.rng);
    uint32_t* s_cost = reinterpret_cast<uint32_t*>(smem + ly.cost);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem + ly.cnt);
    uint32_t* s_seg = reinterpret_cast<uint32_t*>(smem + ly.seg);
    __shared__ uint16_t s_q[65];

    const int y = blockIdx.y;
    const int x0 = blockIdx.x * txc;
    const int xbase = x0 - ha;                   // staged left pixel 0
    const int rbase = xbase - (c.d0 + c.D - 1);  // staged right pixel 0
    const int row = y * c.w;

    if (QLUT) {
        for (int i = tid; i < 65; i += nt) s_q[i] = c.qlut[i];
    } else {
        for (int i = tid; i < kLutSize; i += nt) s_lut[i] = c.lut[i];
    }
    if (CROSS)
        for (int i = tid; i < 2 * ha + 2; i += nt) s_magic[i] = magic[i];
    for (int i = tid; i < nx; i += nt) {
        const int x = xbase + i;
        const bool in = x >= 0 && x < c.w;
        Aux<C64> a{};
        if (in) {
            if constexpr (C64) a.c = c.cl64[row + x];
            else a.c = c.cl[row + x];
            a.g = (uint32_t)c.lgray[row + x] | ((uint32_t)c.lgx[row + x] << 8) | ((uint32_t)c.lgy[row + x] << 16);
        }
        s_left[i] = a;
        if (PRIOR)  // empty range outside the image
            s_rng[i] = in ? ((uint32_t)(uint16_t)c.rmin[row + x] | ((uint32_t)(uint16_t)c.rmax[row + x] << 16)) : 0u;
    }
    for (int i = tid; i < nr; i += nt) {
        const int xr = rbase + i;
        Aux<C64> a{};
        if (xr >= 0 && xr < c.w) {
            if constexpr (C64) a.c = c.cr64[row + xr];
            else a.c = c.cr[row + xr];
            a.g = (uint32_t)c.rgray[row + xr] | ((uint32_t)c.rgx[row + xr] << 8) | ((uint32_t)c.rgy[row + xr] << 16);
        }
        s_right[i] = a;
    }
    __syncthreads();

    // ---- raw quantised costs C(x, d) of the staged pixels (CostComputer::compute_volume,
    // src/cost_computer.cpp:247-264), invalid = 0xFFFF
    for_each_word(nx, W2, nt, [&](int xi, int k) {
        const int x = xbase + xi;
        uint32_t word = kInvalidWord;
        if (x >= 0 && x < c.w) {
            const Aux<C64> la = s_left[xi];
            int lo = 0, hi = 0;
            if (PRIOR) {
                const uint32_t rg = s_rng[xi];
                lo = (int16_t)(rg & 0xFFFFu);
                hi = (int16_t)(rg >> 16);
            }
            word = 0;
            // both disparities of the word valid (the common case): no per-voxel range tests
            const int dw = c.d0 + 2 * k;
            const bool word_ok = !PRIOR && 2 * k + 1 < c.D && x - (dw + 1) >= 0 && x - dw < c.w;
#pragma unroll
            for (int hs = 0; hs < 2; ++hs) {
                const int di = 2 * k + hs;
                const int d = c.d0 + di;
                const int xr = x - d;
                uint32_t q = kInvalidCost;
                // default range [d0, min(dmax, x+1)) and x - d inside the image
                bool ok = word_ok || (di < c.D && xr >= 0 && xr < c.w);
                if (PRIOR) ok = ok && d >= lo && d < hi;
                if (ok) {
                    const Aux<C64> ra = s_right[xi - di + c.D - 1];
                    int pop;
                    if constexpr (C64) pop = __popcll(la.c ^ ra.c);
                    else pop = __popc(la.c ^ ra.c);
                    if (QLUT) {
                        q = s_q[pop];  // census-only: the host pre-quantised LUT (same float ops)
                    } else {
                        float v = s_lut[kLutCensus + pop];
                        const uint32_t ad = __vabsdiffu4(la.g, ra.g);
                        if (c.use_ad) v = __fadd_rn(v, s_lut[kLutAd + (ad & 0xFFu)]);
                        if (c.use_grad) v = __fadd_rn(v, s_lut[kLutGrad + ((ad >> 8) & 0xFFu) + (ad >> 16)]);
                        int qi = __float2int_rz(__fadd_rn(__fmul_rn(v, c.scale), 0.5f));
                        qi = qi < 0 ? 0 : (qi > c.cost_max ? c.cost_max : qi);
                        q = (uint32_t)qi;
                    }
                }
                word |= q << (16 * hs);
            }
        }
        s_cost[xi * CS + k] = word;
    });
    __syncthreads();

    if (RWTA) {
        // right pixels receiving a contribution from this tile's own (non-halo) columns: the
        // first minimum over d of C(xr + d, d) (src/pipeline.cpp:38-53) as key cost<<16 | d-d0
        const uint16_t* s_c16 = reinterpret_cast<const uint16_t*>(s_cost);
        const int xe = min(x0 + txc, c.w);
        const int r_lo = max(0, x0 - c.d0 - c.D + 1), r_hi = min(c.w, xe - c.d0);
        for (int xr = r_lo + tid; xr < r_hi; xr += nt) {
            const int di_lo = max(x0 - xr - c.d0, 0), di_hi = min(xe - xr - c.d0, c.D);
            uint32_t best = kInvalidWord;
            const int xi0 = xr + c.d0 - xbase;  // staged column of di = 0
            for (int di = di_lo; di < di_hi; ++di) {
                const uint32_t v = s_c16[(xi0 + di) * (2 * CS) + di];
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
            for_each_word(txc, W2, nt, [&](int xi, int k) {
                const int x = x0 + xi;
                if (x < c.w) out_vol[((size_t)row + x) * W2 + k] = s_cost[xi * CS + k];
            });
        }
        return;
    }

    // ---- horizontal half of CostAggregator::aggregate_hv (src/cost_aggregator.cpp:65-105)
    if (RWTA) __syncthreads();  // the argmin above still reads the raw costs
    // arms of the tile's pixels (build_cross_arms, src/cost_aggregator.cpp:17-63)
    for (int i = tid; i < txc; i += nt) {
        const int x = x0 + i;
        if (x >= c.w) continue;
        const int sxi = i + ha;
        const int c0 = (int)(s_left[sxi].g & 0xFFu);
        int l = 0, r = 0;
        while (l < lmax && x - l - 1 >= 0 && abs((int)(s_left[sxi - l - 1].g & 0xFFu) - c0) <= tau) ++l;
        while (r < lmax && x + r + 1 < c.w && abs((int)(s_left[sxi + r + 1].g & 0xFFu) - c0) <= tau) ++r;
        s_arm[i] = (uint32_t)l | ((uint32_t)r << 16);
    }
    // inclusive prefix over staged x of the valid costs (and, with per-pixel ranges, of the valid
    // counts), in 16-bit lanes: each word column is cut into `segs` segments scanned in parallel
    const int segs = ly.segs;
    const int seglen = (nx + segs - 1) / segs;
    uint32_t* s_segc = s_seg + segs * W2;
    for (int col = tid; col < W2 * segs; col += nt) {
        const int k = col % W2, sg = col / W2;
        const int a = sg * seglen, b = min(nx, a + seglen);
        uint32_t ps = 0, pc = 0;
        for (int xi = a; xi < b; ++xi) {
            const uint32_t v = s_cost[xi * CS + k];
            const uint32_t inval = __vcmpeq2(v, kInvalidWord);  // 0xFFFF per invalid half
            ps = __vadd2(ps, v & ~inval);
            s_cost[xi * CS + k] = ps;
            if (PRIOR) {
                pc = __vadd2(pc, 0x00010001u & ~inval);
                s_cnt[xi * W2 + k] = pc;
            }
        }
        s_seg[sg * W2 + k] = ps;
        if (PRIOR) s_segc[sg * W2 + k] = pc;
    }
    __syncthreads();
    if (segs > 1) {
        for (int col = tid; col < W2 * segs; col += nt) {
            const int k = col % W2, sg = col / W2;
            if (sg == 0) continue;
            uint32_t os = 0, oc = 0;
            for (int j = 0; j < sg; ++j) {
                os = __vadd2(os, s_seg[j * W2 + k]);
                if (PRIOR) oc = __vadd2(oc, s_segc[j * W2 + k]);
            }
            const int a = sg * seglen, b = min(nx, a + seglen);
            for (int xi = a; xi < b; ++xi) {
                s_cost[xi * CS + k] = __vadd2(s_cost[xi * CS + k], os);
                if (PRIOR) s_cnt[xi * W2 + k] = __vadd2(s_cnt[xi * W2 + k], oc);
            }
        }
        __syncthreads();
    }

    // T(x, d) = floor(window sum / window count) over [x - L(x), x + R(x)]; the window stays inside
    // the image.  A window difference is exact: the true sum is below 2^16.
    for_each_word(txc, W2, nt, [&](int xi, int k) {
        const int x = x0 + xi;
        if (x >= c.w) return;
        const int sxi = xi + ha;
        const uint32_t arm = s_arm[xi];
        const int l = (int)(arm & 0xFFFFu), r = (int)(arm >> 16);
        const int a = sxi - l, b = sxi + r;  // inclusive staged window
        const uint32_t s = __vsub2(s_cost[b * CS + k], a > 0 ? s_cost[(a - 1) * CS + k] : 0u);
        uint32_t n2 = 0;
        int lo = 0, hi = 0;
        if (PRIOR) {
            n2 = __vsub2(s_cnt[b * W2 + k], a > 0 ? s_cnt[(a - 1) * W2 + k] : 0u);
            const uint32_t rg = s_rng[sxi];
            lo = (int16_t)(rg & 0xFFFFu);
            hi = (int16_t)(rg >> 16);
        }
        uint32_t word = 0;
        const int dw = c.d0 + 2 * k;
        if (!PRIOR && 2 * k + 1 < c.D && x - l >= dw + 1 && x + r <= c.w - 1 + dw) {
            // both windows lie where the word's disparities are valid: the count is the window length
            const uint32_t len = (uint32_t)(l + r + 1), mg = s_magic[len];
            word = div_by_magic(s & 0xFFFFu, len, mg) | (div_by_magic(s >> 16, len, mg) << 16);
            out_vol[((size_t)row + x) * W2 + k] = word;
            return;
        }
#pragma unroll
        for (int hs = 0; hs < 2; ++hs) {
            const int di = 2 * k + hs;
            const int d = c.d0 + di;
            const uint32_t sh = (s >> (16 * hs)) & 0xFFFFu;
            int nh;
            bool ok;
            if (PRIOR) {
                nh = (int)((n2 >> (16 * hs)) & 0xFFFFu);
                ok = di < c.D && d >= lo && d < hi && nh > 0;
            } else {
                // valid x' in the window: d <= x' <= w - 1 + d
                nh = min(x + r, c.w - 1 + d) - max(x - l, d) + 1;
                ok = di < c.D && d <= x && nh > 0;
            }
            const uint32_t q = ok ? div_by_magic(sh, (uint32_t)nh, s_magic[nh]) : kInvalidCost;
            word |= q << (16 * hs);
        }
        out_vol[((size_t)row + x) * W2 + k] = word;
    });
}

template <bool C64, bool CROSS, bool STORE, bool RWTA, bool PRIOR, bool QLUT>
cudaError_t launch_cost_t(const CostCtx& c, int txc, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    const int ha = CROSS ? lmax : 0;
    const CostLayout ly = cost_layout(txc, ha, c.D, c.Dp, CROSS, PRIOR, C64);
    auto kern = cost_kernel<C64, CROSS, STORE, RWTA, PRIOR, QLUT>;
    {
        const cudaError_t err = allow_dynamic_smem(kern, ly.total);
        if (err != cudaSuccess) return err;
    }
    dim3 grid((c.w + txc - 1) / txc, c.h);
    kern<<<grid, cost_threads(c.Dp / 2), ly.total, s>>>(c, txc, ha, lmax, tau, vol, rkey, magic);
    return cudaGetLastError();
}

// Tile width: 128 columns where the staged costs fit comfortably (halo overhead 2*lmax/txc), else 64.
int cost_tile(int Dp) { return Dp <= 128 ? 128 : 64; }

// The requested tile width when its shared memory fits, else the default.
int cost_tile_for(const CostCtx& c, int ha, bool cross, bool prior) {
    const int req = c.tile;
    if (req == 64 || req == 128 || req == 256) {
        if (cost_layout(req, ha, c.D, c.Dp, cross, prior, c.census64 != 0).total <= 200 * 1024) return req;
    }
    return cost_tile(c.Dp);
}

template <bool C64, bool PRIOR>
cudaError_t launch_cost_m(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    const int txc = cost_tile_for(c, mode == 1 ? lmax : 0, mode == 1, PRIOR);
    const bool qlut = !c.use_ad && !c.use_grad;
    if (mode == 1) {
        return qlut ? launch_cost_t<C64, true, true, true, PRIOR, true>(c, txc, lmax, tau, vol, rkey, magic, s)
                    : launch_cost_t<C64, true, true, true, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
    }
    if (mode == 0) {
        return qlut ? launch_cost_t<C64, false, true, true, PRIOR, true>(c, txc, lmax, tau, vol, rkey, magic, s)
                    : launch_cost_t<C64, false, true, true, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
    }
    return qlut ? launch_cost_t<C64, false, false, true, PRIOR, true>(c, txc, lmax, tau, vol, rkey, magic, s)
                : launch_cost_t<C64, false, false, true, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
}

}  // namespace

size_t cost_kernel_smem_bytes(int D, int Dp, int lmax, bool cross, bool census64) {
    // the largest variant: per-pixel ranges (count prefix) included
    return cost_layout(cost_tile(Dp), cross ? lmax : 0, D, Dp, cross, true, census64).total;
}

cudaError_t launch_cost(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                        const uint32_t* magic, cudaStream_t s) {
    // mode: 0 = raw volume + right argmin, 1 = cross-H volume + right argmin,
    //       2 = right argmin only (fused Fast path)
    if (cost_runs_supported(c, mode, lmax)) return launch_cost_runs(c, mode, lmax, tau, vol, rkey, magic, s);
    if (c.vol8) return cudaErrorInvalidValue;  // the byte volume is written by the pixel-run kernel only
    if (c.census64) {
        return c.prior_ranges ? launch_cost_m<true, true>(c, mode, lmax, tau, vol, rkey, magic, s)
                              : launch_cost_m<true, false>(c, mode, lmax, tau, vol, rkey, magic, s);
    }
    return c.prior_ranges ? launch_cost_m<false, true>(c, mode, lmax, tau, vol, rkey, magic, s)
                          : launch_cost_m<false, false>(c, mode, lmax, tau, vol, rkey, magic, s);
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
            const int xm = xr + bd - 1, xp = xr + bd + 1;
            if (subpixel && xm >= 0 && xp < c.w && di > 0 && di + 1 < c.D) {
                const int row = y * c.w;
                // C(xl, d) is valid iff d is inside range(xl) and xl - d is inside the image; here
                // xl - d == xr for all three, so only the range test remains, and with the default
                // ranges it always holds (d >= d0, d < dmax, d <= xl).  The right pixel's
                // descriptors are the same for the three costs (src/cost_computer.cpp:247-264).
                const int rg = c.rgray[row + xr], rgx = c.rgx[row + xr], rgy = c.rgy[row + xr];
                uint32_t rc32 = 0;
                unsigned long long rc64 = 0;
                if (C64) rc64 = c.cr64[row + xr];
                else rc32 = c.cr[row + xr];
                auto cost_at = [&](int xl, int d, uint32_t& out) -> bool {
                    if (c.prior_ranges && (d < c.rmin[row + xl] || d >= c.rmax[row + xl])) return false;
                    const int pop = C64 ? __popcll(c.cl64[row + xl] ^ rc64) : __popc(c.cl[row + xl] ^ rc32);
                    float v = s_lut[kLutCensus + pop];
                    if (c.use_ad) v = __fadd_rn(v, s_lut[kLutAd + abs((int)c.lgray[row + xl] - rg)]);
                    if (c.use_grad)
                        v = __fadd_rn(v, s_lut[kLutGrad + abs((int)c.lgx[row + xl] - rgx) + abs((int)c.lgy[row + xl] - rgy)]);
                    int q = __float2int_rz(__fadd_rn(__fmul_rn(v, c.scale), 0.5f));
                    q = q < 0 ? 0 : (q > c.cost_max ? c.cost_max : q);
                    out = (uint32_t)q;
                    return true;
                };
                uint32_t cm, c0v, cp;
                if (cost_at(xm, bd - 1, cm) && cost_at(xm + 1, bd, c0v) && cost_at(xp, bd + 1, cp))
                    dv = __fadd_rn(dv, subpixel_delta((float)cm, (float)c0v, (float)cp, c.sp_method, c.sp_param, 1.0f));
            }
        }
        disp_right[p] = dv;
    }
}

cudaError_t launch_right_wta_finalize(const CostCtx& c, const uint32_t* rkey, int subpixel, float* disp_right,
                                      cudaStream_t s) {
    const int n = c.w * c.h;
    const int blocks = min((n + 255) / 256, 148 * 4);  // each block stages the LUT once
    if (c.census64) right_wta_finalize_kernel<true><<<blocks, 256, 0, s>>>(c, rkey, subpixel, disp_right);
    else right_wta_finalize_kernel<false><<<blocks, 256, 0, s>>>(c, rkey, subpixel, disp_right);
    return cudaGetLastError();
}

}  // namespace apgcu

// Matching-cost volume by pixel runs, fused with the horizontal Cross-arm pass and the
// right-image argmin: the form used for the 32-bit census (Fast, Balanced, and HighQuality with the
// prior's per-pixel ranges), up to 256 padded disparities.  Results are those of cost.cu's tile
// kernel, which keeps the 64-bit census and wider ranges; only the division of the work differs:
//
//   * One warp covers the whole disparity range of a run of consecutive staged pixels: lane l owns
//     the WPL = Dp/64 words k = WPL*l .. WPL*l + WPL-1 (the P = 2*WPL disparities P*l .. P*l+P-1)
//     and walks the run one pixel per step.  The right pixel of (x+1, di+1) is the right pixel of
//     (x, di), so each step loads one new right descriptor per lane into a P-entry register window;
//     the left descriptor is the same for the whole warp (broadcast loads of four pixels at a time).
//   * Quantised costs follow CostComputer::compute_volume (src/cost_computer.cpp:247-264): the
//     census and AD terms come from one table t2[ad][pop] = lut_census[pop] + lut_ad[ad] (the
//     reference's first float add, done once per entry), then + lut_grad[g], * scale, + 0.5,
//     truncation and clamp, each float op rounded on its own.  Census-only costs use the host's
//     pre-quantised table.
//   * The horizontal prefix over a run (CostAggregator::aggregate_hv's row pass,
//     src/cost_aggregator.cpp:65-105) is a plain 32-bit running sum of packed words: the
//     difference of two such sums is exact in each 16-bit half when each half's window sum is
//     below 2^16, which the host checks for the arm length and cost_max.  Runs are joined at query
//     time from the per-run totals.
//   * Per-pixel ranges: each staged left pixel carries [lo, hi); a lane turns it into a mask of its
//     P disparities per step, and the aggregation keeps a second running prefix of valid counts
//     (two 8-bit counts per word, exact for windows of at most 255 pixels).
//   * The right-image argmin (wta_right_from_left_volume, src/pipeline.cpp:24-85): right pixel
//     r = x - d0 - di receives (x, di) at step x in lane di/P.  Each lane keeps the running minimum
//     keys (cost << 16 | di: lowest cost first, then lowest d) of its P right pixels; every step
//     the oldest moves one lane up (a shuffle), and the one leaving lane 31 -- complete over this
//     run -- goes to a per-warp buffer that is merged into rkey with atomicMin at the end of the
//     run, together with the partial minima still held.  min is idempotent, so a halo pixel seen
//     by two tiles changes nothing.
//
// Blocks are persistent: each builds its tables once and then walks (row, column tile) items.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace apgcu {

namespace {

// t2[pop][|dgray|]: one row of 256 per popcount 0..32 of a 32-bit census, so a voxel's index is
// one byte permute of the popcount and the absolute differences
constexpr int kT2Rows = 33;

struct RunGeom {
    int txc, ha, nx, nr, roff, rl, nrun, ntx, ntiles;
    size_t t2, lgt, q, magic, arm, lc, lg, rc, rg, rng, pre, cnt, tot, totc, emit, total;
};

inline size_t a16(size_t v) { return (v + 15) & ~size_t(15); }

inline int run_warps(bool cross) { return cross ? 16 : 8; }

// Staging and table layout of one block for a tile of txc columns with halo ha.  nx (staged left
// pixels) and rl (run length) are multiples of 4 (16-byte loads of four left descriptors); roff
// shifts the staged right row so that each step group's right descriptors start at an even index
// (8-byte loads) and every lane with a disparity inside the range finds its whole window staged.
// One run per warp.
RunGeom run_geom(const CostCtx& c, int txc, int ha, bool cross, bool full, bool prior) {
    RunGeom g{};
    const int W2 = c.Dp / 2;
    g.txc = txc;
    g.ha = ha;
    g.nrun = run_warps(cross);
    g.nx = round_up(txc + 2 * ha, 4);
    g.rl = round_up((g.nx + g.nrun - 1) / g.nrun, 4);
    // even start for every step group, plus P entries so that a lane holding any disparity of the
    // range loads its own window without clamping
    g.roff = ((c.D - 1) % 2 == 0 ? 2 : 1) + c.Dp / 32;
    g.nr = round_up(g.nx + c.D - 1 + g.roff, 4);
    g.ntx = (c.w + txc - 1) / txc;
    g.ntiles = g.ntx * c.h;
    const bool stage_g = full || cross;
    size_t o = 0;
    g.t2 = o; o = a16(o + (full ? 256 * kT2Rows * 4 : 0));
    g.lgt = o; o = a16(o + (full ? 511 * 4 : 0));
    g.q = o; o = a16(o + (full ? 0 : 65 * 4));
    g.magic = o; o = a16(o + (cross ? (2 * ha + 2) * 4 : 0));
    g.arm = o; o = a16(o + (cross ? txc * 4 : 0));
    g.lc = o; o = a16(o + g.nx * 4);
    g.lg = o; o = a16(o + (stage_g ? g.nx * 4 : 0));
    g.rc = o; o = a16(o + g.nr * 4);
    g.rg = o; o = a16(o + (full ? g.nr * 4 : 0));
    g.rng = o; o = a16(o + (prior ? g.nx * 4 : 0));                                // lo | hi << 16
    g.pre = o; o = a16(o + (cross ? (size_t)g.nx * W2 * 4 : 0));
    g.cnt = o; o = a16(o + (cross && prior ? (size_t)g.nx * W2 * 2 : 0));        // valid counts
    g.tot = o; o = a16(o + (cross ? (size_t)g.nrun * W2 * 4 : 0));
    g.totc = o; o = a16(o + (cross && prior ? (size_t)g.nrun * W2 * 2 : 0));
    g.emit = o; o = a16(o + (size_t)g.nrun * g.rl * 4);
    g.total = o;
    return g;
}

__device__ __forceinline__ uint32_t pack_g(const uint8_t* gray, const uint8_t* gx, const uint8_t* gy, int i) {
    return (uint32_t)gray[i] | ((uint32_t)gx[i] << 8) | ((uint32_t)gy[i] << 16);
}

// Quantised costs of two (left, right) descriptor pairs (disparities 2w and 2w + 1 of one lane),
// packed low / high: the reference's float steps (src/cost_computer.cpp:247-264), each rounded on
// its own, two lanes per packed f32x2 instruction.  (int)(v * scale + 0.5f) truncates a value in
// [0.5, 2^23): adding 2^23 rounded toward zero leaves exactly 2^23 + trunc(v), so the integer is
// the low mantissa bits; truncation saturates below zero in the reference, and here v >= 0.5.
__device__ __forceinline__ unsigned long long f2add_rn(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2add_rz(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("add.rz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2mul_rn(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ unsigned long long f2pack(float lo, float hi) {
    return (unsigned long long)__float_as_uint(lo) | ((unsigned long long)__float_as_uint(hi) << 32);
}

template <bool FULL>
__device__ __forceinline__ uint32_t run_cost2(uint32_t lc, uint32_t lg, uint32_t rc0, uint32_t rg0, uint32_t rc1,
                                              uint32_t rg1, const float* s_t2, const float* s_lgt,
                                              const uint32_t* s_q, unsigned long long scale2, uint32_t cmax2) {
    const uint32_t pop0 = __popc(lc ^ rc0), pop1 = __popc(lc ^ rc1);
    if constexpr (!FULL) {
        return __byte_perm(s_q[pop0], s_q[pop1], 0x5410);
    } else {
        const uint32_t ad0 = __vabsdiffu4(lg, rg0), ad1 = __vabsdiffu4(lg, rg1);  // |dgray|, |dgx|, |dgy|
        // t2[pop][|dgray|] at pop * 256 + |dgray| (pop < 256, so its second byte is zero)
        const float t0 = s_t2[__byte_perm(ad0, pop0, 0x5540)];
        const float t1 = s_t2[__byte_perm(ad1, pop1, 0x5540)];
        const float g0 = s_lgt[__dp4a(ad0, 0x00010100u, 0u)];
        const float g1 = s_lgt[__dp4a(ad1, 0x00010100u, 0u)];
        const unsigned long long v = f2add_rn(f2pack(t0, t1), f2pack(g0, g1));
        const unsigned long long u = f2add_rn(f2mul_rn(v, scale2), 0x3F0000003F000000ull);  // + 0.5f
        const unsigned long long q = f2add_rz(u, 0x4B0000004B000000ull);                    // + 2^23, toward 0
        // the low 16 bits of each lane's mantissa are its integer (< 2^16 by the host's cost_max check)
        return __vminu2(__byte_perm((uint32_t)q, (uint32_t)(q >> 32), 0x5410), cmax2);
    }
}

template <int N>
__device__ __forceinline__ void store_words(uint32_t* p, const uint32_t (&w)[N]) {
    if constexpr (N == 4) {
        *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    } else if constexpr (N == 2) {
        *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) p[i] = w[i];
    }
}

// WPL 16-bit count words (two 8-bit valid counts each) at p, which is 4-byte aligned for even WPL.
template <int N>
__device__ __forceinline__ void store_counts(uint16_t* p, const uint32_t (&c)[N]) {
    if constexpr (N % 2 == 0) {
#pragma unroll
        for (int i = 0; i < N; i += 2)
            *reinterpret_cast<uint32_t*>(p + i) = (c[i] & 0xFFFFu) | (c[i + 1] << 16);
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) p[i] = (uint16_t)c[i];
    }
}

// One run of steps of this lane's P disparities.  V: every (x, d) of the run is a valid voxel for
// every lane of the warp (no per-voxel tests).
// PRIOR: every left pixel has its own range [lo, hi) (staged in s_rng); a voxel outside it is
// invalid, and the aggregation also keeps a prefix of valid counts (s_cnt, s_totc).
template <bool V, bool CROSS, bool STORE, bool FULL, int WPL, bool PRIOR, bool U8>
__device__ __forceinline__ void run_steps(const CostCtx& c, const RunGeom& g, int row, int xbase, int xs, int xe,
                                          const uint32_t* s_lc, const uint32_t* s_lg, const uint32_t* s_rc,
                                          const uint32_t* s_rg, const float* s_t2, const float* s_lgt,
                                          const uint32_t* s_q, const uint32_t* s_rng, uint32_t* s_pre,
                                          uint16_t* s_cnt, uint32_t* s_tot, uint16_t* s_totc, uint32_t* s_em,
                                          int run, uint32_t* __restrict__ out_vol, uint32_t* __restrict__ rkey) {
    constexpr int P = 2 * WPL;
    constexpr int W2 = 32 * WPL;
    const int lane = threadIdx.x & 31;
    const int dbase = P * lane;  // first disparity index of this lane
    const unsigned long long scale2 = f2pack(c.scale, c.scale);
    const uint32_t cmax2 = (uint32_t)c.cost_max * 0x00010001u;
    // lanes wholly past the range load at the last in-bounds even base (dl + P <= D + roff keeps
    // every window entry inside the staged row; even keeps the 8-byte loads aligned) and are
    // masked; a lane with any disparity below D has dbase <= D - 1 < D + roff - P, so keeps its own
    const int dl = V ? dbase : min(dbase, (c.D + g.roff - P) & ~1);
    int ri = xs - dl + c.D - 1 + g.roff;  // staged right descriptor of (xs, dl); even
    uint32_t wc[P], wg[P], acc[P], pre[WPL], cnt[WPL];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        // before the first step's shift: wc[j] holds the descriptor of (xs - 1, dl + j)
        wc[j] = j < P - 1 ? s_rc[ri - 1 - j] : 0u;
        wg[j] = (FULL && j < P - 1) ? s_rg[ri - 1 - j] : 0u;
        acc[j] = kInvalidWord;
    }
#pragma unroll
    for (int w = 0; w < WPL; ++w) pre[w] = cnt[w] = 0;
    uint32_t* pp = s_pre + xs * W2 + WPL * lane;                             // prefix words of (xs)
    uint16_t* cp = s_cnt + xs * W2 + WPL * lane;                             // count words of (xs)
    uint32_t* vp = out_vol + ((size_t)row + (xbase + xs)) * W2 + WPL * lane;  // volume words of (xs)
    // byte volume: the lane's 2 * WPL disparities of (xs) as WPL / 2 words
    uint32_t* vp8 = out_vol + ((size_t)row + (xbase + xs)) * (W2 / 2) + (WPL / 2) * lane;
    for (int xi = xs; xi < xe; xi += 4) {
        const uint4 lc4 = *reinterpret_cast<const uint4*>(s_lc + xi);
        uint4 lg4 = make_uint4(0, 0, 0, 0);
        if (FULL) lg4 = *reinterpret_cast<const uint4*>(s_lg + xi);
        const uint2 na = *reinterpret_cast<const uint2*>(s_rc + ri);
        const uint2 nb = *reinterpret_cast<const uint2*>(s_rc + ri + 2);
        uint2 ga = make_uint2(0, 0), gb = make_uint2(0, 0);
        if (FULL) {
            ga = *reinterpret_cast<const uint2*>(s_rg + ri);
            gb = *reinterpret_cast<const uint2*>(s_rg + ri + 2);
        }
        const uint32_t L[4] = {lc4.x, lc4.y, lc4.z, lc4.w};
        const uint32_t LG[4] = {lg4.x, lg4.y, lg4.z, lg4.w};
        const uint32_t NC[4] = {na.x, na.y, nb.x, nb.y};
        const uint32_t NG[4] = {ga.x, ga.y, gb.x, gb.y};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int x = xbase + xi + s;
#pragma unroll
            for (int j = P - 1; j > 0; --j) {
                wc[j] = wc[j - 1];
                wg[j] = wg[j - 1];
            }
            wc[0] = NC[s];
            wg[0] = NG[s];
            uint32_t qp[WPL];  // quantised costs of disparities 2w | 2w + 1 << 16
            uint32_t vm[WPL];  // their validity: 0xFFFF per valid half
            uint32_t rmask = 0xFFFFu;  // this lane's disparities inside the left pixel's range
            if (PRIOR) {
                const uint32_t rg = s_rng[xi + s];
                const int base = c.d0 + dbase;
                const int a0 = min(max((int)(int16_t)(rg & 0xFFFFu) - base, 0), P);
                const int a1 = min(max((int)(int16_t)(rg >> 16) - base, 0), P);
                rmask = ((1u << a1) - 1u) & ~((1u << a0) - 1u);
            }
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                qp[w] = run_cost2<FULL>(L[s], LG[s], wc[2 * w], wg[2 * w], wc[2 * w + 1], wg[2 * w + 1], s_t2, s_lgt,
                                        s_q, scale2, cmax2);
                vm[w] = 0xFFFFFFFFu;
                if (!V || PRIOR) {
                    uint32_t m = 0;
#pragma unroll
                    for (int hs = 0; hs < 2; ++hs) {
                        const int j = 2 * w + hs;
                        bool ok = true;
                        if (!V) {
                            const int di = dbase + j, xr = x - c.d0 - di;
                            ok = x >= 0 && x < c.w && di < c.D && xr >= 0 && xr < c.w;
                        }
                        if (PRIOR) ok = ok && ((rmask >> j) & 1u);
                        if (ok) m |= 0xFFFFu << (16 * hs);
                    }
                    vm[w] = m;
                }
#pragma unroll
                for (int hs = 0; hs < 2; ++hs) {
                    const int j = 2 * w + hs;
                    // key (cost << 16 | disparity index), or the invalid word
                    const uint32_t key = hs == 0 ? ((qp[w] << 16) | (uint32_t)(dbase + j))
                                                 : ((qp[w] & 0xFFFF0000u) | (uint32_t)(dbase + j));
                    const bool ok = (V && !PRIOR) || ((vm[w] >> (16 * hs)) & 1u);
                    acc[j] = min(acc[j], ok ? key : kInvalidWord);
                }
            }
            // the oldest minimum moves one lane up; lane 31's is complete for this run
            const uint32_t out = acc[P - 1];
            if (lane == 31) s_em[xi - xs + s] = out;
            const uint32_t in = __shfl_up_sync(0xFFFFFFFFu, out, 1);
#pragma unroll
            for (int j = P - 1; j > 0; --j) acc[j] = acc[j - 1];
            acc[0] = lane ? in : kInvalidWord;
            if (CROSS) {
#pragma unroll
                for (int w = 0; w < WPL; ++w) pre[w] += qp[w] & vm[w];
                store_words<WPL>(pp + s * W2, pre);
                if (PRIOR) {
#pragma unroll
                    for (int w = 0; w < WPL; ++w) cnt[w] += __byte_perm(vm[w], 0u, 0x4420) & 0x0101u;  // (valid low) | (valid high) << 8
                    store_counts<WPL>(cp + s * W2, cnt);
                }
            } else if (STORE) {
                // without a halo the staged pixels are the tile's; V runs lie inside the image
                if (V || (xi + s < g.txc && x < c.w)) {
                    uint32_t wd[WPL];
#pragma unroll
                    for (int w = 0; w < WPL; ++w) wd[w] = qp[w] | ~vm[w];  // invalid halves: 0xFFFF
                    if constexpr (U8) {
                        // the low byte of each half: costs are below 255, the invalid 0xFFFF becomes 0xFF
                        uint32_t wb[WPL / 2];
#pragma unroll
                        for (int w = 0; w < WPL / 2; ++w) wb[w] = __byte_perm(wd[2 * w], wd[2 * w + 1], 0x6420);
                        store_words<WPL / 2>(vp8 + (size_t)s * (W2 / 2), wb);
                    } else {
                        store_words<WPL>(vp + (size_t)s * W2, wd);
                    }
                }
            }
        }
        ri += 4;
        pp += 4 * W2;
        cp += 4 * W2;
        vp += 4 * (size_t)W2;
        vp8 += 2 * (size_t)W2;
    }
    __syncwarp();
    if (xe > xs) {
        // minima that left lane 31 at step xs + e: right pixel xbase + xs + e - d0 - (Dp - 1)
        const int n = xe - xs;
        const int r0 = xbase + xs - c.d0 - (2 * W2 - 1);
        for (int e = lane; e < n; e += 32) {
            const uint32_t m = s_em[e];
            const int r = r0 + e;
            if (m != kInvalidWord && r >= 0 && r < c.w) atomicMin(rkey + row + r, m);
        }
        // partial minima still held: acc[j] is for right pixel xl + 1 - d0 - dbase - j
        const int r1 = xbase + xe - c.d0 - dbase;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const int r = r1 - j;
            if (acc[j] != kInvalidWord && r >= 0 && r < c.w) atomicMin(rkey + row + r, acc[j]);
        }
    }
    __syncwarp();
    if (CROSS) store_words<WPL>(s_tot + run * W2 + WPL * lane, pre);
    if (CROSS && PRIOR) store_counts<WPL>(s_totc + run * W2 + WPL * lane, cnt);
}

// Aggregated word kk at pixel x from its packed window sum s (cost.cu's tile kernel, same rules).
__device__ __forceinline__ uint32_t agg_word(const CostCtx& c, uint32_t s, int kk, int x, int l, int r,
                                             const uint32_t* s_magic) {
    const int dw = c.d0 + 2 * kk;
    if (2 * kk + 1 < c.D && x - l >= dw + 1 && x + r <= c.w - 1 + dw) {
        const uint32_t len = (uint32_t)(l + r + 1), mg = s_magic[len];
        return div_by_magic(s & 0xFFFFu, len, mg) | (div_by_magic(s >> 16, len, mg) << 16);
    }
    uint32_t word = 0;
#pragma unroll
    for (int hs = 0; hs < 2; ++hs) {
        const int di = 2 * kk + hs;
        const int d = c.d0 + di;
        const uint32_t sh = (s >> (16 * hs)) & 0xFFFFu;
        const int nh = min(x + r, c.w - 1 + d) - max(x - l, d) + 1;  // valid x' in the window
        const bool ok = di < c.D && d <= x && nh > 0;
        const uint32_t q = ok ? div_by_magic(sh, (uint32_t)nh, s_magic[nh]) : kInvalidCost;
        word |= q << (16 * hs);
    }
    return word;
}

// Aggregated word kk from its window sum s and its two 8-bit valid counts n, with per-pixel ranges
// (cost.cu's tile kernel, same rule): a half is valid when its disparity is inside the centre
// pixel's range and its window holds a valid voxel.
__device__ __forceinline__ uint32_t prior_word(const CostCtx& c, uint32_t s, uint32_t n, int kk, int lo, int hi,
                                               const uint32_t* s_magic) {
    uint32_t word = 0;
#pragma unroll
    for (int hs = 0; hs < 2; ++hs) {
        const int di = 2 * kk + hs;
        const int d = c.d0 + di;
        const uint32_t sh = (s >> (16 * hs)) & 0xFFFFu, nh = (n >> (8 * hs)) & 0xFFu;
        const bool ok = di < c.D && d >= lo && d < hi && nh > 0;
        const uint32_t q = ok ? div_by_magic(sh, nh, s_magic[nh]) : kInvalidCost;
        word |= q << (16 * hs);
    }
    return word;
}

// With 192 or 256 padded disparities the aggregating kernel keeps one block per SM (registers for
// the wider lane state, wider tiles: less halo); otherwise two.
template <bool CROSS, bool STORE, bool FULL, int WPL, bool PRIOR, bool U8>
__global__ void __launch_bounds__(CROSS ? 512 : 256, CROSS ? (WPL > 2 ? 1 : 2) : 1)
    cost_run_kernel(CostCtx c, RunGeom g, int lmax, int tau, uint32_t* __restrict__ out_vol,
                    uint32_t* __restrict__ rkey, const uint32_t* __restrict__ magic) {
    constexpr int W2 = 32 * WPL;
    constexpr int P = 2 * WPL;
    extern __shared__ __align__(16) unsigned char smem[];
    float* s_t2 = reinterpret_cast<float*>(smem + g.t2);
    float* s_lgt = reinterpret_cast<float*>(smem + g.lgt);
    uint32_t* s_q = reinterpret_cast<uint32_t*>(smem + g.q);
    uint32_t* s_magic = reinterpret_cast<uint32_t*>(smem + g.magic);
    uint32_t* s_arm = reinterpret_cast<uint32_t*>(smem + g.arm);
    uint32_t* s_lc = reinterpret_cast<uint32_t*>(smem + g.lc);
    uint32_t* s_lg = reinterpret_cast<uint32_t*>(smem + g.lg);
    uint32_t* s_rc = reinterpret_cast<uint32_t*>(smem + g.rc);
    uint32_t* s_rg = reinterpret_cast<uint32_t*>(smem + g.rg);
    uint32_t* s_pre = reinterpret_cast<uint32_t*>(smem + g.pre);
    uint32_t* s_tot = reinterpret_cast<uint32_t*>(smem + g.tot);
    uint32_t* s_rng = reinterpret_cast<uint32_t*>(smem + g.rng);
    uint16_t* s_cnt = reinterpret_cast<uint16_t*>(smem + g.cnt);
    uint16_t* s_totc = reinterpret_cast<uint16_t*>(smem + g.totc);
    const int tid = threadIdx.x, nt = blockDim.x, run = tid >> 5, lane = tid & 31;
    uint32_t* s_em = reinterpret_cast<uint32_t*>(smem + g.emit) + run * g.rl;

    if (FULL) {
        for (int i = tid; i < 256 * kT2Rows; i += nt) {
            const int pop = i >> 8, ad = i & 255;
            const float lc = c.lut[kLutCensus + pop];
            s_t2[i] = c.use_ad ? __fadd_rn(lc, c.lut[kLutAd + ad]) : lc;
        }
        // without the gradient term, + 0.0f leaves every sum as it is
        for (int i = tid; i < 511; i += nt) s_lgt[i] = c.use_grad ? c.lut[kLutGrad + i] : 0.0f;
    } else {
        for (int i = tid; i < 65; i += nt) s_q[i] = c.qlut[i];
    }
    if (CROSS)
        for (int i = tid; i < 2 * g.ha + 2; i += nt) s_magic[i] = magic[i];

    const int xs = min(run * g.rl, g.nx), xe = min(xs + g.rl, g.nx);

    for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
        const int y = tile / g.ntx;
        const int x0 = (tile - y * g.ntx) * g.txc;
        const int xbase = x0 - g.ha;
        const int rbase = xbase - (c.d0 + c.D - 1) - g.roff;  // image column of staged right 0
        const int row = y * c.w;
        __syncthreads();  // the previous item's readers are done with the staging
        for (int i = tid; i < g.nx; i += nt) {
            const int x = xbase + i;
            const bool in = x >= 0 && x < c.w;
            s_lc[i] = in ? c.cl[row + x] : 0u;
            if (FULL || CROSS) s_lg[i] = in ? pack_g(c.lgray, c.lgx, c.lgy, row + x) : 0u;
            // outside the image: an empty range
            if (PRIOR) s_rng[i] = in ? ((uint32_t)(uint16_t)c.rmin[row + x] | ((uint32_t)(uint16_t)c.rmax[row + x] << 16)) : 0u;
        }
        for (int i = tid; i < g.nr; i += nt) {
            const int xr = rbase + i;
            const bool in = xr >= 0 && xr < c.w;
            s_rc[i] = in ? c.cr[row + xr] : 0u;
            if (FULL) s_rg[i] = in ? pack_g(c.rgray, c.rgx, c.rgy, row + xr) : 0u;
        }
        __syncthreads();
        if (CROSS) {
            // arms (build_cross_arms, src/cost_aggregator.cpp:17-63) and the runs each window
            // spans: l | r << 8 | run(a - 1) << 16 | run(b) << 24 over staged [a, b]
            for (int i = tid; i < g.txc; i += nt) {
                const int x = x0 + i;
                if (x >= c.w) break;
                const int sxi = i + g.ha;
                const int c0 = (int)(s_lg[sxi] & 0xFFu);
                int l = 0, r = 0;
                while (l < lmax && x - l - 1 >= 0 && abs((int)(s_lg[sxi - l - 1] & 0xFFu) - c0) <= tau) ++l;
                while (r < lmax && x + r + 1 < c.w && abs((int)(s_lg[sxi + r + 1] & 0xFFu) - c0) <= tau) ++r;
                const int a = sxi - l, b = sxi + r;
                const int rlo = a > 0 ? (a - 1) / g.rl : 0, rhi = b / g.rl;
                s_arm[i] = (uint32_t)l | ((uint32_t)r << 8) | ((uint32_t)rlo << 16) | ((uint32_t)rhi << 24);
            }
        }
        {
            const int xa = xbase + xs, xb = xbase + xe - 1;
            const int dlo = c.d0 + P * lane;
            const bool ok = xa >= 0 && xb < c.w && P * lane + P - 1 < c.D && xa - (dlo + P - 1) >= 0 &&
                            xb - dlo <= c.w - 1;
            if (__all_sync(0xFFFFFFFFu, ok))
                run_steps<true, CROSS, STORE, FULL, WPL, PRIOR, U8>(c, g, row, xbase, xs, xe, s_lc, s_lg, s_rc, s_rg, s_t2,
                                                                s_lgt, s_q, s_rng, s_pre, s_cnt, s_tot, s_totc, s_em,
                                                                run, out_vol, rkey);
            else
                run_steps<false, CROSS, STORE, FULL, WPL, PRIOR, U8>(c, g, row, xbase, xs, xe, s_lc, s_lg, s_rc, s_rg,
                                                                 s_t2, s_lgt, s_q, s_rng, s_pre, s_cnt, s_tot, s_totc,
                                                                 s_em, run, out_vol, rkey);
        }
        if (CROSS) {
            __syncthreads();
            // run offsets: the run totals become an exclusive prefix over the runs, per word, so a
            // window's sum is two lookups whatever number of runs it spans (sums wrap modulo 2^32
            // and counts modulo 2^16; the window differences are exact, as for the prefixes)
            for (int k = tid; k < W2; k += nt) {
                uint32_t acc = 0;
                for (int j = 0; j < g.nrun; ++j) {
                    const uint32_t v = s_tot[j * W2 + k];
                    s_tot[j * W2 + k] = acc;
                    acc += v;
                }
                if (PRIOR) {
                    uint16_t accc = 0;
                    for (int j = 0; j < g.nrun; ++j) {
                        const uint16_t v = s_totc[j * W2 + k];
                        s_totc[j * W2 + k] = accc;
                        accc = (uint16_t)(accc + v);
                    }
                }
            }
            __syncthreads();
            // T(x, d) = floor(window sum / valid count) over [x - L(x), x + R(x)]; a thread takes
            // four words of one pixel, so the pixel's arms, divisor and border tests serve eight
            // disparities and its loads are independent
            constexpr int quads = W2 / 4;
            for (int item = tid; item < g.txc * quads; item += nt) {
                const int xi = item / quads, k4 = 4 * (item - xi * quads);
                const int x = x0 + xi;
                if (x >= c.w) break;
                const uint32_t arm = s_arm[xi];
                const int l = (int)(arm & 0xFFu), r = (int)((arm >> 8) & 0xFFu);
                const int rlo = (int)((arm >> 16) & 0xFFu), rhi = (int)(arm >> 24);
                const int sxi = xi + g.ha, a = sxi - l, b = sxi + r;
                const uint4 pb = *reinterpret_cast<const uint4*>(s_pre + b * W2 + k4);
                const uint4 ob = *reinterpret_cast<const uint4*>(s_tot + rhi * W2 + k4);
                const uint4 oa = *reinterpret_cast<const uint4*>(s_tot + rlo * W2 + k4);
                const uint4 pa = a > 0 ? *reinterpret_cast<const uint4*>(s_pre + (a - 1) * W2 + k4) : make_uint4(0, 0, 0, 0);
                const uint32_t sum[4] = {(pb.x + ob.x) - (pa.x + oa.x), (pb.y + ob.y) - (pa.y + oa.y),
                                         (pb.z + ob.z) - (pa.z + oa.z), (pb.w + ob.w) - (pa.w + oa.w)};
                uint32_t wd[4];
                const uint32_t len = (uint32_t)(l + r + 1);
                if constexpr (PRIOR) {
                    // valid counts of the window from the count prefix (two 8-bit counts per word),
                    // validity from the centre pixel's range (the tile kernel's rule)
                    const uint2 cb = *reinterpret_cast<const uint2*>(s_cnt + b * W2 + k4);
                    const uint2 ca = a > 0 ? *reinterpret_cast<const uint2*>(s_cnt + (a - 1) * W2 + k4) : make_uint2(0, 0);
                    const uint2 tb = *reinterpret_cast<const uint2*>(s_totc + rhi * W2 + k4);
                    const uint2 ta = *reinterpret_cast<const uint2*>(s_totc + rlo * W2 + k4);
                    const uint32_t cw[4] = {(cb.x & 0xFFFFu) + (tb.x & 0xFFFFu) - (ca.x & 0xFFFFu) - (ta.x & 0xFFFFu),
                                            (cb.x >> 16) + (tb.x >> 16) - (ca.x >> 16) - (ta.x >> 16),
                                            (cb.y & 0xFFFFu) + (tb.y & 0xFFFFu) - (ca.y & 0xFFFFu) - (ta.y & 0xFFFFu),
                                            (cb.y >> 16) + (tb.y >> 16) - (ca.y >> 16) - (ta.y >> 16)};
                    const uint32_t rg = s_rng[sxi];
                    const int lo = (int)(int16_t)(rg & 0xFFFFu), hi = (int)(int16_t)(rg >> 16);
#pragma unroll
                    for (int q = 0; q < 4; ++q) wd[q] = prior_word(c, sum[q], cw[q] & 0xFFFFu, k4 + q, lo, hi, s_magic);
                } else if (c.D == c.Dp && len > 1 && x - l >= c.d0 + c.Dp - 1 && x + r <= c.w - 1 + c.d0) {
                    // every word of the pixel has its whole window valid (no padded words, x - d inside
                    // the image over the window for every d): one count, no per-word tests
                    const uint32_t mg = s_magic[len];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        wd[q] = __byte_perm(__umulhi(sum[q] & 0xFFFFu, mg), __umulhi(sum[q] >> 16, mg), 0x5410);
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) wd[q] = agg_word(c, sum[q], k4 + q, x, l, r, s_magic);
                }
                *reinterpret_cast<uint4*>(out_vol + ((size_t)row + x) * W2 + k4) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
            }
        }
    }
}

// Shared memory one SM gives each of `per_sm` resident blocks.
size_t smem_per_block(int per_sm) {
    static size_t sm_total = 0, reserved = 0;
    if (!sm_total) {
        int dev = 0, v = 0, r = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&r, cudaDevAttrReservedSharedMemoryPerBlock, dev) == cudaSuccess) {
            sm_total = (size_t)v;
            reserved = (size_t)r;
        } else {
            cudaGetLastError();
            return 100 * 1024;
        }
    }
    return sm_total / per_sm - reserved;
}

// Tile width of the aggregating form: the fewest tiles per row (least halo) whose staging lets two
// 16-warp blocks share an SM (one block for 192 or 256 padded disparities); a requested width
// (tuning key cost_tile) wins when it fits one block.
int cross_tile(const CostCtx& c, int lmax, bool full) {
    const bool prior = c.prior_ranges != 0;
    if ((c.tile == 64 || c.tile == 128 || c.tile == 256) &&
        run_geom(c, c.tile, lmax, true, full, prior).total <= 200 * 1024)
        return c.tile;
    // one block per SM for the wide forms (see cost_run_kernel), else two
    const size_t budget = smem_per_block(c.Dp > 128 ? 1 : 2);
    for (int ntx = 1; ntx <= c.w; ++ntx) {
        const int txc = round_up((c.w + ntx - 1) / ntx, 4);
        if (run_geom(c, txc, lmax, true, full, prior).total <= budget) return txc;
        if (txc <= 32) break;
    }
    return 32;
}

template <bool CROSS, bool STORE, bool FULL, int WPL, bool PRIOR, bool U8>
cudaError_t launch_runs_w(const CostCtx& c, int txc, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    const RunGeom g = run_geom(c, txc, CROSS ? lmax : 0, CROSS, FULL, PRIOR);
    const int nt = 32 * g.nrun;
    auto kern = cost_run_kernel<CROSS, STORE, FULL, WPL, PRIOR, U8>;
    cudaError_t e = allow_dynamic_smem(kern, g.total);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, nsm = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, g.total);
    if (e != cudaSuccess) return e;
    const int blocks = std::max(1, std::min(g.ntiles, std::max(1, per_sm) * nsm));
    kern<<<blocks, nt, g.total, s>>>(c, g, lmax, tau, vol, rkey, magic);
    return cudaGetLastError();
}

// Words per lane as a compile-time constant: one warp spans Dp = 64 * WPL disparities.
template <bool CROSS, bool STORE, bool FULL, bool PRIOR>
cudaError_t launch_runs_p(const CostCtx& c, int txc, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    if constexpr (STORE && !CROSS && !FULL && !PRIOR) {
        // the byte volume (Fast census-only costs below 255): 128 or 256 padded disparities
        if (c.vol8) {
            if (c.Dp == 128) return launch_runs_w<CROSS, STORE, FULL, 2, PRIOR, true>(c, txc, lmax, tau, vol, rkey, magic, s);
            if (c.Dp == 256) return launch_runs_w<CROSS, STORE, FULL, 4, PRIOR, true>(c, txc, lmax, tau, vol, rkey, magic, s);
            return cudaErrorInvalidValue;
        }
    } else {
        if (c.vol8) return cudaErrorInvalidValue;
    }
    switch (c.Dp) {
        case 64: return launch_runs_w<CROSS, STORE, FULL, 1, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
        case 128: return launch_runs_w<CROSS, STORE, FULL, 2, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
        case 192: return launch_runs_w<CROSS, STORE, FULL, 3, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
        default: return launch_runs_w<CROSS, STORE, FULL, 4, PRIOR, false>(c, txc, lmax, tau, vol, rkey, magic, s);
    }
}

template <bool CROSS, bool STORE, bool FULL>
cudaError_t launch_runs_t(const CostCtx& c, int txc, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                          const uint32_t* magic, cudaStream_t s) {
    if (c.prior_ranges) return launch_runs_p<CROSS, STORE, FULL, true>(c, txc, lmax, tau, vol, rkey, magic, s);
    return launch_runs_p<CROSS, STORE, FULL, false>(c, txc, lmax, tau, vol, rkey, magic, s);
}

}  // namespace

size_t cost_runs_smem_bytes(const CostCtx& c, int mode, int lmax) {
    const bool full = c.use_ad || c.use_grad;
    const bool prior = c.prior_ranges != 0;
    if (mode == 1) return run_geom(c, cross_tile(c, lmax, full), lmax, true, full, prior).total;
    return run_geom(c, 256, 0, false, full, prior).total;
}

bool cost_runs_supported(const CostCtx& c, int mode, int lmax) {
    if (c.kernel == 1 || c.census64) return false;
    if (c.Dp % 64 != 0 || c.Dp > 256) return false;
    const bool full = c.use_ad || c.use_grad;
    if (mode == 2 && (full || c.prior_ranges)) return false;  // the fused form: census-only, default ranges
    if (mode == 1 && lmax > 127) return false;
    // the staging must fit the per-block budget the tile width was chosen for
    return cost_runs_smem_bytes(c, mode, lmax) <= smem_per_block(c.Dp > 128 && mode == 1 ? 1 : 2);
}

cudaError_t launch_cost_runs(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                             const uint32_t* magic, cudaStream_t s) {
    const bool full = c.use_ad || c.use_grad;
    if (mode == 1) {
        const int txc = cross_tile(c, lmax, full);
        return full ? launch_runs_t<true, true, true>(c, txc, lmax, tau, vol, rkey, magic, s)
                    : launch_runs_t<true, true, false>(c, txc, lmax, tau, vol, rkey, magic, s);
    }
    if (mode == 0)
        return full ? launch_runs_t<false, true, true>(c, 256, lmax, tau, vol, rkey, magic, s)
                    : launch_runs_t<false, true, false>(c, 256, lmax, tau, vol, rkey, magic, s);
    return launch_runs_t<false, false, false>(c, 256, lmax, tau, vol, rkey, magic, s);
}

}  // namespace apgcu

// Vertical half of the Cross-arm aggregation, CostAggregator::aggregate_hv
// (src/cost_aggregator.cpp:107-138), and a standalone horizontal pass for the second and later
// aggregation iterations (:77-105).
//
// Vertical kernel: a CTA owns `cols` adjacent pixel columns x and a 256-row segment; each thread
// owns one 32-bit word (two disparities) of one column and slides down the segment keeping the
// column prefix sums (sum and count) of the last 2*Lmax+2 rows in a shared-memory ring, so every
// input voxel is read once (plus a 2*Lmax row halo per segment) and every output
// voxel is written once.  The up/down arms (build_cross_arms, :17-63) are computed once per
// pixel into shared memory.  Bound: HBM, 4 bytes per voxel (read T, write C).
//
// Prefix sums are plain 32-bit running sums of the packed words (two disparities): a carry out of
// the low half moves into the high half of the prefix, but a window's difference of two prefixes
// is the 32-bit sum of the window's words, exact in both halves because the window's low halves
// sum to less than 2^16: valid costs are host-checked ((2 * lmax + 1) * cost_max < 2^16), and an
// invalid low half is either zeroed before it is added or, in the default-range kernel, sits only
// below an invalid high half, whose window is never used.
#include "common.cuh"
#include "kernels.h"

#include <type_traits>

namespace apgcu {

namespace {
constexpr int kSeg = 256;

// Stores the word (two aggregated costs) at word index i of the output volume: as is, or (U8) as
// two bytes of the byte volume, whose pixel slices hold Dp bytes: every valid aggregated cost is
// below 255 (host-checked), and the invalid 0xFFFF keeps its low byte 0xFF as the marker.
template <bool U8, bool STREAM>
__device__ __forceinline__ void store_cost_word(uint32_t* out, size_t i, uint32_t word) {
    if constexpr (U8) {
        unsigned short* o = reinterpret_cast<unsigned short*>(out) + i;
        const unsigned short b = (unsigned short)__byte_perm(word, 0u, 0x0020);  // bytes 0 and 2
        if constexpr (STREAM) __stcs(o, b);
        else *o = b;
    } else {
        if constexpr (STREAM) __stcs(out + i, word);
        else out[i] = word;
    }
}

template <bool U8>
__global__ void cross_v_kernel(int w, int h, int d0, int D, int Dp, int lmax, int tau, int cols,
                               const uint8_t* __restrict__ gray, const int16_t* __restrict__ rmin,
                               const int16_t* __restrict__ rmax, const uint32_t* __restrict__ tin,
                               uint32_t* __restrict__ cout, const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int W2 = Dp / 2;
    const int RS = 2 * lmax + 2;
    const int nthr = W2 * cols;
    uint32_t* ring_s = reinterpret_cast<uint32_t*>(smem);          // [RS][nthr]
    uint32_t* ring_c = ring_s + (size_t)RS * nthr;                  // [RS][nthr]
    uint8_t* armU = reinterpret_cast<uint8_t*>(ring_c + (size_t)RS * nthr);  // [cols][kSeg]
    uint8_t* armD = armU + cols * kSeg;

    const int xb = blockIdx.x * cols;
    const int y0 = blockIdx.y * kSeg;
    const int y1 = min(h, y0 + kSeg);
    const int tid = threadIdx.x;

    for (int i = tid; i < cols * kSeg; i += blockDim.x) {
        const int ci = i / kSeg, yy = y0 + (i - ci * kSeg);
        const int x = xb + ci;
        int u = 0, v = 0;
        if (x < w && yy < h) {
            const int c0 = gray[yy * w + x];
            while (u < lmax && yy - u - 1 >= 0 && abs((int)gray[(yy - u - 1) * w + x] - c0) <= tau) ++u;
            while (v < lmax && yy + v + 1 < h && abs((int)gray[(yy + v + 1) * w + x] - c0) <= tau) ++v;
        }
        armU[i] = (uint8_t)u;
        armD[i] = (uint8_t)v;
    }
    __syncthreads();
    if (tid >= nthr) return;
    const int ci = tid / W2, k = tid - ci * W2;
    const int x = xb + ci;
    if (x >= w) return;

    const int ystart = max(0, y0 - lmax);
    int r_next = ystart;
    uint32_t ps = 0, pc = 0;
    ring_s[(ystart % RS) * nthr + tid] = 0;
    ring_c[(ystart % RS) * nthr + tid] = 0;
    for (int y = y0; y < y1; ++y) {
        const int need = min(h, y + lmax + 1);
        while (r_next < need) {
            const uint32_t v = tin[((size_t)r_next * w + x) * W2 + k];
            const uint32_t inval = __vcmpeq2(v, kInvalidWord);
            ps += v & ~inval;
            pc += 0x00010001u & ~inval;
            ++r_next;
            const int slot = (r_next % RS) * nthr + tid;
            ring_s[slot] = ps;
            ring_c[slot] = pc;
        }
        const int ai = ci * kSeg + (y - y0);
        const int a = y - armU[ai], b = y + armD[ai] + 1;
        const uint32_t s = ring_s[(b % RS) * nthr + tid] - ring_s[(a % RS) * nthr + tid];
        const uint32_t n = ring_c[(b % RS) * nthr + tid] - ring_c[(a % RS) * nthr + tid];
        const int lo = rmin[y * w + x], hi = rmax[y * w + x];
        uint32_t word = 0;
#pragma unroll
        for (int hs = 0; hs < 2; ++hs) {
            const int di = 2 * k + hs;
            const int d = d0 + di;
            const uint32_t sh = (s >> (16 * hs)) & 0xFFFFu, nh = (n >> (16 * hs)) & 0xFFFFu;
            uint32_t q = kInvalidCost;
            if (di < D && d >= lo && d < hi && nh > 0) q = div_by_magic(sh, nh, magic[nh]);
            word |= q << (16 * hs);
        }
        store_cost_word<U8, false>(cout, ((size_t)y * w + x) * W2 + k, word);
    }
}

// Vertical pass when every pixel has the default range [d0, min(dmax, x+1)) and d0 >= 0: then
// T(x, y', d) is valid exactly when d <= x, for every row y', so the window count is the window
// length and no count prefix is needed; lanes with d > x hold the invalid marker in every row and
// their (wrapped) sums are never used, and such a lane is never the low half of a word whose high
// half is valid (d0 >= 0: validity only ends at the top of a pixel's range).  Each thread keeps its column's prefix sums in a power-of-two shared
// ring and loads its input words kB rows at a time, one batch ahead of use (register double
// buffer), so kB loads per thread are in flight; the gray column segment is staged in shared
// memory for the arms.
constexpr int kB = 16;
constexpr int kQ = 8;  // output rows computed together (independent windows: their loads overlap)

// WPT words (of two disparities) per thread: the arms, ring slots, window length and divisor of
// an output row are shared by the thread's words, and its loads, ring accesses and stores are
// WPT words wide.
template <int WPT>
struct Words {
    uint32_t v[WPT];
};
template <int WPT>
__device__ __forceinline__ Words<WPT> load_words(const uint32_t* p) {
    Words<WPT> r;
    if constexpr (WPT == 2) {
        const uint2 t = __ldcs(reinterpret_cast<const uint2*>(p));
        r.v[0] = t.x; r.v[1] = t.y;
    } else {
        r.v[0] = __ldcs(p);
    }
    return r;
}
template <int WPT>
__device__ __forceinline__ void ring_put(uint32_t* p, const uint32_t (&v)[WPT]) {
    if constexpr (WPT == 2) *reinterpret_cast<uint2*>(p) = make_uint2(v[0], v[1]);
    else p[0] = v[0];
}
template <int WPT>
__device__ __forceinline__ void ring_get(const uint32_t* p, uint32_t (&v)[WPT]) {
    if constexpr (WPT == 2) {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = p[0];
    }
}
// Stores WPT words from word index i (a multiple of WPT) of the output volume; see store_cost_word.
template <bool U8, int WPT>
__device__ __forceinline__ void store_cost_words(uint32_t* out, size_t i, const uint32_t (&wd)[WPT]) {
    if constexpr (WPT == 1) {
        store_cost_word<U8, true>(out, i, wd[0]);
    } else if constexpr (U8) {
        __stcs(reinterpret_cast<unsigned int*>(out) + i / 2, __byte_perm(wd[0], wd[1], 0x6420));
    } else {
        __stcs(reinterpret_cast<uint2*>(out + i), make_uint2(wd[0], wd[1]));
    }
}

template <int RS, bool U8, int WPT>
__global__ void __launch_bounds__(128) cross_v_default_kernel(int w, int h, int d0, int D, int Dp, int lmax, int tau,
                                                              int cols, const uint8_t* __restrict__ gray,
                                                              const uint32_t* __restrict__ tin,
                                                              uint32_t* __restrict__ cout,
                                                              const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int W2 = Dp / 2;
    const int tpc = W2 / WPT;      // threads per column
    const int nthr = tpc * cols;   // threads with words
    const int rw = W2 * cols;      // ring words per slot
    uint32_t* ring = reinterpret_cast<uint32_t*>(smem);                      // [RS][rw]
    uint32_t* s_magic = ring + (size_t)RS * rw;                                // [2*lmax+2]
    uint8_t* s_gray = reinterpret_cast<uint8_t*>(s_magic + 2 * lmax + 2);     // [cols][kSeg + 2*lmax]
    uint8_t* armU = s_gray + cols * (kSeg + 2 * lmax);                         // [cols][kSeg]
    uint8_t* armD = armU + cols * kSeg;
    const int xb = blockIdx.x * cols;
    const int y0 = blockIdx.y * kSeg;
    const int y1 = min(h, y0 + kSeg);
    const int tid = threadIdx.x;
    const int gs = kSeg + 2 * lmax;  // staged gray rows [y0 - lmax, y0 + kSeg + lmax)

    for (int i = tid; i < 2 * lmax + 2; i += blockDim.x) s_magic[i] = magic[i];
    for (int i = tid; i < cols * gs; i += blockDim.x) {
        const int r = i / cols, ci = i - r * cols;
        const int yy = y0 - lmax + r, x = xb + ci;
        s_gray[ci * gs + r] = (x < w && yy >= 0 && yy < h) ? gray[yy * w + x] : 0;
    }
    __syncthreads();
    for (int i = tid; i < cols * kSeg; i += blockDim.x) {
        const int ci = i / kSeg, r = i - ci * kSeg;
        const int yy = y0 + r, x = xb + ci;
        int u = 0, v = 0;
        if (x < w && yy < h) {
            const uint8_t* g = s_gray + ci * gs + lmax + r;  // g[0] = gray(x, yy)
            const int c0 = g[0];
            while (u < lmax && yy - u - 1 >= 0 && abs((int)g[-u - 1] - c0) <= tau) ++u;
            while (v < lmax && yy + v + 1 < h && abs((int)g[v + 1] - c0) <= tau) ++v;
        }
        armU[i] = (uint8_t)u;
        armD[i] = (uint8_t)v;
    }
    __syncthreads();
    if (tid >= nthr) return;
    const int ci = tid / tpc, k = (tid - ci * tpc) * WPT;  // the thread's first word
    const int x = xb + ci;
    if (x >= w) return;
    const int roff = ci * W2 + k;  // the thread's words within a ring slot
    // output lanes that can be valid: d < dmax and d <= x
    bool lane_ok[2 * WPT];
#pragma unroll
    for (int hs = 0; hs < 2 * WPT; ++hs) lane_ok[hs] = (2 * k + hs < D) && (d0 + 2 * k + hs <= x);

    const int ystart = max(0, y0 - lmax);
    const int yend = min(h, y1 + lmax);  // rows read: [ystart, yend)
    // ring slot of prefix P(r) (sum over rows [ystart, r]) is (r - ystart + 1) & (RS - 1); slot 0 = P(ystart - 1) = 0
    {
        uint32_t z[WPT] = {};
        ring_put<WPT>(ring + roff, z);
    }
    const size_t rowstride = (size_t)w * W2;
    const uint32_t* src = tin + ((size_t)ystart * w + x) * W2 + k;
    Words<WPT> cur[kB], nxt[kB];
#pragma unroll
    for (int i = 0; i < kB; ++i) cur[i] = ystart + i < yend ? load_words<WPT>(src + i * rowstride) : Words<WPT>{};
#pragma unroll
    for (int i = 0; i < kB; ++i)
        nxt[i] = ystart + kB + i < yend ? load_words<WPT>(src + (kB + i) * rowstride) : Words<WPT>{};
    int pushed = ystart;  // next row to add to the ring
    uint32_t ps[WPT] = {};
    size_t dst = ((size_t)y0 * w + x) * W2 + k;  // word index of (x, y0), word k
    for (int yb = y0; yb < y1; yb += kQ) {
        // prefixes up to the last window of the chunk's rows, then kQ independent rows
        const int need = min(h, min(yb + kQ, y1) + lmax);
        while (pushed < need) {
            // add the buffered batch (rows [pushed, pushed + kB)) and load the one after next
#pragma unroll
            for (int i = 0; i < kB; ++i) {
                if (pushed + i < yend) {
#pragma unroll
                    for (int j = 0; j < WPT; ++j) ps[j] += cur[i].v[j];
                    ring_put<WPT>(ring + ((pushed + i - ystart + 1) & (RS - 1)) * rw + roff, ps);
                }
            }
            pushed += kB;
#pragma unroll
            for (int i = 0; i < kB; ++i) cur[i] = nxt[i];
            const int base = pushed + kB;
#pragma unroll
            for (int i = 0; i < kB; ++i)
                nxt[i] = base + i < yend ? load_words<WPT>(src + (size_t)(base + i - ystart) * rowstride) : Words<WPT>{};
        }
#pragma unroll
        for (int i = 0; i < kQ; ++i) {
            const int y = yb + i;
            if (y >= y1) break;
            const int ai = ci * kSeg + (y - y0);
            const int a = y - armU[ai], b = y + armD[ai];  // inclusive window
            uint32_t pb[WPT], pa[WPT];
            ring_get<WPT>(ring + ((b - ystart + 1) & (RS - 1)) * rw + roff, pb);
            ring_get<WPT>(ring + ((a - ystart) & (RS - 1)) * rw + roff, pa);
            const int len = b - a + 1;
            const uint32_t mg = s_magic[len];
            uint32_t wd[WPT];
#pragma unroll
            for (int j = 0; j < WPT; ++j) {
                const uint32_t sum = pb[j] - pa[j];
                uint32_t word = 0;
#pragma unroll
                for (int hs = 0; hs < 2; ++hs) {
                    const uint32_t sh = (sum >> (16 * hs)) & 0xFFFFu;
                    const uint32_t q = lane_ok[2 * j + hs] ? div_by_magic(sh, (uint32_t)len, mg) : kInvalidCost;
                    word |= q << (16 * hs);
                }
                wd[j] = word;
            }
            store_cost_words<U8, WPT>(cout, dst + (size_t)i * rowstride, wd);
        }
        dst += (size_t)kQ * rowstride;
    }
}

// Vertical pass for any ranges (per-pixel ranges of the prior, negative disparities, wide
// ranges): the batched, power-of-two ring form above plus a prefix of valid counts.  Sums are plain
// 32-bit running sums of the packed words with invalid halves zeroed, and counts are 16-bit running
// sums of (valid low half) | (valid high half) << 8: a window difference is exact in every lane
// because a window's sum is below 2^16 (host-checked for the arm length and cost_max) and its
// counts are at most 2*lmax + 1 <= 255.  The centre pixel's range is staged with the arms.
template <int RS, int KB, bool U8, int WPT>
__global__ void __launch_bounds__(256) cross_v_count_kernel(int w, int h, int d0, int D, int Dp, int lmax, int tau,
                                                            int cols, const uint8_t* __restrict__ gray,
                                                            const int16_t* __restrict__ rmin,
                                                            const int16_t* __restrict__ rmax,
                                                            const uint32_t* __restrict__ tin,
                                                            uint32_t* __restrict__ cout,
                                                            const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int W2 = Dp / 2;
    const int tpc = W2 / WPT;     // threads per column
    const int nthr = tpc * cols;  // threads with words
    const int rw = W2 * cols;     // ring words per slot
    uint32_t* ring = reinterpret_cast<uint32_t*>(smem);                  // [RS][rw] sums
    uint32_t* s_rng = ring + (size_t)RS * rw;                            // [cols][kSeg] lo | hi << 16
    uint32_t* s_magic = s_rng + cols * kSeg;                             // [2*lmax+2]
    uint16_t* ringc = reinterpret_cast<uint16_t*>(s_magic + 2 * lmax + 2);  // [RS][rw] counts
    uint8_t* s_gray = reinterpret_cast<uint8_t*>(ringc + (size_t)RS * rw);  // [cols][kSeg + 2*lmax]
    uint8_t* armU = s_gray + cols * (kSeg + 2 * lmax);                   // [cols][kSeg]
    uint8_t* armD = armU + cols * kSeg;
    const int xb = blockIdx.x * cols;
    const int y0 = blockIdx.y * kSeg;
    const int y1 = min(h, y0 + kSeg);
    const int tid = threadIdx.x;
    const int gs = kSeg + 2 * lmax;

    for (int i = tid; i < 2 * lmax + 2; i += blockDim.x) s_magic[i] = magic[i];
    for (int i = tid; i < cols * gs; i += blockDim.x) {
        const int r = i / cols, ci = i - r * cols;
        const int yy = y0 - lmax + r, x = xb + ci;
        s_gray[ci * gs + r] = (x < w && yy >= 0 && yy < h) ? gray[yy * w + x] : 0;
    }
    __syncthreads();
    for (int i = tid; i < cols * kSeg; i += blockDim.x) {
        const int ci = i / kSeg, r = i - ci * kSeg;
        const int yy = y0 + r, x = xb + ci;
        int u = 0, v = 0;
        uint32_t rg = 0;
        if (x < w && yy < h) {
            const uint8_t* g = s_gray + ci * gs + lmax + r;
            const int c0 = g[0];
            while (u < lmax && yy - u - 1 >= 0 && abs((int)g[-u - 1] - c0) <= tau) ++u;
            while (v < lmax && yy + v + 1 < h && abs((int)g[v + 1] - c0) <= tau) ++v;
            rg = (uint32_t)(uint16_t)rmin[yy * w + x] | ((uint32_t)(uint16_t)rmax[yy * w + x] << 16);
        }
        armU[i] = (uint8_t)u;
        armD[i] = (uint8_t)v;
        s_rng[i] = rg;
    }
    __syncthreads();
    if (tid >= nthr) return;
    const int ci = tid / tpc, k = (tid - ci * tpc) * WPT;  // the thread's first word
    const int x = xb + ci;
    if (x >= w) return;
    const int roff = ci * W2 + k;  // the thread's words within a ring slot

    const int ystart = max(0, y0 - lmax);
    const int yend = min(h, y1 + lmax);
    {
        uint32_t z[WPT] = {};
        ring_put<WPT>(ring + roff, z);
        if constexpr (WPT == 2) *reinterpret_cast<uint32_t*>(ringc + roff) = 0u;
        else ringc[roff] = 0;
    }
    const size_t rowstride = (size_t)w * W2;
    const uint32_t* src = tin + ((size_t)ystart * w + x) * W2 + k;
    Words<WPT> cur[KB], nxt[KB];
#pragma unroll
    for (int i = 0; i < KB; ++i) cur[i] = ystart + i < yend ? load_words<WPT>(src + i * rowstride) : Words<WPT>{};
#pragma unroll
    for (int i = 0; i < KB; ++i)
        nxt[i] = ystart + KB + i < yend ? load_words<WPT>(src + (KB + i) * rowstride) : Words<WPT>{};
    int pushed = ystart;
    uint32_t ps[WPT] = {};
    uint32_t pc[WPT] = {};  // low 16 bits used
    size_t dst = ((size_t)y0 * w + x) * W2 + k;  // word index of (x, y0), word k
    // ring slots kept incrementally (RS need not be a power of two): pslot is the slot of row
    // `pushed`, yslot the slot of the prefix through the output row y, (y - ystart + 1) % RS
    int pslot = 1;
    int yslot = (y0 - ystart + 1) % RS;
    for (int yb = y0; yb < y1; yb += kQ) {
        const int need = min(h, min(yb + kQ, y1) + lmax);
        while (pushed < need) {
#pragma unroll
            for (int i = 0; i < KB; ++i) {
                if (pushed + i < yend) {
#pragma unroll
                    for (int j = 0; j < WPT; ++j) {
                        const uint32_t v = cur[i].v[j];
                        const bool lo_bad = (v & 0xFFFFu) == 0xFFFFu, hi_bad = v >= 0xFFFF0000u;
                        ps[j] += v & ((lo_bad ? 0u : 0x0000FFFFu) | (hi_bad ? 0u : 0xFFFF0000u));
                        pc[j] += (lo_bad ? 0u : 1u) + (hi_bad ? 0u : 0x100u);
                    }
                    const int slot = pslot * rw + roff;
                    ring_put<WPT>(ring + slot, ps);
                    if constexpr (WPT == 2)
                        *reinterpret_cast<uint32_t*>(ringc + slot) = (pc[0] & 0xFFFFu) | (pc[1] << 16);
                    else ringc[slot] = (uint16_t)pc[0];
                }
                pslot = pslot + 1 == RS ? 0 : pslot + 1;
            }
            pushed += KB;
#pragma unroll
            for (int i = 0; i < KB; ++i) cur[i] = nxt[i];
            const int base = pushed + KB;
#pragma unroll
            for (int i = 0; i < KB; ++i)
                nxt[i] = base + i < yend ? load_words<WPT>(src + (size_t)(base + i - ystart) * rowstride) : Words<WPT>{};
        }
#pragma unroll
        for (int i = 0; i < kQ; ++i) {
            const int y = yb + i;
            if (y >= y1) break;
            const int ai = ci * kSeg + (y - y0);
            // inclusive window [y - armU, y + armD]: the prefixes through y + armD and y - armU - 1
            int sb = yslot + armD[ai], sa = yslot - armU[ai] - 1;
            sb = sb >= RS ? sb - RS : sb;
            sa = sa < 0 ? sa + RS : sa;
            sb = sb * rw + roff;
            sa = sa * rw + roff;
            yslot = yslot + 1 == RS ? 0 : yslot + 1;
            uint32_t pb[WPT], pa[WPT], cnt[WPT];
            ring_get<WPT>(ring + sb, pb);
            ring_get<WPT>(ring + sa, pa);
            if constexpr (WPT == 2) {
                const uint32_t cb = *reinterpret_cast<const uint32_t*>(ringc + sb);
                const uint32_t ca = *reinterpret_cast<const uint32_t*>(ringc + sa);
                cnt[0] = (cb - ca) & 0xFFFFu;
                cnt[1] = ((cb >> 16) - (ca >> 16)) & 0xFFFFu;
            } else {
                cnt[0] = (uint32_t)(uint16_t)(ringc[sb] - ringc[sa]);
            }
            const uint32_t rg = s_rng[ai];
            const int lo = (int16_t)(rg & 0xFFFFu), hi = (int16_t)(rg >> 16);
            uint32_t wd[WPT];
#pragma unroll
            for (int j = 0; j < WPT; ++j) {
                const uint32_t sum = pb[j] - pa[j];
                uint32_t word = 0;
#pragma unroll
                for (int hs = 0; hs < 2; ++hs) {
                    const int di = 2 * (k + j) + hs;
                    const int d = d0 + di;
                    const uint32_t sh = (sum >> (16 * hs)) & 0xFFFFu, nh = (cnt[j] >> (8 * hs)) & 0xFFu;
                    uint32_t q = kInvalidCost;
                    if (di < D && d >= lo && d < hi && nh > 0) q = div_by_magic(sh, nh, s_magic[nh]);
                    word |= q << (16 * hs);
                }
                wd[j] = word;
            }
            store_cost_words<U8, WPT>(cout, dst + (size_t)i * rowstride, wd);
        }
        dst += (size_t)kQ * rowstride;
    }
}

// Horizontal pass over a volume (aggregation iterations after the first).  A CTA owns one row
// and a run of `cols` pixels... implemented as the transpose of the vertical kernel: one thread
// per (row, word) sliding along x.
__global__ void cross_h_kernel(int w, int h, int d0, int D, int Dp, int lmax, int tau,
                               const uint8_t* __restrict__ gray, const int16_t* __restrict__ rmin,
                               const int16_t* __restrict__ rmax, const uint32_t* __restrict__ vin,
                               uint32_t* __restrict__ vout, const uint32_t* __restrict__ magic) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int W2 = Dp / 2;
    const int RS = 2 * lmax + 2;
    const int nthr = W2;
    uint32_t* ring_s = reinterpret_cast<uint32_t*>(smem);
    uint32_t* ring_c = ring_s + (size_t)RS * nthr;
    const int y = blockIdx.y;
    const int x0 = blockIdx.x * kSeg, x1 = min(w, x0 + kSeg);
    const int k = threadIdx.x;
    if (k >= W2) return;
    const int xstart = max(0, x0 - lmax);
    int r_next = xstart;
    uint32_t ps = 0, pc = 0;
    ring_s[(xstart % RS) * nthr + k] = 0;
    ring_c[(xstart % RS) * nthr + k] = 0;
    const uint8_t* g = gray + (size_t)y * w;
    for (int x = x0; x < x1; ++x) {
        const int need = min(w, x + lmax + 1);
        while (r_next < need) {
            const uint32_t v = vin[((size_t)y * w + r_next) * W2 + k];
            const uint32_t inval = __vcmpeq2(v, kInvalidWord);
            ps += v & ~inval;
            pc += 0x00010001u & ~inval;
            ++r_next;
            const int slot = (r_next % RS) * nthr + k;
            ring_s[slot] = ps;
            ring_c[slot] = pc;
        }
        const int c0 = g[x];
        int l = 0, r = 0;
        while (l < lmax && x - l - 1 >= 0 && abs((int)g[x - l - 1] - c0) <= tau) ++l;
        while (r < lmax && x + r + 1 < w && abs((int)g[x + r + 1] - c0) <= tau) ++r;
        const int a = x - l, b = x + r + 1;
        const uint32_t s = ring_s[(b % RS) * nthr + k] - ring_s[(a % RS) * nthr + k];
        const uint32_t n = ring_c[(b % RS) * nthr + k] - ring_c[(a % RS) * nthr + k];
        const int lo = rmin[y * w + x], hi = rmax[y * w + x];
        uint32_t word = 0;
#pragma unroll
        for (int hs = 0; hs < 2; ++hs) {
            const int di = 2 * k + hs;
            const int d = d0 + di;
            const uint32_t sh = (s >> (16 * hs)) & 0xFFFFu, nh = (n >> (16 * hs)) & 0xFFFFu;
            uint32_t q = kInvalidCost;
            if (di < D && d >= lo && d < hi && nh > 0) q = div_by_magic(sh, nh, magic[nh]);
            word |= q << (16 * hs);
        }
        vout[((size_t)y * w + x) * W2 + k] = word;
    }
}
template <bool U8>
cudaError_t launch_cross_v_t(int w, int h, int d0, int D, int Dp, int lmax, int tau, const uint8_t* gray,
                             const int16_t* rmin, const int16_t* rmax, const uint32_t* tin, uint32_t* cout,
                             const uint32_t* magic, bool default_ranges, cudaStream_t s) {
    const int W2 = Dp / 2;
    const int cols = W2 >= 128 ? 1 : 128 / W2;
    const int nthr = W2 * cols;
    // fast path: default ranges, non-negative disparities, and a ring holding the windows' prefixes
    // of a chunk of kQ rows plus the batch pushed ahead: rows from yb - lmax - 1 up to
    // yb + kQ + lmax + kB - 2 are live, so a ring of 2*lmax + kB + kQ + 2 slots never overwrites
    // one before its last read
    const int span = 2 * lmax + kB + kQ + 2;
    if (default_ranges && d0 >= 0 && nthr <= 128) {
        const size_t extra = (size_t)(2 * lmax + 2) * 4 + (size_t)cols * (kSeg + 2 * lmax) + (size_t)cols * kSeg * 2;
        // two words per thread from 192 padded disparities (one B200, crossV per frame: 1920x1080
        // D256 0.693 -> 0.590 ms, 1242x375 D192 0.139 -> 0.133; slower with fewer words per pixel:
        // 1280x720 D128 0.176 -> 0.181, 640x480 D64 0.059 -> 0.075, where a block's arms weigh more)
        auto go = [&](auto rs_tag, auto wpt_tag) -> cudaError_t {
            constexpr int RS = decltype(rs_tag)::value;
            constexpr int WPT = decltype(wpt_tag)::value;
            const size_t smem = (size_t)RS * nthr * 4 + extra;
            auto kern = cross_v_default_kernel<RS, U8, WPT>;
            {
                const cudaError_t e = allow_dynamic_smem(kern, smem);
                if (e != cudaSuccess) return e;
            }
            dim3 grid((w + cols - 1) / cols, (h + kSeg - 1) / kSeg);
            kern<<<grid, round_up(nthr / WPT, 32), smem, s>>>(w, h, d0, D, Dp, lmax, tau, cols, gray, tin, cout, magic);
            return cudaGetLastError();
        };
        auto pick = [&](auto rs_tag) -> cudaError_t {
            if (W2 >= 96) return go(rs_tag, std::integral_constant<int, 2>());
            return go(rs_tag, std::integral_constant<int, 1>());
        };
        if (span <= 64) return pick(std::integral_constant<int, 64>());
        if (span <= 128) return pick(std::integral_constant<int, 128>());
        if (span <= 256) return pick(std::integral_constant<int, 256>());
    }
    if (nthr <= 256) {
        // any ranges: sum and count rings, batched loads
        const size_t extra = (size_t)cols * kSeg * 4 + (size_t)(2 * lmax + 2) * 4 + (size_t)cols * (kSeg + 2 * lmax) +
                             (size_t)cols * kSeg * 2;
        // one word per thread: two (WPT = 2) made the kernel slower, 1.162 -> 1.305 ms per frame at
        // HighQuality 1920x1080 D256 (its count ring leaves fewer warps per SM)
        auto go = [&](auto rs_tag, auto kb_tag) -> cudaError_t {
            constexpr int RS = decltype(rs_tag)::value;
            constexpr int KB = decltype(kb_tag)::value;
            const size_t smem = (size_t)RS * nthr * 6 + extra;
            auto launch = [&](auto kern, int wpt) -> cudaError_t {
                const cudaError_t e = allow_dynamic_smem(kern, smem);
                if (e != cudaSuccess) return e;
                dim3 grid((w + cols - 1) / cols, (h + kSeg - 1) / kSeg);
                kern<<<grid, round_up(nthr / wpt, 32), smem, s>>>(w, h, d0, D, Dp, lmax, tau, cols, gray, rmin, rmax, tin,
                                                                  cout, magic);
                return cudaGetLastError();
            };
            return launch(cross_v_count_kernel<RS, KB, U8, 1>, 1);
        };
        auto fits = [&](int rs) { return (size_t)rs * nthr * 6 + extra <= 200 * 1024; };
        // the default arm (lmax <= 17) with 8-row load batches: a ring of exactly the 52 live rows,
        // whose smaller footprint fits five blocks on an SM instead of four
        using I = std::integral_constant<int, 8>;
        if (2 * lmax + 8 + kQ + 2 <= 52 && fits(52)) return go(std::integral_constant<int, 52>(), I());
        if (span <= 64 && fits(64)) return go(std::integral_constant<int, 64>(), std::integral_constant<int, kB>());
        if (span <= 128 && fits(128)) return go(std::integral_constant<int, 128>(), std::integral_constant<int, kB>());
        if (span <= 256 && fits(256)) return go(std::integral_constant<int, 256>(), std::integral_constant<int, kB>());
    }
    const int RS = 2 * lmax + 2;
    const size_t smem = (size_t)RS * nthr * 8 + (size_t)cols * kSeg * 2;
    {
        const cudaError_t e = allow_dynamic_smem(cross_v_kernel<U8>, smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((w + cols - 1) / cols, (h + kSeg - 1) / kSeg);
    cross_v_kernel<U8><<<grid, round_up(nthr, 32), smem, s>>>(w, h, d0, D, Dp, lmax, tau, cols, gray, rmin, rmax,
                                                              tin, cout, magic);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_cross_v(int w, int h, int d0, int D, int Dp, int lmax, int tau, const uint8_t* gray,
                           const int16_t* rmin, const int16_t* rmax, const uint32_t* tin, uint32_t* cout,
                           const uint32_t* magic, bool default_ranges, bool out8, cudaStream_t s) {
    if (out8) return launch_cross_v_t<true>(w, h, d0, D, Dp, lmax, tau, gray, rmin, rmax, tin, cout, magic, default_ranges, s);
    return launch_cross_v_t<false>(w, h, d0, D, Dp, lmax, tau, gray, rmin, rmax, tin, cout, magic, default_ranges, s);
}

cudaError_t launch_cross_h(int w, int h, int d0, int D, int Dp, int lmax, int tau, const uint8_t* gray,
                           const int16_t* rmin, const int16_t* rmax, const uint32_t* vin, uint32_t* vout,
                           const uint32_t* magic, cudaStream_t s) {
    const int W2 = Dp / 2;
    const int RS = 2 * lmax + 2;
    const size_t smem = (size_t)RS * W2 * 8;
    {
        const cudaError_t e = allow_dynamic_smem(cross_h_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((w + kSeg - 1) / kSeg, h);
    cross_h_kernel<<<grid, round_up(W2, 32), smem, s>>>(w, h, d0, D, Dp, lmax, tau, gray, rmin, rmax, vin, vout,
                                                        magic);
    return cudaGetLastError();
}

size_t cross_v_smem_bytes(int Dp, int lmax) {
    const int W2 = Dp / 2;
    const int cols = W2 >= 128 ? 1 : 128 / W2;
    return (size_t)(2 * lmax + 2) * W2 * cols * 8 + (size_t)cols * kSeg * 2;
}

}  // namespace apgcu

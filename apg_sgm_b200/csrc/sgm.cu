// Semi-global matching path sweeps with the path sum accumulated in HBM and the
// winner-take-all fused into the last sweep.
//
// Restates SgmOptimizer::optimize / aggregate_path / process_pixel
// (src/sgm_optimizer.cpp:21-81, 186-274) and wta_impl (:436-555):
//   L(p,d) = C(p,d) + min(L'(d), L'(d-1)+P1, L'(d+1)+P1, m'+P2) - m',  m' = min_k L'(k),
//   L = C at the first pixel of a scanline or when no L' entry is valid, L = INF and S = sentinel
//   where C is invalid; S = sum over the 4 or 8 directions.
//
// Design (one warp per scanline: a row, a column or a diagonal ray):
//   * the disparity axis, padded to Dp = 64*K, is spread over the 32 lanes; lane l holds K
//     32-bit words = 2K consecutive disparities as packed uint16x2;
//   * L' stays in registers between steps; L'(d-1) and L'(d+1) come from funnel shifts inside a
//     lane plus one __shfl_up / __shfl_down across lanes; m' is one __reduce_min_sync;
//   * INF is 0xFFFF and every add that can meet INF saturates (__vaddus2), so the reference's
//     "skip invalid predecessor" tests become plain SIMD min/add;
//   * S uses 16-bit lanes (the host only takes this path when npath*(cost_max+max(P2,P1+1)) <
//     65535, can_use_u16_sgm_accumulator, include/apg_sgm/sgm_optimizer.hpp:9-18), and the
//     sentinel 0xFFFF is sticky through the saturating add;
//   * cost source: the (aggregated) u16 volume, or, in the fused Fast path, the census planes:
//     C = qlut[popc(cl(x,y) ^ cr(x-d,y))] recomputed per step, so no cost volume exists;
//   * the last sweep adds its L to S, keeps the sum in registers and does the reference WTA
//     (first minimum, second minimum outside |d-best|<=1, legacy parabola) with two warp
//     min-reductions, so the final S never goes back to HBM.
// Bound: HBM (S read+write 4 B per voxel per middle sweep) and the per-step latency of the
// shuffle/reduce chain; enough scanlines run concurrently to cover the latter at 720p.
#include "common.cuh"
#include "kernels.h"

namespace apgcu {

namespace {

constexpr int kWarps = 4;

enum Mode { kFirst = 0, kAccum = 1, kLast = 2 };

__device__ __forceinline__ uint32_t min_halves(uint32_t v) {
    const uint32_t lo = v & 0xFFFFu, hi = v >> 16;
    return lo < hi ? lo : hi;
}

template <int K>
__device__ __forceinline__ void load_words(const uint32_t* __restrict__ base, uint32_t (&v)[K]) {
    if constexpr (K == 1) {
        v[0] = __ldg(base);
    } else if constexpr (K == 2) {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(base));
        v[0] = t.x; v[1] = t.y;
    } else if constexpr (K == 4) {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(base));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = __ldg(base + k);
    }
}

template <int K>
__device__ __forceinline__ void load_words_rw(const uint32_t* base, uint32_t (&v)[K]) {
    if constexpr (K == 2) {
        const uint2 t = *reinterpret_cast<const uint2*>(base);
        v[0] = t.x; v[1] = t.y;
    } else if constexpr (K == 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(base);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = base[k];
    }
}

template <int K>
__device__ __forceinline__ void store_words(uint32_t* base, const uint32_t (&v)[K]) {
    if constexpr (K == 2) {
        *reinterpret_cast<uint2*>(base) = make_uint2(v[0], v[1]);
    } else if constexpr (K == 4) {
        *reinterpret_cast<uint4*>(base) = make_uint4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) base[k] = v[k];
    }
}

struct SgmArgs {
    int w, h, d0, D, Dp;
    int dx, dy;
    SgmPen pen;
    const uint8_t* gray;            // left gray (P2 adaptation)
    const uint32_t* cvol;           // cost volume words (VOL source)
    // census source (fused Fast path)
    const uint32_t* cl;
    const uint32_t* cr;
    const uint16_t* qlut;           // 65 quantised census costs
    const int16_t* rmin;
    const int16_t* rmax;
    uint32_t* S;                    // path sum words
    // WTA outputs (last sweep)
    float* disp;
    float* best;
    float* second;
    int subpixel;
    int store_final;
};

// Scanline s of direction (dx, dy): first pixel and length.
__device__ __forceinline__ void scan_start(const SgmArgs& a, int s, int& x, int& y, int& len) {
    if (a.dy == 0) {
        y = s; x = a.dx > 0 ? 0 : a.w - 1; len = a.w;
    } else if (a.dx == 0) {
        x = s; y = a.dy > 0 ? 0 : a.h - 1; len = a.h;
    } else {
        // ray s: start pixel whose predecessor (x-dx, y-dy) is outside (as the reference's
        // packed ray enumeration, src/sgm_optimizer.cpp:325-365)
        if (s < a.w) { x = s; y = a.dy > 0 ? 0 : a.h - 1; }
        else { x = a.dx > 0 ? 0 : a.w - 1; y = a.dy > 0 ? (s - a.w + 1) : (a.h - 1 - (s - a.w + 1)); }
        const int rx = a.dx > 0 ? a.w - x : x + 1;
        const int ry = a.dy > 0 ? a.h - y : y + 1;
        len = rx < ry ? rx : ry;
    }
}

template <int K, int MODE, bool CENSUS>
__global__ void __launch_bounds__(kWarps * 32) sgm_path_kernel(SgmArgs a, int nscan) {
    __shared__ uint16_t s_q[65];
    if (CENSUS) {
        for (int i = threadIdx.x; i < 65; i += blockDim.x) s_q[i] = a.qlut[i];
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kWarps + warp;
    if (s >= nscan) return;
    int x, y, len;
    scan_start(a, s, x, y, len);
    const int W2 = a.Dp / 2;
    const int step_p = a.dy * a.w + a.dx;
    int p = y * a.w + x;

    uint32_t L[K];
    uint32_t m = 0xFFFFu;
    int prev_g = 0;
    const uint32_t p1x2 = (uint32_t)a.pen.P1 * 0x00010001u;

    for (int t = 0; t < len; ++t, p += step_p, x += a.dx) {
        uint32_t c[K];
        if (CENSUS) {
            const uint32_t clv = __ldg(a.cl + p);
            const int lo = __ldg(a.rmin + p), hi = __ldg(a.rmax + p);
            const int row = p - x;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                uint32_t wv = 0;
#pragma unroll
                for (int hs = 0; hs < 2; ++hs) {
                    const int di = 2 * (lane * K + k) + hs;
                    const int d = a.d0 + di;
                    const int xr = x - d;
                    uint32_t q = kInvalidCost;
                    if (di < a.D && d >= lo && d < hi && xr >= 0 && xr < a.w)
                        q = s_q[__popc(clv ^ __ldg(a.cr + row + xr))];
                    wv |= q << (16 * hs);
                }
                c[k] = wv;
            }
        } else {
            load_words<K>(a.cvol + (size_t)p * W2 + lane * K, c);
        }
        const int g = __ldg(a.gray + p);

        uint32_t Ln[K];
        if (t == 0 || m == 0xFFFFu) {
#pragma unroll
            for (int k = 0; k < K; ++k) Ln[k] = c[k];
        } else {
            const int P2 = adaptive_p2(a.pen, g - prev_g);
            const uint32_t mp2 = min(m + (uint32_t)P2, 0xFFFFu) * 0x00010001u;
            const uint32_t m2 = m * 0x00010001u;
            uint32_t up = __shfl_up_sync(0xffffffffu, L[K - 1], 1);
            uint32_t dn = __shfl_down_sync(0xffffffffu, L[0], 1);
            if (lane == 0) up = 0xFFFFFFFFu;
            if (lane == 31) dn = 0xFFFFFFFFu;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint32_t lo_nb = k == 0 ? up : L[k - 1];
                const uint32_t hi_nb = k == K - 1 ? dn : L[k + 1];
                const uint32_t lm = __funnelshift_l(lo_nb, L[k], 16);  // (L[k] << 16) | (lo_nb >> 16)
                const uint32_t lp = __funnelshift_r(L[k], hi_nb, 16);  // (L[k] >> 16) | (hi_nb << 16)
                uint32_t bst = __vminu2(L[k], __vaddus2(__vminu2(lm, lp), p1x2));
                bst = __vminu2(bst, mp2);
                uint32_t v = __vadd2(c[k], __vsub2(bst, m2));
                v |= __vcmpeq2(c[k], 0xFFFFFFFFu);
                Ln[k] = v;
            }
        }
        uint32_t lm_min = 0xFFFFu;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            L[k] = Ln[k];
            lm_min = min(lm_min, min_halves(Ln[k]));
        }
        m = __reduce_min_sync(0xffffffffu, lm_min);
        prev_g = g;

        uint32_t* sp = a.S + (size_t)p * W2 + lane * K;
        if (MODE == kFirst) {
            store_words<K>(sp, Ln);
        } else {
            uint32_t sv[K];
            load_words_rw<K>(sp, sv);
#pragma unroll
            for (int k = 0; k < K; ++k) sv[k] = __vaddus2(sv[k], Ln[k]);
            if (MODE == kAccum) {
                store_words<K>(sp, sv);
            } else {
                if (a.store_final) store_words<K>(sp, sv);
                // winner-take-all on the final sum (wta_impl, src/sgm_optimizer.cpp:465-536)
                uint32_t kmin = kInvalidWord;
#pragma unroll
                for (int k = 0; k < K; ++k) {
#pragma unroll
                    for (int hs = 0; hs < 2; ++hs) {
                        const uint32_t v = (sv[k] >> (16 * hs)) & 0xFFFFu;
                        const uint32_t di = 2 * (lane * K + k) + hs;
                        const uint32_t key = v == 0xFFFFu ? kInvalidWord : ((v << 16) | di);
                        kmin = key < kmin ? key : kmin;
                    }
                }
                const uint32_t bkey = __reduce_min_sync(0xffffffffu, kmin);
                float dval = -1.f, fb = __int_as_float(0x7f800000), fs = __int_as_float(0x7f800000);
                // The reference marks "no winner" with best_d = -1 and tests best_d < 0, so a
                // negative winning disparity also yields -1 / +inf / +inf (:490-495).
                if (bkey != kInvalidWord && a.d0 + (int)(bkey & 0xFFFFu) >= 0) {
                    const int bdi = (int)(bkey & 0xFFFFu);
                    uint32_t smin = 0xFFFFu;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
#pragma unroll
                        for (int hs = 0; hs < 2; ++hs) {
                            const int di = 2 * (lane * K + k) + hs;
                            const uint32_t v = (sv[k] >> (16 * hs)) & 0xFFFFu;
                            if (abs(di - bdi) > 1 && v < smin) smin = v;
                        }
                    }
                    const uint32_t sec = __reduce_min_sync(0xffffffffu, smin);
                    // neighbours of the minimum for the parabola
                    const int wm = (bdi - 1) >> 1, wp = (bdi + 1) >> 1;  // word indices
                    uint32_t selm = 0, selp = 0;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        if (lane * K + k == wm) selm = sv[k];
                        if (lane * K + k == wp) selp = sv[k];
                    }
                    const uint32_t vm_w = __shfl_sync(0xffffffffu, selm, bdi >= 1 ? wm / K : 0);
                    const uint32_t vp_w = __shfl_sync(0xffffffffu, selp, wp / K < 32 ? wp / K : 31);
                    if (lane == 0) {
                        const uint32_t bv = bkey >> 16;
                        dval = (float)(a.d0 + bdi);
                        if (a.subpixel && bdi > 0 && bdi + 1 < a.D) {
                            const uint32_t cm = (vm_w >> (16 * ((bdi - 1) & 1))) & 0xFFFFu;
                            const uint32_t cp = (vp_w >> (16 * ((bdi + 1) & 1))) & 0xFFFFu;
                            if (cm != 0xFFFFu && cp != 0xFFFFu)
                                dval = __fadd_rn(dval, legacy_delta((float)cm, (float)bv, (float)cp));
                        }
                        fb = (float)bv;
                        fs = sec == 0xFFFFu ? __int_as_float(0x7f800000) : (float)sec;
                    }
                }
                if (lane == 0) {
                    a.disp[p] = dval;
                    a.best[p] = fb;
                    a.second[p] = fs;
                }
            }
        }
        y += a.dy;
    }
}

template <int K, int MODE>
cudaError_t launch_k(const SgmArgs& a, bool census, cudaStream_t st) {
    int nscan;
    if (a.dy == 0) nscan = a.h;
    else if (a.dx == 0) nscan = a.w;
    else nscan = a.w + a.h - 1;
    const int blocks = (nscan + kWarps - 1) / kWarps;
    if (census) sgm_path_kernel<K, MODE, true><<<blocks, kWarps * 32, 0, st>>>(a, nscan);
    else sgm_path_kernel<K, MODE, false><<<blocks, kWarps * 32, 0, st>>>(a, nscan);
    return cudaGetLastError();
}

template <int K>
cudaError_t launch_mode(const SgmArgs& a, int mode, bool census, cudaStream_t st) {
    if (mode == kFirst) return launch_k<K, kFirst>(a, census, st);
    if (mode == kAccum) return launch_k<K, kAccum>(a, census, st);
    return launch_k<K, kLast>(a, census, st);
}

}  // namespace

cudaError_t launch_sgm_path(const SgmPathLaunch& l, cudaStream_t st) {
    SgmArgs a;
    a.w = l.w; a.h = l.h; a.d0 = l.d0; a.D = l.D; a.Dp = l.Dp; a.dx = l.dx; a.dy = l.dy;
    a.pen = l.pen; a.gray = l.gray; a.cvol = l.cvol; a.cl = l.cl; a.cr = l.cr; a.qlut = l.qlut;
    a.rmin = l.rmin; a.rmax = l.rmax; a.S = l.S; a.disp = l.disp; a.best = l.best; a.second = l.second;
    a.subpixel = l.subpixel;
    a.store_final = l.store_final;
    const bool census = l.cvol == nullptr;
    switch (l.Dp / 64) {
        case 1: return launch_mode<1>(a, l.mode, census, st);
        case 2: return launch_mode<2>(a, l.mode, census, st);
        case 3: return launch_mode<3>(a, l.mode, census, st);
        case 4: return launch_mode<4>(a, l.mode, census, st);
        case 5: return launch_mode<5>(a, l.mode, census, st);
        case 6: return launch_mode<6>(a, l.mode, census, st);
        case 7: return launch_mode<7>(a, l.mode, census, st);
        case 8: return launch_mode<8>(a, l.mode, census, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace apgcu

// Semi-global matching path sweeps with the path sum in HBM and the winner-take-all fused into
// the last sweep.
//
// Restates SgmOptimizer::optimize / aggregate_path / process_pixel
// (src/sgm_optimizer.cpp:21-81, 186-274) and wta_impl (:436-555):
//   L(p,d) = C(p,d) + min(L'(d), L'(d-1)+P1, L'(d+1)+P1, m'+P2) - m',  m' = min_k L'(k),
//   L = C at the first pixel of a scanline or when no L' entry is valid, L = INF and S = sentinel
//   where C is invalid; S = sum over the 4 or 8 directions (an order-free integer sum).
//
// Design:
//   * the directions whose sweeps do not need another's result run together in ONE launch
//     (left->right, right->left, top->bottom; plus the four diagonals for 8 paths), each chain
//     writing its own path-sum buffer, so a pair puts 3-7x more chains in flight than a sweep at a
//     time; the last sweep (bottom->top) adds the partial sums (Path8: folded into one buffer
//     first) and runs the WTA.  HBM traffic equals sweep-by-sweep accumulation (Path4: 3 writes +
//     3 reads of 2 B per voxel = 12 B per voxel);
//   * a chain (one scanline of one direction) runs on a sub-group of T = 8, 16 or 32 lanes; a
//     warp carries 32/T scanlines in one instruction stream.  Lane j of a group owns 2K
//     consecutive disparities packed as K uint16x2 words, Dp = 2*K*T;
//   * L' stays in registers; L'(d-1) / L'(d+1) come from funnel shifts inside a lane plus one
//     group shuffle each way; m' is one group __reduce_min_sync;
//   * min-plus arithmetic uses the DPX instructions (__viaddmin_u16x2 = min(a+b, c) per
//     halfword): best = min(L', min(L'(d-1), L'(d+1)) + P1, m'+P2) is three SIMD ops.
//     Invalid entries are 0x7FFF: larger than any valid path value (<= cost_max + P2), small
//     enough that 0x7FFF + P2 + P1 never wraps, so the reference's "skip invalid predecessor"
//     tests need no masks.  An invalid cost gives L in [0x7FFF, 0x7FFF+P2]; path sums add with
//     unsigned saturation, so a voxel is invalid iff its sum is >= 0x7FFF (valid sums stay below
//     npath*(cost_max+P2) < 0x7FFF, checked on the host);
//   * cost source: the (aggregated) u16 volume, or in the fused Fast path the census planes,
//     C = qlut[popc(cl(x,y) ^ cr(x-d,y))].  Along a row the right descriptors of a lane slide by
//     one disparity per step, so a horizontal sweep keeps them in a register ring and takes one
//     new descriptor per step from the neighbouring lane (shuffle) or, at the group edge, from
//     memory;
//   * loads run PF steps ahead of use: the census-fed sweeps keep them in a register ring; the
//     volume-fed sweeps (every mode's default) stage costs and partial sums through a per-warp
//     shared-memory ring filled by cp.async, one commit group per step (run_chain_vol);
//   * the volume-fed last sweep runs on two warps per chain: one for the recurrence, one for the
//     partial sums and the WTA (sgm_last_split_kernel);
//   * the last sweep adds its L to S, keeps the final sum in registers and runs the reference WTA
//     (first minimum, second minimum outside |d-best| <= 1, legacy parabola) with two group
//     min-reductions, so the final sum never returns to HBM.
// Bound: HBM (S written once, read-modify-written by the middle sweeps, read by the last) and, on
// the longest scanline, the per-step latency of the shuffle / DPX / reduce chain.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace apgcu {

namespace {

constexpr uint32_t kInf = 0x7FFFu;
constexpr uint32_t kInf2 = 0x7FFF7FFFu;

// One step of the path recurrence per halfword, c + (b - m), as plain 32-bit arithmetic: every half
// of b is at least m (b is a minimum over candidates that are each at least the previous step's
// minimum m) and every result half stays below 0x10000 (costs are at most 0x7FFF and b - m at most
// P2, which the configuration check keeps below 0x7FFF - P1), so no borrow or carry crosses the
// halves and the result equals the per-halfword modular form.
__device__ __forceinline__ uint32_t path_value(uint32_t c, uint32_t b, uint32_t m2) { return c + b - m2; }
// Per-halfword unsigned saturating add: a + min(b, 0xFFFF - a) never carries out of a half.
__device__ __forceinline__ uint32_t addus2(uint32_t a, uint32_t b) { return a + __vminu2(b, ~a); }

enum Mode { kFirst = 0, kLast = 2 };
constexpr int kMaxDirs = 8;

__device__ __forceinline__ uint32_t min_halves(uint32_t v) {
    const uint32_t lo = v & 0xFFFFu, hi = v >> 16;
    return lo < hi ? lo : hi;
}

template <int K>
__device__ __forceinline__ void ld_nc(const uint32_t* __restrict__ base, uint32_t (&v)[K]) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const uint4 t = __ldg(reinterpret_cast<const uint4*>(base + k));
            v[k] = t.x; v[k + 1] = t.y; v[k + 2] = t.z; v[k + 3] = t.w;
        }
    } else if constexpr (K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 2) {
            const uint2 t = __ldg(reinterpret_cast<const uint2*>(base + k));
            v[k] = t.x; v[k + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = __ldg(base + k);
    }
}

// Path sums: L2-coherent, L1-bypassing (.cg); each sum word is touched by one thread per launch.
template <int K>
__device__ __forceinline__ void ld_cg(const uint32_t* base, uint32_t (&v)[K]) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const uint4 t = __ldcg(reinterpret_cast<const uint4*>(base + k));
            v[k] = t.x; v[k + 1] = t.y; v[k + 2] = t.z; v[k + 3] = t.w;
        }
    } else if constexpr (K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 2) {
            const uint2 t = __ldcg(reinterpret_cast<const uint2*>(base + k));
            v[k] = t.x; v[k + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = __ldcg(base + k);
    }
}

template <int K>
__device__ __forceinline__ void st_cg(uint32_t* base, const uint32_t (&v)[K]) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) __stcg(reinterpret_cast<uint4*>(base + k), make_uint4(v[k], v[k + 1], v[k + 2], v[k + 3]));
    } else if constexpr (K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 2) __stcg(reinterpret_cast<uint2*>(base + k), make_uint2(v[k], v[k + 1]));
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) __stcg(base + k, v[k]);
    }
}

struct SgmArgs {
    int w, h, d0, D, Dp, dmax;
    SgmPen pen;
    const uint8_t* gray;
    const uint32_t* cvol;
    const uint32_t* cl;
    const uint32_t* cr;
    const uint16_t* qlut;
    float* disp;
    float* best;
    float* second;
    int subpixel;
    int sp_method;
    float sp_param;
    apg_subpixel_telemetry_t* sp_tel;
    int store_final;
    int cost8;  // cvol holds one byte per voxel (0xFF invalid)
    // a band of the last sweep's steps, [t_begin, t_end) (the banded one-warp kernel only): the
    // chains' L and m enter from `carry` when t_begin > 0 and leave there when t_end is short of
    // the chain's end (32 * (K + 1) words per chain: K words of L, then m, each lane its column)
    int t_begin, t_end;
    uint32_t* carry;
};

// Directions of one launch; warps [warp_begin[i], warp_begin[i+1]) run direction i.
struct DirTable {
    int n;
    int dx[kMaxDirs], dy[kMaxDirs], nscan[kMaxDirs];
    int warp_begin[kMaxDirs + 1];
    uint32_t* out[kMaxDirs];       // first phase: each direction's own path-sum buffer
    const uint32_t* in[kMaxDirs];  // last sweep: the partial sums to add
    int nin;
};

// Scanline s of direction (dx, dy): first pixel and length (0 when s is past the last one).
__device__ __forceinline__ void scan_start(const SgmArgs& a, int dx, int dy, int s, int nscan, int& x, int& y,
                                           int& len) {
    x = 0; y = 0; len = 0;
    if (s >= nscan) return;
    if (dy == 0) {
        y = s; x = dx > 0 ? 0 : a.w - 1; len = a.w;
    } else if (dx == 0) {
        x = s; y = dy > 0 ? 0 : a.h - 1; len = a.h;
    } else {
        // ray s: start pixel whose predecessor (x-dx, y-dy) is outside the image (the reference's
        // ray enumeration, src/sgm_optimizer.cpp:325-365)
        if (s < a.w) { x = s; y = dy > 0 ? 0 : a.h - 1; }
        else { x = dx > 0 ? 0 : a.w - 1; y = dy > 0 ? (s - a.w + 1) : (a.h - 1 - (s - a.w + 1)); }
        const int rx = dx > 0 ? a.w - x : x + 1;
        const int ry = dy > 0 ? a.h - y : y + 1;
        len = rx < ry ? rx : ry;
    }
}

// Data of one future step, loaded ahead of use.
template <int K, bool CENSUS, int HDIR, int NB>
struct Slot {
    static constexpr int NC = CENSUS ? (HDIR != 0 ? 1 : 2 * K) : K;
    uint32_t c[NC];          // volume: cost words; census: right descriptors (sliding: the new one)
    uint32_t s[NB > 0 ? NB : 1][K];  // partial path sums to add (last sweep)
    uint32_t clv;            // census: left descriptor
    int g;                   // left gray
};

template <int K, int T, bool CENSUS, int HDIR, int NB>
__device__ __forceinline__ void fetch(const SgmArgs& a, const DirTable& tab, int j, int p, int x,
                                      Slot<K, CENSUS, HDIR, NB>& sl) {
    const int W2 = a.Dp / 2;
    sl.g = __ldg(a.gray + p);
    if (CENSUS) {
        sl.clv = __ldg(a.cl + p);
        const int row = p - x;
        if (HDIR > 0) {
            // the one descriptor entering the ring at this step: disparity d0 (lane 0 of the group)
            const int xr = x - a.d0;
            sl.c[0] = (j == 0 && xr >= 0 && xr < a.w) ? __ldg(a.cr + row + xr) : 0u;
        } else if (HDIR < 0) {
            // entering at the top: disparity d0 + Dp - 1 (last lane of the group)
            const int xr = x - (a.d0 + a.Dp - 1);
            sl.c[0] = (j == T - 1 && xr >= 0 && xr < a.w) ? __ldg(a.cr + row + xr) : 0u;
        } else {
#pragma unroll
            for (int i = 0; i < 2 * K; ++i) {
                const int xr = x - (a.d0 + 2 * K * j + i);
                sl.c[i] = (xr >= 0 && xr < a.w) ? __ldg(a.cr + row + xr) : 0u;
            }
        }
    } else {
        ld_nc<K>(a.cvol + (size_t)p * W2 + j * K, reinterpret_cast<uint32_t(&)[K]>(sl.c));
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) ld_cg<K>(tab.in[b] + (size_t)p * W2 + j * K, sl.s[b]);
}

// Winner-take-all on the final sums of the group's pixel p (wta_impl, src/sgm_optimizer.cpp:465-536).
template <int K, int T>
__device__ __forceinline__ void wta(const SgmArgs& a, unsigned gmask, int j, int p, const uint32_t (&sv)[K]) {
    uint32_t kmin = kInvalidWord;
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int hs = 0; hs < 2; ++hs) {
            const uint32_t v = (sv[k] >> (16 * hs)) & 0xFFFFu;
            const uint32_t di = 2 * (j * K + k) + hs;
            const uint32_t key = v >= kInf ? kInvalidWord : ((v << 16) | di);
            kmin = key < kmin ? key : kmin;
        }
    const uint32_t bkey = __reduce_min_sync(gmask, kmin);
    float dval = -1.f, fb = __int_as_float(0x7f800000), fs = __int_as_float(0x7f800000);
    // The reference marks "no winner" with best_d = -1 and tests best_d < 0, so a negative
    // winning disparity also yields -1 / +inf / +inf (:490-495).
    if (bkey != kInvalidWord && a.d0 + (int)(bkey & 0xFFFFu) >= 0) {
        const int bdi = (int)(bkey & 0xFFFFu);
        uint32_t smin = kInf;
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int hs = 0; hs < 2; ++hs) {
                const int di = 2 * (j * K + k) + hs;
                const uint32_t v = (sv[k] >> (16 * hs)) & 0xFFFFu;
                if (abs(di - bdi) > 1 && v < smin) smin = v;
            }
        const uint32_t sec = __reduce_min_sync(gmask, smin);
        const int wm = (bdi - 1) >> 1, wp = (bdi + 1) >> 1;
        uint32_t selm = 0, selp = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (j * K + k == wm) selm = sv[k];
            if (j * K + k == wp) selp = sv[k];
        }
        const uint32_t vm_w = __shfl_sync(gmask, selm, bdi >= 1 ? wm / K : 0, T);
        const uint32_t vp_w = __shfl_sync(gmask, selp, wp / K < T ? wp / K : T - 1, T);
        if (j == 0) {
            const uint32_t bv = bkey >> 16;
            dval = (float)(a.d0 + bdi);
            if (a.subpixel && bdi > 0 && bdi + 1 < a.D) {
                const uint32_t cm = (vm_w >> (16 * ((bdi - 1) & 1))) & 0xFFFFu;
                const uint32_t cp = (vp_w >> (16 * ((bdi + 1) & 1))) & 0xFFFFu;
                if (cm < kInf && cp < kInf) {
                    // WTA uniqueness (src/sgm_optimizer.cpp:520-525): (second - best) / max(best, 1)
                    const float u = sec >= kInf ? 1.0f : __fdiv_rn((float)(sec - bv), (float)max(bv, 1u));
                    dval = __fadd_rn(dval, a.sp_tel ? subpixel_delta_tel((float)cm, (float)bv, (float)cp, a.sp_method,
                                                                         a.sp_param, u, a.sp_tel)
                                                    : subpixel_delta((float)cm, (float)bv, (float)cp, a.sp_method,
                                                                     a.sp_param, u));
                }
            }
            fb = (float)bv;
            fs = sec >= kInf ? __int_as_float(0x7f800000) : (float)sec;
        }
    }
    if (j == 0) {
        a.disp[p] = dval;
        a.best[p] = fb;
        a.second[p] = fs;
    }
}


// Sliding census ring: logical entry i (disparity d0 + 2Kj + i) of rotation R lives in register
// (i - R) mod 2K when the row is walked left to right, (i + R) mod 2K right to left.
template <int K, int HDIR>
__device__ __forceinline__ constexpr int ring_idx(int i, int R) {
    return HDIR > 0 ? ((i - R) % (2 * K) + 2 * K) % (2 * K) : (i + R) % (2 * K);
}

// One scanline chain of direction (dx, dy) on this lane group.  MODE kFirst writes the chain's L
// to `out`; MODE kLast adds the NB partial sums of `tab.in`, then runs the WTA.
template <int T, int K, int MODE, bool CENSUS, int HDIR, int PF, int U, int NB>
__device__ __forceinline__ void run_chain(const SgmArgs& a, const DirTable& tab, const uint16_t* s_q, int dx,
                                          int dy, int s, int nscan, uint32_t* out) {
    const int lane = threadIdx.x & 31;
    const int grp = lane / T, j = lane % T;
    const unsigned gmask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << (grp * T));
    int x0, y0, len;
    scan_start(a, dx, dy, s, nscan, x0, y0, len);
    const int maxlen = __reduce_max_sync(0xffffffffu, len);
    if (maxlen == 0) return;
    const int W2 = a.Dp / 2;
    const int step = dy * a.w + dx;
    const int p0 = y0 * a.w + x0;
    const uint32_t p1x2 = (uint32_t)a.pen.P1 * 0x00010001u;
    const int dl0 = a.d0 + 2 * K * j;  // lowest disparity of this lane

    Slot<K, CENSUS, HDIR, NB> ring[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u)
        if (u < len) fetch<K, T, CENSUS, HDIR, NB>(a, tab, j, p0 + u * step, x0 + u * dx, ring[u]);

    // sliding census registers (horizontal census sweeps): descriptors of the first pixel
    uint32_t cw[CENSUS && HDIR != 0 ? 2 * K : 1];
    if (CENSUS && HDIR != 0) {
#pragma unroll
        for (int i = 0; i < 2 * K; ++i) {
            const int xr = x0 - (dl0 + i);
            cw[i] = (len > 0 && xr >= 0 && xr < a.w) ? __ldg(a.cr + y0 * a.w + xr) : 0u;
        }
    }

    uint32_t L[K];
    uint32_t m = kInf;
    int prev_g = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) L[k] = kInf2;

    for (int t0 = 0; t0 < maxlen; t0 += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = t0 + u;
            if (t >= maxlen) break;
            if (t < len) {
                Slot<K, CENSUS, HDIR, NB>& sl = ring[u % PF];
                const int p = p0 + t * step;
                const int x = x0 + t * dx;
                // ---- matching costs of this pixel
                uint32_t c[K];
                if (CENSUS) {
                    // valid disparities: d0 <= d <= min(x, dmax-1) and x - d < w (the default
                    // range [d0, min(dmax, x+1)) of PriorEstimator::estimate)
                    const int dlo = x - a.w + 1, dhi = min(x, a.dmax - 1);
                    const bool all_ok = dl0 >= dlo && dl0 + 2 * K - 1 <= dhi;
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        uint32_t q2[2];
#pragma unroll
                        for (int hs = 0; hs < 2; ++hs) {
                            const int i = 2 * k + hs;
                            const uint32_t desc = HDIR != 0 ? cw[ring_idx<K, HDIR>(i, u % (2 * K))] : sl.c[i];
                            const uint32_t q = s_q[__popc(sl.clv ^ desc)];
                            q2[hs] = (all_ok || (dl0 + i >= dlo && dl0 + i <= dhi)) ? q : kInf;
                        }
                        c[k] = __byte_perm(q2[0], q2[1], 0x5410);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < K; ++k) c[k] = __vminu2(sl.c[k], kInf2);  // 0xFFFF -> 0x7FFF
                }
                // ---- recurrence (process_pixel, src/sgm_optimizer.cpp:44-80)
                if (t == 0 || m >= kInf) {
#pragma unroll
                    for (int k = 0; k < K; ++k) L[k] = c[k];
                } else {
                    const int P2 = adaptive_p2(a.pen, sl.g - prev_g);
                    const uint32_t mp2 = (m + (uint32_t)P2) * 0x00010001u;
                    const uint32_t m2 = m * 0x00010001u;
                    uint32_t up = __shfl_up_sync(gmask, L[K - 1], 1, T);
                    uint32_t dn = __shfl_down_sync(gmask, L[0], 1, T);
                    if (j == 0) up = kInf2;
                    if (j == T - 1) dn = kInf2;
                    uint32_t Ln[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        const uint32_t lo_nb = k == 0 ? up : L[k - 1];
                        const uint32_t hi_nb = k == K - 1 ? dn : L[k + 1];
                        const uint32_t lm = __byte_perm(lo_nb, L[k], 0x5432);  // (L[k] << 16) | (lo_nb >> 16)
                        const uint32_t lp = __byte_perm(L[k], hi_nb, 0x5432);  // (hi_nb << 16) | (L[k] >> 16)
                        const uint32_t b = __vminu2(L[k], __viaddmin_u16x2(__vminu2(lm, lp), p1x2, mp2));
                        Ln[k] = path_value(c[k], b, m2);
                    }
#pragma unroll
                    for (int k = 0; k < K; ++k) L[k] = Ln[k];
                }
                uint32_t mm;
                if constexpr (K == 1) {
                    mm = min_halves(L[0]);
                } else {
                    uint32_t acc = __vminu2(L[0], L[1]);
#pragma unroll
                    for (int k = 2; k < K; k += 2) acc = k + 1 < K ? __vimin3_u16x2(acc, L[k], L[k + 1]) : __vminu2(acc, L[k]);
                    mm = min_halves(acc);
                }
                m = __reduce_min_sync(gmask, mm);
                prev_g = sl.g;
                // ---- path sum
                if (MODE == kFirst) {
                    st_cg<K>(out + (size_t)p * W2 + j * K, L);
                } else {
                    uint32_t sv[K];
#pragma unroll
                    for (int k = 0; k < K; ++k) {
                        uint32_t v = L[k];
#pragma unroll
                        for (int b = 0; b < NB; ++b) v = addus2(v, sl.s[b][k]);
                        sv[k] = v;
                    }
                    if (a.store_final) {
                        uint32_t o[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) o[k] = sv[k] | __vcmpgeu2(sv[k], kInf2);
                        st_cg<K>(const_cast<uint32_t*>(tab.in[0]) + (size_t)p * W2 + j * K, o);
                    }
                    wta<K, T>(a, gmask, j, p, sv);
                }
            }
            // ---- slide the census ring to the next pixel and refill this prefetch slot
            if (CENSUS && HDIR != 0) {
                const int R = u % (2 * K), Rn = (u + 1) % (2 * K);
                // the entry leaving the ring at this step becomes the neighbour's entering entry
                const uint32_t leaving = HDIR > 0 ? cw[ring_idx<K, HDIR>(2 * K - 1, R)] : cw[ring_idx<K, HDIR>(0, R)];
                const uint32_t from_nb = HDIR > 0 ? __shfl_up_sync(gmask, leaving, 1, T) : __shfl_down_sync(gmask, leaving, 1, T);
                if (t + 1 < len) {
                    const bool edge = HDIR > 0 ? (j == 0) : (j == T - 1);
                    const uint32_t entering = edge ? ring[(u + 1) % PF].c[0] : from_nb;
                    if (HDIR > 0) cw[ring_idx<K, HDIR>(0, Rn)] = entering;
                    else cw[ring_idx<K, HDIR>(2 * K - 1, Rn)] = entering;
                }
            }
            {
                const int tn = t + PF;
                if (tn < len) fetch<K, T, CENSUS, HDIR, NB>(a, tab, j, p0 + tn * step, x0 + tn * dx, ring[u % PF]);
            }
        }
    }
}

// ---- volume-fed chains: loads staged through shared memory with cp.async
//
// A register ring cannot keep loads for many future steps independently in flight: completion is
// tracked per warp by a handful of scoreboards, so loads issued for different steps end up waiting
// for one another and each step pays a full HBM latency.  cp.async groups are tracked per step
// instead: step t's group is committed PF steps before use, and cp.async.wait_group(PF-1) waits for
// exactly that group.  Each lane copies its own words into a per-warp ring slot
// [cost: 32 lanes x K][partial sums: NB x 32 x K][gray word: 32], so the reads back are
// conflict-free and need no barrier (a lane reads only what it copied).

__device__ __forceinline__ void cp_async4(uint32_t* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// K words of one lane; the source is 4K-byte aligned (pixel slices are Dp*2 bytes, lanes 4K bytes).
template <int K>
__device__ __forceinline__ void cp_words(uint32_t* dst, const uint32_t* src) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) cp_async16(dst + k, src + k);
    } else if constexpr (K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 2) cp_async8(dst + k, src + k);
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) cp_async4(dst + k, src + k);
    }
}

template <int K>
__device__ __forceinline__ void lds_words(const uint32_t* src, uint32_t (&v)[K]) {
    if constexpr (K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            const uint4 t = *reinterpret_cast<const uint4*>(src + k);
            v[k] = t.x; v[k + 1] = t.y; v[k + 2] = t.z; v[k + 3] = t.w;
        }
    } else if constexpr (K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 2) {
            const uint2 t = *reinterpret_cast<const uint2*>(src + k);
            v[k] = t.x; v[k + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = src[k];
    }
}

template <int K, int NB>
__host__ __device__ constexpr int vol_slot_words() { return (K + NB * K) * 32; }

// Cost words per lane in the volume and in a ring slot: K u16x2 words, or K / 2 words of the byte
// volume.  A lane's words sit together, so a warp's cost loads and reads cover consecutive words.
template <int K, bool C8>
__host__ __device__ constexpr int cost_words() { return C8 ? K / 2 : K; }

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

// The lane's K cost words (u16x2) from its ring slot, the invalid marker clamped to 0x7FFF.  The
// byte volume (C8) widens each byte to a halfword: a byte 0xFF (invalid) gets the high byte 0xFF,
// through prmt's sign-replicating selectors on a word whose bit 7 per byte flags 0xFF, and the
// clamp then gives the same 0x7FFF as the two-byte volume's 0xFFFF.
template <int K, bool C8>
__device__ __forceinline__ void load_costs(const uint32_t* src, uint32_t (&c)[K]) {
    if constexpr (C8) {
        static_assert(K % 2 == 0, "byte volume: an even number of words per lane");
        uint32_t cb[K / 2];
        lds_words<K / 2>(src, cb);
#pragma unroll
        for (int i = 0; i < K / 2; ++i) {
            // per byte b: (~b & 0x7F) + 0x7F has bit 7 set unless the low seven bits of b are all
            // set; with b's own bit 7 that leaves bit 7 set exactly where b == 0xFF
            const uint32_t t = (~cb[i] & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
            const uint32_t inv = ~t & cb[i] & 0x80808080u;
            c[2 * i] = __vminu2(prmt(cb[i], inv, 0xD1C0u), kInf2);      // b0, sign(inv.b0), b1, sign(inv.b1)
            c[2 * i + 1] = __vminu2(prmt(cb[i], inv, 0xF3E2u), kInf2);  // b2, sign(inv.b2), b3, sign(inv.b3)
        }
    } else {
        lds_words<K>(src, c);
#pragma unroll
        for (int k = 0; k < K; ++k) c[k] = __vminu2(c[k], kInf2);  // 0xFFFF -> 0x7FFF
    }
}

// Words per warp of the last sweep's WTA buffer: 32 pixels x (Dp/2 + 1) words (odd row stride, so
// one lane per row reads without bank conflicts).
template <int K, int T>
__host__ __device__ constexpr int wta_buf_words() { return 32 * (K * T + 1); }

// Winner-take-all of one pixel from its final sums, W2 u16x2 words in shared memory, run by one
// lane (wta_impl, src/sgm_optimizer.cpp:465-536): the first minimum, the second minimum outside
// |d - best| <= 1, the legacy parabola.  Sums >= 0x7FFF are invalid.  A negative winning
// disparity reads as "none" like the reference's best_d < 0 test (:490-495).
template <int W2>
__device__ __forceinline__ void wta_row(const SgmArgs& a, const uint32_t* row, int p) {
    // one pass over the row keeps the minimum of each chunk of CS words in registers; the first
    // index and the second minimum then read at most three chunks again
    constexpr int CS = W2 / 16 >= 4 ? W2 / 16 : 4;  // words per chunk (W2 is a multiple of 8)
    constexpr int NC = W2 / CS;
    uint32_t cmin[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        uint32_t v = row[c * CS];
#pragma unroll
        for (int i = 1; i < CS; ++i) v = __vminu2(v, row[c * CS + i]);
        cmin[c] = v;
    }
    uint32_t all = cmin[0];
#pragma unroll
    for (int c = 1; c < NC; ++c) all = __vminu2(all, cmin[c]);
    const uint32_t m = min_halves(all);
    float dval = -1.f, fb = __int_as_float(0x7f800000), fs = __int_as_float(0x7f800000);
    if (m < kInf) {
        // the first chunk whose minimum is m, then the first halfword equal to m inside it
        int fc = 0;
#pragma unroll
        for (int c = NC - 1; c >= 0; --c)
            if (min_halves(cmin[c]) == m) fc = c;
        int bdi = 2 * fc * CS;
        for (int i = 0; i < CS; ++i) {
            const uint32_t v = row[fc * CS + i];
            if ((v & 0xFFFFu) == m) { bdi = 2 * (fc * CS + i); break; }
            if ((v >> 16) == m) { bdi = 2 * (fc * CS + i) + 1; break; }
        }
        if (a.d0 + bdi >= 0) {
            const uint16_t* r16 = reinterpret_cast<const uint16_t*>(row);
            dval = (float)(a.d0 + bdi);
            // second minimum outside |d - best| <= 1: chunks without an excluded halfword keep
            // their minimum; the (at most two) chunks with one are read again with those masked
            const int klo = bdi > 0 ? (bdi - 1) >> 1 : 0, khi = min((bdi + 1) >> 1, W2 - 1);
            const int clo = klo / CS, chi = khi / CS;
            uint32_t sec2 = 0xFFFFFFFFu;
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (c != clo && c != chi) sec2 = __vminu2(sec2, cmin[c]);
            for (int c = clo; c <= chi; ++c) {
                for (int i = 0; i < CS; ++i) {
                    const int k = c * CS + i;
                    uint32_t v = row[k];
                    if (abs(2 * k - bdi) <= 1) v |= 0x0000FFFFu;
                    if (abs(2 * k + 1 - bdi) <= 1) v |= 0xFFFF0000u;
                    sec2 = __vminu2(sec2, v);
                }
            }
            const uint32_t sec = min_halves(sec2);
            if (a.subpixel && bdi > 0 && bdi + 1 < a.D) {
                const uint32_t cm = r16[bdi - 1], cp = r16[bdi + 1];
                if (cm < kInf && cp < kInf) {
                    // WTA uniqueness (src/sgm_optimizer.cpp:520-525): (second - best) / max(best, 1)
                    const float u = sec >= kInf ? 1.0f : __fdiv_rn((float)(sec - m), (float)max(m, 1u));
                    dval = __fadd_rn(dval, a.sp_tel ? subpixel_delta_tel((float)cm, (float)m, (float)cp, a.sp_method,
                                                                         a.sp_param, u, a.sp_tel)
                                                    : subpixel_delta((float)cm, (float)m, (float)cp, a.sp_method,
                                                                     a.sp_param, u));
                }
            }
            fb = (float)m;
            fs = sec >= kInf ? __int_as_float(0x7f800000) : (float)sec;
        }
    }
    a.disp[p] = dval;
    a.best[p] = fb;
    a.second[p] = fs;
}

// One volume-fed scanline chain (same recurrence and WTA as run_chain; loads via cp.async).
// Steps run in blocks of T: at the start of a block lane j loads the gray level of step t0 + j
// (prefetched one block ahead) and computes that step's adaptive P2, so a step costs one shuffle
// for P2 instead of a load and the P2 arithmetic.  Addresses advance by a 32-bit word offset.
//
// BAND: only the steps [a.t_begin, a.t_end) of the chain (t_begin a multiple of T = 32, one chain
// per warp), starting from the L and m a previous band left in a.carry and leaving them there when
// the chain goes on; the steps and the WTA of each step are those of the whole chain.
template <int T, int K, int MODE, int PF, int NB, bool C8 = false, bool BAND = false>
__device__ __forceinline__ void run_chain_vol(const SgmArgs& a, const uint32_t* const* in, uint32_t* s_ring,
                                              uint32_t* s_wta, int dx, int dy, int s, int nscan, uint32_t* out) {
    static_assert((PF & (PF - 1)) == 0 && T % PF == 0, "PF: a power of two dividing T");
    static_assert(!BAND || (T == 32 && MODE == kLast), "bands: the one-warp last sweep");
    constexpr int SW = vol_slot_words<K, NB>();
    const int lane = threadIdx.x & 31;
    const int grp = lane / T, j = lane % T;
    const unsigned gmask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << (grp * T));
    int x0, y0, len;
    scan_start(a, dx, dy, s, nscan, x0, y0, len);
    int tb = 0;             // first step of this launch
    bool carry_out = false;  // the chain goes on after this band
    if constexpr (BAND) {
        tb = a.t_begin;
        carry_out = a.t_end < len;
        len = min(len, a.t_end);
    }
    const int maxlen = __reduce_max_sync(0xffffffffu, len);
    if (maxlen <= tb) return;
    const int W2 = a.Dp / 2;
    const int step = dy * a.w + dx;
    const int p0 = y0 * a.w + x0;
    const uint32_t p1x2 = (uint32_t)a.pen.P1 * 0x00010001u;
    const uint32_t dstep = (uint32_t)(step * W2);  // word offset per step (wraps for negative steps)
    // the cost volume's words: W2 per pixel, or W2 / 2 for the byte volume (K / 2 per lane)
    const uint32_t cstep = C8 ? (uint32_t)(step * (W2 / 2)) : dstep;

    // loads of step t (word offsets off, coff) into slot t % PF; every step commits one group
    auto issue = [&](int t, uint32_t off, uint32_t coff) {
        if (t < len) {
            uint32_t* sl = s_ring + (t & (PF - 1)) * SW;
            cp_words<cost_words<K, C8>()>(sl + lane * cost_words<K, C8>(), a.cvol + coff);
#pragma unroll
            for (int b = 0; b < NB; ++b) cp_words<K>(sl + 32 * K * (1 + b) + lane * K, in[b] + off);
        }
        cp_commit();
    };
    const uint32_t off0 = (uint32_t)p0 * (uint32_t)W2 + (uint32_t)(j * K) + (uint32_t)tb * dstep;
    const uint32_t coff0 =
        C8 ? (uint32_t)p0 * (uint32_t)(W2 / 2) + (uint32_t)(j * (K / 2)) + (uint32_t)tb * cstep : off0;
    uint32_t ioff = off0, icoff = coff0;  // offsets of the next step to issue
#pragma unroll
    for (int t = 0; t < PF; ++t) {
        issue(tb + t, ioff, icoff);
        ioff += dstep;
        icoff += cstep;
    }
    uint32_t off = off0;  // offset of the current step

    uint32_t L[K];
    uint32_t m = kInf;
#pragma unroll
    for (int k = 0; k < K; ++k) L[k] = kInf2;
    int gnext = tb + j < len ? (int)__ldg(a.gray + p0 + (tb + j) * step) : 0;
    int gcarry = 0;
    if constexpr (BAND) {
        if (tb > 0) {
            const uint32_t* cs = a.carry + (size_t)s * (K + 1) * 32 + lane;
#pragma unroll
            for (int k = 0; k < K; ++k) L[k] = __ldcg(cs + k * 32);
            m = __ldcg(cs + K * 32);
            gcarry = (int)__ldg(a.gray + p0 + (tb - 1) * step);
        }
    }

    for (int t0 = tb; t0 < maxlen; t0 += T) {
        // P2 of the steps [t0, t0 + T): lane j holds step t0 + j
        const int gcur = gnext;
        {
            const int tn = t0 + T + j;
            gnext = tn < len ? (int)__ldg(a.gray + p0 + tn * step) : 0;
        }
        int gprev = __shfl_up_sync(gmask, gcur, 1, T);
        if (j == 0) gprev = gcarry;
        gcarry = __shfl_sync(gmask, gcur, T - 1, T);
        const int p2v = adaptive_p2(a.pen, gcur - gprev);

        for (int u0 = 0; u0 < T; u0 += PF) {
            if (t0 + u0 >= maxlen) break;
#pragma unroll
            for (int v = 0; v < PF; ++v) {
                const int t = t0 + u0 + v;
                if (t >= maxlen) break;
                cp_wait<PF - 1>();
                const int P2 = __shfl_sync(gmask, p2v, u0 + v, T);
                if (t < len) {
                    const uint32_t* sl = s_ring + v * SW;
                    uint32_t c[K];
                    load_costs<K, C8>(sl + lane * cost_words<K, C8>(), c);
                    if (t == 0 || m >= kInf) {
#pragma unroll
                        for (int k = 0; k < K; ++k) L[k] = c[k];
                    } else {
                        const uint32_t mp2 = (m + (uint32_t)P2) * 0x00010001u;
                        const uint32_t m2 = m * 0x00010001u;
                        uint32_t up = __shfl_up_sync(gmask, L[K - 1], 1, T);
                        uint32_t dn = __shfl_down_sync(gmask, L[0], 1, T);
                        if (j == 0) up = kInf2;
                        if (j == T - 1) dn = kInf2;
                        uint32_t Ln[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const uint32_t lo_nb = k == 0 ? up : L[k - 1];
                            const uint32_t hi_nb = k == K - 1 ? dn : L[k + 1];
                            const uint32_t lm = __byte_perm(lo_nb, L[k], 0x5432);
                            const uint32_t lp = __byte_perm(L[k], hi_nb, 0x5432);
                            const uint32_t b = __vminu2(L[k], __viaddmin_u16x2(__vminu2(lm, lp), p1x2, mp2));
                            Ln[k] = path_value(c[k], b, m2);
                        }
#pragma unroll
                        for (int k = 0; k < K; ++k) L[k] = Ln[k];
                    }
                    uint32_t mm;
                    if constexpr (K == 1) {
                        mm = min_halves(L[0]);
                    } else {
                        uint32_t acc = __vminu2(L[0], L[1]);
#pragma unroll
                        for (int k = 2; k < K; k += 2)
                            acc = k + 1 < K ? __vimin3_u16x2(acc, L[k], L[k + 1]) : __vminu2(acc, L[k]);
                        mm = min_halves(acc);
                    }
                    m = __reduce_min_sync(gmask, mm);
                    if (MODE == kFirst) {
                        st_cg<K>(out + off, L);
                    } else {
                        uint32_t sv[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) sv[k] = L[k];
#pragma unroll
                        for (int b = 0; b < NB; ++b) {
                            uint32_t sb[K];
                            lds_words<K>(sl + 32 * K * (1 + b) + lane * K, sb);
#pragma unroll
                            for (int k = 0; k < K; ++k) sv[k] = addus2(sv[k], sb[k]);
                        }
                        if (a.store_final) {
                            uint32_t o[K];
#pragma unroll
                            for (int k = 0; k < K; ++k) o[k] = sv[k] | __vcmpgeu2(sv[k], kInf2);
                            st_cg<K>(const_cast<uint32_t*>(in[0]) + off, o);
                        }
                        // final sums of this step's pixel into row (t - t0) of the group's WTA buffer
                        uint32_t* wr = s_wta + grp * T * (K * T + 1) + (u0 + v) * (K * T + 1) + j * K;
#pragma unroll
                        for (int k = 0; k < K; ++k) wr[k] = sv[k];
                    }
                }
                // the slot just read is refilled only after its values were consumed above
                issue(t + PF, ioff, icoff);
                ioff += dstep;
                icoff += cstep;
                off += dstep;
            }
        }
        if (MODE == kLast) {
            // the block's T pixels: lane j of the group runs the WTA of pixel t0 + j of its chain
            __syncwarp();
            if (t0 + j < len)
                wta_row<K * T>(a, s_wta + grp * T * (K * T + 1) + j * (K * T + 1), p0 + (t0 + j) * step);
            __syncwarp();
        }
    }
    if constexpr (BAND) {
        if (carry_out) {
            uint32_t* cs = a.carry + (size_t)s * (K + 1) * 32 + lane;
#pragma unroll
            for (int k = 0; k < K; ++k) __stcg(cs + k * 32, L[k]);
            __stcg(cs + K * 32, m);
        }
    }
    cp_wait<0>();
}

// ---- the last sweep split over two warps of one block
//
// One chain per block of two warps.  Warp 0 runs only the recurrence: its costs come through its
// own cp.async ring, and each step's L goes to a shared-memory ring of kSplitSlots segments of
// kSplitSeg steps.  Warp 1 adds the NB partial sums to each step's L (through its own cp.async
// ring), writes the final sums into the WTA buffer and runs the WTA every 32 steps.  The recurrence
// warp's step is about a third of the instructions of a step that also adds, buffers and
// evaluates the sums, and it shares its SM's issue slots with the other chains' summing warps, so
// the dependent chain of each step is what remains of its time.
//
// Hand-over by named barriers (bar.arrive / bar.sync over the block's 64 threads): warp 0 arrives
// on FULL[s % 2] once segment s is written, warp 1 arrives on FREE[s % 2] once it has read it, and
// each waits for the other's barrier before it touches that slot again.  Both warps walk the same
// number of segments (the block's one chain has one length), so every barrier generation is
// completed by exactly one arrival of each warp, and no warp arrives twice on one barrier before
// the other has passed it.
constexpr int kSplitSlots = 2;
constexpr int kSplitSeg = 8;  // steps per segment (divides the 32-step WTA and P2 blocks)
// Barrier ids are immediates (a register id makes the compiler reserve all sixteen of a block's
// barriers, which capped the SM at four of these blocks); the kernel has no __syncthreads, so ids
// 0..3 are free.
constexpr int kBarFull = 0;   // named barriers 0, 1: segment written
constexpr int kBarFree = 2;   // named barriers 2, 3: segment read

template <int K, int NB, int PFA, int PFB>
struct SplitSmem {
    static constexpr int cring = PFA * 32 * K;                         // warp 0: cost ring
    static constexpr int lseg = kSplitSeg * 32 * K;                    // one segment of L
    static constexpr int lring = kSplitSlots * lseg;
    static constexpr int pring = PFB * NB * 32 * K;                    // warp 1: partial-sum ring
    static constexpr int wta = wta_buf_words<K, 32>();                 // warp 1: final sums
    static constexpr int words = cring + lring + pring + wta;
};

template <int ID>
__device__ __forceinline__ void nbar_sync64() { asm volatile("bar.sync %0, 64;\n" ::"n"(ID) : "memory"); }
template <int ID>
__device__ __forceinline__ void nbar_arrive64() { asm volatile("bar.arrive %0, 64;\n" ::"n"(ID) : "memory"); }
// barrier `base + slot` for a slot of kSplitSlots = 2
template <int BASE>
__device__ __forceinline__ void nbar_sync_slot(int slot) {
    if (slot) nbar_sync64<BASE + 1>();
    else nbar_sync64<BASE>();
}
template <int BASE>
__device__ __forceinline__ void nbar_arrive_slot(int slot) {
    if (slot) nbar_arrive64<BASE + 1>();
    else nbar_arrive64<BASE>();
}

template <int K, int NB, int PFA, int PFB, bool C8 = false>
__global__ void __launch_bounds__(64) sgm_last_split_kernel(SgmArgs a, DirTable tab) {
    static_assert((PFA & (PFA - 1)) == 0 && (PFB & (PFB - 1)) == 0, "ring depths: powers of two");
    using SM = SplitSmem<K, NB, PFA, PFB>;
    extern __shared__ __align__(16) uint32_t s_dyn[];
    uint32_t* s_c = s_dyn;
    uint32_t* s_l = s_c + SM::cring;
    uint32_t* s_p = s_l + SM::lring;
    uint32_t* s_w = s_p + SM::pring;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int x0, y0, len;
    scan_start(a, tab.dx[0], tab.dy[0], blockIdx.x, tab.nscan[0], x0, y0, len);
    if (len == 0) return;  // the whole block (one chain)
    const int W2 = a.Dp / 2;
    const int step = tab.dy[0] * a.w + tab.dx[0];
    const int p0 = y0 * a.w + x0;
    const uint32_t dstep = (uint32_t)(step * W2);
    const uint32_t off0 = (uint32_t)p0 * (uint32_t)W2 + (uint32_t)(lane * K);
    const int nseg = (len + kSplitSeg - 1) / kSplitSeg;

    if (warp == 0) {
        // ---- the recurrence (process_pixel, src/sgm_optimizer.cpp:44-80); the byte volume (C8)
        // has K / 2 words per lane and W2 / 2 per pixel
        auto issue = [&](int t, uint32_t off) {
            if (t < len)
                cp_words<cost_words<K, C8>()>(s_c + (t & (PFA - 1)) * 32 * K + lane * cost_words<K, C8>(), a.cvol + off);
            cp_commit();
        };
        const uint32_t cstep = C8 ? (uint32_t)(step * (W2 / 2)) : dstep;
        uint32_t ioff = C8 ? (uint32_t)p0 * (uint32_t)(W2 / 2) + (uint32_t)(lane * (K / 2)) : off0;
#pragma unroll
        for (int t = 0; t < PFA; ++t) {
            issue(t, ioff);
            ioff += cstep;
        }
        const uint32_t p1x2 = (uint32_t)a.pen.P1 * 0x00010001u;
        uint32_t L[K];
        uint32_t m = kInf;
#pragma unroll
        for (int k = 0; k < K; ++k) L[k] = kInf2;
        int gnext = lane < len ? (int)__ldg(a.gray + p0 + lane * step) : 0;
        int gcarry = 0, p2v = 0;
        for (int seg = 0; seg < nseg; ++seg) {
            if (seg >= kSplitSlots) nbar_sync_slot<kBarFree>(seg % kSplitSlots);
            uint32_t* lslot = s_l + (seg % kSplitSlots) * SM::lseg;
#pragma unroll
            for (int v = 0; v < kSplitSeg; ++v) {
                const int t = seg * kSplitSeg + v;
                if (t < len) {
                    if ((t & 31) == 0) {
                        // P2 of the steps [t, t + 32): lane j holds step t + j
                        const int gcur = gnext;
                        const int tn = t + 32 + lane;
                        gnext = tn < len ? (int)__ldg(a.gray + p0 + tn * step) : 0;
                        int gprev = __shfl_up_sync(0xffffffffu, gcur, 1);
                        if (lane == 0) gprev = gcarry;
                        gcarry = __shfl_sync(0xffffffffu, gcur, 31);
                        p2v = adaptive_p2(a.pen, gcur - gprev);
                    }
                    cp_wait<PFA - 1>();
                    const int P2 = __shfl_sync(0xffffffffu, p2v, t & 31);
                    uint32_t c[K];
                    load_costs<K, C8>(s_c + (t & (PFA - 1)) * 32 * K + lane * cost_words<K, C8>(), c);
                    if (t == 0 || m >= kInf) {
#pragma unroll
                        for (int k = 0; k < K; ++k) L[k] = c[k];
                    } else {
                        const uint32_t mp2 = (m + (uint32_t)P2) * 0x00010001u;
                        const uint32_t m2 = m * 0x00010001u;
                        uint32_t up = __shfl_up_sync(0xffffffffu, L[K - 1], 1);
                        uint32_t dn = __shfl_down_sync(0xffffffffu, L[0], 1);
                        if (lane == 0) up = kInf2;
                        if (lane == 31) dn = kInf2;
                        uint32_t Ln[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const uint32_t lo_nb = k == 0 ? up : L[k - 1];
                            const uint32_t hi_nb = k == K - 1 ? dn : L[k + 1];
                            const uint32_t lm = __byte_perm(lo_nb, L[k], 0x5432);
                            const uint32_t lp = __byte_perm(L[k], hi_nb, 0x5432);
                            const uint32_t b = __vminu2(L[k], __viaddmin_u16x2(__vminu2(lm, lp), p1x2, mp2));
                            Ln[k] = path_value(c[k], b, m2);
                        }
#pragma unroll
                        for (int k = 0; k < K; ++k) L[k] = Ln[k];
                    }
                    uint32_t mm;
                    if constexpr (K == 1) {
                        mm = min_halves(L[0]);
                    } else {
                        uint32_t acc = __vminu2(L[0], L[1]);
#pragma unroll
                        for (int k = 2; k < K; k += 2)
                            acc = k + 1 < K ? __vimin3_u16x2(acc, L[k], L[k + 1]) : __vminu2(acc, L[k]);
                        mm = min_halves(acc);
                    }
                    m = __reduce_min_sync(0xffffffffu, mm);
                    uint32_t* dst = lslot + v * 32 * K + lane * K;
#pragma unroll
                    for (int k = 0; k < K; ++k) dst[k] = L[k];
                    // the cost slot just read is refilled only after its words were consumed above
                    issue(t + PFA, ioff);
                    ioff += cstep;
                }
            }
            __threadfence_block();
            nbar_arrive_slot<kBarFull>(seg % kSplitSlots);
        }
        cp_wait<0>();
    } else {
        // ---- partial sums, final sums, WTA (wta_impl, src/sgm_optimizer.cpp:465-536)
        constexpr int PW = NB * 32 * K;  // words per partial-ring slot
        auto issue = [&](int t, uint32_t off) {
            if (t < len) {
                uint32_t* sl = s_p + (t & (PFB - 1)) * PW;
#pragma unroll
                for (int b = 0; b < NB; ++b) cp_words<K>(sl + 32 * K * b + lane * K, tab.in[b] + off);
            }
            cp_commit();
        };
        uint32_t ioff = off0, off = off0;
#pragma unroll
        for (int t = 0; t < PFB; ++t) {
            issue(t, ioff);
            ioff += dstep;
        }
        for (int seg = 0; seg < nseg; ++seg) {
            nbar_sync_slot<kBarFull>(seg % kSplitSlots);
            const uint32_t* lslot = s_l + (seg % kSplitSlots) * SM::lseg;
#pragma unroll
            for (int v = 0; v < kSplitSeg; ++v) {
                const int t = seg * kSplitSeg + v;
                if (t < len) {
                    cp_wait<PFB - 1>();
                    uint32_t sv[K];
                    lds_words<K>(lslot + v * 32 * K + lane * K, sv);
                    const uint32_t* sl = s_p + (t & (PFB - 1)) * PW;
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        uint32_t sb[K];
                        lds_words<K>(sl + 32 * K * b + lane * K, sb);
#pragma unroll
                        for (int k = 0; k < K; ++k) sv[k] = addus2(sv[k], sb[k]);
                    }
                    if (a.store_final) {
                        uint32_t o[K];
#pragma unroll
                        for (int k = 0; k < K; ++k) o[k] = sv[k] | __vcmpgeu2(sv[k], kInf2);
                        st_cg<K>(const_cast<uint32_t*>(tab.in[0]) + off, o);
                    }
                    uint32_t* wr = s_w + (t & 31) * (32 * K + 1) + lane * K;
#pragma unroll
                    for (int k = 0; k < K; ++k) wr[k] = sv[k];
                    // the partial slot just read is refilled only after its words were consumed
                    issue(t + PFB, ioff);
                    ioff += dstep;
                    off += dstep;
                    if ((t & 31) == 31 || t == len - 1) {
                        // the block's pixels [t0, t]: lane j runs the WTA of pixel t0 + j
                        const int t0 = t & ~31;
                        __syncwarp();
                        if (t0 + lane <= t) wta_row<32 * K>(a, s_w + lane * (32 * K + 1), p0 + (t0 + lane) * step);
                        __syncwarp();
                    }
                }
            }
            __threadfence_block();
            if (seg + kSplitSlots < nseg) nbar_arrive_slot<kBarFree>(seg % kSplitSlots);
        }
        cp_wait<0>();
    }
}

// Prefetch depth PF (steps of loads in flight per chain) and unroll U (a multiple of PF, so ring
// slots are compile-time registers; the sliding census ring also needs a multiple of 2K).  A
// volume-fed sweep has few chains per SM, so it keeps many steps in flight to cover the HBM
// latency under load; the census-fed sweeps load little per step.
#ifndef APGCU_SGM_PF_VOLUME_FIRST
#define APGCU_SGM_PF_VOLUME_FIRST 8  // 16 measured 2% faster per launch, but 27% slower Fast 720p steps beside the side stream's finalize
#endif
#ifndef APGCU_SGM_PF_VOLUME_LAST
#define APGCU_SGM_PF_VOLUME_LAST 8
#endif
#ifndef APGCU_SGM_PF_CENSUS
#define APGCU_SGM_PF_CENSUS 4
#endif
constexpr int kVolPfFirst = APGCU_SGM_PF_VOLUME_FIRST;
constexpr int kVolPfLast = APGCU_SGM_PF_VOLUME_LAST;
// Ring depth of the first phase: the configured depth, at most T (the P2 block of T steps is
// walked in ring-sized pieces).
template <int T>
__host__ __device__ constexpr int first_pf() {
    return kVolPfFirst < T ? kVolPfFirst : T;
}
// Ring depth of the last sweep: the configured depth (at most T) while a warp's ring and WTA buffer
// stay within 17 KB of shared memory (about thirteen chains per SM), else 4 (large disparity
// ranges; the sweep's time does not depend on the depth between 4 and 8, occupancy does).
template <int K, int T, int NB>
__host__ __device__ constexpr int last_pf() {
    constexpr int pf = kVolPfLast < T ? kVolPfLast : T;
    return (pf * vol_slot_words<K, NB>() + wta_buf_words<K, T>()) * 4 <= 17 * 1024 ? pf : (T < 4 ? T : 4);
}

constexpr int multiple_of_both(int pf, int k2) {
    int u = pf;
    while (u % k2) u += pf;
    return u;
}
template <int K, bool CENSUS, int HDIR, int MODE>
struct Unroll {
    static constexpr int PF0 = CENSUS ? APGCU_SGM_PF_CENSUS
                                      : (MODE == kFirst ? APGCU_SGM_PF_VOLUME_FIRST : APGCU_SGM_PF_VOLUME_LAST);
    static constexpr int PF = (CENSUS && HDIR != 0 && multiple_of_both(PF0, 2 * K) > 16) ? 4 : PF0;
    static constexpr int U = (CENSUS && HDIR != 0) ? multiple_of_both(PF, 2 * K) : PF;
};

__device__ __forceinline__ int find_dir(const DirTable& tab, int warp) {
    int d = 0;
#pragma unroll
    for (int i = 1; i < kMaxDirs; ++i)
        if (i < tab.n && warp >= tab.warp_begin[i]) d = i;
    return d;
}

// First phase: every direction of the table at once, each chain writing its own sum buffer.
template <int T, int K, bool CENSUS, bool C8 = false>
__global__ void __launch_bounds__(128) sgm_first_kernel(SgmArgs a, DirTable tab) {
    __shared__ uint16_t s_q[65];
    if (CENSUS) {
        for (int i = threadIdx.x; i < 65; i += blockDim.x) s_q[i] = a.qlut[i];
        __syncthreads();
    }
    constexpr int C = 32 / T;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= tab.warp_begin[tab.n]) return;
    const int d = find_dir(tab, warp);
    const int dx = tab.dx[d], dy = tab.dy[d];
    const int s = (warp - tab.warp_begin[d]) * C + (threadIdx.x & 31) / T;
    if constexpr (!CENSUS) {
        extern __shared__ __align__(16) uint32_t s_dyn[];
        uint32_t* ring = s_dyn + (threadIdx.x >> 5) * first_pf<T>() * vol_slot_words<K, 0>();
        run_chain_vol<T, K, kFirst, first_pf<T>(), 0, C8>(a, tab.in, ring, nullptr, dx, dy, s, tab.nscan[d], tab.out[d]);
        return;
    }
    if (CENSUS && dy == 0) {
        if (dx > 0) {
            using UR = Unroll<K, true, 1, kFirst>;
            run_chain<T, K, kFirst, true, 1, UR::PF, UR::U, 0>(a, tab, s_q, dx, dy, s, tab.nscan[d], tab.out[d]);
        } else {
            using UR = Unroll<K, true, -1, kFirst>;
            run_chain<T, K, kFirst, true, -1, UR::PF, UR::U, 0>(a, tab, s_q, dx, dy, s, tab.nscan[d], tab.out[d]);
        }
    } else {
        using UR = Unroll<K, CENSUS, 0, kFirst>;
        run_chain<T, K, kFirst, CENSUS, 0, UR::PF, UR::U, 0>(a, tab, s_q, dx, dy, s, tab.nscan[d], tab.out[d]);
    }
}

// Last sweep (one direction): add the NB partial sums and run the WTA.
template <int T, int K, bool CENSUS, int NB, bool C8 = false, bool BAND = false>
__global__ void __launch_bounds__(128) sgm_last_kernel(SgmArgs a, DirTable tab) {
    __shared__ uint16_t s_q[65];
    if (CENSUS) {
        for (int i = threadIdx.x; i < 65; i += blockDim.x) s_q[i] = a.qlut[i];
        __syncthreads();
    }
    constexpr int C = 32 / T;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int s = warp * C + (threadIdx.x & 31) / T;
    if constexpr (!CENSUS) {
        extern __shared__ __align__(16) uint32_t s_dyn[];
        constexpr int PF = last_pf<K, T, NB>();
        constexpr int per_warp = PF * vol_slot_words<K, NB>() + wta_buf_words<K, T>();
        uint32_t* ring = s_dyn + (threadIdx.x >> 5) * per_warp;
        run_chain_vol<T, K, kLast, PF, NB, C8, BAND>(a, tab.in, ring, ring + PF * vol_slot_words<K, NB>(), tab.dx[0],
                                                 tab.dy[0], s, tab.nscan[0], nullptr);
        return;
    }
    using UR = Unroll<K, CENSUS, 0, kLast>;
    run_chain<T, K, kLast, CENSUS, 0, UR::PF, UR::U, NB>(a, tab, s_q, tab.dx[0], tab.dy[0], s, tab.nscan[0], nullptr);
}

// Path8: fold the first NBUF first-phase buffers into the first one (saturating per halfword).
struct FoldSrc {
    const uint4* b[6];
};
template <int NBUF>
__global__ void sgm_sum_kernel(uint4* __restrict__ dst, FoldSrc src, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint4 v = __ldcg(dst + i);
#pragma unroll
        for (int b = 0; b < NBUF - 1; ++b) {
            const uint4 t = __ldcs(src.b[b] + i);
            v.x = addus2(v.x, t.x); v.y = addus2(v.y, t.y);
            v.z = addus2(v.z, t.z); v.w = addus2(v.w, t.w);
        }
        __stcg(dst + i, v);
    }
}

int nscan_of(const SgmArgs& a, int dx, int dy) {
    if (dy == 0) return a.h;
    if (dx == 0) return a.w;
    return a.w + a.h - 1;
}

template <int T, int K>
cudaError_t launch_first_tk(const SgmArgs& a, DirTable tab, bool census, cudaStream_t st) {
    constexpr int C = 32 / T;
    tab.warp_begin[0] = 0;
    for (int i = 0; i < tab.n; ++i) {
        tab.nscan[i] = nscan_of(a, tab.dx[i], tab.dy[i]);
        tab.warp_begin[i + 1] = tab.warp_begin[i] + (tab.nscan[i] + C - 1) / C;
    }
    const int blocks = (tab.warp_begin[tab.n] + 3) / 4;
    if (census) {
        sgm_first_kernel<T, K, true><<<blocks, 128, 0, st>>>(a, tab);
    } else {
        // one warp per block: chains of different lengths (directions) end independently
        const size_t smem = (size_t)first_pf<T>() * vol_slot_words<K, 0>() * 4;
        auto kern = sgm_first_kernel<T, K, false>;
        if (a.cost8) {
            if constexpr (T == 32 && K % 2 == 0) kern = sgm_first_kernel<T, K, false, true>;
            else return cudaErrorInvalidValue;
        }
        {
            const cudaError_t e = allow_dynamic_smem(kern, smem);
            if (e != cudaSuccess) return e;
        }
        kern<<<tab.warp_begin[tab.n], 32, smem, st>>>(a, tab);
    }
    return cudaGetLastError();
}

// Whether the volume-fed last sweep runs split over two warps per chain: on request, else for 64
// padded disparities.  Measured at 20 steps (one B200, last-sweep launch): 640x480 D64 0.111 vs
// 0.142 ms split / one warp; 1280x720 D128 0.275 vs 0.272; 1242x375 D192 0.401 vs 0.201 (wider
// ranges need more shared memory per chain than the split saves).
bool use_split(int T, int K, bool census, int split) {
    if (T != 32 || census || split == 1) return false;
    return split == 2 || K == 1;
}

template <int K, int NB>
cudaError_t launch_last_split(const SgmArgs& a, const DirTable& tab, cudaStream_t st) {
    constexpr int PFA = 8;
    constexpr int PFB = K <= 2 ? 8 : 4;
    const size_t smem = (size_t)SplitSmem<K, NB, PFA, PFB>::words * 4;
    auto kern = sgm_last_split_kernel<K, NB, PFA, PFB>;
    if (a.cost8) {
        if constexpr (K % 2 == 0) kern = sgm_last_split_kernel<K, NB, PFA, PFB, true>;
        else return cudaErrorInvalidValue;
    }
    cudaError_t e = allow_dynamic_smem(kern, smem);
    if (e != cudaSuccess) return e;
    // as many chains per SM as shared memory holds: ask for the largest shared-memory carveout
    // (a hint the driver otherwise sizes to other limits)
    if (cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
        cudaSuccess)
        cudaGetLastError();
    kern<<<tab.nscan[0], 64, smem, st>>>(a, tab);
    return cudaGetLastError();
}

template <int T, int K>
cudaError_t launch_last_tk(const SgmArgs& a, DirTable tab, bool census, int split, cudaStream_t st) {
    constexpr int C = 32 / T;
    tab.nscan[0] = nscan_of(a, tab.dx[0], tab.dy[0]);
    const int warps = (tab.nscan[0] + C - 1) / C;
    const int blocks = (warps + 3) / 4;
    if constexpr (T == 32) {
        if (use_split(T, K, census, split)) {
            if (tab.nin == 1) return launch_last_split<K, 1>(a, tab, st);
            if (tab.nin == 3) return launch_last_split<K, 3>(a, tab, st);
            return cudaErrorInvalidValue;
        }
    }
#define APGCU_LAST(NB)                                                                               \
    if (tab.nin == NB) {                                                                             \
        if (census) {                                                                                \
            sgm_last_kernel<T, K, true, NB><<<blocks, 128, 0, st>>>(a, tab);                         \
        } else {                                                                                     \
            /* one warp per block: shared memory is granted per chain, not per four */              \
            const size_t smem = (size_t)(last_pf<K, T, NB>() * vol_slot_words<K, NB>() + wta_buf_words<K, T>()) * 4; \
            auto kern = sgm_last_kernel<T, K, false, NB>;                                            \
            if (a.cost8) {                                                                           \
                if constexpr (T == 32 && K % 2 == 0) kern = sgm_last_kernel<T, K, false, NB, true>;  \
                else return cudaErrorInvalidValue;                                                   \
            }                                                                                        \
            {                                                                                        \
                const cudaError_t e = allow_dynamic_smem(kern, smem);                                \
                if (e != cudaSuccess) return e;                                                      \
            }                                                                                        \
            kern<<<warps, 32, smem, st>>>(a, tab);                                                   \
        }                                                                                            \
        return cudaGetLastError();                                                                   \
    }
    APGCU_LAST(1)
    APGCU_LAST(3)
#undef APGCU_LAST
    return cudaErrorInvalidValue;
}

template <bool FIRST>
cudaError_t dispatch(const SgmArgs& a, const DirTable& tab, bool census, int T, int split, cudaStream_t st) {
#define APGCU_TK(TT, KK) return FIRST ? launch_first_tk<TT, KK>(a, tab, census, st) : launch_last_tk<TT, KK>(a, tab, census, split, st)
    if (T == 8) {
        if (a.Dp == 64) APGCU_TK(8, 4);
        if (a.Dp == 128) APGCU_TK(8, 8);
        return cudaErrorInvalidValue;
    }
    if (T == 16) {
        switch (a.Dp / 32) {
            case 2: APGCU_TK(16, 2);
            case 4: APGCU_TK(16, 4);
            case 6: APGCU_TK(16, 6);
            case 8: APGCU_TK(16, 8);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (a.Dp / 64) {
        case 1: APGCU_TK(32, 1);
        case 2: APGCU_TK(32, 2);
        case 3: APGCU_TK(32, 3);
        case 4: APGCU_TK(32, 4);
        case 5: APGCU_TK(32, 5);
        case 6: APGCU_TK(32, 6);
        case 7: APGCU_TK(32, 7);
        case 8: APGCU_TK(32, 8);
        default: return cudaErrorInvalidValue;
    }
#undef APGCU_TK
}

// ---- batches: the chains of many pairs in one persistent launch
//
// A launch covers one phase (the first-phase directions, or the last sweep) of every pair of a
// batch with the same Dp.  Its work queue is the list of warp units: a unit is 32/T consecutive
// scanlines of one (pair, direction) segment; segments are ordered longest chains first, so the
// tail of the launch is short.  Warps take units from a global counter until the queue is empty.
struct BatchPair {
    SgmArgs a;
    uint32_t* out[kMaxDirs];       // first phase: one path-sum buffer per direction
    const uint32_t* in[kMaxDirs];  // last sweep: the partial sums to add
};
struct BatchSeg {
    int begin;  // first unit of the segment
    int pair, dir, dx, dy, nscan;
};

template <int T, int K, int MODE, int PF, int NB>
__global__ void __launch_bounds__(128) sgm_batch_kernel(const BatchPair* __restrict__ pairs,
                                                        const BatchSeg* __restrict__ segs, int nseg, int total,
                                                        int* __restrict__ queue) {
    extern __shared__ __align__(16) uint32_t s_dyn[];
    constexpr int ring_words = PF * vol_slot_words<K, NB>();
    constexpr int per_warp = ring_words + (MODE == kLast ? wta_buf_words<K, T>() : 0);
    BatchSeg* s_seg = reinterpret_cast<BatchSeg*>(s_dyn + 4 * per_warp);
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) s_seg[i] = segs[i];
    __syncthreads();
    uint32_t* ring = s_dyn + (threadIdx.x >> 5) * per_warp;
    const int lane = threadIdx.x & 31;
    constexpr int C = 32 / T;
    for (;;) {
        int unit = 0;
        if (lane == 0) unit = atomicAdd(queue, 1);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= total) break;
        int lo = 0, hi = nseg - 1;  // the last segment whose first unit is <= unit
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_seg[mid].begin <= unit) lo = mid;
            else hi = mid - 1;
        }
        const BatchSeg sg = s_seg[lo];
        const BatchPair* bp = pairs + sg.pair;
        // private copies: the chain stores through pointers, and arguments read through a global
        // reference would have to be reloaded after every store
        const SgmArgs a = bp->a;
        const uint32_t* in[NB > 0 ? NB : 1];
#pragma unroll
        for (int b = 0; b < NB; ++b) in[b] = bp->in[b];
        uint32_t* out = MODE == kFirst ? bp->out[sg.dir] : nullptr;
        const int scan = (unit - sg.begin) * C + lane / T;
        run_chain_vol<T, K, MODE, PF, NB>(a, in, ring, ring + ring_words, sg.dx, sg.dy, scan, sg.nscan, out);
    }
}

// Pairs of different padded ranges in one launch (32 lanes per chain): a warp's unit names its
// pair, and the chain runs with that pair's words per lane K = Dp / 64 (up to KMAX).  Each warp's
// shared-memory region holds the largest ring (and WTA buffer) any K of the launch needs.
template <int K, int MODE, int NB>
__host__ __device__ constexpr int mixed_pf() {
    return MODE == kFirst ? first_pf<32>() : last_pf<K, 32, NB>();
}
template <int K, int MODE, int NB>
__host__ __device__ constexpr int mixed_ring_words() {
    return mixed_pf<K, MODE, NB>() * vol_slot_words<K, NB>();
}
template <int K, int MODE, int NB>
__host__ __device__ constexpr int mixed_warp_words() {
    return mixed_ring_words<K, MODE, NB>() + (MODE == kLast ? wta_buf_words<K, 32>() : 0);
}
template <int KMAX, int MODE, int NB>
__host__ __device__ constexpr int mixed_region_words() {
    int m = 0;
    if (KMAX >= 1 && mixed_warp_words<1, MODE, NB>() > m) m = mixed_warp_words<1, MODE, NB>();
    if (KMAX >= 2 && mixed_warp_words<2, MODE, NB>() > m) m = mixed_warp_words<2, MODE, NB>();
    if (KMAX >= 3 && mixed_warp_words<3, MODE, NB>() > m) m = mixed_warp_words<3, MODE, NB>();
    if (KMAX >= 4 && mixed_warp_words<4, MODE, NB>() > m) m = mixed_warp_words<4, MODE, NB>();
    return m;
}

template <int K, int MODE, int NB>
__device__ __forceinline__ void run_mixed_unit(const SgmArgs& a, const uint32_t* const* in, uint32_t* region,
                                               const BatchSeg& sg, int scan, uint32_t* out) {
    run_chain_vol<32, K, MODE, mixed_pf<K, MODE, NB>(), NB>(a, in, region, region + mixed_ring_words<K, MODE, NB>(),
                                                            sg.dx, sg.dy, scan, sg.nscan, out);
}

template <int KMAX, int MODE, int NB>
__global__ void __launch_bounds__(128) sgm_batch_mixed_kernel(const BatchPair* __restrict__ pairs,
                                                              const BatchSeg* __restrict__ segs, int nseg, int total,
                                                              int* __restrict__ queue) {
    extern __shared__ __align__(16) uint32_t s_dyn[];
    constexpr int per_warp = mixed_region_words<KMAX, MODE, NB>();
    BatchSeg* s_seg = reinterpret_cast<BatchSeg*>(s_dyn + 4 * per_warp);
    for (int i = threadIdx.x; i < nseg; i += blockDim.x) s_seg[i] = segs[i];
    __syncthreads();
    uint32_t* region = s_dyn + (threadIdx.x >> 5) * per_warp;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int unit = 0;
        if (lane == 0) unit = atomicAdd(queue, 1);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= total) break;
        int lo = 0, hi = nseg - 1;  // the last segment whose first unit is <= unit
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_seg[mid].begin <= unit) lo = mid;
            else hi = mid - 1;
        }
        const BatchSeg sg = s_seg[lo];
        const BatchPair* bp = pairs + sg.pair;
        const SgmArgs a = bp->a;
        const uint32_t* in[NB > 0 ? NB : 1];
#pragma unroll
        for (int b = 0; b < NB; ++b) in[b] = bp->in[b];
        uint32_t* out = MODE == kFirst ? bp->out[sg.dir] : nullptr;
        const int scan = unit - sg.begin;  // one scanline per unit (32 lanes per chain)
        switch (a.Dp >> 6) {
            case 1: run_mixed_unit<1, MODE, NB>(a, in, region, sg, scan, out); break;
            case 2: if constexpr (KMAX >= 2) run_mixed_unit<2, MODE, NB>(a, in, region, sg, scan, out); break;
            case 3: if constexpr (KMAX >= 3) run_mixed_unit<3, MODE, NB>(a, in, region, sg, scan, out); break;
            default: if constexpr (KMAX >= 4) run_mixed_unit<4, MODE, NB>(a, in, region, sg, scan, out); break;
        }
    }
}

template <int KMAX, int MODE, int NB>
cudaError_t launch_batch_mixed_k(const BatchPair* pairs, const BatchSeg* segs, int nseg, int total, int* queue,
                                 int max_blocks_per_sm, cudaStream_t st) {
    auto kern = sgm_batch_mixed_kernel<KMAX, MODE, NB>;
    const size_t smem = (size_t)4 * mixed_region_words<KMAX, MODE, NB>() * 4 + (size_t)nseg * sizeof(BatchSeg);
    {
        const cudaError_t e = allow_dynamic_smem(kern, smem);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    if (max_blocks_per_sm > 0 && occ > max_blocks_per_sm) occ = max_blocks_per_sm;
    int blocks = nsm * occ;
    const int need = (total + 3) / 4;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    kern<<<blocks, 128, smem, st>>>(pairs, segs, nseg, total, queue);
    return cudaGetLastError();
}

template <int MODE, int NB>
cudaError_t launch_batch_mixed(int Dp_max, const BatchPair* pairs, const BatchSeg* segs, int nseg, int total,
                               int* queue, int max_blocks_per_sm, cudaStream_t st) {
    switch (Dp_max >> 6) {
        case 1: return launch_batch_mixed_k<1, MODE, NB>(pairs, segs, nseg, total, queue, max_blocks_per_sm, st);
        case 2: return launch_batch_mixed_k<2, MODE, NB>(pairs, segs, nseg, total, queue, max_blocks_per_sm, st);
        case 3: return launch_batch_mixed_k<3, MODE, NB>(pairs, segs, nseg, total, queue, max_blocks_per_sm, st);
        case 4: return launch_batch_mixed_k<4, MODE, NB>(pairs, segs, nseg, total, queue, max_blocks_per_sm, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int T, int K, int MODE, int NB>
constexpr int batch_pf() {
    return MODE == kFirst ? first_pf<T>() : last_pf<K, T, NB>();
}

template <int T, int K, int MODE, int NB>
size_t batch_smem(int nseg) {
    constexpr int PF = batch_pf<T, K, MODE, NB>();
    constexpr int per_warp = PF * vol_slot_words<K, NB>() + (MODE == kLast ? wta_buf_words<K, T>() : 0);
    return (size_t)4 * per_warp * 4 + (size_t)nseg * sizeof(BatchSeg);
}

template <int T, int K, int MODE, int NB>
cudaError_t launch_batch_tk(const BatchPair* pairs, const BatchSeg* segs, int nseg, int total, int* queue,
                            int max_blocks_per_sm, cudaStream_t st) {
    constexpr int PF = batch_pf<T, K, MODE, NB>();
    auto kern = sgm_batch_kernel<T, K, MODE, PF, NB>;
    const size_t smem = batch_smem<T, K, MODE, NB>(nseg);
    {
        const cudaError_t e = allow_dynamic_smem(kern, smem);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 128, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    if (max_blocks_per_sm > 0 && occ > max_blocks_per_sm) occ = max_blocks_per_sm;
    int blocks = nsm * occ;
    const int need = (total + 3) / 4;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    kern<<<blocks, 128, smem, st>>>(pairs, segs, nseg, total, queue);
    return cudaGetLastError();
}

template <int MODE, int NB>
cudaError_t launch_batch_dispatch(int T, int Dp, const BatchPair* pairs, const BatchSeg* segs, int nseg, int total,
                                  int* queue, int max_blocks_per_sm, cudaStream_t st) {
#define APGCU_BTK(TT, KK) \
    return launch_batch_tk<TT, KK, MODE, NB>(pairs, segs, nseg, total, queue, max_blocks_per_sm, st)
    if (T == 16) {
        switch (Dp) {
            case 64: APGCU_BTK(16, 2);
            case 128: APGCU_BTK(16, 4);
            case 192: APGCU_BTK(16, 6);
            case 256: APGCU_BTK(16, 8);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (Dp) {
        case 64: APGCU_BTK(32, 1);
        case 128: APGCU_BTK(32, 2);
        case 192: APGCU_BTK(32, 3);
        case 256: APGCU_BTK(32, 4);
        default: return cudaErrorInvalidValue;
    }
#undef APGCU_BTK
}

SgmArgs make_args(const SgmLaunch& l) {
    SgmArgs a;
    a.w = l.w; a.h = l.h; a.d0 = l.d0; a.D = l.D; a.Dp = l.Dp; a.dmax = l.d0 + l.D;
    a.pen = l.pen; a.gray = l.gray; a.cvol = l.cvol; a.cl = l.cl; a.cr = l.cr; a.qlut = l.qlut;
    a.disp = l.disp; a.best = l.best; a.second = l.second;
    a.subpixel = l.subpixel;
    a.sp_method = l.sp_method;
    a.sp_param = l.sp_param;
    a.sp_tel = l.sp_tel;
    a.store_final = l.store_final;
    a.cost8 = l.cost8;
    a.t_begin = 0;
    a.t_end = 0x7FFFFFFF;
    a.carry = nullptr;
    return a;
}

}  // namespace

int sgm_lanes_for(int Dp, int requested) {
    // lanes per chain: 32 by default (one warp per chain, K = Dp/64 words per lane): the sweeps are
    // bound by the serial recurrence, and a full warp per chain halves each step's dependent
    // instruction count against 16 lanes (measured 1.9 vs 2.6 ms per 720p pair at D 128); 16 or
    // 8 (Dp 64 / 128 only) on request
    if (requested == 8 && (Dp == 64 || Dp == 128)) return 8;
    if (requested == 16 && Dp <= 256) return 16;
    return 32;
}

cudaError_t launch_sgm_first(const SgmLaunch& l, int ndir, const int (*dirs)[2], uint32_t* const* out,
                             cudaStream_t st) {
    if (ndir < 1 || ndir > kMaxDirs) return cudaErrorInvalidValue;
    const SgmArgs a = make_args(l);
    DirTable tab = {};
    tab.n = ndir;
    for (int i = 0; i < ndir; ++i) {
        tab.dx[i] = dirs[i][0];
        tab.dy[i] = dirs[i][1];
        tab.out[i] = out[i];
    }
    return dispatch<true>(a, tab, l.cvol == nullptr, sgm_lanes_for(l.Dp, l.lanes), l.split, st);
}

cudaError_t launch_sgm_last(const SgmLaunch& l, int dx, int dy, int nin, const uint32_t* const* in,
                            cudaStream_t st) {
    if (nin < 1 || nin > kMaxDirs) return cudaErrorInvalidValue;
    const SgmArgs a = make_args(l);
    DirTable tab = {};
    tab.n = 1;
    tab.dx[0] = dx;
    tab.dy[0] = dy;
    tab.nin = nin;
    for (int i = 0; i < nin; ++i) tab.in[i] = in[i];
    return dispatch<false>(a, tab, l.cvol == nullptr, sgm_lanes_for(l.Dp, l.lanes), l.split, st);
}

// ---- the last sweep in bands of steps (the host-output path copies each band's rows out while
// the next band runs)

namespace {
template <int K, bool C8>
cudaError_t launch_last_band_k(const SgmArgs& a, DirTable tab, cudaStream_t st) {
    constexpr int NB = 3;
    tab.nscan[0] = nscan_of(a, tab.dx[0], tab.dy[0]);
    const size_t smem = (size_t)(last_pf<K, 32, NB>() * vol_slot_words<K, NB>() + wta_buf_words<K, 32>()) * 4;
    auto kern = sgm_last_kernel<32, K, false, NB, C8, true>;
    const cudaError_t e = allow_dynamic_smem(kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<tab.nscan[0], 32, smem, st>>>(a, tab);
    return cudaGetLastError();
}

}  // namespace

// Not at 64 padded disparities, where the last sweep runs on two warps per chain: bands of the
// one-warp kernel there were slower on the host path (Balanced 640x480 D64 e2e 37.6 -> 36.8 G
// voxels/s) than the two-warp sweep followed by its copies.
bool sgm_last_band_supported(const SgmLaunch& l, int nin) {
    if (nin != 3 || !l.cvol || l.store_final || l.sp_tel) return false;
    if (l.Dp != 128 && l.Dp != 192 && l.Dp != 256) return false;
    if (sgm_lanes_for(l.Dp, l.lanes) != 32) return false;
    return !use_split(32, l.Dp / 64, false, l.split);
}

cudaError_t launch_sgm_last_band(const SgmLaunch& l, int dx, int dy, int nin, const uint32_t* const* in, int t_begin,
                                 int t_end, uint32_t* carry, cudaStream_t st) {
    if (!sgm_last_band_supported(l, nin) || t_begin < 0 || (t_begin & 31) || t_end <= t_begin || !carry)
        return cudaErrorInvalidValue;
    SgmArgs a = make_args(l);
    a.t_begin = t_begin;
    a.t_end = t_end;
    a.carry = carry;
    DirTable tab = {};
    tab.n = 1;
    tab.dx[0] = dx;
    tab.dy[0] = dy;
    tab.nin = nin;
    for (int i = 0; i < nin; ++i) tab.in[i] = in[i];
    switch (l.Dp) {
        case 128: return a.cost8 ? launch_last_band_k<2, true>(a, tab, st) : launch_last_band_k<2, false>(a, tab, st);
        case 192: return a.cost8 ? cudaErrorInvalidValue : launch_last_band_k<3, false>(a, tab, st);
        default: return a.cost8 ? launch_last_band_k<4, true>(a, tab, st) : launch_last_band_k<4, false>(a, tab, st);
    }
}

cudaError_t launch_sgm_fold(uint32_t* const* bufs, int nbuf, size_t words, cudaStream_t st) {
    const size_t n = words / 4;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
    FoldSrc src{};
    for (int b = 1; b < nbuf; ++b) src.b[b - 1] = reinterpret_cast<const uint4*>(bufs[b]);
    uint4* dst = reinterpret_cast<uint4*>(bufs[0]);
    if (nbuf == 7) sgm_sum_kernel<7><<<blocks, 256, 0, st>>>(dst, src, n);
    else if (nbuf == 5) sgm_sum_kernel<5><<<blocks, 256, 0, st>>>(dst, src, n);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ---- batch plan (host)

bool sgm_batch_supported(int Dp) { return Dp == 64 || Dp == 128 || Dp == 192 || Dp == 256; }

cudaError_t sgm_batch_plan_create(const SgmLaunch* pl, uint32_t* const* sbufs, int npairs, int nsbuf, int lanes,
                                  SgmBatchPlan* plan) {
    *plan = SgmBatchPlan();
    if (npairs < 1 || (nsbuf != 3 && nsbuf != 7)) return cudaErrorInvalidValue;
    const int T = lanes == 16 ? 16 : 32;
    int Dp = 0;
    bool mixed = false;
    for (int i = 0; i < npairs; ++i) {
        if (!sgm_batch_supported(pl[i].Dp) || !pl[i].cvol) return cudaErrorInvalidValue;
        if (i > 0 && pl[i].Dp != pl[0].Dp) mixed = true;
        Dp = std::max(Dp, pl[i].Dp);
    }
    if (mixed && T != 32) return cudaErrorInvalidValue;  // mixed ranges run one scanline per warp
    const int C = 32 / T;
    static const int first4[3][2] = {{1, 0}, {-1, 0}, {0, 1}};
    static const int first8[7][2] = {{1, 0}, {-1, 0}, {0, 1}, {1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
    std::vector<BatchPair> pairs(npairs);
    struct S { BatchSeg g; int len; };
    std::vector<S> first, last;
    for (int i = 0; i < npairs; ++i) {
        BatchPair& bp = pairs[i];
        std::memset(&bp, 0, sizeof(bp));
        bp.a = make_args(pl[i]);
        for (int d = 0; d < nsbuf; ++d) {
            bp.out[d] = sbufs[i * nsbuf + d];
            bp.in[d] = sbufs[i * nsbuf + d];
        }
        for (int d = 0; d < nsbuf; ++d) {
            const int dx = nsbuf == 7 ? first8[d][0] : first4[d][0];
            const int dy = nsbuf == 7 ? first8[d][1] : first4[d][1];
            S sg;
            sg.g.pair = i; sg.g.dir = d; sg.g.dx = dx; sg.g.dy = dy;
            sg.g.nscan = nscan_of(bp.a, dx, dy);
            sg.len = dy == 0 ? bp.a.w : (dx == 0 ? bp.a.h : std::min(bp.a.w, bp.a.h));
            first.push_back(sg);
        }
        S sl;
        sl.g.pair = i; sl.g.dir = 0; sl.g.dx = 0; sl.g.dy = -1;
        sl.g.nscan = nscan_of(bp.a, 0, -1);
        sl.len = bp.a.h;
        last.push_back(sl);
    }
    // longest chains first; stable, so a pair's segments stay together among equals
    auto order = [](const S& x, const S& y) { return x.len > y.len; };
    std::stable_sort(first.begin(), first.end(), order);
    std::stable_sort(last.begin(), last.end(), order);
    auto units = [&](std::vector<S>& v, int* total) {
        int u = 0;
        for (auto& x : v) {
            x.g.begin = u;
            u += (x.g.nscan + C - 1) / C;
        }
        *total = u;
    };
    units(first, &plan->total_first);
    units(last, &plan->total_last);
    plan->nseg_first = (int)first.size();
    plan->nseg_last = (int)last.size();
    plan->npairs = npairs;
    plan->nsbuf = nsbuf;
    plan->Dp = Dp;
    plan->mixed = mixed;
    plan->lanes = T;
    plan->words.resize(npairs);
    for (int i = 0; i < npairs; ++i) plan->words[i] = (size_t)pl[i].w * pl[i].h * (pl[i].Dp / 2);
    // device tables: pairs | first segments | last segments | 2 queue counters
    const size_t b_pairs = sizeof(BatchPair) * npairs;
    const size_t b_first = sizeof(BatchSeg) * first.size();
    const size_t b_last = sizeof(BatchSeg) * last.size();
    plan->off_first = (b_pairs + 255) & ~size_t(255);
    plan->off_last = (plan->off_first + b_first + 255) & ~size_t(255);
    plan->off_queue = (plan->off_last + b_last + 255) & ~size_t(255);
    const size_t total = plan->off_queue + 256;
    std::vector<unsigned char> host(total, 0);
    std::memcpy(host.data(), pairs.data(), b_pairs);
    for (size_t i = 0; i < first.size(); ++i)
        std::memcpy(host.data() + plan->off_first + i * sizeof(BatchSeg), &first[i].g, sizeof(BatchSeg));
    for (size_t i = 0; i < last.size(); ++i)
        std::memcpy(host.data() + plan->off_last + i * sizeof(BatchSeg), &last[i].g, sizeof(BatchSeg));
    cudaError_t e = cudaMalloc(&plan->dev, total);
    if (e != cudaSuccess) {
        plan->dev = nullptr;
        return e;
    }
    e = cudaMemcpy(plan->dev, host.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) sgm_batch_plan_destroy(plan);
    // the sum buffers of every pair, for the Path8 fold
    plan->sums.assign(sbufs, sbufs + (size_t)npairs * nsbuf);
    return e;
}

void sgm_batch_plan_destroy(SgmBatchPlan* plan) {
    if (plan->dev) cudaFree(plan->dev);
    *plan = SgmBatchPlan();
}

cudaError_t launch_sgm_batch(const SgmBatchPlan& plan, int max_blocks_per_sm, cudaStream_t st) {
    unsigned char* base = static_cast<unsigned char*>(plan.dev);
    const BatchPair* pairs = reinterpret_cast<const BatchPair*>(base);
    int* queue = reinterpret_cast<int*>(base + plan.off_queue);
    const BatchSeg* first = reinterpret_cast<const BatchSeg*>(base + plan.off_first);
    const BatchSeg* last = reinterpret_cast<const BatchSeg*>(base + plan.off_last);
    cudaError_t e = cudaMemsetAsync(queue, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = plan.mixed ? launch_batch_mixed<kFirst, 0>(plan.Dp, pairs, first, plan.nseg_first, plan.total_first, queue,
                                                   max_blocks_per_sm, st)
                   : launch_batch_dispatch<kFirst, 0>(plan.lanes, plan.Dp, pairs, first, plan.nseg_first,
                                                      plan.total_first, queue, max_blocks_per_sm, st);
    if (e != cudaSuccess) return e;
    if (plan.nsbuf == 7) {
        for (int i = 0; i < plan.npairs; ++i) {
            e = launch_sgm_fold(plan.sums.data() + (size_t)i * 7, 7, plan.words[i], st);
            if (e != cudaSuccess) return e;
        }
        return plan.mixed ? launch_batch_mixed<kLast, 1>(plan.Dp, pairs, last, plan.nseg_last, plan.total_last,
                                                         queue + 1, max_blocks_per_sm, st)
                          : launch_batch_dispatch<kLast, 1>(plan.lanes, plan.Dp, pairs, last, plan.nseg_last,
                                                            plan.total_last, queue + 1, max_blocks_per_sm, st);
    }
    return plan.mixed ? launch_batch_mixed<kLast, 3>(plan.Dp, pairs, last, plan.nseg_last, plan.total_last, queue + 1,
                                                     max_blocks_per_sm, st)
                      : launch_batch_dispatch<kLast, 3>(plan.lanes, plan.Dp, pairs, last, plan.nseg_last,
                                                        plan.total_last, queue + 1, max_blocks_per_sm, st);
}

}  // namespace apgcu


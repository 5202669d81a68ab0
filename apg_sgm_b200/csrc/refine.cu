// HighQuality selective refinement, detail::refine_scalar (src/refiner.cpp:42-100).
//
// The reference walks the image in raster order (forward on even passes, backward on odd) and
// updates unreliable pixels in place, so a pixel sees the already-updated values of its causal
// neighbours (left and up forward, right and down backward).
//
// Schedule: a pass is one launch of refine_band_kernel.  A warp owns a band of 32 consecutive
// (pass-order) rows, lane i row i, and walks the columns with lane i one column behind lane i-1:
// at step t lane i updates column t - i, so its up neighbour is what lane i-1 produced at step
// t-1 (one shuffle) and its left neighbour is its own previous value.  The first row of a band
// reads the row above from global memory once the band above has published, through a progress
// counter, that its last row is final that far; the bands therefore run as a wavefront about 40
// columns apart and a pass takes about w + h steps.  Every wait is bounded: on timeout the band
// sets an error flag (read by the host) and stops.  This is exactly the reference's
// read-after-write order.
//
// Random draws: a pixel consumes a draw when it is unreliable, has a non-empty range and holds a
// non-negative value at the start of the pass, so its draw index is an exclusive prefix count of
// such pixels in the pass's raster order.  The reference takes draws from one std::mt19937(12345)
// stream through a fresh std::uniform_int_distribution<int>(-r, r) per pass.  A draw maps one
// accepted engine output to a value and skips rejected outputs, each a function of that single
// output, so per radius the value of every output of the (fixed) stream and the rare rejected
// indices are tabulated once, on the host, by the standard library itself: pass `it` then takes
// the q-th accepted output at or after its start position P_it, and P_{it+1} follows on the device
// from the pass's count.  No host work or synchronisation remains per frame.
#include <algorithm>
#include <map>
#include <mutex>
#include <random>
#include <vector>

#include "engine.h"

namespace apgcu {

namespace {

constexpr int kBand = 32;
constexpr int kPublish = 8;      // steps between progress publications
constexpr int kMaxRejected = 64;  // rejected outputs tabulated per radius (expected: none)

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

// Exclusive prefix sum of the flags in place (the draw index of every pixel, and the pass's count
// at index n): three launches without atomics or waits, so the result does not depend on
// scheduling.  A tile is kScanThreads x kScanPer consecutive entries.
constexpr int kScanThreads = 1024, kScanPer = 4, kScanTile = kScanThreads * kScanPer;

// Exclusive prefix of v over the block and the block's total (s_warp: 32 ints).
__device__ __forceinline__ int block_exclusive(int v, int* s_warp, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        s_warp[lane] = t;
    }
    __syncthreads();
    *total = s_warp[31];
    const int before = wid ? s_warp[wid - 1] : 0;
    __syncthreads();  // s_warp may be reused by the caller
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums_kernel(const int* __restrict__ in, int n,
                                                                      int* __restrict__ sums) {
    __shared__ int s_warp[32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
    int v = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
        if (base + k < (size_t)n) v += in[base + k];
    int total = 0;
    block_exclusive(v, s_warp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// One block: the tile sums [0, nt) into exclusive tile offsets, in place.
__global__ void __launch_bounds__(kScanThreads) scan_tile_offsets_kernel(int* sums, int nt) {
    __shared__ int s_warp[32];
    int carry = 0;
    for (int b = 0; b < nt; b += kScanThreads) {
        const int i = b + (int)threadIdx.x;
        const int v = i < nt ? sums[i] : 0;
        int total = 0;
        const int ex = block_exclusive(v, s_warp, &total);
        if (i < nt) sums[i] = carry + ex;
        carry += total;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(int* data, int n, const int* __restrict__ offs) {
    __shared__ int s_warp[32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
    int v[kScanPer];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = base + k < (size_t)n ? data[base + k] : 0;
        sum += v[k];
    }
    int total = 0;
    int run = offs[blockIdx.x] + block_exclusive(sum, s_warp, &total);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < (size_t)n) data[base + k] = run;
        run += v[k];
    }
}

// Raw index of the q-th accepted output at or after P (rejected indices sorted ascending).
__device__ __forceinline__ unsigned accepted_index(unsigned P, unsigned q, const unsigned* rej, int nrej) {
    unsigned idx = P + q;
    for (int k = 0; k < nrej; ++k) {
        const unsigned r = rej[k];
        if (r < P) continue;
        if (r <= idx) ++idx;
        else break;
    }
    return idx;
}

// Start of pass `it + 1`: the stream position after pass `it`'s count of draws from P[it]; also
// clears the bands' progress counters for the next pass.
__global__ void refine_advance_kernel(unsigned* P, int it, const int* count, const unsigned* rej, int nrej,
                                      int* progress, int nbands) {
    if (threadIdx.x == 0) {
        const unsigned c = (unsigned)*count;
        P[it + 1] = c ? accepted_index(P[it], c - 1, rej, nrej) + 1 : P[it];
    }
    for (int b = threadIdx.x; b < nbands; b += blockDim.x) progress[b] = 0;
}

// Left and right images packed per pixel for the refiner: census (32 bits, or 64 in two words) and
// gray | gx << 8 | gy << 16, so a candidate's cost needs one load of each side.
template <bool C64>
struct RPack;
template <>
struct __align__(8) RPack<false> {
    uint32_t c, g;
};
template <>
struct __align__(16) RPack<true> {
    unsigned long long c;
    uint32_t g, pad;
};

template <bool C64>
__global__ void refine_pack_kernel(CostCtx c, RPack<C64>* __restrict__ lp, RPack<C64>* __restrict__ rp) {
    const int n = c.w * c.h;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        RPack<C64> a, b;
        if constexpr (C64) {
            a.c = c.cl64[i];
            b.c = c.cr64[i];
            a.pad = b.pad = 0;
        } else {
            a.c = c.cl[i];
            b.c = c.cr[i];
        }
        a.g = (uint32_t)c.lgray[i] | ((uint32_t)c.lgx[i] << 8) | ((uint32_t)c.lgy[i] << 16);
        b.g = (uint32_t)c.rgray[i] | ((uint32_t)c.rgx[i] << 8) | ((uint32_t)c.rgy[i] << 16);
        lp[i] = a;
        rp[i] = b;
    }
}

// The refiner's local cost, local_cost (src/refiner.cpp:14-36), from packed pixels: the same LUT
// terms added in the same order.
template <bool C64>
__device__ __forceinline__ float packed_cost(const CostCtx& c, const float* lut, const RPack<C64>& l,
                                             const RPack<C64>& r) {
    int pop;
    if constexpr (C64) pop = __popcll(l.c ^ r.c);
    else pop = __popc(l.c ^ r.c);
    float v = lut[kLutCensus + pop];
    const uint32_t dd = __vabsdiffu4(l.g, r.g);  // |dgray|, |dgx|, |dgy|
    if (c.use_ad) v = __fadd_rn(v, lut[kLutAd + (dd & 0xFFu)]);
    if (c.use_grad) v = __fadd_rn(v, lut[kLutGrad + ((dd >> 8) & 0xFFu) + (dd >> 16)]);
    return v;
}

// Everything about one pixel of a pass that does not depend on the wavefront, computed for all
// pixels at once before the pass and laid out in pass order (index v * w + u): the value at the
// start of the pass, its range, and the two static candidates -- the current value and the
// current value plus the pixel's draw -- with their costs.  The band kernel only costs the two
// dynamic candidates (left and up neighbours) and keeps the reference's candidate order.
struct __align__(16) RStep {
    float cur;     // value at the start of the pass
    float c_cur;   // cost of candidate `cur` (when upd bit 1)
    float c_draw;  // cost of candidate `cur + draw` (when upd bit 2)
    int d_pack;    // d_cur (low 16, signed) | d_draw (high 16, signed)
    int range;     // lo (low 16) | hi (high 16)
    int upd;       // bit 0: unreliable with a non-empty range; bit 1: cur is a candidate; bit 2: cur + draw is
    int rcur;      // the start value as a neighbour candidate: roundf(cur) when cur >= 0, else -1
    int pad1;
};

template <bool C64>
__device__ __forceinline__ float cand_cost(const CostCtx& c, const float* lut, const RPack<C64>& l,
                                           const RPack<C64>* __restrict__ rp, int x, int y, int d, int lo, int hi) {
    const int xr = x - d;
    if (xr >= 0 && xr < c.w && d >= lo && d < hi) return packed_cost<C64>(c, lut, l, rp[y * c.w + xr]);
    return 1e6f;
}

template <bool C64>
__global__ void refine_prep_kernel(CostCtx c, int fwd, const uint8_t* __restrict__ reliable,
                                   const int* __restrict__ prefix, const int16_t* __restrict__ draw_value,
                                   const unsigned* __restrict__ rej, int nrej, const unsigned* __restrict__ P_ptr,
                                   const RPack<C64>* __restrict__ lp, const RPack<C64>* __restrict__ rp,
                                   const float* __restrict__ work, RStep* __restrict__ steps) {
    __shared__ float s_lut[kLutSize];
    for (int i = threadIdx.x; i < kLutSize; i += blockDim.x) s_lut[i] = c.lut[i];
    __syncthreads();
    const int w = c.w, h = c.h, n = w * h;
    const unsigned P = *P_ptr;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int v = j / w, u = j - v * w;
        const int x = fwd ? u : w - 1 - u;
        const int y = fwd ? v : h - 1 - v;
        const int i = y * w + x;
        RStep st;
        st.cur = work[i];
        const int lo = c.rmin[i], hi = c.rmax[i];
        st.range = (lo & 0xFFFF) | (hi << 16);
        st.upd = (!reliable[i] && hi > lo) ? 1 : 0;
        int d_cur = 0, d_draw = 0;
        st.c_cur = st.c_draw = 1e9f;
        st.rcur = st.cur >= 0.f ? (int)roundf(st.cur) : -1;
        st.pad1 = 0;
        if (st.upd && st.cur >= 0.f) {
            const RPack<C64> l = lp[i];
            d_cur = min(max((int)roundf(st.cur), lo), hi - 1);
            st.c_cur = cand_cost<C64>(c, s_lut, l, rp, x, y, d_cur, lo, hi);
            st.upd |= 2;
            const unsigned q = (unsigned)prefix[fwd ? i : n - 1 - i];
            const float dv = __fadd_rn(st.cur, (float)draw_value[accepted_index(P, q, rej, nrej)]);
            if (dv >= 0.f) {
                d_draw = min(max((int)roundf(dv), lo), hi - 1);
                st.c_draw = cand_cost<C64>(c, s_lut, l, rp, x, y, d_draw, lo, hi);
                st.upd |= 4;
            }
        }
        st.d_pack = (d_cur & 0xFFFF) | (d_draw << 16);
        steps[j] = st;
    }
}

constexpr int kRing = 16;  // steps of pixel records in flight per lane
constexpr int kAhead = 32; // steps ahead the right-image window is prefetched into L1

__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];\n" ::"l"(p));
}

// Progress counters between bands use the fence forms of release and acquire: the publishing lane
// fences (acquire-release, device scope) and then stores the counter; the reading band polls the
// counter and fences before reading the row above.
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;\n" ::: "memory"); }

// The loader warp's copies into the step ring carry no compiler memory clobber: their order
// against the compute warp's reads is set by the ring's mbarriers (a slot is refilled only after
// the wait for its empty barrier, and read only after the wait for its full barrier).
__device__ __forceinline__ void cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src));
}

// Shared state of one band's two warps.  The compute warp (warp 0) walks the band; the link warp
// (warp 1) carries every exchange with the other bands, so that no GPU-scope fence or L2 round
// trip sits in the compute warp's step loop:
//   * it polls the band above's progress counter and copies the newly final columns of that
//     band's last row into `up` (a ring of kUpRing columns), then raises `avail`;
//   * it publishes how far this band's last row is final (`done`, raised by the compute warp at
//     CTA scope) to this band's progress counter, behind a GPU-scope fence.
// Causality runs compute warp -> (CTA-scope release / acquire) -> link warp -> (GPU-scope release /
// acquire) -> the next band's link warp, which is the order the reference's in-place raster scan
// implies for the row above.
constexpr int kUpRing = 128;
struct BandLink {
    int up[kUpRing];    // row above the band as neighbour candidates (roundf(value) when value >= 0,
                        // else -1): column c at up[c & (kUpRing - 1)]
    int avail;          // columns [0, avail) of the row above are in `up` (link warp)
    int used;           // columns [0, used) of `up` are no longer read (compute warp)
    int done;           // columns [0, done) of the band's last row are final in `work` (compute warp)
    int abort;          // the link warp gave up waiting (or saw the error word): the compute warp stops
};

// The link warp of band `band` (see BandLink).  Every wait is bounded: after spin_limit polls in
// which nothing moved it sets the error word and `abort`, and after as many again it leaves.
__device__ void band_link(BandLink* s_link, int band, int w, int h, int fwd, const float* work, int* progress,
                          int* err, int spin_limit) {
    const int lane = threadIdx.x & 31;
    volatile BandLink* L = s_link;
    volatile int* vprog = progress;
    const int xs = fwd ? 1 : -1, xb = fwd ? 0 : w - 1;
    const int y_above = band > 0 ? (fwd ? band * kBand - 1 : h - band * kBand) : 0;
    const float* above = work + (size_t)y_above * w;
    int fetched = band > 0 ? 0 : w;  // columns of the row above copied into the ring
    int published = 0;
    int idle = 0;
    bool gave_up = false;
    for (;;) {
        bool moved = false;
        // this band's last row, as far as the compute warp has released it
        const int done = L->done;
        if (done > published) {
            if (lane == 0) {
                fence_acq_rel();
                vprog[band] = done;
            }
            published = done;
            moved = true;
        }
        if (published >= w) break;
        // the row above, as far as the band above has published it and the ring has room
        if (fetched < w && !gave_up) {
            int prog = 0;
            if (lane == 0) prog = vprog[band - 1];
            prog = __shfl_sync(0xffffffffu, prog, 0);
            const int upto = min(min(prog, L->used + kUpRing), w);
            if (upto > fetched) {
                if (lane == 0) fence_acq_rel();
                __syncwarp();
                for (int col = fetched + lane; col < upto; col += 32) {
                    const float a = __ldcg(above + (xb + xs * col));
                    s_link->up[col & (kUpRing - 1)] = a >= 0.f ? (int)roundf(a) : -1;
                }
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    L->avail = upto;
                }
                fetched = upto;
                moved = true;
            }
        }
        if (moved) {
            idle = 0;
            continue;
        }
        ++idle;
        if (!gave_up && (idle > spin_limit || *(volatile int*)err)) {
            if (lane == 0) {
                atomicExch(err, 1);
                L->abort = 1;
            }
            gave_up = true;
            idle = 0;
        } else if (gave_up && idle > spin_limit) {
            break;  // the compute warp did not finish either: leave (the frame is already failed)
        }
        __nanosleep(64);
    }
}

// ---- the band kernel's step ring: mbarriers between the loader warp and the compute warp
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(b)) : "memory");
}
// arrives once every cp.async this thread issued before it has landed
__device__ __forceinline__ void mbar_arrive_copies(uint64_t* b) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_done(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(smem_u32(b)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Waits, in every lane of the warp, for the completed phase `parity` of b; the warp leaves the
// wait together.  False after `limit` polls (each followed by a sleep of `sleep_ns` when non-zero)
// or once *stop is raised.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* b, unsigned parity, int limit, const volatile int* stop,
                                               int sleep_ns) {
    for (int spins = 0;; ++spins) {
        if (__all_sync(0xffffffffu, mbar_done(b, parity))) return true;
        if (spins >= limit || (stop && *stop)) return false;
        if (sleep_ns) __nanosleep(sleep_ns);
    }
}

// Per-lane view of a band's row for one pass: pass-order column u of the lane's row is image
// column xb + xs * u.
template <bool C64>
struct BandRow {
    int lane, v, xs, xb, eoff;
    bool ok;
    const RStep* steps;       // this lane's records, pass order
    const RPack<C64>* left;   // this lane's left pixels
    const RPack<C64>* right;  // this lane's right-image row
    float* work;
    __device__ BandRow(const CostCtx& c, int band, int fwd, const RStep* all_steps, const RPack<C64>* lp,
                       const RPack<C64>* rp, float* all_work) {
        lane = threadIdx.x & 31;
        v = band * kBand + lane;
        ok = v < c.h;
        xs = fwd ? 1 : -1;
        xb = fwd ? 0 : c.w - 1;
        const int yrow = fwd ? v : c.h - 1 - v;
        const size_t rowoff = (size_t)(ok ? yrow : 0) * c.w;
        steps = all_steps + (size_t)(ok ? v : 0) * c.w;
        left = lp + rowoff;
        right = rp + rowoff;
        work = all_work + rowoff;
        eoff = fwd ? c.d0 : c.d0 + c.D - 1;  // entering window pixel of column u: x(u) - eoff
    }
};

// Shared memory of the band kernel besides the link state.
template <bool C64>
struct BandRing {
    RStep rec[kRing][32];       // step t's records in slot t % kRing, one per lane
    RPack<C64> lpk[kRing][32];  // and the lanes' packed left pixels
    uint64_t full[kRing];       // slot filled (32 loader arrivals, each once its copies landed)
    uint64_t empty[kRing];      // slot read (one arrival of the compute warp)
    int stop;                   // the compute warp has stopped: the loader stops too
};

// The loader warp: copies step t's records, packed left pixels and (WIN) the window's entering
// right-image pixels into slot t % kRing and signals full[slot] when they have landed, up to
// kRing steps ahead of the compute warp, refilling a slot only once the compute warp has released
// it.  Without WIN it keeps the right-image window warm in L1 instead: every lane misses L1 at a
// different step and the compute warp waits for the slowest, so the window's first kAhead steps
// are prefetched first and its entering edge kAhead steps ahead of the copies.
template <bool C64, bool WIN>
__device__ void band_loader(const CostCtx& c, const BandRow<C64>& r, BandRing<C64>* ring, RPack<C64>* s_win,
                            int wmask, int spin_limit) {
    const int w = c.w, lane = r.lane;
    auto copy_win = [&](int u) {
        const int pe = r.xb + r.xs * u - r.eoff;
        if ((unsigned)pe < (unsigned)w)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(&s_win[(pe & wmask) * kBand])),
                         "l"(r.right + pe));
    };
    if (WIN && r.ok) {
        // the rest of the window of the lane's first column: columns -(D - 1) .. -lane - 1
        for (int u = -(c.D - 1); u < -lane; ++u) copy_win(u);
    }
    if (!WIN && r.ok) {
        for (int k = -c.D; k <= kAhead; k += 8) prefetch_l1(r.right + min(max(r.xb + r.xs * k - r.eoff, 0), w - 1));
    }
    int pe = r.xb + r.xs * (kAhead - lane) - r.eoff;  // entering pixel kAhead steps ahead
    const int nsteps = w + kBand - 1;
    for (int t = 0; t < nsteps; ++t) {
        const int slot = t % kRing;
        if (t >= kRing &&
            !mbar_wait_warp(&ring->empty[slot], ((t / kRing) - 1) & 1, spin_limit, &ring->stop, 64))
            break;  // the compute warp stopped, or never released the slot: it fails the pass itself
        const int u = t - lane;
        if (r.ok && u >= 0 && u < w) {
            const RStep* src = r.steps + u;
            cp16(&ring->rec[slot][lane], src);
            cp16(reinterpret_cast<unsigned char*>(&ring->rec[slot][lane]) + 16,
                 reinterpret_cast<const unsigned char*>(src) + 16);
            const RPack<C64>* ls = r.left + (r.xb + r.xs * u);
            if constexpr (C64) {
                cp16(&ring->lpk[slot][lane], ls);
            } else {
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(&ring->lpk[slot][lane])),
                             "l"(ls));
            }
        }
        // the window pixel entering at this column (also for the columns before the lane's first)
        if (WIN && r.ok && u < w) copy_win(u);
        if (!WIN && r.ok) prefetch_l1(r.right + min(max(pe, 0), w - 1));
        pe += r.xs;
        mbar_arrive_copies(&ring->full[slot]);
    }
    // no copy may land after the block has left
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// WIN: each lane's right-image window ([x - dmax + 1, x - d0] of its row, sliding one pixel per
// step) lives in shared memory, a ring of wmask + 1 records per lane (a power of two holding the
// window plus the kRing steps copied ahead; the lanes' rings interleaved); the loader copies the
// entering pixel with the step's record, so the candidates' right pixels are shared-memory loads.
// Without WIN they are global loads kept warm in L1 by the loader's prefetches.  Three warps per block: warp 0 computes, warp 1
// links the band to its neighbours (band_link), warp 2 loads the step ring (band_loader), so that
// no copy or address arithmetic sits in the compute warp's step.
template <bool C64, bool WIN>
__global__ void __launch_bounds__(96) refine_band_kernel(CostCtx c, int fwd, const RStep* __restrict__ steps,
                                                         const RPack<C64>* __restrict__ lp,
                                                         const RPack<C64>* __restrict__ rp, float* work,
                                                         int* progress, int* err, int spin_limit, int wmask) {
    __shared__ float s_lut[kLutSize];
    __shared__ __align__(16) BandRing<C64> s_ring;
    __shared__ BandLink s_link;
    for (int i = threadIdx.x; i < kLutSize; i += blockDim.x) s_lut[i] = c.lut[i];
    if (threadIdx.x == 0) {
        s_link.avail = 0;
        s_link.used = 0;
        s_link.done = 0;
        s_link.abort = 0;
        s_ring.stop = 0;
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&s_ring.full[i], 32);
            mbar_init(&s_ring.empty[i], 1);
        }
    }
    __syncthreads();
    const int band = blockIdx.x;
    const int w = c.w;
    const int warp = threadIdx.x >> 5;
    if (warp == 1) {
        band_link(&s_link, band, w, c.h, fwd, work, progress, err, spin_limit);
        return;
    }
    const BandRow<C64> r(c, band, fwd, steps, lp, rp, work);
    extern __shared__ __align__(16) unsigned char s_dyn[];
    // the lanes' window rings interleaved, record i of lane l at i * kBand + l: a step's loads of
    // the 32 lanes fall in distinct banks whatever their offsets
    RPack<C64>* s_win = reinterpret_cast<RPack<C64>*>(s_dyn) + r.lane;
    if (warp == 2) {
        band_loader<C64, WIN>(c, r, &s_ring, s_win, wmask, spin_limit);
        return;
    }
    volatile BandLink* link = &s_link;
    const int lane = r.lane, v = r.v;
    const bool row_ok = r.ok;
    float* wrow = r.work;
    const RPack<C64>* rrow = r.right;
    // Neighbour values travel as candidates: roundf(value) when value >= 0, else -1 (the
    // reference takes a neighbour only when it is non-negative, rounded).  An updated value is an
    // integer already; a start value's candidate comes with its record.
    int prev = -1;  // candidate of this lane's previous column (its left neighbour)
    int avail = band > 0 ? 0 : w;  // columns of the row above known to be in the link's ring
    bool abort = false;
    for (int t = 0; t < w + kBand - 1; ++t) {
        int up_first = -1;  // the row above at column t (lane 0's up neighbour)
        if (band > 0 && t < w) {
            if (t >= avail) {
                // wait until the link warp has the row above at least up to column t (lane 0
                // polls, so that the warp decides together)
                int spins = 0, state = 0;  // 1: available, 2: gave up
                for (;;) {
                    if (lane == 0) {
                        const int a = link->avail;
                        state = a > t ? 1 : ((link->abort || ++spins > spin_limit) ? 2 : 0);
                        if (state == 1) avail = a;
                    }
                    state = __shfl_sync(0xffffffffu, state, 0);
                    if (state) break;
                    __nanosleep(32);
                }
                avail = __shfl_sync(0xffffffffu, avail, 0);
                if (state == 2) {
                    abort = true;
                    if (lane == 0) atomicExch(err, 1);
                    break;
                }
                __threadfence_block();
            }
            if (lane == 0) up_first = s_link.up[t & (kUpRing - 1)];
        }
        // step t's slot has landed
        const int slot = t % kRing;
        if (!mbar_wait_warp(&s_ring.full[slot], (t / kRing) & 1, spin_limit, nullptr, 0)) {
            abort = true;
            if (lane == 0) atomicExch(err, 1);
            break;
        }
        const int up_lane = __shfl_up_sync(0xffffffffu, prev, 1);
        const int u = t - lane;
        if (row_ok && u >= 0 && u < w) {
            const RStep st = s_ring.rec[slot][lane];
            int cand = st.rcur;
            if (st.upd & 1) {
                const int x = r.xb + r.xs * u;
                const int lo = (int)(short)(st.range & 0xFFFF), hi = st.range >> 16;
                const int d_cur = (int)(short)(st.d_pack & 0xFFFF), d_draw = st.d_pack >> 16;
                const bool has_cur = (st.upd & 2) != 0, has_draw = (st.upd & 4) != 0;
                const RPack<C64> l = s_ring.lpk[slot][lane];
                // dynamic candidates: left (forward) / right (backward) and up / down
                const int left = u > 0 ? prev : -1;
                const int up = v > 0 ? (lane > 0 ? up_lane : up_first) : -1;
                const bool has_l = left >= 0, has_u = up >= 0;
                // clamped into [lo, hi - 1] (hi > lo for an updated pixel), so only x - d needs a test
                const int dl = has_l ? min(max(left, lo), hi - 1) : 0;
                const int du = has_u ? min(max(up, lo), hi - 1) : 0;
                const int xl = x - dl, xu = x - du;
                const float cl = (has_l && (unsigned)xl < (unsigned)w)
                                     ? packed_cost<C64>(c, s_lut, l, WIN ? s_win[(xl & wmask) * kBand] : rrow[xl])
                                     : 1e6f;
                const float cu = (has_u && (unsigned)xu < (unsigned)w)
                                     ? packed_cost<C64>(c, s_lut, l, WIN ? s_win[(xu & wmask) * kBand] : rrow[xu])
                                     : 1e6f;
                // the reference's order: cur, left, up, cur + draw; the first strict minimum wins
                float best_c = 1e9f;
                int best_d = st.cur >= 0.f ? d_cur : lo;
                if (has_cur && st.c_cur < best_c) { best_c = st.c_cur; best_d = d_cur; }
                if (has_l && cl < best_c) { best_c = cl; best_d = dl; }
                if (has_u && cu < best_c) { best_c = cu; best_d = du; }
                if (has_draw && st.c_draw < best_c) { best_c = st.c_draw; best_d = d_draw; }
                wrow[x] = (float)best_d;
                cand = best_d >= 0 ? best_d : -1;
            }
            prev = cand;
        }
        // every lane has read the slot (and its window pixels): the loader may refill it
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_ring.empty[slot]);
        if ((t % kPublish) == kPublish - 1) {
            // release to the link warp (CTA scope): how far the last row (lane 31, column t - 31)
            // is final, and that the ring's columns up to t are read
            __threadfence_block();
            if (lane == kBand - 1) link->done = max(0, min(t - (kBand - 1) + 1, w));
            if (lane == 0) link->used = min(t + 1, w);
        }
    }
    if (abort) *(volatile int*)&s_ring.stop = 1;
    __syncwarp();
    __threadfence_block();
    // the whole band is final (or the pass was abandoned: let the next band finish)
    if (lane == kBand - 1) link->done = w;
}

// ---- host: the engine stream, its draw values and rejected indices per radius

struct DrawTable {
    std::vector<int16_t> value;
    std::vector<unsigned> rejected;
};

std::mutex g_rng_mu;
std::vector<uint32_t> g_raw;          // std::mt19937(12345) outputs, generated on demand
std::mt19937 g_engine(12345);
std::map<int, DrawTable> g_tables;   // by radius

// A generator that replays recorded engine outputs, counting how many the distribution takes.
struct Replay {
    using result_type = std::mt19937::result_type;
    const uint32_t* p;
    int calls = 0;
    static constexpr result_type min() { return std::mt19937::min(); }
    static constexpr result_type max() { return std::mt19937::max(); }
    result_type operator()() { return p[calls++]; }
};

const DrawTable& draw_table_locked(int radius, size_t length) {
    while (g_raw.size() < length + 64) g_raw.push_back((uint32_t)g_engine());
    DrawTable& t = g_tables[radius];
    std::uniform_int_distribution<int> dist(-radius, radius);
    for (size_t i = t.value.size(); i < length; ++i) {
        Replay g{g_raw.data() + i};
        const int v = dist(g);
        t.value.push_back((int16_t)v);
        if (g.calls != 1) t.rejected.push_back((unsigned)i);  // output i is skipped by the distribution
    }
    return t;
}

}  // namespace

size_t refine_scan_temp_bytes(int n) { return (size_t)((n + 1 + kScanTile - 1) / kScanTile) * sizeof(int); }

int refine_band_count(int h) { return (h + kBand - 1) / kBand; }

int RefineTables::build(int iterations, int base_radius, int n) {
    release();
    std::vector<const DrawTable*> tabs(iterations);
    std::vector<size_t> len(iterations);
    {
        std::lock_guard<std::mutex> lk(g_rng_mu);
        for (int it = 0; it < iterations; ++it) {
            const int radius = std::max(1, base_radius >> it);
            if (radius > 32767) return 1;
            // pass `it` starts at most it * n outputs (plus rejections) into the stream
            len[it] = (size_t)(it + 1) * n + 64;
            tabs[it] = &draw_table_locked(radius, len[it]);
            if (tabs[it]->rejected.size() > (size_t)kMaxRejected) return 1;
        }
    }
    iters = iterations;
    size_t total = 0;
    for (int it = 0; it < iterations; ++it) total += len[it] * 2 + kMaxRejected * 4 + 256;
    if (cudaMalloc(&dev, total) != cudaSuccess) {
        cudaGetLastError();
        dev = nullptr;
        return 1;
    }
    bytes = total;
    unsigned char* p = static_cast<unsigned char*>(dev);
    for (int it = 0; it < iterations; ++it) {
        const DrawTable& t = *tabs[it];
        value[it] = reinterpret_cast<int16_t*>(p);
        if (cudaMemcpy(p, t.value.data(), len[it] * 2, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
        p += (len[it] * 2 + 255) & ~size_t(255);
        rejected[it] = reinterpret_cast<unsigned*>(p);
        size_t nr = 0;
        for (unsigned r : t.rejected)
            if (r < len[it]) ++nr;
        nrej[it] = (int)nr;
        if (nr && cudaMemcpy(p, t.rejected.data(), nr * 4, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
        p += kMaxRejected * 4;
    }
    n_built = n;
    radius_built = base_radius;
    return 0;
}

void RefineTables::release() {
    if (dev) cudaFree(dev);
    dev = nullptr;
    bytes = 0;
    iters = 0;
    n_built = 0;
}

cudaError_t launch_refine_count(const Layout& L, unsigned char* arena, const float* work, int fwd,
                                cudaStream_t s, unsigned* launches) {
    const int n = L.w * L.h;
    int* flags = reinterpret_cast<int*>(arena + L.rf_prefix);
    const int blocks = min((n + 256) / 256, 148 * 8);
    refine_flags_kernel<<<blocks, 256, 0, s>>>(L.w, L.h, reinterpret_cast<const uint8_t*>(arena + L.reliable),
                                                reinterpret_cast<const int16_t*>(arena + L.rmin),
                                                reinterpret_cast<const int16_t*>(arena + L.rmax), work, fwd, flags);
    // the draw indices: exclusive prefix sum of the n + 1 flags (the last one 0), in place
    const int m = n + 1;
    const int nt = (m + kScanTile - 1) / kScanTile;
    int* sums = reinterpret_cast<int*>(arena + L.rf_scan_tmp);
    scan_tile_sums_kernel<<<nt, kScanThreads, 0, s>>>(flags, m, sums);
    scan_tile_offsets_kernel<<<1, kScanThreads, 0, s>>>(sums, nt);
    scan_apply_kernel<<<nt, kScanThreads, 0, s>>>(flags, m, sums);
    *launches += 4;
    return cudaGetLastError();
}

cudaError_t launch_refine_pack(const CostCtx& c, const Layout& L, unsigned char* arena, cudaStream_t s,
                               unsigned* launches) {
    const int n = L.w * L.h;
    const int blocks = min((n + 255) / 256, 148 * 8);
    if (c.census64)
        refine_pack_kernel<true><<<blocks, 256, 0, s>>>(c, reinterpret_cast<RPack<true>*>(arena + L.rf_pack),
                                                        reinterpret_cast<RPack<true>*>(arena + L.rf_pack) + n);
    else
        refine_pack_kernel<false><<<blocks, 256, 0, s>>>(c, reinterpret_cast<RPack<false>*>(arena + L.rf_pack),
                                                         reinterpret_cast<RPack<false>*>(arena + L.rf_pack) + n);
    ++*launches;
    return cudaGetLastError();
}

size_t refine_pack_bytes(int n, bool c64) { return (size_t)n * 2 * (c64 ? sizeof(RPack<true>) : sizeof(RPack<false>)); }

cudaError_t launch_refine_pass(const CostCtx& c, const Layout& L, unsigned char* arena, const RefineTables& tab,
                               int it, float* work, const RefineTuning& tune, cudaStream_t s, unsigned* launches) {
    const int fwd = (it % 2) == 0;
    const int n = L.w * L.h;
    const int nbands = refine_band_count(L.h);
    const uint8_t* rel = reinterpret_cast<const uint8_t*>(arena + L.reliable);
    const int* prefix = reinterpret_cast<const int*>(arena + L.rf_prefix);
    unsigned* P = reinterpret_cast<unsigned*>(arena + L.rf_state);
    int* err = reinterpret_cast<int*>(arena + L.rf_state) + kRefineErrWord;
    int* progress = reinterpret_cast<int*>(arena + L.rf_state) + kRefineProgWord;
    RStep* steps = reinterpret_cast<RStep*>(arena + L.rf_steps);
    const int blocks = min((n + 255) / 256, 148 * 8);
    if (c.census64) {
        const RPack<true>* lpk = reinterpret_cast<const RPack<true>*>(arena + L.rf_pack);
        refine_prep_kernel<true><<<blocks, 256, 0, s>>>(c, fwd, rel, prefix, tab.value[it], tab.rejected[it], tab.nrej[it],
                                                        P + it, lpk, lpk + n, work, steps);
    } else {
        const RPack<false>* lpk = reinterpret_cast<const RPack<false>*>(arena + L.rf_pack);
        refine_prep_kernel<false><<<blocks, 256, 0, s>>>(c, fwd, rel, prefix, tab.value[it], tab.rejected[it],
                                                         tab.nrej[it], P + it, lpk, lpk + n, work, steps);
    }
    ++*launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // about a second of waiting at most per wait (spins of ~128 ns sleep plus the poll), unless the
    // engine's tuning sets a smaller poll budget
    int spin_limit = tune.spin_limit > 0 ? tune.spin_limit : 1 << 23;
    CostCtx cc = c;
    const void* lpk = arena + L.rf_pack;
    const void* rpk = c.census64 ? (const void*)(reinterpret_cast<const RPack<true>*>(lpk) + n)
                                 : (const void*)(reinterpret_cast<const RPack<false>*>(lpk) + n);
    const RStep* csteps = steps;
    int fwd_arg = fwd;
    // the right-image window in shared memory (32-bit census): a power-of-two ring per lane holding
    // the D window pixels plus the kRing copied ahead, when every band still fits on the device at once
    int wmask = 0;
    size_t wbytes = 0;
    const void* kern = c.census64 ? (const void*)refine_band_kernel<true, false> : (const void*)refine_band_kernel<false, false>;
    if (!c.census64 && tune.window == 0) {
        int rs = 1;
        while (rs < c.D + kRing) rs <<= 1;
        const size_t bytes = (size_t)kBand * (rs + 1) * sizeof(RPack<false>);
        auto wk = refine_band_kernel<false, true>;
        if (rs <= 512 && allow_dynamic_smem(wk, bytes) == cudaSuccess) {
            int per_sm = 0, dev = 0, nsm = 0;
            if (cudaGetDevice(&dev) == cudaSuccess &&
                cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wk, 3 * kBand, bytes) == cudaSuccess &&
                per_sm * nsm >= nbands) {
                wmask = rs - 1;
                wbytes = bytes;
                kern = (const void*)wk;
            }
        }
        cudaGetLastError();
    }
    void* args[] = {&cc, &fwd_arg, (void*)&csteps, (void*)&lpk, (void*)&rpk, &work, &progress, &err, &spin_limit,
                    &wmask};
    e = cudaLaunchCooperativeKernel(kern, dim3(nbands), dim3(3 * kBand), args, wbytes, s);
    if (e != cudaSuccess) return e;
    ++*launches;
    // start of the next pass, and cleared progress counters
    const int* count = prefix + n;
    refine_advance_kernel<<<1, 64, 0, s>>>(P, it, count, tab.rejected[it], tab.nrej[it], progress, nbands);
    ++*launches;
    return cudaGetLastError();
}

size_t refine_steps_bytes(int n) { return (size_t)n * sizeof(RStep); }

}  // namespace apgcu

// HighQuality sparse support prior and search-range shrink, PriorEstimator
// (src/prior_estimator.cpp:13-412), entirely on the device.
//
//   1. candidates (extract_supports :28-110): one warp per 16x16 cell; each lane evaluates the
//      step-2 grid positions (census-only WTA with best/second, uniqueness, right-to-left check)
//      and a ballot keeps the first max_cand passing positions in the cell's raster order;
//   2. selection (:112-165): one CTA reproduces the stratified budget -- base quota per non-empty
//      cell, then round-robin rounds, or the uniform sub-sampling when non-empty cells exceed the
//      budget -- with block-wide prefix counts instead of the serial loops;
//   3. per-cell statistics (:199-251): weighted median and MAD over the cell's supports, sorted
//      with a stable insertion sort (libstdc++'s std::sort is an insertion sort up to 16
//      elements, so the order -- and hence every float sum -- is the reference's whenever a cell
//      holds at most 16 supports, i.e. for every image of 500 or more cells);
//   4. grid hole filling (:253-301): Jacobi sweeps inside one CTA until nothing changes;
//   5. per pixel (:303-412): bilinear prior, then the adaptive search range written to the
//      range planes.
// Float expressions keep the reference order with explicitly rounded intrinsics.
#include "engine.h"

namespace apgcu {

namespace {

struct Support { int x, y; float d, conf; };

constexpr int kCell = 16;

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float stdmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float stdmax(float a, float b) { return (a < b) ? b : a; }

template <bool C64>
__global__ void prior_cand_kernel(CostCtx c, int gw, int n_cells, int max_cand, int tex_thr, float uniq_ratio,
                                  int lr_max, Support* __restrict__ cand, int* __restrict__ ncand) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n_cells) return;
    const int ci = warp, gx = ci % gw, gy = ci / gw;
    const int w = c.w, h = c.h, d0 = c.d0, d1 = c.d0 + c.D;
    const int y_min = max(2, gy * kCell), y_max = min(h - 2, (gy + 1) * kCell);
    const int y_start = (y_min % 2 != 0) ? y_min + 1 : y_min;
    const int x_min = max(2, gx * kCell), x_max = min(w - 2, (gx + 1) * kCell);
    const int x_start = (x_min % 2 != 0) ? x_min + 1 : x_min;
    const int nxs = x_max > x_start ? (x_max - x_start + 1) / 2 : 0;
    const int nys = y_max > y_start ? (y_max - y_start + 1) / 2 : 0;
    const int npos = nxs * nys;
    int count = 0;
    for (int base = 0; base < npos && count < max_cand; base += 32) {
        const int j = base + lane;
        bool pass = false;
        Support m{0, 0, 0.f, 0.f};
        if (j < npos) {
            const int x = x_start + 2 * (j % nxs), y = y_start + 2 * (j / nxs);
            const int row = y * w;
            const int tex = (int)c.lgx[row + x] + (int)c.lgy[row + x];
            if (tex >= tex_thr) {
                int best_d = d0, best = 255, second = 255;
                const uint32_t cl = C64 ? 0u : c.cl[row + x];
                const unsigned long long cl64 = C64 ? c.cl64[row + x] : 0ull;
                for (int d = d0; d < d1; ++d) {
                    const int xr = x - d;
                    if (xr < 0 || xr >= w) continue;
                    const int cc = C64 ? __popcll(cl64 ^ c.cr64[row + xr]) : __popc(cl ^ c.cr[row + xr]);
                    if (cc < best) { second = best; best = cc; best_d = d; }
                    else if (cc < second) second = cc;
                }
                if (second > 0) {
                    const float uniq = __fdiv_rn((float)(second - best), (float)second);
                    const int xr = x - best_d;
                    if (!(uniq < uniq_ratio) && xr >= 1 && xr < w - 1) {
                        int rbest = 255, rbest_d = 0;
                        const uint32_t cr = C64 ? 0u : c.cr[row + xr];
                        const unsigned long long cr64 = C64 ? c.cr64[row + xr] : 0ull;
                        for (int d = d0; d < d1; ++d) {
                            const int xl = xr + d;
                            if (xl < 0 || xl >= w) continue;
                            const int cc = C64 ? __popcll(c.cl64[row + xl] ^ cr64) : __popc(c.cl[row + xl] ^ cr);
                            if (cc < rbest) { rbest = cc; rbest_d = d; }
                        }
                        if (abs(rbest_d - best_d) <= lr_max) {
                            pass = true;
                            m = Support{x, y, (float)best_d, uniq};
                        }
                    }
                }
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, pass);
        const int idx = count + __popc(mask & ((1u << lane) - 1u));
        if (pass && idx < max_cand) cand[(size_t)ci * max_cand + idx] = m;
        count += __popc(mask);
    }
    if (lane == 0) ncand[ci] = min(count, max_cand);
}

// Block-wide exclusive scan of flags[0..n) into out[0..n); returns the total (all threads).
__device__ int block_scan(const int* flags, int* out, int n, int* s_warp) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    int carry = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + tid;
        const int v = i < n ? flags[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) s_warp[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int y = lane < nw ? s_warp[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += t;
            }
            if (lane < nw) s_warp[lane] = y;  // inclusive warp totals
        }
        __syncthreads();
        const int before = (wid > 0 ? s_warp[wid - 1] : 0) + carry;
        if (i < n) out[i] = before + x - v;
        const int total = s_warp[nw - 1];
        __syncthreads();
        carry += total;
    }
    return carry;
}

__global__ void __launch_bounds__(1024) prior_select_kernel(int n_cells, int hard_max, const int* __restrict__ ncand,
                                                            int* __restrict__ taken, int* __restrict__ list,
                                                            int* __restrict__ tmpA, int* __restrict__ tmpB,
                                                            int* __restrict__ count_out) {
    __shared__ int s_warp[32];
    __shared__ int s_int[4];
    const int tid = threadIdx.x;
    for (int i = tid; i < n_cells; i += blockDim.x) { tmpA[i] = ncand[i] > 0; taken[i] = 0; }
    __syncthreads();
    const int nne = block_scan(tmpA, tmpB, n_cells, s_warp);
    for (int i = tid; i < n_cells; i += blockDim.x)
        if (ncand[i] > 0) list[tmpB[i]] = i;
    __syncthreads();
    if (nne <= hard_max) {
        const int base_quota = max(1, hard_max / max(1, nne));
        // pass 1: each non-empty cell in order takes min(base_quota, n), capped by the budget
        for (int k = tid; k < nne; k += blockDim.x) tmpA[k] = min(base_quota, ncand[list[k]]);
        __syncthreads();
        const int t1 = block_scan(tmpA, tmpB, nne, s_warp);
        for (int k = tid; k < nne; k += blockDim.x) {
            const int got = max(0, min(tmpA[k], hard_max - tmpB[k]));
            taken[list[k]] = got;
        }
        __syncthreads();
        int out = min(t1, hard_max);
        // pass 2: round-robin rounds over cells with remaining candidates
        for (int r = 0; out < hard_max; ++r) {
            for (int k = tid; k < nne; k += blockDim.x) {
                const int j = list[k];
                tmpA[k] = (ncand[j] - taken[j]) > 0 ? 1 : 0;
            }
            __syncthreads();
            const int E = block_scan(tmpA, tmpB, nne, s_warp);
            if (E == 0) break;
            const int budget = hard_max - out;
            for (int k = tid; k < nne; k += blockDim.x)
                if (tmpA[k] && tmpB[k] < budget) taken[list[k]] += 1;
            __syncthreads();
            out += min(E, budget);
        }
        if (tid == 0) s_int[0] = out;
    } else {
        for (int k = tid; k < hard_max; k += blockDim.x) {
            const int j = list[(int)(((unsigned long long)k * (unsigned long long)nne) / (unsigned long long)hard_max)];
            taken[j] = 1;  // nne > hard_max: sample indices are strictly increasing, each cell once
        }
        if (tid == 0) s_int[0] = hard_max;
    }
    __syncthreads();
    if (tid == 0) count_out[0] = s_int[0];
}

struct Grid { float *d, *c, *s, *mn, *mx; };

__device__ void sort_pairs(float2* a, int n) {
    for (int i = 1; i < n; ++i) {
        const float2 v = a[i];
        int j = i - 1;
        while (j >= 0 && v.x < a[j].x) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
}

__global__ void prior_cell_kernel(int n_cells, int max_cand, const Support* __restrict__ cand,
                                  const int* __restrict__ taken, float2* __restrict__ scratch, Grid g) {
    const int ci = blockIdx.x * blockDim.x + threadIdx.x;
    if (ci >= n_cells) return;
    const int m = taken[ci];
    g.d[ci] = -1.f; g.c[ci] = 0.f; g.s[ci] = -1.f; g.mn[ci] = -1.f; g.mx[ci] = -1.f;
    if (m == 0) return;
    float2* pts = scratch + (size_t)ci * max_cand * 2;
    float2* devs = pts + max_cand;
    for (int k = 0; k < m; ++k) pts[k] = make_float2(cand[(size_t)ci * max_cand + k].d, cand[(size_t)ci * max_cand + k].conf);
    sort_pairs(pts, m);
    const float mn = pts[0].x, mx = pts[m - 1].x;
    g.mn[ci] = mn;
    g.mx[ci] = mx;
    const float intra_span = __fsub_rn(mx, mn);
    float total_w = 0.f;
    for (int k = 0; k < m; ++k) total_w = __fadd_rn(total_w, pts[k].y);
    if (total_w <= 1e-6f) return;
    const float half_w = __fmul_rn(total_w, 0.5f);
    float cur_w = 0.f, d_med = pts[0].x;
    for (int k = 0; k < m; ++k) {
        cur_w = __fadd_rn(cur_w, pts[k].y);
        if (cur_w >= half_w) { d_med = pts[k].x; break; }
    }
    g.d[ci] = d_med;
    for (int k = 0; k < m; ++k) devs[k] = make_float2(fabsf(__fsub_rn(pts[k].x, d_med)), pts[k].y);
    sort_pairs(devs, m);
    cur_w = 0.f;
    float dev_med = devs[0].x;
    for (int k = 0; k < m; ++k) {
        cur_w = __fadd_rn(cur_w, devs[k].y);
        if (cur_w >= half_w) { dev_med = devs[k].x; break; }
    }
    g.s[ci] = stdmax(__fmul_rn(dev_med, 1.4826f), __fmul_rn(intra_span, 0.5f));
    const float mean_conf = __fdiv_rn(total_w, (float)m);
    const float count_factor = clampf(__fdiv_rn((float)m, 3.f), 0.3f, 1.f);
    g.c[ci] = clampf(__fmul_rn(mean_conf, count_factor), 0.f, 1.f);
}

__global__ void __launch_bounds__(1024) prior_fill_kernel(int gw, int gh, Grid a, Grid b, int* __restrict__ which) {
    const int n = gw * gh;
    Grid cur = a, nxt = b;
    int sel = 0;
    const int max_iters = max(gw, gh);
    for (int iter = 0; iter < max_iters; ++iter) {
        int changed = 0;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int gx = i % gw, gy = i / gw;
            float od = cur.d[i], oc = cur.c[i], os = cur.s[i], omn = cur.mn[i], omx = cur.mx[i];
            if (od < 0.f) {
                float ad = 0.f, ac = 0.f, as = 0.f, ww = 0.f, cmin = 1e9f, cmax = -1e9f;
                for (int oy = -1; oy <= 1; ++oy)
                    for (int ox = -1; ox <= 1; ++ox) {
                        const int nx = gx + ox, ny = gy + oy;
                        if (nx < 0 || ny < 0 || nx >= gw || ny >= gh) continue;
                        const int ni = ny * gw + nx;
                        const float v = cur.d[ni];
                        if (v < 0.f) continue;
                        ad = __fadd_rn(ad, v);
                        ac = __fadd_rn(ac, cur.c[ni]);
                        as = __fadd_rn(as, cur.s[ni] >= 0.f ? cur.s[ni] : 8.f);
                        cmin = stdmin(cmin, cur.mn[ni] >= 0.f ? cur.mn[ni] : v);
                        cmax = stdmax(cmax, cur.mx[ni] >= 0.f ? cur.mx[ni] : v);
                        ww = __fadd_rn(ww, 1.f);
                    }
                if (ww > 0.f) {
                    od = __fdiv_rn(ad, ww);
                    oc = __fmul_rn(__fdiv_rn(ac, ww), 0.85f);
                    os = __fdiv_rn(as, ww);
                    omn = cmin;
                    omx = cmax;
                    changed = 1;
                }
            }
            nxt.d[i] = od; nxt.c[i] = oc; nxt.s[i] = os; nxt.mn[i] = omn; nxt.mx[i] = omx;
        }
        const int any = __syncthreads_or(changed);
        const Grid t = cur; cur = nxt; nxt = t;
        sel ^= 1;
        if (!any) break;
    }
    if (threadIdx.x == 0) which[0] = sel;
}

__global__ void prior_pixel_kernel(int w, int h, int gw, int gh, Grid a, Grid b, const int* __restrict__ which,
                                   const int* __restrict__ count, int min_supports, int default_R, int global_D,
                                   int gmin, int gmax, float* __restrict__ d_prior, int16_t* __restrict__ rmin,
                                   int16_t* __restrict__ rmax) {
    const int n = w * h;
    const bool use = count[0] >= min_supports;
    const Grid g = which[0] ? b : a;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!use) { d_prior[p] = -1.f; continue; }
        const int y = p / w, x = p - y * w;
        const float fy = __fsub_rn(__fdiv_rn(__fadd_rn((float)y, 0.5f), (float)kCell), 0.5f);
        const int gy = min(max((int)floorf(fy), 0), gh - 1);
        const int gy1 = min(gy + 1, gh - 1);
        const float ty = clampf(__fsub_rn(fy, (float)gy), 0.f, 1.f);
        const float fx = __fsub_rn(__fdiv_rn(__fadd_rn((float)x, 0.5f), (float)kCell), 0.5f);
        const int gx = min(max((int)floorf(fx), 0), gw - 1);
        const int gx1 = min(gx + 1, gw - 1);
        const float tx = clampf(__fsub_rn(fx, (float)gx), 0.f, 1.f);
        const int i00 = gy * gw + gx, i10 = gy * gw + gx1, i01 = gy1 * gw + gx, i11 = gy1 * gw + gx1;
        const float d00 = g.d[i00], d10 = g.d[i10], d01 = g.d[i01], d11 = g.d[i11];
        auto pick = [](float v) { return v < 0.f ? 0.f : v; };
        auto wgt = [](float v) { return v < 0.f ? 0.f : 1.f; };
        const float omx = __fsub_rn(1.f, tx), omy = __fsub_rn(1.f, ty);
        const float w00 = __fmul_rn(__fmul_rn(omx, omy), wgt(d00));
        const float w10 = __fmul_rn(__fmul_rn(tx, omy), wgt(d10));
        const float w01 = __fmul_rn(__fmul_rn(omx, ty), wgt(d01));
        const float w11 = __fmul_rn(__fmul_rn(tx, ty), wgt(d11));
        const float ww = __fadd_rn(__fadd_rn(__fadd_rn(w00, w10), w01), w11);
        if (!(ww > 1e-6f)) { d_prior[p] = -1.f; continue; }
        auto wsum = [&](float v00, float v10, float v01, float v11) {
            return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w00, v00), __fmul_rn(w10, v10)), __fmul_rn(w01, v01)),
                             __fmul_rn(w11, v11));
        };
        const float dp = __fdiv_rn(wsum(pick(d00), pick(d10), pick(d01), pick(d11)), ww);
        d_prior[p] = dp;
        const float conf = __fdiv_rn(wsum(g.c[i00], g.c[i10], g.c[i01], g.c[i11]), ww);
        float cmin = 1e9f, cmax = -1e9f;
        const int idx[4] = {i00, i10, i01, i11};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int q = idx[k];
            const float dq = g.d[q];
            if (dq >= 0.f) {
                const float mn = g.mn[q] >= 0.f ? g.mn[q] : dq;
                const float mx = g.mx[q] >= 0.f ? g.mx[q] : dq;
                cmin = stdmin(cmin, mn);
                cmax = stdmax(cmax, mx);
            }
        }
        const float spread = __fdiv_rn(wsum(pick(g.s[i00]), pick(g.s[i10]), pick(g.s[i01]), pick(g.s[i11])), ww);
        const float pmn_v = (cmin <= cmax) ? stdmin(cmin, dp) : dp;
        const float pmx_v = (cmin <= cmax) ? stdmax(cmax, dp) : dp;
        // apply_search_range, :379-409
        const float pmin = pmn_v >= 0.f ? pmn_v : dp;
        const float pmax = pmx_v >= 0.f ? pmx_v : dp;
        int R = default_R;
        if (conf < 0.25f) R = global_D;
        else if (conf > 0.85f && spread < 1.5f) R = 8;
        else if (conf > 0.60f && spread < 3.0f) R = __float2int_rz(__fadd_rn(__fadd_rn(12.f, __fmul_rn(1.5f, spread)), 0.5f));
        else if (conf > 0.40f && spread < 6.0f) R = __float2int_rz(__fadd_rn(__fadd_rn(18.f, __fmul_rn(2.0f, spread)), 0.5f));
        else R = max(24, __float2int_rz(__fadd_rn(__fadd_rn(16.f, __fmul_rn(2.0f, spread)), 0.5f)));
        R = min(R, global_D);
        const int bound_lo = (int)floorf(pmin) - 4;
        const int bound_hi = (int)ceilf(pmax) + 4 + 1;
        int lo = min((int)floorf(dp) - R, bound_lo);
        int hi = max((int)ceilf(dp) + R + 1, bound_hi);
        hi = min(hi, x + 1);
        lo = max(lo, gmin);
        hi = min(hi, gmax);
        if (hi < lo) hi = lo;
        rmin[p] = (int16_t)lo;
        rmax[p] = (int16_t)hi;
    }
}

}  // namespace

cudaError_t launch_prior(const apg_pipeline_config_t& cfg, const CostCtx& c, const Layout& L, unsigned char* arena,
                         cudaStream_t s, unsigned* launches) {
    Support* cand = reinterpret_cast<Support*>(arena + L.pr_cand);
    int* ncand = reinterpret_cast<int*>(arena + L.pr_ncand);
    int* tk = reinterpret_cast<int*>(arena + L.pr_taken);
    int* taken = tk;
    int* list = tk + L.n_cells;
    int* tmpA = tk + 2 * L.n_cells;
    int* tmpB = tk + 3 * L.n_cells;
    int* cnt = reinterpret_cast<int*>(arena + L.pr_count);
    float* gbase = reinterpret_cast<float*>(arena + L.pr_grid);
    Grid ga{gbase, gbase + L.n_cells, gbase + 2 * L.n_cells, gbase + 3 * L.n_cells, gbase + 4 * L.n_cells};
    Grid gb{gbase + 5 * L.n_cells, gbase + 6 * L.n_cells, gbase + 7 * L.n_cells, gbase + 8 * L.n_cells,
            gbase + 9 * L.n_cells};
    const int threads = 256;
    const int blocks = (L.n_cells * 32 + threads - 1) / threads;
    if (c.census64)
        prior_cand_kernel<true><<<blocks, threads, 0, s>>>(c, L.gw, L.n_cells, L.max_cand, cfg.prior_texture_threshold,
                                                           cfg.prior_uniqueness_ratio, cfg.prior_lr_max_diff, cand, ncand);
    else
        prior_cand_kernel<false><<<blocks, threads, 0, s>>>(c, L.gw, L.n_cells, L.max_cand, cfg.prior_texture_threshold,
                                                            cfg.prior_uniqueness_ratio, cfg.prior_lr_max_diff, cand, ncand);
    prior_select_kernel<<<1, 1024, 0, s>>>(L.n_cells, cfg.prior_max_supports, ncand, taken, list, tmpA, tmpB, cnt);
    prior_cell_kernel<<<(L.n_cells + 127) / 128, 128, 0, s>>>(L.n_cells, L.max_cand, cand, taken,
                                                              reinterpret_cast<float2*>(arena + L.pr_scratch), ga);
    prior_fill_kernel<<<1, 1024, 0, s>>>(L.gw, L.gh, ga, gb, cnt + 1);
    const int n = L.w * L.h;
    prior_pixel_kernel<<<min((n + 255) / 256, 148 * 8), 256, 0, s>>>(
        L.w, L.h, L.gw, L.gh, ga, gb, cnt + 1, cnt, cfg.prior_min_supports, cfg.prior_search_radius,
        cfg.max_disparity - cfg.min_disparity, cfg.min_disparity, cfg.max_disparity,
        reinterpret_cast<float*>(arena + L.d_prior), reinterpret_cast<int16_t*>(arena + L.rmin),
        reinterpret_cast<int16_t*>(arena + L.rmax));
    *launches += 5;
    return cudaGetLastError();
}

}  // namespace apgcu

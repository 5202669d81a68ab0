// Host-side launch interface of the apg-sgm sm_100a kernels (internal to the library).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "apg_sgm/pipeline_config.h"

namespace apgcu {

// aux.cu
// One image's input and aux planes (gray, |gx|, |gy|, census 32 or 64 bits).
struct AuxImage {
    const uint8_t* src;
    int stride;
    uint8_t *gray, *gx, *gy;
    uint32_t* census;
    unsigned long long* census64;
};
cudaError_t launch_aux(const AuxImage& left, const AuxImage& right, int ch, int w, int h, int census64,
                       cudaStream_t s);
// One image (the host path runs the left image's while the right one is still being uploaded).
cudaError_t launch_aux_one(const AuxImage& im, int ch, int w, int h, int census64, cudaStream_t s);

// cost.cu: mode 0 raw volume, 1 cross-H volume, 2 right argmin only; all update rkey.
// Pixel-run form of the cost kernel (32-bit census, default ranges); launch_cost uses it where
// cost_runs_supported holds.
bool cost_runs_supported(const CostCtx& c, int mode, int lmax);
size_t cost_runs_smem_bytes(const CostCtx& c, int mode, int lmax);
cudaError_t launch_cost_runs(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                             const uint32_t* magic, cudaStream_t s);
cudaError_t launch_cost(const CostCtx& c, int mode, int lmax, int tau, uint32_t* vol, uint32_t* rkey,
                        const uint32_t* magic, cudaStream_t s);
size_t cost_kernel_smem_bytes(int D, int Dp, int lmax, bool cross, bool census64);
cudaError_t launch_right_wta_finalize(const CostCtx& c, const uint32_t* rkey, int subpixel, float* disp_right,
                                      cudaStream_t s);

// hier.cu: the hierarchical search range around the half-size pass (Engine::run_hier).
cudaError_t launch_hier_downsample(const uint8_t* lg, const uint8_t* rg, int w, int h, uint8_t* cl, uint8_t* cr,
                                   cudaStream_t s);
cudaError_t launch_hier_range(const apg_pipeline_config_t& c, int w, int h, const float* coarse_disp,
                              const float* coarse_conf, int16_t* rmin, int16_t* rmax, float* d_prior,
                              unsigned long long* counts, cudaStream_t s);

// cross.cu.  out8: cout is the byte volume (Dp bytes per pixel, 0xFF invalid; every valid
// aggregated cost below 255).
cudaError_t launch_cross_v(int w, int h, int d0, int D, int Dp, int lmax, int tau, const uint8_t* gray,
                           const int16_t* rmin, const int16_t* rmax, const uint32_t* tin, uint32_t* cout,
                           const uint32_t* magic, bool default_ranges, bool out8, cudaStream_t s);
cudaError_t launch_cross_h(int w, int h, int d0, int D, int Dp, int lmax, int tau, const uint8_t* gray,
                           const int16_t* rmin, const int16_t* rmax, const uint32_t* vin, uint32_t* vout,
                           const uint32_t* magic, cudaStream_t s);
size_t cross_v_smem_bytes(int Dp, int lmax);

// sgm.cu
struct SgmLaunch {
    int w, h, d0, D, Dp;
    SgmPen pen;
    const uint8_t* gray;
    const uint32_t* cvol;  // nullptr -> census source (cl, cr, qlut; default search range only)
    const uint32_t* cl;
    const uint32_t* cr;
    const uint16_t* qlut;
    float* disp;
    float* best;
    float* second;
    int subpixel;
    int sp_method = 0;    // sub-pixel method of the WTA (subpixel_delta), 0 = Legacy
    float sp_param = 0.0f;
    apg_subpixel_telemetry_t* sp_tel = nullptr;  // telemetry counters (ExperimentalSubpixelScope), or none
    int store_final;  // last sweep: also write the final sum into in[0] (stage dumps)
    int lanes;        // lanes per scanline chain (8, 16, 32; 0 = default for Dp)
    int split = 0;    // volume-fed last sweep over two warps per chain: 0 = where it pays (Dp 64),
                      // 1 = never, 2 = always (32 lanes per chain only)
    int cost8 = 0;    // cvol holds one byte per voxel, 0xFF invalid (32 lanes, Dp 128 or 256)
};
// First phase: ndir directions in one launch, direction i writing its path values to out[i].
cudaError_t launch_sgm_first(const SgmLaunch& l, int ndir, const int (*dirs)[2], uint32_t* const* out,
                             cudaStream_t s);
// Last sweep (dx, dy): adds the nin (1 or 3) partial sums in[] and writes the WTA maps.
cudaError_t launch_sgm_last(const SgmLaunch& l, int dx, int dy, int nin, const uint32_t* const* in, cudaStream_t s);
// The last sweep's steps [t_begin, t_end) only (t_begin a multiple of 32), the chains' state
// between bands in `carry` (32 * (Dp / 64 + 1) words per chain): one warp per chain, volume-fed,
// three partial sums, Dp 128 / 192 / 256.  A sequence of bands covering every step gives the maps of
// launch_sgm_last.
bool sgm_last_band_supported(const SgmLaunch& l, int nin);
cudaError_t launch_sgm_last_band(const SgmLaunch& l, int dx, int dy, int nin, const uint32_t* const* in, int t_begin,
                                 int t_end, uint32_t* carry, cudaStream_t s);
// bufs[0] += bufs[1..6] (saturating u16 lanes), `words` 32-bit words each.
// Path8: adds bufs[1 .. nbuf) into bufs[0] (nbuf 5 or 7), saturating per halfword.
cudaError_t launch_sgm_fold(uint32_t* const* bufs, int nbuf, size_t words, cudaStream_t s);
int sgm_lanes_for(int Dp, int requested);

// Batches: the SGM of many pairs (Dp 64, 128, 192 or 256), volume-fed, in two persistent launches
// (every pair's first-phase directions, then every pair's last sweep + WTA).
struct SgmBatchPlan {
    int npairs = 0, nsbuf = 0, Dp = 0, lanes = 32;  // Dp: the widest pair's padded range
    bool mixed = false;                              // pairs of different Dp (one launch per phase all the same)
    int nseg_first = 0, total_first = 0, nseg_last = 0, total_last = 0;
    std::vector<size_t> words;  // per pair: 32-bit words of one path-sum buffer
    void* dev = nullptr;
    size_t off_first = 0, off_last = 0, off_queue = 0;
    std::vector<uint32_t*> sums;  // npairs x nsbuf path-sum buffers
};
bool sgm_batch_supported(int Dp);
// pl[i]: pair i's launch arguments; sbufs[i*nsbuf + d]: its path-sum buffers (nsbuf 3 or 7);
// lanes: 16 or 32 lanes per chain.  Pairs may differ in size and, with 32 lanes, in padded range
// (Dp 64 .. 256): every phase is still one persistent launch whose warps take (pair, direction,
// scanline) units of every pair.  Uploads the work tables (synchronous).
cudaError_t sgm_batch_plan_create(const SgmLaunch* pl, uint32_t* const* sbufs, int npairs, int nsbuf, int lanes,
                                  SgmBatchPlan* plan);
void sgm_batch_plan_destroy(SgmBatchPlan* plan);
// max_blocks_per_sm caps the persistent grid (0 = as many as fit).
cudaError_t launch_sgm_batch(const SgmBatchPlan& plan, int max_blocks_per_sm, cudaStream_t s);

// post.cu
struct ConfLrArgs {
    int w, h;
    const float* disp;
    const float* disp_right;
    const float* best;
    const float* second;
    const uint8_t* lgx;
    const uint8_t* lgy;
    float uniqueness_ratio, min_texture, reliable_threshold;
    int conf_lr_max_diff;
    float* confidence;
    uint8_t* reliable;
    uint8_t* reason;
    int fuse_lr, lr_check, post_lr_max_diff;
    float* disp_out;
};
cudaError_t launch_conf_lr(const ConfLrArgs& a, cudaStream_t s);
cudaError_t launch_lr(int w, int h, int lr_max_diff, const float* dr, const float* din, float* dout,
                      uint8_t* reason, cudaStream_t s);
cudaError_t launch_fill(int w, int h, int gap, int shadow, apg_inpaint_telemetry_t* tel, const float* in,
                        const uint8_t* reason, const uint8_t* gray,
                        const float* d_prior, float* out, cudaStream_t s);
cudaError_t launch_median(int w, int h, int r, const float* in, float* out, cudaStream_t s);
// Rows [y_begin, y_end) only: the ballot fill (gap >= 0) and the 3x3 median; the rows they read
// around the range (one above and one below) must be final.
cudaError_t launch_fill_rows(int w, int h, int y_begin, int y_end, int gap, int shadow, const float* in,
                             const uint8_t* reason, const uint8_t* gray, const float* d_prior, float* out,
                             cudaStream_t s);
cudaError_t launch_median3_rows(int w, int h, int y_begin, int y_end, const float* in, float* out, cudaStream_t s);
cudaError_t launch_frame_stats(int n, const float* disp, const uint8_t* reliable, const uint8_t* reason,
                               const float* before, const float* after, const int16_t* rmin, const int16_t* rmax,
                               unsigned long long range_sum, unsigned long long* out5, cudaStream_t s);

// range.cu (default range, HQ prior, refine)
cudaError_t launch_default_range(int w, int h, int d0, int dmax, int16_t* rmin, int16_t* rmax, cudaStream_t s);

}  // namespace apgcu

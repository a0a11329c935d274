/*
 * Internal declarations shared by the CUDA kernels and the C-ABI layer of
 * the B200-native HPM-MVS PatchMatch path.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "hpm_b200.h"

namespace hpm {

constexpr int kMaxViews = HPM_MAX_IMAGES; /* reference + 32 sources */
constexpr int kMaxSrc = kMaxViews - 1;
constexpr int kTaps = 36; /* 6 x 6 taps of the 11x11 window, stride 2 */
constexpr int kCandRows = 14;  /* 8 NESP directions + 5 refinement candidates + 1 network proposal */
constexpr int kRefineRow = 8; /* first refinement row */

/* Per-view data of one problem, passed to kernels by value. */
struct ViewDev {
    const float *img;        /* h x w gray, linear (reference-window and JBU loads) */
    const float *depth;      /* geometric-consistency depth map or nullptr */
    cudaTextureObject_t tex; /* same image as a float cudaArray texture: linear filter, clamped edges */
    int w, h;
};

/* Camera-pair quantities that do not depend on the hypothesis, computed on
 * the device with the reference's own expressions (HPM.cu:229-255). */
struct PairGeom {
    float Rrel[9];
    float trel[3];
};

/* Everything a PatchMatch kernel needs, passed by value (CUDA 12.1+ allows
 * kernel parameter blocks larger than 4 KB). */
struct PMArgs {
    int n; /* images */
    int W, H;
    int rows_cov; /* rows reached by the reference's checkerboard grid */
    float dmin, dmax;
    int geom, prior;
    uint32_t seed_lo, seed_hi, salt;
    int radius, radius_increment;
    float sigma_spatial, sigma_color;
    int top_k;
    int fix_quirks; /* HpmParams.fix_quirks */
    HpmCamera cam[kMaxViews];
    ViewDev view[kMaxViews];
    const PairGeom *pair; /* [n], entry 0 unused */
    float4 *planes;
    float *costs;
    uint32_t *views;
    const float4 *prior_planes;
    const uint32_t *masks;
    float *cost_cache; /* [S][colour][ceil(H*W/2)] cost vector of the current hypothesis, or nullptr */
    /* hand-off between the two kernels of a half-step (L2-resident):
     * cand_costs [kCandRows*S][ceil(H*W/2)] cost matrix rows (8 NESP
     * directions, the refinement candidates and the proposal), cand_pos
     * [8][ceil(H*W/2)] chosen sites, cand_flags [ceil(H*W/2)] row codes;
     * indexed by (y * W + x) >> 1, dense over the pixels of one colour */
    float *cand_costs;
    int *cand_pos;
    uint32_t *cand_flags;
    unsigned long long *counters; /* [2]: cost vectors, geom terms, or nullptr */
    /* prior-net form: per pixel a proposed plane (ref-frame normal, distance),
     * scored as one more refinement candidate; nullptr in the plain form */
    const float4 *proposals;
    /* HpmParams.variant 1 (ACMM+NESP): acmm selects its refinement kernel
     * (geometric weight 0.2 on the current and refined hypotheses, the
     * threshold rule of a hierarchy pass), geom_max the cap of the geometric
     * cost (5, or 3 in the variant); hier is HpmParams.hierarchy and
     * pre_costs its per-pixel acceptance threshold, written by the
     * initialisation */
    int acmm, hier;
    float geom_max;
    float *pre_costs;
};

/* Launchers (hpm_pm.cu / hpm_jbu.cu). All asynchronous on `s`. */
cudaError_t launch_pair_geom(const PMArgs &a, PairGeom *out, cudaStream_t s);
cudaError_t launch_init(const PMArgs &a, cudaStream_t s);
/* one red/black half-step; ww = pixels of one colour per warp row (4, 8 or 16) */
cudaError_t launch_propagate(const PMArgs &a, int iter, int color, cudaStream_t s, int ww = 8);
cudaError_t launch_depth_normal_filter(const PMArgs &a, float4 *planes, const float *costs, cudaStream_t s);
cudaError_t launch_cost_vectors(const PMArgs &a, const float4 *planes, float *out, cudaStream_t s);
cudaError_t launch_initial_costs(const PMArgs &a, const float4 *planes, float *cost, uint32_t *views,
                                 cudaStream_t s);
cudaError_t launch_geom_costs(const PMArgs &a, const float4 *planes, float *out, cudaStream_t s);
cudaError_t launch_tap_samples(const PMArgs &a, const float4 *planes, const int *pixels, int n, float *out,
                               int *inside, cudaStream_t s);
cudaError_t launch_jbu(const float *guide, int cols, int rows, const float *coarse_depth,
                       const float4 *coarse_normal, int s_cols, int s_rows, int image_scale, float *out_depth,
                       float4 *out_normal, cudaStream_t s);

int rows_covered(int H);

}  // namespace hpm

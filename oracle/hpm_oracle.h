/*
 * CPU oracle for the HPM-MVS PatchMatch hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the checker.
 * The product (hpm-mvs_b200/) never links or calls it.
 *
 * It restates, in plain C99 with FP32 arithmetic where the reference uses
 * FP32, the algorithm of the reference's HPM-MVS/HPM.cu (kernels) and the
 * host prior stages of HPM-MVS/HPM.cpp and main.cpp.  Every function cites
 * the reference lines it follows.  Two documented deviations:
 *   - Random numbers: the reference seeds curand XORWOW with clock64()
 *     (HPM.cu:521), so its runs are not reproducible.  The oracle and the
 *     CUDA product draw from the same counter-based Philox4x32-10 stream,
 *     in the reference's draw order, so that a stochastic half-step can be
 *     compared pixel by pixel.
 *   - Texture fetches: tex2D with cudaFilterModeLinear is emulated in
 *     software (bilinear weights quantised to 8 fractional bits, clamped
 *     edge addressing).  The quantisation rule is pinned against the
 *     hardware by tests/golden (fixtures produced by oracle/_ref, the
 *     reference's own HPM.cu compiled for sm_100a).
 */
#ifndef HPM_ORACLE_H
#define HPM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference's Camera (HPM-MVS/main.h:44-52). */
typedef struct {
    float K[9];
    float R[9];
    float t[3];
    int height;
    int width;
    float depth_min;
    float depth_max;
} OrCamera;

typedef struct {
    int geom_consistency; /* PatchMatchParams::geom_consistency */
    int planar_prior;     /* PatchMatchParams::planar_prior */
    float depth_min;      /* PatchMatchParams::depth_min (already x0.6) */
    float depth_max;      /* PatchMatchParams::depth_max (already x1.2) */
    uint64_t seed;        /* Philox key */
    uint32_t salt;        /* per-pass stream id */
    int half_steps;       /* propagation half-steps to run; the reference runs 6 */
    int finalize;         /* run GetDepthandNormal + the two filters */
    /* The ACMM+NESP variant (ACMM+NESP/windows/ACMM.cu) when variant is 1:
     * geometric weight 0.2 on the current and refined hypotheses and the
     * geometric cost capped at 3 (ACMM.cu:496, 651, 1596); no planar prior;
     * hierarchy 1 (an upsampled pass) or 2 (a pass at the size of the maps it
     * starts from) starts from the (world normal, depth) in planes_io, writes
     * the acceptance threshold of every pixel to pre_costs (caller's buffer,
     * W x H floats) and keeps an update only where its cost is 0.1 below it
     * (ACMM.cu:521-604, 1617-1629). */
    int variant;
    int hierarchy;
    float *pre_costs;
} OrRunOpts;

/* 0: bilinear weight = floor(frac * 256) / 256; 1: round-to-nearest. */
void or_set_tex_rounding(int mode);
int or_get_tex_rounding(void);

float or_tex2d(const float *img, int w, int h, float u, float v);
void or_homography(const OrCamera *ref, const OrCamera *src, const float *plane4, float *H9);

int or_cost_vectors(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float *out);
/* The cost vectors of or_cost_vectors and, per value, what an FP32
 * evaluation may differ by.  out_bound: the first-order effect of moving the
 * taps whose coordinates lie within k_err x their propagated rounding-error
 * bound of a 1/256 texture-weight step across it, or 2 where the centre's
 * in-image test or a variance cut may flip.  out_acc: twice the first-order
 * bound of the FP32 arithmetic on given samples: the accumulation error of
 * the window sums and a relative error of 1e-5 on every bilateral weight
 * (large in flat windows, where the variances cancel).  out_kind: bit 0 a tap lies near a
 * weight step, bit 1 a decision may flip. */
int or_ncc_bounds(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float k_err,
                  float *out_cost, float *out_bound, float *out_acc, int *out_kind);
/* The same at n_pixels listed pixels (index y * W + x): outputs [n_pixels][S]. */
int or_ncc_bounds_px(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float k_err,
                     const int *pixels, int n_pixels, float *out_cost, float *out_bound, float *out_acc, int *out_kind);
int or_initial_costs(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4,
                     float *out_cost, uint32_t *out_views);
int or_geom_costs(int n_img, const OrCamera *cams, const float *const *depths, const float *planes4, float *out);

/* HPM::RunPatchMatch (HPM.cu:1906-1957).  planes_io/costs_io hold the
 * hypothesis state carried between passes; views_out may be NULL. */
int or_run_patchmatch(int n_img, const float *const *imgs, const OrCamera *cams, const OrRunOpts *opts,
                      float *planes_io, float *costs_io, uint32_t *views_io, const float *prior_planes,
                      const uint32_t *plane_masks, const float *const *depth_maps);

int or_depth_normal_filter(const OrCamera *ref, float *planes_io, const float *costs);

int or_jbu(const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal, int s_cols,
           int s_rows, float *out_depth, float *out_normal);
/* The same weights at a given integer scale, also 1 (a 3 x 3 window): the
 * normal average with which the ACMM+NESP variant's hierarchy pass starts
 * (ACMM.cu:538-596) runs whatever the scale. */
int or_jbu_at_scale(const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal,
                    int s_cols, int s_rows, int image_scale, float *out_depth, float *out_normal);

/* Raw Philox4x32-10 block: ctr4 is replaced by the output. */
void or_philox4x32_10(uint32_t k0, uint32_t k1, uint32_t *ctr4);

/* Philox4x32-10 uniform in (0,1] for draw `n` of (pixel, step, salt). */
float or_philox_uniform(uint64_t seed, uint32_t pixel, uint32_t step, uint32_t salt, uint32_t n);

/* ---- host prior stages (HPM.cpp / main.cpp) ---- */

/* GetSupportPoints* (HPM.cpp:759-785, 1125-1179): xy pairs into out (capacity
 * max_points); returns the count. */
int or_support_points(const float *costs, int w, int h, int *out_xy, int max_points);

/* GetPriorPlaneParams_factor (HPM.cpp:811-844). */
void or_plane_from_triangle(const OrCamera *ref, const float *depth, int w, const int *tri6, float factor,
                            float *out4);

/* GetDepthFromPlaneParam_factor (HPM.cpp:846-849). */
float or_depth_from_plane(const OrCamera *ref, const float *plane4, int x, int y, float factor);

/* Triangle raster of main.cpp:96-116: writes idx+1 into mask for every kept
 * triangle, later triangles overwriting earlier ones; returns the number of
 * kept triangles and stores their vertex triples in kept6. */
int or_raster_triangles(const int *tris6, int n_tris, int w, int h, float *mask, int *kept6);
/* 6 nearest points per pixel (mask <= 0, or every pixel), brute force,
 * ties to the lower index: nn6[6 * (y * w + x) + k], -1 elsewhere. */
void or_knn6(const int *pts, int n_pts, int w, int h, const float *mask, int *nn6);

/* DepthsPredictSupplement (HPM.cpp:923-1097) with exact K=6 nearest
 * neighbours, ties to the lower support-point index (the reference uses PCL
 * KdTreeFLANN, an exact kd-tree search).  The neighbours come from a uniform
 * grid search (default) or a brute-force scan (or_set_knn_grid(0)); both are
 * exact and give identical results. */
void or_knn_supplement(const OrCamera *ref, const int *pts_xy, int n_pts, const float *depth, int w, int h,
                       float factor, float dmin, float dmax, float *plane_out4, float *mask);
void or_set_knn_grid(int on);

/* main.cpp:124-162 (coarse levels): prior depth and world normal at the
 * level's resolution from the triangle raster (mask > 0: triangle mask-1,
 * range widened to [0.6 dmin, 1.2 dmax]) and the KNN supplement (mask <
 * -200, range [dmin, dmax]); zero elsewhere. */
void or_prior_coarse(const OrCamera *ref, const float *mask, const float *tri_planes, int n_tri,
                     const float *knn_planes, int w, int h, float factor, float dmin, float dmax, float *out_depth,
                     float *out_normal3);

/* main.cpp:179-203: upsampled depth and world normal to ref-frame prior
 * planes (normal, distance to origin) and 0/1 masks. */
void or_prior_reload(const OrCamera *ref, const float *depth, const float *normal3, int w, int h, float dmin,
                     float dmax, float *out4, unsigned int *out_mask);

/* main.cpp:426-454 with CudaPlanarPriorInitializationSupplement
 * (HPM.cpp:1099-1123): full-scale prior planes, masks (triangle id or
 * 0xFFFFFF17 for KNN planes) and the prior depth map (depths_prior.dmb). */
void or_prior_full(const OrCamera *ref, const float *mask, const float *tri_planes, int n_tri,
                   const float *knn_planes, int w, int h, float dmin, float dmax, float *out4,
                   unsigned int *out_mask, float *out_depth);

/* ---- fusion (RunFusion, main.cpp:502-633) ---- */

/* Fused point cloud of a scene, sequentially as the reference: views in
 * problem order, pixels row by row, the masks of already fused source
 * pixels and the used_list that persists across the pixels of a view.
 * View v's maps (depth h*w, world normal 3 floats/pixel, BGR colour 3 bytes
 * per pixel) and camera match in size; problem p has reference ref_ids[p]
 * and src_counts[p] sources src_ids[p*32 + j] (view ids index the maps).
 * Writes up to cap points (xyz, normal, colour as floats in B, G, R order)
 * and returns the count (more than cap means the output was cut). */
long or_fuse(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
             const unsigned char *const *colors, int n_problems, const int *ref_ids, const int *src_counts,
             const int *src_ids, float *out_xyz, float *out_normal, float *out_color, long cap);
/* The same with the ACMM+NESP variant's rule (ACMM+NESP/windows/main.cpp:
 * 154-297): at least 2 consistent sources, and the point, normal and colour
 * are means over the reference pixel and the agreeing source pixels. */
long or_fuse_acmm(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
                  const unsigned char *const *colors, int n_problems, const int *ref_ids, const int *src_counts,
                  const int *src_ids, float *out_xyz, float *out_normal, float *out_color, long cap);
/* The mask-independent half of RunFusion for the reference view `ref` and
 * its ns sources srcs: pair_src / pair_w [pixel][ns] (source pixel index of
 * a consistent pair or -1, its exp(-error)), points [pixel][3] (the world
 * point of pixels with a positive depth). */
int or_fuse_pairs(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
                  int ref, int ns, const int *srcs, int *pair_src, float *pair_w, float *points);

#ifdef __cplusplus
}
#endif
#endif

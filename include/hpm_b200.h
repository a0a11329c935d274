/*
 * hpm_b200.h - C ABI of the B200-native HPM-MVS PatchMatch path.
 *
 * This is the drop-in boundary: plain pointers and sizes, no C++ or torch
 * types, status codes instead of exit().  Each entry point names the
 * reference interface it replaces (file:line in the HPM-MVS repository).
 *
 * Conventions (those of the reference's host buffers):
 *   images        float32, row-major [height][width], gray 0..255
 *                 (HPM.cpp:492-495 converts the uint8 image to float)
 *   planes        float32 x4 per pixel, row-major: during PatchMatch
 *                 (nx, ny, nz, dist) in the reference camera frame; after a
 *                 pass (world-frame normal, depth)  (HPM.cu:1751-1764)
 *   costs         float32 per pixel
 *   view masks    uint32 per pixel, bit i = source view i selected
 *   prior masks   uint32 per pixel, non-zero = a prior plane is present
 *
 * Every function returns HPM_OK (0) or a negative HpmStatus; the message of
 * the last failure of a context is available from hpm_last_error().
 * A context is used by one host thread at a time; all device work is issued
 * on the context's own CUDA stream.
 */
#ifndef HPM_B200_H
#define HPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HPM_OK = 0,
    HPM_ERR_ARG = -1,     /* invalid argument (null pointer, bad size, too many views) */
    HPM_ERR_CUDA = -2,    /* a CUDA runtime call failed */
    HPM_ERR_IO = -3,      /* a file could not be read or written */
    HPM_ERR_STATE = -4,   /* call out of order (e.g. run before set_views) */
    HPM_ERR_TIMEOUT = -5, /* a bounded device-side wait gave up */
    HPM_ERR_NOMEM = -6    /* device allocation failed */
} HpmStatus;

/* Maximum number of images of one problem: the reference view plus 32
 * sources (cost_vector[32], HPM.cu:402; 32-bit view masks, HPM.cu:55-63). */
#define HPM_MAX_IMAGES 33

/* Same layout as the reference's Camera (HPM-MVS/main.h:44-52). */
typedef struct {
    float K[9];
    float R[9];
    float t[3];
    int height;
    int width;
    float depth_min;
    float depth_max;
} HpmCamera;

/* Mirrors PatchMatchParams (HPM-MVS/HPM.h:29-46).  patch_size,
 * radius_increment, sigma_spatial, sigma_color and top_k keep the
 * reference's defaults (11, 2, 5, 3, 4); max_iterations is accepted but, as in
 * the reference (HPM.cu:1933), every pass runs 3 iterations unless
 * honour_max_iterations is set.
 *
 * fix_quirks = 0 (the default) keeps the reference's behaviour everywhere.
 * fix_quirks = 1 gives these places of the reference the behaviour their
 * code evidently intends (each changes results):
 *   - the right-far strip picks its minimum-cost site, like the other
 *     three strips (the reference keeps the maximum, HPM.cu:1330, 744);
 *   - an invalid direction scores 2 for every view (the reference's
 *     float cost_array[8][32] = { 2.0f } sets only [0][0], HPM.cu:1244);
 *   - the prior pass starts from the previous pass's normal rotated back
 *     to the reference frame (HPM.cu:547-551 reuses the world-frame one);
 *   - the refinement's perturbed depth is drawn again until it lies in the
 *     depth range, at most 8 draws (the reference's do-while never
 *     repeats, HPM.cu:1170-1172);
 *   - every row is propagated and filtered (the reference's grid skips the
 *     last row of an odd height, HPM.cu:1926).
 * Q6 (max_iterations ignored) has its own switch, honour_max_iterations. */
typedef struct {
    int max_iterations;
    int patch_size;
    int radius_increment;
    float sigma_spatial;
    float sigma_color;
    int top_k;
    float depth_min; /* already widened: cam depth_min * 0.6 (HPM.cpp:553) */
    float depth_max; /* already widened: cam depth_max * 1.2 (HPM.cpp:554) */
    int geom_consistency;
    int multi_geometry;
    int planar_prior;
    int honour_max_iterations; /* 0 = reference behaviour (always 3) */
    uint64_t seed;             /* Philox key of this pass's random stream */
    int fix_quirks;            /* 0 = the reference's behaviour (see above) */
    /* 0: the HPM-MVS kernels (HPM.cu).  1: the ACMM+NESP variant's kernels
     * (ACMM+NESP/windows/ACMM.cu, ACMM::RunPatchMatch at ACMM.cu:1810-1862):
     * max_iterations is honoured (ACMM.cu:1836), the geometric term weighs
     * the current and the refined hypotheses by 0.2 (ACMM.cu:651, 1596) and
     * the geometric cost is capped at 3 (ACMM.cu:496); no planar prior.  The
     * reference declares the plane that collects the winner without a value
     * (plane_hypotheses_now, ACMM.cu:1605) and reads it when no neighbour
     * wins; here it starts from the current hypothesis. */
    int variant;
    /* variant 1 only: PatchMatchParams::hierarchy (ACMM.h:50).  The pass
     * starts from the (world normal, depth) of hpm_set_hypotheses, upsampled
     * by the caller, and keeps a pixel's update only where its cost ends 0.1
     * below the initial cost of the plane with a zero normal and the depth
     * as its distance (the reference's half-filled array, ACMM.cpp:707-713,
     * ACMM.cu:596-597).  1: the maps were upsampled (params.upsample); 2: the
     * maps have the pass's size, where the reference leaves that threshold
     * unset (taken as 0: no update is kept). */
    int hierarchy;
} HpmParams;

/* Fills p with the reference defaults (HPM.h:29-46). */
void hpm_default_params(HpmParams *p);

typedef struct hpm_ctx hpm_ctx;

/* Creates a context on `device` (the reference hard-codes cudaSetDevice(0),
 * main.cpp:38).  Replaces the HPM constructor (HPM.cpp:99). */
int hpm_create(hpm_ctx **ctx, int device);
/* Frees every device buffer; replaces HPM::~HPM / Release*Memory
 * (HPM.cpp:101-133, 1283-1307). */
int hpm_destroy(hpm_ctx *ctx);
const char *hpm_last_error(const hpm_ctx *ctx);

/* Uploads the images and cameras of one problem, reference view first.
 * images[i] is cams[i].height x cams[i].width floats.  Replaces the texture
 * set-up of HPM::CudaSpaceInitialization (HPM.cpp:591-633); the 3200-pixel
 * cap of InuputInitialization (HPM.cpp:524-551) is the caller's job. */
int hpm_set_views(hpm_ctx *ctx, const float *const *images, const HpmCamera *cams, int num_images);

/* Depth maps of the reference and source views for the geometric-
 * consistency term (HPM.cpp:561-588, 635-660); depths[i] has the size of
 * cams[i] given to hpm_set_views. */
int hpm_set_geom_depths(hpm_ctx *ctx, const float *const *depths);

/* Seeds the hypothesis state (HPM.cpp:662-695: geometric passes load the
 * previous depths/normals/costs).  planes may hold (world normal, depth) as
 * written by a previous pass.  costs may be NULL (zeros). */
int hpm_set_hypotheses(hpm_ctx *ctx, const float *planes, const float *costs);

/* Planar prior of the next pass: per-pixel ref-frame plane (n, dist) and
 * mask.  Replaces ReloadPlanarPriorInitialization (HPM.cpp:901-921) and
 * CudaPlanarPriorInitializationSupplement (HPM.cpp:1099-1123). */
int hpm_set_prior(hpm_ctx *ctx, const float *prior_planes, const uint32_t *masks);
/* Drops the prior (HPM::ReleasePriorCudaMemory, HPM.cpp:1283-1286). */
int hpm_clear_prior(hpm_ctx *ctx);

/* One PatchMatch pass: initialisation, 3 red/black iterations, depth and
 * normal conversion, checkerboard median filter.  Replaces
 * HPM::RunPatchMatch (HPM.cu:1906-1957).  The hypothesis state stays on the
 * device for the next pass, as in the reference. */
int hpm_run_patchmatch(hpm_ctx *ctx, const HpmParams *params);

/* Parity entry point: the same pass cut after `half_steps` red/black
 * half-steps (the reference runs 6), with or without the depth/normal
 * conversion and filters.  Random streams match hpm_run_patchmatch: the k-th
 * pass of a problem (counting from hpm_set_views) draws from stream k. */
int hpm_run_partial(hpm_ctx *ctx, const HpmParams *params, int half_steps, int finalize);

/* Options of one ProcessProblem call. */
typedef struct {
    int planar_prior;     /* pass set A: plain pass, then the planar-prior pyramid */
    int geom_consistency; /* pass set B: one geometric-consistency pass */
    int multi_geometry;   /* second geometric iteration (reads depths_geom) */
    uint64_t seed;        /* Philox key of the passes of this problem */
    int pyramid_levels;   /* coarse prior levels; -1 = ComputingMultiScaleSettings
                             (HPM.cpp:851-860: halvings until max side <= 1000) */
    int fix_quirks;       /* HpmParams.fix_quirks of every pass; with 1 the coarse levels' triangle planes are
                             also range-checked against the pass's range instead of one widened once more
                             (main.cpp:129, 282) */
} HpmProblemOpts;

/* One reference view through ProcessProblem (main.cpp:35-499) on the
 * device: with planar_prior, the plain pass, then for each pyramid level
 * (ComputingMultiScaleSettings, HPM.cpp:851-860) support points, Delaunay
 * triangles, triangle planes and raster, the KNN supplement, (coarse levels)
 * joint bilateral upsampling, and a PatchMatch pass with the prior; with
 * geom_consistency, one geometric pass over the state and depth maps set by
 * hpm_set_hypotheses / hpm_set_geom_depths.  The depth range is the
 * reference camera's, widened x0.6 / x1.2 (HPM.cpp:553-554).  Outputs (any
 * may be NULL): depth and cost maps, world normals (3 floats per pixel), and
 * the full-scale prior depth map written to depths_prior.dmb by the
 * reference (zeros when no prior ran). */
int hpm_process_problem(hpm_ctx *ctx, const HpmProblemOpts *opts, float *depth, float *normal, float *cost,
                        float *prior_depth);
/* Options of a whole-scene run. */
typedef struct {
    int planar_prior;    /* pass set A with the planar-prior pyramid (the reference's default: 1) */
    int geom_iterations; /* geometric iterations of pass set B (the reference's default: 2) */
    uint64_t seed;
    int pyramid_levels; /* -1 = the reference's rule */
    int iterations;     /* prior-net forms only: PatchMatch iterations of each full-scale pass, the geometric
                           ones included (0 = 3, the reference's count; the plain form always runs 3) */
    int fix_quirks;     /* HpmProblemOpts.fix_quirks of every problem (0 = the reference's behaviour) */
    int geom_pass_iterations; /* prior-net forms only: PatchMatch iterations of each geometric pass
                                 (0 = as `iterations`) */
} HpmSceneOpts;

/* The reference's main() (main.cpp:636-677) over a scene: ProcessProblem
 * with the planar prior for every problem of pair.txt, then
 * geom_iterations geometric passes over every problem, the first reading
 * pass set A's depth maps, the later ones the geometric depth maps as they
 * are being updated (the reference rewrites depths_geom.dmb view by view).
 * All maps stay in HBM; the host only triangulates support points.
 * images[v] / cams[v] describe view v (host or device pointers); problem p
 * has reference ref_ids[p] and src_counts[p] sources
 * src_ids[p * (HPM_MAX_IMAGES-1) + j].  Per-view outputs (arrays of
 * n_views pointers, any may be NULL, host or device): final depth, world
 * normal (3 floats/pixel), cost. */
int hpm_run_scene(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams, int n_problems,
                  const int *ref_ids, const int *src_counts, const int *src_ids, const HpmSceneOpts *opts,
                  float *const *depths, float *const *normals, float *const *costs);
/* hpm_run_scene plus the two other maps the reference's ProcessProblem
 * writes per view in pass set A (main.cpp:481-497): pass_depths[v], the
 * depth map after pass set A (depths.dmb), and prior_depths[v], the
 * full-scale planar-prior depth (depths_prior.dmb; zeros without a prior).
 * Either array, and any entry, may be NULL. */
int hpm_run_scene_ex(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams,
                     int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                     const HpmSceneOpts *opts, float *const *depths, float *const *normals, float *const *costs,
                     float *const *pass_depths, float *const *prior_depths);
/* Options of the ACMM+NESP variant's scene run. */
typedef struct {
    int geom_iterations;     /* geometric iterations at every scale (the reference's: 2, main.cpp:319) */
    uint64_t seed;           /* problem p's k-th pass draws from key seed + 7919 p + k */
    int size_bound;          /* the coarsest scale has every longer side at most this (halvings of
                                the image, main.cpp:38-64); 0 = the reference's 1000 */
    int max_iterations;      /* PatchMatch iterations of the plain and hierarchy passes (0 = 3, ACMM.h:31) */
    int geom_max_iterations; /* of the geometric passes (0 = 2, ACMM.cpp:437) */
} HpmAcmmOpts;

/* The ACMM+NESP variant's main() (ACMM+NESP/windows/main.cpp:299-384) minus
 * fusion: NESP sampling inside ACMM's coarse-to-fine IMAGE pyramid.  Every
 * problem's views are scaled down until their longer side is at most
 * size_bound (ComputeMultiScaleSettings, main.cpp:35-71; images resized as
 * InuputInitialization does, ACMM.cpp:489-516, cameras scaled with them).
 * At the coarsest scale each problem runs a plain pass, then
 * geom_iterations geometric passes over all problems; at every finer scale
 * each problem's last geometric depth map is upsampled by the joint
 * bilateral filter (main.cpp:126-152), a hierarchy pass starts from it
 * (ACMM.cpp:663-719, HpmParams.hierarchy) and the geometric iterations
 * follow.  Passes use HpmParams.variant 1.  The maps stay in HBM between
 * passes (the reference writes .dmb files).  Problem p must have reference
 * view p (ref_ids[p] == p): the reference looks a source's scale up by its
 * image id (ACMM.cpp:490).  Views must be at most 3200 pixels on either
 * side (the cap of ACMM.cpp:448-516 is the caller's job, as for
 * hpm_run_scene), so the outputs have the input sizes.  Inputs and outputs
 * as hpm_run_scene (host or device pointers; any output may be NULL). */
int hpm_run_scene_acmm(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams,
                       int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                       const HpmAcmmOpts *opts, float *const *depths, float *const *normals, float *const *costs);

/* Host threads of hpm_run_scene's pass set A (1 or 2, default 2; no
 * counterpart in the reference).  With 2, pass set A's problems go to this
 * context and a second one on the same device (created on first use, freed
 * with this one; it holds its own working buffers, about as much device
 * memory again) from two host threads.  Only one thread's kernels run at a
 * time; the other thread may meanwhile triangulate support points on the
 * host, so the GPU does not wait for the Delaunay.  The maps do not depend on
 * the setting: each problem draws from its own seed.  The geometric
 * iterations always run on this context, problem after problem.  Counters
 * and CUDA-event profiles (hpm_count_*, hpm_profile_*) cover the work of
 * both contexts. */
int hpm_set_scene_workers(hpm_ctx *ctx, int workers);

/* Parity entry point: the prior of one pyramid level (0: 1/4 scale, 1: 1/2
 * scale, 2: full scale) built from given full-resolution maps of the current
 * reference view (depth, world normal 3 floats/pixel, cost) exactly as
 * hpm_process_problem builds it after a pass.  Outputs (any may be NULL):
 * ref-frame prior planes (4 floats/pixel) and masks of the next pass, and at
 * full scale the prior depth map (zeros at coarse levels). */
int hpm_prior_level(hpm_ctx *ctx, int level, const float *depth, const float *normal, const float *cost,
                    float *prior_planes, uint32_t *masks, float *prior_depth);
/* Support points and kept triangles of the last prior level built. */
int hpm_last_prior_stats(hpm_ctx *ctx, int *points, int *triangles);

/* Copies the pass result to the host: planes = (world normal, depth),
 * costs.  Either pointer may be NULL.  Replaces the D2H copies of
 * HPM.cu:1954-1955 and GetPlaneHypothesis / GetCost (HPM.cpp:739-747). */
int hpm_get_result(hpm_ctx *ctx, float *planes, float *costs);
/* Selected-view masks of the last pass (selected_views_cuda). */
int hpm_get_selected_views(hpm_ctx *ctx, uint32_t *views);

/* Device pointers of the state, for callers that keep data in HBM.
 * Valid until the next hpm_set_views with a larger size or hpm_destroy. */
int hpm_device_state(hpm_ctx *ctx, float **planes, float **costs, uint32_t **views);
/* The context's CUDA stream (cudaStream_t as void*). */
void *hpm_stream(hpm_ctx *ctx);

/* Joint bilateral upsampling of a coarse prior (depth + world normal) to the
 * guide's resolution.  Replaces HPM::JointBilateralUpsampling
 * (HPM.cpp:1215-1281) and JBU::CudaRun / JBU_cu (HPM.cu:1984-2088).
 * coarse_normal and out_normal are 3 floats per pixel.  Returns HPM_OK and
 * leaves the outputs untouched when the integer scale is 1 (HPM.cpp:1219). */
int hpm_jbu(hpm_ctx *ctx, const float *guide, int cols, int rows, const float *coarse_depth,
            const float *coarse_normal, int s_cols, int s_rows, float *out_depth, float *out_normal);

/* Joint bilateral upsampling that allocates nothing.  No counterpart in the
 * reference.  For callers that may not call cudaMalloc while they run (a host
 * that gives its whole device-memory budget to its own pool up front, or
 * that must not add a device synchronisation or a memory-accounting change
 * in its loop): no context is needed, every buffer is the caller's device
 * memory (guide cols x rows floats; coarse_depth s_cols x s_rows floats;
 * coarse_normal and out_normal 3 floats per pixel; out_depth cols x rows
 * floats), and the work is queued on `stream` (cudaStream_t as void*, NULL
 * for the default stream) of `device`.  Same computation as hpm_jbu.
 *
 * Its scratch is a fixed device array of HPM_JBU_NOALLOC_MAX_COARSE float4
 * (16 MiB) that every GPU using this library holds until the process exits;
 * coarse grids with more pixels are rejected with HPM_ERR_ARG.  The array
 * takes its device memory when CUDA loads the library's device code on the
 * device: under CUDA's default lazy module loading that is the first call of
 * this function there.  So make the first call on each device before the
 * caller reserves its memory budget and before any stream capture; later
 * calls allocate nothing.  All calls on a device share the array: calls that
 * overlap on the GPU (different streams, or different host threads) race and
 * must be ordered by the caller.  The caller's current device is restored
 * before returning.  Returns HPM_OK without touching the outputs when the
 * integer scale is 1, like hpm_jbu. */
#define HPM_JBU_NOALLOC_MAX_COARSE (1 << 20)
int hpm_jbu_noalloc(int device, const float *guide, int cols, int rows, const float *coarse_depth,
                    const float *coarse_normal, int s_cols, int s_rows, float *out_depth, float *out_normal,
                    void *stream);

/* ---- Proposal network of the prior-net form (no counterpart in the
 * reference).  Device pointers, work queued on `stream` (cudaStream_t as
 * void*, NULL for the default stream) of the current device. ---- */

/* Packs 3x3 weights [cout][cin][3][3] FP32 (PyTorch's OIHW) into the BF16
 * shared-memory image the convolution reads: 9 * cin * cout BF16 values.
 * mode 0: the layer's forward convolution; mode 1: its data-gradient
 * convolution (kernel flipped, cin and cout exchanged).  Channel counts 16 or
 * 32. */
int hpm_net_pack_weights(const float *weights, int cout, int cin, int mode, void *packed, void *stream);

/* 3x3 convolution, stride 1, zero padding 1, of an h x w NHWC BF16 image with
 * cin channels into cout channels, on the tensor cores (tcgen05, FP32
 * accumulation in TMEM).  epilogue 0: ReLU(acc + bias) as BF16; 1: acc + bias
 * as FP32; 2: acc where aux (NHWC BF16, cout channels) is > 0, else 0, as BF16
 * (the data gradient through the ReLU that produced aux).  use_tma selects
 * TMA staging of the input halo (else thread loads).  err (device int, may be
 * NULL) is set non-zero if a bounded wait ran out. */
int hpm_net_conv3x3(const void *x, int h, int w, int cin, const void *packed, const float *bias, int cout,
                    int epilogue, const void *aux, void *y, int use_tma, int *err, void *stream);

/* Trained weights of the proposal network, device pointers: per layer the
 * packed BF16 weights (hpm_net_pack_weights, mode 0) and the FP32 bias.
 * Layers: 16->32, 32->32, 32->32 (ReLU), 32->16 (linear head). */
typedef struct {
    const void *packed[4];
    const float *bias[4];
} HpmNetWeights;

/* hpm_run_scene_ex in the prior-net form.  Pass set A of each problem is: a
 * plain pass on 1/4-scale views, the coarse planar prior, the network's plane
 * per coarse pixel (from the coarse image, the pass's depth, normal and
 * confidence, and the prior's depth), then ONE full-scale prior pass whose
 * initial hypothesis is the network's proposal (upsampled by JBU) and whose
 * refinement scores the proposal as a sixth candidate with the unchanged NCC
 * cost; the planar prior is the coarse one, upsampled as the plain form's
 * coarsest level.  opts->pyramid_levels > 0 adds that many full-scale
 * prior passes, each with the planar prior rebuilt from the previous pass
 * (the plain form's finest level) and the proposal still a candidate.
 * opts->planar_prior == 2 makes the upsampled proposal itself the first
 * full-scale pass's planar prior instead of the coarse triangulation's.  The
 * geometric iterations are the plain form's. */
int hpm_run_scene_net(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams, int n_problems,
                      const int *ref_ids, const int *src_counts, const int *src_ids, const HpmSceneOpts *opts,
                      const HpmNetWeights *net, float *const *out_depths, float *const *out_normals,
                      float *const *out_costs);

/* hpm_run_scene in the batched form: every problem of the scene advances
 * together, one persistent launch per kernel and half-step covering the
 * tiles of all problems (of any sizes); a pass is captured once as a CUDA
 * graph and replayed; the half-step tile shape is tuned per view size.  Pass
 * set A equals hpm_process_problem's on a fresh context per problem; the
 * geometric iterations read the previous iteration's maps of every view
 * (the reference's in-place order, main.cpp:662-674, would serialise the
 * problems).  Keeps one context per problem inside ctx for later scenes. */
int hpm_run_scene_batched(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams,
                          int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                          const HpmSceneOpts *opts, float *const *out_depths, float *const *out_normals,
                          float *const *out_costs);
/* The batched prior-net form: hpm_run_scene_net's pass set A (options
 * alike) for every problem together: the 1/4-scale plain passes of all
 * problems in one batched pass, per problem the coarse planar prior and
 * the network, then the full-scale passes of all problems batched, each
 * scoring its problem's proposal; then the batched geometric iterations.
 * Pass set A equals hpm_run_scene_net's per problem bit for bit. */
int hpm_run_scene_batched_net(hpm_ctx *ctx, int n_views, const float *const *images, const HpmCamera *cams,
                              int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                              const HpmSceneOpts *opts, const HpmNetWeights *net, float *const *out_depths,
                              float *const *out_normals, float *const *out_costs);

/* The network's input for one problem (views as for hpm_set_views, full
 * scale): the coarse stage of the prior-net form (1/4-scale plain pass with
 * seed, coarse planar prior), written to x0 ([*ch][*cw][16] BF16, host or
 * device, at most cap_px pixels).  Leaves the coarse problem in the context. */
int hpm_net_coarse_inputs(hpm_ctx *ctx, int num_images, const float *const *images, const HpmCamera *cams,
                          uint64_t seed, void *x0, size_t cap_px, int *cw, int *ch);

/* Training targets of a view for the network, at the coarse size cw x ch:
 * the view's final depth and world normal (device), kept where the
 * multi-view test of RunFusion (main.cpp:575-612, without its
 * order-dependent masking) passes against the sources' maps (device
 * pointers); out: depth, reference-frame normal (3 floats) and mask per
 * coarse pixel (device). */
int hpm_net_targets(int device, const HpmCamera *ref_cam, const float *depth, const float *normal, int n_sources,
                    const HpmCamera *src_cams, const float *const *src_depths, const float *const *src_normals, int cw,
                    int ch, float *t_depth, float *t_normal, uint8_t *t_mask, void *stream);

/* Training loss of the head on n pixels (device buffers): masked relative
 * depth error plus lambda (1 - cos) of the normal; dy gets the output
 * gradient (BF16, 16 channels) times inv_count, *loss the loss sum. */
int hpm_net_loss(const float *out16, const float *t_depth, const float *t_normal, const uint8_t *t_mask, int n,
                 float dmin, float dmax, float lambda, float inv_count, void *dy, float *loss, void *stream);

/* One Adam step on n FP32 parameters (device); clears the gradients. */
int hpm_net_adam(float *params, float *grads, float *m, float *v, int n, float lr, float beta1, float beta2, float eps,
                 int step, void *stream);

/* Gradients of a 3x3 convolution layer: dw[cout][cin][3][3] += the weight
 * gradient of input x (NHWC BF16, cin channels) and output gradient dy (NHWC
 * BF16, cout channels), on the tensor cores (pixels as the reduction
 * dimension, FP32 accumulation in TMEM); db[cout] += the bias gradient when
 * db is non-NULL.  Both accumulate into the caller's FP32 buffers. */
int hpm_net_conv_wgrad(const void *x, const void *dy, int h, int w, int cin, int cout, float *dw, float *db,
                       int *err, void *stream);

/* Fusion of a scene's maps into a coloured point cloud: RunFusion
 * (main.cpp:502-633).  View v has depth (h*w floats), world normal (3
 * floats per pixel), colour (3 bytes per pixel, B, G, R as cv::imread gives
 * it, at the depth map's size: the caller resizes it like
 * RescaleImageAndCamera, HPM.cpp:187-208) and camera cams[v] (of the depth
 * map's size).  Problems as in hpm_run_scene; a problem's views are indexed
 * by view id, as the reference indexes them when problem i has reference
 * view i.  Points come in the reference's order (problem by problem, pixel
 * by pixel); up to cap are written (xyz, normal, colour), *n_points gets the
 * full count.  Inputs may be host or device memory.  The consistency tests
 * run on the GPU, the order-dependent masking on the host. */
int hpm_fuse(int device, int n_views, const HpmCamera *cams, const float *const *depths,
             const float *const *normals, const uint8_t *const *colors, int n_problems, const int *ref_ids,
             const int *src_counts, const int *src_ids, float *out_xyz, float *out_normal, uint8_t *out_bgr,
             long long cap, long long *n_points);
/* RunFusion of the ACMM+NESP variant (ACMM+NESP/windows/main.cpp:154-297):
 * hpm_fuse's arguments, consistency tests, order and masking, with the
 * variant's rule: a pixel needs at least 2 agreeing sources, and its point,
 * normal and colour are the means over it and the agreeing source pixels
 * (the colour bytes truncated, as the variant's PLY writer does,
 * ACMM.cpp:395-397). */
int hpm_fuse_acmm(int device, int n_views, const HpmCamera *cams, const float *const *depths,
                  const float *const *normals, const uint8_t *const *colors, int n_problems, const int *ref_ids,
                  const int *src_counts, const int *src_ids, float *out_xyz, float *out_normal, uint8_t *out_bgr,
                  long long cap, long long *n_points);
/* StoreColorPlyFileBinaryPointCloud (HPM.cpp:403-456): binary little-endian
 * PLY, x y z nx ny nz as float, red green blue as uchar, non-finite
 * coordinates written as the origin.  Points are written in order (the
 * reference's OpenMP loop writes them in an order that varies by run). */
int hpm_write_ply(const char *path, long long n, const float *xyz, const float *normal, const uint8_t *bgr);

/* Deterministic building blocks exposed for parity checks. */

/* The order-dependent half of hpm_fuse (rule 0) or hpm_fuse_acmm (rule 1)
 * on the host, without a GPU, given for every problem p what their GPU pass
 * computes: pair_src[p] and pair_w[p], [pixel][src_counts[p]] (the source
 * pixel index of a consistent pair or -1, and its exp(-error)), and
 * points[p], [pixel][3] (the reference pixel's world point).  Other
 * arguments as hpm_fuse's, host memory. */
int hpm_fuse_pass(int rule, int n_views, const HpmCamera *cams, const float *const *depths,
                  const float *const *normals, const uint8_t *const *colors, int n_problems, const int *ref_ids,
                  const int *src_counts, const int *src_ids, const int *const *pair_src,
                  const float *const *pair_w, const float *const *points, float *out_xyz, float *out_normal,
                  uint8_t *out_bgr, long long cap, long long *n_points);

/* Delaunay triangulation of n integer points (xy pairs) used for the planar
 * prior (replaces cv::Subdiv2D in DelaunayTriangulation, HPM.cpp:787-809,
 * plus the inside-image filter of main.cpp:97).  Writes up to cap triangles
 * (6 ints each) when tris is non-NULL; returns the triangle count or a
 * negative status. */
int hpm_delaunay(const int *xy, int n, int w, int h, int *tris, int cap);

/* Triangle raster of the planar prior (main.cpp:96-116): n triangles (6 ints
 * each, every vertex inside the w x h image) walked with the reference's
 * barycentric steps; ids[y * w + x] = index + 1 of the last triangle that
 * reaches the pixel, 0 where none does.  Host buffers; runs the raster kernel
 * of hpm_process_problem on `device`. */
int hpm_raster_triangles(int device, const int *tris, int n, int w, int h, int *ids);

/* The 6 nearest of n support points (xy pairs inside the image) for every
 * pixel whose mask is <= 0 (every pixel when mask is NULL), as the PCL
 * kd-tree search of DepthsPredictSupplement (HPM.cpp:939-962) finds them:
 * nn6[6 * (y * w + x) + k] = index of the k-th nearest by squared distance,
 * ties to the lower index (PCL leaves tie order unspecified), -1 elsewhere.
 * Host buffers; runs the kNN search of hpm_process_problem on `device`. */
int hpm_knn6(int device, const int *xy, int n, int w, int h, const float *mask, int *nn6);

/* ComputeMultiViewCostVector (HPM.cu:438-443) for one ref-frame plane per
 * pixel of the current problem; out holds (num_images-1) floats per pixel. */
int hpm_cost_vectors(hpm_ctx *ctx, const float *planes, float *out);
/* The 36 source-image samples the NCC window of ComputeBilateralNCC
 * (HPM.cu:337-359) weighs, for n listed pixels (index y * w + x) and every
 * source view: out [n][S][36] floats, inside [n][S] = 0 where the warped
 * centre leaves the source image (the NCC is then 2).  Planes as for
 * hpm_cost_vectors.  Lets a parity check tell a tap that the texture unit
 * rounded to another 1/256 step apart from every other difference. */
int hpm_tap_samples(hpm_ctx *ctx, const float *planes, const int *pixels, int n, float *out, int *inside);
/* ComputeMultiViewInitialCostandSelectedViews (HPM.cu:399-436) per pixel. */
int hpm_initial_costs(hpm_ctx *ctx, const float *planes, float *out_cost, uint32_t *out_views);
/* ComputeGeomConsistencyCost (HPM.cu:483-508) per pixel and source view,
 * against the depth maps of hpm_set_geom_depths. */
int hpm_geom_costs(hpm_ctx *ctx, const float *planes, float *out);
/* GetDepthandNormal + Black/RedPixelFilter (HPM.cu:1751-1904) on given
 * ref-frame planes and costs of the current problem (in place). */
int hpm_depth_normal_filter(hpm_ctx *ctx, float *planes, const float *costs);

/* Per-kernel CUDA-event timing of the passes run while enabled. */
int hpm_profile_enable(hpm_ctx *ctx, int enable);
/* kernel times in ms accumulated since enable: [init, propagate, finalize,
 * jbu]; counts = launches of each.  Either pointer may be NULL. */
int hpm_profile_read(hpm_ctx *ctx, float *ms4, int *counts4);
/* Work counters: bilateral NCC window evaluations (one per hypothesis and
 * source view) and geometric-consistency terms, summed over every pass run
 * since hpm_count_enable(ctx, 1), which zeroes them.  Diagnostic; no
 * reference counterpart. */
int hpm_count_enable(hpm_ctx *ctx, int enable);
int hpm_count_read(hpm_ctx *ctx, uint64_t *ncc_windows, uint64_t *geom_terms);

/* Benchmark utility (no counterpart in the reference): measured FP32 FMA
 * throughput of `device` in TFLOP/s, the roofline denominator of the
 * PatchMatch kernels.  sm_clock_mhz_hint (may be NULL) receives the
 * device's nominal SM clock. */
int hpm_fp32_peak(int device, float *tflops, float *sm_clock_mhz_hint);

/* ---- files (drop-in formats) ---- */

/* .dmb: int32 type=1, h, w, nb, then h*w*nb float32 (HPM.cpp:270-401). */
int hpm_write_dmb(const char *path, const float *data, int h, int w, int nb);
/* Reads header into *h,*w,*nb; when data is non-NULL also the payload
 * (capacity cap floats). */
int hpm_read_dmb(const char *path, float *data, size_t cap, int *h, int *w, int *nb);
/* cams/%08d_cam.txt (ReadCamera, HPM.cpp:160-185).  width/height are left 0. */
int hpm_read_camera(const char *path, HpmCamera *cam);
/* An 8-bit grayscale image as cv::imread(path, IMREAD_GRAYSCALE) returns it
 * for the reference's images/%08d.jpg (HPM.cpp:490-492): JPEG (baseline,
 * extended sequential or progressive Huffman; EXIF orientation applied),
 * binary PGM or 8-bit PNG (colour reduced as OpenCV's PNG reader does),
 * recognised by content.  Sets *w, *h; copies the pixels when pixels is
 * non-NULL (capacity cap bytes). */
int hpm_read_gray8(const char *path, uint8_t *pixels, size_t cap, int *w, int *h);
/* A colour image as cv::imread(path, IMREAD_COLOR) returns it for the
 * fusion (main.cpp:520-523): 3 bytes per pixel in B, G, R order; gray JPEG,
 * PGM and gray PNG are replicated to the three channels, alpha is dropped. */
int hpm_read_bgr8(const char *path, uint8_t *pixels, size_t cap, int *w, int *h);
/* cv::resize(src, dst, Size(dw, dh), 0, 0, INTER_LINEAR) of a float map
 * with ch interleaved channels, on the host: the image cap of
 * InuputInitialization (HPM.cpp:525-551).  Same arithmetic as OpenCV 4.x
 * (double-precision fractions, one fused a + f*(b-a) per direction). */
int hpm_resize_linear(const float *src, int sw, int sh, int ch, float *dst, int dw, int dh);
/* cv::resize(src, dst, Size(dw, dh), 0, 0, INTER_LINEAR) of an 8-bit image
 * of ch interleaved channels, byte for byte as OpenCV computes it, as in
 * RescaleImageAndCamera (HPM.cpp:187-208), which resizes the fusion's colour
 * images (cv::Mat_<cv::Vec3b>) to their depth maps. */
int hpm_resize_linear_u8(const uint8_t *src, int sw, int sh, int ch, uint8_t *dst, int dw, int dh);
/* pair.txt (GenerateSampleList, main.cpp:4-33): returns the problem count
 * into *n; ref_ids[n], src_counts[n], src_ids[n][HPM_MAX_IMAGES-1] filled when
 * non-NULL (sources with score <= 0 are dropped). */
int hpm_read_pair(const char *path, int *n, int *ref_ids, int *src_counts, int *src_ids, int cap);

#ifdef __cplusplus
}
#endif
#endif /* HPM_B200_H */

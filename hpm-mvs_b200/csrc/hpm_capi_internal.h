/*
 * The context behind the C ABI (hpm_ctx) and the helpers the pass
 * orchestration (hpm_flow.cu) shares with hpm_capi.cu.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <utility>
#include <vector>

#include "hpm_internal.h"

namespace hpm {

/* Device workspace of the planar-prior stages, grown on demand and reused
 * by every problem of a context. */
struct FlowWorkspace {
    float *full_depth = nullptr, *full_normal = nullptr, *prior_depth = nullptr, *up_depth = nullptr;
    float4 *up_normal = nullptr;
    size_t full_cap = 0;
    float *mask = nullptr;
    int *ids = nullptr;
    float4 *knn_planes = nullptr;
    size_t lvl_cap = 0;
    int2 *blocks = nullptr;
    size_t blocks_cap = 0;
    float *c_depth = nullptr, *c_cost = nullptr, *c_normal = nullptr, *c_prior_depth = nullptr,
          *c_prior_normal = nullptr;
    float4 *c_packed = nullptr;
    size_t coarse_cap = 0;
    int *tris = nullptr;
    float4 *tri_planes = nullptr;
    size_t tri_cap = 0;
    int2 *pts = nullptr;
    int *cell_start = nullptr, *cell_pts = nullptr;
    size_t pts_cap = 0, cells_cap = 0;
    bool has_prior_depth = false;
    int last_points = 0, last_triangles = 0;
};

/* Device buffers of the prior-net form's coarse stage and network, grown on
 * demand and reused by every problem of a context. */
struct NetWorkspace {
    void *x0 = nullptr;            /* network input, [coarse px][16] BF16 */
    void *a[3] = {nullptr, nullptr, nullptr}; /* hidden activations, [coarse px][32] BF16 */
    float *out = nullptr;          /* last layer, [coarse px][16] FP32 */
    float4 *prop = nullptr;        /* head: world normal, depth per coarse pixel */
    size_t cap = 0;
    float *cimg = nullptr;         /* the problem's 1/4-scale images */
    size_t cimg_cap = 0;
    float *up_depth = nullptr;     /* upsampled proposal, full scale */
    float4 *up_normal = nullptr, *cand = nullptr;
    size_t full_cap = 0;
    int *err = nullptr;            /* status of the tensor-core kernels */
};

/* A view's float cudaArray with its texture object. */
struct TexArray {
    int w = 0, h = 0;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
};

}  // namespace hpm

struct hpm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    char err[512] = {0};

    int n = 0;
    HpmCamera cams[hpm::kMaxViews];
    float *d_img[hpm::kMaxViews] = {nullptr};
    size_t img_cap[hpm::kMaxViews] = {0};
    cudaArray_t arr[hpm::kMaxViews] = {nullptr};      /* the current view's array and texture */
    cudaTextureObject_t tex[hpm::kMaxViews] = {0};
    std::vector<hpm::TexArray> tex_pool[hpm::kMaxViews]; /* arrays of the sizes each slot has held */
    float *d_depth[hpm::kMaxViews] = {nullptr};
    size_t depth_cap[hpm::kMaxViews] = {0};
    bool has_depth = false;
    hpm::PairGeom *d_pair = nullptr;

    float4 *d_planes = nullptr;
    float *d_costs = nullptr;
    uint32_t *d_views = nullptr;
    float4 *d_prior = nullptr;
    uint32_t *d_masks = nullptr;
    size_t px_cap = 0;
    bool has_prior = false;
    bool has_state = false;

    unsigned long long *d_counters = nullptr;
    bool counting = false;

    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_events;
    float prof_ms[4] = {0, 0, 0, 0};
    int prof_cnt[4] = {0, 0, 0, 0};

    uint32_t pass_counter = 0;

    void *d_scratch = nullptr;
    size_t scratch_cap = 0;

    float *d_cache = nullptr; /* cost vector of each pixel's current hypothesis, [S][2][ceil(H*W/2)] */
    size_t cache_cap = 0;
    float *d_cand = nullptr; /* half-step hand-off: cost matrix rows [kCandRows*S][ceil(H*W/2)] */
    size_t cand_cap = 0;
    int *d_pos = nullptr; /* chosen NESP sites [8][ceil(H*W/2)] */
    size_t pos_cap = 0;
    uint32_t *d_flags = nullptr; /* direction row codes [ceil(H*W/2)] */
    size_t flags_cap = 0;
    float *d_pre = nullptr; /* ACMM+NESP hierarchy pass: acceptance threshold per pixel */
    size_t pre_cap = 0;

    /* prior-net form: the network's proposed plane per pixel (ref-frame
     * normal, distance) for the next pass, or nullptr (plain form) */
    const float4 *proposals = nullptr;
    hpm::NetWorkspace net;
    /* prior-net form: the context that holds a problem's 1/4-scale views,
     * so that this one keeps its full-scale views and texture arrays */
    hpm_ctx *coarse = nullptr;
    /* batched form: one context per problem of the last batched scene, and
     * the autotuned half-step tile width per view size (width << 32 | rows) */
    std::vector<hpm_ctx *> batch;
    std::vector<std::pair<long long, int>> tile_ww;
    hpm::FlowWorkspace flow;
    /* HpmProblemOpts.fix_quirks of the problem being processed (prior levels) */
    bool fix_quirks = false;
    float *d_scene = nullptr; /* hpm_run_scene's per-view maps, grown on demand */
    size_t scene_cap = 0;

    /* hpm_run_scene hands pass set A's problems to this context and a peer
     * (same device, own stream) from two host threads.  The threads pass a
     * GPU token: a thread holds it while its kernels run and releases it
     * only while its host triangulates support points, so the other
     * problem's kernels fill that gap and the two problems' kernels never
     * share the GPU (their images would compete for L2 and texture caches). */
    int scene_workers = 2;
    hpm_ctx *peer = nullptr;
    std::mutex *gpu_token = nullptr;
};

int ctx_fail(hpm_ctx *c, int code, const char *fmt, ...);
int ctx_cuda_fail(hpm_ctx *c, cudaError_t e, const char *what);
int ctx_select_device(hpm_ctx *c);
/* one pass: init, `half_steps` red/black half-steps, optional finalisation;
 * synchronises the context's stream at the end */
int ctx_run_pass(hpm_ctx *c, const HpmParams *p, int half_steps, int finalize);
/* a context on c's device for c's own use (second worker, coarse views,
 * batched problems), counting and profiling when c does */
int ctx_create_child(hpm_ctx *c, hpm_ctx **child);
float *ctx_planes(hpm_ctx *c);
cudaError_t ctx_scene_arena(hpm_ctx *c, size_t bytes);
float *ctx_scene_base(hpm_ctx *c);
float *ctx_costs(hpm_ctx *c);
float *ctx_prior(hpm_ctx *c);
uint32_t *ctx_masks(hpm_ctx *c);
const float *ctx_image(hpm_ctx *c, int i);
void ctx_mark_prior(hpm_ctx *c);
cudaError_t ws_reserve(hpm_ctx *c, size_t npx, size_t nblocks);
cudaError_t ws_reserve_tris(hpm_ctx *c, size_t ntris);
cudaError_t ws_reserve_grid(hpm_ctx *c, size_t npts, size_t ncells);
cudaError_t ws_reserve_full(hpm_ctx *c, size_t npx);
cudaError_t ws_reserve_coarse(hpm_ctx *c, size_t npx);
void ws_free(hpm_ctx *c);
/* the arguments of one pass (validated as hpm_run_patchmatch; takes the
 * pass's random-stream salt) for a batched launch */
int ctx_pass_args(hpm_ctx *c, const HpmParams *p, hpm::PMArgs *out);
/* restart the context's pass numbering (the salt of its random streams) */
void ctx_reset_salt(hpm_ctx *c);
/* hypotheses written on the device count as the pass state */
void ctx_mark_state(hpm_ctx *c);
cudaError_t net_reserve(hpm_ctx *c, size_t coarse_px, size_t coarse_img_floats);
cudaError_t net_reserve_full(hpm_ctx *c, size_t npx);
void net_free(hpm_ctx *c);

namespace hpm {
/* hpm_flow.cu helpers shared with the prior-net form */
cudaError_t flow_split_state(const float4 *planes, int n, float *depth, float *normal3, cudaStream_t s);
cudaError_t flow_pack4(const float *depth, const float *normal3, int n, float4 *out, cudaStream_t s);
int flow_level_prior(hpm_ctx *c, const HpmCamera &cam, const float *d_cost, const float *d_depth, int w, int h,
                     float factor, float dmin, float dmax);
/* the prior of pyramid level `level` (2: full scale) from flow.full_depth /
 * full_normal and d_cost, into the context's prior planes and masks */
int flow_prior_from_maps(hpm_ctx *c, int level, const float *d_cost, float dmin, float dmax);
/* hpm_priornet.cu: the prior-net form's stages (per problem context) */
int net_coarse_views(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams);
int net_coarse_finish(hpm_ctx *c, float dmin, float dmax);
int net_full_setup(hpm_ctx *c, const HpmNetWeights *net, int prior_mode);
uint64_t net_pass_seed(uint64_t seed, int pass);
int net_status(hpm_ctx *c);
int net_problem(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams, const HpmNetWeights *net,
                uint64_t seed, int extra_passes, int prior_mode, int half_steps, float *depth_out, float *normal_out,
                float *cost_out);
}  // namespace hpm

/*
 * ProcessProblem (HPM-MVS/main.cpp:35-499) for one reference view on the
 * device: the plain pass, the hierarchical planar-prior passes and the
 * geometric-consistency pass, through the context of hpm_capi.cu.
 *
 * Everything stays in HBM between the passes; the host only compacts the
 * support points of a level and triangulates them (hpm_delaunay.cpp).  The
 * reference copies every map to the host between passes and runs the prior
 * stages there (support points, Subdiv2D, PCL kd-tree KNN, per-pixel loops).
 */
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "hpm_capi_internal.h"
#include "hpm_nvtx.h"
#include "hpm_prior.h"

using namespace hpm;

namespace {

__global__ void k_split_state(const float4 *__restrict__ planes, int n, float *__restrict__ depth,
                              float *__restrict__ normal3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = planes[i];
    depth[i] = p.w;
    normal3[3 * i] = p.x;
    normal3[3 * i + 1] = p.y;
    normal3[3 * i + 2] = p.z;
}

__global__ void k_pack4(const float *__restrict__ depth, const float *__restrict__ normal3, int n,
                        float4 *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2], depth[i]);
}

/* ComputingMultiScaleSettings, HPM.cpp:851-860 */
int scale_levels(int w, int h)
{
    int m = w > h ? w : h, k = 0;
    while (m > 1000) {
        m /= 2;
        k++;
    }
    return k;
}

int grid1(int n) { return (n + 255) / 256; }

}  // namespace

#define CK(call, what)                                         \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return ctx_cuda_fail(c, e_, what); \
    } while (0)

cudaError_t hpm::flow_split_state(const float4 *planes, int n, float *depth, float *normal3, cudaStream_t s)
{
    k_split_state<<<grid1(n), 256, 0, s>>>(planes, n, depth, normal3);
    return cudaGetLastError();
}

cudaError_t hpm::flow_pack4(const float *depth, const float *normal3, int n, float4 *out, cudaStream_t s)
{
    k_pack4<<<grid1(n), 256, 0, s>>>(depth, normal3, n, out);
    return cudaGetLastError();
}

/* Support points of a cost map in the reference's block order, the
 * triangulation, raster and plane fits, and the KNN supplement: leaves
 * ws.mask (reference mask values: triangle id, -233 for KNN, 0), ws.ids,
 * ws.tri_planes and ws.knn_planes for a level of size w x h. */
static int build_level_prior(hpm_ctx *c, const HpmCamera &cam, const float *d_cost, const float *d_depth, int w, int h,
                             float factor, float dmin, float dmax)
{
    FlowWorkspace &ws = c->flow;
    cudaStream_t s = c->stream;
    const size_t npx = (size_t)w * h;
    const int nb_max = ((w + 4) / 5) * ((h + 4) / 5);
    CK(ws_reserve(c, npx, nb_max), "prior workspace");
    int nb = 0;
    CK(prior_support_blocks(d_cost, w, h, ws.blocks, &nb, s), "support points");
    std::vector<int2> blocks(nb);
    CK(cudaMemcpyAsync(blocks.data(), ws.blocks, sizeof(int2) * nb, cudaMemcpyDeviceToHost, s), "support points");
    CK(cudaStreamSynchronize(s), "support points");
    std::vector<int> xy;
    xy.reserve(2 * nb);
    for (const int2 &b : blocks)
        if (b.x >= 0) {
            xy.push_back(b.x);
            xy.push_back(b.y);
        }
    const int np = (int)xy.size() / 2;
    std::vector<int> tris;
    /* the stream is idle here: another scene worker may use the GPU while
     * this host thread triangulates */
    if (c->gpu_token) c->gpu_token->unlock();
    delaunay(xy, w, h, tris);
    if (c->gpu_token) c->gpu_token->lock();
    const int nt = (int)tris.size() / 6;
    CK(ws_reserve_tris(c, nt), "triangle buffers");
    if (nt > 0) CK(cudaMemcpyAsync(ws.tris, tris.data(), sizeof(int) * tris.size(), cudaMemcpyHostToDevice, s), "tris");
    CK(prior_triangles(cam, d_depth, w, h, ws.tris, nt, factor, ws.tri_planes, ws.ids, s), "triangle raster");
    CK(prior_ids_to_mask(ws.ids, (int)npx, ws.mask, s), "mask");
    /* KNN supplement over a uniform cell grid (counting sort on the host) */
    if (np >= 6) {
        const int cell = 8;
        int gw, gh;
        std::vector<int> start, order;
        knn_grid(xy.data(), np, w, h, cell, gw, gh, start, order);
        CK(ws_reserve_grid(c, np, gw * gh + 1), "knn grid");
        CK(cudaMemcpyAsync(ws.pts, xy.data(), sizeof(int) * 2 * np, cudaMemcpyHostToDevice, s), "points");
        CK(cudaMemcpyAsync(ws.cell_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, s), "grid");
        CK(cudaMemcpyAsync(ws.cell_pts, order.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s), "grid");
        CK(prior_knn(cam, ws.pts, ws.cell_start, ws.cell_pts, cell, gw, gh, d_depth, w, h, factor, dmin, dmax, ws.mask,
                     ws.knn_planes, s),
           "knn prior");
        CK(cudaStreamSynchronize(s), "knn prior"); /* host vectors above go out of scope */
    }
    ws.last_points = np;
    ws.last_triangles = nt;
    return HPM_OK;
}

/* The prior of pyramid level i (0: 1/4 scale, 1: 1/2 scale, else full
 * scale; main.cpp:78-478) from the full-resolution maps in ws.full_depth,
 * ws.full_normal and d_cost: leaves the ref-frame prior planes and masks of
 * the next pass in the context (and, at full scale, the prior depth map). */
int hpm::flow_level_prior(hpm_ctx *c, const HpmCamera &cam, const float *d_cost, const float *d_depth, int w, int h,
                          float factor, float dmin, float dmax)
{
    return build_level_prior(c, cam, d_cost, d_depth, w, h, factor, dmin, dmax);
}

static int level_prior_from_maps(hpm_ctx *c, int i, const float *d_cost, float dmin, float dmax)
{
    const HpmCamera cam = c->cams[0];
    const int W = cam.width, H = cam.height;
    cudaStream_t s = c->stream;
    FlowWorkspace &ws = c->flow;
    int r;
    if (i == 0 || i == 1) {
        const float f = i == 0 ? 0.25f : 0.5f;
        const int ws_w = (int)std::round(W * (double)f), ws_h = (int)std::round(H * (double)f);
        if (ws_w < 1 || ws_h < 1) return ctx_fail(c, HPM_ERR_ARG, "image too small for pyramid level %d", i);
        const size_t cn = (size_t)ws_w * ws_h;
        CK(ws_reserve_coarse(c, cn), "coarse buffers");
        CK(prior_resize(ws.full_depth, W, H, 1, ws.c_depth, ws_w, ws_h, s), "resize");
        CK(prior_resize(d_cost, W, H, 1, ws.c_cost, ws_w, ws_h, s), "resize");
        CK(prior_resize(ws.full_normal, W, H, 3, ws.c_normal, ws_w, ws_h, s), "resize");
        r = build_level_prior(c, cam, ws.c_cost, ws.c_depth, ws_w, ws_h, f, dmin, dmax);
        if (r) return r;
        CK(prior_coarse(cam, ws_w, ws_h, f, dmin, dmax, ws.mask, ws.ids, ws.tri_planes, ws.knn_planes,
                        ws.c_prior_depth, ws.c_prior_normal, s, !c->fix_quirks),
           "coarse prior");
        k_pack4<<<grid1((int)cn), 256, 0, s>>>(ws.c_prior_depth, ws.c_prior_normal, (int)cn, ws.c_packed);
        const int sr = H / ws_h, sc = W / ws_w;
        CK(launch_jbu(ctx_image(c, 0), W, H, nullptr, ws.c_packed, ws_w, ws_h, sr > sc ? sr : sc, ws.up_depth,
                      ws.up_normal, s),
           "jbu");
        CK(prior_reload(cam, W, H, dmin, dmax, ws.up_depth, ws.up_normal, reinterpret_cast<float4 *>(ctx_prior(c)),
                        ctx_masks(c), s),
           "prior reload");
    } else {
        r = build_level_prior(c, cam, d_cost, ws.full_depth, W, H, 1.0f, dmin, dmax);
        if (r) return r;
        CK(prior_full(cam, W, H, dmin, dmax, ws.mask, ws.ids, ws.tri_planes, ws.knn_planes, ws.prior_depth,
                      reinterpret_cast<float4 *>(ctx_prior(c)), ctx_masks(c), s),
           "full prior");
        ws.has_prior_depth = true;
    }
    ctx_mark_prior(c);
    return HPM_OK;
}

int hpm::flow_prior_from_maps(hpm_ctx *c, int level, const float *d_cost, float dmin, float dmax)
{
    return level_prior_from_maps(c, level, d_cost, dmin, dmax);
}

extern "C" int hpm_prior_level(hpm_ctx *c, int level, const float *depth, const float *normal, const float *cost,
                               float *prior_planes, uint32_t *masks, float *prior_depth)
{
    if (!c || !depth || !normal || !cost) return HPM_ERR_ARG;
    if (c->n < 2) return ctx_fail(c, HPM_ERR_STATE, "hpm_prior_level before hpm_set_views");
    int r = ctx_select_device(c);
    if (r) return r;
    const HpmCamera cam = c->cams[0];
    const size_t npx = (size_t)cam.width * cam.height;
    cudaStream_t s = c->stream;
    FlowWorkspace &ws = c->flow;
    CK(ws_reserve_full(c, npx), "flow workspace");
    CK(ws_reserve_coarse(c, npx), "flow workspace");
    CK(cudaMemcpyAsync(ws.full_depth, depth, sizeof(float) * npx, cudaMemcpyHostToDevice, s), "depth");
    CK(cudaMemcpyAsync(ws.full_normal, normal, sizeof(float) * 3 * npx, cudaMemcpyHostToDevice, s), "normal");
    float *d_hold = nullptr; /* the cost map: must not alias the level's resize targets */
    CK(cudaMalloc(&d_hold, sizeof(float) * npx), "cost");
    CK(cudaMemcpyAsync(d_hold, cost, sizeof(float) * npx, cudaMemcpyHostToDevice, s), "cost");
    r = level_prior_from_maps(c, level, d_hold, cam.depth_min * 0.6f, cam.depth_max * 1.2f);
    if (r == HPM_OK) {
        if (prior_planes)
            CK(cudaMemcpyAsync(prior_planes, ctx_prior(c), sizeof(float4) * npx, cudaMemcpyDeviceToHost, s), "out");
        if (masks) CK(cudaMemcpyAsync(masks, ctx_masks(c), sizeof(uint32_t) * npx, cudaMemcpyDeviceToHost, s), "out");
        if (prior_depth) {
            if (level == 0 || level == 1)
                memset(prior_depth, 0, sizeof(float) * npx);
            else
                CK(cudaMemcpyAsync(prior_depth, ws.prior_depth, sizeof(float) * npx, cudaMemcpyDeviceToHost, s), "out");
        }
        CK(cudaStreamSynchronize(s), "hpm_prior_level");
    }
    cudaFree(d_hold);
    return r;
}

/* hpm_process_problem with `half_steps` half-steps per pass (the reference's
 * 6 everywhere but in the prior-net forms' geometric passes) */
static int process_problem(hpm_ctx *c, const HpmProblemOpts *o, int half_steps, float *depth_out, float *normal_out,
                           float *cost_out, float *prior_depth_out)
{
    if (!c || !o) return HPM_ERR_ARG;
    if (c->n < 2) return ctx_fail(c, HPM_ERR_STATE, "hpm_process_problem before hpm_set_views");
    int r = ctx_select_device(c);
    if (r) return r;
    const HpmCamera cam = c->cams[0];
    const int W = cam.width, H = cam.height;
    const Range range("problem %dx%d geom=%d", W, H, o->geom_consistency);
    const size_t npx = (size_t)W * H;
    cudaStream_t s = c->stream;
    HpmParams p;
    hpm_default_params(&p);
    p.depth_min = cam.depth_min * 0.6f; /* InuputInitialization, HPM.cpp:553-554 */
    p.depth_max = cam.depth_max * 1.2f;
    p.seed = o->seed;
    p.fix_quirks = o->fix_quirks;
    c->fix_quirks = o->fix_quirks != 0;
    FlowWorkspace &ws = c->flow;
    ws.last_points = ws.last_triangles = 0;
    if (o->geom_consistency) {
        p.geom_consistency = 1;
        p.multi_geometry = o->multi_geometry;
        r = ctx_run_pass(c, &p, half_steps, 1);
        if (r) return r;
    } else {
        r = ctx_run_pass(c, &p, half_steps, 1);
        if (r) return r;
        if (o->planar_prior) {
            CK(ws_reserve_full(c, npx), "flow workspace");
            const int k = o->pyramid_levels >= 0 ? o->pyramid_levels : scale_levels(W, H);
            for (int i = 2 - k; i <= 2; ++i) {
                const Range level("prior level %d", i);
                CK(cudaGetLastError(), "flow");
                k_split_state<<<grid1((int)npx), 256, 0, s>>>(reinterpret_cast<const float4 *>(ctx_planes(c)), (int)npx,
                                                              ws.full_depth, ws.full_normal);
                r = level_prior_from_maps(c, i, ctx_costs(c), p.depth_min, p.depth_max);
                if (r) return r;
                p.planar_prior = 1;
                r = ctx_run_pass(c, &p, half_steps, 1);
                if (r) return r;
            }
        }
    }
    /* results: depth, world normal, cost (main.cpp:481-490) */
    CK(ws_reserve_full(c, npx), "flow workspace");
    k_split_state<<<grid1((int)npx), 256, 0, s>>>(reinterpret_cast<const float4 *>(ctx_planes(c)), (int)npx,
                                                  ws.full_depth, ws.full_normal);
    /* outputs may be host or device memory (unified addressing) */
    if (depth_out) CK(cudaMemcpyAsync(depth_out, ws.full_depth, sizeof(float) * npx, cudaMemcpyDefault, s), "out");
    if (normal_out)
        CK(cudaMemcpyAsync(normal_out, ws.full_normal, sizeof(float) * 3 * npx, cudaMemcpyDefault, s), "out");
    if (cost_out) CK(cudaMemcpyAsync(cost_out, ctx_costs(c), sizeof(float) * npx, cudaMemcpyDefault, s), "out");
    if (prior_depth_out) {
        if (ws.has_prior_depth && o->planar_prior && !o->geom_consistency) {
            CK(cudaMemcpyAsync(prior_depth_out, ws.prior_depth, sizeof(float) * npx, cudaMemcpyDefault, s), "out");
        } else {
            cudaPointerAttributes pa;
            if (cudaPointerGetAttributes(&pa, prior_depth_out) == cudaSuccess && pa.type == cudaMemoryTypeDevice)
                CK(cudaMemsetAsync(prior_depth_out, 0, sizeof(float) * npx, s), "out");
            else
                memset(prior_depth_out, 0, sizeof(float) * npx);
        }
    }
    CK(cudaStreamSynchronize(s), "hpm_process_problem");
    return HPM_OK;
}

extern "C" int hpm_process_problem(hpm_ctx *c, const HpmProblemOpts *o, float *depth_out, float *normal_out,
                                   float *cost_out, float *prior_depth_out)
{
    return process_problem(c, o, 6, depth_out, normal_out, cost_out, prior_depth_out);
}

extern "C" int hpm_last_prior_stats(hpm_ctx *c, int *points, int *triangles)
{
    if (!c) return HPM_ERR_ARG;
    if (points) *points = c->flow.last_points;
    if (triangles) *triangles = c->flow.last_triangles;
    return HPM_OK;
}

/* ---------------- whole scene: main.cpp:636-677 ---------------- */

namespace {

__global__ void k_pack_planes(const float *__restrict__ normal3, const float *__restrict__ depth, int n,
                              float4 *__restrict__ planes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    planes[i] = make_float4(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2], depth[i]);
}

/* per-view maps of a scene, carved from one arena kept in the context */
struct SceneMaps {
    std::vector<float *> img, depth_a, depth_g, normal, cost;
};

}  // namespace

extern "C" int hpm_run_scene(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                             int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                             const HpmSceneOpts *o, float *const *out_depths, float *const *out_normals,
                             float *const *out_costs)
{
    return hpm_run_scene_ex(c, n_views, images, cams, n_problems, ref_ids, src_counts, src_ids, o, out_depths,
                            out_normals, out_costs, nullptr, nullptr);
}

static int run_scene_impl(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                          int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                          const HpmSceneOpts *o, const HpmNetWeights *net, float *const *out_depths,
                          float *const *out_normals, float *const *out_costs, float *const *out_pass_depths,
                          float *const *out_prior_depths);

extern "C" int hpm_run_scene_ex(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                                int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                                const HpmSceneOpts *o, float *const *out_depths, float *const *out_normals,
                                float *const *out_costs, float *const *out_pass_depths,
                                float *const *out_prior_depths)
{
    return run_scene_impl(c, n_views, images, cams, n_problems, ref_ids, src_counts, src_ids, o, nullptr, out_depths,
                          out_normals, out_costs, out_pass_depths, out_prior_depths);
}

extern "C" int hpm_run_scene_net(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                                 int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                                 const HpmSceneOpts *o, const HpmNetWeights *net, float *const *out_depths,
                                 float *const *out_normals, float *const *out_costs)
{
    if (!net) return HPM_ERR_ARG;
    for (int l = 0; l < 4; ++l)
        if (!net->packed[l] || !net->bias[l]) return HPM_ERR_ARG;
    return run_scene_impl(c, n_views, images, cams, n_problems, ref_ids, src_counts, src_ids, o, net, out_depths,
                          out_normals, out_costs, nullptr, nullptr);
}

static int run_scene_impl(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                          int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                          const HpmSceneOpts *o, const HpmNetWeights *net, float *const *out_depths,
                          float *const *out_normals, float *const *out_costs, float *const *out_pass_depths,
                          float *const *out_prior_depths)
{
    if (!c || !images || !cams || !ref_ids || !src_counts || !src_ids || !o) return HPM_ERR_ARG;
    if (n_views < 2 || n_problems < 1) return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene: %d views, %d problems", n_views,
                                                       n_problems);
    for (int p = 0; p < n_problems; ++p) {
        if (ref_ids[p] < 0 || ref_ids[p] >= n_views || src_counts[p] < 1 || src_counts[p] > kMaxSrc)
            return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene: problem %d is malformed", p);
        for (int j = 0; j < src_counts[p]; ++j) {
            const int s = src_ids[p * kMaxSrc + j];
            if (s < 0 || s >= n_views) return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene: problem %d source %d", p, s);
        }
    }
    int r = ctx_select_device(c);
    if (r) return r;
    const Range range(net ? "scene %d views (prior-net form)" : "scene %d views", n_views);
    if (o->iterations < 0 || o->iterations > 64 || o->geom_pass_iterations < 0 || o->geom_pass_iterations > 64)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene: iterations outside [0, 64]");
    const int half_steps = net && o->iterations > 0 ? 2 * o->iterations : 6;
    const int geom_half_steps = net && o->geom_pass_iterations > 0 ? 2 * o->geom_pass_iterations : half_steps;
    cudaStream_t s = c->stream;
    SceneMaps m;
    size_t total = 0; /* floats: image, pass-A depth, geometric depth, normal (3), cost */
    for (int v = 0; v < n_views; ++v) total += 7 * (((size_t)cams[v].width * cams[v].height + 63) & ~(size_t)63);
    CK(ctx_scene_arena(c, total * sizeof(float)), "scene buffers");
    float *cur = ctx_scene_base(c);
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height, st = (np + 63) & ~(size_t)63;
        m.img.push_back(cur);
        m.depth_a.push_back(cur + st);
        m.depth_g.push_back(cur + 2 * st);
        m.normal.push_back(cur + 3 * st);
        m.cost.push_back(cur + 6 * st);
        cur += 7 * st;
        CK(cudaMemcpyAsync(m.img[v], images[v], sizeof(float) * np, cudaMemcpyDefault, s), "scene images");
    }
    /* the views of problem p */
    auto gather = [&](int p, const float **pimg, HpmCamera *pcam) -> int {
        const int ref = ref_ids[p], ns = src_counts[p];
        pimg[0] = m.img[ref];
        pcam[0] = cams[ref];
        for (int j = 0; j < ns; ++j) {
            const int sv = src_ids[p * kMaxSrc + j];
            pimg[j + 1] = m.img[sv];
            pcam[j + 1] = cams[sv];
        }
        return ns + 1;
    };
    auto load_problem = [&](hpm_ctx *cc, int p) -> int {
        const float *pimg[kMaxViews];
        HpmCamera pcam[kMaxViews];
        const int n = gather(p, pimg, pcam);
        return hpm_set_views(cc, pimg, pcam, n);
    };
    CK(cudaStreamSynchronize(s), "scene images");
    /* pass set A: ProcessProblem(geom = false, planar_prior) for every view.
     * The problems are independent; with two workers they are handed out to
     * this context and its peer from two host threads that pass the GPU
     * token (see hpm_ctx::gpu_token). */
    {
        const int workers = (c->scene_workers > 1 && n_problems > 1) ? 2 : 1;
        if (workers == 2 && !c->peer) {
            /* the peer's work is profiled and counted with this context's */
            r = ctx_create_child(c, &c->peer);
            if (r) return ctx_fail(c, r, "hpm_run_scene: second context");
        }
        std::mutex token;
        hpm_ctx *ctxs[2] = {c, workers == 2 ? c->peer : nullptr};
        if (workers == 2) c->gpu_token = c->peer->gpu_token = &token;
        std::atomic<int> next{0};
        int rcs[2] = {HPM_OK, HPM_OK};
        auto work = [&](int wi) {
            hpm_ctx *cc = ctxs[wi];
            for (;;) {
                const int p = next.fetch_add(1);
                if (p >= n_problems) return;
                std::unique_lock<std::mutex> hold(token);
                int rr;
                if (net) {
                    const float *pimg[kMaxViews];
                    HpmCamera pcam[kMaxViews];
                    const int n = gather(p, pimg, pcam), ref = ref_ids[p];
                    rr = net_problem(cc, n, pimg, pcam, net, o->seed + (uint64_t)p,
                                     o->pyramid_levels > 0 ? o->pyramid_levels : 0, o->planar_prior, half_steps,
                                     m.depth_a[ref], m.normal[ref], m.cost[ref]);
                    if (rr == HPM_OK && out_prior_depths && out_prior_depths[ref])
                        rr = cudaMemsetAsync(out_prior_depths[ref], 0,
                                             sizeof(float) * cams[ref].width * cams[ref].height, cc->stream) ==
                                     cudaSuccess
                                 ? HPM_OK
                                 : HPM_ERR_CUDA;
                } else {
                    rr = load_problem(cc, p);
                }
                if (!rr && !net) {
                    HpmProblemOpts po = {o->planar_prior, 0, 0, o->seed + (uint64_t)p, o->pyramid_levels,
                                         o->fix_quirks};
                    const int ref = ref_ids[p];
                    float *prior_out = out_prior_depths ? out_prior_depths[ref] : nullptr;
                    rr = hpm_process_problem(cc, &po, m.depth_a[ref], m.normal[ref], m.cost[ref], prior_out);
                }
                if (rr) {
                    rcs[wi] = rr;
                    next.store(n_problems); /* stop the other worker too */
                    return;
                }
            }
        };
        if (workers == 2) {
            std::thread helper(work, 1);
            work(0);
            helper.join();
            c->gpu_token = c->peer->gpu_token = nullptr;
        } else {
            work(0);
        }
        if (rcs[0]) return rcs[0];
        if (rcs[1]) return ctx_fail(c, rcs[1], "hpm_run_scene (second context): %s", hpm_last_error(c->peer));
    }
    float *pdep[kMaxViews];
    /* pass set B: geometric iterations (main.cpp:662-674) */
    for (int gi = 0; gi < o->geom_iterations; ++gi) {
        const Range iteration("geometric iteration %d", gi);
        std::vector<float *> &src_depths = gi == 0 ? m.depth_a : m.depth_g;
        if (gi == 0)
            for (int v = 0; v < n_views; ++v)
                CK(cudaMemcpyAsync(m.depth_g[v], m.depth_a[v], sizeof(float) * cams[v].width * cams[v].height,
                                   cudaMemcpyDeviceToDevice, s),
                   "scene copy");
        for (int p = 0; p < n_problems; ++p) {
            r = load_problem(c, p);
            if (r) return r;
            const int ref = ref_ids[p], ns = src_counts[p];
            pdep[0] = src_depths[ref];
            for (int j = 0; j < ns; ++j) pdep[j + 1] = src_depths[src_ids[p * kMaxSrc + j]];
            r = hpm_set_geom_depths(c, pdep);
            if (r) return r;
            const size_t np = (size_t)cams[ref].width * cams[ref].height;
            k_pack_planes<<<grid1((int)np), 256, 0, s>>>(m.normal[ref], src_depths[ref], (int)np,
                                                         reinterpret_cast<float4 *>(ctx_planes(c)));
            CK(cudaMemcpyAsync(ctx_costs(c), m.cost[ref], sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
            HpmProblemOpts po = {0, 1, gi >= 1, o->seed + 1000003ull * (gi + 1) + (uint64_t)p, o->pyramid_levels,
                                 o->fix_quirks};
            /* the geometric depth map is rewritten view by view (depths_geom.dmb) */
            r = process_problem(c, &po, geom_half_steps, m.depth_g[ref], m.normal[ref], m.cost[ref], nullptr);
            if (r) return r;
        }
    }
    std::vector<float *> &final_depth = o->geom_iterations > 0 ? m.depth_g : m.depth_a;
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height;
        if (out_depths && out_depths[v])
            CK(cudaMemcpyAsync(out_depths[v], final_depth[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
        if (out_normals && out_normals[v])
            CK(cudaMemcpyAsync(out_normals[v], m.normal[v], sizeof(float) * 3 * np, cudaMemcpyDefault, s), "out");
        if (out_costs && out_costs[v])
            CK(cudaMemcpyAsync(out_costs[v], m.cost[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
        if (out_pass_depths && out_pass_depths[v])
            CK(cudaMemcpyAsync(out_pass_depths[v], m.depth_a[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
    }
    CK(cudaStreamSynchronize(s), "hpm_run_scene");
    return HPM_OK;
}

/*
 * The batched form of a scene (hpm_run_scene_batched, and with the network
 * hpm_run_scene_batched_net): every problem of the scene advances together.
 *
 * The reference runs the problems one after another (main.cpp:658-674),
 * each with its own launches (HPM.cu:1906-1957).  Here each problem keeps
 * its own context (views and texture arrays, hypothesis state, hand-off
 * buffers), and one pass of every problem (initialisation, the half-steps,
 * depth/normal and the filter) is one CUDA graph: each problem's kernels
 * form an independent chain of the graph, so that the problems' kernels run
 * side by side and one problem's tail overlaps the others' work.  The
 * kernels are the per-problem launches' own (hpm_pm.cu), with their
 * arguments in the parameter space, so each problem's maps equal
 * hpm_process_problem's on a fresh context bit for bit.
 *
 *  - The graph is captured once per batch and kind of pass and, for every
 *    later pass, re-captured with the pass's arguments (seeds, pass flags)
 *    and applied to the instantiated graph by cudaGraphExecUpdate.
 *  - The half-step tile (pixels of one colour per warp row: 4, 8 or 16) is
 *    picked per view size by timing one half-step of each on the scene's
 *    first problem of that size (kept in the context for later scenes).
 *  - Pass set A advances pass by pass: the plain pass of every problem, then
 *    each pyramid level's prior (built per problem on the host and device,
 *    as in hpm_process_problem) and the batched prior pass.  Problems whose
 *    pyramid is shorter join at its first level (levels aligned at the full
 *    scale).
 *  - The geometric iterations read the previous iteration's maps of every
 *    view (as the view-sharded driver does); the reference's in-place order
 *    would serialise the problems.
 *
 * A first design ran all problems of a half-step as one persistent launch
 * whose CTAs walked a (problem, tile) work list, the arguments read from
 * device memory.  It measured 0.61x the per-problem driver on 24 views of
 * three sizes (argument loads from global memory in the innermost loops,
 * more register spills) and, compiled differently, was not bit-identical
 * to it; the graph form replaced it.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "hpm_capi_internal.h"
#include "hpm_nvtx.h"
#include "hpm_prior.h"

using namespace hpm;

#define CK(call, what)                                            \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return ctx_cuda_fail(c, e_, what); \
    } while (0)

namespace {

int scale_levels_of(int w, int h) /* ComputingMultiScaleSettings, HPM.cpp:851-860 */
{
    int m = w > h ? w : h, k = 0;
    while (m > 1000) {
        m /= 2;
        k++;
    }
    return k;
}

__global__ void k_pack_maps(const float *__restrict__ normal3, const float *__restrict__ depth, int n,
                            float4 *__restrict__ planes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    planes[i] = make_float4(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2], depth[i]);
}

/* f(p) for every problem p < n on up to 4 host threads, so that one
 * problem's host work between passes (the Delaunay of its prior levels,
 * with the synchronisations around it) overlaps the others' device work.
 * f may touch only problem p's own context and stream, and reports a
 * failure there.  Every thread first makes `device` its current device (a
 * new host thread starts on device 0).  Returns the failure of the lowest
 * failing problem (after all threads have stopped) and its index in
 * *failed. */
template <typename F>
int for_each_problem(int device, int n, F f, int *failed)
{
    const int workers = std::max(1, std::min(4, n));
    std::atomic<int> next{0};
    std::atomic<bool> stop{false};
    std::vector<int> rc(n, HPM_OK);
    auto run = [&]() {
        if (cudaSetDevice(device) != cudaSuccess) {
            stop.store(true);
            return;
        }
        for (;;) {
            const int p = next.fetch_add(1);
            if (p >= n || stop.load()) return;
            rc[p] = f(p);
            if (rc[p]) stop.store(true);
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < workers; ++w) pool.emplace_back(run);
    run();
    for (std::thread &t : pool) t.join();
    for (int p = 0; p < n; ++p)
        if (rc[p]) {
            *failed = p;
            return rc[p];
        }
    if (stop.load()) { /* a thread could not select the device */
        *failed = 0;
        return HPM_ERR_CUDA;
    }
    return HPM_OK;
}

/* A batch of problem contexts, their half-step tile widths, and the
 * instantiated graph of each kind of pass (keyed by the number of
 * half-steps). */
struct Plan {
    std::vector<hpm_ctx *> ctxs;
    std::vector<int> ww;
    std::vector<std::pair<int, cudaGraphExec_t>> graphs;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;

    ~Plan()
    {
        for (auto &g : graphs) cudaGraphExecDestroy(g.second);
        if (fork) cudaEventDestroy(fork);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
    }
};

int make_plan(hpm_ctx *c, const std::vector<hpm_ctx *> &ctxs, const std::vector<int> &ww, Plan &pl)
{
    pl.ctxs = ctxs;
    pl.ww = ww;
    CK(cudaEventCreateWithFlags(&pl.fork, cudaEventDisableTiming), "batch events");
    pl.join.assign(ctxs.size(), nullptr);
    for (cudaEvent_t &e : pl.join) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch events");
    return HPM_OK;
}
/* One batched pass with per-problem parameters and `half_steps` half-steps
 * (the reference's 6 unless the prior-net forms ask for fewer iterations).
 * Each problem's chain goes to its own context's stream, forked from and
 * joined back to c's stream, all captured as one graph; the graph of the
 * previous pass of this kind is updated to the new arguments and replayed.
 * A problem whose context holds proposals runs the prior-net form's
 * refinement (the proposal as a candidate). */
int batch_pass(hpm_ctx *c, Plan &pl, const std::vector<HpmParams> &params, int half_steps = 6)
{
    cudaStream_t s = c->stream;
    const size_t n = pl.ctxs.size();
    std::vector<PMArgs> args(n);
    for (size_t i = 0; i < n; ++i) {
        const int r = ctx_pass_args(pl.ctxs[i], &params[i], &args[i]);
        if (r) return ctx_fail(c, r, "batched pass, problem %zu: %s", i, hpm_last_error(pl.ctxs[i]));
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t e = cudaEventRecord(pl.fork, s);
    for (size_t i = 0; i < n && e == cudaSuccess; ++i) {
        hpm_ctx *b = pl.ctxs[i];
        const cudaStream_t bs = b->stream;
        e = cudaStreamWaitEvent(bs, pl.fork, 0);
        if (e == cudaSuccess) e = launch_init(args[i], bs);
        for (int hs = 0; hs < half_steps && e == cudaSuccess; ++hs)
            e = launch_propagate(args[i], hs / 2, hs % 2, bs, pl.ww[i]);
        if (e == cudaSuccess)
            e = launch_depth_normal_filter(args[i], reinterpret_cast<float4 *>(ctx_planes(b)), ctx_costs(b), bs);
        if (e == cudaSuccess) e = cudaEventRecord(pl.join[i], bs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, pl.join[i], 0);
    }
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (e == cudaSuccess) e = ce;
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ctx_cuda_fail(c, e, "batched pass capture");
    }
    cudaGraphExec_t *exec = nullptr;
    for (auto &x : pl.graphs)
        if (x.first == half_steps) exec = &x.second;
    if (exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(*exec, g, &info) != cudaSuccess) {
            cudaGetLastError(); /* topology changed: instantiate anew */
            cudaGraphExecDestroy(*exec);
            *exec = nullptr;
        }
    } else {
        pl.graphs.push_back({half_steps, nullptr});
        exec = &pl.graphs.back().second;
    }
    e = *exec ? cudaSuccess : cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    CK(e, "graph instantiate");
    CK(cudaGraphLaunch(*exec, s), "graph launch");
    CK(cudaStreamSynchronize(s), "batched pass");
    return HPM_OK;
}

/* The half-step tile width for each problem: per view size the fastest of
 * 4, 8 and 16 pixels per warp row, timed on one half-step of the scene's first
 * problem of that size (its state is re-initialised by the real passes). */
int tune_tiles(hpm_ctx *c, const std::vector<hpm_ctx *> &ctxs, const std::vector<HpmParams> &params,
               std::vector<int> &ww)
{
    ww.assign(ctxs.size(), 8);
    for (size_t i = 0; i < ctxs.size(); ++i) {
        const HpmCamera &cam = ctxs[i]->cams[0];
        const long long key = ((long long)cam.width << 32) | (unsigned)cam.height;
        int found = 0;
        for (auto &kv : c->tile_ww)
            if (kv.first == key) found = kv.second;
        if (!found) {
            float best = 1e30f;
            cudaEvent_t e0, e1;
            CK(cudaEventCreate(&e0), "tuning events");
            CK(cudaEventCreate(&e1), "tuning events");
            for (int cand : {4, 8, 16}) {
                PMArgs a;
                const int r = ctx_pass_args(ctxs[i], &params[i], &a);
                if (r) return ctx_fail(c, r, "tile tuning: %s", hpm_last_error(ctxs[i]));
                CK(launch_init(a, c->stream), "tuning init");
                CK(cudaEventRecord(e0, c->stream), "tuning");
                CK(launch_propagate(a, 0, 0, c->stream, cand), "tuning half-step");
                CK(cudaEventRecord(e1, c->stream), "tuning");
                CK(cudaEventSynchronize(e1), "tuning");
                float ms = 0.0f;
                CK(cudaEventElapsedTime(&ms, e0, e1), "tuning");
                if (ms < best) {
                    best = ms;
                    found = cand;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            c->tile_ww.push_back({key, found});
            ctx_reset_salt(ctxs[i]);
        }
        ww[i] = found;
    }
    return HPM_OK;
}
/* Pass set A in the prior-net form for every problem of pc (full-scale
 * views set): the 1/4-scale plain passes as one batched pass over the
 * problems' coarse sub-contexts, per problem the coarse planar prior, the
 * network and the full-scale start (net_full_setup), then 1 + extra_passes
 * batched full-scale passes with the proposal candidate; seeds as
 * net_problem's, so each problem's maps equal it bit for bit. */
int net_pass_set_a(hpm_ctx *c, const std::vector<hpm_ctx *> &pc, const std::vector<HpmParams> &params, Plan &all,
                   const HpmNetWeights *net, int extra_passes, int prior_mode, int half_steps,
                   const std::vector<std::vector<const float *>> &images)
{
    const int n = (int)pc.size();
    int bad = 0;
    int r = for_each_problem(
        c->device, n, [&](int p) { return net_coarse_views(pc[p], pc[p]->n, images[p].data(), pc[p]->cams); }, &bad);
    if (r) return ctx_fail(c, r, "batched prior-net form, problem %d: %s", bad, hpm_last_error(pc[bad]));
    std::vector<hpm_ctx *> cc(n);
    for (int p = 0; p < n; ++p) cc[p] = pc[p]->coarse;
    {
        const Range coarse("batched coarse passes");
        std::vector<int> cww;
        r = tune_tiles(c, cc, params, cww);
        if (r) return r;
        Plan cplan;
        r = make_plan(c, cc, cww, cplan);
        if (!r) r = batch_pass(c, cplan, params);
        if (r) return r;
    }
    r = for_each_problem(
        c->device, n,
        [&](int p) {
            int q = net_coarse_finish(pc[p], params[p].depth_min, params[p].depth_max);
            return q ? q : net_full_setup(pc[p], net, prior_mode);
        },
        &bad);
    if (r) return ctx_fail(c, r, "batched prior-net form, problem %d: %s", bad, hpm_last_error(pc[bad]));
    std::vector<HpmParams> fp(params);
    for (int e = 0; e <= extra_passes; ++e) {
        r = for_each_problem(
            c->device, n,
            [&](int p) {
                hpm_ctx *b = pc[p];
                if (e > 0) {
                    const size_t np = (size_t)b->cams[0].width * b->cams[0].height;
                    const cudaError_t ce = flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(b)), (int)np,
                                                            b->flow.full_depth, b->flow.full_normal, b->stream);
                    if (ce != cudaSuccess) return ctx_cuda_fail(b, ce, "split");
                    const int q = flow_prior_from_maps(b, 2, ctx_costs(b), params[p].depth_min, params[p].depth_max);
                    if (q) return q;
                }
                const cudaError_t ce = cudaStreamSynchronize(b->stream);
                return ce == cudaSuccess ? HPM_OK : ctx_cuda_fail(b, ce, "prior-net set-up");
            },
            &bad);
        if (r) return ctx_fail(c, r, "batched prior-net form, problem %d: %s", bad, hpm_last_error(pc[bad]));
        for (int p = 0; p < n; ++p) {
            fp[p].planar_prior = 1;
            fp[p].seed = net_pass_seed(params[p].seed, e);
        }
        r = batch_pass(c, all, fp, half_steps);
        if (r) return r;
    }
    for (int p = 0; p < n; ++p) {
        pc[p]->proposals = nullptr;
        r = net_status(pc[p]);
        if (r) return ctx_fail(c, r, "batched prior-net form, problem %d: %s", p, hpm_last_error(pc[p]));
    }
    return HPM_OK;
}

int batched_scene(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams, int n_problems,
                  const int *ref_ids, const int *src_counts, const int *src_ids, const HpmSceneOpts *o,
                  const HpmNetWeights *net, float *const *out_depths, float *const *out_normals,
                  float *const *out_costs)
{
    if (!c || !images || !cams || !ref_ids || !src_counts || !src_ids || !o) return HPM_ERR_ARG;
    if (n_views < 2 || n_problems < 1)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_batched: %d views, %d problems", n_views, n_problems);
    for (int p = 0; p < n_problems; ++p) {
        if (ref_ids[p] < 0 || ref_ids[p] >= n_views || src_counts[p] < 1 || src_counts[p] > kMaxSrc)
            return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_batched: problem %d is malformed", p);
        for (int j = 0; j < src_counts[p]; ++j) {
            const int sv = src_ids[p * kMaxSrc + j];
            if (sv < 0 || sv >= n_views)
                return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_batched: problem %d source %d", p, sv);
        }
    }
    int r = ctx_select_device(c);
    if (r) return r;
    const Range range(net ? "batched scene %d views (prior-net form)" : "batched scene %d views", n_views);
    if (o->iterations < 0 || o->iterations > 64 || o->geom_pass_iterations < 0 || o->geom_pass_iterations > 64)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_batched: iterations outside [0, 64]");
    const int half_steps = net && o->iterations > 0 ? 2 * o->iterations : 6;
    const int geom_half_steps = net && o->geom_pass_iterations > 0 ? 2 * o->geom_pass_iterations : half_steps;
    cudaStream_t s = c->stream;
    /* per view: image, pass-A depth, two geometric depth buffers, normal (3), cost */
    std::vector<float *> img(n_views), dep_a(n_views), dep_g0(n_views), dep_g1(n_views), nrm(n_views), cst(n_views);
    size_t total = 0;
    for (int v = 0; v < n_views; ++v) total += 8 * (((size_t)cams[v].width * cams[v].height + 63) & ~(size_t)63);
    CK(ctx_scene_arena(c, total * sizeof(float)), "scene buffers");
    float *cur = ctx_scene_base(c);
    CK(cudaMemsetAsync(cur, 0, total * sizeof(float), s), "scene buffers");
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height, st = (np + 63) & ~(size_t)63;
        img[v] = cur;
        dep_a[v] = cur + st;
        dep_g0[v] = cur + 2 * st;
        dep_g1[v] = cur + 3 * st;
        nrm[v] = cur + 4 * st;
        cst[v] = cur + 7 * st;
        cur += 8 * st;
        CK(cudaMemcpyAsync(img[v], images[v], sizeof(float) * np, cudaMemcpyDefault, s), "scene images");
    }
    CK(cudaStreamSynchronize(s), "scene images");
    /* one context per problem, kept for later scenes */
    while ((int)c->batch.size() < n_problems) {
        hpm_ctx *b = nullptr;
        r = ctx_create_child(c, &b);
        if (b) c->batch.push_back(b); /* owned by c from here, freed with it */
        if (r) return ctx_fail(c, r, "hpm_run_scene_batched: problem context");
    }
    std::vector<hpm_ctx *> pc(c->batch.begin(), c->batch.begin() + n_problems);
    std::vector<HpmParams> params(n_problems);
    std::vector<int> levels(n_problems);
    std::vector<std::vector<const float *>> pimgs(n_problems);
    for (int p = 0; p < n_problems; ++p) {
        HpmCamera pcam[kMaxViews];
        const int ref = ref_ids[p], ns = src_counts[p];
        std::vector<const float *> &pimg = pimgs[p];
        pimg.assign(ns + 1, nullptr);
        pimg[0] = img[ref];
        pcam[0] = cams[ref];
        for (int j = 0; j < ns; ++j) {
            const int sv = src_ids[p * kMaxSrc + j];
            pimg[j + 1] = img[sv];
            pcam[j + 1] = cams[sv];
        }
        r = hpm_set_views(pc[p], pimg.data(), pcam, ns + 1);
        if (r) return ctx_fail(c, r, "hpm_run_scene_batched, problem %d: %s", p, hpm_last_error(pc[p]));
        hpm_clear_prior(pc[p]);
        ctx_reset_salt(pc[p]);
        hpm_default_params(&params[p]);
        params[p].depth_min = cams[ref].depth_min * 0.6f; /* InuputInitialization, HPM.cpp:553-554 */
        params[p].depth_max = cams[ref].depth_max * 1.2f;
        params[p].seed = o->seed + (uint64_t)p;
        params[p].fix_quirks = o->fix_quirks;
        pc[p]->fix_quirks = o->fix_quirks != 0;
        levels[p] = o->pyramid_levels >= 0 ? o->pyramid_levels : scale_levels_of(cams[ref].width, cams[ref].height);
    }
    std::vector<int> ww;
    r = tune_tiles(c, pc, params, ww);
    if (r) return r;

    /* one plan (and graph) for the passes that cover every problem */
    Plan all;
    r = make_plan(c, pc, ww, all);
    if (r) return r;
    if (net) {
        /* pass set A in the prior-net form */
        r = net_pass_set_a(c, pc, params, all, net, o->pyramid_levels > 0 ? o->pyramid_levels : 0,
                           o->planar_prior, half_steps, pimgs);
        if (r) return r;
    } else {
        /* pass set A: the plain pass of every problem */
        r = batch_pass(c, all, params);
        if (r) return r;
    }
    /* the prior passes, levels aligned at the full scale */
    if (o->planar_prior && !net) {
        const int kmax = *std::max_element(levels.begin(), levels.end());
        for (int round = 0; round <= kmax; ++round) {
            const int level = 2 - kmax + round; /* 0: 1/4 scale, 1: 1/2, 2: full */
            std::vector<int> in; /* the problems whose pyramid reaches this level */
            for (int p = 0; p < n_problems; ++p)
                if (level >= 2 - levels[p]) in.push_back(p);
            int bad = 0;
            r = for_each_problem(
                c->device, (int)in.size(),
                [&](int i) {
                    const int p = in[i];
                    hpm_ctx *b = pc[p];
                    const size_t np = (size_t)b->cams[0].width * b->cams[0].height;
                    cudaError_t ce = ws_reserve_full(b, np);
                    if (ce == cudaSuccess)
                        ce = flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(b)), (int)np,
                                              b->flow.full_depth, b->flow.full_normal, b->stream);
                    if (ce != cudaSuccess) return ctx_cuda_fail(b, ce, "prior level");
                    const int q = flow_prior_from_maps(b, level, ctx_costs(b), params[p].depth_min, params[p].depth_max);
                    if (q) return q;
                    ce = cudaStreamSynchronize(b->stream);
                    return ce == cudaSuccess ? HPM_OK : ctx_cuda_fail(b, ce, "prior level");
                },
                &bad);
            if (r) return ctx_fail(c, r, "hpm_run_scene_batched, problem %d: %s", in[bad], hpm_last_error(pc[in[bad]]));
            std::vector<hpm_ctx *> sub;
            std::vector<HpmParams> sp;
            std::vector<int> sw;
            for (int p : in) {
                HpmParams q = params[p];
                q.planar_prior = 1;
                sub.push_back(pc[p]);
                sp.push_back(q);
                sw.push_back(ww[p]);
            }
            if (sub.size() == pc.size()) {
                r = batch_pass(c, all, sp);
            } else {
                Plan pl;
                r = make_plan(c, sub, sw, pl);
                if (!r) r = batch_pass(c, pl, sp);
            }
            if (r) return r;
        }
    }
    for (int p = 0; p < n_problems; ++p) {
        const int ref = ref_ids[p];
        const size_t np = (size_t)cams[ref].width * cams[ref].height;
        CK(flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(pc[p])), (int)np, dep_a[ref], nrm[ref], s),
           "split");
        CK(cudaMemcpyAsync(cst[ref], ctx_costs(pc[p]), sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
    }
    CK(cudaStreamSynchronize(s), "pass set A");

    /* geometric iterations: each reads the previous iteration's maps of every view */
    std::vector<float *> *src = &dep_a, *dst = &dep_g0;
    for (int gi = 0; gi < o->geom_iterations; ++gi) {
        const Range iteration("batched geometric iteration %d", gi);
        std::vector<HpmParams> gp(n_problems);
        for (int p = 0; p < n_problems; ++p) {
            const int ref = ref_ids[p], ns = src_counts[p];
            const float *pd[kMaxViews];
            pd[0] = (*src)[ref];
            for (int j = 0; j < ns; ++j) pd[j + 1] = (*src)[src_ids[p * kMaxSrc + j]];
            r = hpm_set_geom_depths(pc[p], pd);
            if (r) return ctx_fail(c, r, "hpm_run_scene_batched, problem %d: %s", p, hpm_last_error(pc[p]));
            const int np = cams[ref].width * cams[ref].height;
            k_pack_maps<<<(np + 255) / 256, 256, 0, s>>>(nrm[ref], (*src)[ref], np,
                                                          reinterpret_cast<float4 *>(ctx_planes(pc[p])));
            CK(cudaMemcpyAsync(ctx_costs(pc[p]), cst[ref], sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
            gp[p] = params[p];
            gp[p].geom_consistency = 1;
            gp[p].multi_geometry = gi >= 1;
            gp[p].seed = o->seed + 1000003ull * (gi + 1) + (uint64_t)p;
        }
        CK(cudaStreamSynchronize(s), "geometric set-up");
        r = batch_pass(c, all, gp, geom_half_steps);
        if (r) return r;
        for (int p = 0; p < n_problems; ++p) {
            const int ref = ref_ids[p];
            const size_t np = (size_t)cams[ref].width * cams[ref].height;
            CK(flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(pc[p])), (int)np, (*dst)[ref], nrm[ref],
                                s),
               "split");
            CK(cudaMemcpyAsync(cst[ref], ctx_costs(pc[p]), sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
        }
        CK(cudaStreamSynchronize(s), "geometric iteration");
        src = dst;
        dst = (dst == &dep_g0) ? &dep_g1 : &dep_g0;
    }
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height;
        if (out_depths && out_depths[v])
            CK(cudaMemcpyAsync(out_depths[v], (*src)[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
        if (out_normals && out_normals[v])
            CK(cudaMemcpyAsync(out_normals[v], nrm[v], sizeof(float) * 3 * np, cudaMemcpyDefault, s), "out");
        if (out_costs && out_costs[v])
            CK(cudaMemcpyAsync(out_costs[v], cst[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
    }
    CK(cudaStreamSynchronize(s), "hpm_run_scene_batched");
    return HPM_OK;
}

}  // namespace

extern "C" int hpm_run_scene_batched(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                                     int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                                     const HpmSceneOpts *o, float *const *out_depths, float *const *out_normals,
                                     float *const *out_costs)
{
    return batched_scene(c, n_views, images, cams, n_problems, ref_ids, src_counts, src_ids, o, nullptr, out_depths,
                         out_normals, out_costs);
}

extern "C" int hpm_run_scene_batched_net(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                                         int n_problems, const int *ref_ids, const int *src_counts,
                                         const int *src_ids, const HpmSceneOpts *o, const HpmNetWeights *net,
                                         float *const *out_depths, float *const *out_normals, float *const *out_costs)
{
    if (!net) return HPM_ERR_ARG;
    for (int l = 0; l < 4; ++l)
        if (!net->packed[l] || !net->bias[l]) return HPM_ERR_ARG;
    return batched_scene(c, n_views, images, cams, n_problems, ref_ids, src_counts, src_ids, o, net, out_depths,
                         out_normals, out_costs);
}

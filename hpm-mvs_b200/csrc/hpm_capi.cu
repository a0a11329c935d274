/*
 * C ABI of the B200-native HPM-MVS PatchMatch path: context, device memory
 * and pass orchestration.  Declarations and the reference interfaces they
 * replace: include/hpm_b200.h.
 *
 * Memory: a context owns one set of device buffers sized for the largest
 * problem it has seen (images, optional geometric depth maps, hypotheses,
 * costs, view masks, prior planes and masks).  Nothing is freed between
 * passes or problems, unlike the reference which allocates and frees every
 * buffer per problem (HPM.cpp:591-700, 1283-1307).  All work is issued on the
 * context's stream; the only host synchronisations are in the calls that
 * return data to the host.
 */
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_bf16.h>

#include "hpm_capi_internal.h"
#include "hpm_nvtx.h"

using namespace hpm;

namespace {

int fail(hpm_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int cuda_fail(hpm_ctx *c, cudaError_t e, const char *what)
{
    return fail(c, e == cudaErrorMemoryAllocation ? HPM_ERR_NOMEM : HPM_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

cudaError_t ensure(void **p, size_t *cap, size_t bytes)
{
    if (*cap >= bytes && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) *cap = bytes;
    return e;
}

/* Float cudaArray + texture object of view i with the reference's sampling
 * state (HPM.cpp:599-616): linear filter, unnormalised coordinates, element
 * reads.  The reference asks for wrap addressing, which the hardware treats
 * as clamp for unnormalised coordinates (pinned by tests/golden/tex_probe);
 * clamp is requested explicitly here.  A texture's extent is its array's, so
 * each view slot keeps a few arrays of the sizes it has held (kTexPerSlot,
 * most recently used last): problems of a scene whose views differ in size
 * reuse them instead of freeing one (which waits for the whole device) and
 * allocating another for nearly every view. */
constexpr size_t kTexPerSlot = 3;

cudaError_t ensure_texture(hpm_ctx *c, int i, int w, int h)
{
    std::vector<TexArray> &pool = c->tex_pool[i];
    for (size_t k = 0; k < pool.size(); ++k)
        if (pool[k].w == w && pool[k].h == h) {
            const TexArray t = pool[k];
            pool.erase(pool.begin() + (long)k);
            pool.push_back(t);
            c->arr[i] = t.arr;
            c->tex[i] = t.tex;
            return cudaSuccess;
        }
    c->arr[i] = nullptr;
    c->tex[i] = 0;
    if (pool.size() >= kTexPerSlot) {
        cudaDestroyTextureObject(pool.front().tex);
        cudaFreeArray(pool.front().arr);
        pool.erase(pool.begin());
    }
    TexArray t;
    cudaChannelFormatDesc desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaError_t e = cudaMallocArray(&t.arr, &desc, w, h);
    if (e != cudaSuccess) return e;
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = t.arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&t.tex, &res, &td, nullptr);
    if (e != cudaSuccess) {
        cudaFreeArray(t.arr);
        return e;
    }
    t.w = w;
    t.h = h;
    pool.push_back(t);
    c->arr[i] = t.arr;
    c->tex[i] = t.tex;
    return cudaSuccess;
}

int select_device(hpm_ctx *c)
{
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    return HPM_OK;
}

PMArgs make_args(hpm_ctx *c)
{
    PMArgs a;
    memset(&a, 0, sizeof(a));
    a.n = c->n;
    a.W = c->cams[0].width;
    a.H = c->cams[0].height;
    a.rows_cov = rows_covered(a.H);
    a.radius = 5;
    a.radius_increment = 2;
    a.sigma_spatial = 5.0f;
    a.sigma_color = 3.0f;
    a.top_k = 4;
    for (int i = 0; i < c->n; ++i) {
        a.cam[i] = c->cams[i];
        a.view[i].img = c->d_img[i];
        a.view[i].depth = c->has_depth ? c->d_depth[i] : nullptr;
        a.view[i].tex = c->tex[i];
        a.view[i].w = c->cams[i].width;
        a.view[i].h = c->cams[i].height;
    }
    a.pair = c->d_pair;
    a.planes = c->d_planes;
    a.costs = c->d_costs;
    a.views = c->d_views;
    a.prior_planes = c->d_prior;
    a.masks = c->d_masks;
    a.counters = c->counting ? c->d_counters : nullptr;
    a.cost_cache = c->d_cache;
    a.cand_costs = c->d_cand;
    a.cand_pos = c->d_pos;
    a.cand_flags = c->d_flags;
    a.proposals = c->proposals;
    a.geom_max = 5.0f; /* HPM.cu:485 */
    return a;
}

size_t npx(const hpm_ctx *c) { return (size_t)c->cams[0].width * c->cams[0].height; }

void prof_begin(hpm_ctx *c, int kind, cudaEvent_t *e0)
{
    *e0 = nullptr;
    if (!c->profiling) return;
    cudaEventCreate(e0);
    cudaEventRecord(*e0, c->stream);
    (void)kind;
}

void prof_end(hpm_ctx *c, int kind, cudaEvent_t e0)
{
    if (!c->profiling || !e0) return;
    cudaEvent_t e1;
    cudaEventCreate(&e1);
    cudaEventRecord(e1, c->stream);
    c->prof_events.push_back({kind, {e0, e1}});
}

}  // namespace

extern "C" {

void hpm_default_params(HpmParams *p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->max_iterations = 3;
    p->patch_size = 11;
    p->radius_increment = 2;
    p->sigma_spatial = 5.0f;
    p->sigma_color = 3.0f;
    p->top_k = 4;
    p->depth_min = 0.0f;
    p->depth_max = 1.0f;
}

int hpm_create(hpm_ctx **out, int device)
{
    if (!out) return HPM_ERR_ARG;
    *out = nullptr;
    hpm_ctx *c = new (std::nothrow) hpm_ctx();
    if (!c) return HPM_ERR_NOMEM;
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_pair, sizeof(PairGeom) * kMaxViews);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_counters, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        delete c;
        return e == cudaErrorMemoryAllocation ? HPM_ERR_NOMEM : HPM_ERR_CUDA;
    }
    *out = c;
    return HPM_OK;
}

int hpm_destroy(hpm_ctx *c)
{
    if (!c) return HPM_ERR_ARG;
    if (c->peer) hpm_destroy(c->peer);
    c->peer = nullptr;
    if (c->coarse) hpm_destroy(c->coarse);
    c->coarse = nullptr;
    for (hpm_ctx *b : c->batch) hpm_destroy(b);
    c->batch.clear();
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < kMaxViews; ++i) {
        cudaFree(c->d_img[i]);
        cudaFree(c->d_depth[i]);
        for (const TexArray &t : c->tex_pool[i]) {
            cudaDestroyTextureObject(t.tex);
            cudaFreeArray(t.arr);
        }
    }
    cudaFree(c->d_pair);
    cudaFree(c->d_planes);
    cudaFree(c->d_costs);
    cudaFree(c->d_views);
    cudaFree(c->d_prior);
    cudaFree(c->d_masks);
    cudaFree(c->d_counters);
    cudaFree(c->d_scene);
    cudaFree(c->d_scratch);
    cudaFree(c->d_cache);
    cudaFree(c->d_cand);
    cudaFree(c->d_pos);
    cudaFree(c->d_flags);
    cudaFree(c->d_pre);
    ws_free(c);
    net_free(c);
    for (auto &p : c->prof_events) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return HPM_OK;
}

const char *hpm_last_error(const hpm_ctx *c) { return c ? c->err : "null context"; }

void *hpm_stream(hpm_ctx *c) { return c ? (void *)c->stream : nullptr; }

int hpm_set_views(hpm_ctx *c, const float *const *images, const HpmCamera *cams, int num_images)
{
    if (!c) return HPM_ERR_ARG;
    if (!images || !cams) return fail(c, HPM_ERR_ARG, "hpm_set_views: null images or cameras");
    if (num_images < 2 || num_images > kMaxViews)
        return fail(c, HPM_ERR_ARG, "hpm_set_views: num_images=%d outside [2, %d]", num_images, kMaxViews);
    for (int i = 0; i < num_images; ++i) {
        if (!images[i]) return fail(c, HPM_ERR_ARG, "hpm_set_views: image %d is null", i);
        if (cams[i].width < 1 || cams[i].height < 1 || cams[i].width > 16384 || cams[i].height > 16384)
            return fail(c, HPM_ERR_ARG, "hpm_set_views: image %d has size %dx%d", i, cams[i].width,
                        cams[i].height);
    }
    int r = select_device(c);
    if (r) return r;
    for (int i = 0; i < num_images; ++i) {
        const size_t bytes = sizeof(float) * cams[i].width * cams[i].height;
        CK(ensure((void **)&c->d_img[i], &c->img_cap[i], bytes), "image alloc");
        CK(cudaMemcpyAsync(c->d_img[i], images[i], bytes, cudaMemcpyDefault, c->stream), "image upload");
        CK(ensure_texture(c, i, cams[i].width, cams[i].height), "texture set-up");
        CK(cudaMemcpy2DToArrayAsync(c->arr[i], 0, 0, c->d_img[i], sizeof(float) * cams[i].width,
                                    sizeof(float) * cams[i].width, cams[i].height, cudaMemcpyDeviceToDevice,
                                    c->stream),
           "texture upload");
        c->cams[i] = cams[i];
    }
    c->n = num_images;
    c->pass_counter = 0; /* random stream ids restart with every problem */
    c->has_depth = false;
    c->has_prior = false;
    const size_t n = npx(c);
    if (c->px_cap < n) {
        cudaFree(c->d_planes);
        cudaFree(c->d_costs);
        cudaFree(c->d_views);
        cudaFree(c->d_prior);
        cudaFree(c->d_masks);
        c->d_planes = nullptr;
        c->d_costs = nullptr;
        c->d_views = nullptr;
        c->d_prior = nullptr;
        c->d_masks = nullptr;
        c->px_cap = 0;
        CK(cudaMalloc(&c->d_planes, sizeof(float4) * n), "state alloc");
        CK(cudaMalloc(&c->d_costs, sizeof(float) * n), "state alloc");
        CK(cudaMalloc(&c->d_views, sizeof(uint32_t) * n), "state alloc");
        CK(cudaMalloc(&c->d_prior, sizeof(float4) * n), "state alloc");
        CK(cudaMalloc(&c->d_masks, sizeof(uint32_t) * n), "state alloc");
        c->px_cap = n;
    }
    /* per-colour planes of ceil(n / 2) pixels (hpm_pm.cu: Slot) */
    const size_t nh = (n + 1) / 2;
    CK(ensure((void **)&c->d_cache, &c->cache_cap, sizeof(float) * 2 * nh * (num_images - 1)), "cache alloc");
    CK(ensure((void **)&c->d_cand, &c->cand_cap, sizeof(float) * nh * (num_images - 1) * kCandRows), "cand alloc");
    CK(ensure((void **)&c->d_pos, &c->pos_cap, sizeof(int) * nh * 8), "cand alloc");
    CK(ensure((void **)&c->d_flags, &c->flags_cap, sizeof(uint32_t) * nh), "cand alloc");
    CK(cudaMemsetAsync(c->d_planes, 0, sizeof(float4) * n, c->stream), "state clear");
    CK(cudaMemsetAsync(c->d_costs, 0, sizeof(float) * n, c->stream), "state clear");
    CK(cudaMemsetAsync(c->d_views, 0, sizeof(uint32_t) * n, c->stream), "state clear");
    PMArgs a = make_args(c);
    CK(launch_pair_geom(a, c->d_pair, c->stream), "pair geometry");
    c->has_state = false;
    /* synchronous semantics for the caller's host buffers */
    CK(cudaStreamSynchronize(c->stream), "hpm_set_views");
    return HPM_OK;
}

int hpm_set_geom_depths(hpm_ctx *c, const float *const *depths)
{
    if (!c) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_set_geom_depths before hpm_set_views");
    if (!depths) return fail(c, HPM_ERR_ARG, "hpm_set_geom_depths: null");
    int r = select_device(c);
    if (r) return r;
    for (int i = 0; i < c->n; ++i) {
        if (!depths[i]) return fail(c, HPM_ERR_ARG, "hpm_set_geom_depths: depth %d is null", i);
        const size_t bytes = sizeof(float) * c->cams[i].width * c->cams[i].height;
        CK(ensure((void **)&c->d_depth[i], &c->depth_cap[i], bytes), "depth alloc");
        CK(cudaMemcpyAsync(c->d_depth[i], depths[i], bytes, cudaMemcpyDefault, c->stream), "depth upload");
    }
    c->has_depth = true;
    CK(cudaStreamSynchronize(c->stream), "hpm_set_geom_depths");
    return HPM_OK;
}

int hpm_set_hypotheses(hpm_ctx *c, const float *planes, const float *costs)
{
    if (!c) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_set_hypotheses before hpm_set_views");
    if (!planes) return fail(c, HPM_ERR_ARG, "hpm_set_hypotheses: null planes");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c);
    CK(cudaMemcpyAsync(c->d_planes, planes, sizeof(float4) * n, cudaMemcpyDefault, c->stream), "planes");
    if (costs)
        CK(cudaMemcpyAsync(c->d_costs, costs, sizeof(float) * n, cudaMemcpyDefault, c->stream), "costs");
    else
        CK(cudaMemsetAsync(c->d_costs, 0, sizeof(float) * n, c->stream), "costs");
    c->has_state = true;
    CK(cudaStreamSynchronize(c->stream), "hpm_set_hypotheses");
    return HPM_OK;
}

int hpm_set_prior(hpm_ctx *c, const float *prior_planes, const uint32_t *masks)
{
    if (!c) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_set_prior before hpm_set_views");
    if (!prior_planes || !masks) return fail(c, HPM_ERR_ARG, "hpm_set_prior: null input");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c);
    CK(cudaMemcpyAsync(c->d_prior, prior_planes, sizeof(float4) * n, cudaMemcpyDefault, c->stream), "prior");
    CK(cudaMemcpyAsync(c->d_masks, masks, sizeof(uint32_t) * n, cudaMemcpyDefault, c->stream), "masks");
    c->has_prior = true;
    CK(cudaStreamSynchronize(c->stream), "hpm_set_prior");
    return HPM_OK;
}

int hpm_clear_prior(hpm_ctx *c)
{
    if (!c) return HPM_ERR_ARG;
    c->has_prior = false;
    return HPM_OK;
}

/* Checks p against the context's state and fills the pass fields of *out;
 * takes the pass's random-stream salt.  Shared by run_pass and
 * ctx_pass_args. */
static int pass_args(hpm_ctx *c, const HpmParams *p, PMArgs *out)
{
    if (!p) return fail(c, HPM_ERR_ARG, "hpm_run_patchmatch: null params");
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_run_patchmatch before hpm_set_views");
    if (p->patch_size != 11 || p->radius_increment != 2)
        return fail(c, HPM_ERR_ARG, "hpm_run_patchmatch: only the reference window (11, stride 2) is built");
    if (p->geom_consistency && !c->has_depth)
        return fail(c, HPM_ERR_STATE, "geometric consistency needs hpm_set_geom_depths");
    if (p->planar_prior && !c->has_prior) return fail(c, HPM_ERR_STATE, "planar prior needs hpm_set_prior");
    if (!(p->depth_max > p->depth_min)) return fail(c, HPM_ERR_ARG, "depth range is empty");
    if (p->top_k < 1 || p->top_k > kMaxSrc) return fail(c, HPM_ERR_ARG, "top_k outside [1, %d]", kMaxSrc);
    if (p->variant != 0 && p->variant != 1)
        return fail(c, HPM_ERR_ARG, "variant %d: 0 (HPM-MVS) or 1 (ACMM+NESP)", p->variant);
    if (p->variant == 1 && p->planar_prior) return fail(c, HPM_ERR_ARG, "the ACMM+NESP variant has no planar prior");
    if (p->hierarchy < 0 || p->hierarchy > 2) return fail(c, HPM_ERR_ARG, "hierarchy %d outside [0, 2]", p->hierarchy);
    if (p->hierarchy && (p->variant != 1 || p->geom_consistency))
        return fail(c, HPM_ERR_ARG, "a hierarchy pass belongs to the ACMM+NESP variant and has no geometric term");
    if (p->hierarchy && !c->has_state)
        return fail(c, HPM_ERR_STATE, "a hierarchy pass starts from hpm_set_hypotheses");
    if (p->hierarchy) CK(ensure((void **)&c->d_pre, &c->pre_cap, sizeof(float) * npx(c)), "pre-cost alloc");
    PMArgs a = make_args(c);
    a.dmin = p->depth_min;
    a.dmax = p->depth_max;
    a.geom = p->geom_consistency ? 1 : 0;
    a.prior = p->planar_prior ? 1 : 0;
    a.sigma_spatial = p->sigma_spatial;
    a.sigma_color = p->sigma_color;
    a.top_k = p->top_k;
    a.seed_lo = (uint32_t)p->seed;
    a.seed_hi = (uint32_t)(p->seed >> 32);
    a.salt = c->pass_counter++;
    a.fix_quirks = p->fix_quirks ? 1 : 0;
    if (p->fix_quirks) a.rows_cov = a.H; /* every row, also the last of an odd height (HPM.cu:1926) */
    if (p->variant == 1) {
        a.acmm = 1;        /* weight 0.2: ACMM.cu:651, 1596 */
        a.geom_max = 3.0f; /* ACMM.cu:496 */
        a.hier = p->hierarchy;
        a.pre_costs = p->hierarchy ? c->d_pre : nullptr;
    }
    *out = a;
    return HPM_OK;
}

/* The kernel arguments of one pass of context c with parameters p (checks
 * as hpm_run_patchmatch; takes the pass's random-stream salt), for a
 * batched launch. */
extern "C++" int ctx_pass_args(hpm_ctx *c, const HpmParams *p, PMArgs *out)
{
    if (!c) return HPM_ERR_ARG;
    const int r = pass_args(c, p, out);
    if (r) return r;
    c->has_state = true;
    return HPM_OK;
}

extern "C++" void ctx_reset_salt(hpm_ctx *c) { c->pass_counter = 0; }

/* One pass: initialisation, `half_steps` red/black half-steps (the
 * reference runs 2 per iteration), then optionally depth/normal conversion
 * and the two filter kernels.  Nothing waits on the host in between. */
static int run_pass(hpm_ctx *c, const HpmParams *p, int half_steps, int finalize, bool sync)
{
    if (!c) return HPM_ERR_ARG;
    int r = select_device(c);
    if (r) return r;
    PMArgs a;
    r = pass_args(c, p, &a);
    if (r) return r;
    const Range range("pass geom=%d prior=%d", p->geom_consistency ? 1 : 0, p->planar_prior ? 1 : 0);
    cudaEvent_t e0;
    prof_begin(c, 0, &e0);
    CK(launch_init(a, c->stream), "init kernel");
    prof_end(c, 0, e0);
    for (int hs = 0; hs < half_steps; ++hs) {
        prof_begin(c, 1, &e0);
        CK(launch_propagate(a, hs / 2, hs % 2, c->stream), "propagate kernels");
        prof_end(c, 1, e0);
    }
    if (finalize) {
        prof_begin(c, 2, &e0);
        CK(launch_depth_normal_filter(a, c->d_planes, c->d_costs, c->stream), "depth/normal + filter kernels");
        prof_end(c, 2, e0);
    }
    c->has_state = true;
    if (sync) CK(cudaStreamSynchronize(c->stream), "hpm_run_patchmatch");
    return HPM_OK;
}

int hpm_run_patchmatch(hpm_ctx *c, const HpmParams *p)
{
    if (!c || !p) return HPM_ERR_ARG;
    /* HPM.cu:1933 runs 3; the ACMM+NESP variant honours the field (ACMM.cu:1836) */
    const int iters = (p->honour_max_iterations || p->variant == 1) ? p->max_iterations : 3;
    if (iters < 0 || iters > 64) return fail(c, HPM_ERR_ARG, "max_iterations outside [0, 64]");
    return run_pass(c, p, 2 * iters, 1, true);
}

int hpm_run_partial(hpm_ctx *c, const HpmParams *p, int half_steps, int finalize)
{
    if (!c || !p) return HPM_ERR_ARG;
    if (half_steps < 0 || half_steps > 128) return fail(c, HPM_ERR_ARG, "half_steps outside [0, 128]");
    return run_pass(c, p, half_steps, finalize, true);
}

int hpm_get_result(hpm_ctx *c, float *planes, float *costs)
{
    if (!c) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_get_result before hpm_set_views");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c);
    if (planes)
        CK(cudaMemcpyAsync(planes, c->d_planes, sizeof(float4) * n, cudaMemcpyDeviceToHost, c->stream), "planes");
    if (costs) CK(cudaMemcpyAsync(costs, c->d_costs, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream), "costs");
    CK(cudaStreamSynchronize(c->stream), "hpm_get_result");
    return HPM_OK;
}

int hpm_get_selected_views(hpm_ctx *c, uint32_t *views)
{
    if (!c || !views) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_get_selected_views before hpm_set_views");
    int r = select_device(c);
    if (r) return r;
    CK(cudaMemcpyAsync(views, c->d_views, sizeof(uint32_t) * npx(c), cudaMemcpyDeviceToHost, c->stream), "views");
    CK(cudaStreamSynchronize(c->stream), "hpm_get_selected_views");
    return HPM_OK;
}

int hpm_device_state(hpm_ctx *c, float **planes, float **costs, uint32_t **views)
{
    if (!c) return HPM_ERR_ARG;
    if (planes) *planes = (float *)c->d_planes;
    if (costs) *costs = c->d_costs;
    if (views) *views = c->d_views;
    return HPM_OK;
}

static int scratch(hpm_ctx *c, size_t bytes, void **p)
{
    CK(ensure(&c->d_scratch, &c->scratch_cap, bytes), "scratch alloc");
    *p = c->d_scratch;
    return HPM_OK;
}

int hpm_cost_vectors(hpm_ctx *c, const float *planes, float *out)
{
    if (!c || !planes || !out) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_cost_vectors before hpm_set_views");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c), S = c->n - 1;
    void *buf;
    r = scratch(c, n * (sizeof(float4) + S * sizeof(float)), &buf);
    if (r) return r;
    float4 *d_pl = (float4 *)buf;
    float *d_out = (float *)(d_pl + n);
    CK(cudaMemcpyAsync(d_pl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream), "planes");
    PMArgs a = make_args(c);
    CK(launch_cost_vectors(a, d_pl, d_out, c->stream), "cost vector kernel");
    CK(cudaMemcpyAsync(out, d_out, sizeof(float) * n * S, cudaMemcpyDeviceToHost, c->stream), "out");
    CK(cudaStreamSynchronize(c->stream), "hpm_cost_vectors");
    return HPM_OK;
}

int hpm_tap_samples(hpm_ctx *c, const float *planes, const int *pixels, int n, float *out, int *inside)
{
    if (!c || !planes || (!pixels && n > 0) || n < 0 || !out || !inside) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_tap_samples before hpm_set_views");
    const size_t np = npx(c), S = c->n - 1;
    for (int k = 0; k < n; ++k)
        if (pixels[k] < 0 || (size_t)pixels[k] >= np) return fail(c, HPM_ERR_ARG, "pixel index %d outside the view", pixels[k]);
    int r = select_device(c);
    if (r) return r;
    void *buf;
    r = scratch(c, np * sizeof(float4) + (size_t)n * (sizeof(int) + S * (kTaps * sizeof(float) + sizeof(int))), &buf);
    if (r) return r;
    float4 *d_pl = (float4 *)buf;
    float *d_out = (float *)(d_pl + np);
    int *d_in = (int *)(d_out + (size_t)n * S * kTaps);
    int *d_px = d_in + (size_t)n * S;
    CK(cudaMemcpyAsync(d_pl, planes, sizeof(float4) * np, cudaMemcpyHostToDevice, c->stream), "planes");
    if (n > 0) CK(cudaMemcpyAsync(d_px, pixels, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream), "pixels");
    PMArgs a = make_args(c);
    CK(launch_tap_samples(a, d_pl, d_px, n, d_out, d_in, c->stream), "tap sample kernel");
    CK(cudaMemcpyAsync(out, d_out, sizeof(float) * n * S * kTaps, cudaMemcpyDeviceToHost, c->stream), "samples");
    CK(cudaMemcpyAsync(inside, d_in, sizeof(int) * n * S, cudaMemcpyDeviceToHost, c->stream), "inside");
    CK(cudaStreamSynchronize(c->stream), "hpm_tap_samples");
    return HPM_OK;
}

int hpm_initial_costs(hpm_ctx *c, const float *planes, float *out_cost, uint32_t *out_views)
{
    if (!c || !planes || !out_cost || !out_views) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_initial_costs before hpm_set_views");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c);
    void *buf;
    r = scratch(c, n * (sizeof(float4) + sizeof(float) + sizeof(uint32_t)), &buf);
    if (r) return r;
    float4 *d_pl = (float4 *)buf;
    float *d_c = (float *)(d_pl + n);
    uint32_t *d_v = (uint32_t *)(d_c + n);
    CK(cudaMemcpyAsync(d_pl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream), "planes");
    PMArgs a = make_args(c);
    CK(launch_initial_costs(a, d_pl, d_c, d_v, c->stream), "initial cost kernel");
    CK(cudaMemcpyAsync(out_cost, d_c, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream), "cost");
    CK(cudaMemcpyAsync(out_views, d_v, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c->stream), "views");
    CK(cudaStreamSynchronize(c->stream), "hpm_initial_costs");
    return HPM_OK;
}

int hpm_geom_costs(hpm_ctx *c, const float *planes, float *out)
{
    if (!c || !planes || !out) return HPM_ERR_ARG;
    if (c->n < 2 || !c->has_depth) return fail(c, HPM_ERR_STATE, "hpm_geom_costs needs views and depth maps");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c), S = c->n - 1;
    void *buf;
    r = scratch(c, n * (sizeof(float4) + S * sizeof(float)), &buf);
    if (r) return r;
    float4 *d_pl = (float4 *)buf;
    float *d_out = (float *)(d_pl + n);
    CK(cudaMemcpyAsync(d_pl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream), "planes");
    PMArgs a = make_args(c);
    CK(launch_geom_costs(a, d_pl, d_out, c->stream), "geom cost kernel");
    CK(cudaMemcpyAsync(out, d_out, sizeof(float) * n * S, cudaMemcpyDeviceToHost, c->stream), "out");
    CK(cudaStreamSynchronize(c->stream), "hpm_geom_costs");
    return HPM_OK;
}

int hpm_depth_normal_filter(hpm_ctx *c, float *planes, const float *costs)
{
    if (!c || !planes || !costs) return HPM_ERR_ARG;
    if (c->n < 2) return fail(c, HPM_ERR_STATE, "hpm_depth_normal_filter before hpm_set_views");
    int r = select_device(c);
    if (r) return r;
    const size_t n = npx(c);
    void *buf;
    r = scratch(c, n * (sizeof(float4) + sizeof(float)), &buf);
    if (r) return r;
    float4 *d_pl = (float4 *)buf;
    float *d_c = (float *)(d_pl + n);
    CK(cudaMemcpyAsync(d_pl, planes, sizeof(float4) * n, cudaMemcpyHostToDevice, c->stream), "planes");
    CK(cudaMemcpyAsync(d_c, costs, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream), "costs");
    PMArgs a = make_args(c);
    CK(launch_depth_normal_filter(a, d_pl, d_c, c->stream), "depth/normal + filter kernels");
    CK(cudaMemcpyAsync(planes, d_pl, sizeof(float4) * n, cudaMemcpyDeviceToHost, c->stream), "planes");
    CK(cudaStreamSynchronize(c->stream), "hpm_depth_normal_filter");
    return HPM_OK;
}

int hpm_jbu(hpm_ctx *c, const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal,
            int s_cols, int s_rows, float *out_depth, float *out_normal)
{
    if (!c) return HPM_ERR_ARG;
    if (!guide || !coarse_depth || !coarse_normal || !out_depth || !out_normal)
        return fail(c, HPM_ERR_ARG, "hpm_jbu: null input");
    if (cols < 1 || rows < 1 || s_cols < 1 || s_rows < 1 || s_cols > cols || s_rows > rows)
        return fail(c, HPM_ERR_ARG, "hpm_jbu: bad sizes %dx%d <- %dx%d", cols, rows, s_cols, s_rows);
    const int sr = rows / s_rows, sc = cols / s_cols;
    const int image_scale = sr > sc ? sr : sc;
    if (image_scale == 1) return HPM_OK; /* HPM.cpp:1219-1222 */
    int r = select_device(c);
    if (r) return r;
    const size_t fine = (size_t)cols * rows, coarse = (size_t)s_cols * s_rows;
    void *buf;
    r = scratch(c, fine * sizeof(float) + coarse * sizeof(float4) + fine * (sizeof(float) + sizeof(float4)), &buf);
    if (r) return r;
    float4 *d_coarse = (float4 *)buf;
    float4 *d_on = d_coarse + coarse;
    float *d_guide = (float *)(d_on + fine);
    float *d_od = d_guide + fine;
    std::vector<float4> packed(coarse);
    for (size_t i = 0; i < coarse; ++i)
        packed[i] = make_float4(coarse_normal[3 * i], coarse_normal[3 * i + 1], coarse_normal[3 * i + 2],
                                coarse_depth[i]);
    CK(cudaMemcpyAsync(d_coarse, packed.data(), sizeof(float4) * coarse, cudaMemcpyHostToDevice, c->stream),
       "coarse");
    CK(cudaMemcpyAsync(d_guide, guide, sizeof(float) * fine, cudaMemcpyHostToDevice, c->stream), "guide");
    cudaEvent_t e0;
    prof_begin(c, 3, &e0);
    CK(launch_jbu(d_guide, cols, rows, nullptr, d_coarse, s_cols, s_rows, image_scale, d_od, d_on, c->stream),
       "jbu kernel");
    prof_end(c, 3, e0);
    std::vector<float4> on(fine);
    CK(cudaMemcpyAsync(out_depth, d_od, sizeof(float) * fine, cudaMemcpyDeviceToHost, c->stream), "depth");
    CK(cudaMemcpyAsync(on.data(), d_on, sizeof(float4) * fine, cudaMemcpyDeviceToHost, c->stream), "normal");
    CK(cudaStreamSynchronize(c->stream), "hpm_jbu");
    for (size_t i = 0; i < fine; ++i) {
        out_normal[3 * i] = on[i].x;
        out_normal[3 * i + 1] = on[i].y;
        out_normal[3 * i + 2] = on[i].z;
    }
    return HPM_OK;
}

/* The contexts a context runs work on besides itself: the second
 * scene-worker context, the prior-net form's coarse context, the batched
 * form's problem contexts.  Counters and profiles cover them all. */
static std::vector<hpm_ctx *> child_contexts(hpm_ctx *c)
{
    std::vector<hpm_ctx *> out;
    if (c->peer) out.push_back(c->peer);
    if (c->coarse) out.push_back(c->coarse);
    for (hpm_ctx *b : c->batch) out.push_back(b);
    return out;
}

int hpm_profile_enable(hpm_ctx *c, int enable)
{
    if (!c) return HPM_ERR_ARG;
    c->profiling = enable != 0;
    for (int i = 0; i < 4; ++i) {
        c->prof_ms[i] = 0;
        c->prof_cnt[i] = 0;
    }
    for (auto &p : c->prof_events) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    c->prof_events.clear();
    for (hpm_ctx *k : child_contexts(c)) hpm_profile_enable(k, enable);
    return HPM_OK;
}

int hpm_profile_read(hpm_ctx *c, float *ms4, int *counts4)
{
    if (!c) return HPM_ERR_ARG;
    float peer_ms[4] = {0, 0, 0, 0};
    int peer_cnt[4] = {0, 0, 0, 0};
    for (hpm_ctx *k : child_contexts(c)) {
        float ms[4];
        int cnt[4];
        const int r = hpm_profile_read(k, ms, cnt);
        if (r) return fail(c, r, "hpm_profile_read (inner context): %s", hpm_last_error(k));
        for (int i = 0; i < 4; ++i) {
            peer_ms[i] += ms[i];
            peer_cnt[i] += cnt[i];
        }
    }
    CK(cudaStreamSynchronize(c->stream), "hpm_profile_read");
    for (auto &p : c->prof_events) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.second.first, p.second.second);
        c->prof_ms[p.first] += ms;
        c->prof_cnt[p.first] += 1;
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    c->prof_events.clear();
    for (int i = 0; i < 4; ++i) {
        if (ms4) ms4[i] = c->prof_ms[i] + peer_ms[i];
        if (counts4) counts4[i] = c->prof_cnt[i] + peer_cnt[i];
    }
    return HPM_OK;
}

int hpm_set_scene_workers(hpm_ctx *c, int workers)
{
    if (!c) return HPM_ERR_ARG;
    if (workers < 1 || workers > 2) return fail(c, HPM_ERR_ARG, "hpm_set_scene_workers: %d is not 1 or 2", workers);
    c->scene_workers = workers;
    return HPM_OK;
}

int hpm_count_enable(hpm_ctx *c, int enable)
{
    if (!c) return HPM_ERR_ARG;
    /* the counters run from here over every later pass until disabled */
    if (enable) {
        int r = select_device(c);
        if (r) return r;
        CK(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned long long), c->stream), "counters");
        CK(cudaStreamSynchronize(c->stream), "hpm_count_enable");
    }
    c->counting = enable != 0;
    for (hpm_ctx *k : child_contexts(c)) {
        const int r = hpm_count_enable(k, enable);
        if (r) return fail(c, r, "hpm_count_enable (inner context): %s", hpm_last_error(k));
    }
    return HPM_OK;
}

int hpm_count_read(hpm_ctx *c, uint64_t *cv, uint64_t *geom)
{
    if (!c) return HPM_ERR_ARG;
    uint64_t peer_cv = 0, peer_geom = 0;
    for (hpm_ctx *k : child_contexts(c)) {
        uint64_t cv = 0, geom = 0;
        const int r = hpm_count_read(k, &cv, &geom);
        if (r) return fail(c, r, "hpm_count_read (inner context): %s", hpm_last_error(k));
        peer_cv += cv;
        peer_geom += geom;
    }
    unsigned long long h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, c->d_counters, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "counters");
    CK(cudaStreamSynchronize(c->stream), "hpm_count_read");
    if (cv) *cv = h[0] + peer_cv;
    if (geom) *geom = h[1] + peer_geom;
    return HPM_OK;
}

}  // extern "C"

/* ---- helpers shared with the pass orchestration (hpm_flow.cu) ---- */

int ctx_fail(hpm_ctx *c, int code, const char *fmt, ...)
{
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof(c->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int ctx_cuda_fail(hpm_ctx *c, cudaError_t e, const char *what) { return cuda_fail(c, e, what); }
int ctx_create_child(hpm_ctx *c, hpm_ctx **child)
{
    int r = hpm_create(child, c->device);
    if (r) return r;
    (*child)->scene_workers = 1;
    if (c->profiling) hpm_profile_enable(*child, 1);
    if (c->counting) r = hpm_count_enable(*child, 1);
    return r;
}
int ctx_select_device(hpm_ctx *c) { return select_device(c); }
int ctx_run_pass(hpm_ctx *c, const HpmParams *p, int half_steps, int finalize)
{
    return run_pass(c, p, half_steps, finalize, true);
}
float *ctx_planes(hpm_ctx *c) { return reinterpret_cast<float *>(c->d_planes); }
float *ctx_costs(hpm_ctx *c) { return c->d_costs; }
float *ctx_prior(hpm_ctx *c) { return reinterpret_cast<float *>(c->d_prior); }
uint32_t *ctx_masks(hpm_ctx *c) { return c->d_masks; }
const float *ctx_image(hpm_ctx *c, int i) { return c->d_img[i]; }
void ctx_mark_prior(hpm_ctx *c) { c->has_prior = true; }
void ctx_mark_state(hpm_ctx *c) { c->has_state = true; }

template <typename T>
static cudaError_t grow(T **p, size_t *cap, size_t n)
{
    if (*p && *cap >= n) return cudaSuccess;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (n ? n : 1));
    if (e == cudaSuccess) *cap = n;
    return e;
}

cudaError_t ws_reserve(hpm_ctx *c, size_t npx, size_t nblocks)
{
    FlowWorkspace &w = c->flow;
    if (w.lvl_cap < npx) {
        size_t a = 0, b = 0, d = 0;
        cudaError_t e = grow(&w.mask, &a, npx);
        if (e == cudaSuccess) e = grow(&w.ids, &b, npx);
        if (e == cudaSuccess) e = grow(&w.knn_planes, &d, npx);
        if (e != cudaSuccess) return e;
        w.lvl_cap = npx;
    }
    return grow(&w.blocks, &w.blocks_cap, nblocks);
}

cudaError_t ws_reserve_tris(hpm_ctx *c, size_t ntris)
{
    FlowWorkspace &w = c->flow;
    if (w.tri_cap >= ntris && w.tris) return cudaSuccess;
    size_t a = 0;
    cudaError_t e = grow(&w.tris, &a, 6 * ntris);
    if (e == cudaSuccess) e = grow(&w.tri_planes, &w.tri_cap, ntris);
    return e;
}

cudaError_t ws_reserve_grid(hpm_ctx *c, size_t npts, size_t ncells)
{
    FlowWorkspace &w = c->flow;
    if (w.pts_cap < npts || !w.pts) {
        size_t a = 0;
        cudaError_t e = grow(&w.pts, &a, npts);
        if (e == cudaSuccess) e = grow(&w.cell_pts, &w.pts_cap, npts);
        if (e != cudaSuccess) return e;
    }
    return grow(&w.cell_start, &w.cells_cap, ncells);
}

cudaError_t ws_reserve_full(hpm_ctx *c, size_t npx)
{
    FlowWorkspace &w = c->flow;
    if (w.full_cap >= npx && w.full_depth) return cudaSuccess;
    size_t a = 0, b = 0, d = 0, f = 0;
    cudaError_t e = grow(&w.full_depth, &a, npx);
    if (e == cudaSuccess) e = grow(&w.full_normal, &b, 3 * npx);
    if (e == cudaSuccess) e = grow(&w.prior_depth, &d, npx);
    if (e == cudaSuccess) e = grow(&w.up_depth, &f, npx);
    if (e == cudaSuccess) e = grow(&w.up_normal, &w.full_cap, npx);
    return e;
}

cudaError_t ws_reserve_coarse(hpm_ctx *c, size_t npx)
{
    FlowWorkspace &w = c->flow;
    if (w.coarse_cap >= npx && w.c_depth) return cudaSuccess;
    size_t a = 0, b = 0, d = 0, f = 0, g = 0;
    cudaError_t e = grow(&w.c_depth, &a, npx);
    if (e == cudaSuccess) e = grow(&w.c_cost, &b, npx);
    if (e == cudaSuccess) e = grow(&w.c_normal, &d, 3 * npx);
    if (e == cudaSuccess) e = grow(&w.c_prior_depth, &f, npx);
    if (e == cudaSuccess) e = grow(&w.c_prior_normal, &g, 3 * npx);
    if (e == cudaSuccess) e = grow(&w.c_packed, &w.coarse_cap, npx);
    return e;
}

void ws_free(hpm_ctx *c)
{
    FlowWorkspace &w = c->flow;
    void *ptrs[] = {w.full_depth, w.full_normal, w.prior_depth, w.up_depth, w.up_normal, w.mask, w.ids,
                    w.knn_planes, w.blocks, w.c_depth, w.c_cost, w.c_normal, w.c_prior_depth, w.c_prior_normal,
                    w.c_packed, w.tris, w.tri_planes, w.pts, w.cell_start, w.cell_pts};
    for (void *p : ptrs) cudaFree(p);
    w = FlowWorkspace();
}

cudaError_t net_reserve(hpm_ctx *c, size_t coarse_px, size_t coarse_img_floats)
{
    NetWorkspace &w = c->net;
    cudaError_t e = cudaSuccess;
    if (!w.err) {
        e = cudaMalloc((void **)&w.err, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(w.err, 0, sizeof(int));
        if (e != cudaSuccess) return e;
    }
    if (w.cimg_cap < coarse_img_floats || !w.cimg) e = grow(&w.cimg, &w.cimg_cap, coarse_img_floats);
    if (e != cudaSuccess || (w.cap >= coarse_px && w.x0)) return e;
    size_t a = 0, b = 0, d = 0, f = 0, g = 0;
    __nv_bfloat16 *x0 = static_cast<__nv_bfloat16 *>(w.x0), *a0 = static_cast<__nv_bfloat16 *>(w.a[0]),
                  *a1 = static_cast<__nv_bfloat16 *>(w.a[1]), *a2 = static_cast<__nv_bfloat16 *>(w.a[2]);
    e = grow(&x0, &a, 16 * coarse_px);
    if (e == cudaSuccess) e = grow(&a0, &b, 32 * coarse_px);
    if (e == cudaSuccess) e = grow(&a1, &d, 32 * coarse_px);
    if (e == cudaSuccess) e = grow(&a2, &f, 32 * coarse_px);
    if (e == cudaSuccess) e = grow(&w.out, &g, 16 * coarse_px);
    w.x0 = x0;
    w.a[0] = a0;
    w.a[1] = a1;
    w.a[2] = a2;
    if (e == cudaSuccess) e = grow(&w.prop, &w.cap, coarse_px);
    return e;
}

cudaError_t net_reserve_full(hpm_ctx *c, size_t npx)
{
    NetWorkspace &w = c->net;
    if (w.full_cap >= npx && w.up_depth) return cudaSuccess;
    size_t a = 0, b = 0;
    cudaError_t e = grow(&w.up_depth, &a, npx);
    if (e == cudaSuccess) e = grow(&w.up_normal, &b, npx);
    if (e == cudaSuccess) e = grow(&w.cand, &w.full_cap, npx);
    return e;
}

void net_free(hpm_ctx *c)
{
    NetWorkspace &w = c->net;
    void *ptrs[] = {w.x0, w.a[0], w.a[1], w.a[2], w.out, w.prop, w.cimg, w.up_depth, w.up_normal, w.cand, w.err};
    for (void *p : ptrs) cudaFree(p);
    w = NetWorkspace();
}

cudaError_t ctx_scene_arena(hpm_ctx *c, size_t bytes) { return ensure((void **)&c->d_scene, &c->scene_cap, bytes); }
float *ctx_scene_base(hpm_ctx *c) { return c->d_scene; }

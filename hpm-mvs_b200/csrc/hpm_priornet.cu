/*
 * The prior-net form around the tensor-core convolutions of hpm_net.cu: the
 * coarse stage that feeds the network, the network's forward pass and head,
 * the proposal planes handed to PatchMatch, and the training kernels (loss,
 * Adam, the multi-view consistency filter that selects training targets).
 * No counterpart in the reference.
 *
 * Network (4 layers of 3x3 convolutions, BF16 operands, FP32 accumulation):
 *   input  16 channels at the coarse scale (1/4): gray image, the coarse
 *          plain pass's depth, its reference-frame normal and confidence,
 *          the coarse planar prior's depth and presence; 8 channels unused
 *   L1 16->32 ReLU, L2 32->32 ReLU, L3 32->32 ReLU, L4 32->16 linear
 *   head   depth = dmin + sigmoid(o0) (dmax - dmin), reference-frame normal
 *          = normalise(o1, o2, o3)
 */
#include <cuda_bf16.h>

#include <cmath>

#include "hpm_capi_internal.h"
#include "hpm_net.h"
#include "hpm_nvtx.h"
#include "hpm_prior.h"

namespace hpm {
namespace {

__device__ __forceinline__ float3 to_ref(const HpmCamera &c, float x, float y, float z) /* R n */
{
    return make_float3(c.R[0] * x + c.R[1] * y + c.R[2] * z, c.R[3] * x + c.R[4] * y + c.R[5] * z,
                       c.R[6] * x + c.R[7] * y + c.R[8] * z);
}

__device__ __forceinline__ float3 to_world(const HpmCamera &c, float x, float y, float z) /* R^T n */
{
    return make_float3(c.R[0] * x + c.R[3] * y + c.R[6] * z, c.R[1] * x + c.R[4] * y + c.R[7] * z,
                       c.R[2] * x + c.R[5] * y + c.R[8] * z);
}

__device__ __forceinline__ float norm_depth(float d, float dmin, float dmax)
{
    return fminf(fmaxf((d - dmin) / (dmax - dmin), -0.5f), 1.5f) - 0.5f;
}

/* The network's input at the coarse scale (NHWC BF16, 16 channels). */
__global__ void k_net_input(HpmCamera cam, const float *__restrict__ img, const float4 *__restrict__ pass_planes,
                            const float *__restrict__ pass_cost, const float *__restrict__ prior_depth, int n,
                            float dmin, float dmax, __nv_bfloat16 *__restrict__ x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 pl = pass_planes[i]; /* world normal, depth (after the pass's finalisation) */
    const float3 nr = to_ref(cam, pl.x, pl.y, pl.z);
    const float c = pass_cost[i];
    const float conf = c < 2.0f ? __expf(-c * c / 0.18f) : 0.0f;
    const float pd = prior_depth[i];
    float v[16];
    v[0] = img[i] * (1.0f / 255.0f) - 0.5f;
    v[1] = (pl.w > 0.0f) ? norm_depth(pl.w, dmin, dmax) : 0.0f;
    v[2] = conf;
    v[3] = nr.x;
    v[4] = nr.y;
    v[5] = nr.z;
    v[6] = pd > 0.0f ? norm_depth(pd, dmin, dmax) : 0.0f;
    v[7] = pd > 0.0f ? 1.0f : 0.0f;
#pragma unroll
    for (int k = 8; k < 16; ++k) v[k] = 0.0f;
    __align__(16) __nv_bfloat162 o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    reinterpret_cast<uint4 *>(x + (size_t)i * 16)[0] = reinterpret_cast<const uint4 *>(o)[0];
    reinterpret_cast<uint4 *>(x + (size_t)i * 16)[1] = reinterpret_cast<const uint4 *>(o)[1];
}

__device__ __forceinline__ float3 head_normal(const float *o)
{
    const float l2 = o[1] * o[1] + o[2] * o[2] + o[3] * o[3];
    if (!(l2 > 1e-12f)) return make_float3(0.0f, 0.0f, -1.0f);
    const float inv = rsqrtf(l2);
    return make_float3(o[1] * inv, o[2] * inv, o[3] * inv);
}

/* Head: (world normal, depth) per coarse pixel, the layout JBU upsamples. */
__global__ void k_net_head(HpmCamera cam, const float *__restrict__ out16, int n, float dmin, float dmax,
                           float4 *__restrict__ packed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *o = out16 + (size_t)i * 16;
    const float d = dmin + (dmax - dmin) / (1.0f + __expf(-o[0]));
    const float3 nr = head_normal(o);
    const float3 nw = to_world(cam, nr.x, nr.y, nr.z);
    packed[i] = make_float4(nw.x, nw.y, nw.z, d);
}

/* Upsampled proposal (depth, world normal) to the full-scale pass: the
 * initial hypothesis (reference-frame normal, depth: the prior pass's
 * initialisation turns the depth into a distance) and the candidate plane
 * (reference-frame normal, distance, ComputeDepthfromPlaneHypothesis's
 * inverse). */
__global__ void k_proposal_planes(HpmCamera cam, const float *__restrict__ up_depth,
                                  const float4 *__restrict__ up_normal, int w, int h, float4 *__restrict__ init,
                                  float *__restrict__ init_cost, float4 *__restrict__ cand)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = (size_t)y * w + x;
    const float d = up_depth[i];
    const float4 nw = up_normal[i];
    float3 nr = to_ref(cam, nw.x, nw.y, nw.z);
    const float l2 = nr.x * nr.x + nr.y * nr.y + nr.z * nr.z;
    if (!(l2 > 1e-12f) || !(d > 0.0f)) nr = make_float3(0.0f, 0.0f, -1.0f);
    const float X0 = d * (x - cam.K[2]) / cam.K[0], X1 = d * (y - cam.K[5]) / cam.K[4];
    init[i] = make_float4(nr.x, nr.y, nr.z, d);
    init_cost[i] = 0.0f;
    cand[i] = make_float4(nr.x, nr.y, nr.z, -(nr.x * X0 + nr.y * X1 + nr.z * d));
}

/* Masked training loss of the head and its gradient: relative depth error
 * |d - t| / t plus lambda (1 - n . t_n); dy (BF16, 16 channels) = dloss/dout
 * / count, zero in the unused channels; loss[0] += the loss sum. */
__global__ void k_net_loss(const float *__restrict__ out16, const float *__restrict__ t_depth,
                           const float *__restrict__ t_normal, const uint8_t *__restrict__ mask, int n, float dmin,
                           float dmax, float lambda, float inv_count, __nv_bfloat16 *__restrict__ dy,
                           float *__restrict__ loss)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float g[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) g[k] = 0.0f;
    float l = 0.0f;
    if (i < n && mask[i]) {
        const float *o = out16 + (size_t)i * 16;
        const float s = 1.0f / (1.0f + __expf(-o[0]));
        const float d = dmin + (dmax - dmin) * s, t = t_depth[i];
        const float e = (d - t) / t;
        l = fabsf(e);
        g[0] = (e > 0.0f ? 1.0f : (e < 0.0f ? -1.0f : 0.0f)) / t * (dmax - dmin) * s * (1.0f - s);
        const float l2 = o[1] * o[1] + o[2] * o[2] + o[3] * o[3];
        if (l2 > 1e-12f) {
            const float inv = rsqrtf(l2);
            const float n0 = o[1] * inv, n1 = o[2] * inv, n2 = o[3] * inv;
            const float t0 = t_normal[3 * i], t1 = t_normal[3 * i + 1], t2 = t_normal[3 * i + 2];
            const float c = n0 * t0 + n1 * t1 + n2 * t2;
            l += lambda * (1.0f - c);
            /* d(1 - n.t)/do = -(t - c n) / |o| */
            g[1] = -lambda * (t0 - c * n0) * inv;
            g[2] = -lambda * (t1 - c * n1) * inv;
            g[3] = -lambda * (t2 - c * n2) * inv;
        }
    }
    if (i < n) {
        __align__(16) __nv_bfloat162 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __floats2bfloat162_rn(g[2 * k] * inv_count, g[2 * k + 1] * inv_count);
        reinterpret_cast<uint4 *>(dy + (size_t)i * 16)[0] = reinterpret_cast<const uint4 *>(v)[0];
        reinterpret_cast<uint4 *>(dy + (size_t)i * 16)[1] = reinterpret_cast<const uint4 *>(v)[1];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

/* Adam (Kingma and Ba, 2015) on a flat FP32 parameter vector; clears the
 * gradient after the step. */
__global__ void k_adam(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.0f;
}

/* The training filter: the multi-view test of RunFusion (main.cpp:575-612)
 * without its order-dependent masking.  A reference pixel passes when at
 * least one source agrees (reprojection < 2 px, relative depth < 1 %, normal
 * angle < 10 deg) and the summed exp(-(e + 200 rel + 10 angle)) exceeds 0.3
 * per agreeing source. */
struct ConsistArgs {
    HpmCamera ref;
    HpmCamera src[kMaxSrc];
    const float *src_depth[kMaxSrc];
    const float *src_normal[kMaxSrc];
    int ns;
};

__device__ __forceinline__ void world_pt(const HpmCamera &c, float x, float y, float d, float *X)
{
    const float a = d * (x - c.K[2]) / c.K[0], b = d * (y - c.K[5]) / c.K[4];
    for (int k = 0; k < 3; ++k)
        X[k] = c.R[k] * a + c.R[3 + k] * b + c.R[6 + k] * d -
               (c.R[k] * c.t[0] + c.R[3 + k] * c.t[1] + c.R[6 + k] * c.t[2]);
}

__device__ __forceinline__ void project_pt(const float *X, const HpmCamera &c, float *pt, float &depth)
{
    float t[3];
    for (int k = 0; k < 3; ++k) t[k] = c.R[3 * k] * X[0] + c.R[3 * k + 1] * X[1] + c.R[3 * k + 2] * X[2] + c.t[k];
    depth = c.K[6] * t[0] + c.K[7] * t[1] + c.K[8] * t[2];
    pt[0] = (c.K[0] * t[0] + c.K[1] * t[1] + c.K[2] * t[2]) / depth;
    pt[1] = (c.K[3] * t[0] + c.K[4] * t[1] + c.K[5] * t[2]) / depth;
}

__global__ void k_consistency(const __grid_constant__ ConsistArgs a, const float *__restrict__ depth,
                              const float *__restrict__ normal, uint8_t *__restrict__ mask)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int w = a.ref.width, h = a.ref.height;
    if (x >= w || y >= h) return;
    const size_t i = (size_t)y * w + x;
    const float d = depth[i];
    mask[i] = 0;
    if (!(d > 0.0f)) return;
    float X[3];
    world_pt(a.ref, (float)x, (float)y, d, X);
    const float *rn = normal + 3 * i;
    int num = 0;
    float dyn = 0.0f;
    for (int j = 0; j < a.ns; ++j) {
        const HpmCamera &s = a.src[j];
        float pt[2], pd;
        project_pt(X, s, pt, pd);
        const int sr = (int)(pt[1] + 0.5f), sc = (int)(pt[0] + 0.5f);
        if (!(sc >= 0 && sc < s.width && sr >= 0 && sr < s.height)) continue;
        const size_t sp = (size_t)sr * s.width + sc;
        const float sd = a.src_depth[j][sp];
        if (!(sd > 0.0f)) continue;
        float Y[3], tp[2], rd;
        world_pt(s, (float)sc, (float)sr, sd, Y);
        project_pt(Y, a.ref, tp, rd);
        const float e = sqrtf((x - tp[0]) * (x - tp[0]) + (y - tp[1]) * (y - tp[1]));
        const float rel = fabsf(rd - d) / d;
        const float *sn = a.src_normal[j] + 3 * sp;
        float ang = acosf(fminf(fmaxf(rn[0] * sn[0] + rn[1] * sn[1] + rn[2] * sn[2], -1.0f), 1.0f));
        if (e < 2.0f && rel < 0.01f && ang < 0.174533f) {
            num++;
            dyn += __expf(-(e + 200.0f * rel + 10.0f * ang));
        }
    }
    mask[i] = (num >= 1 && dyn > 0.3f * num) ? 1 : 0;
}

/* Training targets at the coarse scale: the full-scale pixel nearest to each
 * coarse pixel's position (the coarse grid's sample points, p / factor). */
__global__ void k_targets(HpmCamera cam, const float *__restrict__ depth, const float *__restrict__ normal,
                          const uint8_t *__restrict__ mask, int W, int H, int cw, int ch, float *__restrict__ t_depth,
                          float *__restrict__ t_normal, uint8_t *__restrict__ t_mask)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= cw || y >= ch) return;
    const int fx = min((int)lrintf((float)x * W / cw), W - 1), fy = min((int)lrintf((float)y * H / ch), H - 1);
    const size_t fi = (size_t)fy * W + fx, ci = (size_t)y * cw + x;
    const float3 nr = to_ref(cam, normal[3 * fi], normal[3 * fi + 1], normal[3 * fi + 2]);
    t_depth[ci] = depth[fi];
    t_normal[3 * ci] = nr.x;
    t_normal[3 * ci + 1] = nr.y;
    t_normal[3 * ci + 2] = nr.z;
    t_mask[ci] = mask[fi];
}

int grid1(size_t n) { return (int)((n + 255) / 256); }

}  // namespace
}  // namespace hpm

using namespace hpm;

#define CK(call, what)                                            \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return ctx_cuda_fail(c, e_, what); \
    } while (0)

namespace hpm {

/* The 1/4-scale views of one problem (the views of images/cams, full scale,
 * host or device) in the context's coarse sub-context (created once), so
 * that this context's full-scale views stay loaded. */
int net_coarse_views(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams)
{
    NetWorkspace &nw = c->net;
    FlowWorkspace &ws = c->flow;
    cudaStream_t s = c->stream;
    const int W = cams[0].width, H = cams[0].height;
    const int w = (int)std::lround(W * 0.25), h = (int)std::lround(H * 0.25);
    if (w < 8 || h < 8) return ctx_fail(c, HPM_ERR_ARG, "prior-net form: image too small");
    HpmCamera ccams[kMaxViews];
    const float *cimgs[kMaxViews];
    size_t need = 0;
    for (int j = 0; j < n; ++j) {
        const int vw = (int)std::lround(cams[j].width * 0.25), vh = (int)std::lround(cams[j].height * 0.25);
        need += ((size_t)vw * vh + 63) & ~(size_t)63;
    }
    CK(net_reserve(c, (size_t)w * h, need), "prior-net buffers");
    float *cur = nw.cimg;
    for (int j = 0; j < n; ++j) {
        HpmCamera cc = cams[j];
        const int vw = (int)std::lround(cams[j].width * 0.25), vh = (int)std::lround(cams[j].height * 0.25);
        const float sx = (float)vw / cams[j].width, sy = (float)vh / cams[j].height;
        cc.K[0] *= sx;
        cc.K[2] *= sx;
        cc.K[4] *= sy;
        cc.K[5] *= sy;
        cc.width = vw;
        cc.height = vh;
        ccams[j] = cc;
        /* full-scale image to the device first when it is host memory */
        const float *src = images[j];
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, src) != cudaSuccess || pa.type != cudaMemoryTypeDevice) {
            cudaGetLastError();
            CK(ws_reserve_full(c, (size_t)cams[j].width * cams[j].height), "staging");
            CK(cudaMemcpyAsync(ws.full_depth, src, sizeof(float) * cams[j].width * cams[j].height,
                               cudaMemcpyHostToDevice, s),
               "image upload");
            src = ws.full_depth;
        }
        CK(prior_resize(src, cams[j].width, cams[j].height, 1, cur, vw, vh, s), "coarse image");
        cimgs[j] = cur;
        cur += ((size_t)vw * vh + 63) & ~(size_t)63;
    }
    if (!c->coarse) {
        const int rc = ctx_create_child(c, &c->coarse);
        if (rc) return ctx_fail(c, rc, "prior-net form: coarse context");
    }
    CK(cudaStreamSynchronize(s), "coarse images");
    const int r = hpm_set_views(c->coarse, cimgs, ccams, n);
    if (r) return ctx_fail(c, r, "prior-net form: %s", hpm_last_error(c->coarse));
    return HPM_OK;
}

/* After the coarse sub-context's plain pass: its planar prior (left in
 * ws.c_prior_depth / c_prior_normal) and the network's input in
 * ws_net.x0. */
int net_coarse_finish(hpm_ctx *c, float dmin, float dmax)
{
    NetWorkspace &nw = c->net;
    FlowWorkspace &ws = c->flow;
    cudaStream_t s = c->stream;
    hpm_ctx *cc = c->coarse;
    const HpmCamera ccam = cc->cams[0];
    const int w = ccam.width, h = ccam.height;
    const size_t cn = (size_t)w * h;
    CK(ws_reserve_coarse(c, cn), "coarse buffers");
    const float4 *cplanes = reinterpret_cast<const float4 *>(ctx_planes(cc));
    const float *ccost = ctx_costs(cc);
    CK(flow_split_state(cplanes, (int)cn, ws.c_depth, ws.c_normal, s), "split");
    const int r = flow_level_prior(c, ccam, ccost, ws.c_depth, w, h, 1.0f, dmin, dmax);
    if (r) return r;
    CK(prior_coarse(ccam, w, h, 1.0f, dmin, dmax, ws.mask, ws.ids, ws.tri_planes, ws.knn_planes, ws.c_prior_depth,
                    ws.c_prior_normal, s),
       "coarse prior");
    k_net_input<<<grid1(cn), 256, 0, s>>>(ccam, ctx_image(cc, 0), cplanes, ccost, ws.c_prior_depth, (int)cn, dmin,
                                          dmax, static_cast<__nv_bfloat16 *>(nw.x0));
    CK(cudaGetLastError(), "net input");
    return HPM_OK;
}

/* Coarse stage of one problem: the 1/4-scale views, the plain pass on them,
 * its planar prior and the network's input; the coarse size in *cw x *ch. */
int net_coarse_stage(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams, uint64_t seed, int *cw,
                     int *ch)
{
    int r = net_coarse_views(c, n, images, cams);
    if (r) return r;
    hpm_ctx *cc = c->coarse;
    HpmParams p;
    hpm_default_params(&p);
    p.depth_min = cams[0].depth_min * 0.6f;
    p.depth_max = cams[0].depth_max * 1.2f;
    p.seed = seed;
    r = ctx_run_pass(cc, &p, 6, 1); /* ends with a synchronisation of its stream */
    if (r) return ctx_fail(c, r, "prior-net form: %s", hpm_last_error(cc));
    r = net_coarse_finish(c, p.depth_min, p.depth_max);
    if (r) return r;
    *cw = cc->cams[0].width;
    *ch = cc->cams[0].height;
    return HPM_OK;
}

/* Forward pass of the network on ws_net.x0 (h x w): the head's packed
 * proposal (world normal, depth) in ws_net.prop. */
int net_forward(hpm_ctx *c, const HpmNetWeights *net, const HpmCamera &ccam, int w, int h, float dmin, float dmax)
{
    NetWorkspace &nw = c->net;
    cudaStream_t s = c->stream;
    int *err = nw.err;
    CK(net_conv3x3(nw.x0, h, w, 16, net->packed[0], net->bias[0], 32, 0, nullptr, nw.a[0], err, true, s), "net L1");
    CK(net_conv3x3(nw.a[0], h, w, 32, net->packed[1], net->bias[1], 32, 0, nullptr, nw.a[1], err, true, s), "net L2");
    CK(net_conv3x3(nw.a[1], h, w, 32, net->packed[2], net->bias[2], 32, 0, nullptr, nw.a[2], err, true, s), "net L3");
    CK(net_conv3x3(nw.a[2], h, w, 32, net->packed[3], net->bias[3], 16, 1, nullptr, nw.out, err, true, s), "net L4");
    const size_t cn = (size_t)w * h;
    k_net_head<<<grid1(cn), 256, 0, s>>>(ccam, nw.out, (int)cn, dmin, dmax, nw.prop);
    CK(cudaGetLastError(), "net head");
    return HPM_OK;
}

/* The full-scale start of the prior-net form, after the coarse stage, with
 * the problem's full-scale views set in c: the network's proposal,
 * upsampled by JBU, as every pixel's initial hypothesis and as the
 * refinement candidate (c->proposals), and the planar prior: the coarse
 * triangulation's, upsampled as the plain form's coarsest level, or with
 * prior_mode 2 the upsampled proposal itself.  The next pass on c (seeded
 * as the caller wants) is the first full-scale pass. */
int net_full_setup(hpm_ctx *c, const HpmNetWeights *net, int prior_mode)
{
    const HpmCamera ccam = c->coarse->cams[0];
    const int cw = ccam.width, ch = ccam.height;
    const HpmCamera cam = c->cams[0];
    const float dmin = cam.depth_min * 0.6f, dmax = cam.depth_max * 1.2f;
    int r;
    {
        const Range network("network %dx%d", cw, ch);
        r = net_forward(c, net, ccam, cw, ch, dmin, dmax);
    }
    if (r) return r;
    NetWorkspace &nw = c->net;
    FlowWorkspace &ws = c->flow;
    cudaStream_t s = c->stream;
    const int W = cam.width, H = cam.height;
    const size_t npx = (size_t)W * H, cn = (size_t)cw * ch;
    CK(ws_reserve_full(c, npx), "flow workspace");
    CK(net_reserve_full(c, npx), "prior-net buffers");
    const int sr = H / ch, sc = W / cw, scale = sr > sc ? sr : sc;
    CK(launch_jbu(ctx_image(c, 0), W, H, nullptr, nw.prop, cw, ch, scale, nw.up_depth, nw.up_normal, s), "jbu");
    if (prior_mode == 2) {
        CK(prior_reload(cam, W, H, dmin, dmax, nw.up_depth, nw.up_normal, reinterpret_cast<float4 *>(ctx_prior(c)),
                        ctx_masks(c), s),
           "prior reload");
    } else {
        CK(flow_pack4(ws.c_prior_depth, ws.c_prior_normal, (int)cn, ws.c_packed, s), "pack");
        CK(launch_jbu(ctx_image(c, 0), W, H, nullptr, ws.c_packed, cw, ch, scale, ws.up_depth, ws.up_normal, s),
           "jbu");
        CK(prior_reload(cam, W, H, dmin, dmax, ws.up_depth, ws.up_normal, reinterpret_cast<float4 *>(ctx_prior(c)),
                        ctx_masks(c), s),
           "prior reload");
    }
    ctx_mark_prior(c);
    dim3 b(16, 16), g((W + 15) / 16, (H + 15) / 16);
    k_proposal_planes<<<g, b, 0, s>>>(cam, nw.up_depth, nw.up_normal, W, H, reinterpret_cast<float4 *>(ctx_planes(c)),
                                     ctx_costs(c), nw.cand);
    CK(cudaGetLastError(), "proposal planes");
    ctx_mark_state(c);
    c->proposals = nw.cand;
    return HPM_OK;
}

/* Seeds of the prior-net form's full-scale passes of a problem seeded s:
 * pass 0 is the first, pass e >= 1 the e-th extra pass. */
uint64_t net_pass_seed(uint64_t s, int pass) { return s + 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull * pass; }

/* Status of the tensor-core kernels of c's network (after a synchronisation). */
int net_status(hpm_ctx *c)
{
    int herr = 0;
    CK(cudaMemcpy(&herr, c->net.err, sizeof(int), cudaMemcpyDeviceToHost), "net status");
    if (herr) return ctx_fail(c, HPM_ERR_CUDA, "prior-net form: a tensor-core wait ran out (status %d)", herr);
    return HPM_OK;
}

/* The whole pass set A of one problem in the prior-net form: the coarse
 * stage, the full-scale start (net_full_setup), one full-scale PatchMatch
 * pass with the proposal as a sixth refinement candidate, then extra_passes
 * more full-scale prior passes, each with the planar prior rebuilt from the
 * previous pass (the plain form's finest level) and the proposal still a
 * candidate; half_steps red/black half-steps per full-scale pass.  Outputs
 * like hpm_process_problem. */
int net_problem(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams, const HpmNetWeights *net,
                uint64_t seed, int extra_passes, int prior_mode, int half_steps, float *depth_out, float *normal_out,
                float *cost_out)
{
    const Range range("prior-net problem %dx%d", cams[0].width, cams[0].height);
    int r = ctx_select_device(c); /* the scene's second worker thread starts on device 0 */
    if (r) return r;
    int cw, ch;
    r = net_coarse_stage(c, n, images, cams, seed, &cw, &ch);
    if (r) return r;
    r = hpm_set_views(c, images, cams, n);
    if (r) return r;
    r = net_full_setup(c, net, prior_mode);
    if (r) return r;
    FlowWorkspace &ws = c->flow;
    cudaStream_t s = c->stream;
    const size_t npx = (size_t)cams[0].width * cams[0].height;
    const float dmin = cams[0].depth_min * 0.6f, dmax = cams[0].depth_max * 1.2f;
    HpmParams p;
    hpm_default_params(&p);
    p.depth_min = dmin;
    p.depth_max = dmax;
    p.planar_prior = 1;
    for (int e = 0; e <= extra_passes && r == HPM_OK; ++e) {
        if (e > 0) {
            r = flow_prior_from_maps(c, 2, ctx_costs(c), dmin, dmax);
            if (r) break;
        }
        p.seed = net_pass_seed(seed, e);
        r = ctx_run_pass(c, &p, half_steps, 1);
        if (r) break;
        CK(flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(c)), (int)npx, ws.full_depth, ws.full_normal,
                            s),
           "split");
    }
    c->proposals = nullptr;
    if (r) return r;
    if (depth_out) CK(cudaMemcpyAsync(depth_out, ws.full_depth, sizeof(float) * npx, cudaMemcpyDefault, s), "out");
    if (normal_out)
        CK(cudaMemcpyAsync(normal_out, ws.full_normal, sizeof(float) * 3 * npx, cudaMemcpyDefault, s), "out");
    if (cost_out) CK(cudaMemcpyAsync(cost_out, ctx_costs(c), sizeof(float) * npx, cudaMemcpyDefault, s), "out");
    CK(cudaStreamSynchronize(s), "prior-net problem");
    return net_status(c);
}

}  // namespace hpm

extern "C" int hpm_net_coarse_inputs(hpm_ctx *c, int n, const float *const *images, const HpmCamera *cams,
                                     uint64_t seed, void *x0, size_t cap_px, int *cw, int *ch)
{
    if (!c || !images || !cams || !x0 || !cw || !ch || n < 2 || n > kMaxViews) return HPM_ERR_ARG;
    int r = ctx_select_device(c);
    if (r) return r;
    r = net_coarse_stage(c, n, images, cams, seed, cw, ch);
    if (r) return r;
    const size_t cn = (size_t)*cw * *ch;
    if (cn > cap_px) return ctx_fail(c, HPM_ERR_ARG, "hpm_net_coarse_inputs: %zu pixels, capacity %zu", cn, cap_px);
    CK(cudaMemcpyAsync(x0, c->net.x0, cn * 16 * sizeof(__nv_bfloat16), cudaMemcpyDefault, c->stream), "out");
    CK(cudaStreamSynchronize(c->stream), "hpm_net_coarse_inputs");
    return HPM_OK;
}

extern "C" int hpm_net_targets(int device, const HpmCamera *ref_cam, const float *depth, const float *normal, int ns,
                               const HpmCamera *src_cams, const float *const *src_depths,
                               const float *const *src_normals, int cw, int ch, float *t_depth, float *t_normal,
                               uint8_t *t_mask, void *stream)
{
    if (!ref_cam || !depth || !normal || ns < 1 || ns > kMaxSrc || !src_cams || !src_depths || !src_normals ||
        !t_depth || !t_normal || !t_mask || cw < 1 || ch < 1)
        return HPM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return HPM_ERR_CUDA;
    ConsistArgs a;
    memset(&a, 0, sizeof(a));
    a.ref = *ref_cam;
    a.ns = ns;
    for (int j = 0; j < ns; ++j) {
        a.src[j] = src_cams[j];
        a.src_depth[j] = src_depths[j];
        a.src_normal[j] = src_normals[j];
    }
    const int W = ref_cam->width, H = ref_cam->height;
    uint8_t *m = nullptr;
    if (cudaMalloc(&m, (size_t)W * H) != cudaSuccess) return HPM_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    dim3 b(16, 16);
    k_consistency<<<dim3((W + 15) / 16, (H + 15) / 16), b, 0, s>>>(a, depth, normal, m);
    k_targets<<<dim3((cw + 15) / 16, (ch + 15) / 16), b, 0, s>>>(*ref_cam, depth, normal, m, W, H, cw, ch, t_depth,
                                                               t_normal, t_mask);
    const cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(m);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
}

extern "C" int hpm_net_loss(const float *out16, const float *t_depth, const float *t_normal, const uint8_t *t_mask,
                            int n, float dmin, float dmax, float lambda, float inv_count, void *dy, float *loss,
                            void *stream)
{
    if (!out16 || !t_depth || !t_normal || !t_mask || !dy || !loss || n < 1) return HPM_ERR_ARG;
    k_net_loss<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        out16, t_depth, t_normal, t_mask, n, dmin, dmax, lambda, inv_count, static_cast<__nv_bfloat16 *>(dy), loss);
    return cudaGetLastError() == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
}

extern "C" int hpm_net_adam(float *params, float *grads, float *m, float *v, int n, float lr, float beta1,
                            float beta2, float eps, int step, void *stream)
{
    if (!params || !grads || !m || !v || n < 1 || step < 1) return HPM_ERR_ARG;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    k_adam<<<grid1(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, n, lr, beta1, beta2, eps, c1,
                                                                     c2);
    return cudaGetLastError() == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
}

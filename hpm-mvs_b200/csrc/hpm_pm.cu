/*
 * PatchMatch kernels of the B200-native HPM-MVS path (sm_100a).
 *
 * Behaviour follows the reference's HPM-MVS/HPM.cu kernel for kernel; the
 * per-function comments cite the lines.  What is different is how the work
 * maps to the machine:
 *
 *  - Reference-window hoisting.  The reference recomputes the 36 bilateral
 *    weights of a pixel's 11x11/stride-2 window (one exp, one sqrt, two
 *    divides each) and all reference-side sums inside every NCC call
 *    (HPM.cu:345-368), i.e. ~23 x S times per pixel per half-step.  Here they
 *    are computed once per pixel per launch, with the reference's own
 *    expressions (so the values are the same bits), and kept in shared memory
 *    as a [tap][thread] array: each NCC tap then costs one shared load of the
 *    weight and one of weight*ref instead of an exp, a sqrt and two texture
 *    fetches.
 *  - Source views are sampled by the texture unit (float cudaArray, linear
 *    filter, clamped edges: the reference's own texture set-up), so the
 *    bilinear samples are the reference's bit for bit.  The filter rounds
 *    coordinates to 1/256 (half up) and only the far corner's weight
 *    A*B/256; a textbook bilinear gather differs by up to ~0.5 gray levels
 *    per tap.
 *  - The per-pixel cost matrix (cost_array[8][32], 1.5 KB of local memory per
 *    thread in the reference) is handed from the site/direction kernel to the
 *    selection/refinement kernel through L2, so that shared memory holds only
 *    the 288-byte reference window per pixel.
 *  - Counter-based Philox random numbers: no 48-byte curand state per pixel
 *    in HBM and no curand_init skip-ahead; draws come in the reference's
 *    order.
 *  - Half-step kernels are launched back to back on one stream with no
 *    host synchronisation (the reference synchronises after every launch).
 */
#include <cfloat>
#include <cstdlib>

#include "hpm_internal.h"

namespace hpm {

namespace {

constexpr double kPiD = 3.14159265358979323846; /* M_PI, HPM-MVS/main.h:41 */
constexpr int kBlockX = 32;
constexpr int kBlockY = 2;
constexpr int kBlock = kBlockX * kBlockY;

/* Pixels of one half-step (one checkerboard colour) per warp: ww per row
 * over 32 / ww rows, so that the 32 lanes sample a compact 2D patch of each
 * source image (the texture cache is tiled in 2D).  A block is two such
 * warps stacked vertically.  ww is 8 unless the batched form's tile tuning
 * picks 4 or 16 for a view size. */
static_assert(kBlock == 64, "two warps per block");

/* (px, py) of this thread in a half-step of `color`, for the block's tile
 * (bx, by) */
__device__ __forceinline__ void half_step_pixel_at(int bx, int by, int ww, int color, int &px, int &py)
{
    const int lane = threadIdx.x, wv = threadIdx.y, wh = 32 / ww;
    py = by * (2 * wh) + wv * wh + lane / ww;
    px = bx * (2 * ww) + 2 * (lane % ww) + ((py + color) & 1);
}

#ifndef HPM_CV_INLINE
#define HPM_CV_INLINE __noinline__
#endif
#ifndef HPM_P1_MIN_BLOCKS
#define HPM_P1_MIN_BLOCKS 10
#endif
#ifndef HPM_P2_MIN_BLOCKS
#define HPM_P2_MIN_BLOCKS 10
#endif

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11), counter = (pixel, step, n/4, salt) */
/* ------------------------------------------------------------------ */
struct Rng {
    uint32_t k0, k1, pixel, step, salt, n;
    uint32_t b0, b1, b2, b3;

    __device__ void init(uint32_t klo, uint32_t khi, uint32_t px, uint32_t st, uint32_t sa)
    {
        k0 = klo;
        k1 = khi;
        pixel = px;
        step = st;
        salt = sa;
        n = 0;
    }

    __device__ void block()
    {
        uint32_t c0 = pixel, c1 = step, c2 = n >> 2, c3 = salt;
        uint32_t a0 = k0, a1 = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
            const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
            const uint32_t n0 = hi1 ^ c1 ^ a0;
            const uint32_t n2 = hi0 ^ c3 ^ a1;
            c0 = n0;
            c1 = lo1;
            c2 = n2;
            c3 = lo0;
            a0 += 0x9E3779B9u;
            a1 += 0xBB67AE85u;
        }
        b0 = c0;
        b1 = c1;
        b2 = c2;
        b3 = c3;
    }

    /* uniform in (0,1]: ((x >> 8) + 1) * 2^-24 */
    __device__ float uniform()
    {
        if ((n & 3u) == 0) block();
        const uint32_t j = n & 3u;
        const uint32_t x = j == 0 ? b0 : (j == 1 ? b1 : (j == 2 ? b2 : b3));
        ++n;
        return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
    }
};

/* ------------------------------------------------------------------ */
/* Sampling                                                            */
/* ------------------------------------------------------------------ */

/* texel at integer position (tex2D at x+0.5, y+0.5), edges repeated */
__device__ __forceinline__ float texel(const float *__restrict__ img, int w, int h, int x, int y)
{
    x = min(max(x, 0), w - 1);
    y = min(max(y, 0), h - 1);
    return __ldg(img + (size_t)y * w + x);
}

/* The hoisted reference window has one entry per tap and pixel in shared
 * memory: (weight, weight x reference pixel) as float2 (WinPair), or the
 * weight alone (WinWeight), the reference pixel then being re-read through
 * L1 at each use.  The weight-only form halves the shared memory; it suits
 * k_init (2.75 against 4.7 ms at 1600x1200), while in the half-step kernels
 * the extra L1 loads compete with the texture path (10.2 against 5.4 ms). */
typedef float2 WinPair;
typedef float WinWeight;

/* ------------------------------------------------------------------ */
/* Geometry (HPM.cu:65-133, 227-316, 445-481)                           */
/* ------------------------------------------------------------------ */

__device__ __forceinline__ void normalize3(float4 &v) /* HPM.cu:77-84 */
{
    const float n2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const float inv = rsqrtf(n2);
    v.x *= inv;
    v.y *= inv;
    v.z *= inv;
}

__device__ __forceinline__ float4 view_direction(const HpmCamera &c, int px, int py, float depth)
{
    float X0 = depth * (px - c.K[2]) / c.K[0];
    float X1 = depth * (py - c.K[5]) / c.K[4];
    float X2 = depth;
    const float norm = sqrtf(X0 * X0 + X1 * X1 + X2 * X2);
    return make_float4(X0 / norm, X1 / norm, X2 / norm, 0.0f);
}

__device__ __forceinline__ float distance_to_origin(const HpmCamera &c, int px, int py, float depth, float4 n)
{
    const float X0 = depth * (px - c.K[2]) / c.K[0];
    const float X1 = depth * (py - c.K[5]) / c.K[4];
    const float X2 = depth;
    return -(n.x * X0 + n.y * X1 + n.z * X2);
}

__device__ __forceinline__ float depth_from_plane(const HpmCamera &c, float4 h, int px, int py)
{
    return -h.w * c.K[0] / ((px - c.K[2]) * h.x + (c.K[0] / c.K[4]) * (py - c.K[5]) * h.y + c.K[0] * h.z);
}

__device__ __forceinline__ float4 transform_normal(const HpmCamera &c, float4 h)
{
    float4 r;
    r.x = c.R[0] * h.x + c.R[3] * h.y + c.R[6] * h.z;
    r.y = c.R[1] * h.x + c.R[4] * h.y + c.R[7] * h.z;
    r.z = c.R[2] * h.x + c.R[5] * h.y + c.R[8] * h.z;
    r.w = h.w;
    return r;
}

__device__ __forceinline__ float4 transform_normal_to_ref(const HpmCamera &c, float4 h)
{
    float4 r;
    r.x = c.R[0] * h.x + c.R[1] * h.y + c.R[2] * h.z;
    r.y = c.R[3] * h.x + c.R[4] * h.y + c.R[5] * h.z;
    r.z = c.R[6] * h.x + c.R[7] * h.y + c.R[8] * h.z;
    r.w = h.w;
    return r;
}

__device__ __forceinline__ float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ float4 random_normal(const HpmCamera &c, int px, int py, Rng &rng, float depth) /* HPM.cu:135-161 */
{
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    while (s >= 1.0f) {
        q1 = 2.0f * rng.uniform() - 1.0f;
        q2 = 2.0f * rng.uniform() - 1.0f;
        s = q1 * q1 + q2 * q2;
    }
    const float sq = sqrtf(1.0f - s);
    float4 n = make_float4(2.0f * q1 * sq, 2.0f * q2 * sq, 1.0f - 2.0f * s, 0.0f);
    const float4 v = view_direction(c, px, py, depth);
    if (n.x * v.x + n.y * v.y + n.z * v.z > 0.0f) {
        n.x = -n.x;
        n.y = -n.y;
        n.z = -n.z;
    }
    normalize3(n);
    return n;
}

__device__ float4 perturbed_normal(const HpmCamera &c, int px, int py, float4 normal, Rng &rng,
                                   float pert) /* HPM.cu:163-198 */
{
    const float4 v = view_direction(c, px, py, 1.0f);
    const float a1 = (rng.uniform() - 0.5f) * pert;
    const float a2 = (rng.uniform() - 0.5f) * pert;
    const float a3 = (rng.uniform() - 0.5f) * pert;
    const float s1 = sinf(a1), s2 = sinf(a2), s3 = sinf(a3);
    const float c1 = cosf(a1), c2 = cosf(a2), c3 = cosf(a3);
    float R[9];
    R[0] = c2 * c3;
    R[1] = c3 * s1 * s2 - c1 * s3;
    R[2] = s1 * s3 + c1 * c3 * s2;
    R[3] = c2 * s3;
    R[4] = c1 * c3 + s1 * s2 * s3;
    R[5] = c1 * s2 * s3 - c3 * s1;
    R[6] = -s2;
    R[7] = c2 * s1;
    R[8] = c1 * c2;
    float4 p;
    p.x = R[0] * normal.x + R[1] * normal.y + R[2] * normal.z;
    p.y = R[3] * normal.x + R[4] * normal.y + R[5] * normal.z;
    p.z = R[6] * normal.x + R[7] * normal.y + R[8] * normal.z;
    p.w = normal.w;
    if (dot3(p, v) >= 0.0f) p = normal;
    normalize3(p);
    return p;
}

/* ComputeHomography (HPM.cu:227-287) with the hypothesis-independent part
 * (relative pose) precomputed per view pair. */
__device__ __forceinline__ void homography(const HpmCamera &rc, const HpmCamera &sc, const PairGeom &g, float4 h,
                                           float *H)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        H[3 * i + 0] = g.Rrel[3 * i + 0] - g.trel[i] * h.x / h.w;
        H[3 * i + 1] = g.Rrel[3 * i + 1] - g.trel[i] * h.y / h.w;
        H[3 * i + 2] = g.Rrel[3 * i + 2] - g.trel[i] * h.z / h.w;
    }
    float tmp[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        tmp[3 * i + 0] = H[3 * i + 0] / rc.K[0];
        tmp[3 * i + 1] = H[3 * i + 1] / rc.K[4];
        tmp[3 * i + 2] = -H[3 * i + 0] * rc.K[2] / rc.K[0] - H[3 * i + 1] * rc.K[5] / rc.K[4] + H[3 * i + 2];
    }
    H[0] = sc.K[0] * tmp[0] + sc.K[2] * tmp[6];
    H[1] = sc.K[0] * tmp[1] + sc.K[2] * tmp[7];
    H[2] = sc.K[0] * tmp[2] + sc.K[2] * tmp[8];
    H[3] = sc.K[4] * tmp[3] + sc.K[5] * tmp[6];
    H[4] = sc.K[4] * tmp[4] + sc.K[5] * tmp[7];
    H[5] = sc.K[4] * tmp[5] + sc.K[5] * tmp[8];
    H[6] = sc.K[8] * tmp[6];
    H[7] = sc.K[8] * tmp[7];
    H[8] = sc.K[8] * tmp[8];
}

/* ComputeCorrespondingPoint (HPM.cu:289-296).  Integer pixel coordinates
 * are passed as floats: (float)(px + i) == (float)px + i exactly. */
__device__ __forceinline__ float2 warp(const float *H, float px, float py)
{
    const float x = H[0] * px + H[1] * py + H[2];
    const float y = H[3] * px + H[4] * py + H[5];
    const float z = H[6] * px + H[7] * py + H[8];
    return make_float2(x / z, y / z);
}

/* ------------------------------------------------------------------ */
/* Hoisted reference window                                            */
/* ------------------------------------------------------------------ */

struct RefStats {
    float inv;  /* 1 / sum of weights */
    float mean; /* weighted mean of the reference window */
    float var;  /* weighted variance of the reference window */
};

/* The reference-side half of ComputeBilateralNCC (HPM.cu:318-386) for pixel
 * (px, py): per-tap (weight, weight*ref) into shared memory as one float2,
 * sums in the reference's row-then-total order.  sWW is [tap][kBlock]. */
template <typename Win>
__device__ RefStats ref_window(const PMArgs &a, int px, int py, Win *sWW, int tid)
{
    const ViewDev &rv = a.view[0];
    const float center = texel(rv.img, rv.w, rv.h, px, py);
    float sum_ref = 0.0f, sum_ref_ref = 0.0f, wsum = 0.0f;
    int t = 0;
    for (int i = -5; i < 6; i += 2) {
        float r_ref = 0.0f, r_rr = 0.0f, r_w = 0.0f;
        for (int j = -5; j < 6; j += 2, ++t) {
            const float rp = texel(rv.img, rv.w, rv.h, px + i, py + j);
            const float x_dist = (float)i, y_dist = (float)j;
            const float spatial_dist = sqrtf(x_dist * x_dist + y_dist * y_dist);
            const float color_dist = fabsf(rp - center);
            const float wgt = expf(-spatial_dist / (2.0f * a.sigma_spatial * a.sigma_spatial) -
                                   color_dist / (2.0f * a.sigma_color * a.sigma_color));
            if constexpr (sizeof(Win) == sizeof(float))
                sWW[t * kBlock + tid] = wgt;
            else
                sWW[t * kBlock + tid] = make_float2(wgt, wgt * rp);
            r_ref += wgt * rp;
            r_rr += wgt * rp * rp;
            r_w += wgt;
        }
        sum_ref += r_ref;
        sum_ref_ref += r_rr;
        wsum += r_w;
    }
    RefStats s;
    s.inv = 1.0f / wsum;
    s.mean = sum_ref * s.inv;
    const float mrr = sum_ref_ref * s.inv;
    s.var = mrr - s.mean * s.mean;
    return s;
}

/* Source sample of tap (i, j) of pixel (fpx, fpy): the warped tap position
 * (ComputeCorrespondingPoint, HPM.cu:289-296) through the texture unit at
 * +0.5 (HPM.cu:358-359).  One definition for the NCC and the tap-sample
 * export, so that both evaluate the same expression. */
__device__ __forceinline__ float tap_sample(cudaTextureObject_t tex, const float *H, float fpx, float fpy, int i, int j)
{
    const float2 q = warp(H, fpx + (float)i, fpy + (float)j);
    return tex2D<float>(tex, q.x + 0.5f, q.y + 0.5f);
}

/* The source-side half of ComputeBilateralNCC (HPM.cu:325-397). */
template <typename Win>
__device__ __forceinline__ float ncc(const PMArgs &a, int v, int px, int py, float4 h, const Win *sWW, int tid,
                                     const RefStats &rs)
{
    const HpmCamera &sc = a.cam[v];
    float H[9];
    homography(a.cam[0], sc, a.pair[v], h, H);
    const float fpx = (float)px, fpy = (float)py;
    const float2 pt = warp(H, fpx, fpy);
    if (pt.x >= sc.width || pt.x < 0.0f || pt.y >= sc.height || pt.y < 0.0f) return 2.0f;
    if (rs.var < 1e-5f) return 2.0f; /* the reference reaches the same result after the taps */
    const cudaTextureObject_t tex = a.view[v].tex;
    float sum_src = 0.0f, sum_src_src = 0.0f, sum_ref_src = 0.0f;
    int t = 0;
#pragma unroll
    for (int i = -5; i < 6; i += 2) {
        float r_src = 0.0f, r_ss = 0.0f, r_rs = 0.0f;
#pragma unroll
        for (int j = -5; j < 6; j += 2, ++t) {
            const float sp = tap_sample(tex, H, fpx, fpy, i, j);
            float2 ww;
            if constexpr (sizeof(Win) == sizeof(float)) {
                const float wt = sWW[t * kBlock + tid];
                ww = make_float2(wt, wt * texel(a.view[0].img, a.view[0].w, a.view[0].h, px + i, py + j));
            } else {
                ww = sWW[t * kBlock + tid];
            }
            r_src += ww.x * sp;
            r_ss += ww.x * sp * sp;
            r_rs += ww.y * sp;
        }
        sum_src += r_src;
        sum_src_src += r_ss;
        sum_ref_src += r_rs;
    }
    sum_src *= rs.inv;
    sum_src_src *= rs.inv;
    sum_ref_src *= rs.inv;
    const float var_src = sum_src_src - sum_src * sum_src;
    if (var_src < 1e-5f) return 2.0f;
    const float covar = sum_ref_src - rs.mean * sum_src;
    const float vv = sqrtf(rs.var * var_src);
    return fmaxf(0.0f, fminf(2.0f, 1.0f - covar / vv));
}

/* One NCC window for the loops that score several candidates view by view
 * (inline by default; -DHPM_NCC_CALL=__noinline__ builds it out of line). */
#ifndef HPM_NCC_CALL
#define HPM_NCC_CALL __forceinline__
#endif
template <typename Win>
__device__ HPM_NCC_CALL float ncc_call(const PMArgs &a, int v, int px, int py, float4 h, const Win *sWW, int tid,
                                        RefStats rs)
{
    return ncc(a, v, px, py, h, sWW, tid, rs);
}

/* ComputeMultiViewCostVector (HPM.cu:438-443) into out[v * stride].  Kept
 * out of line so that the 36-tap loop exists once in the binary. */
template <typename Win>
__device__ HPM_CV_INLINE void cost_vector(const PMArgs &a, int px, int py, float4 h, const Win *sWW, int tid,
                                         RefStats rs, float *out, int stride)
{
    for (int v = 1; v < a.n; ++v) out[(size_t)(v - 1) * stride] = ncc(a, v, px, py, h, sWW, tid, rs);
    if (a.counters) atomicAdd(&a.counters[0], (unsigned long long)(a.n - 1));
}

__device__ __forceinline__ void sort_small(float *d, int n) /* HPM.cu:3-12 */
{
    int j;
    for (int i = 1; i < n; i++) {
        const float tmp = d[i];
        for (j = i; j >= 1 && tmp < d[j - 1]; j--) d[j] = d[j - 1];
        d[j] = tmp;
    }
}

/* ComputeMultiViewInitialCostandSelectedViews (HPM.cu:399-436) from a cost
 * vector cv[v * stride]. */
__device__ float initial_cost_from(const PMArgs &a, const float *cv, int stride, uint32_t *views)
{
    float srt[kMaxSrc];
    const int S = a.n - 1;
    int valid = 0;
    for (int v = 0; v < S; ++v) {
        srt[v] = cv[(size_t)v * stride];
        if (srt[v] < 2.0f) valid++;
    }
    sort_small(srt, S);
    uint32_t sel = 0;
    const int top_k = min(valid, a.top_k);
    float result = 2.0f;
    if (top_k > 0) {
        float cost = 0.0f;
        for (int i = 0; i < top_k; ++i) cost += srt[i];
        const float thr = srt[top_k - 1];
        for (int i = 0; i < S; ++i)
            if (cv[(size_t)i * stride] <= thr) sel |= 1u << i;
        result = cost / top_k;
    }
    *views = sel;
    return result;
}

__device__ __forceinline__ void world_point(const HpmCamera &c, float x, float y, float depth, float *P)
{
    float X0 = depth * (x - c.K[2]) / c.K[0];
    float X1 = depth * (y - c.K[5]) / c.K[4];
    float X2 = depth;
    const float T0 = c.R[0] * X0 + c.R[3] * X1 + c.R[6] * X2;
    const float T1 = c.R[1] * X0 + c.R[4] * X1 + c.R[7] * X2;
    const float T2 = c.R[2] * X0 + c.R[5] * X1 + c.R[8] * X2;
    const float Cx = -(c.R[0] * c.t[0] + c.R[3] * c.t[1] + c.R[6] * c.t[2]);
    const float Cy = -(c.R[1] * c.t[0] + c.R[4] * c.t[1] + c.R[7] * c.t[2]);
    const float Cz = -(c.R[2] * c.t[0] + c.R[5] * c.t[1] + c.R[8] * c.t[2]);
    P[0] = T0 + Cx;
    P[1] = T1 + Cy;
    P[2] = T2 + Cz;
}

__device__ __forceinline__ void project(const float *P, const HpmCamera &c, float *pt, float &depth)
{
    const float t0 = c.R[0] * P[0] + c.R[1] * P[1] + c.R[2] * P[2] + c.t[0];
    const float t1 = c.R[3] * P[0] + c.R[4] * P[1] + c.R[5] * P[2] + c.t[1];
    const float t2 = c.R[6] * P[0] + c.R[7] * P[1] + c.R[8] * P[2] + c.t[2];
    depth = c.K[6] * t0 + c.K[7] * t1 + c.K[8] * t2;
    pt[0] = (c.K[0] * t0 + c.K[1] * t1 + c.K[2] * t2) / depth;
    pt[1] = (c.K[3] * t0 + c.K[4] * t1 + c.K[5] * t2) / depth;
}

/* ComputeGeomConsistencyCost (HPM.cu:483-508; capped at a.geom_max, 5 there
 * and 3 in ACMM.cu:494-519) */
__device__ __noinline__ float geom_cost(const PMArgs &a, int v, float4 h, int px, int py)
{
    const HpmCamera &rc = a.cam[0], &sc = a.cam[v];
    const float depth = depth_from_plane(rc, h, px, py);
    float P[3], spt[2], sd;
    world_point(rc, (float)px, (float)py, depth, P);
    project(P, sc, spt, sd);
    const ViewDev &sv = a.view[v];
    const float src_depth = texel(sv.depth, sv.w, sv.h, __float2int_rz(spt[0]), __float2int_rz(spt[1]));
    if (a.counters) atomicAdd(&a.counters[1], 1ull);
    if (src_depth == 0.0f) return a.geom_max;
    float Q[3], bpt[2], rd;
    world_point(sc, spt[0], spt[1], src_depth, Q);
    project(Q, rc, bpt, rd);
    const float dx = px - bpt[0], dy = py - bpt[1];
    return fminf(a.geom_max, sqrtf(dx * dx + dy * dy));
}

/* ------------------------------------------------------------------ */
/* Kernels                                                             */
/* ------------------------------------------------------------------ */

/* R_relative and t_relative of HPM.cu:229-255, with the same expressions. */
__global__ void k_pair_geom(const __grid_constant__ PMArgs a, PairGeom *out)
{
    const int v = threadIdx.x;
    if (v < 1 || v >= a.n) return;
    const HpmCamera &ref_camera = a.cam[0], &src_camera = a.cam[v];
    float ref_C[3], src_C[3];
    ref_C[0] = -(ref_camera.R[0] * ref_camera.t[0] + ref_camera.R[3] * ref_camera.t[1] + ref_camera.R[6] * ref_camera.t[2]);
    ref_C[1] = -(ref_camera.R[1] * ref_camera.t[0] + ref_camera.R[4] * ref_camera.t[1] + ref_camera.R[7] * ref_camera.t[2]);
    ref_C[2] = -(ref_camera.R[2] * ref_camera.t[0] + ref_camera.R[5] * ref_camera.t[1] + ref_camera.R[8] * ref_camera.t[2]);
    src_C[0] = -(src_camera.R[0] * src_camera.t[0] + src_camera.R[3] * src_camera.t[1] + src_camera.R[6] * src_camera.t[2]);
    src_C[1] = -(src_camera.R[1] * src_camera.t[0] + src_camera.R[4] * src_camera.t[1] + src_camera.R[7] * src_camera.t[2]);
    src_C[2] = -(src_camera.R[2] * src_camera.t[0] + src_camera.R[5] * src_camera.t[1] + src_camera.R[8] * src_camera.t[2]);
    PairGeom g;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            g.Rrel[3 * i + j] = src_camera.R[3 * i + 0] * ref_camera.R[3 * j + 0] +
                                src_camera.R[3 * i + 1] * ref_camera.R[3 * j + 1] +
                                src_camera.R[3 * i + 2] * ref_camera.R[3 * j + 2];
    float C_relative[3];
    C_relative[0] = (ref_C[0] - src_C[0]);
    C_relative[1] = (ref_C[1] - src_C[1]);
    C_relative[2] = (ref_C[2] - src_C[2]);
    for (int i = 0; i < 3; ++i)
        g.trel[i] = src_camera.R[3 * i + 0] * C_relative[0] + src_camera.R[3 * i + 1] * C_relative[1] +
                    src_camera.R[3 * i + 2] * C_relative[2];
    out[v] = g;
}

/* Where a pixel's per-pixel buffers live.  Linear pixel indices 2k and
 * 2k + 1 always have different checkerboard colours (neighbours in a row, or
 * across a row end when W is odd), so center >> 1 numbers the pixels of one
 * colour densely: a half-step's hand-off rows (cand_*, one colour at a time)
 * are indexed by it, and the cost-vector cache keeps one such plane per
 * colour.  A half-step then writes whole 32-byte sectors instead of every
 * other word of them. */
struct Slot {
    size_t nh; /* pixels of one colour, rounded up: ceil(W * H / 2) */
    int hc;    /* hand-off slot: center >> 1 */
    size_t cs; /* cache slot: colour plane + hc */
};

__device__ __forceinline__ Slot slot_of(const PMArgs &a, int px, int py)
{
    Slot sl;
    sl.nh = ((size_t)a.W * a.H + 1) >> 1;
    sl.hc = (py * a.W + px) >> 1;
    sl.cs = (size_t)((px + py) & 1) * sl.nh + (size_t)sl.hc;
    return sl;
}

/* Cost-vector cache: for every pixel the cost vector of its current
 * hypothesis, [view][colour][slot].  Written by the initialisation and by
 * every update, read instead of re-scoring the current hypothesis
 * (HPM.cu:1637-1638): NCC is a pure function of (pixel, plane, view), so the
 * cached values are the ones the re-score would produce. */
__device__ __forceinline__ float *cache_at(const PMArgs &a, int v, const Slot &sl)
{
    return a.cost_cache + (size_t)v * 2 * sl.nh + sl.cs;
}

/* RandomInitialization, HPM.cu:510-558.  One thread per pixel. */
__device__ __forceinline__ void init_body(const PMArgs &a, int px, int py, WinWeight *sWW, float *sCV, int tid)
{
    if (px >= a.W || py >= a.H) return;
    const int center = py * a.W + px;
    const HpmCamera &cam = a.cam[0];
    const RefStats rs = ref_window(a, px, py, sWW, tid);
    Rng rng;
    rng.init(a.seed_lo, a.seed_hi, (uint32_t)center, 0u, a.salt);
    float4 h;
    if (a.geom || a.hier) {
        if (a.hier == 1) {
            /* ACMM+NESP hierarchy pass (ACMM.cu:538-604): the acceptance
             * threshold is the initial cost of the plane the reference holds
             * before the normal is filled in, a zero normal with the depth as
             * its distance (ACMM.cpp:707-713 sets only .w of a fresh,
             * zero-filled array); at the maps' own size (hier 2) the
             * reference leaves it unset, taken as 0 */
            const float4 hz = make_float4(0.0f, 0.0f, 0.0f, a.planes[center].w);
            float *cvz = sCV + tid;
            cost_vector(a, px, py, hz, sWW, tid, rs, cvz, kBlock);
            uint32_t unused;
            a.pre_costs[center] = initial_cost_from(a, cvz, kBlock, &unused);
        } else if (a.hier == 2) {
            a.pre_costs[center] = 0.0f;
        }
        h = transform_normal_to_ref(cam, a.planes[center]);
        const float depth = h.w;
        h.w = distance_to_origin(cam, px, py, depth, h);
    } else if (a.prior) {
        if (a.masks[center] > 0 && a.costs[center] >= 0.1f) {
            const float pert = 0.02f;
            const float4 hp = a.prior_planes[center];
            float dp = hp.w;
            const float lo = (1 - 3 * pert) * dp;
            const float hi = (1 + 3 * pert) * dp;
            dp = rng.uniform() * (hi - lo) + lo;
            h = perturbed_normal(cam, px, py, hp, rng, (float)(3 * pert * kPiD));
            h.w = dp;
        } else {
            /* the previous pass's world-frame normal, reused as it is
             * (HPM.cu:547-551); with fix_quirks rotated back to the
             * reference frame first, as the geometric branch does */
            h = a.fix_quirks ? transform_normal_to_ref(cam, a.planes[center]) : a.planes[center];
            const float depth = h.w;
            h.w = distance_to_origin(cam, px, py, depth, h);
        }
    } else {
        const float depth = rng.uniform() * (a.dmax - a.dmin) + a.dmin;
        h = random_normal(cam, px, py, rng, depth);
        h.w = distance_to_origin(cam, px, py, depth, h);
    }
    float *cv = sCV + tid;
    cost_vector(a, px, py, h, sWW, tid, rs, cv, kBlock);
    uint32_t sel;
    const float c = initial_cost_from(a, cv, kBlock, &sel);
    a.planes[center] = h;
    a.costs[center] = c;
    a.views[center] = sel;
    if (a.cost_cache) {
        const Slot sl = slot_of(a, px, py);
        for (int v = 0; v < a.n - 1; ++v) *cache_at(a, v, sl) = cv[v * kBlock];
    }
}

__global__ void __launch_bounds__(kBlock) k_init(const __grid_constant__ PMArgs a)
{
    __shared__ WinWeight sWW[kTaps * kBlock];
    __shared__ float sCV[kMaxSrc * kBlock];
    const int tid = threadIdx.y * kBlockX + threadIdx.x;
    init_body(a, blockIdx.x * kBlockX + threadIdx.x, blockIdx.y * kBlockY + threadIdx.y, sWW, sCV, tid);
}

/* Validity of the first site of direction k at extension round r (HPM.cu:1252-1445 and the
 * Extended* functions 560-1034).  Directions: 0 left_up, 1 up_far, 2 right_up, 3 down_far,
 * 4 right_down, 5 left_far, 6 left_down, 7 right_far (HPM.cu:1245). */
__device__ __forceinline__ bool first_site_valid(int k, int r, int px, int py, int W, int H)
{
    const int s = 10 * r, d = 8 * r;
    switch (k) {
    case 1: return py > 4 + s;
    case 3: return py < H - 5 - s;
    case 5: return px > 4 + s;
    case 7: return px < W - 5 - s;
    case 0: return px > 4 + d && py > 5 + d;
    case 2: return px < W - 6 - d && py > 4 + d;
    case 4: return px < W - 5 - d && py < H - 6 - d;
    default: return px > 5 + d && py < H - 5 - d;
    }
}

/* NESP site choice of one direction at round r.  Strips: 5 sites 2 apart
 * from +/-(5+10r), the right strip keeps the maximum (HPM.cu:1330, 744;
 * the minimum with fix_quirks).
 * Polylines: start (+/-5|6) shifted 8r outward, then 7 zig-zag steps of 2
 * (HPM.cu:1346-1471). */
__device__ int select_site(const PMArgs &a, int k, int r, int px, int py)
{
    const int W = a.W, H = a.H;
    const float *costs = a.costs;
    if (k & 1) {
        const int dx = (k == 5) ? -1 : (k == 7 ? 1 : 0);
        const int dy = (k == 1) ? -1 : (k == 3 ? 1 : 0);
        const int off = 5 + 10 * r;
        int best = (py + dy * off) * W + (px + dx * off);
        float cmin = costs[best];
        for (int i = 1; i < 5; ++i) {
            bool ok;
            switch (k) {
            case 1: ok = py > 4 + 2 * i + 10 * r; break;
            case 3: ok = py < H - 5 - 2 * i - 10 * r; break;
            case 5: ok = px > 4 + 2 * i + 10 * r; break;
            default: ok = px < W - 5 - 2 * i - 10 * r; break;
            }
            if (!ok) break;
            const int q = (py + dy * (off + 2 * i)) * W + (px + dx * (off + 2 * i));
            const float cq = costs[q];
            if ((k == 7 && !a.fix_quirks) ? (cmin < cq) : (cq < cmin)) {
                cmin = cq;
                best = q;
            }
        }
        return best;
    }
    int sx, sy, ex, ey, ox, oy; /* start, even step, odd step */
    switch (k) {
    case 0: sx = -5 - 8 * r; sy = -6 - 8 * r; ex = -2; ey = 0; ox = 0; oy = -2; break;
    case 2: sx = 6 + 8 * r; sy = -5 - 8 * r; ex = 0; ey = -2; ox = 2; oy = 0; break;
    case 4: sx = 5 + 8 * r; sy = 6 + 8 * r; ex = 2; ey = 0; ox = 0; oy = 2; break;
    default: sx = -6 - 8 * r; sy = 5 + 8 * r; ex = 0; ey = 2; ox = -2; oy = 0; break;
    }
    int x = px + sx, y = py + sy;
    int best = y * W + x;
    float cmin = costs[best];
    for (int i = 0; i < 7; ++i) {
        if ((i & 1) == 0) {
            x += ex;
            y += ey;
        } else {
            x += ox;
            y += oy;
        }
        if (x >= 0 && x < W && y < H && y >= 0) {
            const int q = y * W + x;
            const float cq = costs[q];
            if (cq < cmin) {
                cmin = cq;
                best = q;
            }
        } else {
            break;
        }
    }
    return best;
}

__device__ __forceinline__ float restricted_prior(float depth_diff, float angle_cos, float two_dss, float two_ass)
{
    const float gamma = 0.5f;
    const float angle_diff = acosf(angle_cos);
    return gamma + expf(-depth_diff * depth_diff / two_dss) * expf(-angle_diff * angle_diff / two_ass);
}

__device__ __forceinline__ bool same_plane(float4 p, float4 q)
{
    return __float_as_uint(p.x) == __float_as_uint(q.x) && __float_as_uint(p.y) == __float_as_uint(q.y) &&
           __float_as_uint(p.z) == __float_as_uint(q.z) && __float_as_uint(p.w) == __float_as_uint(q.w);
}

/* One red/black half-step runs as two kernels that hand the per-pixel cost
 * matrix over through L2 instead of holding it in shared memory for the
 * whole pixel update (8 x S floats per pixel is what limits occupancy):
 *
 *   k_prop_dirs    NESP site choice, direction cost vectors, extension
 *                  (HPM.cu:1222-1543)
 *   k_prop_refine  joint view selection, candidate choice and
 *                  PlaneHypothesisRefinement (HPM.cu:1548-1725, 1143-1220)
 *
 * The other colour is read-only during both kernels, so splitting the pixel
 * update changes nothing in what is computed. */

#define CAG(k, v) a.cand_costs[(size_t)((k) * S + (v)) * sl.nh + sl.hc]
/* Hand-off stores use the streaming cache policy (st.global.cs, evict
 * first): the rows are read once by the next kernel, and at ~0.5 GB a
 * half-step they would otherwise push the source images out of L2. */
#define CAG_PUT(k, v, x) __stcs(&CAG(k, v), (x))

/* Where the cost row of direction k lives, 4 bits per direction in the
 * pixel's hand-off code (cand_flags): the row itself, the cost-vector cache
 * (the candidate equals the current hypothesis), the row of an earlier
 * direction with the same plane, or nowhere (an invalid direction, whose row
 * holds 2 at [0][0] and 0 elsewhere because float cost_array[8][32] =
 * { 2.0f } sets only [0][0], HPM.cu:1244).  Copies and invalid rows are
 * resolved on reading instead of being written out. */
constexpr uint32_t kRowCache = 8, kRowOwn = 9, kRowNone = 10;
constexpr uint32_t kCodeAllNone = 0xAAAAAAAAu;

__device__ __forceinline__ bool dir_valid(uint32_t code, int k) { return ((code >> (4 * k)) & 15u) != kRowNone; }

__device__ __forceinline__ float dir_cost(const PMArgs &a, uint32_t code, int k, int v, int S, const Slot &sl)
{
    const uint32_t src = (code >> (4 * k)) & 15u;
    if (src == kRowOwn) return CAG(k, v);
    if (src == kRowCache) return *cache_at(a, v, sl);
    if (src < 8) return CAG(src, v);
    return (a.fix_quirks || (k == 0 && v == 0)) ? 2.0f : 0.0f; /* fix_quirks: the intended {2, 2, ...} */
}

__device__ __forceinline__ void prop_dirs_body(const PMArgs &a, int iter, int px, int py, WinPair *sWW, int tid)
{
    if (px >= a.W || py >= a.rows_cov) return;
    const int W = a.W, H = a.H, S = a.n - 1;
    const int center = py * W + px;
    const Slot sl = slot_of(a, px, py);
    const RefStats rs = ref_window(a, px, py, sWW, tid);
    const float4 cur = a.planes[center];

    int pos[8];
    uint32_t flags = 0;
    pos[0] = center - 5 - 6 * W;
    pos[1] = center - W * 5;
    pos[2] = center + 6 - 5 * W;
    pos[3] = center + W * 5;
    pos[4] = center + 5 + 6 * W;
    pos[5] = center - 5;
    pos[6] = center - 6 + 5 * W;
    pos[7] = center + 5;
    /* 1) NESP sites of the 8 directions.  Identical planes give identical
     * cost vectors: a candidate whose plane equals the current hypothesis
     * (cost vector cached) or an earlier candidate reuses those values
     * (dir_cost resolves the row on reading). */
    uint32_t code = kCodeAllNone; /* 4 bits per direction */
    uint32_t eval_mask = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (!first_site_valid(k, 0, px, py, W, H)) continue;
        flags |= 1u << k;
        pos[k] = select_site(a, k, 0, px, py);
        const float4 c = a.planes[pos[k]];
        uint32_t src = same_plane(c, cur) ? kRowCache : kRowNone;
#pragma unroll
        for (int j = 0; j < k; ++j)
            if (src == kRowNone && ((flags >> j) & 1u) && same_plane(c, a.planes[pos[j]])) src = (uint32_t)j;
        if (src == kRowNone) {
            src = kRowOwn;
            eval_mask |= 1u << k;
        }
        code = (code & ~(15u << (4 * k))) | (src << (4 * k));
    }
    /* 2) the distinct candidates, view by view, so that the threads of a
     * block sample one source image at a time (texture-cache locality) */
    for (int v = 0; v < S; ++v) {
        uint32_t m = eval_mask;
        while (m) {
            const int k = __ffs(m) - 1;
            m &= m - 1;
            CAG_PUT(k, v, ncc_call(a, v + 1, px, py, a.planes[pos[k]], sWW, tid, rs));
        }
    }
    if (a.counters && eval_mask) atomicAdd(&a.counters[0], (unsigned long long)(__popc(eval_mask) * S));

    /* Extension: only the left-up polyline can extend, because
     * bool symbol_eight_orientations[10] = { true } sets index 0 only
     * (HPM.cu:1475).  JudgeExtend: HPM.cu:1036-1059. */
    if (flags & 1u) {
        bool detached = false; /* rows that copy direction 0's first row hold their own copy */
        for (int r = 0; r < 3; ++r) {
            const float good = (float)(0.8 * exp(-iter * iter * (3 - r) / 90.0));
            int good_sum = 0, bad_sum = 0;
            for (int v = 0; v < S; ++v) {
                const float c = dir_cost(a, code, 0, v, S, sl);
                if (c < good) good_sum++;
                if (c > 1.2f) bad_sum++;
            }
            if (good_sum >= 1 && bad_sum <= 2) break;
            if (!first_site_valid(0, r, px, py, W, H)) continue; /* flag[0] is set: keep site and costs */
            const int best = select_site(a, 0, r, px, py);
            if (a.costs[best] > a.costs[pos[0]]) continue; /* the previous site is better: keep it */
            const float4 prev = a.planes[pos[0]];
            pos[0] = best;
            const float4 p = a.planes[best];
            if (same_plane(p, prev)) continue;
            /* direction 0's row changes: the rows that refer to it keep the
             * values it had when they were chosen */
            if (!detached) {
                detached = true;
#pragma unroll
                for (int k = 1; k < 8; ++k)
                    if (((code >> (4 * k)) & 15u) == 0u) {
                        for (int v = 0; v < S; ++v) CAG_PUT(k, v, dir_cost(a, code, 0, v, S, sl));
                        code = (code & ~(15u << (4 * k))) | (kRowOwn << (4 * k));
                    }
            }
            if (same_plane(p, cur)) {
                code = (code & ~15u) | kRowCache;
                continue;
            }
            int src = -1;
#pragma unroll
            for (int j = 1; j < 8; ++j)
                if (src < 0 && ((flags >> j) & 1u) && same_plane(p, a.planes[pos[j]])) src = j;
            if (src >= 0) {
                const uint32_t sj = (code >> (4 * src)) & 15u;
                code = (code & ~15u) | (sj == kRowOwn ? (uint32_t)src : sj);
            } else {
                cost_vector(a, px, py, p, sWW, tid, rs, &CAG(0, 0), (int)sl.nh);
                code = (code & ~15u) | kRowOwn;
            }
        }
    }
    /* 3) every valid direction's row in its own slot: a row that refers to
     * the cost-vector cache or to an earlier direction (always one that owns
     * its row) is copied there, so that the refinement reads each row with
     * one load and no decoding; the code then holds only own and none */
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t src = (code >> (4 * k)) & 15u;
        if (src == kRowOwn || src == kRowNone) continue;
        for (int v = 0; v < S; ++v) CAG_PUT(k, v, src == kRowCache ? *cache_at(a, v, sl) : CAG(src, v));
        code = (code & ~(15u << (4 * k))) | (kRowOwn << (4 * k));
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) __stcs(&a.cand_pos[(size_t)k * sl.nh + sl.hc], pos[k]);
    __stcs(&a.cand_flags[sl.hc], code);
}

/* WW: pixels of one colour per warp row (the half-step tile, tuned per view
 * size by the batched form; 8 elsewhere) */
template <int WW>
__global__ void __launch_bounds__(kBlock, HPM_P1_MIN_BLOCKS) k_prop_dirs(const __grid_constant__ PMArgs a, int iter,
                                                                          int color)
{
    __shared__ WinPair sWW[kTaps * kBlock];
    const int tid = threadIdx.y * kBlockX + threadIdx.x;
    int px, py;
    half_step_pixel_at(blockIdx.x, blockIdx.y, WW, color, px, py);
    prop_dirs_body(a, iter, px, py, sWW, tid);
}

/* PROP: the prior-net form, whose network proposal a.proposals[center] is a
 * sixth refinement candidate, scored by the same NCC (and prior terms) as the
 * other five and accepted by the same rule.  It takes no random draws, so
 * the random stream of the other candidates is unchanged.
 * ACMM: the ACMM+NESP variant (ACMM.cu:1548-1629, 623-667): geometric weight
 * 0.2 on the current and refined hypotheses, no NaN fallback, and in a
 * hierarchy pass the threshold rule on the result.  A separate
 * instantiation, so that the HPM-MVS kernels keep their registers. */
template <int SMAX, bool PROP, bool ACMM>
__device__ __forceinline__ void prop_refine_body(const PMArgs &a, int iter, int px, int py, WinPair *sWW, int tid)
{
    constexpr float kGeomW = ACMM ? 0.2f : 0.1f; /* HPM.cu:1642, 1189; ACMM.cu:1596, 651 */
    if (px >= a.W || py >= a.rows_cov) return;
    const int W = a.W, S = a.n - 1;
    const int center = py * W + px;
    const Slot sl = slot_of(a, px, py);
    const HpmCamera &cam = a.cam[0];
    const uint32_t code = a.cand_flags[sl.hc];
    uint32_t flags = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
        if (dir_valid(code, k)) flags |= 1u << k;
    int pos[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) pos[k] = a.cand_pos[(size_t)k * sl.nh + sl.hc];
#define FLAG(k) (((flags >> (k)) & 1u) != 0)
/* cost of direction k for view v: every valid direction owns its row (step
 * 3 of prop_dirs_body); an invalid one holds the reference's {2, 0, ...}
 * (HPM.cu:1244), or 2 everywhere with fix_quirks */
#define ROWC(k, v) (FLAG(k) ? CAG(k, v) : ((a.fix_quirks || ((k) == 0 && (v) == 0)) ? 2.0f : 0.0f))
    Rng rng;
    rng.init(a.seed_lo, a.seed_hi, (uint32_t)center, (uint32_t)(1 + iter), a.salt);

    /* Multi-hypothesis joint view selection, HPM.cu:1548-1613. */
    float vw[SMAX];
    float sp[SMAX];
    const uint32_t nbm[4] = {FLAG(1) ? a.views[center - W * 5] : 0u, FLAG(3) ? a.views[center + W * 5] : 0u,
                             FLAG(5) ? a.views[center - 5] : 0u, FLAG(7) ? a.views[center + 5] : 0u};
    const float thr = (float)(0.8 * expf((float)(iter * iter) / (-90.0f)));
#pragma unroll
    for (int v = 0; v < SMAX; ++v) {
        vw[v] = 0.0f;
        sp[v] = 0.0f;
        if (v >= S) continue;
        float prior = 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (FLAG(2 * i + 1)) prior += ((nbm[i] >> v) & 1u) ? 0.9f : 0.1f;
        float count = 0;
        int count_false = 0;
        float tmpw = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float c = ROWC(k, v);
            if (c < thr) {
                tmpw += expf(c * c / (-0.18f));
                count++;
            }
            if (c > 1.2f) count_false++;
        }
        float p = 0.0f;
        if (count > 2 && count_false < 3)
            p = tmpw / count;
        else if (count_false < 3)
            p = expf(thr * thr / (-0.32f));
        sp[v] = p * prior;
    }
    {
        float s = 0.0f;
#pragma unroll
        for (int v = 0; v < SMAX; ++v)
            if (v < S) s += sp[v];
        const float inv = 1.0f / s;
        float cum = 0.0f;
#pragma unroll
        for (int v = 0; v < SMAX; ++v)
            if (v < S) {
                cum += sp[v] * inv;
                sp[v] = cum;
            }
    }
    for (int smp = 0; smp < 15; ++smp) {
        const float rp = rng.uniform() - FLT_EPSILON;
        bool done = false;
#pragma unroll
        for (int v = 0; v < SMAX; ++v) {
            if (!done && v < S && sp[v] > rp) {
                vw[v] += 1.0f;
                done = true;
            }
        }
    }
    uint32_t tsv = 0;
    float wn = 0.0f;
    /* the integer view weights, 4 bits per view (at most 15 draws), for
     * loops over the selected views with a run-time index */
    unsigned long long vw_lo = 0, vw_hi = 0;
#pragma unroll
    for (int v = 0; v < SMAX; ++v)
        if (v < S && vw[v] > 0) {
            tsv |= 1u << v;
            wn += vw[v];
            if (v < 16)
                vw_lo |= (unsigned long long)vw[v] << (4 * v);
            else
                vw_hi |= (unsigned long long)vw[v] << (4 * (v - 16));
        }

    float fc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float f = 0.0f;
        float4 hk = make_float4(0, 0, 0, 1);
        if (a.geom && FLAG(k)) hk = a.planes[pos[k]];
#pragma unroll
        for (int v = 0; v < SMAX; ++v) {
            if (v < S && vw[v] > 0) {
                if (a.geom) {
                    if (FLAG(k))
                        f += vw[v] * (ROWC(k, v) + 0.1f * geom_cost(a, v + 1, hk, px, py));
                    else
                        f += vw[v] * (ROWC(k, v) + 0.1f * 5.0f);
                } else {
                    f += vw[v] * ROWC(k, v);
                }
            }
        }
        fc[k] = f / wn;
    }
    int min_idx = 0;
    {
        float m = fc[0];
#pragma unroll
        for (int k = 1; k < 8; ++k)
            if (fc[k] <= m) {
                m = fc[k];
                min_idx = k;
            }
    }

    /* re-score of the current hypothesis (HPM.cu:1637-1650), from the cache */
    const float4 cur = a.planes[center];
    float4 plane = cur;
    int best_row = -1; /* -1: the cached current hypothesis */
    float cost_now = 0.0f;
#pragma unroll
    for (int v = 0; v < SMAX; ++v) {
        if (v < S && vw[v] > 0) {
            if (a.geom)
                cost_now += vw[v] * (*cache_at(a, v, sl) + kGeomW * geom_cost(a, v + 1, plane, px, py));
            else
                cost_now += vw[v] * *cache_at(a, v, sl);
        }
    }
    cost_now /= wn;
    float cost = cost_now;
    uint32_t sel = a.views[center];
    float depth_now = depth_from_plane(cam, plane, px, py);

    float restricted_cost = 0.0f;
    if (a.prior) {
        const float depth_sigma = (a.dmax - a.dmin) / 64.0f;
        const float two_dss = 2 * depth_sigma * depth_sigma;
        const float angle_sigma = (float)(kPiD * (5.0f / 180.0f));
        const float two_ass = 2 * angle_sigma * angle_sigma;
        const float4 pp = a.prior_planes[center];
        const float depth_prior = depth_from_plane(cam, pp, px, py);
        const float beta = 0.18f;
        if (a.masks[center] > 0) {
            float rfc[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                rfc[k] = 0.0f;
                if (FLAG(k)) {
                    const float4 hq = a.planes[pos[k]];
                    const float dn = depth_from_plane(cam, hq, px, py);
                    const float pr = restricted_prior(dn - depth_prior, dot3(pp, hq), two_dss, two_ass);
                    rfc[k] = expf(-fc[k] * fc[k] / beta) * pr;
                }
            }
            int max_idx = 0;
            {
                float m = rfc[0];
#pragma unroll
                for (int k = 1; k < 8; ++k)
                    if (rfc[k] >= m) {
                        m = rfc[k];
                        max_idx = k;
                    }
            }
            const float dn = depth_from_plane(cam, plane, px, py);
            const float pr = restricted_prior(dn - depth_prior, dot3(pp, plane), two_dss, two_ass);
            const float rcn = expf(-cost_now * cost_now / beta) * pr;
            if (FLAG(max_idx)) {
                const float4 hb = a.planes[pos[max_idx]];
                const float db = depth_from_plane(cam, hb, px, py);
                if (db >= a.dmin && db <= a.dmax && rfc[max_idx] > rcn) {
                    depth_now = db;
                    plane = hb;
                    best_row = max_idx;
                    cost = fc[max_idx];
                    restricted_cost = rfc[max_idx];
                    sel = tsv;
                }
            }
        } else if (FLAG(min_idx)) {
            const float4 hb = a.planes[pos[min_idx]];
            const float db = depth_from_plane(cam, hb, px, py);
            if (db >= a.dmin && db <= a.dmax && fc[min_idx] < cost_now) {
                depth_now = db;
                plane = hb;
                best_row = min_idx;
                cost = fc[min_idx];
            }
        }
    }
    if (!a.prior && FLAG(min_idx)) {
        const float4 hb = a.planes[pos[min_idx]];
        const float db = depth_from_plane(cam, hb, px, py);
        if (db >= a.dmin && db <= a.dmax && fc[min_idx] < cost_now) {
            depth_now = db;
            plane = hb;
            best_row = min_idx;
            cost = fc[min_idx];
            sel = tsv;
        }
        if (!ACMM && cost != cost) { /* the ACMM+NESP variant has no such fallback */
            depth_now = db;
            plane = hb;
            best_row = min_idx;
            sel = tsv;
        }
    }

    /* PlaneHypothesisRefinement, HPM.cu:1143-1220 */
    const RefStats rs = ref_window(a, px, py, sWW, tid);
    {
        const float pert = 0.02f;
        const float depth_sigma = (a.dmax - a.dmin) / 64.0f;
        const float two_dss = 2 * depth_sigma * depth_sigma;
        const float angle_sigma = (float)(kPiD * (5.0f / 180.0f));
        const float two_ass = 2 * angle_sigma * angle_sigma;
        const float beta = 0.18f;
        float depth_prior = 0.0f;
        const bool use_prior = a.prior && a.masks[center] > 0;
        float4 pp = make_float4(0, 0, 0, 0);
        float depth_rand;
        float4 n_rand;
        if (use_prior) {
            pp = a.prior_planes[center];
            depth_prior = depth_from_plane(cam, pp, px, py);
            depth_rand = rng.uniform() * 6 * depth_sigma + (depth_prior - 3 * depth_sigma);
            n_rand = perturbed_normal(cam, px, py, pp, rng, angle_sigma);
        } else {
            depth_rand = rng.uniform() * (a.dmax - a.dmin) + a.dmin;
            n_rand = random_normal(cam, px, py, rng, depth_now);
        }
        const float lo = (1 - pert) * depth_now, hi = (1 + pert) * depth_now;
        float depth_pert = rng.uniform() * (hi - lo) + lo;
        /* do { ... } while (d < min && d > max) never repeats (HPM.cu:1170-1172);
         * with fix_quirks the draw repeats while out of range, at most 8 times */
        for (int t = 1; a.fix_quirks && t < 8 && (depth_pert < a.dmin || depth_pert > a.dmax); ++t)
            depth_pert = rng.uniform() * (hi - lo) + lo;
        const float4 n_pert = perturbed_normal(cam, px, py, plane, rng, (float)(pert * kPiD));
        const float depths[5] = {depth_rand, depth_now, depth_rand, depth_now, depth_pert};
        const float4 normals[5] = {plane, n_rand, n_rand, n_pert, plane};
        /* The five candidates are built before any is scored (HPM.cu:1180-
         * 1183), so they are scored view by view with the view index uniform
         * across the warp (one source texture per texture instruction, one
         * source image at a time per block); each NCC value goes to the
         * candidate's hand-off row for the cache. */
        constexpr int NC = PROP ? 6 : 5;
        float4 cand[NC];
        float cand_depth[NC];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            cand[i] = normals[i];
            cand[i].w = distance_to_origin(cam, px, py, depths[i], cand[i]);
            cand_depth[i] = depths[i];
        }
        if constexpr (PROP) {
            cand[5] = a.proposals[center];
            cand_depth[5] = depth_from_plane(cam, cand[5], px, py);
        }
        float tc[NC];
#pragma unroll
        for (int i = 0; i < NC; ++i) tc[i] = 0.0f;
        for (int v = 0; v < S; ++v) {
            const bool selected = (tsv >> v) & 1u;
            const float w = (float)((v < 16 ? (vw_lo >> (4 * v)) : (vw_hi >> (4 * (v - 16)))) & 15ull);
#pragma unroll 1
            for (int k = 0; k < NC; ++k) {
                /* candidates 0 and 2 share the random depth, hence the window
                 * centre in every source view; 1, 3 and 4 sit at or near the
                 * current depth: scoring 0, 2, 1, 3, 4 keeps windows with the
                 * same centre back to back in the texture cache */
                const int i = (0x543120 >> (4 * k)) & 15;
                const float c = ncc_call(a, v + 1, px, py, cand[i], sWW, tid, rs);
                CAG_PUT(kRefineRow + i, v, c);
                if (selected) {
                    if (a.geom)
                        tc[i] += w * (c + kGeomW * geom_cost(a, v + 1, cand[i], px, py));
                    else
                        tc[i] += w * c;
                }
            }
        }
        if (a.counters) atomicAdd(&a.counters[0], (unsigned long long)(NC * S));
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            const float tci = tc[i] / wn;
            const float depth_before = depth_from_plane(cam, cand[i], px, py);
            bool take;
            if (use_prior) {
                const float dd = cand_depth[i] - depth_prior;
                const float pr = restricted_prior(dd, dot3(pp, cand[i]), two_dss, two_ass);
                const float rtc = expf(-tci * tci / beta) * pr;
                take = depth_before >= a.dmin && depth_before <= a.dmax && rtc > restricted_cost;
                if (take) restricted_cost = rtc;
            } else {
                take = depth_before >= a.dmin && depth_before <= a.dmax && tci < cost;
            }
            if (take) {
                depth_now = depth_before;
                plane = cand[i];
                cost = tci;
                best_row = kRefineRow + i;
            }
        }
    }
    /* ACMM+NESP hierarchy pass (ACMM.cu:1617-1624): the update is kept only
     * where it beats the threshold by 0.1; otherwise the pixel keeps its
     * plane with the current hypothesis's cost under this half-step's view
     * weights (its selected views may still have changed) */
    if constexpr (ACMM) {
        if (a.pre_costs && !(cost < a.pre_costs[center] - 0.1f)) {
            plane = cur;
            cost = cost_now;
            best_row = -1;
        }
    }
    a.planes[center] = plane;
    a.costs[center] = cost;
    a.views[center] = sel;
    if (best_row >= kRefineRow) {
        for (int v = 0; v < S; ++v) *cache_at(a, v, sl) = CAG(best_row, v);
    } else if (best_row >= 0) {
        for (int v = 0; v < S; ++v) *cache_at(a, v, sl) = CAG(best_row, v);
    }
#undef ROWC
#undef FLAG
}

template <int SMAX, bool PROP, int WW, bool ACMM = false>
__global__ void __launch_bounds__(kBlock, HPM_P2_MIN_BLOCKS) k_prop_refine(const __grid_constant__ PMArgs a, int iter,
                                                                            int color)
{
    __shared__ WinPair sWW[kTaps * kBlock];
    const int tid = threadIdx.y * kBlockX + threadIdx.x;
    int px, py;
    half_step_pixel_at(blockIdx.x, blockIdx.y, WW, color, px, py);
    prop_refine_body<SMAX, PROP, ACMM>(a, iter, px, py, sWW, tid);
}
#undef CAG_PUT
#undef CAG

/* GetDepthandNormal, HPM.cu:1751-1764 */
__global__ void k_depth_normal(const __grid_constant__ PMArgs a, float4 *planes)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= a.W || py >= a.H) return;
    const int c = py * a.W + px;
    float4 h = planes[c];
    h.w = depth_from_plane(a.cam[0], h, px, py);
    planes[c] = transform_normal(a.cam[0], h);
}

/* CheckerboardFilter, HPM.cu:1766-1904 */
__global__ void k_filter(const __grid_constant__ PMArgs a, float4 *pl, const float *costs, int color)
{
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    const int px = blockIdx.x * (2 * blockDim.x) + 2 * threadIdx.x + ((py + color) & 1);
    const int W = a.W, H = a.H;
    if (px >= W || py >= a.rows_cov) return;
    const int center = py * W + px;
    if (costs[center] < 0.001f) return;
    float f[21];
    int n = 0;
    f[n++] = pl[center].w;
    const int left = center - 1, leftleft = center - 3, up = center - W, upup = center - 3 * W;
    const int down = center + W, downdown = center + 3 * W, right = center + 1, rightright = center + 3;
    if (py > 0) f[n++] = pl[up].w;
    if (py > 2) f[n++] = pl[upup].w;
    if (py > 4) f[n++] = pl[upup - W * 2].w;
    if (py < H - 1) f[n++] = pl[down].w;
    if (py < H - 3) f[n++] = pl[downdown].w;
    if (py < H - 5) f[n++] = pl[downdown + W * 2].w;
    if (px > 0) f[n++] = pl[left].w;
    if (px > 2) f[n++] = pl[leftleft].w;
    if (px > 4) f[n++] = pl[leftleft - 2].w;
    if (px < W - 1) f[n++] = pl[right].w;
    if (px < W - 3) f[n++] = pl[rightright].w;
    if (px < W - 5) f[n++] = pl[rightright + 2].w;
    if (py > 0 && px < W - 2) f[n++] = pl[up + 2].w;
    if (py < H - 1 && px < W - 2) f[n++] = pl[down + 2].w;
    if (py > 0 && px > 1) f[n++] = pl[up - 2].w;
    if (py < H - 1 && px > 1) f[n++] = pl[down - 2].w;
    if (px > 0 && py > 2) f[n++] = pl[left - W * 2].w;
    if (px < W - 1 && py > 2) f[n++] = pl[right - W * 2].w;
    if (px > 0 && py < H - 2) f[n++] = pl[left + W * 2].w;
    if (px < W - 1 && py < H - 2) f[n++] = pl[right + W * 2].w;
    sort_small(f, n);
    const int m = n / 2;
    pl[center].w = (n % 2 == 0) ? (f[m - 1] + f[m]) / 2 : f[m];
}

__global__ void __launch_bounds__(kBlock) k_cost_vectors(const __grid_constant__ PMArgs a, const float4 *planes,
                                                          float *out)
{
    __shared__ WinPair sWW[kTaps * kBlock];
    const int tid = threadIdx.y * kBlockX + threadIdx.x;
    const int px = blockIdx.x * kBlockX + threadIdx.x;
    const int py = blockIdx.y * kBlockY + threadIdx.y;
    if (px >= a.W || py >= a.H) return;
    const RefStats rs = ref_window(a, px, py, sWW, tid);
    const int c = py * a.W + px;
    const int S = a.n - 1;
    cost_vector(a, px, py, planes[c], sWW, tid, rs, out + (size_t)c * S, 1);
}

__global__ void __launch_bounds__(kBlock) k_initial_costs(const __grid_constant__ PMArgs a, const float4 *planes,
                                                          float *cost, uint32_t *views)
{
    __shared__ WinPair sWW[kTaps * kBlock];
    __shared__ float sCV[kMaxSrc * kBlock];
    const int tid = threadIdx.y * kBlockX + threadIdx.x;
    const int px = blockIdx.x * kBlockX + threadIdx.x;
    const int py = blockIdx.y * kBlockY + threadIdx.y;
    if (px >= a.W || py >= a.H) return;
    const RefStats rs = ref_window(a, px, py, sWW, tid);
    const int c = py * a.W + px;
    cost_vector(a, px, py, planes[c], sWW, tid, rs, sCV + tid, kBlock);
    cost[c] = initial_cost_from(a, sCV + tid, kBlock, &views[c]);
}

__global__ void k_geom_costs(const __grid_constant__ PMArgs a, const float4 *planes, float *out)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= a.W || py >= a.H) return;
    const int c = py * a.W + px;
    const int S = a.n - 1;
    for (int v = 1; v < a.n; ++v) out[(size_t)c * S + v - 1] = geom_cost(a, v, planes[c], px, py);
}

/* The 36 source samples of the NCC window of listed pixels, per source view
 * (the values ncc() weighs), and whether the warped centre is inside. */
__global__ void k_tap_samples(const __grid_constant__ PMArgs a, const float4 *planes, const int *pixels, int n,
                              float *out, int *inside)
{
    const int S = a.n - 1;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * S) return;
    const int pi = k / S, v = k % S + 1;
    const int px = pixels[pi] % a.W, py = pixels[pi] / a.W;
    const HpmCamera &sc = a.cam[v];
    float H[9];
    homography(a.cam[0], sc, a.pair[v], planes[pixels[pi]], H);
    const float fpx = (float)px, fpy = (float)py;
    const float2 pt = warp(H, fpx, fpy);
    inside[k] = !(pt.x >= sc.width || pt.x < 0.0f || pt.y >= sc.height || pt.y < 0.0f);
    int t = 0;
#pragma unroll
    for (int i = -5; i < 6; i += 2)
#pragma unroll
        for (int j = -5; j < 6; j += 2, ++t) out[(size_t)k * kTaps + t] = tap_sample(a.view[v].tex, H, fpx, fpy, i, j);
}

template <int SMAX, int WW>
cudaError_t launch_prop_t(const PMArgs &a, int iter, int color, cudaStream_t s)
{
    constexpr int WH = 32 / WW;
    const dim3 grid((a.W + 2 * WW - 1) / (2 * WW), (a.rows_cov + 2 * WH - 1) / (2 * WH)), b(kBlockX, kBlockY);
    k_prop_dirs<WW><<<grid, b, 0, s>>>(a, iter, color);
    if constexpr (WW == 8) { /* the ACMM+NESP variant runs the default tile */
        if (a.acmm) {
            k_prop_refine<SMAX, false, WW, true><<<grid, b, 0, s>>>(a, iter, color);
            return cudaGetLastError();
        }
    }
    if (a.proposals)
        k_prop_refine<SMAX, true, WW><<<grid, b, 0, s>>>(a, iter, color);
    else
        k_prop_refine<SMAX, false, WW><<<grid, b, 0, s>>>(a, iter, color);
    return cudaGetLastError();
}

template <int WW>
cudaError_t launch_prop_w(const PMArgs &a, int iter, int color, cudaStream_t s)
{
    const int S = a.n - 1;
    if (S <= 4) return launch_prop_t<4, WW>(a, iter, color, s);
    if (S <= 8) return launch_prop_t<8, WW>(a, iter, color, s);
    if (S <= 12) return launch_prop_t<12, WW>(a, iter, color, s);
    if (S <= 16) return launch_prop_t<16, WW>(a, iter, color, s);
    return launch_prop_t<kMaxSrc, WW>(a, iter, color, s);
}

}  // namespace

int rows_covered(int H)
{
    const int cov = 2 * (((H / 2) + 15) / 16) * 16;
    return cov < H ? cov : H;
}

cudaError_t launch_pair_geom(const PMArgs &a, PairGeom *out, cudaStream_t s)
{
    k_pair_geom<<<1, 64, 0, s>>>(a, out);
    return cudaGetLastError();
}

static dim3 pixel_grid(int W, int H) { return dim3((W + kBlockX - 1) / kBlockX, (H + kBlockY - 1) / kBlockY); }

cudaError_t launch_init(const PMArgs &a, cudaStream_t s)
{
    k_init<<<pixel_grid(a.W, a.H), dim3(kBlockX, kBlockY), 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_propagate(const PMArgs &a, int iter, int color, cudaStream_t s, int ww)
{
    if (a.rows_cov <= 0) return cudaSuccess;
    if (a.acmm) ww = 8; /* its refinement kernel exists for this tile only */
    switch (ww) {
    case 4: return launch_prop_w<4>(a, iter, color, s);
    case 8: return launch_prop_w<8>(a, iter, color, s);
    case 16: return launch_prop_w<16>(a, iter, color, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_depth_normal_filter(const PMArgs &a, float4 *planes, const float *costs, cudaStream_t s)
{
    dim3 b(16, 16), g((a.W + 15) / 16, (a.H + 15) / 16);
    k_depth_normal<<<g, b, 0, s>>>(a, planes);
    if (a.rows_cov > 0) {
        dim3 fb(32, 8), fg((a.W + 63) / 64, (a.rows_cov + 7) / 8);
        k_filter<<<fg, fb, 0, s>>>(a, planes, costs, 0);
        k_filter<<<fg, fb, 0, s>>>(a, planes, costs, 1);
    }
    return cudaGetLastError();
}

cudaError_t launch_cost_vectors(const PMArgs &a, const float4 *planes, float *out, cudaStream_t s)
{
    k_cost_vectors<<<pixel_grid(a.W, a.H), dim3(kBlockX, kBlockY), 0, s>>>(a, planes, out);
    return cudaGetLastError();
}

cudaError_t launch_initial_costs(const PMArgs &a, const float4 *planes, float *cost, uint32_t *views,
                                 cudaStream_t s)
{
    k_initial_costs<<<pixel_grid(a.W, a.H), dim3(kBlockX, kBlockY), 0, s>>>(a, planes, cost, views);
    return cudaGetLastError();
}

cudaError_t launch_tap_samples(const PMArgs &a, const float4 *planes, const int *pixels, int n, float *out,
                               int *inside, cudaStream_t s)
{
    const int total = n * (a.n - 1);
    if (total > 0) k_tap_samples<<<(total + 127) / 128, 128, 0, s>>>(a, planes, pixels, n, out, inside);
    return cudaGetLastError();
}

cudaError_t launch_geom_costs(const PMArgs &a, const float4 *planes, float *out, cudaStream_t s)
{
    dim3 b(16, 16), g((a.W + 15) / 16, (a.H + 15) / 16);
    k_geom_costs<<<g, b, 0, s>>>(a, planes, out);
    return cudaGetLastError();
}

}  // namespace hpm

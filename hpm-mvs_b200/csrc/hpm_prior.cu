/*
 * Planar-prior construction on the GPU (the host stages of the reference's
 * ProcessProblem, HPM-MVS/main.cpp:73-480, and HPM.cpp:759-1123).
 *
 *   k_resize          cv::resize INTER_LINEAR of depth / cost / normal maps
 *                     (main.cpp:84-86, 238-240)
 *   k_support_blocks  GetSupportPoints* (HPM.cpp:759-785, 1125-1179): argmin
 *                     cost per 5x5 block, kept when < 0.1
 *   k_tri_planes      GetPriorPlaneParams_factor (HPM.cpp:811-844)
 *   k_tri_raster      triangle raster of main.cpp:96-116 (later triangles win:
 *                     atomicMax on the triangle index)
 *   k_knn_prior       DepthsPredictSupplement (HPM.cpp:923-1097): exact 6
 *                     nearest support points from a uniform cell grid instead
 *                     of PCL's kd-tree on the host
 *   k_prior_coarse    prior depth + world normal at a coarse level
 *                     (main.cpp:124-162, 277-314)
 *   k_prior_reload    JBU output -> ref-frame prior planes (main.cpp:179-203)
 *   k_prior_full      full-scale prior planes, masks and prior depths
 *                     (main.cpp:426-454, HPM.cpp:1099-1123)
 *
 * Discrete decisions (raster pixel, collinearity test, depth range checks)
 * use round-to-nearest operations without fused multiply-adds, as the host
 * code they restate; plane fits run in double precision.
 */
#include "hpm_internal.h"
#include "hpm_prior.h"

namespace hpm {
namespace {

/* ---------------- resize ---------------- */

/* Source index pair and weight of output coordinate d (cv::resize
 * INTER_LINEAR for float data, as OpenCV 4.x computes it: the fraction is
 * taken in double precision and rounded once to float; edges clamp). */
__device__ __forceinline__ void resize_coef(int d, int sn, int dn, int &s0, int &s1, float &f)
{
    const double fd = (d + 0.5) * ((double)sn / dn) - 0.5;
    int s = (int)floor(fd);
    f = (float)(fd - s);
    if (s < 0) f = 0.0f, s = 0;
    if (s >= sn - 1) f = 0.0f, s = sn - 1;
    s0 = s;
    s1 = min(s + 1, sn - 1);
}

/* Each pass blends a + f * (b - a) with one fused multiply-add, rows first,
 * then columns; bit-exact with cv::resize (OpenCV 4.13) on float maps for
 * every ratio tried, 2:1 and 4:1 included. */
__global__ void k_resize(const float *__restrict__ src, int sw, int sh, int ch, float *__restrict__ dst, int dw,
                         int dh)
{
    const int dx = blockIdx.x * blockDim.x + threadIdx.x;
    const int dy = blockIdx.y * blockDim.y + threadIdx.y;
    if (dx >= dw || dy >= dh) return;
    int sx0, sx1, sy0, sy1;
    float fx, fy;
    resize_coef(dx, sw, dw, sx0, sx1, fx);
    resize_coef(dy, sh, dh, sy0, sy1, fy);
    for (int c = 0; c < ch; ++c) {
        const float a0 = src[((size_t)sy0 * sw + sx0) * ch + c], b0 = src[((size_t)sy0 * sw + sx1) * ch + c];
        const float a1 = src[((size_t)sy1 * sw + sx0) * ch + c], b1 = src[((size_t)sy1 * sw + sx1) * ch + c];
        const float r0 = __fmaf_rn(fx, __fsub_rn(b0, a0), a0);
        const float r1 = __fmaf_rn(fx, __fsub_rn(b1, a1), a1);
        dst[((size_t)dy * dw + dx) * ch + c] = __fmaf_rn(fy, __fsub_rn(r1, r0), r0);
    }
}

/* ---------------- support points ---------------- */

/* One thread per 5x5 block, blocks in the reference's column-major order
 * (HPM.cpp:765-766): out[b] = (x, y) or (-1, -1). */
__global__ void k_support_blocks(const float *__restrict__ costs, int w, int h, int nbr, int nb, int2 *__restrict__ out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int col = (b / nbr) * 5, row = (b % nbr) * 5;
    float min_cost = 2.0f;
    int tx = 0, ty = 0;
    const int cb = min(w, col + 5), rb = min(h, row + 5);
    for (int c = col; c < cb; ++c)
        for (int r = row; r < rb; ++r) {
            const float v = costs[(size_t)r * w + c];
            if (v < 2.0f && min_cost > v) {
                tx = c;
                ty = r;
                min_cost = v;
            }
        }
    out[b] = (min_cost < 0.1f) ? make_int2(tx, ty) : make_int2(-1, -1);
}

/* ---------------- plane fit ---------------- */

__device__ double det3(double a, double b, double c, double d, double e, double f, double g, double h, double i)
{
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

/* GetPriorPlaneParams_factor (HPM.cpp:811-844): plane n.X + w = 0 through the
 * three back-projected vertices, |n| = 1, w >= 0.  The null vector of the
 * 3x4 system (cv::SVD::solveZ in the reference) by cofactors. */
__device__ float4 plane_from_vertices(const HpmCamera &cam, const float *__restrict__ depth, int w, const int *v,
                                      float factor)
{
    double P[3][3];
    for (int k = 0; k < 3; ++k) {
        const int x = v[2 * k], y = v[2 * k + 1];
        const float d = depth[(size_t)y * w + x];
        const float X = __fdiv_rn(__fmul_rn(d, __fsub_rn((float)x, __fmul_rn(cam.K[2], factor))),
                                  __fmul_rn(cam.K[0], factor));
        const float Y = __fdiv_rn(__fmul_rn(d, __fsub_rn((float)y, __fmul_rn(cam.K[5], factor))),
                                  __fmul_rn(cam.K[4], factor));
        P[k][0] = X;
        P[k][1] = Y;
        P[k][2] = d;
    }
    double n[4];
    n[0] = det3(P[0][1], P[0][2], 1, P[1][1], P[1][2], 1, P[2][1], P[2][2], 1);
    n[1] = -det3(P[0][0], P[0][2], 1, P[1][0], P[1][2], 1, P[2][0], P[2][2], 1);
    n[2] = det3(P[0][0], P[0][1], 1, P[1][0], P[1][1], 1, P[2][0], P[2][1], 1);
    n[3] = -det3(P[0][0], P[0][1], P[0][2], P[1][0], P[1][1], P[1][2], P[2][0], P[2][1], P[2][2]);
    const double s = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + n[3] * n[3]);
    const float n4[4] = {(float)(n[0] / s), (float)(n[1] / s), (float)(n[2] / s), (float)(n[3] / s)};
    float norm2 = (float)sqrt((double)n4[0] * n4[0] + (double)n4[1] * n4[1] + (double)n4[2] * n4[2]);
    if (n4[3] < 0) norm2 = -norm2;
    return make_float4(n4[0] / norm2, n4[1] / norm2, n4[2] / norm2, n4[3] / norm2);
}

/* GetDepthFromPlaneParam_factor (HPM.cpp:846-849), IEEE without contraction. */
__device__ float depth_from_plane_f(const HpmCamera &c, float4 p, int x, int y, float f)
{
    const float num = __fmul_rn(-p.w, __fmul_rn(c.K[0], f));
    const float t0 = __fmul_rn(__fsub_rn((float)x, __fmul_rn(c.K[2], f)), p.x);
    const float t1 = __fmul_rn(__fmul_rn(__fdiv_rn(c.K[0], c.K[4]), __fsub_rn((float)y, __fmul_rn(c.K[5], f))), p.y);
    const float t2 = __fmul_rn(__fmul_rn(c.K[0], f), p.z);
    return __fdiv_rn(num, __fadd_rn(__fadd_rn(t0, t1), t2));
}

__global__ void k_tri_planes(HpmCamera cam, const float *__restrict__ depth, int w, const int *__restrict__ tris, int n,
                             float factor, float4 *__restrict__ planes)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int v[6];
    for (int k = 0; k < 6; ++k) v[k] = tris[6 * t + k];
    planes[t] = plane_from_vertices(cam, depth, w, v, factor);
}

/* Raster of main.cpp:96-116 for kept triangle t (id t+1).  The loops run in
 * float with the reference's mixed float/double expression; the largest id
 * wins a pixel, as sequential overwriting in triangle order does.
 *
 * One warp per triangle.  Both loop variables start at 0 and advance by the
 * same float step, so they walk the same sequence of partial sums: lane 0
 * writes it to shared memory once, and the lanes split the outer loop.  A
 * triangle whose sequence does not fit (an edge longer than kSeq pixels)
 * runs the reference's two loops on lane 0. */
constexpr int kSeq = 2048;

__device__ __forceinline__ void raster_px(const int *v, float p, float q, int w, int *ids, int id)
{
    const double rest = __dsub_rn(__dsub_rn(1.0, (double)p), (double)q);
    const double xs = __dadd_rn((double)__fadd_rn(__fmul_rn(p, (float)v[0]), __fmul_rn(q, (float)v[2])),
                                __dmul_rn(rest, (double)v[4]));
    const double ys = __dadd_rn((double)__fadd_rn(__fmul_rn(p, (float)v[1]), __fmul_rn(q, (float)v[3])),
                                __dmul_rn(rest, (double)v[5]));
    atomicMax(&ids[(size_t)(int)ys * w + (int)xs], id);
}

__global__ void __launch_bounds__(128) k_tri_raster(const int *__restrict__ tris, int n, int w, int *__restrict__ ids)
{
    __shared__ float seq_s[4][kSeq];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * 4 + warp;
    if (t >= n) return;
    const int *v = tris + 6 * t;
    const float L01 = (float)sqrt((double)(v[0] - v[2]) * (v[0] - v[2]) + (double)(v[1] - v[3]) * (v[1] - v[3]));
    const float L02 = (float)sqrt((double)(v[0] - v[4]) * (v[0] - v[4]) + (double)(v[1] - v[5]) * (v[1] - v[5]));
    const float L12 = (float)sqrt((double)(v[2] - v[4]) * (v[2] - v[4]) + (double)(v[3] - v[5]) * (v[3] - v[5]));
    const float mx = fmaxf(L01, fmaxf(L02, L12));
    const float step = (float)(1.0 / (double)mx);
    float *seq = seq_s[warp];
    int len = 0, fits = 1;
    if (lane == 0) {
        float p = 0;
        while ((double)p < 1.0 && len < kSeq) {
            seq[len++] = p;
            p = __fadd_rn(p, step);
        }
        fits = (double)p >= 1.0;
    }
    len = __shfl_sync(0xffffffffu, len, 0);
    fits = __shfl_sync(0xffffffffu, fits, 0);
    __syncwarp();
    if (!fits) {
        if (lane == 0)
            for (float p = 0; (double)p < 1.0; p = __fadd_rn(p, step))
                for (float q = 0; (double)q < 1.0 - (double)p; q = __fadd_rn(q, step)) raster_px(v, p, q, w, ids, t + 1);
        return;
    }
    for (int k = lane; k < len; k += 32) {
        const float p = seq[k];
        const double lim = 1.0 - (double)p;
        for (int m = 0; m < len && (double)seq[m] < lim; ++m) raster_px(v, p, seq[m], w, ids, t + 1);
    }
}

/* ---------------- kNN prior ---------------- */

__device__ float dist_f(int x1, int y1, int x2, int y2) /* Distance, HPM.cpp:923-926 */
{
    return __fsqrt_rn((float)((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2)));
}

__device__ bool not_on_line(int2 a, int2 b, int2 c) /* JudgeNotOnline, HPM.cpp:928-937 */
{
    const float l1 = dist_f(a.x, a.y, b.x, b.y);
    const float l2 = dist_f(a.x, a.y, c.x, c.y);
    const float l3 = dist_f(c.x, c.y, b.x, b.y);
    const float area = (float)(0.5 * (double)__fadd_rn(__fadd_rn(l1, l2), l3));
    return __fmul_rn(__fmul_rn(__fmul_rn(area, __fsub_rn(area, l1)), __fsub_rn(area, l2)), __fsub_rn(area, l3)) > 0;
}

/* triple order of HPM.cpp:982-1081 */
__constant__ unsigned char kTriples[20][3] = {{0, 1, 2}, {0, 1, 3}, {0, 1, 4}, {0, 2, 3}, {0, 2, 4}, {0, 3, 4},
                                              {1, 2, 3}, {1, 2, 4}, {1, 3, 4}, {2, 3, 4}, {0, 1, 5}, {0, 2, 5},
                                              {0, 3, 5}, {0, 4, 5}, {1, 2, 5}, {1, 3, 5}, {1, 4, 5}, {2, 3, 5},
                                              {2, 4, 5}, {3, 4, 5}};

/* The 6 support points nearest to (x, y) (squared distance, ties to the
 * lower point index): rings of cells of a uniform grid around the query's
 * cell, a ring searched only while it can still hold a point closer than the
 * current 6th.  Returns how many were found (fewer than 6 only when there
 * are fewer points); bi gets their indices nearest first. */
__device__ int knn6(int x, int y, const int2 *__restrict__ pts, const int *__restrict__ cell_start,
                    const int *__restrict__ cell_pts, int cell, int gw, int gh, int *bi)
{
    long long bd[6];
    int nb = 0;
    const int cx = min(x / cell, gw - 1), cy = min(y / cell, gh - 1);
    const int max_ring = max(gw, gh);
    for (int ring = 0; ring <= max_ring; ++ring) {
        if (nb == 6) {
            /* nearest possible distance of any point in this ring */
            const long long lim = (long long)(ring - 1) * cell;
            if (lim > 0 && lim * lim > bd[5]) break;
        }
        const int x0 = cx - ring, x1 = cx + ring, y0 = cy - ring, y1 = cy + ring;
        for (int gy = y0; gy <= y1; ++gy) {
            if (gy < 0 || gy >= gh) continue;
            const bool edge_row = (gy == y0 || gy == y1);
            for (int gx = x0; gx <= x1; gx += (edge_row ? 1 : (x1 - x0 > 0 ? x1 - x0 : 1))) {
                if (gx < 0 || gx >= gw) continue;
                const int cid = gy * gw + gx;
                for (int s = cell_start[cid]; s < cell_start[cid + 1]; ++s) {
                    const int k = cell_pts[s];
                    const long long dx = pts[k].x - x, dy = pts[k].y - y;
                    const long long d = dx * dx + dy * dy;
                    if (nb < 6 || d < bd[nb - 1] || (d == bd[nb - 1] && k < bi[nb - 1])) {
                        int pos = nb < 6 ? nb : 5;
                        while (pos > 0 && (bd[pos - 1] > d || (bd[pos - 1] == d && bi[pos - 1] > k))) {
                            bd[pos] = bd[pos - 1];
                            bi[pos] = bi[pos - 1];
                            pos--;
                        }
                        bd[pos] = d;
                        bi[pos] = k;
                        if (nb < 6) nb++;
                    }
                }
            }
        }
    }
    return nb;
}

/* One thread per pixel whose mask is <= 0: its 6 nearest support points
 * (knn6), then the first non-collinear triple, the plane fit and the
 * depth-range test of HPM.cpp:982-1093. */
__global__ void k_knn_prior(HpmCamera cam, const int2 *__restrict__ pts, const int *__restrict__ cell_start,
                            const int *__restrict__ cell_pts, int cell, int gw, int gh, const float *__restrict__ depth,
                            int w, int h, float factor, float dmin, float dmax, float *__restrict__ mask,
                            float4 *__restrict__ planes)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    if (mask[c] > 0) return;
    int bi[6];
    const int nb = knn6(x, y, pts, cell_start, cell_pts, cell, gw, gh, bi);
    if (nb < 6) return;
    int sel = -1;
    for (int t = 0; t < 20 && sel < 0; ++t)
        if (not_on_line(pts[bi[kTriples[t][0]]], pts[bi[kTriples[t][1]]], pts[bi[kTriples[t][2]]])) sel = t;
    if (sel < 0) return;
    int v[6];
    for (int k = 0; k < 3; ++k) {
        v[2 * k] = pts[bi[kTriples[sel][k]]].x;
        v[2 * k + 1] = pts[bi[kTriples[sel][k]]].y;
    }
    const float4 n4 = plane_from_vertices(cam, depth, w, v, factor);
    const float d = depth_from_plane_f(cam, n4, x, y, factor);
    if (d <= dmax && d >= dmin) {
        mask[c] = -233.0f;
        planes[c] = n4;
    }
}

/* The index sets alone: nn6[6 c + k] = k-th nearest support point of pixel c
 * (mask <= 0, or every pixel without a mask), -1 elsewhere or past the
 * number of points. */
__global__ void k_knn6_ids(const int2 *__restrict__ pts, const int *__restrict__ cell_start,
                           const int *__restrict__ cell_pts, int cell, int gw, int gh, int w, int h,
                           const float *__restrict__ mask, int *__restrict__ nn6)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    int bi[6] = {-1, -1, -1, -1, -1, -1};
    if (!mask || mask[c] <= 0) {
        const int nb = knn6(x, y, pts, cell_start, cell_pts, cell, gw, gh, bi);
        for (int k = nb; k < 6; ++k) bi[k] = -1;
    }
    for (int k = 0; k < 6; ++k) nn6[6 * c + k] = bi[k];
}

/* ---------------- prior assembly ---------------- */

__device__ float4 to_world(const HpmCamera &c, float4 h) /* TransformNormal, HPM.cpp:872-880 */
{
    float4 r;
    r.x = c.R[0] * h.x + c.R[3] * h.y + c.R[6] * h.z;
    r.y = c.R[1] * h.x + c.R[4] * h.y + c.R[7] * h.z;
    r.z = c.R[2] * h.x + c.R[5] * h.y + c.R[8] * h.z;
    r.w = h.w;
    return r;
}

/* Coarse level, main.cpp:124-162: prior depth and world normal (zero where
 * the mask ends up 0).  Triangle planes are range-checked against the
 * pass's range widened once more (x1.2 / x0.6, main.cpp:129; hi_widen /
 * lo_widen, 1 with fixed quirks), kNN planes against the pass's range. */
__global__ void k_prior_coarse(HpmCamera cam, int w, int h, float factor, float dmin, float dmax, float hi_widen,
                               float lo_widen, float *__restrict__ mask, const int *__restrict__ ids, const float4 *__restrict__ tri_planes,
                               const float4 *__restrict__ knn_planes, float *__restrict__ out_depth,
                               float *__restrict__ out_normal)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    float m = mask[c];
    float d = 0.0f;
    float4 n = make_float4(0, 0, 0, 0);
    if (m > 0) {
        const float4 p = tri_planes[ids[c] - 1];
        d = depth_from_plane_f(cam, p, x, y, factor);
        if (d <= __fmul_rn(dmax, hi_widen) && d >= __fmul_rn(dmin, lo_widen))
            n = to_world(cam, p);
        else
            m = 0, d = 0.0f;
    } else if (m < -200.0f) {
        const float4 p = knn_planes[c];
        d = depth_from_plane_f(cam, p, x, y, factor);
        if (d <= dmax && d >= dmin)
            n = to_world(cam, p);
        else
            m = 0, d = 0.0f;
    } else {
        m = 0;
    }
    mask[c] = m;
    out_depth[c] = d;
    out_normal[3 * c] = n.x;
    out_normal[3 * c + 1] = n.y;
    out_normal[3 * c + 2] = n.z;
}

/* main.cpp:179-203: upsampled prior -> ref-frame plane (n, dist) with the
 * full-resolution intrinsics (GetDistance2Origin_factor ignores its factor). */
__global__ void k_prior_reload(HpmCamera cam, int w, int h, float dmin, float dmax, const float *__restrict__ up_depth,
                               const float4 *__restrict__ up_normal, float4 *__restrict__ prior, uint32_t *__restrict__ masks)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    const float d = up_depth[c];
    if (d <= dmax && d >= dmin) {
        const float4 nw = up_normal[c];
        float4 t; /* TransformNormal2RefCam, HPM.cpp:882-890 */
        t.x = cam.R[0] * nw.x + cam.R[1] * nw.y + cam.R[2] * nw.z;
        t.y = cam.R[3] * nw.x + cam.R[4] * nw.y + cam.R[5] * nw.z;
        t.z = cam.R[6] * nw.x + cam.R[7] * nw.y + cam.R[8] * nw.z;
        const float X0 = d * (x - cam.K[2]) / cam.K[0];
        const float X1 = d * (y - cam.K[5]) / cam.K[4];
        t.w = -(t.x * X0 + t.y * X1 + t.z * d);
        prior[c] = t;
        masks[c] = 1u;
    } else {
        masks[c] = 0u;
    }
}

/* Full scale, main.cpp:426-454 and HPM.cpp:1099-1123: prior depth map,
 * planes and masks.  A kNN mask of -233.0f becomes (unsigned int)-233.0f:
 * non-zero, so the pixel carries a prior. */
__global__ void k_prior_full(HpmCamera cam, int w, int h, float dmin, float dmax, const float *__restrict__ mask,
                             const int *__restrict__ ids, const float4 *__restrict__ tri_planes,
                             const float4 *__restrict__ knn_planes, float *__restrict__ prior_depth,
                             float4 *__restrict__ prior, uint32_t *__restrict__ masks)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t c = (size_t)y * w + x;
    const float m = mask[c];
    float d = 0.0f;
    uint32_t mk = 0u;
    float4 p = make_float4(0, 0, 0, 0);
    if (m > 0) {
        p = tri_planes[ids[c] - 1];
        const float dd = depth_from_plane_f(cam, p, x, y, 1.0f);
        if (dd <= dmax && dd >= dmin) {
            d = dd;
            mk = (uint32_t)ids[c];
        }
    } else if (m < -200.0f) {
        p = knn_planes[c];
        const float dd = depth_from_plane_f(cam, p, x, y, 1.0f);
        if (dd <= dmax && dd >= dmin) {
            d = dd;
            mk = 0xFFFFFF17u; /* (unsigned int)-233.0f */
        }
    }
    prior_depth[c] = d;
    masks[c] = mk;
    prior[c] = mk ? p : make_float4(0, 0, 0, 0);
}

/* ids (int) -> reference mask values (float, id + 1.0 or 0) */
__global__ void k_ids_to_mask(const int *__restrict__ ids, int n, float *__restrict__ mask)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) mask[i] = (float)ids[i];
}

}  // namespace

static dim3 grid2(int w, int h) { return dim3((w + 15) / 16, (h + 15) / 16); }

cudaError_t prior_resize(const float *src, int sw, int sh, int ch, float *dst, int dw, int dh, cudaStream_t s)
{
    k_resize<<<grid2(dw, dh), dim3(16, 16), 0, s>>>(src, sw, sh, ch, dst, dw, dh);
    return cudaGetLastError();
}

cudaError_t prior_support_blocks(const float *costs, int w, int h, int2 *out, int *nblocks, cudaStream_t s)
{
    const int nbr = (h + 4) / 5, nbc = (w + 4) / 5, nb = nbr * nbc;
    *nblocks = nb;
    k_support_blocks<<<(nb + 255) / 256, 256, 0, s>>>(costs, w, h, nbr, nb, out);
    return cudaGetLastError();
}

cudaError_t prior_triangles(const HpmCamera &cam, const float *depth, int w, int h, const int *tris, int n,
                            float factor, float4 *planes, int *ids, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(ids, 0, sizeof(int) * (size_t)w * h, s);
    if (e != cudaSuccess || n == 0) return e;
    k_tri_planes<<<(n + 127) / 128, 128, 0, s>>>(cam, depth, w, tris, n, factor, planes);
    k_tri_raster<<<(n + 3) / 4, 128, 0, s>>>(tris, n, w, ids);
    return cudaGetLastError();
}

cudaError_t prior_raster(const int *tris, int n, int w, int *ids, cudaStream_t s)
{
    if (n > 0) k_tri_raster<<<(n + 3) / 4, 128, 0, s>>>(tris, n, w, ids);
    return cudaGetLastError();
}

cudaError_t prior_knn_ids(const int2 *pts, const int *cell_start, const int *cell_pts, int cell, int gw, int gh, int w,
                          int h, const float *mask, int *nn6, cudaStream_t s)
{
    k_knn6_ids<<<grid2(w, h), dim3(16, 16), 0, s>>>(pts, cell_start, cell_pts, cell, gw, gh, w, h, mask, nn6);
    return cudaGetLastError();
}

cudaError_t prior_ids_to_mask(const int *ids, int n, float *mask, cudaStream_t s)
{
    k_ids_to_mask<<<(n + 255) / 256, 256, 0, s>>>(ids, n, mask);
    return cudaGetLastError();
}

cudaError_t prior_knn(const HpmCamera &cam, const int2 *pts, const int *cell_start, const int *cell_pts, int cell,
                      int gw, int gh, const float *depth, int w, int h, float factor, float dmin, float dmax, float *mask,
                      float4 *planes, cudaStream_t s)
{
    k_knn_prior<<<grid2(w, h), dim3(16, 16), 0, s>>>(cam, pts, cell_start, cell_pts, cell, gw, gh, depth, w, h, factor,
                                                     dmin, dmax, mask, planes);
    return cudaGetLastError();
}

cudaError_t prior_coarse(const HpmCamera &cam, int w, int h, float factor, float dmin, float dmax, float *mask,
                         const int *ids, const float4 *tri_planes, const float4 *knn_planes, float *out_depth,
                         float *out_normal, cudaStream_t s, bool widen)
{
    k_prior_coarse<<<grid2(w, h), dim3(16, 16), 0, s>>>(cam, w, h, factor, dmin, dmax, widen ? 1.2f : 1.0f,
                                                        widen ? 0.6f : 1.0f, mask, ids, tri_planes, knn_planes,
                                                        out_depth, out_normal);
    return cudaGetLastError();
}

cudaError_t prior_reload(const HpmCamera &cam, int w, int h, float dmin, float dmax, const float *up_depth,
                         const float4 *up_normal, float4 *prior, uint32_t *masks, cudaStream_t s)
{
    k_prior_reload<<<grid2(w, h), dim3(16, 16), 0, s>>>(cam, w, h, dmin, dmax, up_depth, up_normal, prior, masks);
    return cudaGetLastError();
}

cudaError_t prior_full(const HpmCamera &cam, int w, int h, float dmin, float dmax, const float *mask, const int *ids,
                       const float4 *tri_planes, const float4 *knn_planes, float *prior_depth, float4 *prior,
                       uint32_t *masks, cudaStream_t s)
{
    k_prior_full<<<grid2(w, h), dim3(16, 16), 0, s>>>(cam, w, h, dmin, dmax, mask, ids, tri_planes, knn_planes,
                                                      prior_depth, prior, masks);
    return cudaGetLastError();
}

}  // namespace hpm

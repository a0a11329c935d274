/*
 * Fusion of the depth/normal maps of a scene into a coloured point cloud:
 * RunFusion (HPM-MVS/main.cpp:502-633) and StoreColorPlyFileBinaryPointCloud
 * (HPM-MVS/HPM.cpp:403-456).
 *
 * The reference fuses sequentially: views in problem order, pixels row by
 * row; a pixel consistent with at least one source (reprojection error < 2
 * px, relative depth difference < 1 %, normal angle < 10 degrees, mean
 * exp(-error) > 0.3) becomes a point and masks the source pixels it agreed
 * with, and masked pixels are skipped later, as references and as sources.
 * The list of agreeing source pixels (used_list) is declared per view, not
 * per pixel (main.cpp:557), so a point also masks source pixels that agreed
 * with earlier pixels of the same view.
 *
 * Everything that does not depend on the masks is computed on the GPU, one
 * thread per (reference pixel, source view): the world point, its
 * projection, the source pixel, the back-projection and the consistency
 * test, leaving for each pair the source pixel index (or -1) and its weight
 * exp(-error).  The order-dependent part, which only reads those pairs and
 * the masks, runs on the host in the reference's order.
 *
 * Arithmetic follows the reference's host code operation by operation
 * (round-to-nearest, no fused multiply-adds; the reprojection distance in
 * double as pow/sqrt promote it); acosf and expf are CUDA's.
 */
#include <cfloat>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "hpm_internal.h"
#include "hpm_nvtx.h"

namespace {

using hpm::kMaxSrc;

struct Cam {
    float K[9], R[9], t[3];
    int w, h;
};

Cam make_cam(const HpmCamera &c)
{
    Cam o;
    memcpy(o.K, c.K, sizeof(o.K));
    memcpy(o.R, c.R, sizeof(o.R));
    memcpy(o.t, c.t, sizeof(o.t));
    o.w = c.width;
    o.h = c.height;
    return o;
}

/* (int)f as the reference's x86 host code computes it: truncation, and the
 * "integer indefinite" INT_MIN for NaN and out-of-range values (CUDA's
 * conversion would give 0 for NaN, a pixel inside the image) */
__device__ __forceinline__ int host_int(float f)
{
    return (f != f || f >= 2147483648.0f || f < -2147483648.0f) ? INT_MIN : __float2int_rz(f);
}

__device__ __forceinline__ float m(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float ad(float a, float b) { return __fadd_rn(a, b); }

/* Get3DPointonWorld (HPM.cpp:210-234) */
__device__ void world_point(const Cam &c, int x, int y, float depth, float *X)
{
    const float px = __fdiv_rn(m(depth, __fsub_rn((float)x, c.K[2])), c.K[0]);
    const float py = __fdiv_rn(m(depth, __fsub_rn((float)y, c.K[5])), c.K[4]);
    const float pz = depth;
    const float *R = c.R, *t = c.t;
    const float tx = ad(ad(m(R[0], px), m(R[3], py)), m(R[6], pz));
    const float ty = ad(ad(m(R[1], px), m(R[4], py)), m(R[7], pz));
    const float tz = ad(ad(m(R[2], px), m(R[5], py)), m(R[8], pz));
    const float cx = -ad(ad(m(R[0], t[0]), m(R[3], t[1])), m(R[6], t[2]));
    const float cy = -ad(ad(m(R[1], t[0]), m(R[4], t[1])), m(R[7], t[2]));
    const float cz = -ad(ad(m(R[2], t[0]), m(R[5], t[1])), m(R[8], t[2]));
    X[0] = ad(tx, cx);
    X[1] = ad(ty, cy);
    X[2] = ad(tz, cz);
}

/* ProjectonCamera (HPM.cpp:247-257) */
__device__ void project(const float *X, const Cam &c, float *pt, float *depth)
{
    const float *R = c.R, *K = c.K, *t = c.t;
    const float x = ad(ad(ad(m(R[0], X[0]), m(R[1], X[1])), m(R[2], X[2])), t[0]);
    const float y = ad(ad(ad(m(R[3], X[0]), m(R[4], X[1])), m(R[5], X[2])), t[1]);
    const float z = ad(ad(ad(m(R[6], X[0]), m(R[7], X[1])), m(R[8], X[2])), t[2]);
    const float d = ad(ad(m(K[6], x), m(K[7], y)), m(K[8], z));
    *depth = d;
    pt[0] = __fdiv_rn(ad(ad(m(K[0], x), m(K[1], y)), m(K[2], z)), d);
    pt[1] = __fdiv_rn(ad(ad(m(K[3], x), m(K[4], y)), m(K[5], z)), d);
}

struct FuseArgs {
    Cam ref;
    Cam src[kMaxSrc];
    const float *ref_depth, *ref_normal;
    const float *src_depth[kMaxSrc];
    const float *src_normal[kMaxSrc];
    int ns;
    int *pair_src;     /* [pixel][ns] source pixel index, or -1 */
    float *pair_w;     /* [pixel][ns] exp(-error) */
    float *point;      /* [pixel][3] world point */
};

/* One thread per (reference pixel, source view): main.cpp:565-612 without
 * the masks. */
__global__ void k_fuse_pairs(const __grid_constant__ FuseArgs a, int npx)
{
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)npx * a.ns) return;
    const int p = (int)(gid / a.ns), j = (int)(gid % a.ns);
    const int cols = a.ref.w;
    const int r = p / cols, c = p % cols;
    const float ref_depth = a.ref_depth[p];
    a.pair_src[gid] = -1;
    a.pair_w[gid] = 0.0f;
    if (ref_depth <= 0.0f) return; /* main.cpp:562-563; a NaN depth goes on, as in the reference */
    float X[3];
    world_point(a.ref, c, r, ref_depth, X);
    if (j == 0) {
        a.point[3 * (size_t)p] = X[0];
        a.point[3 * (size_t)p + 1] = X[1];
        a.point[3 * (size_t)p + 2] = X[2];
    }
    const Cam &s = a.src[j];
    float pt[2], proj_depth;
    project(X, s, pt, &proj_depth);
    const int sr = host_int(ad(pt[1], 0.5f)), sc = host_int(ad(pt[0], 0.5f));
    if (!(sc >= 0 && sc < s.w && sr >= 0 && sr < s.h)) return;
    const size_t sp = (size_t)sr * s.w + sc;
    const float src_depth = a.src_depth[j][sp];
    if (src_depth <= 0.0f) return;
    float Y[3], tp[2];
    world_point(s, sc, sr, src_depth, Y);
    project(Y, a.ref, tp, &proj_depth);
    const double dx = (double)__fsub_rn((float)c, tp[0]), dy = (double)__fsub_rn((float)r, tp[1]);
    const float reproj = (float)sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    const float rel = __fdiv_rn(fabsf(__fsub_rn(proj_depth, ref_depth)), ref_depth);
    const float *rn = a.ref_normal + 3 * (size_t)p, *sn = a.src_normal[j] + 3 * sp;
    const float dot = ad(ad(m(rn[0], sn[0]), m(rn[1], sn[1])), m(rn[2], sn[2]));
    float ang = acosf(dot);
    if (ang != ang) ang = 0.0f; /* GetAngle, HPM.cpp:259-268 */
    if (reproj < 2.0f && rel < 0.01f && ang < 0.174533f) {
        const float idx = ad(ad(reproj, m(200.0f, rel)), m(ang, 10.0f));
        a.pair_src[gid] = (int)sp;
        a.pair_w[gid] = expf(-idx);
    }
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * (n ? n : 1)); }
};

/* What the ordered pass reads of a view besides the pairs (host memory). */
struct PassView {
    HpmCamera cam;
    const float *depth;   /* the ACMM+NESP rule only */
    const float *normal;  /* 3 floats per pixel */
    const uint8_t *color; /* B, G, R */
};

/* Get3DPointonWorld (HPM.cpp:210-234, ACMM.cpp:187-211) on the host: the
 * float operations of world_point above, in order (the x86-64 host build
 * has no fused multiply-add). */
void host_world_point(const HpmCamera &c, int x, int y, float depth, float *X)
{
    const float px = depth * ((float)x - c.K[2]) / c.K[0];
    const float py = depth * ((float)y - c.K[5]) / c.K[4];
    const float pz = depth;
    const float *R = c.R, *t = c.t;
    const float tx = R[0] * px + R[3] * py + R[6] * pz;
    const float ty = R[1] * px + R[4] * py + R[7] * pz;
    const float tz = R[2] * px + R[5] * py + R[8] * pz;
    const float cx = -(R[0] * t[0] + R[3] * t[1] + R[6] * t[2]);
    const float cy = -(R[1] * t[0] + R[4] * t[1] + R[7] * t[2]);
    const float cz = -(R[2] * t[0] + R[5] * t[1] + R[8] * t[2]);
    X[0] = tx + cx;
    X[1] = ty + cy;
    X[2] = tz + cz;
}

/* The order-dependent half of RunFusion for one problem (reference view i,
 * sources srcs), reading the pairs of the GPU pass and the masks in the
 * reference's order.  rule 0: HPM-MVS (main.cpp:553-620): a pixel with at
 * least one agreeing source whose mean exp(-error) exceeds 0.3 gives its own
 * point, normal and colour.  rule 1: the ACMM+NESP variant
 * (ACMM+NESP/windows/main.cpp:205-292): a pixel with at least 2 agreeing
 * sources gives the mean point, normal and colour over it and those source
 * pixels (cv::Vec3f /= divides by multiplying with the float reciprocal,
 * OpenCV core/matx.hpp; the PLY writer truncates colours,
 * ACMM.cpp:395-397).  Either way the accepted pixel masks the source pixels
 * recorded in the per-view used list (main.cpp:557). */
void ordered_problem(int rule, int i, int ns, const int *srcs, const std::vector<PassView> &views,
                     std::vector<std::vector<uint8_t>> &masks, const int *h_src, const float *h_w, const float *h_pt,
                     float *out_xyz, float *out_normal, uint8_t *out_bgr, long long cap, long long &n_out)
{
    const PassView &ref = views[i];
    const size_t npx = (size_t)ref.cam.width * ref.cam.height;
    int used[kMaxSrc];
    uint8_t *msrc[kMaxSrc];
    for (int j = 0; j < ns; ++j) {
        used[j] = -1;
        msrc[j] = masks[srcs[j]].data();
    }
    std::vector<uint8_t> &mi = masks[i];
    for (size_t p = 0; p < npx; ++p) {
        if (mi[p] == 1) continue;
        const int *ps = &h_src[p * ns];
        const float *pw = &h_w[p * ns];
        int num = 0;
        float dyn = 0.0f;
        float sp[3], sn[3], sc[3]; /* the variant's sums: point, normal, colour */
        if (rule == 1)
            for (int k = 0; k < 3; ++k) {
                sp[k] = h_pt[3 * p + k];
                sn[k] = ref.normal[3 * p + k];
                sc[k] = (float)ref.color[3 * p + k];
            }
        for (int j = 0; j < ns; ++j) {
            if (ps[j] < 0) continue;
            if (msrc[j][ps[j]] == 1) continue;
            if (rule == 1) {
                const PassView &s = views[srcs[j]];
                const int sx = ps[j] % s.cam.width, sy = ps[j] / s.cam.width;
                float Y[3];
                host_world_point(s.cam, sx, sy, s.depth[ps[j]], Y);
                for (int k = 0; k < 3; ++k) {
                    sp[k] += Y[k];
                    sn[k] = sn[k] + s.normal[3 * (size_t)ps[j] + k];
                    sc[k] += (float)s.color[3 * (size_t)ps[j] + k];
                }
            }
            used[j] = ps[j];
            dyn += pw[j];
            num++;
        }
        if (rule == 1 ? num < 2 : !(num >= 1 && (dyn > 0.3 * num))) continue;
        if (n_out < cap) {
            if (rule == 1) {
                const float div = num + 1.0f, inv = 1.f / div;
                for (int k = 0; k < 3; ++k) {
                    if (out_xyz) out_xyz[3 * n_out + k] = sp[k] / div;
                    if (out_normal) out_normal[3 * n_out + k] = sn[k] * inv;
                    if (out_bgr) out_bgr[3 * n_out + k] = (uint8_t)(int)(sc[k] / div);
                }
            } else {
                if (out_xyz) memcpy(out_xyz + 3 * n_out, &h_pt[3 * p], 3 * sizeof(float));
                if (out_normal) memcpy(out_normal + 3 * n_out, &ref.normal[3 * p], 3 * sizeof(float));
                if (out_bgr) memcpy(out_bgr + 3 * n_out, &ref.color[3 * p], 3);
            }
        }
        n_out++;
        for (int j = 0; j < ns; ++j)
            if (used[j] != -1) msrc[j][used[j]] = 1;
    }
}

/* hpm_fuse's argument checks (problems as hpm_run_scene's) */
bool fuse_args_ok(int n_views, const HpmCamera *cams, const float *const *depths, const float *const *normals,
                  const uint8_t *const *colors, int n_problems, const int *ref_ids, const int *src_counts,
                  const int *src_ids, long long cap, long long *n_points)
{
    if (!cams || !depths || !normals || !colors || !ref_ids || !src_counts || !src_ids || !n_points || n_views < 1 ||
        n_problems < 0 || cap < 0)
        return false;
    for (int v = 0; v < n_views; ++v)
        if (!depths[v] || !normals[v] || !colors[v] || cams[v].width < 1 || cams[v].height < 1) return false;
    for (int p = 0; p < n_problems; ++p) {
        if (ref_ids[p] < 0 || ref_ids[p] >= n_views || src_counts[p] < 0 || src_counts[p] > kMaxSrc) return false;
        for (int j = 0; j < src_counts[p]; ++j)
            if (src_ids[p * kMaxSrc + j] < 0 || src_ids[p * kMaxSrc + j] >= n_views) return false;
    }
    return true;
}

int fuse_impl(int rule, int device, int n_views, const HpmCamera *cams, const float *const *depths,
              const float *const *normals, const uint8_t *const *colors, int n_problems, const int *ref_ids,
              const int *src_counts, const int *src_ids, float *out_xyz, float *out_normal, uint8_t *out_bgr,
              long long cap, long long *n_points);

}  // namespace

extern "C" int hpm_fuse(int device, int n_views, const HpmCamera *cams, const float *const *depths,
                        const float *const *normals, const uint8_t *const *colors, int n_problems,
                        const int *ref_ids, const int *src_counts, const int *src_ids, float *out_xyz,
                        float *out_normal, uint8_t *out_bgr, long long cap, long long *n_points)
{
    return fuse_impl(0, device, n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids,
                     out_xyz, out_normal, out_bgr, cap, n_points);
}

extern "C" int hpm_fuse_acmm(int device, int n_views, const HpmCamera *cams, const float *const *depths,
                             const float *const *normals, const uint8_t *const *colors, int n_problems,
                             const int *ref_ids, const int *src_counts, const int *src_ids, float *out_xyz,
                             float *out_normal, uint8_t *out_bgr, long long cap, long long *n_points)
{
    return fuse_impl(1, device, n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids,
                     out_xyz, out_normal, out_bgr, cap, n_points);
}

extern "C" int hpm_fuse_pass(int rule, int n_views, const HpmCamera *cams, const float *const *depths,
                             const float *const *normals, const uint8_t *const *colors, int n_problems,
                             const int *ref_ids, const int *src_counts, const int *src_ids,
                             const int *const *pair_src, const float *const *pair_w, const float *const *points,
                             float *out_xyz, float *out_normal, uint8_t *out_bgr, long long cap,
                             long long *n_points)
{
    if ((rule != 0 && rule != 1) || !pair_src || !pair_w || !points ||
        !fuse_args_ok(n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids, cap,
                      n_points))
        return HPM_ERR_ARG;
    for (int p = 0; p < n_problems; ++p)
        if (src_counts[p] > 0 && (!pair_src[p] || !pair_w[p] || !points[p])) return HPM_ERR_ARG;
    std::vector<PassView> views(n_views);
    std::vector<std::vector<uint8_t>> masks(n_views);
    for (int v = 0; v < n_views; ++v) {
        views[v] = {cams[v], depths[v], normals[v], colors[v]};
        masks[v].assign((size_t)cams[v].width * cams[v].height, 0);
    }
    long long n_out = 0;
    for (int p = 0; p < n_problems; ++p)
        if (src_counts[p] > 0)
            ordered_problem(rule, ref_ids[p], src_counts[p], src_ids + p * kMaxSrc, views, masks, pair_src[p],
                            pair_w[p], points[p], out_xyz, out_normal, out_bgr, cap, n_out);
    *n_points = n_out;
    return HPM_OK;
}

namespace {

int fuse_impl(int rule, int device, int n_views, const HpmCamera *cams, const float *const *depths,
              const float *const *normals, const uint8_t *const *colors, int n_problems, const int *ref_ids,
              const int *src_counts, const int *src_ids, float *out_xyz, float *out_normal, uint8_t *out_bgr,
              long long cap, long long *n_points)
{
    if (!fuse_args_ok(n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids, cap,
                      n_points))
        return HPM_ERR_ARG;

    if (cudaSetDevice(device) != cudaSuccess) return HPM_ERR_CUDA;
    const hpm::Range range("fusion %d problems", n_problems);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return HPM_ERR_CUDA;
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } guard{st};
#define FCK(x)                                       \
    do {                                             \
        if ((x) != cudaSuccess) return HPM_ERR_CUDA; \
    } while (0)
    /* the maps on the device (inputs may be host or device memory) and on
     * the host (the sequential pass reads colours and normals of points) */
    std::vector<DevBuf<float>> d_depth(n_views), d_normal(n_views);
    std::vector<std::vector<float>> h_normal(n_views), h_depth(n_views);
    std::vector<std::vector<uint8_t>> h_color(n_views);
    std::vector<std::vector<uint8_t>> masks(n_views);
    size_t max_px = 0;
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height;
        max_px = np > max_px ? np : max_px;
        FCK(d_depth[v].alloc(np));
        FCK(d_normal[v].alloc(3 * np));
        FCK(cudaMemcpyAsync(d_depth[v].p, depths[v], sizeof(float) * np, cudaMemcpyDefault, st));
        FCK(cudaMemcpyAsync(d_normal[v].p, normals[v], sizeof(float) * 3 * np, cudaMemcpyDefault, st));
        h_normal[v].resize(3 * np);
        h_color[v].resize(3 * np);
        FCK(cudaMemcpyAsync(h_normal[v].data(), normals[v], sizeof(float) * 3 * np, cudaMemcpyDefault, st));
        FCK(cudaMemcpyAsync(h_color[v].data(), colors[v], 3 * np, cudaMemcpyDefault, st));
        if (rule == 1) { /* the variant also averages the agreeing source points */
            h_depth[v].resize(np);
            FCK(cudaMemcpyAsync(h_depth[v].data(), depths[v], sizeof(float) * np, cudaMemcpyDefault, st));
        }
        masks[v].assign(np, 0);
    }
    FCK(cudaStreamSynchronize(st));
    std::vector<PassView> views(n_views);
    for (int v = 0; v < n_views; ++v)
        views[v] = {cams[v], rule == 1 ? h_depth[v].data() : nullptr, h_normal[v].data(), h_color[v].data()};
    int max_ns = 1;
    for (int p = 0; p < n_problems; ++p) max_ns = src_counts[p] > max_ns ? src_counts[p] : max_ns;
    /* Two slots of pair data.  A producer thread runs the kernel of problem
     * p + 1 and copies its pairs to the host (pageable memory, so each copy
     * holds its thread until done) while this thread runs problem p's
     * ordered pass. */
    struct Slot {
        DevBuf<int> d_src;
        DevBuf<float> d_w, d_pt;
        std::vector<int> h_src;
        std::vector<float> h_w, h_pt;
    } slots[2];
    for (Slot &sl : slots) {
        FCK(sl.d_src.alloc(max_px * max_ns));
        FCK(sl.d_w.alloc(max_px * max_ns));
        FCK(sl.d_pt.alloc(3 * max_px));
        sl.h_src.resize(max_px * max_ns);
        sl.h_w.resize(max_px * max_ns);
        sl.h_pt.resize(3 * max_px);
    }
    auto produce = [&](int pi, Slot &sl) -> int {
        const int i = ref_ids[pi], ns = src_counts[pi];
        const size_t npx = (size_t)cams[i].width * cams[i].height;
        FuseArgs a;
        memset(&a, 0, sizeof(a));
        a.ref = make_cam(cams[i]);
        a.ns = ns;
        a.ref_depth = d_depth[i].p;
        a.ref_normal = d_normal[i].p;
        for (int j = 0; j < ns; ++j) {
            const int s = src_ids[pi * kMaxSrc + j];
            a.src[j] = make_cam(cams[s]);
            a.src_depth[j] = d_depth[s].p;
            a.src_normal[j] = d_normal[s].p;
        }
        a.pair_src = sl.d_src.p;
        a.pair_w = sl.d_w.p;
        a.point = sl.d_pt.p;
        if (ns > 0) {
            const long long total = (long long)npx * ns;
            k_fuse_pairs<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, (int)npx);
            FCK(cudaGetLastError());
            FCK(cudaMemcpyAsync(sl.h_src.data(), sl.d_src.p, sizeof(int) * total, cudaMemcpyDeviceToHost, st));
            FCK(cudaMemcpyAsync(sl.h_w.data(), sl.d_w.p, sizeof(float) * total, cudaMemcpyDeviceToHost, st));
            FCK(cudaMemcpyAsync(sl.h_pt.data(), sl.d_pt.p, sizeof(float) * 3 * npx, cudaMemcpyDeviceToHost, st));
        }
        FCK(cudaStreamSynchronize(st));
        return HPM_OK;
    };
    std::mutex mu;
    std::condition_variable cv;
    int ready[2] = {-1, -1}; /* problem whose pairs a slot holds, -1 while free */
    bool stop = false;
    int produce_rc = HPM_OK;
    std::thread producer([&] {
        const int rc0 = cudaSetDevice(device) == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
        for (int pi = 0; pi < n_problems; ++pi) {
            const int k = pi & 1;
            {
                std::unique_lock<std::mutex> l(mu);
                cv.wait(l, [&] { return ready[k] == -1 || stop; });
                if (stop) return;
            }
            const int rc = rc0 ? rc0 : produce(pi, slots[k]);
            {
                std::lock_guard<std::mutex> l(mu);
                if (rc) produce_rc = rc;
                else ready[k] = pi;
            }
            cv.notify_all();
            if (rc) return;
        }
    });
    struct Joiner {
        std::thread &t;
        std::mutex &mu;
        std::condition_variable &cv;
        bool &stop;
        ~Joiner()
        {
            {
                std::lock_guard<std::mutex> l(mu);
                stop = true;
            }
            cv.notify_all();
            t.join();
        }
    } joiner{producer, mu, cv, stop};
    long long n_out = 0;
    for (int pi = 0; pi < n_problems; ++pi) {
        const int i = ref_ids[pi], ns = src_counts[pi];
        const int k = pi & 1;
        {
            std::unique_lock<std::mutex> l(mu);
            cv.wait(l, [&] { return ready[k] == pi || produce_rc != HPM_OK; });
            if (ready[k] != pi) return produce_rc;
        }
        struct Release {
            int &slot;
            std::mutex &mu;
            std::condition_variable &cv;
            ~Release()
            {
                {
                    std::lock_guard<std::mutex> l(mu);
                    slot = -1;
                }
                cv.notify_all();
            }
        } release{ready[k], mu, cv};
        if (ns == 0) continue; /* no source: no pixel can be consistent */
        ordered_problem(rule, i, ns, src_ids + pi * kMaxSrc, views, masks, slots[k].h_src.data(),
                        slots[k].h_w.data(), slots[k].h_pt.data(), out_xyz, out_normal, out_bgr, cap, n_out);
    }
#undef FCK
    *n_points = n_out;
    return HPM_OK;
}

}  // namespace

extern "C" int hpm_write_ply(const char *path, long long n, const float *xyz, const float *normal, const uint8_t *bgr)
{
    if (!path || n < 0 || (n > 0 && (!xyz || !normal || !bgr))) return HPM_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return HPM_ERR_IO;
    fprintf(f, "ply\nformat binary_little_endian 1.0\nelement vertex %d\n", (int)n);
    fprintf(f, "property float x\nproperty float y\nproperty float z\n");
    fprintf(f, "property float nx\nproperty float ny\nproperty float nz\n");
    fprintf(f, "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n");
    bool ok = true;
    for (long long k = 0; k < n && ok; ++k) {
        float X[3] = {xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]};
        /* non-finite coordinates are written as the origin (HPM.cpp:431-435) */
        if (!(X[0] < FLT_MAX && X[0] > -FLT_MAX) || !(X[1] < FLT_MAX && X[1] > -FLT_MAX) ||
            !(X[2] < FLT_MAX && X[2] >= -FLT_MAX))
            X[0] = X[1] = X[2] = 0.0f;
        unsigned char rec[27];
        memcpy(rec, X, 12);
        memcpy(rec + 12, normal + 3 * k, 12);
        rec[24] = bgr[3 * k + 2]; /* red */
        rec[25] = bgr[3 * k + 1]; /* green */
        rec[26] = bgr[3 * k];     /* blue */
        ok = fwrite(rec, 1, 27, f) == 27;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? HPM_OK : HPM_ERR_IO;
}

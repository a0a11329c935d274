/*
 * The ACMM+NESP variant's scene flow (ACMM+NESP/windows/main.cpp:299-384,
 * minus fusion) on the device: NESP propagation inside ACMM's coarse-to-fine
 * image pyramid.
 *
 * Per scale, every view is resized on the device from its full-size image
 * (k_resize, bit-exact with cv::resize INTER_LINEAR on float images); the
 * depth, normal and cost maps of every view stay in HBM from pass to pass
 * (the reference writes and reads .dmb files); between scales the last
 * geometric depth map and the normals are upsampled together by one JBU
 * launch (their weights are the same: main.cpp:126-152 for the depth,
 * ACMM.cu:538-596 for the normals).  The passes are the context's own
 * (hpm_run_patchmatch with HpmParams.variant 1).
 */
#include <cmath>
#include <cstring>
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

constexpr int kMaxImageSize = 3200; /* PatchMatchParams::max_image_size, ACMM.h:34 */

/* A view at one scale: its size and camera (InuputInitialization,
 * ACMM.cpp:489-516: resized to fit cur x cur unless it already fits, K
 * scaled by the new/old size ratios, all in float as the reference). */
struct ScaledView {
    int w, h;
    HpmCamera cam;
};

ScaledView scale_view(const HpmCamera &full, int cur)
{
    ScaledView s{full.width, full.height, full};
    if (full.width <= cur && full.height <= cur) return s;
    const float fx = static_cast<float>(cur) / full.width, fy = static_cast<float>(cur) / full.height;
    const float factor = fx < fy ? fx : fy;
    s.w = (int)std::round(full.width * factor);
    s.h = (int)std::round(full.height * factor);
    const float sx = s.w / static_cast<float>(full.width), sy = s.h / static_cast<float>(full.height);
    s.cam.K[0] *= sx;
    s.cam.K[2] *= sx;
    s.cam.K[4] *= sy;
    s.cam.K[5] *= sy;
    s.cam.width = s.w;
    s.cam.height = s.h;
    return s;
}

/* Per-view maps, at the view's current scale, carved from the context's
 * scene arena: the resized image, depths.dmb, depths_geom.dmb, normals.dmb
 * (3 floats per pixel), costs.dmb. */
struct AcmmMaps {
    std::vector<float *> img, depth, depth_g, normal, cost;
    std::vector<ScaledView> at;
    float4 *coarse = nullptr, *up_normal = nullptr; /* JBU input and output */
    float *up_depth = nullptr;
};

}  // namespace

extern "C" int hpm_run_scene_acmm(hpm_ctx *c, int n_views, const float *const *images, const HpmCamera *cams,
                                  int n_problems, const int *ref_ids, const int *src_counts, const int *src_ids,
                                  const HpmAcmmOpts *o, float *const *out_depths, float *const *out_normals,
                                  float *const *out_costs)
{
    if (!c || !images || !cams || !ref_ids || !src_counts || !src_ids || !o) return HPM_ERR_ARG;
    if (n_views < 2 || n_problems != n_views)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: %d views and %d problems (one problem per view)",
                        n_views, n_problems);
    for (int p = 0; p < n_problems; ++p) {
        if (ref_ids[p] != p)
            return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: problem %d must have reference view %d", p, p);
        if (src_counts[p] < 1 || src_counts[p] > kMaxSrc)
            return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: problem %d has %d sources", p, src_counts[p]);
        for (int j = 0; j < src_counts[p]; ++j) {
            const int s = src_ids[p * kMaxSrc + j];
            if (s < 0 || s >= n_views)
                return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: problem %d source %d", p, s);
        }
    }
    for (int v = 0; v < n_views; ++v)
        if (!images[v] || cams[v].width < 1 || cams[v].height < 1 || cams[v].width > kMaxImageSize ||
            cams[v].height > kMaxImageSize)
            return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: view %d is %dx%d (at most %d a side)", v,
                            cams[v].width, cams[v].height, kMaxImageSize);
    if (o->geom_iterations < 0 || o->geom_iterations > 16 || o->size_bound < 0 || o->max_iterations < 0 ||
        o->max_iterations > 64 || o->geom_max_iterations < 0 || o->geom_max_iterations > 64)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: options out of range");
    int r = ctx_select_device(c);
    if (r) return r;
    const int size_bound = o->size_bound > 0 ? o->size_bound : 1000; /* main.cpp:38 */
    const int iters = o->max_iterations > 0 ? o->max_iterations : 3;
    const int geom_iters = o->geom_max_iterations > 0 ? o->geom_max_iterations : 2;
    cudaStream_t s = c->stream;

    /* ComputeMultiScaleSettings (main.cpp:35-71) */
    std::vector<int> max_size(n_views), nd(n_views), cur(n_views, 0);
    int max_down = -1;
    for (int v = 0; v < n_views; ++v) {
        int m = cams[v].width > cams[v].height ? cams[v].width : cams[v].height;
        max_size[v] = m;
        int k = 0;
        while (m > size_bound) {
            m /= 2;
            k++;
        }
        nd[v] = k;
        if (k > max_down) max_down = k;
    }
    if (max_down > 0 && o->geom_iterations < 1)
        return ctx_fail(c, HPM_ERR_ARG, "hpm_run_scene_acmm: the finer scales start from the geometric maps "
                                        "(geom_iterations >= 1)");
    const Range range("ACMM+NESP scene %d views, %d scales", n_views, max_down + 1);

    /* arena: per view the full image and five maps at full size (a view's
     * scales only grow), and the JBU's buffers at the largest size */
    AcmmMaps m;
    size_t total = 0, largest = 0;
    auto st = [](size_t np) { return (np + 63) & ~(size_t)63; };
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height;
        total += 8 * st(np);
        if (np > largest) largest = np;
    }
    total += 9 * st(largest);
    CK(ctx_scene_arena(c, total * sizeof(float)), "scene buffers");
    float *base = ctx_scene_base(c);
    std::vector<float *> full(n_views);
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)cams[v].width * cams[v].height, sp = st(np);
        full[v] = base;
        m.img.push_back(base + sp);
        m.depth.push_back(base + 2 * sp);
        m.depth_g.push_back(base + 3 * sp);
        m.normal.push_back(base + 4 * sp);
        m.cost.push_back(base + 7 * sp);
        base += 8 * sp;
        CK(cudaMemcpyAsync(full[v], images[v], sizeof(float) * np, cudaMemcpyDefault, s), "scene images");
    }
    m.coarse = reinterpret_cast<float4 *>(base);
    m.up_normal = reinterpret_cast<float4 *>(base + 4 * st(largest));
    m.up_depth = base + 8 * st(largest);
    m.at.resize(n_views);

    std::vector<int> pass_no(n_views, 0);
    /* one pass of problem p on the context: its views at their current
     * scales, the pass's parameters, then the maps out of the state */
    auto load = [&](int p) -> int {
        const float *pimg[kMaxViews];
        HpmCamera pcam[kMaxViews];
        pimg[0] = m.img[p];
        pcam[0] = m.at[p].cam;
        for (int j = 0; j < src_counts[p]; ++j) {
            const int sv = src_ids[p * kMaxSrc + j];
            pimg[j + 1] = m.img[sv];
            pcam[j + 1] = m.at[sv].cam;
        }
        return hpm_set_views(c, pimg, pcam, src_counts[p] + 1);
    };
    auto params = [&](int p, int max_it) {
        HpmParams pp;
        hpm_default_params(&pp);
        pp.depth_min = cams[p].depth_min * 0.6f; /* ACMM.cpp:518-519 */
        pp.depth_max = cams[p].depth_max * 1.2f;
        pp.seed = o->seed + 7919ull * (uint64_t)p + (uint64_t)pass_no[p]++;
        pp.variant = 1;
        pp.max_iterations = max_it;
        return pp;
    };
    /* ProcessProblem's outputs (main.cpp:96-121): depth to depths.dmb or
     * depths_geom.dmb, normals.dmb, costs.dmb */
    auto store = [&](int p, bool geom) -> int {
        const size_t np = (size_t)m.at[p].w * m.at[p].h;
        CK(flow_split_state(reinterpret_cast<const float4 *>(ctx_planes(c)), (int)np,
                            geom ? m.depth_g[p] : m.depth[p], m.normal[p], s),
           "maps");
        CK(cudaMemcpyAsync(m.cost[p], ctx_costs(c), sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
        return HPM_OK;
    };
    auto plain = [&](int p) -> int {
        int rr = load(p);
        if (rr) return rr;
        const HpmParams pp = params(p, iters);
        rr = hpm_run_patchmatch(c, &pp);
        return rr ? rr : store(p, false);
    };
    auto geometric = [&](int p, bool multi) -> int {
        int rr = load(p);
        if (rr) return rr;
        std::vector<float *> &src = multi ? m.depth_g : m.depth;
        const float *pdep[kMaxViews];
        pdep[0] = src[p];
        for (int j = 0; j < src_counts[p]; ++j) pdep[j + 1] = src[src_ids[p * kMaxSrc + j]];
        rr = hpm_set_geom_depths(c, pdep);
        if (rr) return rr;
        const size_t np = (size_t)m.at[p].w * m.at[p].h;
        /* ACMM.cpp:636-660: the previous depth (suffix), normals and costs */
        CK(flow_pack4(src[p], m.normal[p], (int)np, reinterpret_cast<float4 *>(ctx_planes(c)), s), "planes");
        CK(cudaMemcpyAsync(ctx_costs(c), m.cost[p], sizeof(float) * np, cudaMemcpyDeviceToDevice, s), "costs");
        ctx_mark_state(c);
        HpmParams pp = params(p, geom_iters);
        pp.geom_consistency = 1;
        pp.multi_geometry = multi ? 1 : 0;
        rr = hpm_run_patchmatch(c, &pp);
        return rr ? rr : store(p, true);
    };
    /* JointBilateralUpsampling (main.cpp:126-152) and the hierarchy block of
     * CudaSpaceInitialization (ACMM.cpp:663-719): the depth of depths.dmb
     * (the geometric depth upsampled by RunJBU, ACMM.cpp:804-855, unless
     * the integer scale is 1) and the last normals averaged with the JBU's
     * weights at the new size, which happens whenever the normal map's
     * width differs from the image's ROWS or its height from the image's
     * columns (the reference's comparison, ACMM.cpp:682) */
    auto hierarchy = [&](int p, int prev_w, int prev_h) -> int {
        const int W = m.at[p].w, H = m.at[p].h;
        const size_t np = (size_t)W * H, cp = (size_t)prev_w * prev_h;
        const int sr = H / prev_h, sc = W / prev_w, scale = sr > sc ? sr : sc;
        const bool up = prev_w != H || prev_h != W;
        int rr = load(p);
        if (rr) return rr;
        float4 *planes = reinterpret_cast<float4 *>(ctx_planes(c));
        if (up) {
            CK(flow_pack4(m.depth_g[p], m.normal[p], (int)cp, m.coarse, s), "jbu input");
            CK(launch_jbu(m.img[p], W, H, nullptr, m.coarse, prev_w, prev_h, scale, m.up_depth, m.up_normal, s),
               "jbu");
            if (scale > 1)
                CK(cudaMemcpyAsync(m.depth[p], m.up_depth, sizeof(float) * np, cudaMemcpyDeviceToDevice, s),
                   "depths.dmb");
            /* the upsampled normals become the view's normal map; the
             * split's depth output lands in the JBU scratch, unused */
            CK(flow_split_state(m.up_normal, (int)np, m.up_depth, m.normal[p], s), "normals");
        }
        CK(flow_pack4(m.depth[p], m.normal[p], (int)np, planes, s), "planes");
        ctx_mark_state(c);
        HpmParams pp = params(p, iters);
        pp.hierarchy = up ? 1 : 2;
        rr = hpm_run_patchmatch(c, &pp);
        return rr ? rr : store(p, false);
    };

    bool first = true;
    std::vector<int> prev_w(n_views), prev_h(n_views);
    while (max_down >= 0) {
        const Range scale_range("scale %d", max_down);
        for (int v = 0; v < n_views; ++v) {
            if (nd[v] >= 0) {
                cur[v] = (int)(max_size[v] / std::pow(2.0, nd[v])); /* main.cpp:331-336 */
                nd[v]--;
            }
            prev_w[v] = m.at[v].w;
            prev_h[v] = m.at[v].h;
            m.at[v] = scale_view(cams[v], cur[v]);
            const int w = m.at[v].w, h = m.at[v].h;
            CK(prior_resize(full[v], cams[v].width, cams[v].height, 1, m.img[v], w, h, s), "view resize");
        }
        if (first) {
            first = false;
            for (int p = 0; p < n_problems; ++p)
                if ((r = plain(p))) return r;
        } else {
            for (int p = 0; p < n_problems; ++p)
                if ((r = hierarchy(p, prev_w[p], prev_h[p]))) return r;
        }
        for (int gi = 0; gi < o->geom_iterations; ++gi)
            for (int p = 0; p < n_problems; ++p)
                if ((r = geometric(p, gi > 0))) return r;
        max_down--;
    }
    for (int v = 0; v < n_views; ++v) {
        const size_t np = (size_t)m.at[v].w * m.at[v].h;
        const float *d = o->geom_iterations > 0 ? m.depth_g[v] : m.depth[v];
        if (out_depths && out_depths[v])
            CK(cudaMemcpyAsync(out_depths[v], d, sizeof(float) * np, cudaMemcpyDefault, s), "out");
        if (out_normals && out_normals[v])
            CK(cudaMemcpyAsync(out_normals[v], m.normal[v], sizeof(float) * 3 * np, cudaMemcpyDefault, s), "out");
        if (out_costs && out_costs[v])
            CK(cudaMemcpyAsync(out_costs[v], m.cost[v], sizeof(float) * np, cudaMemcpyDefault, s), "out");
    }
    CK(cudaStreamSynchronize(s), "hpm_run_scene_acmm");
    return HPM_OK;
}

/*
 * Reference shim: compiles the reference's own HPM-MVS/HPM.cu (unchanged, from
 * where it lies) for sm_100a and exposes its kernels and __device__ functions
 * through a small C ABI, so that tests can produce golden vectors from the
 * reference's own code on a B200 and the reference arm of bench.py can time
 * the reference's RunPatchMatch.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref): never linked into the product.
 *
 * Host set-up restates what the reference's HPM.cpp does before its kernels
 * run (HPM.cpp needs OpenCV/PCL and cannot be compiled here):
 *   texture objects        HPM.cpp:595-617 (float cudaArray, linear filter,
 *                          wrap address mode, unnormalised coordinates)
 *   device buffers         HPM.cpp:618-633
 *   geometric-consistency  HPM.cpp:635-699
 *   JBU buffers            HPM.cpp:1181-1212, 1215-1247, 1322-1339
 * Build recipe: oracle/Makefile (target `ref`).
 */
#include "ref_stub.h"
#include "HPM.cu"

cudaError_t hpm_ref_first_error = cudaSuccess;

namespace {

struct Tex {
    cudaArray *array = nullptr;
    cudaTextureObject_t tex = 0;
};

cudaError_t make_texture(const float *host, int cols, int rows, Tex *out)
{
    cudaChannelFormatDesc desc = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaError_t e = cudaMallocArray(&out->array, &desc, cols, rows);
    if (e != cudaSuccess) return e;
    e = cudaMemcpy2DToArray(out->array, 0, 0, host, sizeof(float) * cols, sizeof(float) * cols, rows,
                            cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = out->array;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeWrap;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    return cudaCreateTextureObject(&out->tex, &res, &td, nullptr);
}

void free_texture(Tex *t)
{
    if (t->tex) cudaDestroyTextureObject(t->tex);
    if (t->array) cudaFreeArray(t->array);
    t->tex = 0;
    t->array = nullptr;
}

/* Owns the textures and device buffers of one reference problem. */
struct Problem {
    int n = 0;
    std::vector<Tex> images, depths;
    cudaTextureObjects *tex_d = nullptr, *depth_tex_d = nullptr;
    Camera *cams_d = nullptr;

    cudaError_t init(int num_images, const float *const *imgs, const Camera *cams, const float *const *depth_maps)
    {
        n = num_images;
        images.resize(n);
        cudaTextureObjects host;
        memset(&host, 0, sizeof(host));
        for (int i = 0; i < n; ++i) {
            cudaError_t e = make_texture(imgs[i], cams[i].width, cams[i].height, &images[i]);
            if (e != cudaSuccess) return e;
            host.images[i] = images[i].tex;
        }
        cudaError_t e = cudaMalloc(&tex_d, sizeof(cudaTextureObjects));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(tex_d, &host, sizeof(host), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        cudaTextureObjects dhost;
        memset(&dhost, 0, sizeof(dhost));
        if (depth_maps) {
            depths.resize(n);
            for (int i = 0; i < n; ++i) {
                e = make_texture(depth_maps[i], cams[i].width, cams[i].height, &depths[i]);
                if (e != cudaSuccess) return e;
                dhost.images[i] = depths[i].tex;
            }
        }
        e = cudaMalloc(&depth_tex_d, sizeof(cudaTextureObjects));
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(depth_tex_d, &dhost, sizeof(dhost), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        e = cudaMalloc(&cams_d, sizeof(Camera) * n);
        if (e != cudaSuccess) return e;
        return cudaMemcpy(cams_d, cams, sizeof(Camera) * n, cudaMemcpyHostToDevice);
    }

    ~Problem()
    {
        for (auto &t : images) free_texture(&t);
        for (auto &t : depths) free_texture(&t);
        cudaFree(tex_d);
        cudaFree(depth_tex_d);
        cudaFree(cams_d);
    }
};

PatchMatchParams make_params(int num_images, float depth_min, float depth_max)
{
    PatchMatchParams p;
    p.num_images = num_images;
    p.depth_min = depth_min;
    p.depth_max = depth_max;
    return p;
}

__global__ void k_cost_vectors(cudaTextureObjects *tex, Camera *cams, const float4 *planes, float *out,
                               PatchMatchParams params)
{
    const int2 p = make_int2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    const int w = cams[0].width, h = cams[0].height;
    if (p.x >= w || p.y >= h) return;
    const int c = p.y * w + p.x;
    float cv[32];
    ComputeMultiViewCostVector(tex[0].images, cams, p, planes[c], cv, params);
    for (int i = 0; i < params.num_images - 1; ++i) out[(size_t)c * (params.num_images - 1) + i] = cv[i];
}

__global__ void k_initial_costs(cudaTextureObjects *tex, Camera *cams, const float4 *planes, float *cost,
                                unsigned int *views, PatchMatchParams params)
{
    const int2 p = make_int2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    const int w = cams[0].width, h = cams[0].height;
    if (p.x >= w || p.y >= h) return;
    const int c = p.y * w + p.x;
    cost[c] = ComputeMultiViewInitialCostandSelectedViews(tex[0].images, cams, p, planes[c], &views[c], params);
}

__global__ void k_geom_costs(cudaTextureObjects *depth_tex, Camera *cams, const float4 *planes, float *out,
                             int num_images)
{
    const int2 p = make_int2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    const int w = cams[0].width, h = cams[0].height;
    if (p.x >= w || p.y >= h) return;
    const int c = p.y * w + p.x;
    for (int i = 1; i < num_images; ++i)
        out[(size_t)c * (num_images - 1) + i - 1] =
            ComputeGeomConsistencyCost(depth_tex[0].images[i], cams[0], cams[i], planes[c], p);
}

__global__ void k_homography(Camera ref, Camera src, const float4 *planes, int n, float *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float H[9];
    ComputeHomography(ref, src, planes[i], H);
    for (int k = 0; k < 9; ++k) out[i * 9 + k] = H[k];
}

__global__ void k_tex_fetch(cudaTextureObject_t t, const float2 *coords, int n, float *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = tex2D<float>(t, coords[i].x, coords[i].y);
}

/* The 36 source-texture samples of ComputeBilateralNCC (HPM.cu:337-359) for
 * listed pixels and every source view, with the reference's own
 * ComputeHomography and ComputeCorrespondingPoint; inside[k] = 0 where the
 * warped centre leaves the source image (the NCC is then 2). */
__global__ void k_tap_samples(cudaTextureObjects *tex, Camera *cams, const float4 *planes, const int *pixels, int n,
                              int num_images, float *out, int *inside)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int S = num_images - 1;
    if (k >= n * S) return;
    const int pi = k / S, v = k % S + 1;
    const int w = cams[0].width;
    const int2 p = make_int2(pixels[pi] % w, pixels[pi] / w);
    float H[9];
    ComputeHomography(cams[0], cams[v], planes[pixels[pi]], H);
    const float2 pt = ComputeCorrespondingPoint(H, p);
    inside[k] = !(pt.x >= cams[v].width || pt.x < 0.0f || pt.y >= cams[v].height || pt.y < 0.0f);
    int t = 0;
    for (int i = -5; i < 6; i += 2)
        for (int j = -5; j < 6; j += 2, ++t) {
            const float2 src_pt = ComputeCorrespondingPoint(H, make_int2(p.x + i, p.y + j));
            out[(size_t)k * 36 + t] = tex2D<float>(tex[0].images[v], src_pt.x + 0.5f, src_pt.y + 0.5f);
        }
}

int status(cudaError_t e)
{
    if (e == cudaSuccess && hpm_ref_first_error != cudaSuccess) e = hpm_ref_first_error;
    hpm_ref_first_error = cudaSuccess;
    return (int)e;
}

}  // namespace

extern "C" {

/* Options of one RunPatchMatch call (the PatchMatchParams fields the
 * reference's host code sets: HPM.cpp:468-480, 553-559). */
typedef struct {
    int geom_consistency;
    int planar_prior;
    int multi_geometry;
    float depth_min;
    float depth_max;
    unsigned long long seed;
} HpmRefRunOpts;

int hpm_ref_sizeof_camera(void) { return (int)sizeof(Camera); }
int hpm_ref_sizeof_params(void) { return (int)sizeof(PatchMatchParams); }

}  // extern "C"

namespace {

/* HPM::RunPatchMatch (HPM.cu:1906-1957) with a CUDA event pair around each of
 * its launches: the same grids, kernels and arguments, in the same order,
 * with the reference's synchronisation after each.  ms_out gets 10 kernel
 * times: RandomInitialization, the 6 Black/RedPixelUpdate half-steps,
 * GetDepthandNormal, BlackPixelFilter, RedPixelFilter. */
cudaError_t run_patchmatch_timed(HPM &hpm, float *ms_out)
{
    const int width = hpm.cameras[0].width, height = hpm.cameras[0].height;
    const dim3 gi((width + 15) / 16, (height + 15) / 16), bi(16, 16);
    const dim3 gc((width + 31) / 32, ((height / 2) + 15) / 16), bc(32, 16);
    cudaEvent_t ev[20];
    for (auto &e : ev) cudaEventCreate(&e);
    int k = 0;
    cudaEventRecord(ev[2 * k]);
    RandomInitialization<<<gi, bi>>>(hpm.texture_objects_cuda, hpm.cameras_cuda, hpm.plane_hypotheses_cuda,
                                     hpm.costs_cuda, hpm.rand_states_cuda, hpm.selected_views_cuda,
                                     hpm.prior_planes_cuda, hpm.plane_masks_cuda, hpm.params);
    cudaEventRecord(ev[2 * k + 1]);
    cudaDeviceSynchronize();
    ++k;
    for (int i = 0; i < 3; ++i) {
        for (int color = 0; color < 2; ++color) {
            cudaEventRecord(ev[2 * k]);
            if (color == 0)
                BlackPixelUpdate<<<gc, bc>>>(hpm.texture_objects_cuda, hpm.texture_depths_cuda, hpm.cameras_cuda,
                                             hpm.plane_hypotheses_cuda, hpm.costs_cuda, hpm.rand_states_cuda,
                                             hpm.selected_views_cuda, hpm.prior_planes_cuda, hpm.plane_masks_cuda,
                                             hpm.params, i);
            else
                RedPixelUpdate<<<gc, bc>>>(hpm.texture_objects_cuda, hpm.texture_depths_cuda, hpm.cameras_cuda,
                                           hpm.plane_hypotheses_cuda, hpm.costs_cuda, hpm.rand_states_cuda,
                                           hpm.selected_views_cuda, hpm.prior_planes_cuda, hpm.plane_masks_cuda,
                                           hpm.params, i);
            cudaEventRecord(ev[2 * k + 1]);
            cudaDeviceSynchronize();
            ++k;
        }
    }
    cudaEventRecord(ev[2 * k]);
    GetDepthandNormal<<<gi, bi>>>(hpm.cameras_cuda, hpm.plane_hypotheses_cuda, hpm.params);
    cudaEventRecord(ev[2 * k + 1]);
    cudaDeviceSynchronize();
    ++k;
    cudaEventRecord(ev[2 * k]);
    BlackPixelFilter<<<gc, bc>>>(hpm.cameras_cuda, hpm.plane_hypotheses_cuda, hpm.costs_cuda);
    cudaEventRecord(ev[2 * k + 1]);
    cudaDeviceSynchronize();
    ++k;
    cudaEventRecord(ev[2 * k]);
    RedPixelFilter<<<gc, bc>>>(hpm.cameras_cuda, hpm.plane_hypotheses_cuda, hpm.costs_cuda);
    cudaEventRecord(ev[2 * k + 1]);
    cudaError_t e = cudaDeviceSynchronize();
    ++k;
    for (int j = 0; j < k; ++j) cudaEventElapsedTime(&ms_out[j], ev[2 * j], ev[2 * j + 1]);
    for (auto &x : ev) cudaEventDestroy(x);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpy(hpm.plane_hypotheses_host, hpm.plane_hypotheses_cuda, sizeof(float4) * width * height,
                       cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(hpm.costs_host, hpm.costs_cuda, sizeof(float) * width * height, cudaMemcpyDeviceToHost);
    return e;
}

int run_patchmatch_impl(int num_images, const float *const *images, const Camera *cams, const HpmRefRunOpts *o,
                        float *planes_io, float *costs_io, const float *prior_planes, const unsigned int *plane_masks,
                        const float *const *depth_maps, float *ms_out)
{
    Problem pr;
    cudaError_t e = pr.init(num_images, images, cams, o->geom_consistency ? depth_maps : nullptr);
    if (e != cudaSuccess) return status(e);
    const int w = cams[0].width, h = cams[0].height;
    const size_t npx = (size_t)w * h;
    HPM hpm;
    hpm.cameras.assign(cams, cams + num_images);
    hpm.params = make_params(num_images, o->depth_min, o->depth_max);
    hpm.params.geom_consistency = o->geom_consistency != 0;
    hpm.params.planar_prior = o->planar_prior != 0;
    hpm.params.multi_geometry = o->multi_geometry != 0;
    if (o->geom_consistency) hpm.params.max_iterations = 2;
    hpm.plane_hypotheses_host = new float4[npx];
    hpm.costs_host = new float[npx];
    hpm.texture_objects_cuda = pr.tex_d;
    hpm.texture_depths_cuda = pr.depth_tex_d;
    hpm.cameras_cuda = pr.cams_d;
    e = cudaSetDevice(0);
    cudaMalloc(&hpm.plane_hypotheses_cuda, sizeof(float4) * npx);
    cudaMalloc(&hpm.costs_cuda, sizeof(float) * npx);
    cudaMalloc(&hpm.rand_states_cuda, sizeof(curandState) * npx);
    cudaMalloc(&hpm.selected_views_cuda, sizeof(unsigned int) * npx);
    cudaMalloc(&hpm.prior_planes_cuda, sizeof(float4) * npx);
    e = cudaMalloc(&hpm.plane_masks_cuda, sizeof(unsigned int) * npx);
    if (e == cudaSuccess) e = cudaMemset(hpm.plane_hypotheses_cuda, 0, sizeof(float4) * npx);
    if (e == cudaSuccess) e = cudaMemset(hpm.costs_cuda, 0, sizeof(float) * npx);
    if (e == cudaSuccess) e = cudaMemset(hpm.prior_planes_cuda, 0, sizeof(float4) * npx);
    if (e == cudaSuccess) e = cudaMemset(hpm.plane_masks_cuda, 0, sizeof(unsigned int) * npx);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(hpm_ref_seed, &o->seed, sizeof(o->seed));
    if (e == cudaSuccess && planes_io)
        e = cudaMemcpy(hpm.plane_hypotheses_cuda, planes_io, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && costs_io)
        e = cudaMemcpy(hpm.costs_cuda, costs_io, sizeof(float) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && prior_planes)
        e = cudaMemcpy(hpm.prior_planes_cuda, prior_planes, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && plane_masks)
        e = cudaMemcpy(hpm.plane_masks_cuda, plane_masks, sizeof(unsigned int) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ms_out) {
        e = run_patchmatch_timed(hpm, ms_out);
    } else if (e == cudaSuccess) {
        hpm.RunPatchMatch();
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) {
        if (planes_io) memcpy(planes_io, hpm.plane_hypotheses_host, sizeof(float4) * npx);
        if (costs_io) memcpy(costs_io, hpm.costs_host, sizeof(float) * npx);
    }
    cudaFree(hpm.plane_hypotheses_cuda);
    cudaFree(hpm.costs_cuda);
    cudaFree(hpm.rand_states_cuda);
    cudaFree(hpm.selected_views_cuda);
    cudaFree(hpm.prior_planes_cuda);
    cudaFree(hpm.plane_masks_cuda);
    delete[] hpm.plane_hypotheses_host;
    delete[] hpm.costs_host;
    return status(e);
}

}  // namespace

extern "C" {

/* One HPM::RunPatchMatch (HPM.cu:1906-1957) on a fresh problem.  planes_io /
 * costs_io seed the hypothesis state (the reference keeps that state on the
 * device between passes of one HPM object); on return they hold the result. */
int hpm_ref_run_patchmatch(int num_images, const float *const *images, const Camera *cams, const HpmRefRunOpts *o,
                           float *planes_io, float *costs_io, const float *prior_planes,
                           const unsigned int *plane_masks, const float *const *depth_maps)
{
    return run_patchmatch_impl(num_images, images, cams, o, planes_io, costs_io, prior_planes, plane_masks,
                               depth_maps, nullptr);
}

/* The same pass with each kernel timed by CUDA events (ms_out: 10 floats,
 * see run_patchmatch_timed). */
int hpm_ref_run_patchmatch_timed(int num_images, const float *const *images, const Camera *cams,
                                 const HpmRefRunOpts *o, float *planes_io, float *costs_io, const float *prior_planes,
                                 const unsigned int *plane_masks, const float *const *depth_maps, float *ms_out)
{
    return run_patchmatch_impl(num_images, images, cams, o, planes_io, costs_io, prior_planes, plane_masks,
                               depth_maps, ms_out);
}

/* Tap samples of listed pixels (k_tap_samples): out [n][S][36], inside [n][S]. */
int hpm_ref_tap_samples(int num_images, const float *const *images, const Camera *cams, const float *planes,
                        const int *pixels, int n, float *out, int *inside)
{
    Problem pr;
    cudaError_t e = pr.init(num_images, images, cams, nullptr);
    if (e != cudaSuccess) return status(e);
    const size_t npx = (size_t)cams[0].width * cams[0].height;
    const int S = num_images - 1;
    float4 *d_planes = nullptr;
    int *d_pix = nullptr, *d_in = nullptr;
    float *d_out = nullptr;
    e = cudaMalloc(&d_planes, sizeof(float4) * npx);
    if (e == cudaSuccess) e = cudaMalloc(&d_pix, sizeof(int) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_in, sizeof(int) * (size_t)n * S);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * (size_t)n * S * 36);
    if (e == cudaSuccess) e = cudaMemcpy(d_planes, planes, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_pix, pixels, sizeof(int) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_tap_samples<<<(n * S + 127) / 128, 128>>>(pr.tex_d, pr.cams_d, d_planes, d_pix, n, num_images, d_out, d_in);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, sizeof(float) * (size_t)n * S * 36, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(inside, d_in, sizeof(int) * (size_t)n * S, cudaMemcpyDeviceToHost);
    cudaFree(d_planes);
    cudaFree(d_pix);
    cudaFree(d_in);
    cudaFree(d_out);
    return status(e);
}

/* ComputeMultiViewCostVector (HPM.cu:438-443) for one ref-frame plane per pixel. */
int hpm_ref_cost_vectors(int num_images, const float *const *images, const Camera *cams, const float *planes,
                         float *out)
{
    Problem pr;
    cudaError_t e = pr.init(num_images, images, cams, nullptr);
    if (e != cudaSuccess) return status(e);
    const int w = cams[0].width, h = cams[0].height;
    const size_t npx = (size_t)w * h;
    float4 *planes_d = nullptr;
    float *out_d = nullptr;
    cudaMalloc(&planes_d, sizeof(float4) * npx);
    e = cudaMalloc(&out_d, sizeof(float) * npx * (num_images - 1));
    if (e == cudaSuccess) e = cudaMemcpy(planes_d, planes, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        dim3 b(16, 16), g((w + 15) / 16, (h + 15) / 16);
        k_cost_vectors<<<g, b>>>(pr.tex_d, pr.cams_d, planes_d, out_d, make_params(num_images, 0.f, 1.f));
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, out_d, sizeof(float) * npx * (num_images - 1), cudaMemcpyDeviceToHost);
    cudaFree(planes_d);
    cudaFree(out_d);
    return status(e);
}

/* ComputeMultiViewInitialCostandSelectedViews (HPM.cu:399-436) per pixel. */
int hpm_ref_initial_costs(int num_images, const float *const *images, const Camera *cams, const float *planes,
                          float *out_cost, unsigned int *out_views)
{
    Problem pr;
    cudaError_t e = pr.init(num_images, images, cams, nullptr);
    if (e != cudaSuccess) return status(e);
    const int w = cams[0].width, h = cams[0].height;
    const size_t npx = (size_t)w * h;
    float4 *planes_d = nullptr;
    float *cost_d = nullptr;
    unsigned int *views_d = nullptr;
    cudaMalloc(&planes_d, sizeof(float4) * npx);
    cudaMalloc(&cost_d, sizeof(float) * npx);
    e = cudaMalloc(&views_d, sizeof(unsigned int) * npx);
    if (e == cudaSuccess) e = cudaMemcpy(planes_d, planes, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        dim3 b(16, 16), g((w + 15) / 16, (h + 15) / 16);
        k_initial_costs<<<g, b>>>(pr.tex_d, pr.cams_d, planes_d, cost_d, views_d, make_params(num_images, 0.f, 1.f));
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out_cost, cost_d, sizeof(float) * npx, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out_views, views_d, sizeof(unsigned int) * npx, cudaMemcpyDeviceToHost);
    cudaFree(planes_d);
    cudaFree(cost_d);
    cudaFree(views_d);
    return status(e);
}

/* ComputeGeomConsistencyCost (HPM.cu:483-508) per pixel and source view. */
int hpm_ref_geom_costs(int num_images, const Camera *cams, const float *const *depth_maps, const float *planes,
                       float *out)
{
    Problem pr;
    cudaError_t e = pr.init(num_images, depth_maps, cams, depth_maps);
    if (e != cudaSuccess) return status(e);
    const int w = cams[0].width, h = cams[0].height;
    const size_t npx = (size_t)w * h;
    float4 *planes_d = nullptr;
    float *out_d = nullptr;
    cudaMalloc(&planes_d, sizeof(float4) * npx);
    e = cudaMalloc(&out_d, sizeof(float) * npx * (num_images - 1));
    if (e == cudaSuccess) e = cudaMemcpy(planes_d, planes, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        dim3 b(16, 16), g((w + 15) / 16, (h + 15) / 16);
        k_geom_costs<<<g, b>>>(pr.depth_tex_d, pr.cams_d, planes_d, out_d, num_images);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, out_d, sizeof(float) * npx * (num_images - 1), cudaMemcpyDeviceToHost);
    cudaFree(planes_d);
    cudaFree(out_d);
    return status(e);
}

/* ComputeHomography (HPM.cu:227-287) for n planes. */
int hpm_ref_homography(const Camera *ref, const Camera *src, const float *planes, int n, float *out9)
{
    float4 *planes_d = nullptr;
    float *out_d = nullptr;
    cudaMalloc(&planes_d, sizeof(float4) * n);
    cudaError_t e = cudaMalloc(&out_d, sizeof(float) * 9 * n);
    if (e == cudaSuccess) e = cudaMemcpy(planes_d, planes, sizeof(float4) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_homography<<<(n + 127) / 128, 128>>>(*ref, *src, planes_d, n, out_d);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out9, out_d, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost);
    cudaFree(planes_d);
    cudaFree(out_d);
    return status(e);
}

/* tex2D<float> on a texture built exactly like the reference's image
 * textures: pins the hardware's bilinear weights and edge addressing. */
int hpm_ref_tex_fetch(const float *img, int cols, int rows, const float *coords, int n, float *out)
{
    Tex t;
    cudaError_t e = make_texture(img, cols, rows, &t);
    float2 *c_d = nullptr;
    float *o_d = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&c_d, sizeof(float2) * n);
    if (e == cudaSuccess) e = cudaMalloc(&o_d, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemcpy(c_d, coords, sizeof(float2) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_tex_fetch<<<(n + 127) / 128, 128>>>(t.tex, c_d, n, o_d);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, o_d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(c_d);
    cudaFree(o_d);
    free_texture(&t);
    return status(e);
}

/* GetDepthandNormal then BlackPixelFilter / RedPixelFilter, launched as in
 * HPM.cu:1946-1952.  planes_io: ref-frame planes in, (world normal, depth) out. */
int hpm_ref_depth_normal_filter(const Camera *ref, float *planes_io, const float *costs)
{
    const int w = ref->width, h = ref->height;
    const size_t npx = (size_t)w * h;
    Camera *cam_d = nullptr;
    float4 *planes_d = nullptr;
    float *costs_d = nullptr;
    cudaMalloc(&cam_d, sizeof(Camera));
    cudaMalloc(&planes_d, sizeof(float4) * npx);
    cudaError_t e = cudaMalloc(&costs_d, sizeof(float) * npx);
    if (e == cudaSuccess) e = cudaMemcpy(cam_d, ref, sizeof(Camera), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(planes_d, planes_io, sizeof(float4) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(costs_d, costs, sizeof(float) * npx, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        PatchMatchParams params;
        dim3 b1(16, 16), g1((w + 15) / 16, (h + 15) / 16);
        dim3 b2(32, 16), g2((w + 31) / 32, ((h / 2) + 15) / 16);
        GetDepthandNormal<<<g1, b1>>>(cam_d, planes_d, params);
        BlackPixelFilter<<<g2, b2>>>(cam_d, planes_d, costs_d);
        RedPixelFilter<<<g2, b2>>>(cam_d, planes_d, costs_d);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(planes_io, planes_d, sizeof(float4) * npx, cudaMemcpyDeviceToHost);
    cudaFree(cam_d);
    cudaFree(planes_d);
    cudaFree(costs_d);
    return status(e);
}

/* HPM::JointBilateralUpsampling (HPM.cpp:1215-1281) through JBU::CudaRun
 * (HPM.cu:2054-2088).  coarse_normal: s_rows*s_cols*3; out_normal: rows*cols*3.
 * Returns 0 without output when the integer scale is 1, as the reference does. */
int hpm_ref_jbu(const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal,
                int s_cols, int s_rows, float *out_depth, float *out_normal)
{
    int scale_r = rows / s_rows, scale_c = cols / s_cols;
    int image_scale = scale_r > scale_c ? scale_r : scale_c;
    if (image_scale == 1) return 0;
    JBU jbu;
    jbu.jp_h.height = rows;
    jbu.jp_h.width = cols;
    jbu.jp_h.s_height = s_rows;
    jbu.jp_h.s_width = s_cols;
    jbu.jp_h.Imagescale = image_scale;
    Tex t0, t1;
    cudaError_t e = make_texture(guide, cols, rows, &t0);
    if (e == cudaSuccess) e = make_texture(coarse_depth, s_cols, s_rows, &t1);
    jbu.jt_h.imgs[0] = t0.tex;
    jbu.jt_h.imgs[1] = t1.tex;
    const size_t n = (size_t)rows * cols, on = (size_t)s_rows * s_cols;
    std::vector<float4> origin(on);
    for (size_t i = 0; i < on; ++i)
        origin[i] = make_float4(coarse_normal[3 * i], coarse_normal[3 * i + 1], coarse_normal[3 * i + 2], coarse_depth[i]);
    jbu.depth_h = (float *)malloc(sizeof(float) * n);
    jbu.normal_h = new float4[n];
    cudaMalloc(&jbu.depth_d, sizeof(float) * n);
    cudaMalloc(&jbu.normal_d, sizeof(float4) * n);
    cudaMalloc(&jbu.normal_origin_cuda, sizeof(float4) * on);
    cudaMalloc(&jbu.jp_d, sizeof(JBUParameters));
    if (e == cudaSuccess) e = cudaMalloc(&jbu.jt_d, sizeof(JBUTexObj));
    if (e == cudaSuccess) e = cudaMemcpy(jbu.normal_origin_cuda, origin.data(), sizeof(float4) * on, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(jbu.jp_d, &jbu.jp_h, sizeof(JBUParameters), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(jbu.jt_d, &jbu.jt_h, sizeof(JBUTexObj), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        jbu.CudaRun();
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) {
        for (size_t i = 0; i < n; ++i) {
            out_depth[i] = jbu.depth_h[i];
            out_normal[3 * i] = jbu.normal_h[i].x;
            out_normal[3 * i + 1] = jbu.normal_h[i].y;
            out_normal[3 * i + 2] = jbu.normal_h[i].z;
        }
    }
    cudaFree(jbu.depth_d);
    cudaFree(jbu.normal_d);
    cudaFree(jbu.normal_origin_cuda);
    cudaFree(jbu.jp_d);
    cudaFree(jbu.jt_d);
    free(jbu.depth_h);
    delete[] jbu.normal_h;
    free_texture(&t0);
    free_texture(&t1);
    return status(e);
}

}  // extern "C"

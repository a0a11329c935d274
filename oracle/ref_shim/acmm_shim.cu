/*
 * ACMM+NESP reference shim: compiles the reference's own
 * ACMM+NESP/windows/ACMM.cu (unchanged, from where it lies) for sm_100a and
 * runs its RandomInitialization kernel (ACMM.cu:521-621) through a small C
 * ABI, so that tests can pin the variant's hierarchy initialisation against
 * the reference's own code on a B200.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/_ref): never linked into the product.
 *
 * Host set-up restates what ACMM.cpp does before the kernel runs:
 *   texture objects   ACMM.cpp:559-580 (float cudaArray, linear filter, wrap
 *                     address mode, unnormalised coordinates)
 *   hierarchy inputs  ACMM.cpp:663-719: scaled_plane_hypotheses = the previous
 *                     scale's (normal, cost) per pixel when upsampling; the
 *                     full-size plane_hypotheses with only .w = depth set, the
 *                     rest of the freshly allocated array zero-filled
 * Build recipe: oracle/Makefile (target `acmm`).
 */
#include "acmm_stub.h"
#include "ACMM.cu"

cudaError_t acmm_ref_first_error = cudaSuccess;

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

}  // namespace

/* RandomInitialization of a hierarchy pass with upsample set (ACMM.cu:538-604).
 * planes4: W*H float4 with (0, 0, 0, depth) as the host leaves them; scaled4:
 * sw*sh float4 (previous scale's world normal, cost).  Outputs: planes
 * (ref-frame normal, distance), costs, pre_costs, selected views. */
extern "C" int acmm_ref_hier_init(int n_img, const float *const *imgs, const Camera *cams, const float *planes4,
                                  const float *scaled4, int sw, int sh, float depth_min, float depth_max,
                                  float *out_planes4, float *out_costs, float *out_pre, unsigned *out_views)
{
    if (n_img < 2 || n_img > 33) return -1;
    acmm_ref_first_error = cudaSuccess;
    const int W = cams[0].width, H = cams[0].height;
    const size_t n = (size_t)W * H, ns = (size_t)sw * sh;
    std::vector<Tex> tex(n_img);
    cudaTextureObjects to;
    memset(&to, 0, sizeof(to));
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < n_img && e == cudaSuccess; ++i) {
        e = make_texture(imgs[i], cams[i].width, cams[i].height, &tex[i]);
        to.images[i] = tex[i].tex;
    }
    cudaTextureObjects *d_to = nullptr;
    Camera *d_cams = nullptr;
    float4 *d_planes = nullptr, *d_scaled = nullptr;
    float *d_costs = nullptr, *d_pre = nullptr;
    curandState *d_rand = nullptr;
    unsigned *d_views = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d_to, sizeof(to));
    if (e == cudaSuccess) e = cudaMemcpy(d_to, &to, sizeof(to), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d_cams, sizeof(Camera) * n_img);
    if (e == cudaSuccess) e = cudaMemcpy(d_cams, cams, sizeof(Camera) * n_img, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d_planes, sizeof(float4) * n);
    if (e == cudaSuccess) e = cudaMemcpy(d_planes, planes4, sizeof(float4) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d_scaled, sizeof(float4) * ns);
    if (e == cudaSuccess) e = cudaMemcpy(d_scaled, scaled4, sizeof(float4) * ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&d_costs, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_pre, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemset(d_pre, 0, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_rand, sizeof(curandState) * n);
    if (e == cudaSuccess) e = cudaMalloc(&d_views, sizeof(unsigned) * n);
    if (e == cudaSuccess) {
        PatchMatchParams p;
        p.num_images = n_img;
        p.depth_min = depth_min;
        p.depth_max = depth_max;
        p.hierarchy = true;
        p.upsample = true;
        p.scaled_cols = (float)sw;
        p.scaled_rows = (float)sh;
        unsigned long long seed = 1;
        e = cudaMemcpyToSymbol(acmm_ref_seed, &seed, sizeof(seed));
        /* the launch shape of ACMM::RunPatchMatch (ACMM.cu:1817-1840) */
        dim3 grid((W + 15) / 16, (H + 15) / 16), block(16, 16);
        if (e == cudaSuccess) {
            RandomInitialization<<<grid, block>>>(d_to, d_cams, d_planes, d_scaled, d_costs, d_pre, d_rand, d_views,
                                                  p);
            e = cudaDeviceSynchronize();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpy(out_planes4, d_planes, sizeof(float4) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out_costs, d_costs, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out_pre, d_pre, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(out_views, d_views, sizeof(unsigned) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_to);
    cudaFree(d_cams);
    cudaFree(d_planes);
    cudaFree(d_scaled);
    cudaFree(d_costs);
    cudaFree(d_pre);
    cudaFree(d_rand);
    cudaFree(d_views);
    for (Tex &t : tex) {
        if (t.tex) cudaDestroyTextureObject(t.tex);
        if (t.array) cudaFreeArray(t.array);
    }
    return e == cudaSuccess ? 0 : -2;
}

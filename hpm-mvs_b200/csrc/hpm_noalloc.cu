/*
 * Joint bilateral upsampling that allocates nothing: hpm_jbu_noalloc.
 *
 * Who needs it: callers that may not allocate device memory while they run,
 * e.g. a host application that hands its whole GPU memory budget to its own
 * pool allocator up front, or a plugin invoked from a real-time or
 * graph-capturing host loop where a cudaMalloc/cudaFree would synchronise the
 * device or break the caller's memory accounting.  hpm_jbu needs a context,
 * whose creation and whose scratch buffers use cudaMalloc; this variant works
 * on device buffers the caller already owns and keeps its only scratch (the
 * coarse depth and normal packed into one float4 per coarse pixel) in a
 * fixed, file-scope device array.
 *
 * When that array takes device memory: it belongs to this library's device
 * code, which CUDA loads on a device when the code is first used there.  With
 * CUDA's default lazy module loading (CUDA_MODULE_LOADING=LAZY) that is the
 * first hpm_jbu_noalloc call on the device (the symbol lookup below), not
 * the library's load; with eager loading it is context creation.  Either way
 * the 16 MiB stay allocated until the process exits, and no later call
 * allocates anything.  So make the first call on each device before the
 * caller reserves its memory budget and before any stream capture.
 *
 * Limit: the coarse grid may hold at most HPM_JBU_NOALLOC_MAX_COARSE pixels
 * (1,048,576: 16 MiB of float4 per device).
 */
#include <cuda_runtime.h>

#include "hpm_b200.h"
#include "hpm_jbu_pixel.cuh"

namespace {

constexpr int kMaxCoarse = HPM_JBU_NOALLOC_MAX_COARSE;

/* The scratch: one float4 (nx, ny, nz, depth) per coarse pixel. */
static __device__ __align__(256) float4 g_jbu_scratch[kMaxCoarse];

__global__ void k_pack_coarse(const float *__restrict__ depth, const float *__restrict__ normal, int n,
                              float4 *__restrict__ packed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    packed[i] = make_float4(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2], depth[i]);
}

/* The context path's JBU (hpm::jbu_pixel), writing the normal as 3 floats
 * per pixel as the caller's buffers hold it. */
__global__ void k_jbu_noalloc(const float *__restrict__ guide, int cols, int rows, const float4 *__restrict__ coarse,
                              int s_cols, int s_rows, int image_scale, float *__restrict__ out_depth,
                              float *__restrict__ out_normal)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= cols || py >= rows) return;
    const float4 n = hpm::jbu_pixel(guide, cols, rows, coarse, s_cols, s_rows, image_scale, px, py);
    const size_t o = (size_t)py * cols + px;
    out_depth[o] = n.w;
    out_normal[3 * o] = n.x;
    out_normal[3 * o + 1] = n.y;
    out_normal[3 * o + 2] = n.z;
}

/* Makes `device` current for the lifetime of the object and gives the
 * caller's current device back on every return path. */
struct DeviceGuard {
    int saved = -1;
    bool ok = false;
    explicit DeviceGuard(int device)
    {
        if (cudaGetDevice(&saved) != cudaSuccess) return;
        ok = saved == device || cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

}  // namespace

extern "C" int hpm_jbu_noalloc(int device, const float *guide, int cols, int rows, const float *coarse_depth,
                               const float *coarse_normal, int s_cols, int s_rows, float *out_depth,
                               float *out_normal, void *stream)
{
    if (!guide || !coarse_depth || !coarse_normal || !out_depth || !out_normal) return HPM_ERR_ARG;
    if (cols < 1 || rows < 1 || s_cols < 1 || s_rows < 1 || s_cols > cols || s_rows > rows) return HPM_ERR_ARG;
    if ((long long)s_cols * s_rows > kMaxCoarse) return HPM_ERR_ARG; /* coarse grid above the fixed scratch */
    if (device < 0) return HPM_ERR_ARG;
    const int sr = rows / s_rows, sc = cols / s_cols;
    const int image_scale = sr > sc ? sr : sc;
    if (image_scale == 1) return HPM_OK; /* as hpm_jbu: nothing to upsample */
    DeviceGuard guard(device);
    if (!guard.ok) return HPM_ERR_CUDA;
    /* The array's address on this device, looked up on every call (cheap
     * once the code is loaded; never stale after a cudaDeviceReset).  In host
     * code g_jbu_scratch names a host-side stand-in, not device memory. */
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_jbu_scratch) != cudaSuccess || !p) return HPM_ERR_CUDA;
    float4 *scratch = static_cast<float4 *>(p);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int n = s_cols * s_rows;
    /* every scratch entry the upsampling reads is written first: nothing has
     * to start at zero.  cudaLaunchKernel returns each launch's own status,
     * so an earlier unrelated error of the caller is neither reported nor
     * cleared here. */
    {
        void *args[] = {(void *)&coarse_depth, (void *)&coarse_normal, (void *)&n, (void *)&scratch};
        if (cudaLaunchKernel((const void *)k_pack_coarse, dim3((n + 255) / 256), dim3(256), args, 0, s) !=
            cudaSuccess)
            return HPM_ERR_CUDA;
    }
    {
        const float4 *coarse = scratch;
        int image_scale_arg = image_scale;
        void *args[] = {(void *)&guide,  (void *)&cols,   (void *)&rows,           (void *)&coarse,
                        (void *)&s_cols, (void *)&s_rows, (void *)&image_scale_arg, (void *)&out_depth,
                        (void *)&out_normal};
        if (cudaLaunchKernel((const void *)k_jbu_noalloc, dim3((cols + 15) / 16, (rows + 15) / 16), dim3(16, 16),
                             args, 0, s) != cudaSuccess)
            return HPM_ERR_CUDA;
    }
    return HPM_OK;
}

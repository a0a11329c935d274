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
 * fixed, file-scope device array that exists from the moment the library is
 * loaded on a device until the process exits.
 *
 * Limit: the coarse grid may hold at most HPM_JBU_NOALLOC_MAX_COARSE pixels
 * (1,048,576: 16 MiB of float4 per device).
 */
#include <cuda_runtime.h>

#include <mutex>

#include "hpm_b200.h"

namespace {

constexpr int kMaxCoarse = HPM_JBU_NOALLOC_MAX_COARSE;
constexpr int kMaxDevices = 64;

/* The scratch: one float4 (nx, ny, nz, depth) per coarse pixel. */
static __device__ __align__(256) float4 g_jbu_scratch[kMaxCoarse];

/* Device address of g_jbu_scratch, looked up once per device. */
float4 *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

int scratch_for_device(int device, float4 **out)
{
    if (device < 0 || device >= kMaxDevices) return HPM_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        /* the device is current here: the address is that device's copy */
        const cudaError_t e = cudaGetSymbolAddress(&p, g_jbu_scratch);
        if (e != cudaSuccess || !p) return HPM_ERR_CUDA;
        g_scratch_ptr[device] = static_cast<float4 *>(p);
    }
    *out = g_scratch_ptr[device];
    return HPM_OK;
}

__global__ void k_pack_coarse(const float *__restrict__ depth, const float *__restrict__ normal, int n,
                              float4 *__restrict__ packed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    packed[i] = make_float4(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2], depth[i]);
}

/* Same computation as the context path's JBU kernel (reference JBU_cu,
 * HPM-MVS/HPM.cu:1984-2052), writing the normal as 3 floats per pixel. */
__global__ void k_jbu_noalloc(const float *__restrict__ guide, int cols, int rows, const float4 *__restrict__ coarse,
                              int s_cols, int s_rows, int image_scale, float *__restrict__ out_depth,
                              float *__restrict__ out_normal)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= cols || py >= rows) return;
    const float scale = (float)(1.0 * s_cols / cols);
    const int nn = (image_scale * image_scale + 1) / 2;
    const float oy = py * scale, ox = px * scale;
    const float ref_pix = __ldg(guide + (size_t)py * cols + px);
    const float inv_2sd2 = 1.0f / (2.0f * 0.5f * 0.5f);
    const float inv_2sr2 = 1.0f / (2.0f * 25.5f * 25.5f);
    float nf = 0.0f, ctot = 0.0f, nx = 0.0f, ny = 0.0f, nz = 0.0f;
    for (int j = -nn; j <= nn; ++j) {
        int ry = __float2int_rz(oy + (float)j);
        ry = ry > 0 ? (ry < s_rows ? ry : s_rows - 1) : 0;
        const int rys = min(max(py + j, 0), rows - 1);
        const float dy = oy - (float)ry;
        const float *grow = guide + (size_t)rys * cols;
        for (int i = -nn; i <= nn; ++i) {
            int rx = __float2int_rz(ox + (float)i);
            rx = rx > 0 ? (rx < s_cols ? rx : s_cols - 1) : 0;
            const float4 c = coarse[(size_t)ry * s_cols + rx];
            const int rxs = min(max(px + i, 0), cols - 1);
            const float nb = __ldg(grow + rxs);
            const float dx = ox - (float)rx;
            const float sg = expf(-(dx * dx + dy * dy) * inv_2sd2);
            const float xp = fabsf(ref_pix - nb);
            const float rg = expf(-(xp * xp) * inv_2sr2);
            const float tg = sg * rg;
            nf += tg;
            ctot += c.w * tg;
            nx += c.x * tg;
            ny += c.y * tg;
            nz += c.z * tg;
        }
    }
    float ax = nx / nf, ay = ny / nf, az = nz / nf;
    const float inv = rsqrtf(ax * ax + ay * ay + az * az);
    const size_t o = (size_t)py * cols + px;
    out_depth[o] = ctot / nf;
    out_normal[3 * o] = ax * inv;
    out_normal[3 * o + 1] = ay * inv;
    out_normal[3 * o + 2] = az * inv;
}

}  // namespace

extern "C" int hpm_jbu_noalloc(int device, const float *guide, int cols, int rows, const float *coarse_depth,
                               const float *coarse_normal, int s_cols, int s_rows, float *out_depth,
                               float *out_normal, void *stream)
{
    if (!guide || !coarse_depth || !coarse_normal || !out_depth || !out_normal) return HPM_ERR_ARG;
    if (cols < 1 || rows < 1 || s_cols < 1 || s_rows < 1 || s_cols > cols || s_rows > rows) return HPM_ERR_ARG;
    if ((long long)s_cols * s_rows > kMaxCoarse) return HPM_ERR_ARG; /* coarse grid above the fixed scratch */
    const int sr = rows / s_rows, sc = cols / s_cols;
    const int image_scale = sr > sc ? sr : sc;
    if (image_scale == 1) return HPM_OK; /* as hpm_jbu: nothing to upsample */
    if (cudaSetDevice(device) != cudaSuccess) return HPM_ERR_CUDA;
    float4 *scratch = nullptr;
    int rc = scratch_for_device(device, &scratch);
    if (rc != HPM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = s_cols * s_rows;
    /* every scratch entry the upsampling reads is written first: nothing has
     * to start at zero */
    k_pack_coarse<<<(n + 255) / 256, 256, 0, s>>>(coarse_depth, coarse_normal, n, scratch);
    dim3 b(16, 16), g((cols + 15) / 16, (rows + 15) / 16);
    k_jbu_noalloc<<<g, b, 0, s>>>(guide, cols, rows, scratch, s_cols, s_rows, image_scale, out_depth, out_normal);
    return cudaGetLastError() == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
}

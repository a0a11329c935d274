/*
 * Joint bilateral upsampling of a coarse prior (depth + world normal) to
 * full resolution, guided by the full-resolution gray image: the reference's
 * JBU_cu (HPM-MVS/HPM.cu:1971-2052).  The per-pixel computation is
 * hpm::jbu_pixel (hpm_jbu_pixel.cuh); this file maps it onto the machine:
 * one thread per fine pixel in 16x16 tiles, the coarse depth and normal
 * packed by the caller into one float4 per coarse pixel.
 */
#include "hpm_internal.h"
#include "hpm_jbu_pixel.cuh"

namespace hpm {
namespace {

__global__ void k_jbu(const float *__restrict__ guide, int cols, int rows, const float4 *__restrict__ coarse,
                      int s_cols, int s_rows, int image_scale, float *__restrict__ out_depth,
                      float4 *__restrict__ out_normal)
{
    const int px = blockIdx.x * blockDim.x + threadIdx.x;
    const int py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= cols || py >= rows) return;
    float4 n = jbu_pixel(guide, cols, rows, coarse, s_cols, s_rows, image_scale, px, py);
    const size_t c = (size_t)py * cols + px;
    out_depth[c] = n.w;
    n.w = 0.0f;
    out_normal[c] = n;
}

}  // namespace

cudaError_t launch_jbu(const float *guide, int cols, int rows, const float *coarse_depth, const float4 *coarse_normal,
                       int s_cols, int s_rows, int image_scale, float *out_depth, float4 *out_normal, cudaStream_t s)
{
    (void)coarse_depth; /* packed into coarse_normal.w by the caller */
    dim3 b(16, 16), g((cols + 15) / 16, (rows + 15) / 16);
    k_jbu<<<g, b, 0, s>>>(guide, cols, rows, coarse_normal, s_cols, s_rows, image_scale, out_depth, out_normal);
    return cudaGetLastError();
}

}  // namespace hpm

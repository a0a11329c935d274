/*
 * One fine pixel of the joint bilateral upsampling, shared by the context
 * path's k_jbu (hpm_jbu.cu) and the allocation-free k_jbu_noalloc
 * (hpm_noalloc.cu), so that the two cannot drift apart.
 *
 * Behaviour of the reference's JBU_cu (HPM-MVS/HPM.cu:1971-2052): for a fine
 * pixel p the window is (s*s+1) x (s*s+1) taps of the coarse grid around
 * o = p * (coarse_w / fine_w) (coordinates truncated, then clamped), the
 * spatial weight is exp(-d^2 / (2 * 0.5^2)) in coarse units and the range
 * weight exp(-dI^2 / (2 * 25.5^2)) compares the guide at p with the guide at
 * p + (i, j) in FINE pixels (the mixed-space window of the reference is kept).
 * Depth is the weighted mean; the normal is the normalised weighted sum.
 *
 * The coarse depth and normal come packed as one float4 (nx, ny, nz, depth)
 * per coarse pixel, so that every tap is a single 16-byte read-only load.
 * The reference computes both gaussians in double precision (pow/exp of a
 * double); here they are FP32 expf of the same arguments.
 */
#pragma once

#include <cuda_runtime.h>

namespace hpm {

/* Returns (nx, ny, nz, depth) of fine pixel (px, py). */
__device__ __forceinline__ float4 jbu_pixel(const float *__restrict__ guide, int cols, int rows,
                                            const float4 *__restrict__ coarse, int s_cols, int s_rows,
                                            int image_scale, int px, int py)
{
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
            const float4 c = __ldg(coarse + (size_t)ry * s_cols + rx);
            const int rxs = min(max(px + i, 0), cols - 1);
            const float nb = __ldg(grow + rxs);
            const float dx = ox - (float)rx;
            const float dis = dx * dx + dy * dy;
            const float sg = expf(-dis * inv_2sd2);
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
    float4 n = make_float4(nx / nf, ny / nf, nz / nf, 0.0f);
    const float inv = rsqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
    n.x *= inv;
    n.y *= inv;
    n.z *= inv;
    n.w = ctot / nf;
    return n;
}

}  // namespace hpm

/*
 * The integer stages of the planar prior as stand-alone C-ABI calls, for
 * exact parity checks: the triangle raster (main.cpp:96-116) and the
 * 6-nearest-neighbour search of DepthsPredictSupplement (HPM.cpp:939-962).
 * Both run the same kernels as hpm_prior_level and hpm_process_problem.
 */
#include <vector>

#include "hpm_prior.h"

namespace hpm {

void knn_grid(const int *xy, int n, int w, int h, int cell, int &gw, int &gh, std::vector<int> &start,
              std::vector<int> &order)
{
    gw = (w + cell - 1) / cell;
    gh = (h + cell - 1) / cell;
    start.assign((size_t)gw * gh + 1, 0);
    order.assign(n, 0);
    for (int k = 0; k < n; ++k) start[(xy[2 * k + 1] / cell) * gw + xy[2 * k] / cell + 1]++;
    for (int i = 0; i < gw * gh; ++i) start[i + 1] += start[i];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int k = 0; k < n; ++k) order[fill[(xy[2 * k + 1] / cell) * gw + xy[2 * k] / cell]++] = k;
}

}  // namespace hpm

namespace {

/* device buffers of one call, freed on every return path */
struct Buffers {
    std::vector<void *> p;
    template <typename T>
    cudaError_t get(T **out, size_t n)
    {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, n > 0 ? n * sizeof(T) : 1);
        if (e == cudaSuccess) p.push_back(q);
        *out = static_cast<T *>(q);
        return e;
    }
    ~Buffers()
    {
        for (void *q : p) cudaFree(q);
    }
};

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

extern "C" int hpm_raster_triangles(int device, const int *tris, int n, int w, int h, int *ids)
{
    if ((!tris && n > 0) || n < 0 || w < 1 || h < 1 || !ids) return HPM_ERR_ARG;
    for (int k = 0; k < 6 * n; ++k)
        if (tris[k] < 0 || tris[k] >= ((k & 1) ? h : w)) return HPM_ERR_ARG; /* vertices inside the image */
    DeviceGuard guard(device);
    if (!guard.ok) return HPM_ERR_CUDA;
    Buffers b;
    int *d_tris = nullptr, *d_ids = nullptr;
    const size_t npx = (size_t)w * h;
    if (b.get(&d_tris, 6 * (size_t)n) != cudaSuccess || b.get(&d_ids, npx) != cudaSuccess) return HPM_ERR_CUDA;
    if (n > 0 && cudaMemcpy(d_tris, tris, sizeof(int) * 6 * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return HPM_ERR_CUDA;
    if (cudaMemset(d_ids, 0, sizeof(int) * npx) != cudaSuccess) return HPM_ERR_CUDA;
    if (hpm::prior_raster(d_tris, n, w, d_ids, 0) != cudaSuccess) return HPM_ERR_CUDA;
    return cudaMemcpy(ids, d_ids, sizeof(int) * npx, cudaMemcpyDeviceToHost) == cudaSuccess ? HPM_OK : HPM_ERR_CUDA;
}

extern "C" int hpm_knn6(int device, const int *xy, int n, int w, int h, const float *mask, int *nn6)
{
    if ((!xy && n > 0) || n < 0 || w < 1 || h < 1 || !nn6) return HPM_ERR_ARG;
    for (int k = 0; k < n; ++k)
        if (xy[2 * k] < 0 || xy[2 * k] >= w || xy[2 * k + 1] < 0 || xy[2 * k + 1] >= h) return HPM_ERR_ARG;
    DeviceGuard guard(device);
    if (!guard.ok) return HPM_ERR_CUDA;
    const int cell = 8; /* the cell size hpm_process_problem uses */
    int gw, gh;
    std::vector<int> start, order;
    hpm::knn_grid(xy, n, w, h, cell, gw, gh, start, order);
    Buffers b;
    int2 *d_pts = nullptr;
    int *d_start = nullptr, *d_order = nullptr, *d_nn = nullptr;
    float *d_mask = nullptr;
    const size_t npx = (size_t)w * h;
    if (b.get(&d_pts, (size_t)n) != cudaSuccess || b.get(&d_start, start.size()) != cudaSuccess ||
        b.get(&d_order, (size_t)n) != cudaSuccess || b.get(&d_nn, 6 * npx) != cudaSuccess)
        return HPM_ERR_CUDA;
    if (mask && (b.get(&d_mask, npx) != cudaSuccess ||
                 cudaMemcpy(d_mask, mask, sizeof(float) * npx, cudaMemcpyHostToDevice) != cudaSuccess))
        return HPM_ERR_CUDA;
    if (n > 0 && (cudaMemcpy(d_pts, xy, sizeof(int) * 2 * n, cudaMemcpyHostToDevice) != cudaSuccess ||
                  cudaMemcpy(d_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice) != cudaSuccess))
        return HPM_ERR_CUDA;
    if (cudaMemcpy(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return HPM_ERR_CUDA;
    if (hpm::prior_knn_ids(d_pts, d_start, d_order, cell, gw, gh, w, h, d_mask, d_nn, 0) != cudaSuccess)
        return HPM_ERR_CUDA;
    return cudaMemcpy(nn6, d_nn, sizeof(int) * 6 * npx, cudaMemcpyDeviceToHost) == cudaSuccess ? HPM_OK
                                                                                              : HPM_ERR_CUDA;
}

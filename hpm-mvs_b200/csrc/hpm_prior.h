/*
 * Planar-prior construction: GPU launchers (hpm_prior.cu) and the host
 * Delaunay triangulation (hpm_delaunay.cpp).
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "hpm_b200.h"

namespace hpm {

cudaError_t prior_resize(const float *src, int sw, int sh, int ch, float *dst, int dw, int dh, cudaStream_t s);
cudaError_t prior_support_blocks(const float *costs, int w, int h, int2 *out, int *nblocks, cudaStream_t s);
cudaError_t prior_triangles(const HpmCamera &cam, const float *depth, int w, int h, const int *tris, int n,
                            float factor, float4 *planes, int *ids, cudaStream_t s);
cudaError_t prior_raster(const int *tris, int n, int w, int *ids, cudaStream_t s);
cudaError_t prior_knn_ids(const int2 *pts, const int *cell_start, const int *cell_pts, int cell, int gw, int gh, int w,
                          int h, const float *mask, int *nn6, cudaStream_t s);
/* Uniform grid of `cell`-pixel cells over w x h for the kNN search (CSR:
 * start[gw*gh+1], order[n] point indices ascending within a cell). */
void knn_grid(const int *xy, int n, int w, int h, int cell, int &gw, int &gh, std::vector<int> &start,
              std::vector<int> &order);
cudaError_t prior_ids_to_mask(const int *ids, int n, float *mask, cudaStream_t s);
cudaError_t prior_knn(const HpmCamera &cam, const int2 *pts, const int *cell_start, const int *cell_pts, int cell,
                      int gw, int gh, const float *depth, int w, int h, float factor, float dmin, float dmax, float *mask,
                      float4 *planes, cudaStream_t s);
/* widen: range-check triangle planes against [dmin, dmax] widened once
 * more (x0.6 / x1.2), as the reference does (main.cpp:129, 282); false
 * checks them against [dmin, dmax] */
cudaError_t prior_coarse(const HpmCamera &cam, int w, int h, float factor, float dmin, float dmax, float *mask,
                         const int *ids, const float4 *tri_planes, const float4 *knn_planes, float *out_depth,
                         float *out_normal, cudaStream_t s, bool widen = true);
cudaError_t prior_reload(const HpmCamera &cam, int w, int h, float dmin, float dmax, const float *up_depth,
                         const float4 *up_normal, float4 *prior, uint32_t *masks, cudaStream_t s);
cudaError_t prior_full(const HpmCamera &cam, int w, int h, float dmin, float dmax, const float *mask, const int *ids,
                       const float4 *tri_planes, const float4 *knn_planes, float *prior_depth, float4 *prior,
                       uint32_t *masks, cudaStream_t s);

/* Delaunay triangulation of integer points (DelaunayTriangulation,
 * HPM.cpp:787-809, which uses cv::Subdiv2D): triangles as 6 ints each,
 * counter-clockwise, those with all three vertices inside [0,w) x [0,h)
 * (the reference's imageRC.contains filter, main.cpp:97).  Co-circular
 * point sets have several Delaunay triangulations; this one keeps a point
 * that lies exactly on a circumcircle outside the cavity. */
void delaunay(const std::vector<int> &xy, int w, int h, std::vector<int> &tris_out);

}  // namespace hpm

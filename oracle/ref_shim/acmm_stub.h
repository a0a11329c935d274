/*
 * Stub declarations that let the reference's own ACMM+NESP/windows/ACMM.cu
 * compile for sm_100a without OpenCV or <direct.h>.
 *
 * TEST INFRASTRUCTURE ONLY: the shim built from this header is the checker
 * (oracle/_ref), never the product.  It is included before ACMM.cu so that the
 * include guards of the reference's main.h / ACMM.h are already defined and
 * those headers (which pull in OpenCV) are skipped.
 *
 * The types below restate the reference's data layouts because the compiled
 * reference kernels read them by value/pointer:
 *   Camera             ACMM+NESP/windows/main.h:36-44
 *   cudaTextureObjects ACMM+NESP/windows/ACMM.h:26-28
 *   PatchMatchParams   ACMM+NESP/windows/ACMM.h:30-52 (same defaults)
 *   JBUParameters/JBUTexObj/JBU  ACMM+NESP/windows/ACMM.h:100-131
 *   ACMM (only the members RunPatchMatch touches)  ACMM+NESP/windows/ACMM.h:54-99
 */
#pragma once
#define _MAIN_H_
#define _ACMM_H_

#include <cuda_runtime.h>
#include <cuda.h>
#include <cuda_runtime_api.h>
#include <cuda_texture_types.h>
#include <curand_kernel.h>
#include <vector_types.h>
#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define MAX_IMAGES 256
#define JBU_NUM 2
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

struct Camera {
    float K[9];
    float R[9];
    float t[3];
    int height;
    int width;
    float depth_min;
    float depth_max;
};

/* The reference aborts the process on a CUDA error; the shim records the
 * first error instead so that the harness can report it. */
extern cudaError_t acmm_ref_first_error;
inline void CudaSafeCall(const cudaError_t error, const std::string &, const int)
{
    if (error != cudaSuccess && acmm_ref_first_error == cudaSuccess) acmm_ref_first_error = error;
}
#define CUDA_SAFE_CALL(error) CudaSafeCall(error, __FILE__, __LINE__)

struct cudaTextureObjects {
    cudaTextureObject_t images[MAX_IMAGES];
};

struct PatchMatchParams {
    int max_iterations = 3;
    int patch_size = 11;
    int num_images = 5;
    int max_image_size = 3200;
    int radius_increment = 2;
    float sigma_spatial = 5.0f;
    float sigma_color = 3.0f;
    int top_k = 4;
    float baseline = 0.54f;
    float depth_min = 0.0f;
    float depth_max = 1.0f;
    float disparity_min = 0.0f;
    float disparity_max = 1.0f;

    float scaled_cols;
    float scaled_rows;

    bool geom_consistency = false;
    bool multi_geometry = false;
    bool hierarchy = false;
    bool upsample = false;
};

class ACMM {
public:
    void RunPatchMatch();

    std::vector<Camera> cameras;
    PatchMatchParams params;
    float4 *plane_hypotheses_host = nullptr;
    float *costs_host = nullptr;

    Camera *cameras_cuda = nullptr;
    cudaTextureObjects *texture_objects_cuda = nullptr;
    cudaTextureObjects *texture_depths_cuda = nullptr;
    float4 *plane_hypotheses_cuda = nullptr;
    float4 *scaled_plane_hypotheses_cuda = nullptr;
    float *costs_cuda = nullptr;
    float *pre_costs_cuda = nullptr;
    curandState *rand_states_cuda = nullptr;
    unsigned int *selected_views_cuda = nullptr;
};

struct JBUParameters {
    int height;
    int width;
    int s_height;
    int s_width;
    int Imagescale;
};

struct JBUTexObj {
    cudaTextureObject_t imgs[JBU_NUM];
};

class JBU {
public:
    float *depth_h = nullptr;
    JBUTexObj jt_h;
    JBUParameters jp_h;

    float *depth_d = nullptr;
    cudaArray *cuArray[JBU_NUM];
    JBUTexObj *jt_d = nullptr;
    JBUParameters *jp_d = nullptr;

    void CudaRun();
};

/* The reference seeds curand with clock64() (ACMM.cu:532); the shim makes
 * that seed settable so that its runs are reproducible. */
__device__ unsigned long long acmm_ref_seed;
#define clock64() (acmm_ref_seed)

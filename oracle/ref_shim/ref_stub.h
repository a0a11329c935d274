/*
 * Stub declarations that let the reference's own HPM-MVS/HPM.cu compile for
 * sm_100a without OpenCV, PCL or <direct.h>.
 *
 * TEST INFRASTRUCTURE ONLY: the shim built from this header is the checker
 * (oracle/_ref), never the product.  It is included before HPM.cu so that the
 * include guards of the reference's main.h / HPM.h are already defined and
 * those headers (which pull in OpenCV/PCL) are skipped.
 *
 * The types below restate the reference's data layouts because the compiled
 * reference kernels read them by value/pointer:
 *   Camera            HPM-MVS/main.h:44-52
 *   cudaTextureObjects HPM-MVS/HPM.h:27-29
 *   PatchMatchParams  HPM-MVS/HPM.h:29-46 (same defaults)
 *   JBUParameters/JBUTexObj/JBU  HPM-MVS/main.h:70-110
 *   HPM (only the members RunPatchMatch touches)  HPM-MVS/HPM.h:48-112
 */
#pragma once
#define _MAIN_H_
#define _HPM_H_

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

#define MAX_IMAGES 512
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define JBU_NUM 2

struct Camera {
    float K[9];
    float R[9];
    float t[3];
    int height;
    int width;
    float depth_min;
    float depth_max;
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
    float4 *normal_h = nullptr;
    JBUTexObj jt_h;
    JBUParameters jp_h;
    float4 *normal_origin_host = nullptr;

    float *depth_d = nullptr;
    cudaArray *cuArray[JBU_NUM];
    JBUTexObj *jt_d = nullptr;
    JBUParameters *jp_d = nullptr;
    float4 *normal_d = nullptr;
    float4 *normal_origin_cuda = nullptr;

    void CudaRun();
};

/* The reference aborts the process on a CUDA error; the shim records the
 * first error instead so that the harness can report it. */
extern cudaError_t hpm_ref_first_error;
inline void CudaSafeCall(const cudaError_t error, const std::string &, const int)
{
    if (error != cudaSuccess && hpm_ref_first_error == cudaSuccess) {
        hpm_ref_first_error = error;
    }
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
    bool geom_consistency = false;
    bool multi_geometry = false;
    bool planar_prior = false;
};

class HPM {
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
    float *costs_cuda = nullptr;
    curandState *rand_states_cuda = nullptr;
    unsigned int *selected_views_cuda = nullptr;
    float4 *prior_planes_cuda = nullptr;
    unsigned int *plane_masks_cuda = nullptr;
};

/* The reference seeds curand with clock64() (HPM-MVS/HPM.cu:521), which makes
 * every run different.  The shim replaces that one call site with a fixed,
 * host-settable seed so that reference runs are reproducible. */
__device__ unsigned long long hpm_ref_seed;
#define clock64() (hpm_ref_seed)

/*
 * C++ host side of the B200 path, mirroring the reference's HPM class
 * (HPM-MVS/HPM.h:48-84), GenerateSampleList / ProcessProblem / main()
 * (HPM-MVS/main.cpp:4-33, 35-499, 636-677) over the C ABI of
 * include/hpm_b200.h.  Method names, argument meaning and the on-disk layout
 * (images/, cams/%08d_cam.txt, pair.txt in; HPM/2333_%08d/{depths,
 * depths_geom, normals, costs, depths_prior}.dmb out) are the reference's.
 *
 * Differences a caller sees:
 *   - images are float vectors (row-major) instead of cv::Mat;
 *   - failures throw hpm_host::Error instead of printing and exit();
 *   - the planar-prior pyramid of one problem (support points, Delaunay,
 *     KNN prior, JBU) runs inside RunProblem on the device, so the per-stage
 *     methods of the reference that only shuttle cv::Mat between host loops
 *     are not mirrored one by one;
 *   - random streams come from a seed (counter-based) instead of clock64().
 */
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <vector_types.h>

#include "hpm_b200.h"

namespace hpm_host {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &what) : std::runtime_error(what), code(c) {}
};

/* Problem (main.h:54-57). */
struct Problem {
    int ref_image_id = 0;
    std::vector<int> src_image_ids;
};

/* GenerateSampleList (main.cpp:4-33). */
void GenerateSampleList(const std::string &dense_folder, std::vector<Problem> &problems);

class HPM {
public:
    explicit HPM(int device = 0);
    ~HPM();
    HPM(const HPM &) = delete;
    HPM &operator=(const HPM &) = delete;

    /* HPM.cpp:482-577: gray images (images/%08d.{jpg,png,pgm}; JPEG needs the
     * Python front end), cameras, the 3200-pixel cap, the depth range
     * widened x0.6 / x1.2, and in geometric mode the depth maps of the
     * reference and its sources. */
    void InuputInitialization(const std::string &dense_folder, const Problem &problem);
    /* HPM.cpp:579-700: upload to the device; in geometric mode also the
     * previous pass's planes and costs of the reference view. */
    void CudaSpaceInitialization(const std::string &dense_folder, const Problem &problem);
    /* HPM.cu:1906-1957 */
    void RunPatchMatch();
    /* ProcessProblem's device work for the current problem: the plain pass
     * and, with the planar prior, every pyramid level; or the geometric pass. */
    void RunProblem(bool planar_prior, uint64_t seed, int pyramid_levels = -1);

    void SetGeomConsistencyParams(bool multi_geometry = false); /* HPM.cpp:468-475 */
    void SetPlanarPriorParams();                                 /* HPM.cpp:477-480 */
    void SetSeed(uint64_t seed) { params_.seed = seed; }
    /* true (the default): the reference's behaviour everywhere; false fixes
     * the quirks listed at HpmParams in hpm_b200.h (no counterpart in the
     * reference) */
    void SetReferenceCompat(bool on) { params_.fix_quirks = on ? 0 : 1; }

    int GetReferenceImageWidth() const;
    int GetReferenceImageHeight() const;
    const std::vector<float> &GetReferenceImage() const;
    float4 GetPlaneHypothesis(int index) const; /* (world normal, depth) after a pass */
    float GetCost(int index) const;
    /* the full-scale prior depth map of the last RunProblem (depths_prior.dmb) */
    const std::vector<float> &GetPriorDepths() const { return prior_depth_; }
    float GetMinDepth() const { return params_.depth_min; }
    float GetMaxDepth() const { return params_.depth_max; }

    int ComputingMultiScaleSettings(int width, int height) const; /* HPM.cpp:851-860 */
    float4 TransformNormal(float4 plane_hypothesis) const;        /* HPM.cpp:872-880 */
    float4 TransformNormal2RefCam(float4 plane_hypothesis) const; /* HPM.cpp:882-890 */
    float GetDistance2Origin_factor(int2 p, float depth, float4 normal, float factor) const; /* HPM.cpp:892-899 */
    float GetDepthFromPlaneParam_factor(float4 plane_hypothesis, int x, int y, float factor) const; /* HPM.cpp:846-849 */

    /* HPM.cpp:787-809 over hpm_delaunay: triangles (x0,y0,x1,y1,x2,y2) inside
     * [0,w) x [0,h) of the given points (x,y pairs). */
    std::vector<int> DelaunayTriangulation(int w, int h, const std::vector<int> &points) const;
    /* HPM.cpp:1215-1281 over hpm_jbu: coarse depth + world normal (3 floats
     * per pixel) to the reference image's resolution. */
    void JointBilateralUpsampling(const std::vector<float> &guide, const std::vector<float> &src_depth,
                                  const std::vector<float> &src_normal, int s_cols, int s_rows,
                                  std::vector<float> &up_depth, std::vector<float> &up_normal) const;
    /* HPM.cpp:901-921 / 1099-1123: prior planes (4 floats per pixel, ref
     * frame) and masks for the next RunPatchMatch. */
    void SetPlanarPrior(const std::vector<float> &prior_planes, const std::vector<uint32_t> &masks);

    void ReleasePriorCudaMemory();   /* HPM.cpp:1283-1286 */
    void ReleaseProblemCudaMemory(); /* HPM.cpp:1288-1298: the context keeps its arena for the next problem */
    void ReleaseProblemHostMemory(); /* HPM.cpp:1300-1306 */

    hpm_ctx *context() const { return ctx_; }
    const std::vector<HpmCamera> &cameras() const { return cameras_; }

private:
    void check(int rc, const char *what) const;
    void fetch_result();

    hpm_ctx *ctx_ = nullptr;
    HpmParams params_{};
    std::vector<std::vector<float>> images_;
    std::vector<std::vector<float>> depths_;
    std::vector<HpmCamera> cameras_;
    std::vector<float> planes_host_, costs_host_, prior_depth_;
    std::vector<float> seed_planes_, seed_costs_;
};

/* RunFusion (main.cpp:502-633): fuses the depth maps of every problem
 * (depths_geom.dmb with geom_consistency, else depths.dmb) and normals.dmb
 * into dense_folder/HPM/HPM_model.ply; returns the number of points.
 * Colours come from images/ (JPEG, PNG or PGM); an image whose size differs
 * from its depth map is resized as RescaleImageAndCamera does it
 * (HPM.cpp:187-208, OpenCV's 8-bit bilinear, byte for byte). */
long long RunFusion(const std::string &dense_folder, const std::vector<Problem> &problems, bool geom_consistency,
                    int device = 0);
/* The ACMM+NESP variant's RunFusion (ACMM+NESP/windows/main.cpp:154-297,
 * hpm_fuse_acmm: points averaged over at least 2 agreeing sources) over its
 * tree: ACMM_NESP/2333_%08d/ into ACMM_NESP/ACMM_NESP_model.ply. */
long long RunFusionAcmm(const std::string &dense_folder, const std::vector<Problem> &problems, int device = 0);

/* The ACMM+NESP variant's main() minus fusion (ACMM+NESP/windows/main.cpp:
 * 299-384) in one hpm_run_scene_acmm call, then its files for every problem
 * (ACMM_NESP/2333_%08d/{depths_geom,normals,costs}.dmb).  Problem p must have
 * reference view p.  Returns the depth pixels of all reference views. */
long long RunSceneAcmm(const std::string &dense_folder, const std::vector<Problem> &problems, int geom_iterations,
                       uint64_t seed, int device);

/* ProcessProblem (main.cpp:35-499): one reference view, outputs written
 * under dense_folder/HPM/2333_%08d/; returns the depth pixels written. */
long long ProcessProblem(const std::string &dense_folder, const Problem &problem, bool geom_consistency,
                    bool planar_prior, bool multi_geometry = false, uint64_t seed = 0, int pyramid_levels = -1,
                    int device = 0, bool reference_compat = true);

/* main()'s depth estimation (main.cpp:646-674) in one hpm_run_scene_ex
 * call: pass set A, then geom_iterations geometric iterations, over every
 * problem, with the maps kept in device memory between passes; then, for
 * every problem, the files the per-problem loop leaves (depths.dmb,
 * depths_prior.dmb, depths_geom.dmb, normals.dmb, costs.dmb).  Seeds as in
 * that loop (S + p, S + 1000003 (g + 1) + p), hence the same files.  Host
 * memory: about 20 bytes per pixel of each reference view, plus the images.
 * Returns the depth pixels of all reference views. */
long long RunScene(const std::string &dense_folder, const std::vector<Problem> &problems, bool planar_prior,
              int geom_iterations, uint64_t seed, int pyramid_levels, int device, bool reference_compat = true);

/* What main() has finished in a dense folder, so that a run can stop and be
 * resumed (the reference has no such log; its passes only exchange .dmb
 * files).  dense_folder/HPM/progress.txt holds a line naming the run's
 * settings, then one line per finished step, appended and flushed after
 * that step's files are written:
 *   "A <ref_id>"        pass set A of a problem (ProcessProblem)
 *   "G<g> <ref_id>"     geometric iteration g of a problem
 *   "scene"             the whole depth estimation of the scene form
 *   "fusion"            HPM/HPM_model.ply
 * A fresh run (resume false) starts an empty log; resuming a log written
 * with other settings throws.  A step cut off while its files were being
 * written is not in the log and runs again from the files as they are. */
class Progress {
public:
    Progress(const std::string &dense_folder, const std::string &settings, bool resume);
    bool done(const std::string &step) const;
    void mark(const std::string &step);

private:
    std::string path_;
    std::vector<std::string> steps_;
};

}  // namespace hpm_host

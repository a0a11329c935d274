/*
 * HPM class, GenerateSampleList and ProcessProblem over the C ABI; see
 * hpm_host.h for what mirrors what.
 */
#include "hpm_host.h"

#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>

namespace hpm_host {

namespace {

std::string id_path(const std::string &folder, int id, const char *suffix)
{
    std::ostringstream s;
    s << folder << "/" << std::setw(8) << std::setfill('0') << id << suffix;
    return s.str();
}

std::string result_folder(const std::string &dense_folder, int ref_id, const char *tree = "HPM")
{
    std::ostringstream s;
    s << dense_folder << "/" << tree << "/2333_" << std::setw(8) << std::setfill('0') << ref_id;
    return s.str();
}

float4 f4(float x, float y, float z, float w)
{
    float4 r;
    r.x = x;
    r.y = y;
    r.z = z;
    r.w = w;
    return r;
}

bool exists(const std::string &p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

void make_dir(const std::string &p)
{
    if (mkdir(p.c_str(), 0755) != 0 && !exists(p)) throw Error(HPM_ERR_IO, "cannot create " + p);
}

/* images/%08d.jpg in the reference (HPM.cpp:490); .png and .pgm are also
 * accepted, in that order after .jpg. */
std::string image_path(const std::string &dense_folder, int id)
{
    const std::string base = dense_folder + "/images";
    for (const char *ext : {".jpg", ".png", ".pgm"}) {
        const std::string p = id_path(base, id, ext);
        if (exists(p)) return p;
    }
    throw Error(HPM_ERR_IO, "no image for view " + std::to_string(id) + " under " + base);
}

/* Decoded images, kept for the whole process: the reference decodes every
 * view again for each problem and pass (11 views x 3 passes per problem of
 * a plain scene); here each file is decoded once while its size and
 * modification time stay the same.  HPM_IMAGE_CACHE_MB bounds the bytes
 * kept (default 8192, 0 disables); the oldest entries leave first. */
class ImageCache {
public:
    using Pixels = std::shared_ptr<const std::vector<uint8_t>>;

    /* keep false: decode without storing (a file read once) */
    Pixels get(const std::string &path, int channels, int *w, int *h, bool keep = true)
    {
        struct stat st;
        if (stat(path.c_str(), &st) != 0) throw Error(HPM_ERR_IO, "cannot read " + path);
        const std::string key = path + (channels == 3 ? "#bgr" : "#gray");
        {
            std::lock_guard<std::mutex> g(mu_);
            auto it = map_.find(key);
            if (it != map_.end() && it->second.size == (long long)st.st_size &&
                it->second.mtime_ns == mtime_ns(st)) {
                *w = it->second.w;
                *h = it->second.h;
                return it->second.px;
            }
        }
        auto read = channels == 3 ? hpm_read_bgr8 : hpm_read_gray8;
        int rc = read(path.c_str(), nullptr, 0, w, h);
        if (rc != HPM_OK) throw Error(rc, "cannot decode " + path);
        auto px = std::make_shared<std::vector<uint8_t>>((size_t)*w * *h * channels);
        rc = read(path.c_str(), px->data(), px->size(), w, h);
        if (rc != HPM_OK) throw Error(rc, "cannot decode " + path);
        std::lock_guard<std::mutex> g(mu_);
        const size_t cap = cap_bytes();
        if (keep && px->size() <= cap) {
            auto old = map_.find(key);
            if (old != map_.end()) {
                bytes_ -= old->second.px->size();
                map_.erase(old);
            }
            while (bytes_ + px->size() > cap && !map_.empty()) {
                auto oldest = std::min_element(map_.begin(), map_.end(), [](const auto &a, const auto &b) {
                    return a.second.order < b.second.order;
                });
                bytes_ -= oldest->second.px->size();
                map_.erase(oldest);
            }
            map_[key] = Entry{px, *w, *h, (long long)st.st_size, mtime_ns(st), next_++};
            bytes_ += px->size();
        }
        return px;
    }

private:
    struct Entry {
        Pixels px;
        int w, h;
        long long size, mtime_ns;
        unsigned long long order;
    };
    static long long mtime_ns(const struct stat &st) { return (long long)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec; }
    static size_t cap_bytes()
    {
        const char *e = getenv("HPM_IMAGE_CACHE_MB");
        const long long mb = e ? atoll(e) : 8192;
        return mb > 0 ? (size_t)mb << 20 : 0;
    }
    std::mutex mu_;
    std::map<std::string, Entry> map_;
    size_t bytes_ = 0;
    unsigned long long next_ = 0;
};

ImageCache &image_cache()
{
    static ImageCache c;
    return c;
}

std::vector<float> read_image(const std::string &dense_folder, int id, int *w, int *h)
{
    const auto px = image_cache().get(image_path(dense_folder, id), 1, w, h);
    return std::vector<float>(px->begin(), px->end()); /* convertTo(CV_32FC1), HPM.cpp:494 */
}

/* One view as InuputInitialization reads it (HPM.cpp:482-551): the gray
 * image as floats, its camera, both scaled down to the 3200-pixel cap. */
void load_view(const std::string &dense_folder, int id, std::vector<float> &img, HpmCamera &cam)
{
    int w = 0, h = 0;
    img = read_image(dense_folder, id, &w, &h);
    cam = HpmCamera{};
    const std::string cp = id_path(dense_folder + "/cams", id, "_cam.txt");
    int rc = hpm_read_camera(cp.c_str(), &cam);
    if (rc != HPM_OK) throw Error(rc, "cannot read " + cp);
    const int cap = 3200; /* HPM.cpp:525-551 */
    if (w > cap || h > cap) {
        const float factor = std::min((float)cap / w, (float)cap / h);
        const int nw = (int)std::round(w * factor), nh = (int)std::round(h * factor);
        const float sx = nw / (float)w, sy = nh / (float)h;
        std::vector<float> scaled((size_t)nw * nh);
        rc = hpm_resize_linear(img.data(), w, h, 1, scaled.data(), nw, nh);
        if (rc != HPM_OK) throw Error(rc, "image cap");
        img.swap(scaled);
        cam.K[0] *= sx;
        cam.K[2] *= sx;
        cam.K[4] *= sy;
        cam.K[5] *= sy;
        w = nw;
        h = nh;
    }
    cam.width = w;
    cam.height = h;
}

/* f(i) for i in [0, n) on up to `threads` host threads; the first exception
 * is rethrown */
template <typename F>
void parallel_for(size_t n, unsigned threads, F f)
{
    std::atomic<size_t> next{0};
    std::vector<std::exception_ptr> errors(n);
    auto run = [&] {
        for (size_t i; (i = next.fetch_add(1)) < n;) {
            try {
                f(i);
            } catch (...) {
                errors[i] = std::current_exception();
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < std::min<size_t>(threads, n); ++t) pool.emplace_back(run);
    run();
    for (auto &t : pool) t.join();
    for (auto &e : errors)
        if (e) std::rethrow_exception(e);
}

std::vector<float> read_dmb(const std::string &path, int *w, int *h, int want_nb)
{
    int nb = 0;
    int rc = hpm_read_dmb(path.c_str(), nullptr, 0, h, w, &nb);
    if (rc != HPM_OK || nb != want_nb) throw Error(rc ? rc : HPM_ERR_IO, "cannot read " + path);
    std::vector<float> v((size_t)*w * *h * nb);
    rc = hpm_read_dmb(path.c_str(), v.data(), v.size(), h, w, &nb);
    if (rc != HPM_OK) throw Error(rc, "cannot read " + path);
    return v;
}

void write_dmb(const std::string &path, const std::vector<float> &v, int w, int h, int nb)
{
    const int rc = hpm_write_dmb(path.c_str(), v.data(), h, w, nb);
    if (rc != HPM_OK) throw Error(rc, "cannot write " + path);
}

}  // namespace

void GenerateSampleList(const std::string &dense_folder, std::vector<Problem> &problems)
{
    const std::string path = dense_folder + "/pair.txt";
    int n = 0;
    int rc = hpm_read_pair(path.c_str(), &n, nullptr, nullptr, nullptr, 0);
    if (rc != HPM_OK) throw Error(rc, "cannot read " + path);
    std::vector<int> refs(n), counts(n), srcs((size_t)n * (HPM_MAX_IMAGES - 1));
    rc = hpm_read_pair(path.c_str(), &n, refs.data(), counts.data(), srcs.data(), n);
    if (rc != HPM_OK) throw Error(rc, "cannot read " + path);
    problems.clear();
    for (int i = 0; i < n; ++i) {
        Problem p;
        p.ref_image_id = refs[i];
        p.src_image_ids.assign(srcs.begin() + (size_t)i * (HPM_MAX_IMAGES - 1),
                               srcs.begin() + (size_t)i * (HPM_MAX_IMAGES - 1) + counts[i]);
        problems.push_back(p);
    }
}

HPM::HPM(int device)
{
    hpm_default_params(&params_);
    check(hpm_create(&ctx_, device), "hpm_create");
}

HPM::~HPM()
{
    if (ctx_) hpm_destroy(ctx_);
}

void HPM::check(int rc, const char *what) const
{
    if (rc == HPM_OK) return;
    std::string msg = what;
    if (ctx_) msg += std::string(": ") + hpm_last_error(ctx_);
    throw Error(rc, msg);
}

void HPM::InuputInitialization(const std::string &dense_folder, const Problem &problem)
{
    images_.clear();
    cameras_.clear();
    std::vector<int> ids{problem.ref_image_id};
    ids.insert(ids.end(), problem.src_image_ids.begin(), problem.src_image_ids.end());
    if ((int)ids.size() > HPM_MAX_IMAGES) throw Error(HPM_ERR_ARG, "more than 32 source images");
    const size_t n = ids.size();
    images_.resize(n);
    cameras_.resize(n);
    /* the views of a problem are read and decoded on threads of their own */
    parallel_for(n, (unsigned)n, [&](size_t i) { load_view(dense_folder, ids[i], images_[i], cameras_[i]); });
    params_.depth_min = cameras_[0].depth_min * 0.6f;
    params_.depth_max = cameras_[0].depth_max * 1.2f;
    depths_.clear();
    seed_planes_.clear();
    seed_costs_.clear();
    if (params_.geom_consistency) {
        const char *suffix = params_.multi_geometry ? "/depths_geom.dmb" : "/depths.dmb";
        for (size_t i = 0; i < ids.size(); ++i) {
            int w = 0, h = 0;
            depths_.push_back(read_dmb(result_folder(dense_folder, ids[i]) + suffix, &w, &h, 1));
            if (w != cameras_[i].width || h != cameras_[i].height)
                throw Error(HPM_ERR_ARG, "depth map size differs from its image: view " + std::to_string(ids[i]));
        }
    }
}

void HPM::CudaSpaceInitialization(const std::string &dense_folder, const Problem &problem)
{
    std::vector<const float *> ptrs;
    for (auto &img : images_) ptrs.push_back(img.data());
    check(hpm_set_views(ctx_, ptrs.data(), cameras_.data(), (int)images_.size()), "hpm_set_views");
    if (!params_.geom_consistency) return;
    std::vector<const float *> dptrs;
    for (auto &d : depths_) dptrs.push_back(d.data());
    check(hpm_set_geom_depths(ctx_, dptrs.data()), "hpm_set_geom_depths");
    /* the previous pass's hypotheses of the reference view (HPM.cpp:661-697) */
    const std::string folder = result_folder(dense_folder, problem.ref_image_id);
    int w = 0, h = 0;
    const std::vector<float> normal = read_dmb(folder + "/normals.dmb", &w, &h, 3);
    const std::vector<float> cost = read_dmb(folder + "/costs.dmb", &w, &h, 1);
    const std::vector<float> &depth = depths_[0];
    if (w != cameras_[0].width || h != cameras_[0].height) throw Error(HPM_ERR_ARG, "normals.dmb size");
    seed_planes_.resize((size_t)4 * w * h);
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        seed_planes_[4 * i] = normal[3 * i];
        seed_planes_[4 * i + 1] = normal[3 * i + 1];
        seed_planes_[4 * i + 2] = normal[3 * i + 2];
        seed_planes_[4 * i + 3] = depth[i];
    }
    seed_costs_ = cost;
    check(hpm_set_hypotheses(ctx_, seed_planes_.data(), seed_costs_.data()), "hpm_set_hypotheses");
}

void HPM::fetch_result()
{
    const size_t n = (size_t)GetReferenceImageWidth() * GetReferenceImageHeight();
    planes_host_.resize(4 * n);
    costs_host_.resize(n);
    check(hpm_get_result(ctx_, planes_host_.data(), costs_host_.data()), "hpm_get_result");
}

void HPM::RunPatchMatch()
{
    check(hpm_run_patchmatch(ctx_, &params_), "hpm_run_patchmatch");
    fetch_result();
}

void HPM::RunProblem(bool planar_prior, uint64_t seed, int pyramid_levels)
{
    const size_t n = (size_t)GetReferenceImageWidth() * GetReferenceImageHeight();
    std::vector<float> depth(n), normal(3 * n), cost(n);
    prior_depth_.assign(n, 0.0f);
    HpmProblemOpts o{};
    o.planar_prior = planar_prior && !params_.geom_consistency;
    o.geom_consistency = params_.geom_consistency;
    o.multi_geometry = params_.multi_geometry;
    o.seed = seed;
    o.pyramid_levels = pyramid_levels;
    o.fix_quirks = params_.fix_quirks;
    check(hpm_process_problem(ctx_, &o, depth.data(), normal.data(), cost.data(), prior_depth_.data()),
          "hpm_process_problem");
    planes_host_.resize(4 * n);
    costs_host_ = cost;
    for (size_t i = 0; i < n; ++i) {
        planes_host_[4 * i] = normal[3 * i];
        planes_host_[4 * i + 1] = normal[3 * i + 1];
        planes_host_[4 * i + 2] = normal[3 * i + 2];
        planes_host_[4 * i + 3] = depth[i];
    }
}

void HPM::SetGeomConsistencyParams(bool multi_geometry)
{
    params_.geom_consistency = 1;
    params_.max_iterations = 2; /* recorded, not used: every pass runs 3 iterations (HPM.cu:1933) */
    if (multi_geometry) params_.multi_geometry = 1;
}

void HPM::SetPlanarPriorParams() { params_.planar_prior = 1; }

int HPM::GetReferenceImageWidth() const { return cameras_.empty() ? 0 : cameras_[0].width; }
int HPM::GetReferenceImageHeight() const { return cameras_.empty() ? 0 : cameras_[0].height; }

const std::vector<float> &HPM::GetReferenceImage() const
{
    if (images_.empty()) throw Error(HPM_ERR_STATE, "GetReferenceImage before InuputInitialization");
    return images_[0];
}

float4 HPM::GetPlaneHypothesis(int index) const
{
    if (index < 0 || (size_t)index * 4 >= planes_host_.size()) throw Error(HPM_ERR_ARG, "plane index");
    return f4(planes_host_[4 * (size_t)index], planes_host_[4 * (size_t)index + 1],
                       planes_host_[4 * (size_t)index + 2], planes_host_[4 * (size_t)index + 3]);
}

float HPM::GetCost(int index) const
{
    if (index < 0 || (size_t)index >= costs_host_.size()) throw Error(HPM_ERR_ARG, "cost index");
    return costs_host_[index];
}

int HPM::ComputingMultiScaleSettings(int width, int height) const
{
    int max_size = std::max(width, height), k = 0;
    while (max_size > 1000) {
        max_size /= 2;
        k++;
    }
    return k;
}

float4 HPM::TransformNormal(float4 p) const
{
    const float *R = cameras_.at(0).R;
    return f4(R[0] * p.x + R[3] * p.y + R[6] * p.z, R[1] * p.x + R[4] * p.y + R[7] * p.z,
                       R[2] * p.x + R[5] * p.y + R[8] * p.z, p.w);
}

float4 HPM::TransformNormal2RefCam(float4 p) const
{
    const float *R = cameras_.at(0).R;
    return f4(R[0] * p.x + R[1] * p.y + R[2] * p.z, R[3] * p.x + R[4] * p.y + R[5] * p.z,
                       R[6] * p.x + R[7] * p.y + R[8] * p.z, p.w);
}

float HPM::GetDistance2Origin_factor(int2 p, float depth, float4 normal, float /*factor: unused, as in the reference*/) const
{
    const float *K = cameras_.at(0).K;
    const float X0 = depth * (p.x - K[2]) / K[0], X1 = depth * (p.y - K[5]) / K[4], X2 = depth;
    return -(normal.x * X0 + normal.y * X1 + normal.z * X2);
}

float HPM::GetDepthFromPlaneParam_factor(float4 n, int x, int y, float factor) const
{
    const float *K = cameras_.at(0).K;
    return -n.w * (K[0] * factor) /
           ((x - K[2] * factor) * n.x + (K[0] / K[4]) * (y - K[5] * factor) * n.y + K[0] * factor * n.z);
}

std::vector<int> HPM::DelaunayTriangulation(int w, int h, const std::vector<int> &points) const
{
    const int n = (int)points.size() / 2;
    const int cnt = hpm_delaunay(points.data(), n, w, h, nullptr, 0);
    if (cnt < 0) throw Error(cnt, "hpm_delaunay");
    std::vector<int> tris((size_t)6 * cnt);
    const int got = hpm_delaunay(points.data(), n, w, h, tris.data(), cnt);
    if (got < 0) throw Error(got, "hpm_delaunay");
    tris.resize((size_t)6 * got);
    return tris;
}

void HPM::JointBilateralUpsampling(const std::vector<float> &guide, const std::vector<float> &src_depth,
                                   const std::vector<float> &src_normal, int s_cols, int s_rows,
                                   std::vector<float> &up_depth, std::vector<float> &up_normal) const
{
    const int cols = GetReferenceImageWidth(), rows = GetReferenceImageHeight();
    up_depth.assign((size_t)cols * rows, 0.0f);
    up_normal.assign((size_t)3 * cols * rows, 0.0f);
    check(hpm_jbu(ctx_, guide.data(), cols, rows, src_depth.data(), src_normal.data(), s_cols, s_rows,
                  up_depth.data(), up_normal.data()),
          "hpm_jbu");
}

void HPM::SetPlanarPrior(const std::vector<float> &prior_planes, const std::vector<uint32_t> &masks)
{
    check(hpm_set_prior(ctx_, prior_planes.data(), masks.data()), "hpm_set_prior");
    params_.planar_prior = 1;
}

void HPM::ReleasePriorCudaMemory()
{
    hpm_clear_prior(ctx_);
    params_.planar_prior = 0;
}

void HPM::ReleaseProblemCudaMemory() {}

void HPM::ReleaseProblemHostMemory()
{
    std::vector<std::vector<float>>().swap(images_);
    std::vector<std::vector<float>>().swap(depths_);
    std::vector<float>().swap(seed_planes_);
    std::vector<float>().swap(seed_costs_);
}

static long long fuse_tree(const std::string &dense_folder, const std::vector<Problem> &problems,
                           bool geom_consistency, int device, const char *tree, const char *ply_name, bool acmm);

long long RunFusion(const std::string &dense_folder, const std::vector<Problem> &problems, bool geom_consistency,
                    int device)
{
    return fuse_tree(dense_folder, problems, geom_consistency, device, "HPM", "HPM_model.ply", false);
}

long long RunFusionAcmm(const std::string &dense_folder, const std::vector<Problem> &problems, int device)
{
    return fuse_tree(dense_folder, problems, true, device, "ACMM_NESP", "ACMM_NESP_model.ply", true);
}

static long long fuse_tree(const std::string &dense_folder, const std::vector<Problem> &problems,
                           bool geom_consistency, int device, const char *tree, const char *ply_name, bool acmm)
{
    const int n = (int)problems.size();
    std::vector<HpmCamera> cams(n);
    std::vector<std::vector<float>> depths(n), normals(n);
    std::vector<std::vector<uint8_t>> colors(n);
    std::vector<int> refs(n), counts(n), srcs((size_t)n * (HPM_MAX_IMAGES - 1), 0);
    for (int i = 0; i < n; ++i) {
        /* the reference indexes views by problem order (main.cpp:517-546) */
        const int id = problems[i].ref_image_id;
        const std::string folder = result_folder(dense_folder, id, tree);
        int w = 0, h = 0;
        depths[i] = read_dmb(folder + (geom_consistency ? "/depths_geom.dmb" : "/depths.dmb"), &w, &h, 1);
        normals[i] = read_dmb(folder + "/normals.dmb", &w, &h, 3);
        HpmCamera cam{};
        const std::string cp = id_path(dense_folder + "/cams", id, "_cam.txt");
        int rc = hpm_read_camera(cp.c_str(), &cam);
        if (rc != HPM_OK) throw Error(rc, "cannot read " + cp);
        int iw = 0, ih = 0;
        const std::string ip = image_path(dense_folder, id);
        std::vector<uint8_t> bgr(*image_cache().get(ip, 3, &iw, &ih, false));
        if (iw != w || ih != h) {
            /* RescaleImageAndCamera, HPM.cpp:187-208: OpenCV's 8-bit bilinear */
            std::vector<uint8_t> g((size_t)3 * w * h);
            int r2 = hpm_resize_linear_u8(bgr.data(), iw, ih, 3, g.data(), w, h);
            if (r2 != HPM_OK) throw Error(r2, "colour resize");
            bgr.swap(g);
            const float sx = w / (float)iw, sy = h / (float)ih;
            cam.K[0] *= sx;
            cam.K[2] *= sx;
            cam.K[4] *= sy;
            cam.K[5] *= sy;
        }
        cam.width = w;
        cam.height = h;
        cams[i] = cam;
        colors[i] = std::move(bgr);
        refs[i] = i;
        counts[i] = (int)problems[i].src_image_ids.size();
        for (int j = 0; j < counts[i]; ++j) srcs[(size_t)i * (HPM_MAX_IMAGES - 1) + j] = problems[i].src_image_ids[j];
    }
    std::vector<const float *> dp(n), np_(n);
    std::vector<const uint8_t *> cp(n);
    size_t cap = 0;
    for (int i = 0; i < n; ++i) {
        dp[i] = depths[i].data();
        np_[i] = normals[i].data();
        cp[i] = colors[i].data();
        cap += depths[i].size();
    }
    std::vector<float> xyz(3 * cap), nrm(3 * cap);
    std::vector<uint8_t> col(3 * cap);
    long long count = 0;
    int rc = (acmm ? hpm_fuse_acmm : hpm_fuse)(device, n, cams.data(), dp.data(), np_.data(), cp.data(), n,
                                               refs.data(), counts.data(), srcs.data(), xyz.data(), nrm.data(),
                                               col.data(), (long long)cap, &count);
    if (rc != HPM_OK) throw Error(rc, acmm ? "hpm_fuse_acmm" : "hpm_fuse");
    const std::string ply = dense_folder + "/" + tree + "/" + ply_name;
    rc = hpm_write_ply(ply.c_str(), count, xyz.data(), nrm.data(), col.data());
    if (rc != HPM_OK) throw Error(rc, "cannot write " + ply);
    return count;
}

long long ProcessProblem(const std::string &dense_folder, const Problem &problem, bool geom_consistency,
                    bool planar_prior, bool multi_geometry, uint64_t seed, int pyramid_levels, int device,
                    bool reference_compat)
{
    std::cout << "Processing image " << std::setw(8) << std::setfill('0') << problem.ref_image_id << "..."
              << std::endl;
    const std::string folder = result_folder(dense_folder, problem.ref_image_id);
    make_dir(dense_folder + "/HPM");
    make_dir(folder);
    HPM hpm(device);
    hpm.SetReferenceCompat(reference_compat);
    if (geom_consistency) hpm.SetGeomConsistencyParams(multi_geometry);
    hpm.InuputInitialization(dense_folder, problem);
    hpm.CudaSpaceInitialization(dense_folder, problem);
    hpm.RunProblem(planar_prior, seed, pyramid_levels);

    const int w = hpm.GetReferenceImageWidth(), h = hpm.GetReferenceImageHeight();
    const size_t n = (size_t)w * h;
    std::vector<float> depths(n), normals(3 * n), costs(n);
    for (size_t i = 0; i < n; ++i) {
        const float4 p = hpm.GetPlaneHypothesis((int)i);
        depths[i] = p.w;
        normals[3 * i] = p.x;
        normals[3 * i + 1] = p.y;
        normals[3 * i + 2] = p.z;
        costs[i] = hpm.GetCost((int)i);
    }
    if (planar_prior && !geom_consistency) write_dmb(folder + "/depths_prior.dmb", hpm.GetPriorDepths(), w, h, 1);
    write_dmb(folder + (geom_consistency ? "/depths_geom.dmb" : "/depths.dmb"), depths, w, h, 1);
    write_dmb(folder + "/normals.dmb", normals, w, h, 3);
    write_dmb(folder + "/costs.dmb", costs, w, h, 1);
    std::cout << "Processing image " << std::setw(8) << std::setfill('0') << problem.ref_image_id << " done!"
              << std::endl;
    return (long long)n;
}

long long RunScene(const std::string &dense_folder, const std::vector<Problem> &problems, bool planar_prior,
              int geom_iterations, uint64_t seed, int pyramid_levels, int device, bool reference_compat)
{
    /* every view a problem names, numbered in order of appearance */
    std::map<int, int> index;
    std::vector<int> ids;
    auto add = [&](int id) {
        if (index.emplace(id, (int)ids.size()).second) ids.push_back(id);
    };
    for (const Problem &p : problems) {
        if ((int)p.src_image_ids.size() + 1 > HPM_MAX_IMAGES) throw Error(HPM_ERR_ARG, "more than 32 source images");
        add(p.ref_image_id);
        for (int sid : p.src_image_ids) add(sid);
    }
    const size_t n = ids.size(), np = problems.size();
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<float>> images(n);
    std::vector<HpmCamera> cams(n);
    parallel_for(n, threads, [&](size_t i) { load_view(dense_folder, ids[i], images[i], cams[i]); });
    std::vector<int> refs(np), counts(np), srcs(np * (HPM_MAX_IMAGES - 1), 0);
    for (size_t p = 0; p < np; ++p) {
        refs[p] = index[problems[p].ref_image_id];
        counts[p] = (int)problems[p].src_image_ids.size();
        for (int j = 0; j < counts[p]; ++j) srcs[p * (HPM_MAX_IMAGES - 1) + j] = index[problems[p].src_image_ids[j]];
    }
    /* outputs for the views that are references: final depth, normal and
     * cost, pass set A's depth and the prior depth */
    std::vector<std::vector<float>> depth(n), normal(n), cost(n), pass(n), prior(n);
    std::vector<const float *> img_ptr(n);
    std::vector<float *> pd(n, nullptr), pn(n, nullptr), pc(n, nullptr), pp(n, nullptr), pr(n, nullptr);
    for (size_t i = 0; i < n; ++i) img_ptr[i] = images[i].data();
    for (size_t p = 0; p < np; ++p) {
        const int v = refs[p];
        const size_t npx = (size_t)cams[v].width * cams[v].height;
        depth[v].resize(npx);
        normal[v].resize(3 * npx);
        cost[v].resize(npx);
        pass[v].resize(npx);
        if (planar_prior) prior[v].resize(npx);
        pd[v] = depth[v].data();
        pn[v] = normal[v].data();
        pc[v] = cost[v].data();
        pp[v] = pass[v].data();
        if (planar_prior) pr[v] = prior[v].data();
    }
    hpm_ctx *ctx = nullptr;
    int rc = hpm_create(&ctx, device);
    if (rc != HPM_OK) throw Error(rc, "hpm_create");
    struct Destroy {
        hpm_ctx *c;
        ~Destroy() { hpm_destroy(c); }
    } destroy{ctx};
    const HpmSceneOpts o = {planar_prior ? 1 : 0, geom_iterations, seed, pyramid_levels, 0, reference_compat ? 0 : 1,
                            0};
    rc = hpm_run_scene_ex(ctx, (int)n, img_ptr.data(), cams.data(), (int)np, refs.data(), counts.data(), srcs.data(),
                          &o, pd.data(), pn.data(), pc.data(), pp.data(), pr.data());
    if (rc != HPM_OK) throw Error(rc, std::string("hpm_run_scene_ex: ") + hpm_last_error(ctx));
    /* the files ProcessProblem leaves behind for each reference view:
     * pass set A's depth, prior depth, normal and cost, then the geometric
     * passes' depth, normal and cost over them (main.cpp:481-497) */
    make_dir(dense_folder + "/HPM");
    parallel_for(np, threads, [&](size_t p) {
        const int v = refs[p], w = cams[v].width, h = cams[v].height;
        const std::string folder = result_folder(dense_folder, problems[p].ref_image_id);
        make_dir(folder);
        if (planar_prior) write_dmb(folder + "/depths_prior.dmb", prior[v], w, h, 1);
        write_dmb(folder + "/depths.dmb", pass[v], w, h, 1);
        if (geom_iterations > 0) write_dmb(folder + "/depths_geom.dmb", depth[v], w, h, 1);
        write_dmb(folder + "/normals.dmb", normal[v], w, h, 3);
        write_dmb(folder + "/costs.dmb", cost[v], w, h, 1);
    });
    std::cout << "Processed " << np << " problems (" << n << " views) in one scene run" << std::endl;
    long long px = 0;
    for (size_t p = 0; p < np; ++p) px += (long long)cams[refs[p]].width * cams[refs[p]].height;
    return px;
}

Progress::Progress(const std::string &dense_folder, const std::string &settings, bool resume)
    : path_(dense_folder + "/HPM/progress.txt")
{
    make_dir(dense_folder + "/HPM");
    const std::string head = "settings " + settings;
    if (resume) {
        std::ifstream in(path_);
        std::string line;
        if (in && std::getline(in, line)) {
            if (line != head) throw Error(HPM_ERR_ARG, "cannot resume: " + path_ + " was written with " + line);
            while (std::getline(in, line))
                if (!line.empty()) steps_.push_back(line);
            return;
        }
    }
    std::ofstream out(path_, std::ios::trunc);
    out << head << "\n";
    out.flush();
    if (!out) throw Error(HPM_ERR_IO, "cannot write " + path_);
}

long long RunSceneAcmm(const std::string &dense_folder, const std::vector<Problem> &problems, int geom_iterations,
                       uint64_t seed, int device)
{
    const size_t n = problems.size();
    for (size_t p = 0; p < n; ++p) {
        if (problems[p].ref_image_id != (int)p)
            throw Error(HPM_ERR_ARG, "the ACMM+NESP variant needs pair.txt to list views 0, 1, ... in order (the "
                                     "reference looks a source's scale up by its image id)");
        if ((int)problems[p].src_image_ids.size() + 1 > HPM_MAX_IMAGES)
            throw Error(HPM_ERR_ARG, "more than 32 source images");
    }
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<float>> images(n);
    std::vector<HpmCamera> cams(n);
    parallel_for(n, threads, [&](size_t i) { load_view(dense_folder, (int)i, images[i], cams[i]); });
    std::vector<int> refs(n), counts(n), srcs(n * (HPM_MAX_IMAGES - 1), 0);
    std::vector<std::vector<float>> depth(n), normal(n), cost(n);
    std::vector<const float *> img_ptr(n);
    std::vector<float *> pd(n), pn(n), pc(n);
    for (size_t p = 0; p < n; ++p) {
        refs[p] = (int)p;
        counts[p] = (int)problems[p].src_image_ids.size();
        for (int j = 0; j < counts[p]; ++j) srcs[p * (HPM_MAX_IMAGES - 1) + j] = problems[p].src_image_ids[j];
        const size_t npx = (size_t)cams[p].width * cams[p].height;
        depth[p].resize(npx);
        normal[p].resize(3 * npx);
        cost[p].resize(npx);
        img_ptr[p] = images[p].data();
        pd[p] = depth[p].data();
        pn[p] = normal[p].data();
        pc[p] = cost[p].data();
    }
    hpm_ctx *ctx = nullptr;
    int rc = hpm_create(&ctx, device);
    if (rc != HPM_OK) throw Error(rc, "hpm_create");
    struct Destroy {
        hpm_ctx *c;
        ~Destroy() { hpm_destroy(c); }
    } destroy{ctx};
    const HpmAcmmOpts o = {geom_iterations, seed, 0, 0, 0};
    rc = hpm_run_scene_acmm(ctx, (int)n, img_ptr.data(), cams.data(), (int)n, refs.data(), counts.data(),
                            srcs.data(), &o, pd.data(), pn.data(), pc.data());
    if (rc != HPM_OK) throw Error(rc, std::string("hpm_run_scene_acmm: ") + hpm_last_error(ctx));
    /* the files the variant's ProcessProblem leaves (ACMM+NESP/windows/main.cpp:96-121) */
    make_dir(dense_folder + "/ACMM_NESP");
    long long pixels = 0;
    for (size_t p = 0; p < n; ++p) pixels += (long long)depth[p].size();
    parallel_for(n, threads, [&](size_t p) {
        const int w = cams[p].width, h = cams[p].height;
        const std::string folder = result_folder(dense_folder, (int)p, "ACMM_NESP");
        make_dir(folder);
        write_dmb(folder + (geom_iterations > 0 ? "/depths_geom.dmb" : "/depths.dmb"), depth[p], w, h, 1);
        write_dmb(folder + "/normals.dmb", normal[p], w, h, 3);
        write_dmb(folder + "/costs.dmb", cost[p], w, h, 1);
    });
    return pixels;
}

bool Progress::done(const std::string &step) const
{
    return std::find(steps_.begin(), steps_.end(), step) != steps_.end();
}

void Progress::mark(const std::string &step)
{
    std::ofstream out(path_, std::ios::app);
    out << step << "\n";
    out.flush();
    if (!out) throw Error(HPM_ERR_IO, "cannot write " + path_);
    steps_.push_back(step);
}

}  // namespace hpm_host

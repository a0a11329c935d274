/*
 * Stub declarations that let the reference's own RunFusion (HPM-MVS/main.cpp
 * 502-633) and the HPM.cpp helpers it calls (ReadCamera, readDepthDmb,
 * readNormalDmb, RescaleImageAndCamera, Get3DPointonWorld, ProjectonCamera,
 * GetAngle, StoreColorPlyFileBinaryPointCloud: HPM.cpp:135-456) compile on
 * the host without OpenCV or PCL; likewise the ACMM+NESP variant's RunFusion
 * (ACMM+NESP/windows/main.cpp:154-297) with its ACMM.cpp helpers
 * (ACMM.cpp:137-422).
 *
 * TEST INFRASTRUCTURE ONLY: the library built from this header is the
 * checker of the fusion oracle (oracle/_ref/libfusion_ref.so), never the
 * product.  The reference's source text is extracted at build time from
 * where it lies (oracle/Makefile, target `fusion`); nothing of it is kept in
 * the repository.
 *
 * Restated because the reference's code reads them: Camera (main.h:44-52),
 * Problem (main.h:54-57), PointList (main.h:64-68).  cv::Mat / cv::Mat_ keep
 * rows x cols elements of one type in one contiguous buffer; cv::imread reads
 * the test's raw image files (a "RAW3" header, height and width as int32,
 * then BGR bytes row by row) whatever their extension.
 */
#pragma once

#include <cuda_runtime.h>
#include <vector_functions.h>
#include <vector_types.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

struct Camera {
    float K[9];
    float R[9];
    float t[3];
    int height;
    int width;
    float depth_min;
    float depth_max;
};

struct Problem {
    int ref_image_id;
    std::vector<int> src_image_ids;
};

struct PointList {
    float3 coord;
    float3 normal;
    float3 color;
};

typedef unsigned char uchar;

namespace cv {

enum { CV_8UC1_ = 0 };
constexpr int IMREAD_COLOR = 1;
constexpr int INTER_LINEAR = 1;

struct Vec3b {
    uchar v[3];
    uchar &operator[](int i) { return v[i]; }
    const uchar &operator[](int i) const { return v[i]; }
};

struct Vec3f {
    float v[3];
    float &operator[](int i) { return v[i]; }
    const float &operator[](int i) const { return v[i]; }
};

/* Element-wise sum, and division by a scalar as OpenCV's Vec does it
 * (core/matx.hpp: a multiplication by the float reciprocal); used by the
 * ACMM+NESP variant's RunFusion (ACMM+NESP/windows/main.cpp:259, 275). */
inline Vec3f operator+(const Vec3f &a, const Vec3f &b)
{
    Vec3f r;
    for (int i = 0; i < 3; ++i) r.v[i] = a.v[i] + b.v[i];
    return r;
}
inline Vec3f &operator/=(Vec3f &a, float alpha)
{
    const float ialpha = 1.f / alpha;
    for (int i = 0; i < 3; ++i) a.v[i] = a.v[i] * ialpha;
    return a;
}

struct Size {
    int width, height;
    Size(int w, int h) : width(w), height(h) {}
};

class Mat {
public:
    int rows = 0, cols = 0, esize = 1;
    uchar *data = nullptr;
    std::shared_ptr<std::vector<uchar>> buf;

    Mat() {}
    Mat(int r, int c, int elem_size) : rows(r), cols(c), esize(elem_size)
    {
        buf = std::make_shared<std::vector<uchar>>((size_t)r * c * elem_size, 0);
        data = buf->data();
    }
    static Mat zeros(int r, int c, int elem_size) { return Mat(r, c, elem_size); }
    template <typename T>
    T &at(int r, int c)
    {
        return reinterpret_cast<T *>(data)[(size_t)r * cols + c];
    }
    template <typename T>
    const T &at(int r, int c) const
    {
        return reinterpret_cast<const T *>(data)[(size_t)r * cols + c];
    }
    Mat clone() const
    {
        Mat m(rows, cols, esize);
        if (data) memcpy(m.data, data, (size_t)rows * cols * esize);
        return m;
    }
};

template <typename T>
class Mat_ : public Mat {
public:
    Mat_() {}
    Mat_(const Mat &m) : Mat(m) {}
    Mat_ &operator=(const Mat &m)
    {
        Mat::operator=(m);
        return *this;
    }
    Mat_ clone() const { return Mat_(Mat::clone()); }
};

/* element sizes stand in for the OpenCV type codes the helpers pass */
}  // namespace cv

#define CV_8UC1 1
#define CV_32F 4
#define CV_32FC3 12

namespace cv {

inline Mat imread(const std::string &path, int)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return Mat();
    char magic[4];
    int32_t h = 0, w = 0;
    if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "RAW3", 4) != 0 || fread(&h, 4, 1, f) != 1 ||
        fread(&w, 4, 1, f) != 1) {
        fclose(f);
        return Mat();
    }
    Mat m(h, w, 3);
    const size_t n = (size_t)h * w * 3;
    if (fread(m.data, 1, n, f) != n) m = Mat();
    fclose(f);
    return m;
}

template <typename A, typename B>
inline void resize(const A &, B &, Size, double, double, int)
{
    /* the checker's scenes keep images at the size of their depth maps */
    fprintf(stderr, "fusion checker: cv::resize is not provided\n");
    abort();
}

}  // namespace cv

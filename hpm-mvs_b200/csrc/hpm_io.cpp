/*
 * Drop-in file formats of HPM-MVS: .dmb maps, cams/%08d_cam.txt, pair.txt.
 *
 *   .dmb      int32 type (=1), int32 h, int32 w, int32 nb, then h*w*nb float32
 *             row-major, channels interleaved (HPM.cpp:270-401)
 *   cam file  token "extrinsic", 4x4 [R|t] row-major, token "intrinsic", 3x3 K,
 *             then depth_min interval depth_num depth_max (ReadCamera,
 *             HPM.cpp:160-185)
 *   pair.txt  N, then per problem: ref_id, n_src, n_src x (id score); sources
 *             with score <= 0 are dropped (GenerateSampleList, main.cpp:4-33)
 *
 * Unlike the reference (which prints and carries on, or dereferences NULL on
 * a failed fopen), every failure returns HPM_ERR_IO.
 */
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>

#include "hpm_b200.h"

extern "C" {

int hpm_write_dmb(const char *path, const float *data, int h, int w, int nb)
{
    if (!path || !data || h < 0 || w < 0 || nb < 1) return HPM_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return HPM_ERR_IO;
    const int32_t hdr[4] = {1, h, w, nb};
    bool ok = fwrite(hdr, sizeof(int32_t), 4, f) == 4;
    const size_t n = (size_t)h * w * nb;
    ok = ok && fwrite(data, sizeof(float), n, f) == n;
    ok = (fclose(f) == 0) && ok;
    return ok ? HPM_OK : HPM_ERR_IO;
}

int hpm_read_dmb(const char *path, float *data, size_t cap, int *h, int *w, int *nb)
{
    if (!path) return HPM_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return HPM_ERR_IO;
    int32_t hdr[4] = {-1, 0, 0, 0};
    if (fread(hdr, sizeof(int32_t), 4, f) != 4 || hdr[0] != 1 || hdr[1] < 0 || hdr[2] < 0 || hdr[3] < 1) {
        fclose(f);
        return HPM_ERR_IO;
    }
    if (h) *h = hdr[1];
    if (w) *w = hdr[2];
    if (nb) *nb = hdr[3];
    int rc = HPM_OK;
    if (data) {
        const size_t n = (size_t)hdr[1] * hdr[2] * hdr[3];
        if (n > cap)
            rc = HPM_ERR_ARG;
        else if (fread(data, sizeof(float), n, f) != n)
            rc = HPM_ERR_IO;
    }
    fclose(f);
    return rc;
}

int hpm_read_camera(const char *path, HpmCamera *cam)
{
    if (!path || !cam) return HPM_ERR_ARG;
    std::ifstream file(path);
    if (!file) return HPM_ERR_IO;
    memset(cam, 0, sizeof(*cam));
    std::string token;
    file >> token;
    if (token != "extrinsic") return HPM_ERR_IO;
    for (int i = 0; i < 3; ++i) file >> cam->R[3 * i + 0] >> cam->R[3 * i + 1] >> cam->R[3 * i + 2] >> cam->t[i];
    float tmp[4];
    file >> tmp[0] >> tmp[1] >> tmp[2] >> tmp[3];
    file >> token;
    if (token != "intrinsic") return HPM_ERR_IO;
    for (int i = 0; i < 3; ++i) file >> cam->K[3 * i + 0] >> cam->K[3 * i + 1] >> cam->K[3 * i + 2];
    float interval = 0.0f, depth_num = 0.0f;
    file >> cam->depth_min >> interval >> depth_num >> cam->depth_max;
    if (file.fail()) return HPM_ERR_IO;
    return HPM_OK;
}

int hpm_read_pair(const char *path, int *n_out, int *ref_ids, int *src_counts, int *src_ids, int cap)
{
    if (!path || !n_out) return HPM_ERR_ARG;
    std::ifstream file(path);
    if (!file) return HPM_ERR_IO;
    int n = 0;
    file >> n;
    if (file.fail() || n < 0) return HPM_ERR_IO;
    *n_out = n;
    if (!ref_ids && !src_counts && !src_ids) return HPM_OK;
    if (n > cap) return HPM_ERR_ARG;
    for (int i = 0; i < n; ++i) {
        int ref = 0, ns = 0;
        file >> ref >> ns;
        if (file.fail() || ns < 0) return HPM_ERR_IO;
        int kept = 0;
        for (int j = 0; j < ns; ++j) {
            int id = 0;
            float score = 0.0f;
            file >> id >> score;
            if (file.fail()) return HPM_ERR_IO;
            if (score <= 0.0f) continue;
            if (kept < HPM_MAX_IMAGES - 1 && src_ids) src_ids[(size_t)i * (HPM_MAX_IMAGES - 1) + kept] = id;
            kept++;
        }
        if (ref_ids) ref_ids[i] = ref;
        if (src_counts) src_counts[i] = kept < HPM_MAX_IMAGES - 1 ? kept : HPM_MAX_IMAGES - 1;
    }
    return HPM_OK;
}

}  // extern "C"

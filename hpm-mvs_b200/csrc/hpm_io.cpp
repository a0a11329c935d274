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
 *   images    8-bit grayscale as cv::imread(path, IMREAD_GRAYSCALE) returns it
 *             (HPM.cpp:492), and B, G, R as IMREAD_COLOR (main.cpp:523):
 *             JPEG (hpm_jpeg.cpp), binary PGM (P5, maxval 255) and PNG (8-bit
 *             gray, gray+alpha, RGB, RGBA, palette; not interlaced).  PNG
 *             colour is reduced the way libpng's rgb_to_gray does it for
 *             OpenCV's coefficients 0.299/0.587: (9797 R + 19234 G + 3737 B)
 *             >> 15, alpha is dropped.
 *
 * Unlike the reference (which prints and carries on, or dereferences NULL on
 * a failed fopen), every failure returns HPM_ERR_IO.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include <zlib.h>

#include "hpm_b200.h"
#include "hpm_jpeg.h"

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

namespace {

bool read_file(const char *path, std::vector<uint8_t> &out)
{
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    out.clear();
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) out.insert(out.end(), buf, buf + n);
    const bool ok = !ferror(f);
    fclose(f);
    return ok;
}

/* P5 header: magic, width, height, maxval, each separated by whitespace and
 * '#' comments, then one whitespace byte before the raster. */
int decode_pgm(const std::vector<uint8_t> &b, std::vector<uint8_t> &px, int *w, int *h)
{
    size_t i = 2;
    long v[3];
    for (int k = 0; k < 3; ++k) {
        for (;;) {
            if (i >= b.size()) return HPM_ERR_IO;
            if (b[i] == '#') {
                while (i < b.size() && b[i] != '\n') ++i;
            } else if (b[i] == ' ' || b[i] == '\t' || b[i] == '\n' || b[i] == '\r') {
                ++i;
            } else {
                break;
            }
        }
        if (b[i] < '0' || b[i] > '9') return HPM_ERR_IO;
        v[k] = 0;
        while (i < b.size() && b[i] >= '0' && b[i] <= '9' && v[k] < (1L << 20)) v[k] = v[k] * 10 + (b[i++] - '0');
    }
    if (i >= b.size() || v[0] <= 0 || v[1] <= 0 || v[0] >= (1L << 16) || v[1] >= (1L << 16) || v[2] != 255)
        return HPM_ERR_IO;
    ++i; /* the single whitespace byte */
    const size_t n = (size_t)v[0] * v[1];
    if (b.size() - i < n) return HPM_ERR_IO;
    px.assign(b.begin() + i, b.begin() + i + n);
    *w = (int)v[0];
    *h = (int)v[1];
    return HPM_OK;
}

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

int paeth(int a, int b, int c)
{
    const int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    return (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
}

/* out_ch 1: gray as IMREAD_GRAYSCALE; 3: B, G, R as IMREAD_COLOR */
int decode_png(const std::vector<uint8_t> &b, std::vector<uint8_t> &px, int *w_out, int *h_out, int out_ch)
{
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (b.size() < 33 || memcmp(b.data(), sig, 8) != 0) return HPM_ERR_IO;
    size_t i = 8;
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, palette;
    bool seen_end = false;
    while (i + 12 <= b.size() && !seen_end) {
        const uint32_t len = be32(&b[i]);
        if (len > b.size() - i - 12) return HPM_ERR_IO;
        const uint8_t *type = &b[i + 4], *data = &b[i + 8];
        if (!memcmp(type, "IHDR", 4) && len >= 13) {
            w = be32(data);
            h = be32(data + 4);
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
        } else if (!memcmp(type, "PLTE", 4)) {
            palette.assign(data, data + len);
        } else if (!memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!memcmp(type, "IEND", 4)) {
            seen_end = true;
        }
        i += 12 + (size_t)len;
    }
    if (w == 0 || h == 0 || w >= (1u << 16) || h >= (1u << 16) || depth != 8 || interlace != 0) return HPM_ERR_IO;
    int ch;
    switch (ctype) {
    case 0: ch = 1; break;
    case 2: ch = 3; break;
    case 3: ch = 1; break;
    case 4: ch = 2; break;
    case 6: ch = 4; break;
    default: return HPM_ERR_IO;
    }
    if (ctype == 3 && (palette.size() < 3 || palette.size() % 3)) return HPM_ERR_IO;
    const size_t stride = (size_t)w * ch;
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf raw_len = (uLongf)raw.size();
    if (uncompress(raw.data(), &raw_len, idat.data(), (uLong)idat.size()) != Z_OK || raw_len != raw.size())
        return HPM_ERR_IO;
    /* undo the per-row filters (PNG spec, section 9) */
    std::vector<uint8_t> img(stride * h);
    for (uint32_t y = 0; y < h; ++y) {
        const uint8_t f = raw[y * (stride + 1)];
        const uint8_t *src = &raw[y * (stride + 1) + 1];
        uint8_t *dst = &img[y * stride];
        const uint8_t *up = y ? &img[(y - 1) * stride] : nullptr;
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= (size_t)ch ? dst[x - ch] : 0, u = up ? up[x] : 0,
                      c = (up && x >= (size_t)ch) ? up[x - ch] : 0;
            int pred;
            switch (f) {
            case 0: pred = 0; break;
            case 1: pred = a; break;
            case 2: pred = u; break;
            case 3: pred = (a + u) >> 1; break;
            case 4: pred = paeth(a, u, c); break;
            default: return HPM_ERR_IO;
            }
            dst[x] = (uint8_t)(src[x] + pred);
        }
    }
    px.resize((size_t)w * h * out_ch);
    for (size_t p = 0; p < (size_t)w * h; ++p) {
        int r, g, bl;
        if (ctype == 0 || ctype == 4) {
            r = g = bl = img[p * ch];
        } else if (ctype == 3) {
            const size_t k = 3 * (size_t)img[p];
            if (k + 2 >= palette.size()) return HPM_ERR_IO;
            r = palette[k], g = palette[k + 1], bl = palette[k + 2];
        } else {
            r = img[p * ch], g = img[p * ch + 1], bl = img[p * ch + 2];
        }
        if (out_ch == 3) {
            px[3 * p] = (uint8_t)bl;
            px[3 * p + 1] = (uint8_t)g;
            px[3 * p + 2] = (uint8_t)r;
        } else if (ctype == 0 || ctype == 4) {
            px[p] = (uint8_t)r;
        } else {
            px[p] = (uint8_t)((9797 * r + 19234 * g + 3737 * bl) >> 15);
        }
    }
    *w_out = (int)w;
    *h_out = (int)h;
    return HPM_OK;
}

}  // namespace

extern "C" int hpm_resize_linear(const float *src, int sw, int sh, int ch, float *dst, int dw, int dh)
{
    if (!src || !dst || sw < 1 || sh < 1 || dw < 1 || dh < 1 || ch < 1) return HPM_ERR_ARG;
    auto coef = [](int d, int sn, int dn, int &s0, int &s1, float &f) {
        const double fd = (d + 0.5) * ((double)sn / dn) - 0.5;
        int si = (int)std::floor(fd);
        f = (float)(fd - si);
        if (si < 0) f = 0.0f, si = 0;
        if (si >= sn - 1) f = 0.0f, si = sn - 1;
        s0 = si;
        s1 = si + 1 < sn ? si + 1 : sn - 1;
    };
    std::vector<int> xs0(dw), xs1(dw);
    std::vector<float> fxs(dw);
    for (int x = 0; x < dw; ++x) coef(x, sw, dw, xs0[x], xs1[x], fxs[x]);
    for (int y = 0; y < dh; ++y) {
        int sy0, sy1;
        float fy;
        coef(y, sh, dh, sy0, sy1, fy);
        const float *r0 = src + (size_t)sy0 * sw * ch, *r1 = src + (size_t)sy1 * sw * ch;
        float *o = dst + (size_t)y * dw * ch;
        for (int x = 0; x < dw; ++x) {
            const float fx = fxs[x];
            for (int c = 0; c < ch; ++c) {
                const float a0 = r0[(size_t)xs0[x] * ch + c], b0 = r0[(size_t)xs1[x] * ch + c];
                const float a1 = r1[(size_t)xs0[x] * ch + c], b1 = r1[(size_t)xs1[x] * ch + c];
                const float h0 = std::fmaf(fx, b0 - a0, a0), h1 = std::fmaf(fx, b1 - a1, a1);
                o[(size_t)x * ch + c] = std::fmaf(fy, h1 - h0, h0);
            }
        }
    }
    return HPM_OK;
}

/* cv::resize(INTER_LINEAR) of an 8-bit image as OpenCV 4.13 computes it:
 * 11-bit fixed-point weights round((1 - f) 2048) and round(f 2048) from the
 * float source coordinate (d + 0.5) s - 0.5; horizontally the fraction is
 * zeroed where the left or right tap leaves the image, vertically both rows
 * are clamped into it and the fraction is kept; the vertical blend is
 * ((H0 >> 4) b0 >> 16) + ((H1 >> 4) b1 >> 16), rounded by (x + 2) >> 2.
 * Checked byte for byte against cv2.resize for down- and upscales. */
extern "C" int hpm_resize_linear_u8(const uint8_t *src, int sw, int sh, int ch, uint8_t *dst, int dw, int dh)
{
    if (!src || !dst || sw < 1 || sh < 1 || dw < 1 || dh < 1 || ch < 1) return HPM_ERR_ARG;
    /* the scale as OpenCV forms it, 1 / (dst / src): sw / dw can differ from
     * it by one ulp, which can move a floor or an 11-bit weight */
    const double scale_x = 1.0 / ((double)dw / sw), scale_y = 1.0 / ((double)dh / sh);
    std::vector<int> x0(dw), x1(dw), a0(dw), a1(dw);
    for (int x = 0; x < dw; ++x) {
        float f = (float)((x + 0.5) * scale_x - 0.5);
        int sx = (int)std::floor(f);
        f -= (float)sx;
        if (sx < 0) f = 0.0f, sx = 0;
        if (sx >= sw - 1) f = 0.0f, sx = sw - 1;
        x0[x] = sx;
        x1[x] = std::min(sx + 1, sw - 1);
        a0[x] = (int)std::lrintf((1.0f - f) * 2048.0f);
        a1[x] = (int)std::lrintf(f * 2048.0f);
    }
    std::vector<int> h0((size_t)dw * ch), h1((size_t)dw * ch);
    auto horizontal = [&](int row, std::vector<int> &out) {
        const uint8_t *r = src + (size_t)row * sw * ch;
        for (int x = 0; x < dw; ++x)
            for (int c = 0; c < ch; ++c)
                out[(size_t)x * ch + c] = r[(size_t)x0[x] * ch + c] * a0[x] + r[(size_t)x1[x] * ch + c] * a1[x];
    };
    for (int y = 0; y < dh; ++y) {
        float f = (float)((y + 0.5) * scale_y - 0.5);
        const int sy = (int)std::floor(f);
        f -= (float)sy;
        const int r0 = std::min(std::max(sy, 0), sh - 1), r1 = std::min(std::max(sy + 1, 0), sh - 1);
        const int b0 = (int)std::lrintf((1.0f - f) * 2048.0f), b1 = (int)std::lrintf(f * 2048.0f);
        horizontal(r0, h0);
        horizontal(r1, h1);
        uint8_t *o = dst + (size_t)y * dw * ch;
        for (size_t k = 0; k < (size_t)dw * ch; ++k) {
            const int v = ((((h0[k] >> 4) * b0) >> 16) + (((h1[k] >> 4) * b1) >> 16) + 2) >> 2;
            o[k] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
    return HPM_OK;
}

static int read_image8(const char *path, uint8_t *pixels, size_t cap, int *w, int *h, int out_ch)
{
    if (!path || !w || !h) return HPM_ERR_ARG;
    std::vector<uint8_t> bytes, px;
    if (!read_file(path, bytes) || bytes.size() < 2) return HPM_ERR_IO;
    int r;
    if (bytes[0] == 0xFF && bytes[1] == 0xD8) {
        if (!pixels) return hpm_jpeg_size(bytes.data(), bytes.size(), w, h); /* size query: markers only */
        r = hpm_decode_jpeg(bytes.data(), bytes.size(), px, w, h, out_ch);
    } else if (bytes[0] == 'P' && bytes[1] == '5') {
        r = decode_pgm(bytes, px, w, h);
        if (!r && out_ch == 3) {
            std::vector<uint8_t> c(px.size() * 3);
            for (size_t p = 0; p < px.size(); ++p) c[3 * p] = c[3 * p + 1] = c[3 * p + 2] = px[p];
            px.swap(c);
        }
    } else {
        r = decode_png(bytes, px, w, h, out_ch);
    }
    if (r) return r;
    if (!pixels) return HPM_OK;
    if (cap < px.size()) return HPM_ERR_ARG;
    memcpy(pixels, px.data(), px.size());
    return HPM_OK;
}

extern "C" int hpm_read_gray8(const char *path, uint8_t *pixels, size_t cap, int *w, int *h)
{
    return read_image8(path, pixels, cap, w, h, 1);
}

extern "C" int hpm_read_bgr8(const char *path, uint8_t *pixels, size_t cap, int *w, int *h)
{
    return read_image8(path, pixels, cap, w, h, 3);
}

/*
 * CPU oracle for the HPM-MVS PatchMatch hot path (see hpm_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of it.
 *
 * Every routine restates the reference's algorithm in the reference's own
 * arithmetic types (float where the reference computes in float, double where
 * a double literal or double math function promotes it).  Build with
 * -ffp-contract=off so that no multiply-add is fused behind our back.
 */
#include "hpm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846 /* M_PI of HPM-MVS/main.h:41 */
#define MAXV 32                      /* cost_vector[32], HPM.cu:402 */

typedef struct {
    float x, y, z, w;
} F4;

static int g_tex_round = 1;

void or_set_tex_rounding(int mode) { g_tex_round = mode; }
int or_get_tex_rounding(void) { return g_tex_round; }

/* ------------------------------------------------------------------ */
/* Counter-based RNG (Philox4x32-10, Salmon et al., SC'11).            */
/* ------------------------------------------------------------------ */

static void philox4x32_10(uint32_t k0, uint32_t k1, uint32_t c[4])
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* uniform in (0,1]: ((x >> 8) + 1) * 2^-24 */
static float u32_to_uniform(uint32_t x) { return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f); }

typedef struct {
    uint32_t k0, k1, pixel, step, salt, n;
    uint32_t buf[4];
} Rng;

static void rng_init(Rng *r, uint64_t seed, uint32_t pixel, uint32_t step, uint32_t salt)
{
    r->k0 = (uint32_t)seed;
    r->k1 = (uint32_t)(seed >> 32);
    r->pixel = pixel;
    r->step = step;
    r->salt = salt;
    r->n = 0;
}

static float rng_uniform(Rng *r)
{
    if ((r->n & 3u) == 0) {
        r->buf[0] = r->pixel;
        r->buf[1] = r->step;
        r->buf[2] = r->n >> 2;
        r->buf[3] = r->salt;
        philox4x32_10(r->k0, r->k1, r->buf);
    }
    return u32_to_uniform(r->buf[r->n++ & 3u]);
}

void or_philox4x32_10(uint32_t k0, uint32_t k1, uint32_t *ctr4) { philox4x32_10(k0, k1, ctr4); }

float or_philox_uniform(uint64_t seed, uint32_t pixel, uint32_t step, uint32_t salt, uint32_t n)
{
    uint32_t c[4] = {pixel, step, n >> 2, salt};
    philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c);
    return u32_to_uniform(c[n & 3u]);
}

/* ------------------------------------------------------------------ */
/* Texture emulation: tex2D<float> on a float cudaArray with            */
/* cudaFilterModeLinear, unnormalised coordinates (HPM.cpp:599-616).    */
/* ------------------------------------------------------------------ */

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* float -> int conversion with CUDA's saturating semantics (NaN -> 0). */
static int f2i_rz_sat(float f)
{
    if (f != f) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return (-2147483647 - 1);
    return (int)f;
}

/* Fixed-point coordinate of one axis: texel index pair and the 8-bit
 * fraction A (0..255).  Mode 1 (the hardware's, pinned by the probe in
 * tests/golden/tex_probe.npz): A = round-half-up of 256 * (u - 0.5). */
static void tex_coord(float u, int n, int *i0, int *i1, int *A)
{
    double xb = (double)u - 0.5; /* texel-centre convention */
    if (xb != xb) xb = 0.0;
    if (xb < -2.0) xb = -2.0; /* beyond the edge every tap reads the edge texel */
    if (xb > (double)n + 1.0) xb = (double)n + 1.0;
    const double s = xb * 256.0;
    const double q = g_tex_round ? floor(s + 0.5) : floor(s);
    const double i = floor(q / 256.0);
    *A = (int)(q - i * 256.0);
    *i0 = clampi((int)i, 0, n - 1);
    *i1 = clampi((int)i + 1, 0, n - 1);
}

/* Bilinear filter of the texture unit for float textures, as measured on a
 * B200 with single-texel and random textures (tests/golden/tex_probe.npz):
 * only the far corner's weight is rounded, w11 = round-half-up(A*B/256), and
 * the other three follow by subtraction so that the four weights are
 * integers summing to 256.  Exact for every probe sample. */
float or_tex2d(const float *img, int w, int h, float u, float v)
{
    int x0, x1, y0, y1, A, B;
    tex_coord(u, w, &x0, &x1, &A);
    tex_coord(v, h, &y0, &y1, &B);
    const int w11 = (A * B + 128) >> 8;
    const int w10 = A - w11, w01 = B - w11, w00 = 256 - A - B + w11;
    const double t00 = img[(size_t)y0 * w + x0], t10 = img[(size_t)y0 * w + x1];
    const double t01 = img[(size_t)y1 * w + x0], t11 = img[(size_t)y1 * w + x1];
    return (float)((w00 * t00 + w10 * t10 + w01 * t01 + w11 * t11) / 256.0);
}

/* texel fetch at an integer position + 0.5 (no interpolation), clamped */
static float texel(const float *img, int w, int h, int x, int y)
{
    return img[(size_t)clampi(y, 0, h - 1) * w + clampi(x, 0, w - 1)];
}

/* ------------------------------------------------------------------ */
/* Plane / camera utilities (HPM.cu:65-133, 227-316, 445-481)          */
/* ------------------------------------------------------------------ */

static void normalize3(F4 *v) /* NormalizeVec3, HPM.cu:77-84 */
{
    const float n2 = v->x * v->x + v->y * v->y + v->z * v->z;
    const float inv = 1.0f / sqrtf(n2);
    v->x *= inv;
    v->y *= inv;
    v->z *= inv;
}

static void get3dpoint(const OrCamera *c, int px, int py, float depth, float *X) /* HPM.cu:102-107 */
{
    X[0] = depth * ((float)px - c->K[2]) / c->K[0];
    X[1] = depth * ((float)py - c->K[5]) / c->K[4];
    X[2] = depth;
}

static F4 view_direction(const OrCamera *c, int px, int py, float depth) /* HPM.cu:109-121 */
{
    float X[3];
    get3dpoint(c, px, py, depth, X);
    const float norm = sqrtf(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    F4 v = {X[0] / norm, X[1] / norm, X[2] / norm, 0.0f};
    return v;
}

static float distance_to_origin(const OrCamera *c, int px, int py, float depth, F4 n) /* HPM.cu:123-128 */
{
    float X[3];
    get3dpoint(c, px, py, depth, X);
    return -(n.x * X[0] + n.y * X[1] + n.z * X[2]);
}

static float depth_from_plane(const OrCamera *c, F4 h, int px, int py) /* HPM.cu:130-133 */
{
    return -h.w * c->K[0] /
           (((float)px - c->K[2]) * h.x + (c->K[0] / c->K[4]) * ((float)py - c->K[5]) * h.y + c->K[0] * h.z);
}

static F4 transform_normal(const OrCamera *c, F4 h) /* R^T n, HPM.cu:298-306 */
{
    F4 r;
    r.x = c->R[0] * h.x + c->R[3] * h.y + c->R[6] * h.z;
    r.y = c->R[1] * h.x + c->R[4] * h.y + c->R[7] * h.z;
    r.z = c->R[2] * h.x + c->R[5] * h.y + c->R[8] * h.z;
    r.w = h.w;
    return r;
}

static F4 transform_normal_to_ref(const OrCamera *c, F4 h) /* R n, HPM.cu:308-316 */
{
    F4 r;
    r.x = c->R[0] * h.x + c->R[1] * h.y + c->R[2] * h.z;
    r.y = c->R[3] * h.x + c->R[4] * h.y + c->R[5] * h.z;
    r.z = c->R[6] * h.x + c->R[7] * h.y + c->R[8] * h.z;
    r.w = h.w;
    return r;
}

static float dot3(F4 a, F4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static F4 random_normal(const OrCamera *c, int px, int py, Rng *rng, float depth) /* HPM.cu:135-161 */
{
    float q1 = 1.0f, q2 = 1.0f, s = 2.0f;
    while (s >= 1.0f) {
        q1 = 2.0f * rng_uniform(rng) - 1.0f;
        q2 = 2.0f * rng_uniform(rng) - 1.0f;
        s = q1 * q1 + q2 * q2;
    }
    const float sq = sqrtf(1.0f - s);
    F4 n = {2.0f * q1 * sq, 2.0f * q2 * sq, 1.0f - 2.0f * s, 0.0f};
    const F4 v = view_direction(c, px, py, depth);
    if (n.x * v.x + n.y * v.y + n.z * v.z > 0.0f) {
        n.x = -n.x;
        n.y = -n.y;
        n.z = -n.z;
    }
    normalize3(&n);
    return n;
}

static F4 perturbed_normal(const OrCamera *c, int px, int py, F4 normal, Rng *rng, float pert) /* HPM.cu:163-198 */
{
    const F4 v = view_direction(c, px, py, 1.0f);
    const float a1 = (rng_uniform(rng) - 0.5f) * pert;
    const float a2 = (rng_uniform(rng) - 0.5f) * pert;
    const float a3 = (rng_uniform(rng) - 0.5f) * pert;
    const float s1 = sinf(a1), s2 = sinf(a2), s3 = sinf(a3);
    const float c1 = cosf(a1), c2 = cosf(a2), c3 = cosf(a3);
    float R[9];
    R[0] = c2 * c3;
    R[1] = c3 * s1 * s2 - c1 * s3;
    R[2] = s1 * s3 + c1 * c3 * s2;
    R[3] = c2 * s3;
    R[4] = c1 * c3 + s1 * s2 * s3;
    R[5] = c1 * s2 * s3 - c3 * s1;
    R[6] = -s2;
    R[7] = c2 * s1;
    R[8] = c1 * c2;
    F4 p;
    p.x = R[0] * normal.x + R[1] * normal.y + R[2] * normal.z;
    p.y = R[3] * normal.x + R[4] * normal.y + R[5] * normal.z;
    p.z = R[6] * normal.x + R[7] * normal.y + R[8] * normal.z;
    p.w = normal.w;
    if (dot3(p, v) >= 0.0f) p = normal;
    normalize3(&p);
    return p;
}

static F4 random_plane(const OrCamera *c, int px, int py, Rng *rng, float dmin, float dmax) /* HPM.cu:200-206 */
{
    const float depth = rng_uniform(rng) * (dmax - dmin) + dmin;
    F4 h = random_normal(c, px, py, rng, depth);
    h.w = distance_to_origin(c, px, py, depth, h);
    return h;
}

static void homography(const OrCamera *ref, const OrCamera *src, F4 h, float *H) /* HPM.cu:227-287 */
{
    const float *rR = ref->R, *sR = src->R, *rt = ref->t, *st = src->t;
    float rC[3], sC[3];
    rC[0] = -(rR[0] * rt[0] + rR[3] * rt[1] + rR[6] * rt[2]);
    rC[1] = -(rR[1] * rt[0] + rR[4] * rt[1] + rR[7] * rt[2]);
    rC[2] = -(rR[2] * rt[0] + rR[5] * rt[1] + rR[8] * rt[2]);
    sC[0] = -(sR[0] * st[0] + sR[3] * st[1] + sR[6] * st[2]);
    sC[1] = -(sR[1] * st[0] + sR[4] * st[1] + sR[7] * st[2]);
    sC[2] = -(sR[2] * st[0] + sR[5] * st[1] + sR[8] * st[2]);
    float Rr[9], Cr[3], tr[3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Rr[3 * i + j] = sR[3 * i + 0] * rR[3 * j + 0] + sR[3 * i + 1] * rR[3 * j + 1] + sR[3 * i + 2] * rR[3 * j + 2];
    Cr[0] = rC[0] - sC[0];
    Cr[1] = rC[1] - sC[1];
    Cr[2] = rC[2] - sC[2];
    for (int i = 0; i < 3; ++i) tr[i] = sR[3 * i + 0] * Cr[0] + sR[3 * i + 1] * Cr[1] + sR[3 * i + 2] * Cr[2];
    for (int i = 0; i < 3; ++i) {
        H[3 * i + 0] = Rr[3 * i + 0] - tr[i] * h.x / h.w;
        H[3 * i + 1] = Rr[3 * i + 1] - tr[i] * h.y / h.w;
        H[3 * i + 2] = Rr[3 * i + 2] - tr[i] * h.z / h.w;
    }
    const float *rK = ref->K, *sK = src->K;
    float tmp[9];
    for (int i = 0; i < 3; ++i) {
        tmp[3 * i + 0] = H[3 * i + 0] / rK[0];
        tmp[3 * i + 1] = H[3 * i + 1] / rK[4];
        tmp[3 * i + 2] = -H[3 * i + 0] * rK[2] / rK[0] - H[3 * i + 1] * rK[5] / rK[4] + H[3 * i + 2];
    }
    H[0] = sK[0] * tmp[0] + sK[2] * tmp[6];
    H[1] = sK[0] * tmp[1] + sK[2] * tmp[7];
    H[2] = sK[0] * tmp[2] + sK[2] * tmp[8];
    H[3] = sK[4] * tmp[3] + sK[5] * tmp[6];
    H[4] = sK[4] * tmp[4] + sK[5] * tmp[7];
    H[5] = sK[4] * tmp[5] + sK[5] * tmp[8];
    H[6] = sK[8] * tmp[6];
    H[7] = sK[8] * tmp[7];
    H[8] = sK[8] * tmp[8];
}

void or_homography(const OrCamera *ref, const OrCamera *src, const float *plane4, float *H9)
{
    F4 h = {plane4[0], plane4[1], plane4[2], plane4[3]};
    homography(ref, src, h, H9);
}

static void warp(const float *H, int px, int py, float *ox, float *oy) /* HPM.cu:289-296 */
{
    const float x = H[0] * (float)px + H[1] * (float)py + H[2];
    const float y = H[3] * (float)px + H[4] * (float)py + H[5];
    const float z = H[6] * (float)px + H[7] * (float)py + H[8];
    *ox = x / z;
    *oy = y / z;
}

/* ------------------------------------------------------------------ */
/* Problem context                                                     */
/* ------------------------------------------------------------------ */

typedef struct {
    int n;
    const float *const *imgs;
    const OrCamera *cams;
    const float *const *depths; /* geometric-consistency depth maps, may be NULL */
    int W, H;
    int geom, prior;
    float dmin, dmax;
    uint64_t seed;
    uint32_t salt;
    F4 *planes;
    float *costs;
    uint32_t *views;
    const F4 *prior_planes;
    const uint32_t *masks;
    /* ACMM+NESP variant (ACMM+NESP/windows/ACMM.cu): acmm selects its
     * weights and update rule, hier its hierarchy pass (1 upsampled, 2 at the
     * same size), pre_costs the hierarchy's acceptance threshold */
    int acmm, hier;
    float *pre_costs;
} Ctx;

/* ComputeBilateralNCC, HPM.cu:318-397 (patch 11, increment 2, sigma 5/3). */
static float bilateral_ncc(const Ctx *c, int v, int px, int py, F4 h)
{
    const float cost_max = 2.0f;
    const int radius = 11 / 2;
    const float sigma_spatial = 5.0f, sigma_color = 3.0f;
    const OrCamera *ref = &c->cams[0], *src = &c->cams[v];
    const float *rimg = c->imgs[0], *simg = c->imgs[v];
    float H[9];
    homography(ref, src, h, H);
    float cx, cy;
    warp(H, px, py, &cx, &cy);
    if (cx >= (float)src->width || cx < 0.0f || cy >= (float)src->height || cy < 0.0f) return cost_max;

    float sum_ref = 0.f, sum_ref_ref = 0.f, sum_src = 0.f, sum_src_src = 0.f, sum_ref_src = 0.f, wsum = 0.f;
    const float rc = texel(rimg, ref->width, ref->height, px, py);
    for (int i = -radius; i < radius + 1; i += 2) {
        float r_ref = 0.f, r_src = 0.f, r_rr = 0.f, r_ss = 0.f, r_rs = 0.f, r_w = 0.f;
        for (int j = -radius; j < radius + 1; j += 2) {
            const int qx = px + i, qy = py + j;
            const float rp = texel(rimg, ref->width, ref->height, qx, qy);
            float sx, sy;
            warp(H, qx, qy, &sx, &sy);
            const float sp = or_tex2d(simg, src->width, src->height, sx + 0.5f, sy + 0.5f);
            const float sd = sqrtf((float)(i * i + j * j));
            const float cd = fabsf(rp - rc);
            const float wgt =
                expf(-sd / (2.0f * sigma_spatial * sigma_spatial) - cd / (2.0f * sigma_color * sigma_color));
            r_ref += wgt * rp;
            r_rr += wgt * rp * rp;
            r_src += wgt * sp;
            r_ss += wgt * sp * sp;
            r_rs += wgt * rp * sp;
            r_w += wgt;
        }
        sum_ref += r_ref;
        sum_ref_ref += r_rr;
        sum_src += r_src;
        sum_src_src += r_ss;
        sum_ref_src += r_rs;
        wsum += r_w;
    }
    const float inv = 1.0f / wsum;
    sum_ref *= inv;
    sum_ref_ref *= inv;
    sum_src *= inv;
    sum_src_src *= inv;
    sum_ref_src *= inv;
    const float var_ref = sum_ref_ref - sum_ref * sum_ref;
    const float var_src = sum_src_src - sum_src * sum_src;
    if (var_ref < 1e-5f || var_src < 1e-5f) return cost_max;
    const float covar = sum_ref_src - sum_ref * sum_src;
    const float vv = sqrtf(var_ref * var_src);
    return fmaxf(0.0f, fminf(cost_max, 1.0f - covar / vv));
}

static void cost_vector(const Ctx *c, int px, int py, F4 h, float *cv) /* HPM.cu:438-443 */
{
    for (int i = 1; i < c->n; ++i) cv[i - 1] = bilateral_ncc(c, i, px, py, h);
}

static void sort_small(float *d, int n) /* HPM.cu:3-12 */
{
    int j;
    for (int i = 1; i < n; i++) {
        const float tmp = d[i];
        for (j = i; j >= 1 && tmp < d[j - 1]; j--) d[j] = d[j - 1];
        d[j] = tmp;
    }
}

/* ComputeMultiViewInitialCostandSelectedViews, HPM.cu:399-436 (top_k = 4) */
static float initial_cost(const Ctx *c, int px, int py, F4 h, uint32_t *views)
{
    float cv[MAXV], cp[MAXV];
    memset(cv, 0, sizeof(cv));
    memset(cp, 0, sizeof(cp));
    cv[0] = cp[0] = 2.0f;
    int count = 0, valid = 0;
    for (int i = 1; i < c->n; ++i) {
        const float x = bilateral_ncc(c, i, px, py, h);
        cv[i - 1] = x;
        cp[i - 1] = x;
        count++;
        if (x < 2.0f) valid++;
    }
    sort_small(cv, count);
    *views = 0;
    const int top_k = valid < 4 ? valid : 4;
    if (top_k > 0) {
        float cost = 0.0f;
        for (int i = 0; i < top_k; ++i) cost += cv[i];
        const float thr = cv[top_k - 1];
        for (int i = 0; i < c->n - 1; ++i)
            if (cp[i] <= thr) *views |= (1u << i);
        return cost / (float)top_k;
    }
    return 2.0f;
}

static void world_point(const OrCamera *c, float x, float y, float depth, float *P) /* HPM.cu:445-469 */
{
    float X[3], T[3];
    X[0] = depth * (x - c->K[2]) / c->K[0];
    X[1] = depth * (y - c->K[5]) / c->K[4];
    X[2] = depth;
    T[0] = c->R[0] * X[0] + c->R[3] * X[1] + c->R[6] * X[2];
    T[1] = c->R[1] * X[0] + c->R[4] * X[1] + c->R[7] * X[2];
    T[2] = c->R[2] * X[0] + c->R[5] * X[1] + c->R[8] * X[2];
    const float Cx = -(c->R[0] * c->t[0] + c->R[3] * c->t[1] + c->R[6] * c->t[2]);
    const float Cy = -(c->R[1] * c->t[0] + c->R[4] * c->t[1] + c->R[7] * c->t[2]);
    const float Cz = -(c->R[2] * c->t[0] + c->R[5] * c->t[1] + c->R[8] * c->t[2]);
    P[0] = T[0] + Cx;
    P[1] = T[1] + Cy;
    P[2] = T[2] + Cz;
}

static void project(const float *P, const OrCamera *c, float *pt, float *depth) /* HPM.cu:471-481 */
{
    float t[3];
    t[0] = c->R[0] * P[0] + c->R[1] * P[1] + c->R[2] * P[2] + c->t[0];
    t[1] = c->R[3] * P[0] + c->R[4] * P[1] + c->R[5] * P[2] + c->t[1];
    t[2] = c->R[6] * P[0] + c->R[7] * P[1] + c->R[8] * P[2] + c->t[2];
    *depth = c->K[6] * t[0] + c->K[7] * t[1] + c->K[8] * t[2];
    pt[0] = (c->K[0] * t[0] + c->K[1] * t[1] + c->K[2] * t[2]) / *depth;
    pt[1] = (c->K[3] * t[0] + c->K[4] * t[1] + c->K[5] * t[2]) / *depth;
}

/* ComputeGeomConsistencyCost, HPM.cu:483-508 */
/* ComputeGeomConsistencyCost, HPM.cu:483-508; max_cost 5 there and 3 in the
 * ACMM+NESP variant (ACMM.cu:496) */
static float geom_cost_m(const OrCamera *ref, const OrCamera *src, const float *sdepth, F4 h, int px, int py,
                         float max_cost)
{
    const float depth = depth_from_plane(ref, h, px, py);
    float P[3], spt[2], sd;
    world_point(ref, (float)px, (float)py, depth, P);
    project(P, src, spt, &sd);
    const int ix = f2i_rz_sat(spt[0]), iy = f2i_rz_sat(spt[1]);
    const float src_depth = or_tex2d(sdepth, src->width, src->height, (float)ix + 0.5f, (float)iy + 0.5f);
    if (src_depth == 0.0f) return max_cost;
    float Q[3], bpt[2], rd;
    world_point(src, spt[0], spt[1], src_depth, Q);
    project(Q, ref, bpt, &rd);
    const float dx = (float)px - bpt[0], dy = (float)py - bpt[1];
    return fminf(max_cost, sqrtf(dx * dx + dy * dy));
}

static float geom_cost(const OrCamera *ref, const OrCamera *src, const float *sdepth, F4 h, int px, int py)
{
    return geom_cost_m(ref, src, sdepth, h, px, py, 5.0f);
}

/* the pass's geometric term: weight w times the variant's capped cost */
static float geom_term(const Ctx *c, int j, F4 h, int px, int py, float w)
{
    return w * geom_cost_m(&c->cams[0], &c->cams[j], c->depths[j], h, px, py, c->acmm ? 3.0f : 5.0f);
}

/* ------------------------------------------------------------------ */
/* RandomInitialization, HPM.cu:510-558                                 */
/* ------------------------------------------------------------------ */

static void init_pixel(Ctx *c, int px, int py)
{
    const int center = py * c->W + px;
    const OrCamera *cam = &c->cams[0];
    Rng rng;
    rng_init(&rng, c->seed, (uint32_t)center, 0u, c->salt);
    if (c->geom || c->hier) {
        /* ACMM.cu:538-604: the hierarchy pass starts from the upsampled
         * (world normal, depth).  Its acceptance threshold pre_costs is the
         * initial cost of the plane held before the normal is filled in:
         * normal (0, 0, 0), w = the depth itself (ACMM.cpp:707-713 sets only
         * .w of a freshly allocated array, which is zero-filled); at the same
         * size (upsample false) the reference leaves pre_costs unset, taken
         * here as zero, which accepts no update. */
        if (c->hier == 1) {
            uint32_t v_unused;
            F4 hz = {0.0f, 0.0f, 0.0f, c->planes[center].w};
            c->pre_costs[center] = initial_cost(c, px, py, hz, &v_unused);
        } else if (c->hier == 2) {
            c->pre_costs[center] = 0.0f;
        }
        F4 h = transform_normal_to_ref(cam, c->planes[center]);
        const float depth = h.w;
        h.w = distance_to_origin(cam, px, py, depth, h);
        c->planes[center] = h;
        c->costs[center] = initial_cost(c, px, py, h, &c->views[center]);
    } else if (c->prior) {
        if (c->masks[center] > 0 && c->costs[center] >= 0.1f) {
            const float pert = 0.02f;
            const F4 h = c->prior_planes[center];
            float dp = h.w;
            const float lo = (1 - 3 * pert) * dp;
            const float hi = (1 + 3 * pert) * dp;
            dp = rng_uniform(&rng) * (hi - lo) + lo;
            F4 hp = perturbed_normal(cam, px, py, h, &rng, (float)(3 * pert * OR_PI));
            hp.w = dp;
            c->planes[center] = hp;
            c->costs[center] = initial_cost(c, px, py, hp, &c->views[center]);
        } else {
            F4 h = c->planes[center];
            const float depth = h.w;
            h.w = distance_to_origin(cam, px, py, depth, h);
            c->planes[center] = h;
            c->costs[center] = initial_cost(c, px, py, h, &c->views[center]);
        }
    } else {
        const F4 h = random_plane(cam, px, py, &rng, c->dmin, c->dmax);
        c->planes[center] = h;
        c->costs[center] = initial_cost(c, px, py, h, &c->views[center]);
    }
}

/* ------------------------------------------------------------------ */
/* CheckerboardPropagation, HPM.cu:1222-1725                           */
/* ------------------------------------------------------------------ */

/* Direction order of HPM.cu:1245: 0 left_up, 1 up_far, 2 right_up,
 * 3 down_far, 4 right_down, 5 left_far, 6 left_down, 7 right_far. */
static const int kStripDir[8][2] = {{0, 0}, {0, -1}, {0, 0}, {0, 1}, {0, 0}, {-1, 0}, {0, 0}, {1, 0}};
/* polyline start (dx, dy) and the two alternating step axes */
static const int kPolyStart[8][2] = {{-5, -6}, {0, 0}, {6, -5}, {0, 0}, {5, 6}, {0, 0}, {-6, 5}, {0, 0}};
/* step for even i, step for odd i */
static const int kPolyStep[8][2][2] = {
    {{-2, 0}, {0, -2}}, {{0, 0}, {0, 0}}, {{0, -2}, {2, 0}}, {{0, 0}, {0, 0}},
    {{2, 0}, {0, 2}},   {{0, 0}, {0, 0}}, {{0, 2}, {-2, 0}}, {{0, 0}, {0, 0}}};

/* Validity of the first site of direction k at extension round r (r = 0 is
 * the initial sampling): HPM.cu:1252-1445 and the Extended* functions. */
static int first_site_valid(int k, int r, int px, int py, int W, int H)
{
    const int s = 10 * r, d = 8 * r;
    switch (k) {
    case 1: return py > 4 + s;
    case 3: return py < H - 5 - s;
    case 5: return px > 4 + s;
    case 7: return px < W - 5 - s;
    case 0: return px > 4 + d && py > 5 + d;
    case 2: return px < W - 6 - d && py > 4 + d;
    case 4: return px < W - 5 - d && py < H - 6 - d;
    default: return px > 5 + d && py < H - 5 - d;
    }
}

/* Site selection of one direction at round r; returns the chosen pixel index.
 * Strips: 5 sites 2 apart from +/-(5 + 10r) (right strip keeps the maximum,
 * HPM.cu:1330, 744).  Polylines: start shifted by 8r, then 7 zig-zag steps of
 * 2 (HPM.cu:1346-1471, 780-1034). */
static int select_site(const Ctx *c, int k, int r, int px, int py)
{
    const int W = c->W, H = c->H;
    if (k & 1) {
        const int dx = kStripDir[k][0], dy = kStripDir[k][1];
        const int off = 5 + 10 * r;
        int best = (py + dy * off) * W + (px + dx * off);
        float cmin = c->costs[best];
        for (int i = 1; i < 5; ++i) {
            int ok;
            switch (k) {
            case 1: ok = py > 4 + 2 * i + 10 * r; break;
            case 3: ok = py < H - 5 - 2 * i - 10 * r; break;
            case 5: ok = px > 4 + 2 * i + 10 * r; break;
            default: ok = px < W - 5 - 2 * i - 10 * r; break;
            }
            if (!ok) break;
            const int q = (py + dy * (off + 2 * i)) * W + (px + dx * (off + 2 * i));
            if (k == 7) {
                if (cmin < c->costs[q]) {
                    cmin = c->costs[q];
                    best = q;
                }
            } else if (c->costs[q] < cmin) {
                cmin = c->costs[q];
                best = q;
            }
        }
        return best;
    }
    const int sx = (kPolyStart[k][0] < 0 ? -1 : 1), sy = (kPolyStart[k][1] < 0 ? -1 : 1);
    int x = px + kPolyStart[k][0] + sx * 8 * r;
    int y = py + kPolyStart[k][1] + sy * 8 * r;
    int best = y * W + x;
    float cmin = c->costs[best];
    for (int i = 0; i < 7; ++i) {
        x += kPolyStep[k][i & 1][0];
        y += kPolyStep[k][i & 1][1];
        if (x >= 0 && x < W && y < H && y >= 0) {
            const int q = y * W + x;
            if (c->costs[q] < cmin) {
                cmin = c->costs[q];
                best = q;
            }
        } else {
            break;
        }
    }
    return best;
}

/* JudgeExtend, HPM.cu:1036-1059 */
static int judge_extend(int iter, int round, const float *cv, int nv, int flag)
{
    if (!flag) return 0;
    const int iter_tmp = 3 - round;
    const float good = (float)(0.8 * exp(-iter * iter * iter_tmp / 90.0));
    const float bad = 1.2f;
    int good_sum = 0, bad_sum = 0;
    for (int i = 0; i < nv; i++) {
        if (cv[i] < good) good_sum++;
        if (cv[i] > bad) bad_sum++;
    }
    return !(good_sum >= 1 && bad_sum <= 2);
}

static float restricted_prior(float depth_diff, float angle_cos, float two_dss, float two_ass)
{
    const float gamma = 0.5f;
    const float angle_diff = acosf(angle_cos);
    return gamma + expf(-depth_diff * depth_diff / two_dss) * expf(-angle_diff * angle_diff / two_ass);
}

/* PlaneHypothesisRefinement, HPM.cu:1143-1220 */
static void refine(Ctx *c, int px, int py, F4 *plane, float *depth, float *cost, Rng *rng, const float *vw, float wn,
                   float *restricted_cost)
{
    const OrCamera *cam = &c->cams[0];
    const int center = py * c->W + px;
    const float pert = 0.02f;
    const float depth_sigma = (c->dmax - c->dmin) / 64.0f;
    const float two_dss = 2 * depth_sigma * depth_sigma;
    const float angle_sigma = (float)(OR_PI * (5.0f / 180.0f));
    const float two_ass = 2 * angle_sigma * angle_sigma;
    const float beta = 0.18f;
    float depth_prior = 0.0f;
    const int use_prior = c->prior && c->masks[center] > 0;

    float depth_rand;
    F4 n_rand;
    if (use_prior) {
        depth_prior = depth_from_plane(cam, c->prior_planes[center], px, py);
        depth_rand = rng_uniform(rng) * 6 * depth_sigma + (depth_prior - 3 * depth_sigma);
        n_rand = perturbed_normal(cam, px, py, c->prior_planes[center], rng, angle_sigma);
    } else {
        depth_rand = rng_uniform(rng) * (c->dmax - c->dmin) + c->dmin;
        n_rand = random_normal(cam, px, py, rng, *depth);
    }
    float depth_pert = *depth;
    const float lo = (1 - pert) * depth_pert, hi = (1 + pert) * depth_pert;
    depth_pert = rng_uniform(rng) * (hi - lo) + lo; /* do { } while (false-condition): one draw */
    const F4 n_pert = perturbed_normal(cam, px, py, *plane, rng, (float)(pert * OR_PI));

    const float depths[5] = {depth_rand, *depth, depth_rand, *depth, depth_pert};
    const F4 normals[5] = {*plane, n_rand, n_rand, n_pert, *plane};
    for (int i = 0; i < 5; ++i) {
        float cv[MAXV];
        F4 t = normals[i];
        t.w = distance_to_origin(cam, px, py, depths[i], t);
        cost_vector(c, px, py, t, cv);
        float tc = 0.0f;
        for (int j = 0; j < c->n - 1; ++j) {
            if (vw[j] > 0) {
                if (c->geom)
                    tc += vw[j] * (cv[j] + geom_term(c, j + 1, t, px, py, c->acmm ? 0.2f : 0.1f));
                else
                    tc += vw[j] * cv[j];
            }
        }
        tc /= wn;
        const float depth_before = depth_from_plane(cam, t, px, py);
        if (use_prior) {
            const float dd = depths[i] - depth_prior;
            const float pr = restricted_prior(dd, dot3(c->prior_planes[center], t), two_dss, two_ass);
            const float rtc = expf(-tc * tc / beta) * pr;
            if (depth_before >= c->dmin && depth_before <= c->dmax && rtc > *restricted_cost) {
                *depth = depth_before;
                *plane = t;
                *cost = tc;
                *restricted_cost = rtc;
            }
        } else {
            if (depth_before >= c->dmin && depth_before <= c->dmax && tc < *cost) {
                *depth = depth_before;
                *plane = t;
                *cost = tc;
            }
        }
    }
}

static void propagate_pixel(Ctx *c, int px, int py, int iter)
{
    const int W = c->W, H = c->H, nv = c->n - 1;
    const int center = py * W + px;
    const OrCamera *cam = &c->cams[0];
    Rng rng;
    rng_init(&rng, c->seed, (uint32_t)center, (uint32_t)(1 + iter), c->salt);

    float ca[8][MAXV];
    memset(ca, 0, sizeof(ca));
    ca[0][0] = 2.0f; /* float cost_array[8][32] = { 2.0f } (HPM.cu:1244) */
    int flag[8] = {0};
    int pos[8];
    /* default positions when a direction is invalid (HPM.cu:1231-1241) */
    pos[0] = center - 5 - 6 * W;
    pos[1] = center - W * 5;
    pos[2] = center + 6 - 5 * W;
    pos[3] = center + W * 5;
    pos[4] = center + 5 + 6 * W;
    pos[5] = center - 5;
    pos[6] = center - 6 + 5 * W;
    pos[7] = center + 5;
    /* evaluation order of the reference: strips 1,3,5,7 then polylines 0,2,4,6 */
    static const int order[8] = {1, 3, 5, 7, 0, 2, 4, 6};
    for (int oi = 0; oi < 8; ++oi) {
        const int k = order[oi];
        if (!first_site_valid(k, 0, px, py, W, H)) continue;
        flag[k] = 1;
        pos[k] = select_site(c, k, 0, px, py);
        cost_vector(c, px, py, c->planes[pos[k]], ca[k]);
    }

    /* extension: bool symbol_eight_orientations[10] = { true } (HPM.cu:1475) */
    int symbol[8] = {1, 0, 0, 0, 0, 0, 0, 0};
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 8; ++k) {
            if (!symbol[k]) continue;
            if (judge_extend(iter, r, ca[k], nv, flag[k])) {
                if (first_site_valid(k, r, px, py, W, H)) {
                    int best = select_site(c, k, r, px, py);
                    int fresh = 1;
                    if (c->costs[best] > c->costs[pos[k]]) {
                        best = pos[k];
                        fresh = 0;
                    }
                    pos[k] = best;
                    if (fresh) cost_vector(c, px, py, c->planes[best], ca[k]);
                }
                /* else flag[k] is set: position and costs are kept */
            } else {
                symbol[k] = 0;
            }
        }
    }

    /* multi-hypothesis joint view selection, HPM.cu:1548-1613 */
    float vw[MAXV], vp[MAXV], sp[MAXV];
    memset(vw, 0, sizeof(vw));
    memset(vp, 0, sizeof(vp));
    memset(sp, 0, sizeof(sp));
    const int nb[4] = {center - W * 5, center + W * 5, center - 5, center + 5};
    for (int i = 0; i < 4; ++i) {
        if (flag[2 * i + 1]) {
            for (int j = 0; j < nv; ++j) vp[j] += ((c->views[nb[i]] >> j) & 1u) ? 0.9f : 0.1f;
        }
    }
    const float thr = (float)(0.8 * expf((float)(iter * iter) / (-90.0f)));
    for (int i = 0; i < nv; i++) {
        float count = 0;
        int count_false = 0;
        float tmpw = 0;
        for (int j = 0; j < 8; j++) {
            if (ca[j][i] < thr) {
                tmpw += expf(ca[j][i] * ca[j][i] / (-0.18f));
                count++;
            }
            if (ca[j][i] > 1.2f) count_false++;
        }
        if (count > 2 && count_false < 3)
            sp[i] = tmpw / count;
        else if (count_false < 3)
            sp[i] = expf(thr * thr / (-0.32f));
        sp[i] = sp[i] * vp[i];
    }
    { /* TransformPDFToCDF, HPM.cu:86-100 */
        float s = 0.0f;
        for (int i = 0; i < nv; ++i) s += sp[i];
        const float inv = 1.0f / s;
        float cum = 0.0f;
        for (int i = 0; i < nv; ++i) {
            cum += sp[i] * inv;
            sp[i] = cum;
        }
    }
    for (int s = 0; s < 15; ++s) {
        const float rp = rng_uniform(&rng) - FLT_EPSILON;
        for (int i = 0; i < nv; ++i) {
            if (sp[i] > rp) {
                vw[i] += 1.0f;
                break;
            }
        }
    }
    uint32_t tsv = 0;
    float wn = 0;
    for (int i = 0; i < nv; ++i) {
        if (vw[i] > 0) {
            tsv |= 1u << i;
            wn += vw[i];
        }
    }

    float fc[8] = {0};
    for (int i = 0; i < 8; ++i) {
        for (int j = 0; j < nv; ++j) {
            if (vw[j] > 0) {
                if (c->geom) {
                    if (flag[i])
                        fc[i] += vw[j] * (ca[i][j] + geom_term(c, j + 1, c->planes[pos[i]], px, py, 0.1f));
                    else
                        fc[i] += vw[j] * (ca[i][j] + 0.1f * 5.0f);
                } else {
                    fc[i] += vw[j] * ca[i][j];
                }
            }
        }
        fc[i] /= wn;
    }
    int min_idx = 0;
    {
        float m = fc[0];
        for (int i = 1; i < 8; ++i)
            if (fc[i] <= m) {
                m = fc[i];
                min_idx = i;
            }
    }

    float cvn[MAXV];
    cost_vector(c, px, py, c->planes[center], cvn);
    float cost_now = 0.0f;
    for (int i = 0; i < nv; ++i) {
        if (c->geom)
            cost_now += vw[i] * (cvn[i] + geom_term(c, i + 1, c->planes[center], px, py, c->acmm ? 0.2f : 0.1f));
        else
            cost_now += vw[i] * cvn[i];
    }
    cost_now /= wn;
    c->costs[center] = cost_now;
    float depth_now = depth_from_plane(cam, c->planes[center], px, py);

    if (c->acmm) {
        /* ACMM.cu:1602-1629: the winner is built in plane_hypotheses_now,
         * which the reference declares without a value and reads when no
         * direction wins; it starts here from the current hypothesis, the
         * in-place update of HPM.cu:1707-1724 that the variant restructures.
         * No planar prior and no NaN fallback; a hierarchy pass keeps the
         * result only if it beats the upsampled plane's cost by 0.1. */
        F4 now = c->planes[center];
        float cost = cost_now;
        if (flag[min_idx]) {
            const float db = depth_from_plane(cam, c->planes[pos[min_idx]], px, py);
            if (db >= c->dmin && db <= c->dmax && fc[min_idx] < cost_now) {
                depth_now = db;
                now = c->planes[pos[min_idx]];
                cost = fc[min_idx];
                c->views[center] = tsv;
            }
        }
        float unused = 0.0f;
        refine(c, px, py, &now, &depth_now, &cost, &rng, vw, wn, &unused);
        if (!c->hier || cost < c->pre_costs[center] - 0.1f) {
            c->costs[center] = cost;
            c->planes[center] = now;
        }
        return;
    }

    float restricted_cost = 0.0f;
    if (c->prior) {
        const float depth_sigma = (c->dmax - c->dmin) / 64.0f;
        const float two_dss = 2 * depth_sigma * depth_sigma;
        const float angle_sigma = (float)(OR_PI * (5.0f / 180.0f));
        const float two_ass = 2 * angle_sigma * angle_sigma;
        const float depth_prior = depth_from_plane(cam, c->prior_planes[center], px, py);
        const float beta = 0.18f;
        if (c->masks[center] > 0) {
            float rfc[8] = {0};
            for (int i = 0; i < 8; i++) {
                if (flag[i]) {
                    const F4 hq = c->planes[pos[i]];
                    const float dn = depth_from_plane(cam, hq, px, py);
                    const float pr = restricted_prior(dn - depth_prior, dot3(c->prior_planes[center], hq), two_dss,
                                                      two_ass);
                    rfc[i] = expf(-fc[i] * fc[i] / beta) * pr;
                }
            }
            int max_idx = 0;
            {
                float m = rfc[0];
                for (int i = 1; i < 8; ++i)
                    if (rfc[i] >= m) {
                        m = rfc[i];
                        max_idx = i;
                    }
            }
            const float dn = depth_from_plane(cam, c->planes[center], px, py);
            const float pr =
                restricted_prior(dn - depth_prior, dot3(c->prior_planes[center], c->planes[center]), two_dss, two_ass);
            const float rcn = expf(-cost_now * cost_now / beta) * pr;
            if (flag[max_idx]) {
                const float db = depth_from_plane(cam, c->planes[pos[max_idx]], px, py);
                if (db >= c->dmin && db <= c->dmax && rfc[max_idx] > rcn) {
                    depth_now = db;
                    c->planes[center] = c->planes[pos[max_idx]];
                    c->costs[center] = fc[max_idx];
                    restricted_cost = rfc[max_idx];
                    c->views[center] = tsv;
                }
            }
        } else if (flag[min_idx]) {
            const float db = depth_from_plane(cam, c->planes[pos[min_idx]], px, py);
            if (db >= c->dmin && db <= c->dmax && fc[min_idx] < cost_now) {
                depth_now = db;
                c->planes[center] = c->planes[pos[min_idx]];
                c->costs[center] = fc[min_idx];
            }
        }
    }
    if (!c->prior && flag[min_idx]) {
        const float db = depth_from_plane(cam, c->planes[pos[min_idx]], px, py);
        if (db >= c->dmin && db <= c->dmax && fc[min_idx] < cost_now) {
            depth_now = db;
            c->planes[center] = c->planes[pos[min_idx]];
            c->costs[center] = fc[min_idx];
            c->views[center] = tsv;
        }
        if (c->costs[center] != c->costs[center]) {
            depth_now = db;
            c->planes[center] = c->planes[pos[min_idx]];
            cost_now = fc[min_idx];
            c->views[center] = tsv;
        }
    }
    F4 plane = c->planes[center];
    float cost = c->costs[center];
    refine(c, px, py, &plane, &depth_now, &cost, &rng, vw, wn, &restricted_cost);
    c->planes[center] = plane;
    c->costs[center] = cost;
}

/* rows reached by the checkerboard grid of HPM.cu:1924-1931 */
static int rows_covered(int H) { return 2 * (((H / 2) + 15) / 16) * 16; }

static void half_step(Ctx *c, int color, int iter)
{
    const int hc = rows_covered(c->H) < c->H ? rows_covered(c->H) : c->H;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int y = 0; y < hc; ++y) {
        for (int x = ((y + color) & 1); x < c->W; x += 2) propagate_pixel(c, x, y, iter);
    }
}

/* CheckerboardFilter, HPM.cu:1766-1880 */
static void filter_pixel(F4 *pl, const float *costs, int W, int H, int px, int py)
{
    const int center = py * W + px;
    float f[21];
    int n = 0;
    f[n++] = pl[center].w;
    const int left = center - 1, leftleft = center - 3, up = center - W, upup = center - 3 * W;
    const int down = center + W, downdown = center + 3 * W, right = center + 1, rightright = center + 3;
    if (costs[center] < 0.001f) return;
    if (py > 0) f[n++] = pl[up].w;
    if (py > 2) f[n++] = pl[upup].w;
    if (py > 4) f[n++] = pl[upup - W * 2].w;
    if (py < H - 1) f[n++] = pl[down].w;
    if (py < H - 3) f[n++] = pl[downdown].w;
    if (py < H - 5) f[n++] = pl[downdown + W * 2].w;
    if (px > 0) f[n++] = pl[left].w;
    if (px > 2) f[n++] = pl[leftleft].w;
    if (px > 4) f[n++] = pl[leftleft - 2].w;
    if (px < W - 1) f[n++] = pl[right].w;
    if (px < W - 3) f[n++] = pl[rightright].w;
    if (px < W - 5) f[n++] = pl[rightright + 2].w;
    if (py > 0 && px < W - 2) f[n++] = pl[up + 2].w;
    if (py < H - 1 && px < W - 2) f[n++] = pl[down + 2].w;
    if (py > 0 && px > 1) f[n++] = pl[up - 2].w;
    if (py < H - 1 && px > 1) f[n++] = pl[down - 2].w;
    if (px > 0 && py > 2) f[n++] = pl[left - W * 2].w;
    if (px < W - 1 && py > 2) f[n++] = pl[right - W * 2].w;
    if (px > 0 && py < H - 2) f[n++] = pl[left + W * 2].w;
    if (px < W - 1 && py < H - 2) f[n++] = pl[right + W * 2].w;
    sort_small(f, n);
    const int m = n / 2;
    pl[center].w = (n % 2 == 0) ? (f[m - 1] + f[m]) / 2 : f[m];
}

int or_depth_normal_filter(const OrCamera *ref, float *planes_io, const float *costs)
{
    const int W = ref->width, H = ref->height;
    F4 *pl = (F4 *)planes_io;
    for (int y = 0; y < H; ++y) /* GetDepthandNormal, HPM.cu:1751-1764 */
        for (int x = 0; x < W; ++x) {
            F4 h = pl[y * W + x];
            h.w = depth_from_plane(ref, h, x, y);
            pl[y * W + x] = transform_normal(ref, h);
        }
    const int hc = rows_covered(H) < H ? rows_covered(H) : H;
    for (int color = 0; color < 2; ++color)
        for (int y = 0; y < hc; ++y)
            for (int x = ((y + color) & 1); x < W; x += 2) filter_pixel(pl, costs, W, H, x, y);
    return 0;
}

int or_run_patchmatch(int n_img, const float *const *imgs, const OrCamera *cams, const OrRunOpts *o,
                      float *planes_io, float *costs_io, uint32_t *views_io, const float *prior_planes,
                      const uint32_t *plane_masks, const float *const *depth_maps)
{
    if (n_img < 2 || n_img > MAXV + 1) return -1;
    Ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n_img;
    c.imgs = imgs;
    c.cams = cams;
    c.depths = depth_maps;
    c.W = cams[0].width;
    c.H = cams[0].height;
    c.geom = o->geom_consistency;
    c.prior = o->planar_prior;
    c.dmin = o->depth_min;
    c.dmax = o->depth_max;
    c.seed = o->seed;
    c.salt = o->salt;
    c.planes = (F4 *)planes_io;
    c.costs = costs_io;
    c.acmm = o->variant == 1;
    c.hier = c.acmm ? o->hierarchy : 0;
    c.pre_costs = o->pre_costs;
    if (c.hier && !c.pre_costs) return -3;
    if (c.acmm && c.prior) return -4;
    const size_t npx = (size_t)c.W * c.H;
    uint32_t *views = views_io ? views_io : (uint32_t *)calloc(npx, sizeof(uint32_t));
    uint32_t *zero_masks = NULL;
    c.views = views;
    c.prior_planes = (const F4 *)prior_planes;
    c.masks = plane_masks;

    if (c.prior && !c.masks) {
        zero_masks = (uint32_t *)calloc(npx, sizeof(uint32_t));
        c.masks = zero_masks;
    }
    if (c.geom && !c.depths) return -2;

#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int y = 0; y < c.H; ++y)
        for (int x = 0; x < c.W; ++x) init_pixel(&c, x, y);
    int hs = 0;
    for (int iter = 0; iter < 3 && hs < o->half_steps; ++iter) {
        for (int color = 0; color < 2 && hs < o->half_steps; ++color, ++hs) half_step(&c, color, iter);
    }
    if (o->finalize) or_depth_normal_filter(&cams[0], planes_io, costs_io);
    if (!views_io) free(views);
    free(zero_masks);
    return 0;
}

int or_cost_vectors(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float *out)
{
    Ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n_img;
    c.imgs = imgs;
    c.cams = cams;
    c.W = cams[0].width;
    c.H = cams[0].height;
    const F4 *pl = (const F4 *)planes4;
#ifdef _OPENMP
#pragma omp parallel for
#endif
    for (int y = 0; y < c.H; ++y)
        for (int x = 0; x < c.W; ++x) {
            float cv[MAXV];
            cost_vector(&c, x, y, pl[y * c.W + x], cv);
            for (int i = 0; i < n_img - 1; ++i) out[((size_t)y * c.W + x) * (n_img - 1) + i] = cv[i];
        }
    return 0;
}

int or_initial_costs(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4,
                     float *out_cost, uint32_t *out_views)
{
    Ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n_img;
    c.imgs = imgs;
    c.cams = cams;
    c.W = cams[0].width;
    c.H = cams[0].height;
    const F4 *pl = (const F4 *)planes4;
#ifdef _OPENMP
#pragma omp parallel for
#endif
    for (int y = 0; y < c.H; ++y)
        for (int x = 0; x < c.W; ++x)
            out_cost[y * c.W + x] = initial_cost(&c, x, y, pl[y * c.W + x], &out_views[y * c.W + x]);
    return 0;
}

int or_geom_costs(int n_img, const OrCamera *cams, const float *const *depths, const float *planes4, float *out)
{
    const int W = cams[0].width, H = cams[0].height;
    const F4 *pl = (const F4 *)planes4;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int i = 1; i < n_img; ++i)
                out[((size_t)y * W + x) * (n_img - 1) + i - 1] =
                    geom_cost(&cams[0], &cams[i], depths[i], pl[y * W + x], x, y);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Joint bilateral upsampling: JBU_cu, HPM.cu:1971-2052                */
/* ------------------------------------------------------------------ */

int or_jbu(const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal, int s_cols,
           int s_rows, float *out_depth, float *out_normal)
{
    const int sr = rows / s_rows, sc = cols / s_cols;
    const int image_scale = sr > sc ? sr : sc;
    if (image_scale == 1) return 1;
    return or_jbu_at_scale(guide, cols, rows, coarse_depth, coarse_normal, s_cols, s_rows, image_scale, out_depth,
                           out_normal);
}

int or_jbu_at_scale(const float *guide, int cols, int rows, const float *coarse_depth, const float *coarse_normal,
                    int s_cols, int s_rows, int image_scale, float *out_depth, float *out_normal)
{
    const float scale = (float)(1.0 * s_cols / cols);
    const float sigmad = 0.50f, sigmar = 25.5f;
    const int win = image_scale * image_scale + 1;
    const int nn = win / 2;
#ifdef _OPENMP
#pragma omp parallel for
#endif
    for (int py = 0; py < rows; ++py) {
        for (int px = 0; px < cols; ++px) {
            const float oy = (float)py * scale, ox = (float)px * scale;
            const float ref_pix = texel(guide, cols, rows, px, py);
            float nf = 0.0f, ctot = 0.0f, nx = 0.0f, ny = 0.0f, nz = 0.0f;
            for (int j = -nn; j <= nn; ++j) {
                int ry = f2i_rz_sat(oy + (float)j);
                ry = ry > 0 ? (ry < s_rows ? ry : s_rows - 1) : 0;
                const int rys = py + j;
                for (int i = -nn; i <= nn; ++i) {
                    int rx = f2i_rz_sat(ox + (float)i);
                    rx = rx > 0 ? (rx < s_cols ? rx : s_cols - 1) : 0;
                    const size_t sc_i = (size_t)ry * s_cols + rx;
                    const float src_pix = coarse_depth[sc_i];
                    const int rxs = px + i;
                    const float nb_pix = texel(guide, cols, rows, rxs, rys);
                    /* SpatialGauss: pow(float,2) promotes to double, exp is double */
                    const float dis = (float)(pow((double)(ox - (float)rx), 2) + pow((double)(oy - (float)ry), 2) - 0.0);
                    const float sg = (float)exp(-1.0 * dis / (double)(2 * sigmad * sigmad));
                    const float xp = fabsf(ref_pix - nb_pix) - 0.0f;
                    const float rg = (float)exp(-1.0 * (double)(xp * xp) / (double)(2 * sigmar * sigmar));
                    const float tg = sg * rg;
                    nf += tg;
                    ctot += src_pix * tg;
                    nx += coarse_normal[3 * sc_i] * tg;
                    ny += coarse_normal[3 * sc_i + 1] * tg;
                    nz += coarse_normal[3 * sc_i + 2] * tg;
                }
            }
            F4 n = {nx / nf, ny / nf, nz / nf, 0.0f};
            normalize3(&n);
            const size_t c = (size_t)py * cols + px;
            out_depth[c] = ctot / nf;
            out_normal[3 * c] = n.x;
            out_normal[3 * c + 1] = n.y;
            out_normal[3 * c + 2] = n.z;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Host prior stages                                                   */
/* ------------------------------------------------------------------ */

int or_support_points(const float *costs, int w, int h, int *out_xy, int max_points)
{
    const int step = 5;
    int n = 0;
    for (int col = 0; col < w; col += step) {
        for (int row = 0; row < h; row += step) {
            float min_cost = 2.0f;
            int tx = 0, ty = 0;
            const int cb = w < col + step ? w : col + step;
            const int rb = h < row + step ? h : row + step;
            for (int cc = col; cc < cb; ++cc)
                for (int r = row; r < rb; ++r) {
                    const float v = costs[(size_t)r * w + cc];
                    if (v < 2.0f && min_cost > v) {
                        tx = cc;
                        ty = r;
                        min_cost = v;
                    }
                }
            if (min_cost < 0.1f) {
                if (n < max_points) {
                    out_xy[2 * n] = tx;
                    out_xy[2 * n + 1] = ty;
                }
                n++;
            }
        }
    }
    return n;
}

static double det3(double a, double b, double c, double d, double e, double f, double g, double h, double i)
{
    return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

void or_plane_from_triangle(const OrCamera *ref, const float *depth, int w, const int *t, float factor, float *out4)
{
    float P[3][3];
    for (int k = 0; k < 3; ++k) {
        const int x = t[2 * k], y = t[2 * k + 1];
        const float d = depth[(size_t)y * w + x];
        /* Get3DPointonRefCam_factor, HPM.cpp:236-245 */
        P[k][0] = d * ((float)x - ref->K[2] * factor) / (ref->K[0] * factor);
        P[k][1] = d * ((float)y - ref->K[5] * factor) / (ref->K[4] * factor);
        P[k][2] = d;
    }
    /* null vector of [P 1] (cv::SVD::solveZ in HPM.cpp:832) by cofactors */
    double n[4];
    n[0] = det3(P[0][1], P[0][2], 1, P[1][1], P[1][2], 1, P[2][1], P[2][2], 1);
    n[1] = -det3(P[0][0], P[0][2], 1, P[1][0], P[1][2], 1, P[2][0], P[2][2], 1);
    n[2] = det3(P[0][0], P[0][1], 1, P[1][0], P[1][1], 1, P[2][0], P[2][1], 1);
    n[3] = -det3(P[0][0], P[0][1], P[0][2], P[1][0], P[1][1], P[1][2], P[2][0], P[2][1], P[2][2]);
    const double s = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + n[3] * n[3]);
    float n4[4] = {(float)(n[0] / s), (float)(n[1] / s), (float)(n[2] / s), (float)(n[3] / s)};
    float norm2 = (float)sqrt(pow(n4[0], 2) + pow(n4[1], 2) + pow(n4[2], 2));
    if (n4[3] < 0) norm2 *= -1;
    for (int k = 0; k < 4; ++k) out4[k] = n4[k] / norm2;
}

float or_depth_from_plane(const OrCamera *ref, const float *p, int x, int y, float factor)
{
    return -p[3] * (ref->K[0] * factor) /
           (((float)x - ref->K[2] * factor) * p[0] + (ref->K[0] / ref->K[4]) * ((float)y - ref->K[5] * factor) * p[1] +
            ref->K[0] * factor * p[2]);
}

int or_raster_triangles(const int *tris, int n_tris, int w, int h, float *mask, int *kept6)
{
    unsigned int idx = 0;
    for (int t = 0; t < n_tris; ++t) {
        const int *v = tris + 6 * t;
        int inside = 1;
        for (int k = 0; k < 3; ++k)
            if (!(v[2 * k] >= 0 && v[2 * k] < w && v[2 * k + 1] >= 0 && v[2 * k + 1] < h)) inside = 0;
        if (!inside) continue;
        const float L01 = (float)sqrt(pow(v[0] - v[2], 2) + pow(v[1] - v[3], 2));
        const float L02 = (float)sqrt(pow(v[0] - v[4], 2) + pow(v[1] - v[5], 2));
        const float L12 = (float)sqrt(pow(v[2] - v[4], 2) + pow(v[3] - v[5], 2));
        const float mx = L01 > (L02 > L12 ? L02 : L12) ? L01 : (L02 > L12 ? L02 : L12);
        const float step = (float)(1.0 / mx);
        for (float p = 0; p < 1.0; p += step) {
            for (float q = 0; q < 1.0 - p; q += step) {
                const int x = (int)(p * v[0] + q * v[2] + (1.0 - p - q) * v[4]);
                const int y = (int)(p * v[1] + q * v[3] + (1.0 - p - q) * v[5]);
                mask[(size_t)y * w + x] = (float)(idx + 1.0);
            }
        }
        if (kept6) memcpy(kept6 + 6 * idx, v, 6 * sizeof(int));
        idx++;
    }
    return (int)idx;
}

static float distf(int x1, int y1, int x2, int y2) /* Distance, HPM.cpp:923-926 */
{
    const float tmp = (float)((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2));
    return sqrtf(tmp);
}

static int not_on_line(const int *a, const int *b, const int *c) /* JudgeNotOnline, HPM.cpp:928-937 */
{
    const float l1 = distf(a[0], a[1], b[0], b[1]);
    const float l2 = distf(a[0], a[1], c[0], c[1]);
    const float l3 = distf(c[0], c[1], b[0], b[1]);
    const float area = (float)(0.5 * (l1 + l2 + l3));
    return area * (area - l1) * (area - l2) * (area - l3) > 0;
}

/* triple order of HPM.cpp:982-1081 (0-based indices into the 6 neighbours) */
static const int kTriples[20][3] = {{0, 1, 2}, {0, 1, 3}, {0, 1, 4}, {0, 2, 3}, {0, 2, 4}, {0, 3, 4}, {1, 2, 3},
                                    {1, 2, 4}, {1, 3, 4}, {2, 3, 4}, {0, 1, 5}, {0, 2, 5}, {0, 3, 5}, {0, 4, 5},
                                    {1, 2, 5}, {1, 3, 5}, {1, 4, 5}, {2, 3, 5}, {2, 4, 5}, {3, 4, 5}};

/* Insert (d, k) into the sorted 6-list, ordered by distance, then index. */
static void knn6_insert(long d, int k, long *bd, int *best, int *nb)
{
    if (*nb == 6 && (d > bd[5] || (d == bd[5] && k > best[5]))) return;
    int pos = *nb < 6 ? (*nb)++ : 5;
    while (pos > 0 && (bd[pos - 1] > d || (bd[pos - 1] == d && best[pos - 1] > k))) {
        bd[pos] = bd[pos - 1];
        best[pos] = best[pos - 1];
        pos--;
    }
    bd[pos] = d;
    best[pos] = k;
}

static void knn6_brute(const int *pts, int n_pts, int x, int y, int *best)
{
    long bd[6];
    int nb = 0;
    for (int k = 0; k < n_pts; ++k) {
        const long dx = pts[2 * k] - x, dy = pts[2 * k + 1] - y;
        knn6_insert(dx * dx + dy * dy, k, bd, best, &nb);
    }
}

/* Uniform grid of kGridCell-pixel cells (CSR, indices ascending per cell). */
enum { kGridCell = 8 };
typedef struct {
    int gw, gh;
    int *start, *idx;
} KnnGrid;

static void knn_grid_build(KnnGrid *g, const int *pts, int n_pts, int w, int h)
{
    g->gw = (w + kGridCell - 1) / kGridCell;
    g->gh = (h + kGridCell - 1) / kGridCell;
    const int nc = g->gw * g->gh;
    g->start = (int *)calloc((size_t)nc + 1, sizeof(int));
    g->idx = (int *)malloc(sizeof(int) * (size_t)(n_pts > 0 ? n_pts : 1));
    for (int k = 0; k < n_pts; ++k) g->start[1 + (pts[2 * k + 1] / kGridCell) * g->gw + pts[2 * k] / kGridCell]++;
    for (int c = 0; c < nc; ++c) g->start[c + 1] += g->start[c];
    int *fill = (int *)malloc(sizeof(int) * (size_t)nc);
    memcpy(fill, g->start, sizeof(int) * (size_t)nc);
    for (int k = 0; k < n_pts; ++k) g->idx[fill[(pts[2 * k + 1] / kGridCell) * g->gw + pts[2 * k] / kGridCell]++] = k;
    free(fill);
}

/* Exact: rings of cells around the query's cell until the 6th distance is
 * below the distance to anything outside the visited block. */
static void knn6_grid(const KnnGrid *g, const int *pts, int x, int y, int *best)
{
    long bd[6];
    int nb = 0;
    const int cx = x / kGridCell, cy = y / kGridCell;
    for (int r = 0;; ++r) {
        for (int gy = cy - r; gy <= cy + r; ++gy) {
            if (gy < 0 || gy >= g->gh) continue;
            const int step = (gy == cy - r || gy == cy + r) ? 1 : 2 * r;
            for (int gx = cx - r; gx <= cx + r; gx += step > 0 ? step : 1) {
                if (gx < 0 || gx >= g->gw) continue;
                const int c = gy * g->gw + gx;
                for (int q = g->start[c]; q < g->start[c + 1]; ++q) {
                    const int k = g->idx[q];
                    const long dx = pts[2 * k] - x, dy = pts[2 * k + 1] - y;
                    knn6_insert(dx * dx + dy * dy, k, bd, best, &nb);
                }
            }
        }
        if (cx - r <= 0 && cy - r <= 0 && cx + r >= g->gw - 1 && cy + r >= g->gh - 1) return;
        if (nb == 6) {
            /* nearest integer position outside cells [cx-r, cx+r] x [cy-r, cy+r] */
            long b = x - ((long)(cx - r) * kGridCell - 1);
            const long bx2 = (long)(cx + r + 1) * kGridCell - x;
            const long by1 = y - ((long)(cy - r) * kGridCell - 1), by2 = (long)(cy + r + 1) * kGridCell - y;
            if (bx2 < b) b = bx2;
            if (by1 < b) b = by1;
            if (by2 < b) b = by2;
            if (bd[5] < b * b) return;
        }
    }
}

/* The 6 nearest of n_pts points for every pixel whose mask is <= 0 (every
 * pixel without a mask), by brute force; -1 elsewhere and past n_pts. */
void or_knn6(const int *pts, int n_pts, int w, int h, const float *mask, int *nn6)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            int *o = nn6 + 6 * ((size_t)y * w + x);
            for (int k = 0; k < 6; ++k) o[k] = -1;
            if (mask && mask[(size_t)y * w + x] > 0) continue;
            knn6_brute(pts, n_pts, x, y, o);
        }
}

static int g_knn_grid = 1;

void or_set_knn_grid(int on) { g_knn_grid = on; }

void or_knn_supplement(const OrCamera *ref, const int *pts, int n_pts, const float *depth, int w, int h, float factor,
                       float dmin, float dmax, float *plane_out, float *mask)
{
    if (n_pts < 6) return;
    KnnGrid g = {0, 0, NULL, NULL};
    if (g_knn_grid) knn_grid_build(&g, pts, n_pts, w, h);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int i = 0; i < h; i++) {
        for (int j = 0; j < w; j++) {
            if (mask[(size_t)i * w + j] > 0) continue;
            /* exact 6 nearest support points; ties broken by insertion order */
            int best[6];
            if (g_knn_grid)
                knn6_grid(&g, pts, j, i, best);
            else
                knn6_brute(pts, n_pts, j, i, best);
            int sel = -1;
            for (int tI = 0; tI < 20; ++tI) {
                if (not_on_line(pts + 2 * best[kTriples[tI][0]], pts + 2 * best[kTriples[tI][1]],
                                pts + 2 * best[kTriples[tI][2]])) {
                    sel = tI;
                    break;
                }
            }
            if (sel < 0) continue;
            int tri[6];
            for (int k = 0; k < 3; ++k) {
                tri[2 * k] = pts[2 * best[kTriples[sel][k]]];
                tri[2 * k + 1] = pts[2 * best[kTriples[sel][k]] + 1];
            }
            float n4[4];
            or_plane_from_triangle(ref, depth, w, tri, factor, n4);
            const float d = or_depth_from_plane(ref, n4, j, i, factor);
            if (d <= dmax && d >= dmin) {
                mask[(size_t)i * w + j] = -233.0f;
                memcpy(plane_out + 4 * ((size_t)i * w + j), n4, sizeof(n4));
            }
        }
    }
    free(g.start);
    free(g.idx);
}

/* TransformNormal (HPM.cpp:872-880): ref-frame normal to world, R^T n. */
static void to_world(const OrCamera *ref, const float *n, float *out)
{
    const float *R = ref->R;
    out[0] = R[0] * n[0] + R[3] * n[1] + R[6] * n[2];
    out[1] = R[1] * n[0] + R[4] * n[1] + R[7] * n[2];
    out[2] = R[2] * n[0] + R[5] * n[1] + R[8] * n[2];
}

void or_prior_coarse(const OrCamera *ref, const float *mask, const float *tri_planes, int n_tri,
                     const float *knn_planes, int w, int h, float factor, float dmin, float dmax, float *out_depth,
                     float *out_normal3)
{
    for (size_t i = 0; i < (size_t)w * h; ++i) {
        out_depth[i] = 0.0f;
        out_normal3[3 * i] = out_normal3[3 * i + 1] = out_normal3[3 * i + 2] = 0.0f;
    }
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const size_t c = (size_t)y * w + x;
            const float m = mask[c];
            const float *pl = NULL;
            float lo = dmin, hi = dmax;
            if (m > 0) {
                const int t = (int)m - 1;
                if (t < 0 || t >= n_tri) continue;
                pl = tri_planes + 4 * t;
                lo = dmin * 0.6f; /* main.cpp:129 widens the range once more */
                hi = dmax * 1.2f;
            } else if (m < -200) {
                pl = knn_planes + 4 * c;
            } else {
                continue;
            }
            const float d = or_depth_from_plane(ref, pl, x, y, factor);
            if (d <= hi && d >= lo) {
                out_depth[c] = d;
                to_world(ref, pl, out_normal3 + 3 * c);
            }
        }
    }
}

void or_prior_reload(const OrCamera *ref, const float *depth, const float *normal3, int w, int h, float dmin,
                     float dmax, float *out4, unsigned int *out_mask)
{
    const float *R = ref->R, *K = ref->K;
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const size_t c = (size_t)y * w + x;
            const float d = depth[c];
            out4[4 * c] = out4[4 * c + 1] = out4[4 * c + 2] = out4[4 * c + 3] = 0.0f;
            out_mask[c] = 0;
            if (!(d <= dmax && d >= dmin)) continue;
            const float *n = normal3 + 3 * c;
            /* TransformNormal2RefCam (HPM.cpp:882-890), GetDistance2Origin_factor (HPM.cpp:892-899) */
            const float nx = R[0] * n[0] + R[1] * n[1] + R[2] * n[2];
            const float ny = R[3] * n[0] + R[4] * n[1] + R[5] * n[2];
            const float nz = R[6] * n[0] + R[7] * n[1] + R[8] * n[2];
            const float X0 = d * ((float)x - K[2]) / K[0];
            const float X1 = d * ((float)y - K[5]) / K[4];
            out4[4 * c] = nx;
            out4[4 * c + 1] = ny;
            out4[4 * c + 2] = nz;
            out4[4 * c + 3] = -(nx * X0 + ny * X1 + nz * d);
            out_mask[c] = 1;
        }
    }
}

void or_prior_full(const OrCamera *ref, const float *mask, const float *tri_planes, int n_tri,
                   const float *knn_planes, int w, int h, float dmin, float dmax, float *out4,
                   unsigned int *out_mask, float *out_depth)
{
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) {
            const size_t c = (size_t)y * w + x;
            const float m = mask[c];
            out4[4 * c] = out4[4 * c + 1] = out4[4 * c + 2] = out4[4 * c + 3] = 0.0f;
            out_mask[c] = 0;
            out_depth[c] = 0.0f;
            const float *pl = NULL;
            unsigned int mv = 0;
            if (m > 0) {
                const int t = (int)m - 1;
                if (t < 0 || t >= n_tri) continue;
                pl = tri_planes + 4 * t;
                mv = (unsigned int)(int)m;
            } else if (m < -200) {
                pl = knn_planes + 4 * c;
                mv = 0xFFFFFF17u; /* (unsigned int)-233.0f, HPM.cpp:1112 */
            } else {
                continue;
            }
            const float d = or_depth_from_plane(ref, pl, x, y, 1.0f);
            if (d <= dmax && d >= dmin) {
                out_depth[c] = d;
                memcpy(out4 + 4 * c, pl, 4 * sizeof(float));
                out_mask[c] = mv;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Fusion (RunFusion, main.cpp:502-633)                                */
/* ------------------------------------------------------------------ */

/* Get3DPointonWorld (HPM.cpp:210-234) */
static void fu_world(const OrCamera *c, int x, int y, float depth, float *X)
{
    const float px = depth * ((float)x - c->K[2]) / c->K[0];
    const float py = depth * ((float)y - c->K[5]) / c->K[4];
    const float pz = depth;
    const float *R = c->R, *t = c->t;
    const float tx = R[0] * px + R[3] * py + R[6] * pz;
    const float ty = R[1] * px + R[4] * py + R[7] * pz;
    const float tz = R[2] * px + R[5] * py + R[8] * pz;
    const float cx = -(R[0] * t[0] + R[3] * t[1] + R[6] * t[2]);
    const float cy = -(R[1] * t[0] + R[4] * t[1] + R[7] * t[2]);
    const float cz = -(R[2] * t[0] + R[5] * t[1] + R[8] * t[2]);
    X[0] = tx + cx;
    X[1] = ty + cy;
    X[2] = tz + cz;
}

/* ProjectonCamera (HPM.cpp:247-257) */
static void fu_project(const float *X, const OrCamera *c, float *pt, float *depth)
{
    const float *R = c->R, *K = c->K, *t = c->t;
    const float x = R[0] * X[0] + R[1] * X[1] + R[2] * X[2] + t[0];
    const float y = R[3] * X[0] + R[4] * X[1] + R[5] * X[2] + t[1];
    const float z = R[6] * X[0] + R[7] * X[1] + R[8] * X[2] + t[2];
    *depth = K[6] * x + K[7] * y + K[8] * z;
    pt[0] = (K[0] * x + K[1] * y + K[2] * z) / *depth;
    pt[1] = (K[3] * x + K[4] * y + K[5] * z) / *depth;
}

/* (int)f of the reference's x86 host build: truncation, INT_MIN (the
 * "integer indefinite" of cvttss2si) for NaN and out-of-range values */
static int trunc_int(float f)
{
    if (f != f || f >= 2147483648.0f || f < -2147483648.0f) return (-2147483647 - 1);
    return (int)f;
}

/* GetAngle (HPM.cpp:259-268) */
static float fu_angle(const float *a, const float *b)
{
    const float d = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    const float ang = acosf(d);
    return ang != ang ? 0.0f : ang;
}

/* RunFusion of HPM-MVS (main.cpp:502-633, acmm 0) or of the ACMM+NESP
 * variant (ACMM+NESP/windows/main.cpp:154-297, acmm 1).  The variant keeps a
 * pixel consistent with at least 2 sources and writes the mean of its point,
 * normal and colour with those of the agreeing source pixels; HPM-MVS keeps
 * one with at least 1 source whose mean exp(-error) exceeds 0.3 and writes
 * the reference pixel's own. */
static long fuse_impl(int acmm, int n_views, const OrCamera *cams, const float *const *depths,
                      const float *const *normals, const unsigned char *const *colors, int n_problems,
                      const int *ref_ids, const int *src_counts, const int *src_ids, float *out_xyz,
                      float *out_normal, float *out_color, long cap)
{
    unsigned char **masks = (unsigned char **)calloc((size_t)n_views, sizeof(*masks));
    for (int v = 0; v < n_views; ++v) masks[v] = (unsigned char *)calloc((size_t)cams[v].width * cams[v].height, 1);
    long n_out = 0;
    for (int pi = 0; pi < n_problems; ++pi) {
        const int i = ref_ids[pi];
        const OrCamera *ci = &cams[i];
        const int cols = ci->width, rows = ci->height, ns = src_counts[pi];
        int used_x[32], used_y[32];
        for (int j = 0; j < ns; ++j) used_x[j] = used_y[j] = -1; /* kept across pixels (main.cpp:557) */
        for (int r = 0; r < rows; ++r) {
            for (int c = 0; c < cols; ++c) {
                const size_t ctr = (size_t)r * cols + c;
                if (masks[i][ctr] == 1) continue;
                const float ref_depth = depths[i][ctr];
                const float *ref_n = normals[i] + 3 * ctr;
                if (ref_depth <= 0.0) continue;
                float X[3];
                fu_world(ci, c, r, ref_depth, X);
                int num = 0;
                float dyn = 0;
                /* the variant's sums: point, normal (cv::Vec3f), colour */
                float sp[3] = {X[0], X[1], X[2]}, sn[3] = {ref_n[0], ref_n[1], ref_n[2]}, scol[3];
                for (int k = 0; k < 3; ++k) scol[k] = (float)colors[i][3 * ctr + k];
                for (int j = 0; j < ns; ++j) {
                    const int s = src_ids[pi * 32 + j];
                    const OrCamera *cs = &cams[s];
                    float pt[2], proj_depth;
                    fu_project(X, cs, pt, &proj_depth);
                    const int sr = trunc_int(pt[1] + 0.5f), sc = trunc_int(pt[0] + 0.5f);
                    if (sc >= 0 && sc < cs->width && sr >= 0 && sr < cs->height) {
                        const size_t sctr = (size_t)sr * cs->width + sc;
                        if (masks[s][sctr] == 1) continue;
                        const float src_depth = depths[s][sctr];
                        const float *src_n = normals[s] + 3 * sctr;
                        if (src_depth <= 0.0) continue;
                        float Y[3], tp[2];
                        fu_world(cs, sc, sr, src_depth, Y);
                        fu_project(Y, ci, tp, &proj_depth);
                        const float dx = (float)c - tp[0], dy = (float)r - tp[1];
                        const float reproj = (float)sqrt((double)dx * dx + (double)dy * dy);
                        const float rel = fabsf(proj_depth - ref_depth) / ref_depth;
                        const float ang = fu_angle(ref_n, src_n);
                        if (reproj < 2.0f && rel < 0.01f && ang < 0.174533f) {
                            if (acmm) { /* ACMM+NESP/windows/main.cpp:254-261 */
                                for (int k = 0; k < 3; ++k) {
                                    sp[k] += Y[k];
                                    sn[k] = sn[k] + src_n[k];
                                    scol[k] += (float)colors[s][3 * sctr + k];
                                }
                            }
                            used_x[j] = sc;
                            used_y[j] = sr;
                            const float idx = reproj + 200 * rel + ang * 10;
                            if (!acmm) dyn += expf(-idx);
                            num++;
                        }
                    }
                }
                if (acmm ? num >= 2 : (num >= 1 && (dyn > 0.3 * num))) {
                    if (acmm) { /* ACMM+NESP/windows/main.cpp:270-277 */
                        const float div = num + 1.0f;
                        /* cv::Vec3f /= float multiplies by the float reciprocal (OpenCV core/matx.hpp) */
                        const float inv = 1.f / div;
                        for (int k = 0; k < 3; ++k) {
                            sp[k] /= div;
                            sn[k] = sn[k] * inv;
                            scol[k] /= div;
                        }
                    }
                    if (n_out < cap) {
                        memcpy(out_xyz + 3 * n_out, acmm ? sp : X, sizeof(X));
                        memcpy(out_normal + 3 * n_out, acmm ? sn : ref_n, 3 * sizeof(float));
                        for (int k = 0; k < 3; ++k)
                            out_color[3 * n_out + k] = acmm ? scol[k] : (float)colors[i][3 * ctr + k];
                    }
                    n_out++;
                    for (int j = 0; j < ns; ++j) {
                        if (used_x[j] == -1) continue;
                        const int s = src_ids[pi * 32 + j];
                        masks[s][(size_t)used_y[j] * cams[s].width + used_x[j]] = 1;
                    }
                }
            }
        }
    }
    for (int v = 0; v < n_views; ++v) free(masks[v]);
    free(masks);
    return n_out;
}

long or_fuse(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
             const unsigned char *const *colors, int n_problems, const int *ref_ids, const int *src_counts,
             const int *src_ids, float *out_xyz, float *out_normal, float *out_color, long cap)
{
    return fuse_impl(0, n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids, out_xyz,
                     out_normal, out_color, cap);
}

long or_fuse_acmm(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
                  const unsigned char *const *colors, int n_problems, const int *ref_ids, const int *src_counts,
                  const int *src_ids, float *out_xyz, float *out_normal, float *out_color, long cap)
{
    return fuse_impl(1, n_views, cams, depths, normals, colors, n_problems, ref_ids, src_counts, src_ids, out_xyz,
                     out_normal, out_color, cap);
}

/* The mask-independent half of RunFusion for problem pi, as the product's
 * GPU pass computes it: per reference pixel its world point, and per
 * (pixel, source) the source pixel index of a consistent pair (-1
 * otherwise) and its exp(-error). */
int or_fuse_pairs(int n_views, const OrCamera *cams, const float *const *depths, const float *const *normals,
                  int ref, int ns, const int *srcs, int *pair_src, float *pair_w, float *points)
{
    (void)n_views;
    const OrCamera *ci = &cams[ref];
    const int cols = ci->width, rows = ci->height;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) {
            const size_t ctr = (size_t)r * cols + c;
            const float ref_depth = depths[ref][ctr];
            const float *ref_n = normals[ref] + 3 * ctr;
            for (int j = 0; j < ns; ++j) {
                pair_src[ctr * ns + j] = -1;
                pair_w[ctr * ns + j] = 0.0f;
            }
            if (ref_depth <= 0.0) continue;
            float X[3];
            fu_world(ci, c, r, ref_depth, X);
            memcpy(points + 3 * ctr, X, sizeof(X));
            for (int j = 0; j < ns; ++j) {
                const int s = srcs[j];
                const OrCamera *cs = &cams[s];
                float pt[2], proj_depth;
                fu_project(X, cs, pt, &proj_depth);
                const int sr = trunc_int(pt[1] + 0.5f), sc = trunc_int(pt[0] + 0.5f);
                if (!(sc >= 0 && sc < cs->width && sr >= 0 && sr < cs->height)) continue;
                const size_t sctr = (size_t)sr * cs->width + sc;
                const float src_depth = depths[s][sctr];
                const float *src_n = normals[s] + 3 * sctr;
                if (src_depth <= 0.0) continue;
                float Y[3], tp[2];
                fu_world(cs, sc, sr, src_depth, Y);
                fu_project(Y, ci, tp, &proj_depth);
                const float dx = (float)c - tp[0], dy = (float)r - tp[1];
                const float reproj = (float)sqrt((double)dx * dx + (double)dy * dy);
                const float rel = fabsf(proj_depth - ref_depth) / ref_depth;
                const float ang = fu_angle(ref_n, src_n);
                if (reproj < 2.0f && rel < 0.01f && ang < 0.174533f) {
                    pair_src[ctr * ns + j] = (int)sctr;
                    pair_w[ctr * ns + j] = expf(-(reproj + 200 * rel + ang * 10));
                }
            }
        }
    return 0;
}

/* ------------------------------------------------------------------ */
/* NCC error bound: what an FP32 evaluation of ComputeBilateralNCC may  */
/* differ by, tap coordinates being rounded differently                 */
/* ------------------------------------------------------------------ */

/* Value with a first-order bound on the rounding error that an FP32
 * evaluation of the same expression accumulates: each add or multiply may
 * round by one unit in the last place (2^-23 relative covers it), each
 * divide by two (fast-math division), and errors of the operands propagate.
 * The value itself is computed in double precision. */
typedef struct {
    double v, e;
} EV;

#define EV_EPS (1.0 / 8388608.0) /* 2^-23 */
static EV ev(double v) { EV r = {v, 0.0}; return r; }
static EV ev_add(EV a, EV b) { EV r = {a.v + b.v, 0}; r.e = a.e + b.e + EV_EPS * fabs(r.v); return r; }
static EV ev_sub(EV a, EV b) { EV r = {a.v - b.v, 0}; r.e = a.e + b.e + EV_EPS * fabs(r.v); return r; }
static EV ev_mul(EV a, EV b)
{
    EV r = {a.v * b.v, 0};
    r.e = fabs(a.v) * b.e + fabs(b.v) * a.e + a.e * b.e + EV_EPS * fabs(r.v);
    return r;
}
static EV ev_div(EV a, EV b)
{
    EV r = {a.v / b.v, 0};
    const double den = fabs(b.v) - b.e;
    r.e = den > 0 ? (a.e + fabs(r.v) * b.e) / den + 2.0 * EV_EPS * fabs(r.v) : INFINITY;
    return r;
}
static EV ev_neg(EV a) { EV r = {-a.v, a.e}; return r; }

/* ComputeHomography (HPM.cu:227-287), the same steps, with error bounds. */
static void homography_e(const OrCamera *ref, const OrCamera *src, F4 hf, EV *H)
{
    EV rR[9], sR[9], rt[3], st[3], rK[9], sK[9];
    for (int i = 0; i < 9; ++i) rR[i] = ev(ref->R[i]), sR[i] = ev(src->R[i]), rK[i] = ev(ref->K[i]), sK[i] = ev(src->K[i]);
    for (int i = 0; i < 3; ++i) rt[i] = ev(ref->t[i]), st[i] = ev(src->t[i]);
    const EV h[4] = {ev(hf.x), ev(hf.y), ev(hf.z), ev(hf.w)};
    EV rC[3], sC[3], Rr[9], Cr[3], tr[3], tmp[9];
    for (int i = 0; i < 3; ++i) {
        rC[i] = ev_neg(ev_add(ev_add(ev_mul(rR[i], rt[0]), ev_mul(rR[3 + i], rt[1])), ev_mul(rR[6 + i], rt[2])));
        sC[i] = ev_neg(ev_add(ev_add(ev_mul(sR[i], st[0]), ev_mul(sR[3 + i], st[1])), ev_mul(sR[6 + i], st[2])));
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Rr[3 * i + j] = ev_add(ev_add(ev_mul(sR[3 * i], rR[j]), ev_mul(sR[3 * i + 1], rR[3 + j])),
                                   ev_mul(sR[3 * i + 2], rR[6 + j]));
    for (int i = 0; i < 3; ++i) Cr[i] = ev_sub(rC[i], sC[i]);
    for (int i = 0; i < 3; ++i)
        tr[i] = ev_add(ev_add(ev_mul(sR[3 * i], Cr[0]), ev_mul(sR[3 * i + 1], Cr[1])), ev_mul(sR[3 * i + 2], Cr[2]));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) H[3 * i + j] = ev_sub(Rr[3 * i + j], ev_div(ev_mul(tr[i], h[j]), h[3]));
    for (int i = 0; i < 3; ++i) {
        tmp[3 * i + 0] = ev_div(H[3 * i + 0], rK[0]);
        tmp[3 * i + 1] = ev_div(H[3 * i + 1], rK[4]);
        tmp[3 * i + 2] = ev_add(ev_sub(ev_div(ev_mul(ev_neg(H[3 * i + 0]), rK[2]), rK[0]),
                                       ev_div(ev_mul(H[3 * i + 1], rK[5]), rK[4])),
                                H[3 * i + 2]);
    }
    H[0] = ev_add(ev_mul(sK[0], tmp[0]), ev_mul(sK[2], tmp[6]));
    H[1] = ev_add(ev_mul(sK[0], tmp[1]), ev_mul(sK[2], tmp[7]));
    H[2] = ev_add(ev_mul(sK[0], tmp[2]), ev_mul(sK[2], tmp[8]));
    H[3] = ev_add(ev_mul(sK[4], tmp[3]), ev_mul(sK[5], tmp[6]));
    H[4] = ev_add(ev_mul(sK[4], tmp[4]), ev_mul(sK[5], tmp[7]));
    H[5] = ev_add(ev_mul(sK[4], tmp[5]), ev_mul(sK[5], tmp[8]));
    H[6] = ev_mul(sK[8], tmp[6]);
    H[7] = ev_mul(sK[8], tmp[7]);
    H[8] = ev_mul(sK[8], tmp[8]);
}

/* ComputeCorrespondingPoint (HPM.cu:289-296) with error bounds. */
static void warp_e(const EV *H, int px, int py, EV *u, EV *v)
{
    const EV x = ev(px), y = ev(py);
    const EV a = ev_add(ev_add(ev_mul(H[0], x), ev_mul(H[1], y)), H[2]);
    const EV b = ev_add(ev_add(ev_mul(H[3], x), ev_mul(H[4], y)), H[5]);
    const EV z = ev_add(ev_add(ev_mul(H[6], x), ev_mul(H[7], y)), H[8]);
    *u = ev_div(a, z);
    *v = ev_div(b, z);
}

static double ulpf(float u)
{
    const float a = fabsf(u);
    return (double)(nextafterf(a, INFINITY) - a);
}

/* Texture sample with the fixed-point coordinate of each axis moved by
 * dq steps of 1/256 (the neighbouring rounding of the same coordinate). */
static float tex2d_q(const float *img, int w, int h, float u, float v, int dqa, int dqb)
{
    int ia[2], A[2];
    const float uv[2] = {u, v};
    const int n[2] = {w, h}, dq[2] = {dqa, dqb};
    int i0[2], i1[2];
    for (int ax = 0; ax < 2; ++ax) {
        double xb = (double)uv[ax] - 0.5;
        if (xb != xb) xb = 0.0;
        if (xb < -2.0) xb = -2.0;
        if (xb > (double)n[ax] + 1.0) xb = (double)n[ax] + 1.0;
        const double q = floor(xb * 256.0 + 0.5) + dq[ax];
        const double i = floor(q / 256.0);
        A[ax] = (int)(q - i * 256.0);
        ia[ax] = (int)i;
        i0[ax] = clampi(ia[ax], 0, n[ax] - 1);
        i1[ax] = clampi(ia[ax] + 1, 0, n[ax] - 1);
    }
    const int w11 = (A[0] * A[1] + 128) >> 8;
    const int w10 = A[0] - w11, w01 = A[1] - w11, w00 = 256 - A[0] - A[1] + w11;
    const double t00 = img[(size_t)i0[1] * w + i0[0]], t10 = img[(size_t)i0[1] * w + i1[0]];
    const double t01 = img[(size_t)i1[1] * w + i0[0]], t11 = img[(size_t)i1[1] * w + i1[0]];
    return (float)((w00 * t00 + w10 * t10 + w01 * t01 + w11 * t11) / 256.0);
}

/* Distance (in 1/256 steps) of a coordinate's scaled value from the rounding
 * boundary of the texture unit's 8-bit fraction, and the direction to the
 * other rounding: A = floor(256 (u - 0.5) + 1/2). */
static double step_margin(double u, int *dq)
{
    const double s = (u - 0.5) * 256.0 + 0.5;
    const double f = s - floor(s); /* boundary at f = 0 (and 1) */
    *dq = f < 0.5 ? -1 : 1;
    return f < 0.5 ? f : 1.0 - f;
}

/* One NCC with its bound.  Returns the oracle's cost; *bound is the largest
 * change that moving any subset of the taps whose coordinates lie within
 * the coordinate tolerance of a 1/256 rounding step across that step can
 * cause, to first order (sum of |d cost / d sample| x |sample change|), or 2
 * when the centre lies within the tolerance of the image border or a
 * variance cut lies within reach (either decision may then flip).
 * Coordinate tolerance of a tap: k_err times the propagated rounding-error
 * bound of its FP32 coordinate (homography_e, warp_e). */
static float ncc_with_bound(const Ctx *c, int v, int px, int py, F4 h, float k_err, float *bound, float *acc,
                            int *kind)
{
    *acc = 0.0f;
    *kind = 0; /* bit 0: a tap near a weight step; bit 1: a decision may flip */
    const OrCamera *ref = &c->cams[0], *src = &c->cams[v];
    const float *rimg = c->imgs[0], *simg = c->imgs[v];
    *bound = 0.0f;
    float H[9];
    EV He[9];
    homography(ref, src, h, H);
    homography_e(ref, src, h, He);
    float cx, cy;
    warp(H, px, py, &cx, &cy);
    {
        EV ue, ve;
        warp_e(He, px, py, &ue, &ve);
        const double cxd = ue.v, cyd = ve.v, tx = k_err * ue.e, ty = k_err * ve.e;
        if (fabs(cxd) <= tx || fabs(cxd - src->width) <= tx || fabs(cyd) <= ty || fabs(cyd - src->height) <= ty) {
            *bound = 2.0f;
            *kind = 2;
            return bilateral_ncc(c, v, px, py, h);
        }
    }
    const float cost = bilateral_ncc(c, v, px, py, h);
    if (cx >= (float)src->width || cx < 0.0f || cy >= (float)src->height || cy < 0.0f) return cost;
    double w[36], r[36], s[36], ds[36];
    const float rc = texel(rimg, ref->width, ref->height, px, py);
    int t = 0;
    for (int i = -5; i < 6; i += 2)
        for (int j = -5; j < 6; j += 2, ++t) {
            const int qx = px + i, qy = py + j;
            const float rp = texel(rimg, ref->width, ref->height, qx, qy);
            float sx, sy;
            warp(H, qx, qy, &sx, &sy);
            EV ue, ve;
            warp_e(He, qx, qy, &ue, &ve);
            const double sxd = ue.v, syd = ve.v;
            const float u = sx + 0.5f, vv = sy + 0.5f;
            const float sp = or_tex2d(simg, src->width, src->height, u, vv);
            /* the + 0.5 rounds once more */
            const double tx = k_err * (ue.e + EV_EPS * fabs(sxd + 0.5)), ty = k_err * (ve.e + EV_EPS * fabs(syd + 0.5));
            int dqa = 0, dqb = 0;
            const int near_a = step_margin(sxd + 0.5, &dqa) <= 256.0 * tx;
            const int near_b = step_margin(syd + 0.5, &dqb) <= 256.0 * ty;
            double d = 0.0;
            if (near_a) d = fmax(d, fabs((double)tex2d_q(simg, src->width, src->height, u, vv, dqa, 0) - sp));
            if (near_b) d = fmax(d, fabs((double)tex2d_q(simg, src->width, src->height, u, vv, 0, dqb) - sp));
            if (near_a && near_b)
                d = fmax(d, fabs((double)tex2d_q(simg, src->width, src->height, u, vv, dqa, dqb) - sp));
            /* the oracle's own rounding may sit on either side: include the
             * current rounding's neighbours in both directions */
            if (near_a) d = fmax(d, fabs((double)tex2d_q(simg, src->width, src->height, u, vv, -dqa, 0) - sp));
            if (near_b) d = fmax(d, fabs((double)tex2d_q(simg, src->width, src->height, u, vv, 0, -dqb) - sp));
            const double sdist = sqrt((double)(i * i + j * j));
            w[t] = exp(-sdist / 50.0 - fabs((double)rp - rc) / 18.0);
            r[t] = rp;
            s[t] = sp;
            ds[t] = d;
            if (d > 0.0) *kind |= 1;
        }
    double W = 0, mr = 0, mrr = 0, ms = 0, mss = 0, mrs = 0;
    for (t = 0; t < 36; ++t) {
        W += w[t];
        mr += w[t] * r[t];
        mrr += w[t] * r[t] * r[t];
        ms += w[t] * s[t];
        mss += w[t] * s[t] * s[t];
        mrs += w[t] * r[t] * s[t];
    }
    mr /= W, mrr /= W, ms /= W, mss /= W, mrs /= W;
    const double var_r = mrr - mr * mr, var_s = mss - ms * ms;
    if (fabs(var_r - 1e-5) <= 1e-8 || fabs(var_s - 1e-5) <= 1e-8 + 1e-3 * 1e-5) {
        *bound = 2.0f;
        *kind |= 2;
        return cost;
    }
    if (var_r < 1e-5 || var_s < 1e-5) {
        /* a sample change can still lift var_s over the cut */
        double dv = 0;
        for (t = 0; t < 36; ++t) dv += w[t] / W * (2 * fabs(s[t] - ms) + ds[t]) * ds[t];
        if (var_r >= 1e-5 && var_s + dv >= 1e-5) *bound = 2.0f, *kind |= 2;
        return cost;
    }
    const double covar = mrs - mr * ms, vv = sqrt(var_r * var_s);
    /* FP32 accumulation: each weighted sum is 36 terms of at most three
     * rounded factors, added as 6 rows of 6 and scaled by 1/W, so it lies
     * within g = 16 units of 2^-24 of its exact value (all terms positive);
     * the variances and the covariance then cancel, most of all in flat
     * windows.  Any two FP32 evaluations lie within twice this of each other. */
    const double u = 1.0 / 16777216.0, g = 16.0 * u;
    const double e_var_r = g * mrr + 2.0 * mr * g * mr + u * (mrr + mr * mr);
    const double e_var_s = g * mss + 2.0 * ms * g * ms + u * (mss + ms * ms);
    const double e_cov = g * mrs + mr * g * ms + ms * g * mr + u * (mrs + mr * ms);
    const double e_c = e_cov / vv + fabs(covar) / vv * (0.5 * (e_var_r / var_r + e_var_s / var_s) + u) + u;
    /* The bilateral weights: an FP32 evaluation's exp of an argument formed
     * with approximate division differs from the exact weight by a few
     * parts in 1e6 (CUDA documents __expf to 2 + floor(1.173 |x|) ulp, and
     * |x| < 15 here; the argument adds ~2 ulp of |x|).  First-order effect
     * of a relative error eps_w on every weight, signs taken worst case:
     * d cost / d w_t from the weighted means (d m / d w_t = (v_t - m) / W). */
    const double eps_w = 1e-5;
    double e_w = 0.0;
    for (t = 0; t < 36; ++t) {
        const double dmr = (r[t] - mr) / W, dms = (s[t] - ms) / W;
        const double dmrr = (r[t] * r[t] - mrr) / W, dmss = (s[t] * s[t] - mss) / W, dmrs = (r[t] * s[t] - mrs) / W;
        const double dvr = dmrr - 2.0 * mr * dmr, dvs = dmss - 2.0 * ms * dms, dcov = dmrs - mr * dms - ms * dmr;
        const double dc = -(dcov / vv - covar / (2.0 * vv) * (dvr / var_r + dvs / var_s));
        e_w += fabs(dc) * eps_w * w[t];
    }
    *acc = (float)(2.0 * (e_c + e_w));
    double b = 0, dvar_tot = 0;
    for (t = 0; t < 36; ++t) {
        if (ds[t] == 0.0) continue;
        const double dvar = w[t] / W * 2.0 * (s[t] - ms);
        const double dcov = w[t] / W * (r[t] - mr);
        const double dvv = var_r * dvar / (2.0 * vv);
        b += fabs((dcov * vv - covar * dvv) / (vv * vv)) * ds[t];
        dvar_tot += (fabs(dvar) + w[t] / W * ds[t]) * ds[t];
    }
    if (var_s - dvar_tot < 1e-5) b = 2.0, *kind |= 2; /* the variance cut itself is within reach */
    *bound = (float)b;
    return cost;
}

int or_ncc_bounds_px(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float k_err,
                     const int *pixels, int n_pixels, float *out_cost, float *out_bound, float *out_acc, int *out_kind)
{
    Ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n_img;
    c.imgs = imgs;
    c.cams = cams;
    c.W = cams[0].width;
    c.H = cams[0].height;
    const F4 *pl = (const F4 *)planes4;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int k = 0; k < n_pixels; ++k) {
        const int x = pixels[k] % c.W, y = pixels[k] / c.W;
        for (int v = 1; v < n_img; ++v) {
            const size_t o = (size_t)k * (n_img - 1) + v - 1;
            out_cost[o] = ncc_with_bound(&c, v, x, y, pl[pixels[k]], k_err, &out_bound[o], &out_acc[o], &out_kind[o]);
        }
    }
    return 0;
}

int or_ncc_bounds(int n_img, const float *const *imgs, const OrCamera *cams, const float *planes4, float k_err,
                  float *out_cost, float *out_bound, float *out_acc, int *out_kind)
{
    Ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n_img;
    c.imgs = imgs;
    c.cams = cams;
    c.W = cams[0].width;
    c.H = cams[0].height;
    const F4 *pl = (const F4 *)planes4;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int y = 0; y < c.H; ++y)
        for (int x = 0; x < c.W; ++x)
            for (int v = 1; v < n_img; ++v) {
                const size_t o = ((size_t)y * c.W + x) * (n_img - 1) + v - 1;
                out_cost[o] = ncc_with_bound(&c, v, x, y, pl[y * c.W + x], k_err, &out_bound[o], &out_acc[o],
                                             &out_kind[o]);
            }
    return 0;
}

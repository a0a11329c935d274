/*
 * JPEG decoding for the image reader: the bytes cv::imread returns for the
 * reference's images/%08d.jpg (OpenCV 4.13 over libjpeg-turbo) with
 * IMREAD_GRAYSCALE (HPM.cpp:490-492, main.cpp:168) and IMREAD_COLOR
 * (main.cpp:521-523).
 *
 * Decoded: Huffman-coded baseline (SOF0), extended sequential 8-bit (SOF1)
 * and progressive (SOF2) frames of 1 or 3 components, any integral sampling
 * factors, restart intervals, and the EXIF orientation tag (APP1), which
 * imread applies.  Rejected with HPM_ERR_IO: arithmetic coding, lossless and
 * hierarchical frames, 12-bit samples, 2 or 4 components (CMYK, YCCK),
 * truncated or corrupt entropy data.
 *
 * The steps that fix the output bytes follow ISO/IEC 10918-1 as libjpeg
 * implements it by default, and have to be alike for the bytes to be equal:
 *   - the integer inverse DCT of the Loeffler-Ligtenberg-Moschytz
 *     factorisation with 13-bit constants, 2 extra bits kept between the
 *     column and the row pass, and a wrap-around range limit (libjpeg's
 *     "islow", its default method);
 *   - "fancy" upsampling of subsampled components: a triangle filter, 3/4 of
 *     the nearer sample and 1/4 of the further one, with libjpeg's rounding
 *     biases and edge samples repeated; factors other than 2 replicate;
 *   - YCbCr -> RGB with 16-bit fixed-point coefficient tables; grayscale
 *     output of a YCbCr file is its Y component, unconverted;
 *   - the colour space of a 3-component file from its JFIF / Adobe markers or
 *     component ids.
 * Progressive files are decoded to their final coefficients before the
 * transform; when every coefficient is refined to its last bit (what
 * encoders write) libjpeg applies no block smoothing either.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "hpm_b200.h"
#include "hpm_jpeg.h"

namespace {

/* natural (row-major) index of the k-th coefficient in zig-zag order; 16
 * extra entries map overlong runs in corrupt data onto the last coefficient */
struct ZigZag {
    int pos[80];
    ZigZag()
    {
        int k = 0, x = 0, y = 0;
        for (int d = 0; d < 15; ++d) {
            /* anti-diagonal d, walked up-right on even d, down-left on odd d */
            for (int i = 0; i <= d; ++i) {
                x = (d & 1) ? d - i : i;
                y = d - x;
                if (x < 8 && y < 8) pos[k++] = y * 8 + x;
            }
        }
        for (; k < 80; ++k) pos[k] = 63;
    }
};
const ZigZag kZZ;

constexpr int kLook = 9; /* Huffman codes up to this length decode by table */

struct Huffman {
    bool present = false;
    uint8_t look_len[1 << kLook]; /* 0: the code is longer than kLook */
    uint8_t look_sym[1 << kLook];
    int32_t maxcode[18]; /* largest code of each length, -1 if none */
    int32_t valoff[17];  /* symbol index of a code of length l = valoff[l] + code */
    uint8_t sym[256];
    /* AC tables: a code and its value bits that fit in kLook bits together,
     * decoded in one lookup: value << 8 | run << 4 | total length; 0 if not */
    int32_t fast_ac[1 << kLook];

    bool build(const uint8_t counts[16], const uint8_t *syms, int nsyms)
    {
        memcpy(sym, syms, nsyms);
        memset(look_len, 0, sizeof(look_len));
        int code = 0, k = 0;
        for (int l = 1; l <= 16; ++l) {
            valoff[l] = k - code;
            for (int i = 0; i < counts[l - 1]; ++i, ++k, ++code) {
                if (code >= (1 << l)) return false; /* more codes than the length allows */
                if (l <= kLook) {
                    const int lo = code << (kLook - l), n = 1 << (kLook - l);
                    for (int j = 0; j < n; ++j) {
                        look_len[lo + j] = (uint8_t)l;
                        look_sym[lo + j] = syms[k];
                    }
                }
            }
            maxcode[l] = counts[l - 1] ? code - 1 : -1;
            code <<= 1;
        }
        maxcode[17] = 0x7fffffff;
        for (int i = 0; i < (1 << kLook); ++i) {
            fast_ac[i] = 0;
            const int l = look_len[i];
            if (!l) continue;
            const int rs = look_sym[i], r = rs >> 4, sz = rs & 15;
            if (sz == 0 || l + sz > kLook) continue;
            const int bits = (i >> (kLook - l - sz)) & ((1 << sz) - 1);
            const int v = bits < (1 << (sz - 1)) ? bits - (1 << sz) + 1 : bits;
            fast_ac[i] = (int32_t)((uint32_t)v << 8) | r << 4 | (l + sz);
        }
        present = true;
        return true;
    }
};

/* Entropy-coded data: stuffed zero bytes removed; at a marker (or the end
 * of the data) the reader stops and supplies zero bits.  As in libjpeg, a
 * decoder that consumes one of those zero bits has run out of data
 * (insufficient): the unit in progress is finished with zero bits and the
 * units after it, up to the next restart, are left as they are. */
struct BitReader {
    const uint8_t *d;
    size_t n, pos;
    uint64_t acc = 0;
    int cnt = 0;  /* bits in acc */
    int real = 0; /* of those, bits from the data (the leading ones) */
    bool at_marker = false, insufficient = false;

    BitReader(const uint8_t *data, size_t size, size_t start) : d(data), n(size), pos(start) {}

    void fill()
    {
        if (!at_marker && pos + 8 <= n) {
            /* eight bytes at once when none of them is 0xFF */
            uint64_t w;
            memcpy(&w, d + pos, 8);
            const uint64_t x = ~w;
            if (((x - 0x0101010101010101ull) & ~x & 0x8080808080808080ull) == 0) {
                w = __builtin_bswap64(w);
                const int k = (64 - cnt) >> 3;
                acc |= (k == 8 ? w : (w >> (64 - 8 * k))) << (64 - cnt - 8 * k);
                pos += k;
                cnt += 8 * k;
                real += 8 * k;
                return;
            }
        }
        while (cnt <= 56) {
            uint32_t b = 0;
            bool data = false;
            if (!at_marker && pos < n) {
                if (d[pos] != 0xFF) {
                    b = d[pos++];
                    data = true;
                } else {
                    size_t q = pos + 1;
                    while (q < n && d[q] == 0xFF) ++q; /* fill bytes */
                    if (q < n && d[q] == 0x00) {
                        b = 0xFF;
                        pos = q + 1;
                        data = true;
                    } else {
                        at_marker = true;
                    }
                }
            } else if (pos >= n) {
                at_marker = true;
            }
            acc |= (uint64_t)b << (56 - cnt);
            cnt += 8;
            if (data) real += 8;
        }
    }
    void consume(int k)
    {
        acc <<= k;
        cnt -= k;
        if (k > real) {
            insufficient = true;
            real = 0;
        } else {
            real -= k;
        }
    }
    int bits(int k)
    {
        if (k == 0) return 0;
        if (cnt < k) fill();
        const int v = (int)(acc >> (64 - k));
        consume(k);
        return v;
    }
    int bit() { return bits(1); }
    /* -1 on a code that no table entry has */
    int decode(const Huffman &h)
    {
        if (cnt < 16) fill();
        const int look = (int)(acc >> (64 - kLook));
        const int len = h.look_len[look];
        if (len) {
            consume(len);
            return h.look_sym[look];
        }
        for (int l = kLook + 1; l <= 16; ++l) {
            const int code = (int)(acc >> (64 - l));
            if (code <= h.maxcode[l]) {
                consume(l);
                const int i = h.valoff[l] + code;
                return (i >= 0 && i < 256) ? h.sym[i] : -1;
            }
        }
        return -1;
    }
    /* at a restart boundary: the padding bits go, reading resumes at pos */
    void discard_buffer()
    {
        acc = 0;
        cnt = 0;
        real = 0;
        at_marker = false;
        insufficient = false;
    }
};

inline int extend(int v, int s) { return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v; }

}  // namespace

namespace {

struct Component {
    int id = 0, h = 1, v = 1, tq = 0;
    int bw = 0, bh = 0; /* blocks held: the frame's MCUs times h (v) */
    int dw = 0, dh = 0; /* samples: ceil(W h / Hmax), ceil(H v / Vmax) */
    int dc_tbl = 0, ac_tbl = 0;
    int pred = 0;
    bool quant_latched = false;
    uint16_t quant[64]; /* natural order, latched at the component's first scan */
    std::vector<int16_t> coef; /* bw * bh blocks of 64, natural order */
    std::vector<uint8_t> plane; /* (8 bw) x (8 bh) samples after the inverse DCT */
};

struct Frame {
    int W = 0, H = 0, ncomp = 0;
    int hmax = 1, vmax = 1, mcux = 0, mcuy = 0;
    bool progressive = false, have_frame = false;
    bool jfif = false, adobe = false;
    int adobe_transform = -1;
    int restart_interval = 0;
    int orientation = 1;
    bool qt_present[4] = {false, false, false, false};
    uint16_t qt[4][64]; /* natural order */
    Huffman dc[4], ac[4];
    Component comp[3];
};

/* The islow inverse DCT.  Constants are round(x * 2^13) of
 *   0.298631336 = sqrt2 (-c1 + c3 + c5 - c7)   0.390180644 = sqrt2 (c3 - c5)
 *   0.541196100 = sqrt2 c6                     0.765366865 = sqrt2 (c2 - c6)
 *   0.899976223 = sqrt2 (c3 - c7)              1.175875602 = sqrt2 c3
 *   1.501321110 = sqrt2 (c1 + c3 - c5 - c7)    1.847759065 = sqrt2 (c2 + c6)
 *   1.961570560 = sqrt2 (c3 + c5)              2.053119869 = sqrt2 (c1 + c3 - c5 + c7)
 *   2.562915447 = sqrt2 (c1 + c3)              3.072711026 = sqrt2 (c1 + c3 + c5 - c7)
 * with ck = cos(k pi / 16). */
constexpr int kConstBits = 13, kPass1Bits = 2;
constexpr uint32_t F0_298 = 2446, F0_390 = 3196, F0_541 = 4433, F0_765 = 6270, F0_899 = 7373, F1_175 = 9633,
                   F1_501 = 12299, F1_847 = 15137, F1_961 = 16069, F2_053 = 16819, F2_562 = 20995, F3_072 = 25172;

/* One 1-D pass over the 8 lanes of each input row: in[k * 8 + lane] is the
 * k-th input of that lane's transform, out[k * 8 + lane] its k-th output
 * descaled by n bits.  32-bit arithmetic, modulo 2^32 (it does not wrap for
 * the coefficients encoders produce; libjpeg-turbo's SIMD transform, which
 * cv::imread runs, also works in 16- and 32-bit lanes). */
inline void idct_pass(const int32_t *in, int32_t *out, int n)
{
    const uint32_t half = 1u << (n - 1);
    for (int x = 0; x < 8; ++x) {
        const uint32_t s0 = (uint32_t)in[x], s1 = (uint32_t)in[8 + x], s2 = (uint32_t)in[16 + x],
                       s3 = (uint32_t)in[24 + x], s4 = (uint32_t)in[32 + x], s5 = (uint32_t)in[40 + x],
                       s6 = (uint32_t)in[48 + x], s7 = (uint32_t)in[56 + x];
        /* even part */
        const uint32_t z1 = (s2 + s6) * F0_541;
        const uint32_t e2 = z1 - s6 * F1_847, e3 = z1 + s2 * F0_765;
        const uint32_t e0 = (s0 + s4) << kConstBits, e1 = (s0 - s4) << kConstBits;
        const uint32_t t10 = e0 + e3, t13 = e0 - e3, t11 = e1 + e2, t12 = e1 - e2;
        /* odd part */
        const uint32_t y5 = (s7 + s3 + s5 + s1) * F1_175;
        const uint32_t y1 = (s7 + s1) * (0u - F0_899), y2 = (s5 + s3) * (0u - F2_562);
        const uint32_t y3 = (s7 + s3) * (0u - F1_961) + y5, y4 = (s5 + s1) * (0u - F0_390) + y5;
        const uint32_t a0 = s7 * F0_298 + y1 + y3, a1 = s5 * F2_053 + y2 + y4;
        const uint32_t a2 = s3 * F3_072 + y2 + y3, a3 = s1 * F1_501 + y1 + y4;
        out[x] = (int32_t)(t10 + a3 + half) >> n;
        out[56 + x] = (int32_t)(t10 - a3 + half) >> n;
        out[8 + x] = (int32_t)(t11 + a2 + half) >> n;
        out[48 + x] = (int32_t)(t11 - a2 + half) >> n;
        out[16 + x] = (int32_t)(t12 + a1 + half) >> n;
        out[40 + x] = (int32_t)(t12 - a1 + half) >> n;
        out[24 + x] = (int32_t)(t13 + a0 + half) >> n;
        out[32 + x] = (int32_t)(t13 - a0 + half) >> n;
    }
}

/* the range limit of the transform's output: v + 128 clamped to [0, 255]
 * for v in [-512, 511], wrapping outside (index v & 1023) */
struct RangeLimit {
    uint8_t t[1024];
    RangeLimit()
    {
        for (int x = 0; x < 1024; ++x) t[x] = x < 128 ? (uint8_t)(x + 128) : x < 512 ? 255 : x < 896 ? 0 : (uint8_t)(x - 896);
    }
};
const RangeLimit kRange;

/* dequantise, columns, rows: the column pass keeps 2 extra bits
 * (descale by 13 - 2), the row pass removes them and the factor 8 of the
 * 2-D transform (descale by 13 + 2 + 3) */
__attribute__((target_clones("avx2", "default"))) void idct_block(const int16_t *c, const uint16_t *q, uint8_t *out,
                                                                  int stride)
{
    int32_t deq[64], ws[64], wt[64], res[64];
    for (int i = 0; i < 64; ++i) deq[i] = (int32_t)c[i] * (int32_t)q[i];
    idct_pass(deq, ws, kConstBits - kPass1Bits);
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) wt[x * 8 + y] = ws[y * 8 + x];
    idct_pass(wt, res, kConstBits + kPass1Bits + 3);
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) out[(size_t)y * stride + x] = kRange.t[res[x * 8 + y] & 1023];
}

}  // namespace

namespace {

inline int be16(const uint8_t *p) { return p[0] << 8 | p[1]; }

/* EXIF orientation from an APP1 "Exif\0\0" payload: the TIFF header, IFD0,
 * tag 0x0112 (SHORT).  Values outside 1..8 leave the image as decoded. */
int exif_orientation(const uint8_t *p, size_t n)
{
    if (n < 14 || memcmp(p, "Exif\0\0", 6) != 0) return 1;
    const uint8_t *t = p + 6;
    const size_t tn = n - 6;
    bool le;
    if (t[0] == 'I' && t[1] == 'I')
        le = true;
    else if (t[0] == 'M' && t[1] == 'M')
        le = false;
    else
        return 1;
    auto u16 = [&](size_t o) -> uint32_t { return le ? (t[o] | t[o + 1] << 8) : (t[o] << 8 | t[o + 1]); };
    auto u32 = [&](size_t o) -> uint32_t {
        return le ? (uint32_t)(t[o] | t[o + 1] << 8 | t[o + 2] << 16 | (uint32_t)t[o + 3] << 24)
                  : ((uint32_t)t[o] << 24 | t[o + 1] << 16 | t[o + 2] << 8 | t[o + 3]);
    };
    if (u16(2) != 42) return 1;
    const size_t ifd = u32(4);
    if (ifd + 2 > tn) return 1;
    const uint32_t count = u16(ifd);
    for (uint32_t i = 0; i < count; ++i) {
        const size_t e = ifd + 2 + 12 * (size_t)i;
        if (e + 12 > tn) break;
        if (u16(e) == 0x0112 && u16(e + 2) == 3) {
            const int v = (int)u16(e + 8);
            return (v >= 1 && v <= 8) ? v : 1;
        }
    }
    return 1;
}

/* Marker segments up to and including the next SOS; returns the offset of
 * the SOS length field (pos then at the entropy-coded data), 0 at EOI, -2 at
 * the end of the data without EOI, -1 on an error. */
long parse_to_scan(const uint8_t *d, size_t n, size_t &pos, Frame &f)
{
    while (true) {
        /* the next marker: 0xFF, any fill bytes, a code other than 0 */
        while (pos < n && d[pos] != 0xFF) ++pos;
        while (pos < n && d[pos] == 0xFF) ++pos;
        if (pos >= n) return -2;
        const int m = d[pos++];
        /* 0x00: a stuffed byte of entropy data left behind a scan; SOI, RSTn, TEM */
        if (m == 0x00 || m == 0xD8 || (m >= 0xD0 && m <= 0xD7) || m == 0x01) continue;
        if (m == 0xD9) return 0;                                            /* EOI */
        if (pos + 2 > n) return -1;
        const size_t len = (size_t)be16(d + pos);
        if (len < 2 || pos + len > n) return -1;
        const uint8_t *s = d + pos + 2;
        const size_t sl = len - 2;
        const size_t seg = pos;
        pos += len;
        switch (m) {
        case 0xDB: { /* DQT */
            size_t i = 0;
            while (i < sl) {
                const int pq = s[i] >> 4, tq = s[i] & 15;
                ++i;
                if (tq > 3 || pq > 1 || i + 64 * (pq + 1) > sl) return -1;
                for (int k = 0; k < 64; ++k) {
                    f.qt[tq][kZZ.pos[k]] = pq ? (uint16_t)be16(s + i + 2 * k) : s[i + k];
                }
                i += 64 * (pq + 1);
                f.qt_present[tq] = true;
            }
            break;
        }
        case 0xC4: { /* DHT */
            size_t i = 0;
            while (i < sl) {
                if (i + 17 > sl) return -1;
                const int tc = s[i] >> 4, th = s[i] & 15;
                if (tc > 1 || th > 3) return -1;
                int total = 0;
                for (int l = 0; l < 16; ++l) total += s[i + 1 + l];
                if (total > 256 || i + 17 + total > sl) return -1;
                Huffman &h = tc ? f.ac[th] : f.dc[th];
                if (!h.build(s + i + 1, s + i + 17, total)) return -1;
                i += 17 + total;
            }
            break;
        }
        case 0xC0:
        case 0xC1:
        case 0xC2: { /* SOF0 baseline, SOF1 extended sequential, SOF2 progressive */
            if (f.have_frame || sl < 6) return -1;
            if (s[0] != 8) return -1; /* 12-bit samples */
            f.H = be16(s + 1);
            f.W = be16(s + 3);
            f.ncomp = s[5];
            if (f.W < 1 || f.H < 1 || (f.ncomp != 1 && f.ncomp != 3) || sl < 6 + 3 * (size_t)f.ncomp) return -1;
            f.progressive = m == 0xC2;
            for (int c = 0; c < f.ncomp; ++c) {
                Component &k = f.comp[c];
                k.id = s[6 + 3 * c];
                k.h = s[7 + 3 * c] >> 4;
                k.v = s[7 + 3 * c] & 15;
                k.tq = s[8 + 3 * c];
                if (k.h < 1 || k.h > 4 || k.v < 1 || k.v > 4 || k.tq > 3) return -1;
                f.hmax = std::max(f.hmax, k.h);
                f.vmax = std::max(f.vmax, k.v);
            }
            f.have_frame = true;
            break;
        }
        case 0xDD: /* DRI */
            if (sl < 2) return -1;
            f.restart_interval = be16(s);
            break;
        case 0xE0: /* APP0: JFIF */
            if (sl >= 5 && memcmp(s, "JFIF\0", 5) == 0) f.jfif = true;
            break;
        case 0xE1: /* APP1: EXIF */
            if (f.orientation == 1 && sl >= 6 && memcmp(s, "Exif\0\0", 6) == 0) f.orientation = exif_orientation(s, sl);
            break;
        case 0xEE: /* APP14: Adobe */
            if (sl >= 12 && memcmp(s, "Adobe", 5) == 0) {
                f.adobe = true;
                f.adobe_transform = s[11];
            }
            break;
        case 0xDA: /* SOS */
            if (!f.have_frame) return -1;
            return (long)seg; /* pos is at the entropy-coded data */
        default:
            /* arithmetic (SOF9-SOF15 but DHT's neighbours), lossless,
             * hierarchical frames; other segments are skipped */
            if ((m >= 0xC3 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC)) return -1;
            break;
        }
    }
}

}  // namespace

namespace {

struct Scan {
    int ns = 0;
    int ci[3] = {0, 0, 0};
    int ss = 0, se = 63, ah = 0, al = 0;
};

bool setup_frame(Frame &f)
{
    if ((int64_t)f.W * f.H > ((int64_t)1 << 29)) return false; /* 512 Mpixel */
    f.mcux = (f.W + 8 * f.hmax - 1) / (8 * f.hmax);
    f.mcuy = (f.H + 8 * f.vmax - 1) / (8 * f.vmax);
    for (int c = 0; c < f.ncomp; ++c) {
        Component &k = f.comp[c];
        k.bw = f.mcux * k.h;
        k.bh = f.mcuy * k.v;
        k.dw = (int)(((int64_t)f.W * k.h + f.hmax - 1) / f.hmax);
        k.dh = (int)(((int64_t)f.H * k.v + f.vmax - 1) / f.vmax);
        k.coef.assign((size_t)k.bw * k.bh * 64, 0);
    }
    return true;
}

bool parse_scan_header(const uint8_t *d, size_t seg, Frame &f, Scan &sc)
{
    const size_t len = (size_t)be16(d + seg);
    const uint8_t *s = d + seg + 2;
    if (len < 3) return false;
    sc.ns = s[0];
    if (sc.ns < 1 || sc.ns > f.ncomp || len != 6 + 2 * (size_t)sc.ns) return false;
    for (int i = 0; i < sc.ns; ++i) {
        const int id = s[1 + 2 * i];
        int c = -1;
        for (int j = 0; j < f.ncomp; ++j)
            if (f.comp[j].id == id) c = j;
        if (c < 0) return false;
        for (int j = 0; j < i; ++j)
            if (sc.ci[j] == c) return false;
        sc.ci[i] = c;
        f.comp[c].dc_tbl = s[2 + 2 * i] >> 4;
        f.comp[c].ac_tbl = s[2 + 2 * i] & 15;
        if (f.comp[c].dc_tbl > 3 || f.comp[c].ac_tbl > 3) return false;
    }
    const uint8_t *t = s + 1 + 2 * sc.ns;
    sc.ss = t[0];
    sc.se = t[1];
    sc.ah = t[2] >> 4;
    sc.al = t[2] & 15;
    if (f.progressive) {
        if (sc.ss == 0 ? sc.se != 0 : (sc.se < sc.ss || sc.se > 63 || sc.ns != 1)) return false;
        if (sc.al > 13 || sc.ah > 13) return false;
    } else {
        sc.ss = 0, sc.se = 63, sc.ah = 0, sc.al = 0; /* fixed in sequential mode */
    }
    int blocks = 0;
    for (int i = 0; i < sc.ns; ++i) blocks += f.comp[sc.ci[i]].h * f.comp[sc.ci[i]].v;
    if (sc.ns > 1 && blocks > 10) return false; /* the MCU limit of ISO/IEC 10918-1 */
    return true;
}

bool block_sequential(BitReader &br, const Huffman &dc, const Huffman &ac, int &pred, int16_t *blk)
{
    int s = br.decode(dc);
    if (s < 0 || s > 16) return false;
    pred += s ? extend(br.bits(s), s) : 0;
    blk[0] = (int16_t)pred;
    for (int k = 1; k < 64; ++k) {
        if (br.cnt < 16) br.fill();
        const int32_t fa = ac.fast_ac[br.acc >> (64 - kLook)];
        if (fa) { /* code and value bits in one lookup */
            k += (fa >> 4) & 15;
            br.consume(fa & 15);
            blk[kZZ.pos[k]] = (int16_t)(fa >> 8);
            continue;
        }
        const int rs = br.decode(ac);
        if (rs < 0) return false;
        const int r = rs >> 4;
        s = rs & 15;
        if (s) {
            k += r;
            blk[kZZ.pos[k]] = (int16_t)extend(br.bits(s), s);
        } else {
            if (r != 15) break;
            k += 15;
        }
    }
    return true;
}

bool block_dc_first(BitReader &br, const Huffman &dc, int &pred, int al, int16_t *blk)
{
    const int s = br.decode(dc);
    if (s < 0 || s > 16) return false;
    pred += s ? extend(br.bits(s), s) : 0;
    blk[0] = (int16_t)((uint32_t)pred << al);
    return true;
}

bool block_dc_refine(BitReader &br, int al, int16_t *blk)
{
    if (br.bit()) blk[0] = (int16_t)(blk[0] | (1 << al));
    return true;
}

bool block_ac_first(BitReader &br, const Huffman &ac, const Scan &sc, int &eobrun, int16_t *blk)
{
    if (eobrun > 0) {
        --eobrun;
        return true;
    }
    for (int k = sc.ss; k <= sc.se; ++k) {
        const int rs = br.decode(ac);
        if (rs < 0) return false;
        const int r = rs >> 4, s = rs & 15;
        if (s) {
            k += r;
            blk[kZZ.pos[k]] = (int16_t)((uint32_t)extend(br.bits(s), s) << sc.al);
        } else if (r == 15) {
            k += 15;
        } else {
            eobrun = (1 << r) - 1;
            if (r) eobrun += br.bits(r);
            break;
        }
    }
    return true;
}

/* Successive-approximation refinement of AC coefficients (ISO/IEC 10918-1
 * G.1.2.3): newly nonzero coefficients get +-1 at bit al, coefficients
 * already nonzero get a correction bit each time the run passes them. */
bool block_ac_refine(BitReader &br, const Huffman &ac, const Scan &sc, int &eobrun, int16_t *blk)
{
    const int p1 = 1 << sc.al, m1 = -p1;
    auto correct = [&](int16_t &c) {
        if (br.bit() && (c & p1) == 0) c = (int16_t)(c >= 0 ? c + p1 : c + m1);
    };
    int k = sc.ss;
    if (eobrun == 0) {
        for (; k <= sc.se; ++k) {
            const int rs = br.decode(ac);
            if (rs < 0) return false;
            int r = rs >> 4, s = rs & 15;
            if (s) { /* a size other than 1 is read as 1, as libjpeg does */
                s = br.bit() ? p1 : m1;
            } else if (r != 15) {
                eobrun = 1 << r;
                if (r) eobrun += br.bits(r);
                break; /* the rest of the band goes through the end-of-band pass */
            }
            /* skip r zero coefficients (correcting nonzero ones on the way),
             * then place s on the next zero one */
            while (k <= sc.se) {
                int16_t &c = blk[kZZ.pos[k]];
                if (c != 0) {
                    correct(c);
                } else {
                    if (r == 0) break;
                    --r;
                }
                ++k;
            }
            if (s) blk[kZZ.pos[k]] = (int16_t)s;
        }
    }
    if (eobrun > 0) {
        for (; k <= sc.se; ++k) {
            int16_t &c = blk[kZZ.pos[k]];
            if (c != 0) correct(c);
        }
        --eobrun;
    }
    return true;
}

/* One scan; pos enters at the entropy-coded data and leaves after it. */
bool decode_scan(const uint8_t *d, size_t n, size_t &pos, Frame &f, const Scan &sc)
{
    for (int i = 0; i < sc.ns; ++i) {
        Component &c = f.comp[sc.ci[i]];
        c.pred = 0;
        if (!c.quant_latched) {
            if (!f.qt_present[c.tq]) return false;
            memcpy(c.quant, f.qt[c.tq], sizeof(c.quant));
            c.quant_latched = true;
        }
        const bool need_dc = sc.ss == 0 && sc.ah == 0, need_ac = sc.se > 0;
        if (need_dc && !f.dc[c.dc_tbl].present) return false;
        if (need_ac && !f.ac[c.ac_tbl].present) return false;
    }
    BitReader br(d, n, pos);
    int eobrun = 0;
    const Component &c0 = f.comp[sc.ci[0]];
    const int ux = sc.ns == 1 ? (c0.dw + 7) / 8 : f.mcux;
    const int uy = sc.ns == 1 ? (c0.dh + 7) / 8 : f.mcuy;
    const int64_t total = (int64_t)ux * uy;
    for (int64_t u = 0; u < total; ++u) {
        if (f.restart_interval && u > 0 && u % f.restart_interval == 0) {
            const bool out_of_data = br.insufficient;
            br.discard_buffer();
            size_t p = br.pos;
            while (p + 1 < n && !(d[p] == 0xFF && d[p + 1] != 0x00 && d[p + 1] != 0xFF)) ++p;
            if (p + 1 < n && d[p + 1] >= 0xD0 && d[p + 1] <= 0xD7)
                p += 2;
            else /* no restart marker (another marker, or the end): libjpeg keeps its out-of-data state */
                br.insufficient = out_of_data;
            br.pos = p;
            eobrun = 0;
            for (int i = 0; i < sc.ns; ++i) f.comp[sc.ci[i]].pred = 0;
        }
        if (br.insufficient) continue; /* out of data: left as it is */
        const int my = (int)(u / ux), mx = (int)(u % ux);
        for (int i = 0; i < sc.ns; ++i) {
            Component &c = f.comp[sc.ci[i]];
            const int nbx = sc.ns == 1 ? 1 : c.h, nby = sc.ns == 1 ? 1 : c.v;
            for (int by = 0; by < nby; ++by)
                for (int bx = 0; bx < nbx; ++bx) {
                    const int gx = mx * nbx + bx, gy = my * nby + by;
                    int16_t *blk = &c.coef[((size_t)gy * c.bw + gx) * 64];
                    bool ok;
                    if (!f.progressive)
                        ok = block_sequential(br, f.dc[c.dc_tbl], f.ac[c.ac_tbl], c.pred, blk);
                    else if (sc.ss == 0 && sc.ah == 0)
                        ok = block_dc_first(br, f.dc[c.dc_tbl], c.pred, sc.al, blk);
                    else if (sc.ss == 0)
                        ok = block_dc_refine(br, sc.al, blk);
                    else if (sc.ah == 0)
                        ok = block_ac_first(br, f.ac[c.ac_tbl], sc, eobrun, blk);
                    else
                        ok = block_ac_refine(br, f.ac[c.ac_tbl], sc, eobrun, blk);
                    if (!ok) return false;
                }
        }
    }
    pos = br.pos;
    return true;
}

}  // namespace

namespace {

void transform_component(Component &c)
{
    const int ps = c.bw * 8;
    const int nbx = (c.dw + 7) / 8, nby = (c.dh + 7) / 8;
    c.plane.assign((size_t)ps * c.bh * 8, 0);
    for (int by = 0; by < nby; ++by)
        for (int bx = 0; bx < nbx; ++bx)
            idct_block(&c.coef[((size_t)by * c.bw + bx) * 64], c.quant, &c.plane[(size_t)by * 8 * ps + bx * 8], ps);
}

/* Horizontal triangle filter of one row: n input samples to 2n outputs,
 * the edge samples repeated (libjpeg's h2v1 filter) */
__attribute__((target_clones("avx2", "default"))) void h2_row(const uint8_t *in, int n, uint8_t *out)
{
    out[0] = in[0];
    for (int k = 0; k + 1 < n; ++k) {
        out[2 * k + 1] = (uint8_t)((3 * in[k] + in[k + 1] + 2) >> 2);
        out[2 * k + 2] = (uint8_t)((3 * in[k + 1] + in[k] + 1) >> 2);
    }
    out[2 * n - 1] = in[n - 1];
}

/* The 2-D filter of libjpeg's h2v2: column sums 3 near + far of the two
 * input rows, then 3/4 - 1/4 across, over 16 with biases 8 and 7 */
__attribute__((target_clones("avx2", "default"))) void h2v2_row(const uint8_t *near, const uint8_t *far, int n,
                                                                uint8_t *out, int *cs)
{
    for (int k = 0; k < n; ++k) cs[k] = 3 * near[k] + far[k];
    out[0] = (uint8_t)((4 * cs[0] + 8) >> 4);
    for (int k = 0; k + 1 < n; ++k) {
        out[2 * k + 1] = (uint8_t)((3 * cs[k] + cs[k + 1] + 7) >> 4);
        out[2 * k + 2] = (uint8_t)((3 * cs[k + 1] + cs[k] + 8) >> 4);
    }
    out[2 * n - 1] = (uint8_t)((4 * cs[n - 1] + 7) >> 4);
}

/* A component's dw x dh samples to the W x H image grid.  Factors of 2 use
 * libjpeg's triangle filters (horizontal ones only on components more than 2
 * samples wide); other integral factors replicate samples. */
bool upsample(const Component &c, const Frame &f, std::vector<uint8_t> &out)
{
    if (f.hmax % c.h || f.vmax % c.v) return false;
    const int hr = f.hmax / c.h, vr = f.vmax / c.v;
    const int W = f.W, H = f.H, ps = c.bw * 8, dw = c.dw, dh = c.dh;
    const uint8_t *in = c.plane.data();
    out.resize((size_t)W * H);
    std::vector<uint8_t> wide(2 * (size_t)dw);
    std::vector<int> cs(dw);
    for (int y = 0; y < H; ++y) {
        uint8_t *o = &out[(size_t)y * W];
        const int r = y / vr;
        const uint8_t *row = in + (size_t)r * ps;
        const bool lower = y & 1;
        if (hr == 1 && vr == 1) {
            memcpy(o, row, W);
        } else if (hr == 2 && vr == 1 && dw > 2) {
            h2_row(row, dw, wide.data());
            memcpy(o, wide.data(), W);
        } else if (hr == 1 && vr == 2) {
            const uint8_t *nb = in + (size_t)(lower ? std::min(r + 1, dh - 1) : std::max(r - 1, 0)) * ps;
            const int bias = lower ? 2 : 1;
            for (int x = 0; x < W; ++x) o[x] = (uint8_t)((3 * row[x] + nb[x] + bias) >> 2);
        } else if (hr == 2 && vr == 2 && dw > 2) {
            const uint8_t *nb = in + (size_t)(lower ? std::min(r + 1, dh - 1) : std::max(r - 1, 0)) * ps;
            h2v2_row(row, nb, dw, wide.data(), cs.data());
            memcpy(o, wide.data(), W);
        } else {
            for (int x = 0; x < W; ++x) o[x] = row[x / hr];
        }
    }
    return true;
}

/* 16-bit fixed point of a conversion coefficient, rounded */
constexpr int fix16(double x) { return (int)(x * 65536.0 + 0.5); }

inline uint8_t clamp8(int v) { return (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v); }

/* JFIF YCbCr -> B, G, R: R = Y + 1.402 Cr', G = Y - 0.34414 Cb' - 0.71414 Cr',
 * B = Y + 1.772 Cb' (Cb' = Cb - 128, ...) in 16-bit fixed point, each
 * chroma term rounded as libjpeg's conversion tables round it */
__attribute__((target_clones("avx2", "default"))) void ycc_to_bgr(const uint8_t *Y, const uint8_t *Cb, const uint8_t *Cr,
                                                                  size_t n, uint8_t *out)
{
    constexpr int kR = fix16(1.40200), kB = fix16(1.77200), kGr = fix16(0.71414), kGb = fix16(0.34414);
    for (size_t p = 0; p < n; ++p) {
        const int y = Y[p], cb = Cb[p] - 128, cr = Cr[p] - 128;
        const int r = y + ((kR * cr + (1 << 15)) >> 16);
        const int g = y + ((-kGb * cb + (1 << 15) - kGr * cr) >> 16);
        const int b = y + ((kB * cb + (1 << 15)) >> 16);
        out[3 * p] = clamp8(b);
        out[3 * p + 1] = clamp8(g);
        out[3 * p + 2] = clamp8(r);
    }
}

/* EXIF orientation as imread applies it: 2 mirror, 3 rotate 180, 4 flip,
 * 5 transpose, 6 rotate 90 clockwise, 7 transverse, 8 rotate 90
 * counter-clockwise. */
void orient(std::vector<uint8_t> &px, int &w, int &h, int ch, int o)
{
    if (o <= 1 || o > 8) return;
    const bool tr = o >= 5;
    const bool fx = o == 2 || o == 3 || o == 6 || o == 7, fy = o == 3 || o == 4 || o == 7 || o == 8;
    const int ow = tr ? h : w, oh = tr ? w : h;
    std::vector<uint8_t> out((size_t)ow * oh * ch);
    for (int y = 0; y < oh; ++y)
        for (int x = 0; x < ow; ++x) {
            const int tx = fx ? ow - 1 - x : x, ty = fy ? oh - 1 - y : y; /* in the transposed image */
            const int sx = tr ? ty : tx, sy = tr ? tx : ty;
            memcpy(&out[((size_t)y * ow + x) * ch], &px[((size_t)sy * w + sx) * ch], ch);
        }
    px.swap(out);
    w = ow;
    h = oh;
}

}  // namespace

int hpm_decode_jpeg(const uint8_t *d, size_t n, std::vector<uint8_t> &px, int *w_out, int *h_out, int out_ch)
{
    if (!d || n < 4 || d[0] != 0xFF || d[1] != 0xD8 || (out_ch != 1 && out_ch != 3)) return HPM_ERR_IO;
    try {
        Frame f;
        size_t pos = 2;
        int scans = 0;
        while (true) {
            const long seg = parse_to_scan(d, n, pos, f);
            if (seg == -2 && scans > 0) break; /* no EOI: decode what was read */
            if (seg < 0) return HPM_ERR_IO;
            if (seg == 0) break;
            if (scans == 0 && !setup_frame(f)) return HPM_ERR_IO;
            Scan sc;
            if (!parse_scan_header(d, (size_t)seg, f, sc)) return HPM_ERR_IO;
            if (!decode_scan(d, n, pos, f, sc)) return HPM_ERR_IO;
            ++scans;
        }
        if (!scans) return HPM_ERR_IO;
        bool rgb = false; /* colour space of a 3-component file */
        if (f.ncomp == 3 && !f.jfif) {
            if (f.adobe)
                rgb = f.adobe_transform == 0;
            else
                rgb = f.comp[0].id == 'R' && f.comp[1].id == 'G' && f.comp[2].id == 'B';
        }
        const int W = f.W, H = f.H;
        const size_t npx = (size_t)W * H;
        const int needed = (out_ch == 1 && !rgb) ? 1 : f.ncomp;
        std::vector<uint8_t> full[3];
        for (int c = 0; c < needed; ++c) {
            transform_component(f.comp[c]);
            if (!upsample(f.comp[c], f, full[c])) return HPM_ERR_IO;
            std::vector<int16_t>().swap(f.comp[c].coef);
            std::vector<uint8_t>().swap(f.comp[c].plane);
        }
        px.resize(npx * out_ch);
        if (out_ch == 1) {
            if (!rgb) {
                memcpy(px.data(), full[0].data(), npx);
            } else {
                for (size_t p = 0; p < npx; ++p)
                    px[p] = (uint8_t)((fix16(0.29900) * full[0][p] + fix16(0.58700) * full[1][p] +
                                       fix16(0.11400) * full[2][p] + (1 << 15)) >> 16);
            }
        } else if (f.ncomp == 1) {
            for (size_t p = 0; p < npx; ++p) px[3 * p] = px[3 * p + 1] = px[3 * p + 2] = full[0][p];
        } else if (rgb) {
            for (size_t p = 0; p < npx; ++p) {
                px[3 * p] = full[2][p];
                px[3 * p + 1] = full[1][p];
                px[3 * p + 2] = full[0][p];
            }
        } else {
            ycc_to_bgr(full[0].data(), full[1].data(), full[2].data(), npx, px.data());
        }
        int w = W, h = H;
        orient(px, w, h, out_ch, f.orientation);
        *w_out = w;
        *h_out = h;
        return HPM_OK;
    } catch (const std::bad_alloc &) {
        return HPM_ERR_IO;
    }
}

int hpm_jpeg_size(const uint8_t *d, size_t n, int *w_out, int *h_out)
{
    if (!d || n < 4 || d[0] != 0xFF || d[1] != 0xD8) return HPM_ERR_IO;
    Frame f;
    size_t pos = 2;
    if (parse_to_scan(d, n, pos, f) <= 0) return HPM_ERR_IO;
    const bool tr = f.orientation >= 5;
    *w_out = tr ? f.H : f.W;
    *h_out = tr ? f.W : f.H;
    return HPM_OK;
}

"""JPEG decoding of the image reader (hpm-mvs_b200/csrc/hpm_jpeg.cpp) against
cv::imread, which the reference calls on images/%08d.jpg with
IMREAD_GRAYSCALE (HPM.cpp:490-492, main.cpp:168) and IMREAD_COLOR
(main.cpp:521-523); cv2 4.13 here, over libjpeg-turbo.  Every case is
bit-exact: baseline and progressive files, all chroma samplings OpenCV
writes, restart intervals, optimised Huffman tables, gray files, sizes that
are not multiples of the MCU, EXIF orientation, RGB-coded files, and
sequential files cut short."""
import os
import struct

import numpy as np
import pytest

import hpm_b200 as hb

cv2 = pytest.importorskip("cv2")

SAMPLINGS = {"444": "IMWRITE_JPEG_SAMPLING_FACTOR_444", "420": "IMWRITE_JPEG_SAMPLING_FACTOR_420",
             "422": "IMWRITE_JPEG_SAMPLING_FACTOR_422", "440": "IMWRITE_JPEG_SAMPLING_FACTOR_440",
             "411": "IMWRITE_JPEG_SAMPLING_FACTOR_411"}


def picture(seed, w, h, color=True):
    """Gradients with noise: every coefficient band is populated."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    base = np.stack([xx * 255 // max(w - 1, 1), yy * 255 // max(h - 1, 1), ((xx + yy) * 7) % 256], -1).astype(float)
    a = np.clip(base + rng.normal(0, 40, base.shape), 0, 255).astype(np.uint8)
    return a if color else a[..., 0].copy()


def encode(a, quality=90, sampling="420", progressive=0, restart=0, optimize=0):
    params = [cv2.IMWRITE_JPEG_QUALITY, quality, cv2.IMWRITE_JPEG_PROGRESSIVE, progressive,
              cv2.IMWRITE_JPEG_RST_INTERVAL, restart, cv2.IMWRITE_JPEG_OPTIMIZE, optimize]
    if a.ndim == 3:
        params += [cv2.IMWRITE_JPEG_SAMPLING_FACTOR, getattr(cv2, SAMPLINGS[sampling])]
    ok, buf = cv2.imencode(".jpg", a, params)
    assert ok
    return buf.tobytes()


def check_same(path, gray=True, color=True):
    if gray:
        ref = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        got = hb.read_gray8(path)
        assert got.shape == ref.shape
        np.testing.assert_array_equal(got, ref)
    if color:
        ref = cv2.imread(path, cv2.IMREAD_COLOR)
        got = hb.read_bgr8(path)
        assert got.shape == ref.shape
        np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("progressive", [0, 1])
@pytest.mark.parametrize("sampling", list(SAMPLINGS))
def test_colour_files_match_imread(tmp_path, sampling, progressive):
    path = str(tmp_path / "x.jpg")
    for (w, h) in [(1, 1), (3, 2), (17, 9), (64, 48), (101, 77)]:
        for quality, restart, optimize in [(5, 0, 0), (75, 3, 0), (100, 0, 1), (92, 1, 1)]:
            with open(path, "wb") as f:
                f.write(encode(picture(w * 131 + h, w, h), quality, sampling, progressive, restart, optimize))
            check_same(path)


@pytest.mark.parametrize("progressive", [0, 1])
def test_gray_files_match_imread(tmp_path, progressive):
    path = str(tmp_path / "x.jpg")
    for (w, h) in [(1, 1), (9, 17), (64, 48), (101, 77)]:
        for quality, restart in [(10, 0), (95, 2)]:
            with open(path, "wb") as f:
                f.write(encode(picture(w + h, w, h, color=False), quality, progressive=progressive, restart=restart))
            check_same(path)


def test_full_size_view(tmp_path):
    """A 1600x1200 view, the size of the benchmark scene's images."""
    rng = np.random.default_rng(5)
    a = cv2.resize(np.clip(rng.normal(128, 50, (300, 400, 3)), 0, 255).astype(np.uint8), (1600, 1200))
    path = str(tmp_path / "00000000.jpg")
    with open(path, "wb") as f:
        f.write(encode(a, 95))
    check_same(path)


def exif_segment(orientation, little_endian=True):
    bo = "<" if little_endian else ">"
    tiff = (b"II" if little_endian else b"MM") + struct.pack(bo + "HI", 42, 8)
    entries = [(0x010F, 2, 4, b"cam\0"), (0x0112, 3, 1, struct.pack(bo + "HH", orientation, 0))]
    ifd = struct.pack(bo + "H", len(entries))
    ifd += b"".join(struct.pack(bo + "HHI", t, ty, c) + v for t, ty, c, v in entries) + b"\0\0\0\0"
    payload = b"Exif\0\0" + tiff + ifd
    return b"\xff\xe1" + struct.pack(">H", len(payload) + 2) + payload


@pytest.mark.parametrize("little_endian", [True, False])
def test_exif_orientation_is_applied(tmp_path, little_endian):
    path = str(tmp_path / "x.jpg")
    buf = encode(picture(3, 53, 37), 90, "420")
    for orientation in range(0, 10):
        with open(path, "wb") as f:
            f.write(buf[:2] + exif_segment(orientation, little_endian) + buf[2:])
        check_same(path)
        ref = cv2.imread(path, cv2.IMREAD_GRAYSCALE)
        w, h = hb.ctypes.c_int(), hb.ctypes.c_int()  # the size query reads markers only
        assert hb.lib().hpm_read_gray8(path.encode(), None, 0, hb.ctypes.byref(w), hb.ctypes.byref(h)) == 0
        assert (h.value, w.value) == ref.shape


def segments(buf):
    """(marker, start, end) of each segment up to and including SOS"""
    i, out = 2, []
    while True:
        m = buf[i + 1]
        n = struct.unpack(">H", buf[i + 2:i + 4])[0]
        out.append((m, i, i + 2 + n))
        if m == 0xDA:
            return out
        i += 2 + n


def test_colour_space_from_markers_and_ids(tmp_path):
    """A 3-component file without JFIF is RGB when Adobe's transform is 0 or
    its component ids are 'R', 'G', 'B'; YCbCr otherwise."""
    buf = encode(picture(9, 40, 24), 90, "444")
    app0 = [s for s in segments(buf) if s[0] == 0xE0][0]
    bare = buf[:app0[1]] + buf[app0[2]:]
    segs = segments(bare)
    sof = [s for s in segs if s[0] in (0xC0, 0xC1, 0xC2)][0]
    sos = [s for s in segs if s[0] == 0xDA][0]

    def with_ids(b, ids):
        b = bytearray(b)
        for k, cid in enumerate(ids):
            b[sof[1] + 10 + 3 * k] = cid
            b[sos[1] + 5 + 2 * k] = cid
        return bytes(b)

    def adobe(b, transform):
        return b[:2] + b"\xff\xee" + struct.pack(">H", 14) + b"Adobe" + struct.pack(">HHHB", 100, 0, 0, transform) + b[2:]

    path = str(tmp_path / "x.jpg")
    for variant in [bare, with_ids(bare, b"RGB"), with_ids(bare, b"\x05\x06\x07"), adobe(bare, 0), adobe(bare, 1),
                    adobe(with_ids(bare, b"RGB"), 1)]:
        with open(path, "wb") as f:
            f.write(variant)
        check_same(path)


@pytest.mark.parametrize("restart", [0, 2])
def test_truncated_sequential_files(tmp_path, restart):
    """Cut inside the entropy-coded data: the unit being decoded is finished
    with zero bits and the units after it stay zero, as libjpeg does."""
    buf = encode(picture(4, 160, 120), 90, "420", restart=restart)
    start = buf.index(b"\xff\xda") + 14
    path = str(tmp_path / "x.jpg")
    for frac in np.linspace(0.02, 0.999, 17):
        with open(path, "wb") as f:
            f.write(buf[:start + int((len(buf) - start) * frac)])
        check_same(path)


def test_rejected_files(tmp_path):
    path = str(tmp_path / "x.jpg")
    buf = bytearray(encode(picture(1, 16, 16), 90, "444"))
    sof = buf.index(b"\xff\xc0")
    for patch in [(sof + 1, 0xC9),  # arithmetic coding
                  (sof + 4, 12)]:   # 12-bit samples
        bad = bytearray(buf)
        bad[patch[0]] = patch[1]
        with open(path, "wb") as f:
            f.write(bytes(bad))
        with pytest.raises(hb.HpmError):
            hb.read_bgr8(path)
    with open(path, "wb") as f:
        f.write(b"\xff\xd8\xff\xd9")  # no frame
    with pytest.raises(hb.HpmError):
        hb.read_gray8(path)
    with open(path, "wb") as f:
        f.write(bytes(buf[:sof + 6]))  # ends inside the frame header
    with pytest.raises(hb.HpmError):
        hb.read_gray8(path)


def test_huffman_table_with_too_many_codes_is_rejected(tmp_path):
    """A DHT whose counts ask for more codes of a length than that length
    has (3 one-bit codes) is an error, not a write past the decode table."""
    buf = bytearray(encode(picture(2, 24, 16), 90, "444"))
    i = buf.index(b"\xff\xc4") + 5  # the 16 code counts of the first table
    counts = buf[i:i + 16]
    last = max(k for k in range(16) if counts[k] >= 2)
    buf[i] += 3
    buf[i + last] -= 3 if counts[last] >= 3 else 2
    if counts[last] < 3:
        buf[i] -= 1
    path = str(tmp_path / "x.jpg")
    with open(path, "wb") as f:
        f.write(bytes(buf))
    with pytest.raises(hb.HpmError):
        hb.read_gray8(path)


def test_damaged_files_decode_or_fail_cleanly(tmp_path):
    """Bytes changed, inserted or removed anywhere in valid files, or the file
    cut short: every read either returns an image or raises HpmError."""
    rng = np.random.default_rng(0)
    bases = [encode(picture(s, 40, 28), 85, smp, prog, rst) for s, smp, prog, rst in
             [(1, "420", 0, 0), (2, "444", 1, 0), (3, "422", 0, 2), (4, "420", 1, 3)]]
    path = str(tmp_path / "x.jpg")
    for it in range(300):
        b = bytearray(bases[it % len(bases)])
        for _ in range(int(rng.integers(1, 6))):
            i = int(rng.integers(2, len(b)))
            op = int(rng.integers(0, 3))
            if op == 0:
                b[i] = int(rng.integers(0, 256))
            elif op == 1:
                b.insert(i, int(rng.integers(0, 256)))
            elif len(b) > 10:
                del b[i]
        if rng.random() < 0.2:
            b = b[:int(rng.integers(2, len(b)))]
        with open(path, "wb") as f:
            f.write(bytes(b))
        for read in (hb.read_gray8, hb.read_bgr8):
            try:
                img = read(path)
                assert img.dtype == np.uint8 and img.size > 0
            except hb.HpmError:
                pass

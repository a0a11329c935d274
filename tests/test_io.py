"""Host-side I/O of the drop-in: images/ decoding and the 3200-pixel image
cap (InuputInitialization, HPM.cpp:482-554) against the OpenCV calls the
reference makes (cv2 4.13 here)."""
import os

import numpy as np
import pytest

import hpm_b200 as hb

cv2 = pytest.importorskip("cv2")


@pytest.mark.parametrize("shape", [(37, 53), (64, 80, 3), (21, 33, 4), (100, 7, 3)])
@pytest.mark.parametrize("ext", [".png", ".pgm"])
def test_read_gray8_matches_imread(tmp_path, shape, ext):
    if ext == ".pgm" and len(shape) == 3:
        pytest.skip("PGM is single-channel")
    rng = np.random.default_rng(sum(shape))
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    for level in ([0, 6, 9] if ext == ".png" else [None]):
        path = str(tmp_path / f"img{ext}")
        cv2.imwrite(path, img, [] if level is None else [cv2.IMWRITE_PNG_COMPRESSION, level])
        np.testing.assert_array_equal(hb.read_gray8(path), cv2.imread(path, cv2.IMREAD_GRAYSCALE))


def test_read_gray8_rejects_bad_files(tmp_path):
    bad = tmp_path / "x.png"
    bad.write_bytes(b"\x89PNG\r\n\x1a\nnot a png")
    with pytest.raises(hb.HpmError):
        hb.read_gray8(str(bad))
    with pytest.raises(hb.HpmError):
        hb.read_gray8(str(tmp_path / "missing.png"))


@pytest.mark.parametrize("src,dst,ch", [((1600, 1200), (400, 300), 1), ((1600, 1200), (800, 600), 3),
                                        ((6048, 4032), (3200, 2133), 1), ((605, 403), (1000, 666), 1),
                                        ((7, 5), (3, 2), 3)])
def test_resize_linear_matches_cv2(src, dst, ch):
    rng = np.random.default_rng(src[0])
    shape = (src[1], src[0]) if ch == 1 else (src[1], src[0], ch)
    a = rng.uniform(-300, 300, shape).astype(np.float32)
    np.testing.assert_array_equal(hb.resize_linear(a, *dst), cv2.resize(a, dst, interpolation=cv2.INTER_LINEAR))


def test_synthetic_scene_command_writes_a_dense_folder(tmp_path):
    """python hpm-mvs_b200/synthetic.py FOLDER writes images/%08d.jpg,
    cams/%08d_cam.txt and pair.txt in the reference's layout, plus the
    ground-truth depth maps as gt/%08d.dmb, all readable through the C ABI."""
    import synthetic as syn

    folder = str(tmp_path / "scene")
    syn.main([folder, "--views", "3", "--size", "64x48", "--sources", "2", "--planes", "2", "--spheres", "0"])
    assert hb.read_pair(os.path.join(folder, "pair.txt")) == [(0, [1, 2]), (1, [0, 2]), (2, [1, 0])]
    for v in range(3):
        assert hb.read_gray8(os.path.join(folder, "images", f"{v:08d}.jpg")).shape == (48, 64)
        assert hb.read_camera(os.path.join(folder, "cams", f"{v:08d}_cam.txt"))["depth_max"] > 0
        gt = hb.read_dmb(os.path.join(folder, "gt", f"{v:08d}.dmb"))
        assert gt.shape == (48, 64) and (gt > 0).mean() > 0.9


@pytest.mark.parametrize("src,dst,ch", [((4000, 3000), (3200, 2400), 3), ((3301, 2001), (3200, 1940), 3),
                                        ((641, 479), (500, 377), 3), ((640, 480), (320, 240), 3),
                                        ((97, 61), (200, 130), 3), ((33, 17), (34, 18), 1), ((1600, 1200), (1599, 1199), 1)])
def test_resize_linear_u8_matches_cv2(src, dst, ch):
    """RescaleImageAndCamera (HPM.cpp:187-208) resizes the fusion's 8-bit
    colour images with cv::resize INTER_LINEAR: the fixed-point result is
    reproduced byte for byte, downscales (the 3200-pixel cap), 2:1 and
    upscales alike."""
    rng = np.random.default_rng(src[0] + dst[0] + ch)
    shape = (src[1], src[0], ch) if ch > 1 else (src[1], src[0])
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    np.testing.assert_array_equal(hb.resize_linear_u8(img, *dst), cv2.resize(img, dst, interpolation=cv2.INTER_LINEAR))


def test_resize_linear_u8_random_sizes_match_cv2():
    """A seeded sweep of source and destination sizes (down, up, mixed, one
    axis unchanged), so that the byte equality does not rest on the handful
    of sizes above."""
    rng = np.random.default_rng(2024)
    for _ in range(300):
        sw, sh = (int(x) for x in rng.integers(1, 260, 2))
        dw, dh = (int(x) for x in rng.integers(1, 260, 2))
        ch = int(rng.choice([1, 3]))
        shape = (sh, sw, ch) if ch > 1 else (sh, sw)
        img = rng.integers(0, 256, shape, dtype=np.uint8)
        np.testing.assert_array_equal(hb.resize_linear_u8(img, dw, dh),
                                      cv2.resize(img, (dw, dh), interpolation=cv2.INTER_LINEAR),
                                      err_msg=f"{sw}x{sh} -> {dw}x{dh}, {ch} channels")


@pytest.mark.parametrize("shape", [(2201, 3300), (3300, 2201), (3201, 3201)])
def test_python_front_end_caps_views_like_the_reference(tmp_path, shape):
    """hpm_mvs.load_view: views over 3200 pixels are resized as
    InuputInitialization does (HPM.cpp:524-551): factor = min(3200/w,
    3200/h) in float, new size = std::round of the float product (halves
    away from zero), K scaled by the float size ratios, the image by
    cv::resize INTER_LINEAR on the float image."""
    import hpm_mvs

    h, w = shape
    rng = np.random.default_rng(h * 7 + w)
    img = rng.integers(0, 256, (h, w), dtype=np.uint8)
    os.makedirs(tmp_path / "images")
    os.makedirs(tmp_path / "cams")
    cv2.imwrite(str(tmp_path / "images" / "00000000.pgm"), img)
    with open(tmp_path / "cams" / "00000000_cam.txt", "w") as f:
        f.write("extrinsic\n1 0 0 0\n0 1 0 0\n0 0 1 0\n0 0 0 1\n\nintrinsic\n"
                f"1000 0 {w / 2}\n0 1000 {h / 2}\n0 0 1\n\n2 0.02 192 6\n")
    out, cam = hpm_mvs.load_view(str(tmp_path), 0)
    f32 = np.float32
    factor = min(f32(3200) / f32(w), f32(3200) / f32(h))
    nw = int(np.floor(np.float64(f32(w) * factor) + 0.5))
    nh = int(np.floor(np.float64(f32(h) * factor) + 0.5))
    assert out.shape == (nh, nw) and (cam["width"], cam["height"]) == (nw, nh)
    np.testing.assert_array_equal(out, cv2.resize(img.astype(np.float32), (nw, nh), interpolation=cv2.INTER_LINEAR))
    sx, sy = f32(nw) / f32(w), f32(nh) / f32(h)
    assert cam["K"][0] == f32(1000) * sx and cam["K"][4] == f32(1000) * sy

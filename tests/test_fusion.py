"""Fusion (RunFusion, main.cpp:502-633) on the CPU: the oracle's sequential
restatement on scenes with known geometry, the colour reader against
cv::imread(IMREAD_COLOR), and the PLY writer's format
(StoreColorPlyFileBinaryPointCloud, HPM.cpp:403-456)."""
import numpy as np
import pytest

import hpm_b200 as hb
import oracle as orc
import synthetic as syn

cv2 = pytest.importorskip("cv2")


def fusion_inputs(seed, w, h, nv, noise=0.0):
    """Ground-truth depth and world normals of every view (optionally with
    multiplicative depth noise), a colour image per view with distinct B, G,
    R channels, and the scene's problems."""
    sc = syn.make_scene(seed, w, h, nv, n_planes=4, n_spheres=1)
    rng = np.random.default_rng(seed)
    depths = [(d * (1 + noise * rng.standard_normal(d.shape))).astype(np.float32) for d in sc.gt_depth]
    normals = [n.astype(np.float32) for n in sc.gt_normal]
    colors = [np.stack([g, 255 - g, (g.astype(np.int32) * 7 % 256).astype(np.uint8)], -1) for g in sc.images]
    problems = [(v, list(sc.pairs[v][1])) for v in range(nv)]
    return sc, depths, normals, colors, problems


def test_oracle_fusion_on_true_geometry():
    sc, depths, normals, colors, problems = fusion_inputs(1, 96, 72, 4)
    xyz, nrm, col = orc.fuse(sc.cams, depths, normals, colors, problems)
    n_px = 4 * 96 * 72
    # exact geometry agrees across views wherever the views overlap: a large
    # share of pixels becomes points, and each source pixel is used once
    assert 0.2 * n_px < len(xyz) < n_px
    assert np.isfinite(xyz).all()
    np.testing.assert_allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-4)
    # colours come from the reference pixel, B G R
    assert set(np.unique(col[:, 0] + col[:, 1])) == {255.0}


def test_oracle_fusion_rejects_inconsistent_maps():
    sc, depths, normals, colors, problems = fusion_inputs(2, 64, 48, 3)
    rng = np.random.default_rng(0)
    scrambled = [d * rng.uniform(0.5, 1.5, d.shape).astype(np.float32) for d in depths]
    xyz_ok, _, _ = orc.fuse(sc.cams, depths, normals, colors, problems)
    xyz_bad, _, _ = orc.fuse(sc.cams, scrambled, normals, colors, problems)
    assert len(xyz_bad) < 0.2 * len(xyz_ok)
    empty = [np.zeros_like(d) for d in depths]
    assert len(orc.fuse(sc.cams, empty, normals, colors, problems)[0]) == 0
    assert len(orc.fuse(sc.cams, depths, normals, colors, [(0, [])])[0]) == 0


@pytest.mark.parametrize("shape", [(21, 33), (40, 24, 3), (17, 9, 4)])
@pytest.mark.parametrize("ext", [".png", ".pgm"])
def test_read_bgr8_matches_imread_color(tmp_path, shape, ext):
    if ext == ".pgm" and len(shape) == 3:
        pytest.skip("PGM is single-channel")
    img = np.random.default_rng(sum(shape)).integers(0, 256, shape, dtype=np.uint8)
    path = str(tmp_path / f"i{ext}")
    cv2.imwrite(path, img)
    np.testing.assert_array_equal(hb.read_bgr8(path), cv2.imread(path, cv2.IMREAD_COLOR))


def test_ply_layout(tmp_path):
    xyz = np.array([[1, 2, 3], [np.inf, 0, 1], [4, 5, np.nan]], np.float32)
    nrm = np.array([[0, 0, 1], [0, 1, 0], [1, 0, 0]], np.float32)
    bgr = np.array([[10, 20, 30], [40, 50, 60], [70, 80, 90]], np.uint8)
    path = str(tmp_path / "m.ply")
    hb.write_ply(path, xyz, nrm, bgr)
    data = open(path, "rb").read()
    head, body = data.split(b"end_header\n")
    assert head.decode().splitlines() == [
        "ply", "format binary_little_endian 1.0", "element vertex 3", "property float x", "property float y",
        "property float z", "property float nx", "property float ny", "property float nz", "property uchar red",
        "property uchar green", "property uchar blue"]
    rec = np.frombuffer(body, dtype=np.dtype([("xyz", "<f4", 3), ("n", "<f4", 3), ("rgb", "u1", 3)]))
    assert len(rec) == 3
    np.testing.assert_array_equal(rec["xyz"], [[1, 2, 3], [0, 0, 0], [0, 0, 0]])  # non-finite -> origin
    np.testing.assert_array_equal(rec["n"], nrm)
    np.testing.assert_array_equal(rec["rgb"], bgr[:, ::-1])  # red, green, blue


@pytest.mark.parametrize("acmm", [False, True])
def test_product_ordered_pass_matches_oracle(acmm):
    """hpm_fuse_pass, the host half of hpm_fuse (acmm False) and of
    hpm_fuse_acmm (acmm True), on the oracle's pairs (or_fuse_pairs, the
    restatement of their GPU pass) against the oracle's whole RunFusion
    (or_fuse / or_fuse_acmm, each pinned to the reference's own code in
    tests/test_fusion_reference.py): the same points in the same order, bit
    for bit; colour bytes as the reference's PLY writer truncates them."""
    sc, depths, normals, colors, problems = fusion_inputs(3, 160, 120, 5, noise=0.002)
    pairs = [orc.fuse_pairs(sc.cams, depths, normals, ref, srcs) for ref, srcs in problems]
    xyz, nrm, bgr = hb.fuse_pass(sc.cams, depths, normals, colors, problems, pairs, acmm=acmm)
    oxyz, onrm, ocol = orc.fuse(sc.cams, depths, normals, colors, problems, acmm=acmm)
    assert len(xyz) == len(oxyz) and len(xyz) > 1000, (len(xyz), len(oxyz))
    np.testing.assert_array_equal(xyz, oxyz)
    np.testing.assert_array_equal(nrm, onrm)
    np.testing.assert_array_equal(bgr, ocol.astype(np.int32).astype(np.uint8))

"""The COLMAP -> dense-folder converter (hpm-mvs_b200/colmap.py) against the
files the reference's own converter (ACMM+NESP/windows/colmap2mvsnet_acm.py)
wrote for the same sparse model (tests/golden/colmap/, made by
make_colmap_golden.py): cams/*_cam.txt and pair.txt byte for byte, for the
text and binary models and for the inverse-depth depth count (max_d 0)."""
import os
import shutil

import pytest

import colmap

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "colmap")


@pytest.mark.parametrize("tag,ext,max_d", [("txt", ".txt", 192), ("bin", ".bin", 192), ("txt_maxd0", ".txt", 0)])
def test_converter_matches_reference_files(tmp_path, tag, ext, max_d):
    pytest.importorskip("cv2")
    dense = tmp_path / "dense"
    shutil.copytree(os.path.join(GOLD, "model", "images"), dense / "images")
    shutil.copytree(os.path.join(GOLD, "model", "sparse" if ext == ".txt" else "sparse_bin"), dense / "sparse")
    out = tmp_path / "out"
    out.mkdir()
    n = colmap.convert(str(dense), str(out), max_d=max_d, model_ext=ext)
    exp = os.path.join(GOLD, "expected_" + tag)
    assert n == 8
    assert open(out / "pair.txt").read() == open(os.path.join(exp, "pair.txt")).read()
    names = sorted(os.listdir(os.path.join(exp, "cams")))
    assert sorted(os.listdir(out / "cams")) == names
    for name in names:
        assert open(out / "cams" / name).read() == open(os.path.join(exp, "cams", name)).read(), name
    assert sorted(os.listdir(out / "images")) == [f"{i:08d}.jpg" for i in range(8)]


def test_converted_folder_reads_back(tmp_path):
    """The drop-in readers take what the converter writes."""
    pytest.importorskip("cv2")
    import hpm_b200 as hb

    dense = tmp_path / "dense"
    shutil.copytree(os.path.join(GOLD, "model", "images"), dense / "images")
    shutil.copytree(os.path.join(GOLD, "model", "sparse"), dense / "sparse")
    out = tmp_path / "out"
    out.mkdir()
    colmap.convert(str(dense), str(out), png=True)
    pairs = hb.read_pair(str(out / "pair.txt"))
    assert len(pairs) == 8 and all(0 < len(s) <= 7 for _, s in pairs)
    cam = hb.read_camera(str(out / "cams" / "00000003_cam.txt"))
    assert cam["K"][0] > 0 and cam["depth_max"] > cam["depth_min"] > 0
    assert hb.read_gray8(str(out / "images" / "00000003.png")).shape == (48, 64)

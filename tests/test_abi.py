"""The C ABI boundary (include/hpm_b200.h) without a GPU: the library loads,
exports every declared entry point, and its host-only functions (file
formats, argument checks) behave like the reference's readers and writers."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

import hpm_b200 as hb
import synthetic as syn


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hpm_b200.h")).read()
    return sorted(set(re.findall(r"\b(hpm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = hb.lib()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(hb.EXPORTED) == sorted(names)


def test_dmb_round_trip(tmp_path):
    d = np.random.default_rng(0).random((7, 5)).astype(np.float32)
    n = np.random.default_rng(1).random((7, 5, 3)).astype(np.float32)
    hb.write_dmb(str(tmp_path / "depths.dmb"), d)
    hb.write_dmb(str(tmp_path / "normals.dmb"), n)
    np.testing.assert_array_equal(hb.read_dmb(str(tmp_path / "depths.dmb")), d)
    np.testing.assert_array_equal(hb.read_dmb(str(tmp_path / "normals.dmb")), n)
    raw = (tmp_path / "depths.dmb").read_bytes()
    # header int32 type=1, h, w, nb then row-major float32 (HPM.cpp:270-295)
    assert np.frombuffer(raw[:16], "<i4").tolist() == [1, 7, 5, 1]
    assert len(raw) == 16 + 7 * 5 * 4


def test_dmb_errors(tmp_path):
    with pytest.raises(hb.HpmError):
        hb.read_dmb(str(tmp_path / "missing.dmb"))
    bad = tmp_path / "bad.dmb"
    bad.write_bytes(np.array([2, 3, 3, 1], "<i4").tobytes() + bytes(36))
    with pytest.raises(hb.HpmError):
        hb.read_dmb(str(bad))
    short = tmp_path / "short.dmb"
    short.write_bytes(np.array([1, 3, 3, 1], "<i4").tobytes() + bytes(10))
    with pytest.raises(hb.HpmError):
        hb.read_dmb(str(short))
    with pytest.raises(hb.HpmError):
        hb.write_dmb(str(tmp_path / "no" / "dir" / "x.dmb"), np.zeros((2, 2), np.float32))


def test_camera_and_pair_files(tmp_path):
    sc = syn.make_scene(0, 40, 30, 4, n_planes=2)
    syn.write_dense_folder(sc, str(tmp_path))
    for i in range(4):
        c = hb.read_camera(str(tmp_path / "cams" / f"{i:08d}_cam.txt"))
        np.testing.assert_allclose(c["K"], sc.cams[i]["K"], rtol=1e-6)
        np.testing.assert_allclose(c["R"], sc.cams[i]["R"], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(c["t"], sc.cams[i]["t"], rtol=1e-6, atol=1e-6)
        assert abs(c["depth_min"] - sc.depth_min) < 1e-6 and abs(c["depth_max"] - sc.depth_max) < 1e-6
    pairs = hb.read_pair(str(tmp_path / "pair.txt"))
    assert [p[0] for p in pairs] == [0, 1, 2, 3]
    assert pairs[1][1] == sc.pairs[1][1]


def test_pair_drops_non_positive_scores(tmp_path):
    p = tmp_path / "pair.txt"
    p.write_text("2\n0\n3 1 2.5 2 0 3 -1.0\n1\n2 0 1.0 2 4.0\n")
    assert hb.read_pair(str(p)) == [(0, [1]), (1, [0, 2])]
    (tmp_path / "broken.txt").write_text("3\n0\n2 1")
    with pytest.raises(hb.HpmError):
        hb.read_pair(str(tmp_path / "broken.txt"))


def test_camera_errors(tmp_path):
    with pytest.raises(hb.HpmError):
        hb.read_camera(str(tmp_path / "none.txt"))
    (tmp_path / "c.txt").write_text("intrinsic\n1 0 0\n")
    with pytest.raises(hb.HpmError):
        hb.read_camera(str(tmp_path / "c.txt"))


def test_null_context_is_an_argument_error():
    L = hb.lib()
    for name in ["hpm_destroy", "hpm_run_patchmatch", "hpm_set_views", "hpm_get_result", "hpm_clear_prior"]:
        fn = getattr(L, name)
        fn.restype = ctypes.c_int
    assert L.hpm_destroy(None) == -1
    assert L.hpm_clear_prior(None) == -1
    assert L.hpm_get_result(None, None, None) == -1
    assert L.hpm_create(None, 0) == -1
    assert L.hpm_run_scene_acmm(None, 2, None, None, 2, None, None, None, None, None, None, None) == -1
    # the fusion's host pass checks its arguments before touching any
    assert L.hpm_fuse_pass(2, 1, None, None, None, None, 0, None, None, None, None, None, None, None, None, None,
                           ctypes.c_longlong(0), None) == -1


@pytest.mark.skipif(gpu_available(), reason="checks the behaviour on a machine without a GPU")
def test_create_without_gpu_reports_cuda_error():
    h = ctypes.c_void_p()
    rc = hb.lib().hpm_create(ctypes.byref(h), 0)
    assert rc == -2 and not h.value


def test_default_params_are_the_reference_defaults():
    p = hb.default_params(1.2, 9.6)
    assert (p.max_iterations, p.patch_size, p.radius_increment, p.top_k) == (3, 11, 2, 4)
    # the HPM-MVS kernels unless the ACMM+NESP variant is asked for
    assert (p.variant, p.hierarchy) == (0, 0)
    assert (p.sigma_spatial, p.sigma_color) == (5.0, 3.0)
    assert p.geom_consistency == 0 and p.planar_prior == 0


def test_host_binary_builds_and_runs_without_a_gpu_call():
    """The C++ host mirror links against the C ABI and answers --help; a
    missing dense folder is a clean error, not a crash."""
    import os
    import subprocess

    exe = os.path.join(os.path.dirname(os.path.abspath(hb.__file__)), "hpm_mvs")
    assert os.path.exists(exe), "make -C hpm-mvs_b200 builds hpm_mvs"
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "dense_folder" in r.stdout
    r = subprocess.run([exe, "/nonexistent/folder"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "pair.txt" in r.stderr

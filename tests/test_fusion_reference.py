"""The fusion oracle (or_fuse) against the reference's own RunFusion.

oracle/_ref/libfusion_ref.so is RunFusion (HPM-MVS/main.cpp:502-633) and the
HPM.cpp helpers it calls, compiled unchanged from the reference tree on the
host (oracle/Makefile, target `fusion`).  Both run on the same dense folder:
the reference reads its files (cameras as text, .dmb depth and normal maps,
images through the checker's cv::imread stand-in) and writes its PLY; the
oracle gets the same arrays.  Every point must agree bit for bit, in order.
The product's hpm_fuse is checked against the oracle point for point in
tests/test_gpu_fusion.py, so this pins the product's fusion too.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import ROOT

import oracle as orc
import synthetic as syn

LIB = os.path.join(ROOT, "oracle", "_ref", "libfusion_ref.so")
LIB_ACMM = os.path.join(ROOT, "oracle", "_ref", "libfusion_acmm_ref.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="reference fusion checker not built "
                                                                 "(make -C oracle fusion REF_DIR=...)")


def _write_dmb(path, a):
    a = np.ascontiguousarray(a, np.float32)
    h, w = a.shape[:2]
    nb = 1 if a.ndim == 2 else a.shape[2]
    with open(path, "wb") as f:
        f.write(np.array([1, h, w, nb], np.int32).tobytes())
        f.write(a.tobytes())


def _write_raw(path, bgr):
    h, w = bgr.shape[:2]
    with open(path, "wb") as f:
        f.write(b"RAW3" + np.array([h, w], np.int32).tobytes())
        f.write(np.ascontiguousarray(bgr, np.uint8).tobytes())


def _read_ply(path):
    with open(path, "rb") as f:
        data = f.read()
    head, body = data.split(b"end_header\n", 1)
    n = int([ln for ln in head.split(b"\n") if ln.startswith(b"element vertex")][0].split()[-1])
    dt = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
                   ("r", "u1"), ("g", "u1"), ("b", "u1")])
    return np.frombuffer(body, dt, count=n)


def _scene_folder(tmp_path, geom, seed, tree="HPM"):
    sc = syn.make_scene(seed, 120, 90, 6, n_planes=5, n_spheres=1)
    folder = str(tmp_path / f"scene{seed}_{geom}")
    syn.write_dense_folder(sc, folder)  # cameras and pair.txt (the images are replaced below)
    rng = np.random.default_rng(seed)
    nv = len(sc.images)
    depths, normals, colors = [], [], []
    for v in range(nv):
        # maps as a pass leaves them: 0.3 % depth noise, some holes, some
        # normals off by more than the 10-degree test
        d = sc.gt_depth[v] * rng.uniform(0.997, 1.003, sc.gt_depth[v].shape)
        d[rng.random(d.shape) < 0.03] = 0.0
        n = sc.gt_normal[v] + rng.normal(0, 0.05, sc.gt_normal[v].shape) * (rng.random(d.shape) < 0.2)[..., None]
        n /= np.linalg.norm(n, axis=-1, keepdims=True)
        depths.append(d.astype(np.float32))
        normals.append(n.astype(np.float32))
        colors.append(rng.integers(0, 256, d.shape + (3,), dtype=np.uint8))
        out = os.path.join(folder, tree, f"2333_{v:08d}")
        os.makedirs(out, exist_ok=True)
        _write_dmb(os.path.join(out, "depths_geom.dmb" if geom else "depths.dmb"), depths[-1])
        _write_dmb(os.path.join(out, "normals.dmb"), normals[-1])
        _write_raw(os.path.join(folder, "images", f"{v:08d}.jpg"), colors[-1])
    problems = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(nv)]
    return sc, folder, depths, normals, colors, problems


def _run_reference(lib_path, folder, problems, geom):
    lib = ctypes.CDLL(lib_path)
    refs = np.array([p[0] for p in problems], np.int32)
    counts = np.array([len(p[1]) for p in problems], np.int32)
    srcs = np.zeros((len(problems), 32), np.int32)
    for i, (_, s) in enumerate(problems):
        srcs[i, :len(s)] = s
    rc = lib.ref_run_fusion(folder.encode(), len(problems), refs.ctypes.data_as(ctypes.c_void_p),
                            counts.ctypes.data_as(ctypes.c_void_p), srcs.ctypes.data_as(ctypes.c_void_p), geom)
    assert rc == 0


@pytest.mark.parametrize("geom", [0, 1])
def test_oracle_fusion_matches_the_reference_run_fusion(tmp_path, geom):
    sc, folder, depths, normals, colors, problems = _scene_folder(tmp_path, geom, seed=3 + geom)
    _run_reference(LIB, folder, problems, geom)
    ref = _read_ply(os.path.join(folder, "HPM", "HPM_model.ply"))
    xyz, nrm, col = orc.fuse(sc.cams, depths, normals, colors, problems)
    _check(ref, xyz, nrm, col)


@pytest.mark.skipif(not os.path.exists(LIB_ACMM), reason="reference ACMM+NESP fusion checker not built")
def test_oracle_fusion_matches_the_reference_run_fusion_acmm(tmp_path):
    """The ACMM+NESP variant's RunFusion (ACMM+NESP/windows/main.cpp:154-297,
    always from depths_geom.dmb): at least 2 agreeing sources, and the mean
    of the point, normal and colour with the agreeing source pixels'."""
    sc, folder, depths, normals, colors, problems = _scene_folder(tmp_path, 1, seed=9, tree="ACMM_NESP")
    _run_reference(LIB_ACMM, folder, problems, 1)
    ref = _read_ply(os.path.join(folder, "ACMM_NESP", "ACMM_NESP_model.ply"))
    xyz, nrm, col = orc.fuse(sc.cams, depths, normals, colors, problems, acmm=True)
    _check(ref, xyz, nrm, col)
    # the variant's rule is another one than HPM-MVS's
    assert len(xyz) != len(orc.fuse(sc.cams, depths, normals, colors, problems)[0])


def _check(ref, xyz, nrm, col):
    assert len(ref) > 1000 and len(ref) == len(xyz), (len(ref), len(xyz))
    # the reference's writer replaces non-finite coordinates by 0 (HPM.cpp:433-437)
    bad = ~(np.isfinite(xyz).all(1))
    xyz = np.where(bad[:, None], 0.0, xyz).astype(np.float32)
    np.testing.assert_array_equal(np.stack([ref["x"], ref["y"], ref["z"]], 1), xyz)
    np.testing.assert_array_equal(np.stack([ref["nx"], ref["ny"], ref["nz"]], 1), nrm)
    np.testing.assert_array_equal(np.stack([ref["r"], ref["g"], ref["b"]], 1),
                                  col[:, ::-1].astype(np.int32).astype(np.uint8))

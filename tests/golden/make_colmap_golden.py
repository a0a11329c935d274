"""Generate tests/golden/colmap/: a small synthetic COLMAP sparse model and
what the reference's converter (ACMM+NESP/windows/colmap2mvsnet_acm.py)
writes for it (cams/*_cam.txt, pair.txt).

The model comes from a seeded synthetic scene (hpm-mvs_b200/synthetic.py):
8 images with PINHOLE and SIMPLE_RADIAL cameras, 3D points sampled on the
true surfaces, each observed by the images that see it (depth test against
the true depth maps), plus unmatched observations (point id -1).  The model
is written in COLMAP's text and binary layouts.

The reference script runs in this process, from the reference tree, through
its processing_single_scene().  It calls np.asscalar, which NumPy 2 no
longer has, so that one name is provided (as ndarray.item) before the
script runs; nothing else is changed.

Usage (from the repository root, where the reference tree is available):
    python tests/golden/make_colmap_golden.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import shutil
import struct
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "hpm-mvs_b200")]


def rot_to_quat(R):
    """Unit quaternion (w, x, y, z) of a rotation matrix (Shepperd's method)."""
    t = np.trace(R)
    if t > 0:
        s = np.sqrt(t + 1.0) * 2
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k]) * 2
        q = [0.0] * 4
        q[0] = (R[k, j] - R[j, k]) / s
        q[1 + i] = 0.25 * s
        q[1 + j] = (R[j, i] + R[i, j]) / s
        q[1 + k] = (R[k, i] + R[i, k]) / s
    q = np.array(q)
    return q if q[0] >= 0 else -q


def build_model(seed=7, n_views=8, w=64, h=48):
    import synthetic as syn

    sc = syn.make_scene(seed, w, h, n_views, n_planes=4, n_spheres=1)
    rng = np.random.default_rng(seed)
    cams, images, points = [], [], []
    obs = [[] for _ in range(n_views)]
    for v in range(n_views):
        K = sc.cams[v]["K"].reshape(3, 3).astype(np.float64)
        model = "PINHOLE" if v % 2 == 0 else "SIMPLE_RADIAL"
        params = [K[0, 0], K[1, 1], K[0, 2], K[1, 2]] if model == "PINHOLE" else [K[0, 0], K[0, 2], K[1, 2], 0.0]
        cams.append((v + 1, model, w, h, params))
    # points: random pixels of every view lifted to the true surface
    for v in range(n_views):
        c = sc.cams[v]
        K, R, t = c["K"].reshape(3, 3).astype(np.float64), c["R"].reshape(3, 3).astype(np.float64), c["t"].astype(np.float64)
        for _ in range(40):
            x, y = rng.uniform(2, w - 3), rng.uniform(2, h - 3)
            d = float(sc.gt_depth[v][int(y), int(x)])
            Xc = d * np.linalg.inv(K) @ [x, y, 1.0]
            points.append(R.T @ (Xc - t))
    for pid, X in enumerate(points):
        for v in range(n_views):
            c = sc.cams[v]
            K, R, t = c["K"].reshape(3, 3).astype(np.float64), c["R"].reshape(3, 3).astype(np.float64), c["t"].astype(np.float64)
            Xc = R @ X + t
            if Xc[2] <= 0:
                continue
            u = K @ Xc
            x, y = u[0] / u[2], u[1] / u[2]
            if not (0 <= x < w - 1 and 0 <= y < h - 1):
                continue
            if abs(float(sc.gt_depth[v][int(round(y)), int(round(x))]) - Xc[2]) < 0.01 * Xc[2]:
                obs[v].append((x, y, pid + 1))
    for v in range(n_views):
        for _ in range(5):
            obs[v].append((rng.uniform(0, w), rng.uniform(0, h), -1))
        rng.shuffle(obs[v])
        c = sc.cams[v]
        R = c["R"].reshape(3, 3).astype(np.float64)
        images.append((v + 1, rot_to_quat(R), c["t"].astype(np.float64), v + 1, f"view_{v}.png", obs[v]))
    return sc, cams, images, points


def write_text(folder, cams, images, points):
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "cameras.txt"), "w") as f:
        f.write("# Camera list\n")
        for cid, model, w, h, params in cams:
            f.write(f"{cid} {model} {w} {h} " + " ".join(repr(float(p)) for p in params) + "\n")
    with open(os.path.join(folder, "images.txt"), "w") as f:
        f.write("# Image list\n")
        for iid, q, t, cid, name, ob in images:
            f.write(f"{iid} " + " ".join(repr(float(x)) for x in list(q) + list(t)) + f" {cid} {name}\n")
            f.write(" ".join(f"{repr(float(x))} {repr(float(y))} {p}" for x, y, p in ob) + "\n")
    with open(os.path.join(folder, "points3D.txt"), "w") as f:
        f.write("# 3D point list\n")
        for pid, X in enumerate(points):
            f.write(f"{pid + 1} " + " ".join(repr(float(x)) for x in X) + " 128 128 128 0.5\n")


def write_binary(folder, cams, images, points):
    ids = {"PINHOLE": 1, "SIMPLE_RADIAL": 2}
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "cameras.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(cams)))
        for cid, model, w, h, params in cams:
            f.write(struct.pack("<iiQQ", cid, ids[model], w, h) + struct.pack("<" + "d" * len(params), *params))
    with open(os.path.join(folder, "images.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(images)))
        for iid, q, t, cid, name, ob in images:
            f.write(struct.pack("<idddddddi", iid, *q, *t, cid) + name.encode() + b"\x00")
            f.write(struct.pack("<Q", len(ob)))
            for x, y, p in ob:
                f.write(struct.pack("<ddq", x, y, p))
    with open(os.path.join(folder, "points3D.bin"), "wb") as f:
        f.write(struct.pack("<Q", len(points)))
        for pid, X in enumerate(points):
            f.write(struct.pack("<QdddBBBd", pid + 1, *X, 128, 128, 128, 0.5) + struct.pack("<Q", 0))


def run_reference(script, dense, save, model_ext, max_d):
    np.asscalar = lambda a: a.item()  # removed from NumPy 2; the script still calls it
    spec = importlib.util.spec_from_file_location("colmap2mvsnet_acm", script)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["colmap2mvsnet_acm"] = mod  # its worker pool pickles calc_score by module name
    spec.loader.exec_module(mod)
    args = argparse.Namespace(dense_folder=dense, save_folder=save, max_d=max_d, interval_scale=1.0, theta0=5,
                              sigma1=1, sigma2=10, model_ext=model_ext)
    mod.processing_single_scene(args)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference tree")
    ap.add_argument("--out", default=os.path.join(HERE, "colmap"))
    a = ap.parse_args()
    import cv2

    script = os.path.join(a.reference, "ACMM+NESP", "windows", "colmap2mvsnet_acm.py")
    sc, cams, images, points = build_model()
    if os.path.exists(a.out):
        shutil.rmtree(a.out)
    model = os.path.join(a.out, "model")
    write_text(os.path.join(model, "sparse"), cams, images, points)
    write_binary(os.path.join(model, "sparse_bin"), cams, images, points)
    os.makedirs(os.path.join(model, "images"))
    for v in range(len(images)):
        cv2.imwrite(os.path.join(model, "images", f"view_{v}.png"), sc.images[v])
    with tempfile.TemporaryDirectory() as tmp:
        for tag, ext, max_d in [("txt", ".txt", 192), ("bin", ".bin", 192), ("txt_maxd0", ".txt", 0)]:
            dense = os.path.join(tmp, tag)
            shutil.copytree(os.path.join(model, "images"), os.path.join(dense, "images"))
            shutil.copytree(os.path.join(model, "sparse" if ext == ".txt" else "sparse_bin"),
                            os.path.join(dense, "sparse"))
            save = os.path.join(tmp, tag + "_out")
            os.makedirs(save)
            run_reference(script, dense, save, ext, max_d)
            exp = os.path.join(a.out, "expected_" + tag)
            shutil.copytree(os.path.join(save, "cams"), os.path.join(exp, "cams"))
            shutil.copyfile(os.path.join(save, "pair.txt"), os.path.join(exp, "pair.txt"))
    print("wrote", a.out)


if __name__ == "__main__":
    main()

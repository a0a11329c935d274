#!/usr/bin/env python
"""COLMAP sparse model -> HPM-MVS dense folder (images/, cams/, pair.txt):
the input side of the path, as ACMM+NESP/windows/colmap2mvsnet_acm.py
prepares it for the reference.

    python hpm-mvs_b200/colmap.py --dense_folder D --save_folder S
           [--max_d 192] [--interval_scale 1] [--model_ext .txt|.bin] [--png]

D holds images/ and sparse/{cameras,images,points3D}{.txt,.bin} (COLMAP's
documented text and binary layouts).  Written, as the reference's script
writes them (colmap2mvsnet_acm.py:304-451):
  cams/%08d_cam.txt  4x4 extrinsic and 3x3 intrinsic (Python's float repr),
                     then "depth_min interval depth_num depth_max" (%f);
                     the depth range is the 1st/99th percentile of the
                     image's observed points' depths, widened x0.75/x1.25
  pair.txt           per image the min(20, N-1) best views by shared 3D
                     points (integer scores); a pair whose 75th-percentile
                     triangulation angle is under 1 degree scores 0
  images/%08d.jpg    the images, renumbered in image-id order (--png: PNG
                     instead)
The view scores need no host pool: one pass over the 3D points' tracks
accumulates every pair at once.
"""
from __future__ import annotations

import argparse
import os
import shutil
import struct
from collections import defaultdict

import numpy as np

# COLMAP camera models: id -> (name, parameter names)
CAMERA_MODELS = {
    0: ("SIMPLE_PINHOLE", ["f", "cx", "cy"]),
    1: ("PINHOLE", ["fx", "fy", "cx", "cy"]),
    2: ("SIMPLE_RADIAL", ["f", "cx", "cy", "k"]),
    3: ("RADIAL", ["f", "cx", "cy", "k1", "k2"]),
    4: ("OPENCV", ["fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2"]),
    5: ("OPENCV_FISHEYE", ["fx", "fy", "cx", "cy", "k1", "k2", "k3", "k4"]),
    6: ("FULL_OPENCV", ["fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2", "k3", "k4", "k5", "k6"]),
    7: ("FOV", ["fx", "fy", "cx", "cy", "omega"]),
    8: ("SIMPLE_RADIAL_FISHEYE", ["f", "cx", "cy", "k"]),
    9: ("RADIAL_FISHEYE", ["f", "cx", "cy", "k1", "k2"]),
    10: ("THIN_PRISM_FISHEYE", ["fx", "fy", "cx", "cy", "k1", "k2", "p1", "p2", "k3", "k4", "sx1", "sy1"]),
}
PARAMS_BY_NAME = {name: params for name, params in CAMERA_MODELS.values()}


class Model:
    """cameras: id -> (model name, width, height, params);
    images: id -> (qvec, tvec, camera id, name, point3D ids);
    points: id -> xyz."""

    def __init__(self):
        self.cameras, self.images, self.points = {}, {}, {}


def _lines(path):
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line and not line.startswith("#"):
                yield line


def read_text_model(folder: str) -> Model:
    m = Model()
    for line in _lines(os.path.join(folder, "cameras.txt")):
        e = line.split()
        m.cameras[int(e[0])] = (e[1], int(e[2]), int(e[3]), np.array([float(x) for x in e[4:]]))
    with open(os.path.join(folder, "images.txt")) as f:
        rows = [ln.strip() for ln in f if not ln.startswith("#")]
    # an image takes two lines; the second (observations) may be empty
    for k in range(0, len(rows) - 1, 2):
        e = rows[k].split()
        if not e:
            continue
        obs = rows[k + 1].split()
        ids = np.array([int(x) for x in obs[2::3]], dtype=np.int64)
        m.images[int(e[0])] = (np.array([float(x) for x in e[1:5]]), np.array([float(x) for x in e[5:8]]), int(e[8]),
                               e[9], ids)
    for line in _lines(os.path.join(folder, "points3D.txt")):
        e = line.split()
        m.points[int(e[0])] = np.array([float(x) for x in e[1:4]])
    return m


def read_binary_model(folder: str) -> Model:
    m = Model()
    with open(os.path.join(folder, "cameras.bin"), "rb") as f:
        (n,) = struct.unpack("<Q", f.read(8))
        for _ in range(n):
            cid, model_id, w, h = struct.unpack("<iiQQ", f.read(24))
            name, params = CAMERA_MODELS[model_id]
            m.cameras[cid] = (name, w, h, np.array(struct.unpack("<" + "d" * len(params), f.read(8 * len(params)))))
    with open(os.path.join(folder, "images.bin"), "rb") as f:
        (n,) = struct.unpack("<Q", f.read(8))
        for _ in range(n):
            v = struct.unpack("<idddddddi", f.read(64))
            name = b""
            c = f.read(1)
            while c != b"\x00":
                name += c
                c = f.read(1)
            (n2,) = struct.unpack("<Q", f.read(8))
            obs = struct.unpack("<" + "ddq" * n2, f.read(24 * n2))
            m.images[v[0]] = (np.array(v[1:5]), np.array(v[5:8]), v[8], name.decode("utf-8"),
                              np.array(obs[2::3], dtype=np.int64))
    with open(os.path.join(folder, "points3D.bin"), "rb") as f:
        (n,) = struct.unpack("<Q", f.read(8))
        for _ in range(n):
            v = struct.unpack("<QdddBBBd", f.read(43))
            (tl,) = struct.unpack("<Q", f.read(8))
            f.read(8 * tl)
            m.points[v[0]] = np.array(v[1:4])
    return m


def quat_to_rot(q) -> np.ndarray:
    """Rotation of the unit quaternion (w, x, y, z), COLMAP's convention."""
    w, x, y, z = q
    return np.array([[1 - 2 * y ** 2 - 2 * z ** 2, 2 * x * y - 2 * w * z, 2 * z * x + 2 * w * y],
                     [2 * x * y + 2 * w * z, 1 - 2 * x ** 2 - 2 * z ** 2, 2 * y * z - 2 * w * x],
                     [2 * z * x - 2 * w * y, 2 * y * z + 2 * w * x, 1 - 2 * x ** 2 - 2 * y ** 2]])


def intrinsic(camera) -> np.ndarray:
    name, _, _, params = camera
    p = dict(zip(PARAMS_BY_NAME[name], params))
    fx, fy = (p["f"], p["f"]) if "f" in p else (p["fx"], p["fy"])
    return np.array([[fx, 0, p["cx"]], [0, fy, p["cy"]], [0, 0, 1]])


def depth_range(K, E, xyzs, max_d, interval_scale):
    """(depth_min, interval, depth_num, depth_max) of one image."""
    zs = sorted(float((E @ np.array([x[0], x[1], x[2], 1.0]))[2]) for x in xyzs)
    dmin = zs[int(len(zs) * 0.01)] * 0.75
    dmax = zs[int(len(zs) * 0.99)] * 1.25
    if max_d == 0:  # one inverse-depth step per pixel at depth_min
        R, t = E[:3, :3], E[:3, 3]
        P1 = np.linalg.inv(R) @ (np.linalg.inv(K) @ [K[0, 2], K[1, 2], 1] * dmin - t)
        P2 = np.linalg.inv(R) @ (np.linalg.inv(K) @ [K[0, 2] + 1, K[1, 2], 1] * dmin - t)
        num = (1 / dmin - 1 / dmax) / (1 / dmin - 1 / (dmin + np.linalg.norm(P2 - P1)))
    else:
        num = max_d
    return dmin, (dmax - dmin) / (num - 1) / interval_scale, num, dmax


def view_scores(point_ids, centers, points) -> np.ndarray:
    """Pair scores from the images' observation lists: for i < j, the number
    of i's observations (repeats counted) whose 3D point j also observes;
    0 when the 75th-percentile triangulation angle of those observations is
    under 1 degree.  Symmetric."""
    n = len(point_ids)
    # point -> {image: observation count}
    tracks = defaultdict(dict)
    for i, ids in enumerate(point_ids):
        for pid in ids:
            if pid != -1:
                tracks[int(pid)][i] = tracks[int(pid)].get(i, 0) + 1
    counts = np.zeros((n, n))
    angles = defaultdict(list)
    for pid, obs in tracks.items():
        imgs = sorted(obs)
        if len(imgs) < 2:
            continue
        p = points[pid]
        for a in range(len(imgs)):
            i = imgs[a]
            di = centers[i] - p
            ni = np.linalg.norm(di)
            for b in range(a + 1, len(imgs)):
                j = imgs[b]
                dj = centers[j] - p
                theta = (180 / np.pi) * np.arccos(np.dot(di, dj) / ni / np.linalg.norm(dj))
                c = obs[i]
                counts[i, j] += c
                angles[(i, j)].extend([theta] * c)
    score = np.zeros((n, n))
    for (i, j), th in angles.items():
        s = counts[i, j]
        if sorted(th)[int(len(th) * 0.75)] < 1:
            s = 0.0
        score[i, j] = score[j, i] = s
    return score


def convert(dense_folder, save_folder, max_d=192, interval_scale=1.0, model_ext=".txt", png=False):
    model_dir = os.path.join(dense_folder, "sparse")
    m = read_text_model(model_dir) if model_ext == ".txt" else read_binary_model(model_dir)
    ids = sorted(m.images)
    n = len(ids)
    Ks, Es, centers, point_ids = [], [], [], []
    for iid in ids:
        q, t, cid, _, pids = m.images[iid]
        E = np.zeros((4, 4))
        E[:3, :3] = quat_to_rot(q)
        E[:3, 3] = t
        E[3, 3] = 1
        Es.append(E)
        Ks.append(intrinsic(m.cameras[cid]))
        centers.append(-(E[:3, :3].T @ E[:3, 3:4])[:, 0])
        point_ids.append(pids)
    ranges = [depth_range(Ks[i], Es[i], [m.points[p] for p in point_ids[i] if p != -1], max_d, interval_scale)
              for i in range(n)]
    score = view_scores(point_ids, centers, m.points)
    keep = min(20, n - 1)
    cam_dir, img_dir = os.path.join(save_folder, "cams"), os.path.join(save_folder, "images")
    for d in (cam_dir, img_dir):
        if os.path.exists(d):
            shutil.rmtree(d)
        os.makedirs(d)
    for i in range(n):
        with open(os.path.join(cam_dir, f"{i:08d}_cam.txt"), "w") as f:
            f.write("extrinsic\n")
            for r in range(4):
                f.write("".join(str(Es[i][r, k]) + " " for k in range(4)) + "\n")
            f.write("\nintrinsic\n")
            for r in range(3):
                f.write("".join(str(Ks[i][r, k]) + " " for k in range(3)) + "\n")
            f.write("\n%f %f %f %f\n" % ranges[i])
    with open(os.path.join(save_folder, "pair.txt"), "w") as f:
        f.write("%d\n" % n)
        for i in range(n):
            # best views by score; ties keep NumPy's argsort order
            order = np.argsort(score[i])[::-1][:keep]
            f.write("%d\n%d " % (i, len(order)) + "".join("%d %d " % (k, score[i, k]) for k in order) + "\n")
    for i, iid in enumerate(ids):
        src = os.path.join(dense_folder, "images", m.images[iid][3])
        ext = ".png" if png else ".jpg"
        dst = os.path.join(img_dir, f"{i:08d}{ext}")
        if src.lower().endswith(ext):
            shutil.copyfile(src, dst)
        else:
            import cv2

            cv2.imwrite(dst, cv2.imread(src))
    return n


def main(argv=None):
    ap = argparse.ArgumentParser(description="COLMAP sparse model to an HPM-MVS dense folder")
    ap.add_argument("--dense_folder", required=True)
    ap.add_argument("--save_folder", required=True)
    ap.add_argument("--max_d", type=int, default=192)
    ap.add_argument("--interval_scale", type=float, default=1)
    ap.add_argument("--model_ext", default=".txt", choices=[".txt", ".bin"])
    ap.add_argument("--png", action="store_true", help="write images/ as PNG instead of JPEG")
    a = ap.parse_args(argv)
    convert(a.dense_folder, a.save_folder, a.max_d, a.interval_scale, a.model_ext, a.png)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

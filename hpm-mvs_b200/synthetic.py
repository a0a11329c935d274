"""Seeded synthetic multi-view scenes with known geometry.

No public MVS dataset travels with this project, so benchmarks and parity runs
use procedurally rendered scenes with the shapes, sizes and value
distributions of the benchmark configurations:

* textures: band-limited 1/f^2 noise (mean 128, std 40) with low-texture
  patches (std 2) covering a chosen fraction of every surface;
* shading: Lambertian under one directional light plus ambient;
* pixel noise: Gaussian, sigma 2, then rounded to uint8 gray;
* cameras: pinhole fx = fy (512 at 640 px width, scaled with width),
  principal point at the image centre, placed on a 5 m arc around the scene
  centre, 8 degrees apart, all looking at the scene centre;
* scene: one backdrop plane, random planar rectangles and spheres at 2-8 m.

The camera model is the reference's (HPM-MVS/main.h:44-52): X_cam = R X + t,
x = K X_cam, pixel (x, y) is the sample at integer coordinates.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

CAMERA_DTYPE = np.dtype(
    [("K", "<f4", 9), ("R", "<f4", 9), ("t", "<f4", 3), ("height", "<i4"), ("width", "<i4"),
     ("depth_min", "<f4"), ("depth_max", "<f4")]
)


@dataclasses.dataclass
class Scene:
    images: list            # uint8 [H, W] per view
    cams: np.ndarray        # CAMERA_DTYPE [N]
    gt_depth: list          # float32 [H, W] per view (0 = no surface)
    gt_normal: list         # float32 [H, W, 3] world-frame normals per view
    pairs: list             # [(ref_id, [src ids ranked by angle], [scores])]
    depth_min: float        # cam-file depth range (before the x0.6 / x1.2 widening)
    depth_max: float


def _noise_texture(rng: np.random.Generator, size: int, std: float = 40.0, mean: float = 128.0) -> np.ndarray:
    """Periodic band-limited noise with a 1/f^2 power spectrum."""
    fy = np.fft.fftfreq(size)[:, None]
    fx = np.fft.rfftfreq(size)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    amp = 1.0 / np.maximum(f, 1.0 / size)
    amp[f > 0.25] = 0.0  # band limit: nothing finer than 4 texels
    amp[0, 0] = 0.0
    phase = rng.uniform(0, 2 * np.pi, amp.shape)
    spec = amp * np.exp(1j * phase)
    tex = np.fft.irfft2(spec, s=(size, size))
    tex = (tex - tex.mean()) / (tex.std() + 1e-12)
    return (mean + std * tex).astype(np.float32)


def _flat_mask(rng: np.random.Generator, size: int, frac: float) -> np.ndarray:
    """Blobby low-frequency mask covering about `frac` of the texture."""
    if frac <= 0:
        return np.zeros((size, size), bool)
    fy = np.fft.fftfreq(size)[:, None]
    fx = np.fft.rfftfreq(size)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    amp = np.where((f > 0) & (f < 4.0 / size), 1.0, 0.0)
    phase = rng.uniform(0, 2 * np.pi, amp.shape)
    field = np.fft.irfft2(amp * np.exp(1j * phase), s=(size, size))
    return field > np.quantile(field, 1.0 - frac)


def _bilinear_wrap(tex: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    n = tex.shape[0]
    u0 = np.floor(u)
    v0 = np.floor(v)
    a = (u - u0).astype(np.float32)
    b = (v - v0).astype(np.float32)
    x0 = u0.astype(np.int64) % n
    y0 = v0.astype(np.int64) % n
    x1 = (x0 + 1) % n
    y1 = (y0 + 1) % n
    return ((1 - a) * (1 - b) * tex[y0, x0] + a * (1 - b) * tex[y0, x1] + (1 - a) * b * tex[y1, x0]
            + a * b * tex[y1, x1])


def look_at(pos: np.ndarray, target: np.ndarray):
    z = target - pos
    z = z / np.linalg.norm(z)
    x = np.cross(np.array([0.0, 1.0, 0.0]), z)
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z])
    t = -R @ pos
    return R, t


def _random_unit_facing(rng, max_tilt_deg):
    """Unit normal within max_tilt of -z (facing cameras that look along +z)."""
    tilt = math.radians(rng.uniform(0, max_tilt_deg))
    az = rng.uniform(0, 2 * math.pi)
    return np.array([math.sin(tilt) * math.cos(az), math.sin(tilt) * math.sin(az), -math.cos(tilt)])


def _basis(n):
    a = np.array([0.0, 1.0, 0.0]) if abs(n[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    u = np.cross(a, n)
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    return u, v


def make_scene(seed: int, width: int, height: int, n_views: int, *, n_planes: int = 6, n_spheres: int = 0,
               low_texture: float = 0.25, depth_range=(2.0, 8.0), fx: float | None = None,
               arc_radius: float = 5.0, arc_step_deg: float = 8.0, noise_sigma: float = 2.0,
               n_sources: int | None = None, texel_m: float | None = None, tex_size: int = 1024,
               sizes=None) -> Scene:
    """sizes: per-view (width, height) for scenes of uneven resolution; each
    view's focal length scales with its width (fx given for `width`), so all
    views see the same field of view."""
    rng = np.random.default_rng(seed)
    sizes = [(width, height)] * n_views if sizes is None else [(int(w), int(h)) for w, h in sizes]
    assert len(sizes) == n_views
    if fx is None:
        fx = 512.0 * width / 640.0
    dmin, dmax = depth_range
    center = np.array([0.0, 0.0, 0.5 * (dmin + dmax)])
    if texel_m is None:
        # about 1.6 texels per pixel at the scene centre, whatever the resolution
        texel_m = 0.6 * center[2] / fx

    # ---- objects -------------------------------------------------------
    objs = []
    light = np.array([0.3, -0.5, 0.8])
    light /= np.linalg.norm(light)
    for k in range(n_planes):
        n = _random_unit_facing(rng, 25.0 if k == 0 else 55.0)
        if k == 0:
            p0 = np.array([0.0, 0.0, dmax - 0.6])
            half = (1e3, 1e3)
        else:
            z = rng.uniform(dmin + 0.3, dmax - 1.2)
            ext = np.tan(np.radians(20)) * z
            p0 = np.array([rng.uniform(-ext, ext), rng.uniform(-0.7 * ext, 0.7 * ext), z])
            half = (rng.uniform(0.3, 0.9) * z * 0.25, rng.uniform(0.3, 0.9) * z * 0.25)
        u, v = _basis(n)
        objs.append(dict(kind="plane", n=n, p0=p0, u=u, v=v, half=half,
                         tex=_noise_texture(rng, tex_size), flat=_flat_mask(rng, tex_size, low_texture),
                         flat_level=rng.uniform(70, 190)))
    for _ in range(n_spheres):
        z = rng.uniform(dmin + 0.8, dmax - 1.5)
        ext = np.tan(np.radians(18)) * z
        c = np.array([rng.uniform(-ext, ext), rng.uniform(-0.7 * ext, 0.7 * ext), z])
        r = rng.uniform(0.25, 0.7)
        objs.append(dict(kind="sphere", c=c, r=r, tex=_noise_texture(rng, tex_size),
                         flat=_flat_mask(rng, tex_size, low_texture), flat_level=rng.uniform(70, 190)))
    for o in objs:
        o["tex"] = np.where(o["flat"], o["flat_level"], o["tex"]).astype(np.float32)
        # fine std-2 noise on the flat patches (low texture, not textureless)
        o["tex"] += np.where(o["flat"], rng.normal(0, 2.0, o["tex"].shape), 0).astype(np.float32)

    # ---- cameras -------------------------------------------------------
    Ks = [np.array([[fx * w / width, 0, w / 2.0], [0, fx * w / width, h / 2.0], [0, 0, 1.0]]) for w, h in sizes]
    cams = np.zeros(n_views, CAMERA_DTYPE)
    angles = [(i - (n_views - 1) / 2.0) * math.radians(arc_step_deg) for i in range(n_views)]
    for i, a in enumerate(angles):
        pos = center + arc_radius * np.array([math.sin(a), 0.0, -math.cos(a)])
        R, t = look_at(pos, center)
        cams[i]["K"] = Ks[i].reshape(-1)
        cams[i]["R"] = R.reshape(-1)
        cams[i]["t"] = t
        cams[i]["width"], cams[i]["height"] = sizes[i]
        cams[i]["depth_min"] = dmin
        cams[i]["depth_max"] = dmax

    # ---- render --------------------------------------------------------
    images, gt_depth, gt_normal = [], [], []
    for i in range(n_views):
        width, height = sizes[i]
        ys, xs = np.mgrid[0:height, 0:width].astype(np.float64)
        Kinv = np.linalg.inv(Ks[i])
        R = cams[i]["R"].reshape(3, 3).astype(np.float64)
        t = cams[i]["t"].astype(np.float64)
        C = -R.T @ t
        dcam = np.stack([xs, ys, np.ones_like(xs)], -1) @ Kinv.T  # z = 1
        dw = dcam @ R  # world directions (R^T d), camera z-component 1
        best_t = np.full((height, width), np.inf)
        col = np.zeros((height, width), np.float32)
        nrm = np.zeros((height, width, 3), np.float32)
        for o in objs:
            if o["kind"] == "plane":
                n = o["n"]
                denom = dw @ n
                with np.errstate(divide="ignore", invalid="ignore"):
                    tt = (o["p0"] - C) @ n / denom
                hit = C + tt[..., None] * dw
                rel = hit - o["p0"]
                su, sv = rel @ o["u"], rel @ o["v"]
                ok = (tt > 0.05) & (np.abs(su) <= o["half"][0]) & (np.abs(sv) <= o["half"][1]) & (tt < best_t)
                nn = np.broadcast_to(n, hit.shape)
            else:
                oc = C - o["c"]
                a = np.einsum("ijk,ijk->ij", dw, dw)
                b = 2.0 * (dw @ oc)
                cc = oc @ oc - o["r"] ** 2
                disc = b * b - 4 * a * cc
                with np.errstate(invalid="ignore"):
                    tt = (-b - np.sqrt(np.maximum(disc, 0))) / (2 * a)
                hit = C + tt[..., None] * dw
                nn = (hit - o["c"]) / o["r"]
                lat = np.arcsin(np.clip(nn[..., 1], -1, 1))
                lon = np.arctan2(nn[..., 0], -nn[..., 2])
                su = lon * o["r"]
                sv = lat * o["r"]
                ok = (disc > 0) & (tt > 0.05) & (tt < best_t)
            if not ok.any():
                continue
            tex = _bilinear_wrap(o["tex"], su[ok] / texel_m, sv[ok] / texel_m)
            nk = nn[ok]
            facing = np.einsum("ij,ij->i", nk, dw[ok]) > 0
            nk = np.where(facing[:, None], -nk, nk)
            shade = 0.45 + 0.55 * np.clip(-(nk @ light), 0.0, 1.0)
            col[ok] = tex * shade / 0.8
            nrm[ok] = nk
            best_t[ok] = tt[ok]
        depth = np.where(np.isfinite(best_t), best_t, 0.0).astype(np.float32)
        img = col + rng.normal(0.0, noise_sigma, col.shape)
        images.append(np.clip(np.rint(img), 0, 255).astype(np.uint8))
        gt_depth.append(depth)
        gt_normal.append(nrm)

    # ---- view selection (pair.txt) -------------------------------------
    ns = n_views - 1 if n_sources is None else min(n_sources, n_views - 1)
    pairs = []
    for i in range(n_views):
        others = sorted((j for j in range(n_views) if j != i), key=lambda j: (abs(angles[j] - angles[i]), j))[:ns]
        scores = [round(100.0 / (1.0 + math.degrees(abs(angles[j] - angles[i]))), 3) for j in others]
        pairs.append((i, others, scores))
    return Scene(images, cams, gt_depth, gt_normal, pairs, dmin, dmax)


def view_set(scene: Scene, ref_id: int):
    """(float images, cameras) of one problem in the reference's order: the
    reference view first, then its sources (HPM.cpp:482-522)."""
    _, srcs, _ = scene.pairs[ref_id]
    ids = [ref_id] + list(srcs)
    images = [scene.images[i].astype(np.float32) for i in ids]
    cams = scene.cams[ids].copy()
    return images, cams


def write_dense_folder(scene: Scene, folder: str, image_ext: str = ".png") -> None:
    """images/%08d<ext>, cams/%08d_cam.txt and pair.txt in the reference's
    layout (main.cpp:4-33, HPM.cpp:160-185).  PNG keeps the pixels exact."""
    import os

    import cv2

    os.makedirs(os.path.join(folder, "images"), exist_ok=True)
    os.makedirs(os.path.join(folder, "cams"), exist_ok=True)
    for i, img in enumerate(scene.images):
        cv2.imwrite(os.path.join(folder, "images", f"{i:08d}{image_ext}"), img)
        c = scene.cams[i]
        R = c["R"].reshape(3, 3)
        with open(os.path.join(folder, "cams", f"{i:08d}_cam.txt"), "w") as f:
            f.write("extrinsic\n")
            for r in range(3):
                f.write(" ".join(f"{R[r, k]:.9g}" for k in range(3)) + f" {c['t'][r]:.9g}\n")
            f.write("0 0 0 1\n\nintrinsic\n")
            K = c["K"].reshape(3, 3)
            for r in range(3):
                f.write(" ".join(f"{K[r, k]:.9g}" for k in range(3)) + "\n")
            interval = (scene.depth_max - scene.depth_min) / 192.0
            f.write(f"\n{scene.depth_min:.9g} {interval:.9g} 192 {scene.depth_max:.9g}\n")
    with open(os.path.join(folder, "pair.txt"), "w") as f:
        f.write(f"{len(scene.pairs)}\n")
        for ref_id, srcs, scores in scene.pairs:
            f.write(f"{ref_id}\n{len(srcs)} " + " ".join(f"{s} {sc}" for s, sc in zip(srcs, scores)) + "\n")


def gt_planes_ref_frame(scene: Scene, ref_id: int) -> np.ndarray:
    """Ground-truth hypotheses (n_ref, dist) of the reference view in the
    PatchMatch parametrisation (ref-camera normal, dist = -n . X)."""
    cam = scene.cams[ref_id]
    R = cam["R"].reshape(3, 3).astype(np.float64)
    K = cam["K"].reshape(3, 3).astype(np.float64)
    d = scene.gt_depth[ref_id].astype(np.float64)
    nw = scene.gt_normal[ref_id].astype(np.float64)
    h, w = d.shape
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)
    X = np.stack([d * (xs - K[0, 2]) / K[0, 0], d * (ys - K[1, 2]) / K[1, 1], d], -1)
    n = nw @ R.T
    dist = -(n * X).sum(-1)
    out = np.concatenate([n, dist[..., None]], -1).astype(np.float32)
    return out


def depth_accuracy(depth: np.ndarray, gt: np.ndarray, rel: float = 0.01) -> float:
    """Fraction of pixels with a ground-truth surface whose relative depth
    error is below `rel` (the benchmark's %px metric)."""
    m = gt > 0
    if not m.any():
        return 0.0
    err = np.abs(depth[m] - gt[m]) / gt[m]
    return float((err < rel).mean())


def normal_error_deg(normal: np.ndarray, gt: np.ndarray, gt_depth: np.ndarray) -> float:
    """Median angle in degrees between estimated and ground-truth normals."""
    m = gt_depth > 0
    a = normal[m].astype(np.float64)
    b = gt[m].astype(np.float64)
    na = np.linalg.norm(a, axis=-1)
    ok = na > 0
    cos = (a[ok] * b[ok]).sum(-1) / na[ok]
    return float(np.degrees(np.median(np.arccos(np.clip(cos, -1, 1))))) if ok.any() else 180.0


def _read_dmb(path):
    """A .dmb map (int32 type, h, w, channels; then float32) as [h, w] or [h, w, c]."""
    raw = np.fromfile(path, np.uint8)
    _, h, w, nb = np.frombuffer(raw[:16].tobytes(), np.int32)
    a = np.frombuffer(raw[16:].tobytes(), np.float32).reshape(h, w, nb)
    return a[..., 0] if nb == 1 else a


def main(argv=None) -> None:
    """Write a seeded scene as a dense folder (images/, cams/, pair.txt) for
    hpm_mvs or the reference's executable, with the ground-truth depth maps
    as gt/%08d.dmb."""
    import argparse
    import os

    ap = argparse.ArgumentParser(description="seeded synthetic scene as an HPM-MVS dense folder")
    ap.add_argument("folder")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--views", type=int, default=11)
    ap.add_argument("--size", default="1600x1200", help="WxH")
    ap.add_argument("--sources", type=int, default=10)
    ap.add_argument("--planes", type=int, default=20)
    ap.add_argument("--spheres", type=int, default=5)
    ap.add_argument("--low-texture", type=float, default=0.4)
    ap.add_argument("--ext", default=".jpg", choices=[".jpg", ".png", ".pgm"])
    ap.add_argument("--score", action="store_true",
                    help="instead of writing, score FOLDER/HPM/2333_%%08d/depths_geom.dmb against FOLDER/gt")
    a = ap.parse_args(argv)
    if a.score:
        accs = []
        for name in sorted(os.listdir(os.path.join(a.folder, "gt"))):
            v = int(name.split(".")[0])
            res = os.path.join(a.folder, "HPM", f"2333_{v:08d}", "depths_geom.dmb")
            if os.path.exists(res):
                accs.append(depth_accuracy(_read_dmb(res), _read_dmb(os.path.join(a.folder, "gt", name))))
        print(f"views {len(accs)} px_relerr_lt_1pct {np.mean(accs) if accs else float('nan'):.4f}")
        return
    w, h = (int(x) for x in a.size.lower().split("x"))
    sc = make_scene(a.seed, w, h, a.views, n_planes=a.planes, n_spheres=a.spheres, low_texture=a.low_texture,
                    n_sources=a.sources)
    write_dense_folder(sc, a.folder, a.ext)
    os.makedirs(os.path.join(a.folder, "gt"), exist_ok=True)
    for i, d in enumerate(sc.gt_depth):
        with open(os.path.join(a.folder, "gt", f"{i:08d}.dmb"), "wb") as f:  # .dmb: type 1, h, w, 1 channel
            f.write(np.array([1, d.shape[0], d.shape[1], 1], np.int32).tobytes())
            f.write(np.ascontiguousarray(d, np.float32).tobytes())
    print(f"wrote {a.views} views of {w}x{h} to {a.folder}")


if __name__ == "__main__":
    main()

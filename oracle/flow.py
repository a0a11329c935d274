"""ProcessProblem (HPM-MVS/main.cpp:35-499) restated on the CPU for small
images, from the oracle's kernels (liboracle.so) and the OpenCV calls the
reference makes (cv2.resize INTER_LINEAR, cv2.Subdiv2D).

TEST INFRASTRUCTURE ONLY: the checker of hpm_process_problem and
hpm_prior_level.

The reference's kd-tree KNN (PCL) is the oracle's exact brute-force 6-NN
(ties to the lower support-point index); the Delaunay is OpenCV's own.
"""
from __future__ import annotations

import numpy as np

import oracle as orc


def scale_levels(w: int, h: int) -> int:
    """ComputingMultiScaleSettings, HPM.cpp:851-860."""
    m, k = max(w, h), 0
    while m > 1000:
        m //= 2
        k += 1
    return k


def cv_triangles(pts: np.ndarray, w: int, h: int) -> np.ndarray:
    """DelaunayTriangulation (HPM.cpp:787-809) with the inside filter of
    main.cpp:97, through OpenCV's Subdiv2D."""
    import cv2

    if len(pts) == 0:
        return np.zeros((0, 6), np.int32)
    sd = cv2.Subdiv2D((0, 0, w, h))
    for x, y in pts:
        sd.insert((float(x), float(y)))
    t = sd.getTriangleList().astype(np.int64).astype(np.int32)  # (int) casts, HPM.cpp:803-805
    keep = ((t[:, 0::2] >= 0) & (t[:, 0::2] < w) & (t[:, 1::2] >= 0) & (t[:, 1::2] < h)).all(1)
    return t[keep]


def level_masks(cam, depth, cost, factor, dmin, dmax, triangles=None):
    """Support points, triangles, raster, planes and KNN of one level: the
    reference's mask (float), triangle planes and KNN planes."""
    h, w = depth.shape
    pts = orc.support_points(cost)
    tris = cv_triangles(pts, w, h) if triangles is None else triangles(pts, w, h)
    mask, kept = orc.raster_triangles(tris, w, h)
    tri_planes = np.array([orc.plane_from_triangle(cam, depth, t, factor) for t in kept], np.float32).reshape(-1, 4)
    knn_planes, mask = orc.knn_supplement(cam, pts, depth, factor, dmin, dmax, mask)
    return mask, tri_planes, knn_planes


def prior_level(cam, level, depth, normal, cost, guide, dmin, dmax, triangles=None, jbu=None):
    """Prior planes (ref frame), masks and (full scale) prior depth of one
    pyramid level from full-resolution maps (main.cpp:78-478).  jbu: the
    joint bilateral upsampler (default: the oracle's)."""
    import cv2

    H, W = depth.shape
    dmin, dmax = np.float32(dmin), np.float32(dmax)
    if level in (0, 1):
        f = 0.25 if level == 0 else 0.5
        ws, hs = int(round(W * f)), int(round(H * f))
        d_s = cv2.resize(depth, (ws, hs), interpolation=cv2.INTER_LINEAR)
        c_s = cv2.resize(cost, (ws, hs), interpolation=cv2.INTER_LINEAR)
        mask, tri_planes, knn_planes = level_masks(cam, d_s, c_s, f, dmin, dmax, triangles)
        pd, pn = orc.prior_coarse(cam, mask, tri_planes, knn_planes, f, dmin, dmax)
        ud, un = (jbu or orc.jbu)(guide, pd, pn)
        prior, pmask = orc.prior_reload(cam, ud, un, dmin, dmax)
        return prior, pmask, np.zeros((H, W), np.float32)
    mask, tri_planes, knn_planes = level_masks(cam, depth, cost, 1.0, dmin, dmax, triangles)
    return orc.prior_full(cam, mask, tri_planes, knn_planes, dmin, dmax)


def _oracle_pass(images, cams, **kw):
    return orc.run_patchmatch(images, cams, **kw)


def _reference_pass(images, cams, *, salt=0, views=None, **kw):
    """HPM::RunPatchMatch of the reference's own kernels (oracle/_ref); the
    reference draws its random streams from clock64(), so salt and the
    selected-view map do not apply."""
    p, c = orc.ref_run_patchmatch(images, cams, **kw)
    return p, c, None


def process_problem(images, cams, *, seed=0, planar_prior=True, geom=False, multi_geometry=False, planes=None,
                    costs=None, depth_maps=None, guide=None, pyramid_levels=-1, backend="oracle"):
    """Returns (depth, world normal, cost, prior depth) of the reference view.
    backend "oracle": the oracle's CPU passes and JBU; "reference": the
    reference's own CUDA kernels (oracle/_ref) for the passes and the JBU,
    with the host stages above."""
    ref = backend == "reference"
    run = _reference_pass if ref else _oracle_pass
    jbu = orc.ref_jbu if ref else orc.jbu
    cam = cams[0]
    H, W = images[0].shape
    dmin = np.float32(cam["depth_min"]) * np.float32(0.6)
    dmax = np.float32(cam["depth_max"]) * np.float32(1.2)
    salt = 0
    if geom:
        extra = {"multi_geometry": multi_geometry} if ref else {}
        p, c, v = run(images, cams, depth_min=dmin, depth_max=dmax, seed=seed, salt=salt, geom=True,
                      planes=planes, costs=costs, depth_maps=depth_maps, **extra)
        return p[..., 3].copy(), p[..., :3].copy(), c, np.zeros((H, W), np.float32)
    p, c, v = run(images, cams, depth_min=dmin, depth_max=dmax, seed=seed, salt=salt)
    prior_depth = np.zeros((H, W), np.float32)
    if planar_prior:
        guide = images[0] if guide is None else guide
        k = pyramid_levels if pyramid_levels >= 0 else scale_levels(W, H)
        for i in range(2 - k, 3):
            prior, pmask, pd = prior_level(cam, i, p[..., 3].copy(), p[..., :3].copy(), c, guide, dmin, dmax,
                                           jbu=jbu)
            if i not in (0, 1):
                prior_depth = pd
            salt += 1
            p, c, v = run(images, cams, depth_min=dmin, depth_max=dmax, seed=seed + (salt if ref else 0), salt=salt,
                          prior=True, planes=p, costs=c, views=v, prior_planes=prior, masks=pmask)
    return p[..., 3].copy(), p[..., :3].copy(), c, prior_depth

"""The ACMM+NESP variant's main() (ACMM+NESP/windows/main.cpp:299-384)
restated on the CPU for small images, from the oracle's kernels
(liboracle.so, variant 1) and the OpenCV resize the reference calls.

TEST INFRASTRUCTURE ONLY: the checker of hpm_run_scene_acmm.

The flow: every problem's images are scaled down until their longer side is
at most `size_bound` (1000 in ComputeMultiScaleSettings, main.cpp:35-71; a
parameter here so that small test scenes get several scales).  At the
coarsest scale a plain pass and the geometric iterations run for every
problem; at each finer scale the last geometric depth map is upsampled by
the joint bilateral filter (main.cpp:126-152, RunJBU in ACMM.cpp:804-855),
a hierarchy pass starts from it (ACMM.cpp:663-719, ACMM.cu:521-604) and
the geometric iterations follow.  Problem p must have reference view p, as
the reference indexes problems by source image id (ACMM.cpp:490).
"""
from __future__ import annotations

import numpy as np

import oracle as orc

MAX_IMAGE_SIZE = 3200  # PatchMatchParams::max_image_size (ACMM.h:34)


def multiscale_settings(shapes, size_bound=1000):
    """ComputeMultiScaleSettings (main.cpp:35-71): per problem the capped
    longer side and the number of halvings down to size_bound; returns
    (max_sizes, downscales, max_downscale)."""
    max_sizes, ks = [], []
    for h, w in shapes:
        m = min(max(h, w), MAX_IMAGE_SIZE)
        max_sizes.append(m)
        k = 0
        while m > size_bound:
            m //= 2
            k += 1
        ks.append(k)
    return max_sizes, ks, max(ks)


def scaled_view(image, cam, cur):
    """InuputInitialization's scaling (ACMM.cpp:489-516): the image resized
    by cv::resize INTER_LINEAR to fit cur x cur, the camera's K scaled with
    it; views that already fit are kept."""
    import cv2

    h, w = image.shape
    cam = cam.copy()
    if w <= cur and h <= cur:
        return image, cam
    f32 = np.float32
    factor = min(f32(cur) / f32(w), f32(cur) / f32(h))
    # std::round of a float: halves away from zero
    nw, nh = int(np.floor(np.float64(f32(w) * factor) + 0.5)), int(np.floor(np.float64(f32(h) * factor) + 0.5))
    sx, sy = f32(nw) / f32(w), f32(nh) / f32(h)
    out = cv2.resize(image, (nw, nh), interpolation=cv2.INTER_LINEAR)
    K = cam["K"].astype(np.float32)
    K[0] *= sx
    K[2] *= sx
    K[4] *= sy
    K[5] *= sy
    cam["K"] = K
    cam["width"], cam["height"] = nw, nh
    return out, cam


def run_scene(images, cams, problems, *, seed=0, size_bound=1000, geom_iterations=2, half_steps_plain=6,
              half_steps_geom=4, run=None):
    """Returns per-view (depth, world normal, cost) at the final scale and
    the per-scale sizes.  images: float32 [H, W] per view at full size;
    cams: CAMERA_DTYPE array; problems: [(ref, [sources])] with ref == index.
    run: the pass (default the oracle's, orc.run_patchmatch)."""
    run = run or orc.run_patchmatch
    n = len(problems)
    for p, (ref, _) in enumerate(problems):
        if ref != p:
            raise ValueError("problem p must have reference view p")
    max_sizes, nd, max_down = multiscale_settings([images[p].shape for p in range(n)], size_bound)
    nd = list(nd)
    cur = [0] * n
    # per-view maps of the reference's files: depths.dmb, depths_geom.dmb,
    # normals.dmb, costs.dmb
    depth, depth_geom, normal, cost = [None] * n, [None] * n, [None] * n, [None] * n
    pass_no = [0] * n

    def views_of(p):
        ids = [p] + list(problems[p][1])
        out = [scaled_view(images[v], cams[v], cur[v]) for v in ids]
        return ids, [o[0].astype(np.float32) for o in out], np.array([o[1] for o in out], dtype=orc.CAMERA_DTYPE)

    def finish(p, planes, c, geom):
        (depth_geom if geom else depth)[p] = planes[..., 3].copy()
        normal[p] = planes[..., :3].copy()
        cost[p] = c

    def one_pass(p, **kw):
        ids, imgs, vcams = views_of(p)
        dmin = np.float32(cams[p]["depth_min"]) * np.float32(0.6)
        dmax = np.float32(cams[p]["depth_max"]) * np.float32(1.2)
        s = seed + 7919 * p + pass_no[p]
        pass_no[p] += 1
        return ids, imgs, vcams, dict(depth_min=dmin, depth_max=dmax, seed=s, variant=1, **kw)

    def plain(p):
        ids, imgs, vcams, kw = one_pass(p)
        planes, c, _ = run(imgs, vcams, half_steps=half_steps_plain, **kw)
        finish(p, planes, c, False)

    def geometric(p, multi):
        ids, imgs, vcams, kw = one_pass(p)
        src = depth_geom if multi else depth
        dm = [src[v] for v in ids]
        planes = np.concatenate([normal[p], src[p][..., None]], -1)
        planes, c, _ = run(imgs, vcams, half_steps=half_steps_geom, geom=True, planes=planes, costs=cost[p],
                           depth_maps=dm, **kw)
        finish(p, planes, c, True)

    def upsample(p):
        """JointBilateralUpsampling (main.cpp:126-152): depths.dmb becomes
        the geometric depth map upsampled to the new scale, unless the
        integer scale is 1 (RunJBU returns early, ACMM.cpp:810-813)."""
        ids, imgs, vcams = views_of(p)
        guide = imgs[0]
        src = depth_geom[p]
        scale = max(guide.shape[0] // src.shape[0], guide.shape[1] // src.shape[1])
        if scale == 1:
            return
        d, _ = orc.jbu_at_scale(guide, src, np.zeros(src.shape + (3,), np.float32), scale)
        depth[p] = d

    def hierarchy(p):
        """CudaSpaceInitialization's hierarchy block (ACMM.cpp:663-719) and
        the pass: the normals of the last geometric pass, averaged with the
        JBU's weights at the new size (upsample; the reference compares the
        normal map's width with the image's rows, ACMM.cpp:682), the depth of
        depths.dmb."""
        ids, imgs, vcams, kw = one_pass(p)
        guide = imgs[0]
        H, W = guide.shape
        nh, nw = normal[p].shape[:2]
        up = nw != H or nh != W
        if up:
            scale = max(W // nw, H // nh)
            _, n_up = orc.jbu_at_scale(guide, cost[p], normal[p], scale)
        else:
            n_up = normal[p]
        planes = np.concatenate([n_up, depth[p][..., None]], -1).astype(np.float32)
        pre = np.zeros((H, W), np.float32)
        planes, c, _ = run(imgs, vcams, half_steps=half_steps_plain, planes=planes, hierarchy=1 if up else 2,
                           pre_costs=pre, **kw)
        finish(p, planes, c, False)

    sizes = []
    first = True
    while max_down >= 0:
        for p in range(n):
            if nd[p] >= 0:
                cur[p] = int(max_sizes[p] / 2.0 ** nd[p])
                nd[p] -= 1
        sizes.append(list(cur))
        if first:
            first = False
            for p in range(n):
                plain(p)
        else:
            for p in range(n):
                upsample(p)
            for p in range(n):
                hierarchy(p)
        for gi in range(geom_iterations):
            for p in range(n):
                geometric(p, gi > 0)
        max_down -= 1
    final = depth_geom if geom_iterations > 0 else depth
    return [final[p] for p in range(n)], [normal[p] for p in range(n)], [cost[p] for p in range(n)], sizes

"""ctypes binding of the CPU oracle (liboracle.so) and of the reference shim
(_ref/libhpm_ref.so, the reference's own HPM-MVS/HPM.cu compiled for sm_100a).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm use this module as the checker.  The product never
imports it.

Array conventions (match the reference's host buffers):
  images        list of float32 [H, W] arrays (gray values, HPM.cpp:492-495)
  cams          numpy structured array of CAMERA_DTYPE (HPM-MVS/main.h:44-52)
  planes        float32 [H, W, 4] = (nx, ny, nz, w)
  costs         float32 [H, W]
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhpm_ref.so")
ACMM_REF_SO = os.path.join(HERE, "_ref", "libacmm_ref.so")

CAMERA_DTYPE = np.dtype(
    [("K", "<f4", 9), ("R", "<f4", 9), ("t", "<f4", 3), ("height", "<i4"), ("width", "<i4"),
     ("depth_min", "<f4"), ("depth_max", "<f4")]
)
assert CAMERA_DTYPE.itemsize == 100


class OrRunOpts(ctypes.Structure):
    _fields_ = [("geom_consistency", ctypes.c_int), ("planar_prior", ctypes.c_int),
                ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float),
                ("seed", ctypes.c_uint64), ("salt", ctypes.c_uint32),
                ("half_steps", ctypes.c_int), ("finalize", ctypes.c_int),
                ("variant", ctypes.c_int), ("hierarchy", ctypes.c_int), ("pre_costs", ctypes.c_void_p)]


class RefRunOpts(ctypes.Structure):
    _fields_ = [("geom_consistency", ctypes.c_int), ("planar_prior", ctypes.c_int),
                ("multi_geometry", ctypes.c_int), ("depth_min", ctypes.c_float),
                ("depth_max", ctypes.c_float), ("seed", ctypes.c_ulonglong)]


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.or_tex2d.restype = ctypes.c_float
        _lib.or_philox_uniform.restype = ctypes.c_float
        _lib.or_philox_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_uint32]
        _lib.or_depth_from_plane.restype = ctypes.c_float
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
    return _ref


_acmm_ref = None


def acmm_ref_available() -> bool:
    return os.path.exists(ACMM_REF_SO)


def ref_acmm_hier_init(images, cams, planes, scaled):
    """The reference's own RandomInitialization of an ACMM+NESP hierarchy
    pass with upsample set (ACMM.cu:538-604, oracle/_ref/libacmm_ref.so on a
    GPU).  planes: [H, W, 4] as the host leaves them ((0, 0, 0, depth));
    scaled: [sh, sw, 4] (previous scale's world normal, cost).  Returns
    (planes, costs, pre_costs, selected views)."""
    global _acmm_ref
    if _acmm_ref is None:
        _acmm_ref = ctypes.CDLL(ACMM_REF_SO)
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    pl = np.ascontiguousarray(planes, dtype=np.float32)
    sc = np.ascontiguousarray(scaled, dtype=np.float32)
    cam0 = np.asarray(cams)[0]
    dmin = np.float32(cam0["depth_min"]) * np.float32(0.6)
    dmax = np.float32(cam0["depth_max"]) * np.float32(1.2)
    op = np.empty((h, w, 4), np.float32)
    oc = np.empty((h, w), np.float32)
    pre = np.empty((h, w), np.float32)
    ov = np.empty((h, w), np.uint32)
    rc = _acmm_ref.acmm_ref_hier_init(len(imgs), arr, _p(c), _p(pl), _p(sc), sc.shape[1], sc.shape[0],
                                      ctypes.c_float(dmin), ctypes.c_float(dmax), _p(op), _p(oc), _p(pre), _p(ov))
    if rc != 0:
        raise RuntimeError(f"acmm_ref_hier_init failed: {rc}")
    return op, oc, pre, ov


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _img_ptrs(images):
    imgs = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
    arr = (ctypes.c_void_p * len(imgs))(*[i.ctypes.data for i in imgs])
    return imgs, arr


def _cams(cams):
    c = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
    return c


def set_tex_rounding(mode: int) -> None:
    lib().or_set_tex_rounding(ctypes.c_int(mode))


def tex2d(img: np.ndarray, u: float, v: float) -> float:
    img = np.ascontiguousarray(img, dtype=np.float32)
    h, w = img.shape
    return lib().or_tex2d(_p(img), w, h, ctypes.c_float(u), ctypes.c_float(v))


def homography(ref_cam, src_cam, plane) -> np.ndarray:
    out = np.zeros(9, np.float32)
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    s = _cams(np.array([src_cam], dtype=CAMERA_DTYPE))
    pl = np.ascontiguousarray(plane, dtype=np.float32)
    lib().or_homography(_p(r), _p(s), _p(pl), _p(out))
    return out


def cost_vectors(images, cams, planes) -> np.ndarray:
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    out = np.zeros((h, w, len(imgs) - 1), np.float32)
    lib().or_cost_vectors(len(imgs), arr, _p(c), _p(planes), _p(out))
    return out


def ncc_bounds(images, cams, planes, k_err=1.0, pixels=None):
    """Cost vectors with per-value bounds (or_ncc_bounds): (cost, bound,
    acc, kind).  bound: what rounding the tap coordinates differently (up to
    k_err x their propagated first-order error bound) can change, 2 where a
    decision may flip; acc: twice the first-order bound of the FP32
    arithmetic on given samples (window sums, and 1e-5 relative on every
    bilateral weight); kind: bit 0 a tap near a texture-weight step, bit 1 a
    decision may flip.  pixels: flat indices y*W+x to evaluate only those
    (outputs [len(pixels)][S])."""
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    if pixels is not None:
        px = np.ascontiguousarray(pixels, dtype=np.int32)
        shp = (len(px), len(imgs) - 1)
        cost, bound, acc = (np.zeros(shp, np.float32) for _ in range(3))
        kind = np.zeros(shp, np.int32)
        lib().or_ncc_bounds_px(len(imgs), arr, _p(c), _p(planes), ctypes.c_float(k_err), _p(px), len(px), _p(cost),
                               _p(bound), _p(acc), _p(kind))
        return cost, bound, acc, kind
    cost = np.zeros((h, w, len(imgs) - 1), np.float32)
    bound = np.zeros_like(cost)
    acc = np.zeros_like(cost)
    kind = np.zeros(cost.shape, np.int32)
    lib().or_ncc_bounds(len(imgs), arr, _p(c), _p(planes), ctypes.c_float(k_err), _p(cost), _p(bound), _p(acc),
                        _p(kind))
    return cost, bound, acc, kind


def initial_costs(images, cams, planes):
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    cost = np.zeros((h, w), np.float32)
    views = np.zeros((h, w), np.uint32)
    lib().or_initial_costs(len(imgs), arr, _p(c), _p(planes), _p(cost), _p(views))
    return cost, views


def geom_costs(cams, depth_maps, planes) -> np.ndarray:
    dm, arr = _img_ptrs(depth_maps)
    c = _cams(cams)
    h, w = dm[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    out = np.zeros((h, w, len(dm) - 1), np.float32)
    lib().or_geom_costs(len(dm), _p(c), arr, _p(planes), _p(out))
    return out


def run_patchmatch(images, cams, *, depth_min, depth_max, seed=0, salt=0, geom=False, prior=False,
                   planes=None, costs=None, views=None, prior_planes=None, masks=None, depth_maps=None,
                   half_steps=6, finalize=True, variant=0, hierarchy=0, pre_costs=None):
    """HPM::RunPatchMatch restated on the CPU; returns (planes, costs, views).
    variant 1: ACMM::RunPatchMatch of the ACMM+NESP variant; with hierarchy
    (1 upsampled, 2 same size) planes hold the upsampled (world normal,
    depth) and pre_costs, a float32 [H, W] array, receives the acceptance
    thresholds."""
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = (np.zeros((h, w, 4), np.float32) if planes is None
              else np.array(planes, dtype=np.float32, copy=True, order="C"))
    costs = (np.zeros((h, w), np.float32) if costs is None
             else np.array(costs, dtype=np.float32, copy=True, order="C"))
    views = (np.zeros((h, w), np.uint32) if views is None
             else np.array(views, dtype=np.uint32, copy=True, order="C"))
    if hierarchy and (pre_costs is None or pre_costs.shape != (h, w) or pre_costs.dtype != np.float32
                      or not pre_costs.flags.c_contiguous):
        raise ValueError("run_patchmatch: hierarchy needs a float32 [H, W] pre_costs array")
    o = OrRunOpts(int(geom), int(prior), float(depth_min), float(depth_max), int(seed), int(salt),
                  int(half_steps), int(finalize), int(variant), int(hierarchy),
                  None if pre_costs is None else pre_costs.ctypes.data)
    pp = None if prior_planes is None else np.ascontiguousarray(prior_planes, dtype=np.float32)
    mk = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint32)
    dms, darr = (None, None) if depth_maps is None else _img_ptrs(depth_maps)
    rc = lib().or_run_patchmatch(len(imgs), arr, _p(c), ctypes.byref(o), _p(planes), _p(costs), _p(views),
                                 None if pp is None else _p(pp), None if mk is None else _p(mk), darr)
    if rc != 0:
        raise RuntimeError(f"or_run_patchmatch failed: {rc}")
    return planes, costs, views


def depth_normal_filter(ref_cam, planes, costs):
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    planes = np.array(planes, dtype=np.float32, copy=True, order="C")
    costs = np.ascontiguousarray(costs, dtype=np.float32)
    lib().or_depth_normal_filter(_p(r), _p(planes), _p(costs))
    return planes


def jbu(guide, coarse_depth, coarse_normal):
    guide = np.ascontiguousarray(guide, dtype=np.float32)
    cd = np.ascontiguousarray(coarse_depth, dtype=np.float32)
    cn = np.ascontiguousarray(coarse_normal, dtype=np.float32)
    rows, cols = guide.shape
    s_rows, s_cols = cd.shape
    od = np.zeros((rows, cols), np.float32)
    on = np.zeros((rows, cols, 3), np.float32)
    rc = lib().or_jbu(_p(guide), cols, rows, _p(cd), _p(cn), s_cols, s_rows, _p(od), _p(on))
    if rc == 1:
        return None, None
    return od, on


def jbu_at_scale(guide, coarse_depth, coarse_normal, image_scale):
    """or_jbu_at_scale: the JBU's weights at a given integer scale (1 too)."""
    guide = np.ascontiguousarray(guide, dtype=np.float32)
    cd = np.ascontiguousarray(coarse_depth, dtype=np.float32)
    cn = np.ascontiguousarray(coarse_normal, dtype=np.float32)
    rows, cols = guide.shape
    s_rows, s_cols = cd.shape
    od = np.zeros((rows, cols), np.float32)
    on = np.zeros((rows, cols, 3), np.float32)
    lib().or_jbu_at_scale(_p(guide), cols, rows, _p(cd), _p(cn), s_cols, s_rows, int(image_scale), _p(od), _p(on))
    return od, on


def philox_uniform(seed, pixel, step, salt, n) -> float:
    return lib().or_philox_uniform(seed, pixel, step, salt, n)


def support_points(costs) -> np.ndarray:
    costs = np.ascontiguousarray(costs, dtype=np.float32)
    h, w = costs.shape
    cap = ((w + 4) // 5) * ((h + 4) // 5)
    out = np.zeros((cap, 2), np.int32)
    n = lib().or_support_points(_p(costs), w, h, _p(out), cap)
    return out[:n].copy()


def plane_from_triangle(ref_cam, depth, tri, factor) -> np.ndarray:
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    t = np.ascontiguousarray(tri, dtype=np.int32).reshape(6)
    out = np.zeros(4, np.float32)
    lib().or_plane_from_triangle(_p(r), _p(depth), depth.shape[1], _p(t), ctypes.c_float(factor), _p(out))
    return out


def depth_from_plane(ref_cam, plane, x, y, factor) -> float:
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    p = np.ascontiguousarray(plane, dtype=np.float32)
    return lib().or_depth_from_plane(_p(r), _p(p), int(x), int(y), ctypes.c_float(factor))


def raster_triangles(tris, w, h, mask=None):
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 6)
    mask = np.zeros((h, w), np.float32) if mask is None else np.array(mask, np.float32, copy=True, order="C")
    kept = np.zeros_like(t)
    n = lib().or_raster_triangles(_p(t), len(t), w, h, _p(mask), _p(kept))
    return mask, kept[:n].copy()


def knn6(pts, w, h, mask=None):
    """(h, w, 6) indices of the 6 nearest points per pixel (brute force)."""
    pts = np.ascontiguousarray(pts, dtype=np.int32).reshape(-1, 2)
    out = np.zeros((h, w, 6), np.int32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
    lib().or_knn6(_p(pts), len(pts), w, h, None if m is None else _p(m), _p(out))
    return out


def knn_supplement(ref_cam, pts, depth, factor, dmin, dmax, mask):
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    pts = np.ascontiguousarray(pts, dtype=np.int32).reshape(-1, 2)
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    h, w = depth.shape
    mask = np.array(mask, np.float32, copy=True, order="C")
    planes = np.zeros((h, w, 4), np.float32)
    lib().or_knn_supplement(_p(r), _p(pts), len(pts), _p(depth), w, h, ctypes.c_float(factor),
                            ctypes.c_float(dmin), ctypes.c_float(dmax), _p(planes), _p(mask))
    return planes, mask


def set_knn_grid(on: bool) -> None:
    """Neighbour search of knn_supplement: exact grid search (default) or the
    brute-force scan; both give identical results."""
    lib().or_set_knn_grid(ctypes.c_int(int(on)))


def _f(x):
    return ctypes.c_float(float(x))


def prior_coarse(ref_cam, mask, tri_planes, knn_planes, factor, dmin, dmax):
    """main.cpp:124-162: (prior depth, world normal) at the level's size."""
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    mask = np.ascontiguousarray(mask, dtype=np.float32)
    h, w = mask.shape
    tp = np.ascontiguousarray(tri_planes, dtype=np.float32).reshape(-1, 4)
    kp = np.ascontiguousarray(knn_planes, dtype=np.float32).reshape(h, w, 4)
    d = np.zeros((h, w), np.float32)
    n = np.zeros((h, w, 3), np.float32)
    lib().or_prior_coarse(_p(r), _p(mask), _p(tp), len(tp), _p(kp), w, h, _f(factor), _f(dmin), _f(dmax), _p(d), _p(n))
    return d, n


def prior_reload(ref_cam, depth, normal, dmin, dmax):
    """main.cpp:179-203: (ref-frame prior planes, 0/1 masks)."""
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    normal = np.ascontiguousarray(normal, dtype=np.float32)
    h, w = depth.shape
    out = np.zeros((h, w, 4), np.float32)
    m = np.zeros((h, w), np.uint32)
    lib().or_prior_reload(_p(r), _p(depth), _p(normal), w, h, _f(dmin), _f(dmax), _p(out), _p(m))
    return out, m


def prior_full(ref_cam, mask, tri_planes, knn_planes, dmin, dmax):
    """main.cpp:426-454 + HPM.cpp:1099-1123: (prior planes, masks, prior depth)."""
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    mask = np.ascontiguousarray(mask, dtype=np.float32)
    h, w = mask.shape
    tp = np.ascontiguousarray(tri_planes, dtype=np.float32).reshape(-1, 4)
    kp = np.ascontiguousarray(knn_planes, dtype=np.float32).reshape(h, w, 4)
    out = np.zeros((h, w, 4), np.float32)
    m = np.zeros((h, w), np.uint32)
    d = np.zeros((h, w), np.float32)
    lib().or_prior_full(_p(r), _p(mask), _p(tp), len(tp), _p(kp), w, h, _f(dmin), _f(dmax), _p(out), _p(m), _p(d))
    return out, m, d


def fuse_pairs(cams, depths, normals, ref, srcs):
    """or_fuse_pairs: (pair_src [H*W, ns], pair_w [H*W, ns], points [H*W, 3])
    of reference view `ref` against sources `srcs`."""
    n = len(cams)
    c = _cams(cams)
    ds = [np.ascontiguousarray(d, dtype=np.float32) for d in depths]
    ns_ = [np.ascontiguousarray(x, dtype=np.float32) for x in normals]
    arr = lambda xs: (ctypes.c_void_p * n)(*[x.ctypes.data for x in xs])  # noqa: E731
    npx = ds[ref].size
    s = np.array(srcs, np.int32)
    ps = np.empty((npx, len(srcs)), np.int32)
    pw = np.empty((npx, len(srcs)), np.float32)
    pt = np.zeros((npx, 3), np.float32)
    lib().or_fuse_pairs(n, _p(c), arr(ds), arr(ns_), int(ref), len(srcs), _p(s), _p(ps), _p(pw), _p(pt))
    return ps, pw, pt


def fuse(cams, depths, normals, colors, problems, acmm=False):
    """or_fuse: the reference's sequential RunFusion (xyz, normal, colour as
    floats B G R), in the reference's order; acmm: the ACMM+NESP variant's
    rule (or_fuse_acmm)."""
    n = len(cams)
    c = _cams(cams)
    ds = [np.ascontiguousarray(d, dtype=np.float32) for d in depths]
    ns_ = [np.ascontiguousarray(x, dtype=np.float32) for x in normals]
    cs = [np.ascontiguousarray(x, dtype=np.uint8) for x in colors]
    arr = lambda xs: (ctypes.c_void_p * n)(*[x.ctypes.data for x in xs])  # noqa: E731
    refs = np.array([p[0] for p in problems], np.int32)
    counts = np.array([len(p[1]) for p in problems], np.int32)
    srcs = np.zeros((max(len(problems), 1), 32), np.int32)
    for i, (_, s) in enumerate(problems):
        srcs[i, :len(s)] = s
    cap = sum(d.size for d in ds)
    xyz = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    col = np.empty((cap, 3), np.float32)
    fn = lib().or_fuse_acmm if acmm else lib().or_fuse
    fn.restype = ctypes.c_long
    k = fn(n, _p(c), arr(ds), arr(ns_), arr(cs), len(problems), _p(refs), _p(counts), _p(srcs), _p(xyz), _p(nrm),
           _p(col), ctypes.c_long(cap))
    return xyz[:k].copy(), nrm[:k].copy(), col[:k].copy()


# ---------------------------------------------------------------- reference shim

def ref_cost_vectors(images, cams, planes) -> np.ndarray:
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    out = np.zeros((h, w, len(imgs) - 1), np.float32)
    rc = ref().hpm_ref_cost_vectors(len(imgs), arr, _p(c), _p(planes), _p(out))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_cost_vectors: cuda error {rc}")
    return out


def ref_initial_costs(images, cams, planes):
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    cost = np.zeros((h, w), np.float32)
    views = np.zeros((h, w), np.uint32)
    rc = ref().hpm_ref_initial_costs(len(imgs), arr, _p(c), _p(planes), _p(cost), _p(views))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_initial_costs: cuda error {rc}")
    return cost, views


def ref_geom_costs(cams, depth_maps, planes) -> np.ndarray:
    dm, arr = _img_ptrs(depth_maps)
    c = _cams(cams)
    h, w = dm[0].shape
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    out = np.zeros((h, w, len(dm) - 1), np.float32)
    rc = ref().hpm_ref_geom_costs(len(dm), _p(c), arr, _p(planes), _p(out))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_geom_costs: cuda error {rc}")
    return out


def ref_tap_samples(images, cams, planes, pixels):
    """The reference's 36 source-texture samples per (listed pixel, source
    view) of ComputeBilateralNCC, and whether the warped centre is inside."""
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    px = np.ascontiguousarray(pixels, dtype=np.int32)
    S = len(imgs) - 1
    out = np.zeros((len(px), S, 36), np.float32)
    inside = np.zeros((len(px), S), np.int32)
    rc = ref().hpm_ref_tap_samples(len(imgs), arr, _p(c), _p(planes), _p(px), len(px), _p(out), _p(inside))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_tap_samples: cuda error {rc}")
    return out, inside.astype(bool)


def ref_homography(ref_cam, src_cam, planes) -> np.ndarray:
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    s = _cams(np.array([src_cam], dtype=CAMERA_DTYPE))
    planes = np.ascontiguousarray(planes, dtype=np.float32).reshape(-1, 4)
    out = np.zeros((len(planes), 9), np.float32)
    rc = ref().hpm_ref_homography(_p(r), _p(s), _p(planes), len(planes), _p(out))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_homography: cuda error {rc}")
    return out


def ref_tex_fetch(img, coords) -> np.ndarray:
    img = np.ascontiguousarray(img, dtype=np.float32)
    coords = np.ascontiguousarray(coords, dtype=np.float32).reshape(-1, 2)
    out = np.zeros(len(coords), np.float32)
    h, w = img.shape
    rc = ref().hpm_ref_tex_fetch(_p(img), w, h, _p(coords), len(coords), _p(out))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_tex_fetch: cuda error {rc}")
    return out


def ref_depth_normal_filter(ref_cam, planes, costs):
    r = _cams(np.array([ref_cam], dtype=CAMERA_DTYPE))
    planes = np.array(planes, dtype=np.float32, copy=True, order="C")
    costs = np.ascontiguousarray(costs, dtype=np.float32)
    rc = ref().hpm_ref_depth_normal_filter(_p(r), _p(planes), _p(costs))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_depth_normal_filter: cuda error {rc}")
    return planes


def ref_jbu(guide, coarse_depth, coarse_normal):
    guide = np.ascontiguousarray(guide, dtype=np.float32)
    cd = np.ascontiguousarray(coarse_depth, dtype=np.float32)
    cn = np.ascontiguousarray(coarse_normal, dtype=np.float32)
    rows, cols = guide.shape
    s_rows, s_cols = cd.shape
    od = np.zeros((rows, cols), np.float32)
    on = np.zeros((rows, cols, 3), np.float32)
    rc = ref().hpm_ref_jbu(_p(guide), cols, rows, _p(cd), _p(cn), s_cols, s_rows, _p(od), _p(on))
    if rc != 0:
        raise RuntimeError(f"hpm_ref_jbu: cuda error {rc}")
    return od, on


def ref_run_patchmatch(images, cams, *, depth_min, depth_max, seed=0, geom=False, prior=False, multi_geometry=False,
                       planes=None, costs=None, prior_planes=None, masks=None, depth_maps=None, timed=False):
    """HPM::RunPatchMatch of the reference (shim).  timed=True launches the
    same kernels with CUDA events around each and also returns their times
    (ms): init, the six half-steps, GetDepthandNormal, the two filters."""
    imgs, arr = _img_ptrs(images)
    c = _cams(cams)
    h, w = imgs[0].shape
    planes = (np.zeros((h, w, 4), np.float32) if planes is None
              else np.array(planes, dtype=np.float32, copy=True, order="C"))
    costs = (np.zeros((h, w), np.float32) if costs is None
             else np.array(costs, dtype=np.float32, copy=True, order="C"))
    o = RefRunOpts(int(geom), int(prior), int(multi_geometry), float(depth_min), float(depth_max), int(seed))
    pp = None if prior_planes is None else np.ascontiguousarray(prior_planes, dtype=np.float32)
    mk = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint32)
    dms, darr = (None, None) if depth_maps is None else _img_ptrs(depth_maps)
    args = (len(imgs), arr, _p(c), ctypes.byref(o), _p(planes), _p(costs), None if pp is None else _p(pp),
            None if mk is None else _p(mk), darr)
    if timed:
        ms = np.zeros(10, np.float32)
        rc = ref().hpm_ref_run_patchmatch_timed(*args, _p(ms))
    else:
        rc = ref().hpm_ref_run_patchmatch(*args)
    if rc != 0:
        raise RuntimeError(f"hpm_ref_run_patchmatch: cuda error {rc}")
    if timed:
        return planes, costs, {"init": float(ms[0]), "half_steps": [float(x) for x in ms[1:7]],
                               "depth_normal": float(ms[7]), "filter": [float(ms[8]), float(ms[9])]}
    return planes, costs

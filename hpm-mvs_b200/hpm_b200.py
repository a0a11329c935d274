"""Python binding of libhpm_b200.so (the C ABI in include/hpm_b200.h).

This module is a thin ctypes layer for tests, the benchmark and Python
callers; the product is the CUDA/C++ library.  It fails loudly when the
library is missing: there is no CPU fallback.

Array conventions follow the reference's host buffers:
  images  float32 [H, W];  cams  structured array of CAMERA_DTYPE;
  planes  float32 [H, W, 4];  costs  float32 [H, W].
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("HPM_B200_LIB", os.path.join(HERE, "libhpm_b200.so"))

CAMERA_DTYPE = np.dtype(
    [("K", "<f4", 9), ("R", "<f4", 9), ("t", "<f4", 3), ("height", "<i4"), ("width", "<i4"),
     ("depth_min", "<f4"), ("depth_max", "<f4")]
)
MAX_IMAGES = 33

HPM_OK = 0
STATUS_NAMES = {0: "HPM_OK", -1: "HPM_ERR_ARG", -2: "HPM_ERR_CUDA", -3: "HPM_ERR_IO", -4: "HPM_ERR_STATE",
                -5: "HPM_ERR_TIMEOUT", -6: "HPM_ERR_NOMEM"}

# every symbol include/hpm_b200.h declares
EXPORTED = [
    "hpm_default_params", "hpm_create", "hpm_destroy", "hpm_last_error", "hpm_set_views", "hpm_set_geom_depths",
    "hpm_set_hypotheses", "hpm_set_prior", "hpm_clear_prior", "hpm_run_patchmatch", "hpm_run_partial",
    "hpm_get_result",
    "hpm_get_selected_views", "hpm_device_state", "hpm_stream", "hpm_jbu", "hpm_cost_vectors",
    "hpm_initial_costs", "hpm_geom_costs", "hpm_depth_normal_filter", "hpm_profile_enable", "hpm_profile_read",
    "hpm_count_enable", "hpm_count_read", "hpm_write_dmb", "hpm_read_dmb", "hpm_read_camera", "hpm_read_pair",
    "hpm_fp32_peak", "hpm_jbu_noalloc", "hpm_process_problem", "hpm_last_prior_stats", "hpm_delaunay",
    "hpm_prior_level", "hpm_run_scene", "hpm_run_scene_ex", "hpm_read_gray8", "hpm_resize_linear",
    "hpm_fuse", "hpm_write_ply", "hpm_read_bgr8", "hpm_set_scene_workers", "hpm_resize_linear_u8",
    "hpm_raster_triangles", "hpm_knn6", "hpm_tap_samples", "hpm_net_pack_weights", "hpm_net_conv3x3",
    "hpm_net_conv_wgrad", "hpm_run_scene_net", "hpm_net_coarse_inputs", "hpm_net_targets", "hpm_net_loss",
    "hpm_net_adam", "hpm_run_scene_batched", "hpm_run_scene_batched_net", "hpm_run_scene_acmm",
    "hpm_fuse_acmm", "hpm_fuse_pass",
]


class HpmSceneOpts(ctypes.Structure):
    _fields_ = [("planar_prior", ctypes.c_int), ("geom_iterations", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("pyramid_levels", ctypes.c_int), ("iterations", ctypes.c_int), ("fix_quirks", ctypes.c_int),
                ("geom_pass_iterations", ctypes.c_int)]


class HpmAcmmOpts(ctypes.Structure):
    _fields_ = [("geom_iterations", ctypes.c_int), ("seed", ctypes.c_uint64), ("size_bound", ctypes.c_int),
                ("max_iterations", ctypes.c_int), ("geom_max_iterations", ctypes.c_int)]


class HpmNetWeights(ctypes.Structure):
    _fields_ = [("packed", ctypes.c_void_p * 4), ("bias", ctypes.c_void_p * 4)]


class HpmProblemOpts(ctypes.Structure):
    _fields_ = [("planar_prior", ctypes.c_int), ("geom_consistency", ctypes.c_int), ("multi_geometry", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("pyramid_levels", ctypes.c_int), ("fix_quirks", ctypes.c_int)]


def delaunay(points: np.ndarray, w: int, h: int) -> np.ndarray:
    """Triangles (n, 6) of the prior triangulation of integer points (n, 2)."""
    pts = np.ascontiguousarray(points, dtype=np.int32).reshape(-1, 2)
    n = lib().hpm_delaunay(_p(pts), len(pts), w, h, None, 0)
    if n < 0:
        raise HpmError(f"hpm_delaunay: {STATUS_NAMES.get(n, n)}")
    out = np.zeros((max(n, 1), 6), np.int32)
    n2 = lib().hpm_delaunay(_p(pts), len(pts), w, h, _p(out), len(out))
    return out[:n2]


def raster_triangles(tris: np.ndarray, w: int, h: int, device: int = 0) -> np.ndarray:
    """Triangle-id raster (h, w) int32 of the prior: index + 1 of the last
    triangle reaching each pixel, 0 where none does."""
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 6)
    ids = np.zeros((h, w), np.int32)
    rc = lib().hpm_raster_triangles(device, _p(t), len(t), w, h, _p(ids))
    if rc != HPM_OK:
        raise HpmError(f"hpm_raster_triangles: {STATUS_NAMES.get(rc, rc)}")
    return ids


def knn6(points: np.ndarray, w: int, h: int, mask=None, device: int = 0) -> np.ndarray:
    """(h, w, 6) int32 indices of the 6 nearest support points per pixel
    (mask <= 0, or all pixels), nearest first, -1 where not searched."""
    pts = np.ascontiguousarray(points, dtype=np.int32).reshape(-1, 2)
    out = np.zeros((h, w, 6), np.int32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float32)
    rc = lib().hpm_knn6(device, _p(pts), len(pts), w, h, None if m is None else _p(m), _p(out))
    if rc != HPM_OK:
        raise HpmError(f"hpm_knn6: {STATUS_NAMES.get(rc, rc)}")
    return out


def fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA throughput of the device in TFLOP/s."""
    t = ctypes.c_float()
    rc = lib().hpm_fp32_peak(device, ctypes.byref(t), None)
    if rc != HPM_OK:
        raise HpmError(f"hpm_fp32_peak: {STATUS_NAMES.get(rc, rc)}")
    return float(t.value)


class HpmParams(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int), ("patch_size", ctypes.c_int), ("radius_increment", ctypes.c_int),
                ("sigma_spatial", ctypes.c_float), ("sigma_color", ctypes.c_float), ("top_k", ctypes.c_int),
                ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float), ("geom_consistency", ctypes.c_int),
                ("multi_geometry", ctypes.c_int), ("planar_prior", ctypes.c_int),
                ("honour_max_iterations", ctypes.c_int), ("seed", ctypes.c_uint64), ("fix_quirks", ctypes.c_int),
                ("variant", ctypes.c_int), ("hierarchy", ctypes.c_int)]


class HpmError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HpmError(f"{LIB_PATH} is missing: build it with `make -C hpm-mvs_b200`")
        L = ctypes.CDLL(LIB_PATH)
        L.hpm_last_error.restype = ctypes.c_char_p
        L.hpm_last_error.argtypes = [ctypes.c_void_p]
        L.hpm_stream.restype = ctypes.c_void_p
        L.hpm_stream.argtypes = [ctypes.c_void_p]
        L.hpm_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        for name in ["hpm_destroy", "hpm_clear_prior"]:
            getattr(L, name).argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def default_params(depth_min: float, depth_max: float, *, seed: int = 0, geom: bool = False,
                   prior: bool = False, multi_geometry: bool = False, fix_quirks: bool = False, variant: int = 0,
                   hierarchy: int = 0, max_iterations: int = 3) -> HpmParams:
    """HpmParams with the reference's defaults; fix_quirks: see HpmParams in
    include/hpm_b200.h (False keeps the reference's behaviour).  variant 1:
    the ACMM+NESP variant's kernels (max_iterations honoured, hierarchy
    1 or 2 for its hierarchy pass)."""
    p = HpmParams()
    lib().hpm_default_params(ctypes.byref(p))
    p.depth_min = depth_min
    p.depth_max = depth_max
    p.seed = seed
    p.geom_consistency = int(geom)
    p.planar_prior = int(prior)
    p.multi_geometry = int(multi_geometry)
    p.fix_quirks = int(fix_quirks)
    p.variant = int(variant)
    p.hierarchy = int(hierarchy)
    p.max_iterations = int(max_iterations)
    return p


class Context:
    """One hpm_ctx: device buffers of one problem plus its CUDA stream."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        rc = lib().hpm_create(ctypes.byref(self._h), device)
        if rc != HPM_OK:
            raise HpmError(f"hpm_create failed: {STATUS_NAMES.get(rc, rc)}")
        self.shape = None
        self.n = 0

    def close(self):
        if self._h:
            lib().hpm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc: int, what: str) -> None:
        if rc != HPM_OK:
            msg = lib().hpm_last_error(self._h)
            raise HpmError(f"{what}: {STATUS_NAMES.get(rc, rc)}: {msg.decode() if msg else ''}")

    def set_views(self, images, cams) -> None:
        imgs = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
        cams = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
        for i, im in enumerate(imgs):
            if im.shape != (int(cams[i]["height"]), int(cams[i]["width"])):
                raise ValueError(f"image {i} shape {im.shape} does not match its camera")
        arr = (ctypes.c_void_p * len(imgs))(*[i.ctypes.data for i in imgs])
        self._check(lib().hpm_set_views(self._h, arr, _p(cams), len(imgs)), "hpm_set_views")
        self._imgs = imgs  # keep alive until the synchronous upload returned (it has)
        self.shape = imgs[0].shape
        self.n = len(imgs)

    def set_geom_depths(self, depths) -> None:
        ds = [np.ascontiguousarray(d, dtype=np.float32) for d in depths]
        arr = (ctypes.c_void_p * len(ds))(*[d.ctypes.data for d in ds])
        self._check(lib().hpm_set_geom_depths(self._h, arr), "hpm_set_geom_depths")

    def set_hypotheses(self, planes, costs=None) -> None:
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        costs = None if costs is None else np.ascontiguousarray(costs, dtype=np.float32)
        self._check(lib().hpm_set_hypotheses(self._h, _p(planes), _p(costs)), "hpm_set_hypotheses")

    def set_prior(self, prior_planes, masks) -> None:
        pp = np.ascontiguousarray(prior_planes, dtype=np.float32)
        mk = np.ascontiguousarray(masks, dtype=np.uint32)
        self._check(lib().hpm_set_prior(self._h, _p(pp), _p(mk)), "hpm_set_prior")

    def clear_prior(self) -> None:
        self._check(lib().hpm_clear_prior(self._h), "hpm_clear_prior")

    def run_patchmatch(self, params: HpmParams) -> None:
        self._check(lib().hpm_run_patchmatch(self._h, ctypes.byref(params)), "hpm_run_patchmatch")

    def run_partial(self, params: HpmParams, half_steps: int, finalize: bool) -> None:
        self._check(lib().hpm_run_partial(self._h, ctypes.byref(params), int(half_steps), int(finalize)),
                    "hpm_run_partial")

    def process_problem(self, *, planar_prior=True, geom=False, multi_geometry=False, seed=0, pyramid_levels=-1,
                        fix_quirks=False):
        """ProcessProblem for the current views: returns (depth, normal, cost, prior_depth)."""
        h, w = self.shape
        depth = np.empty((h, w), np.float32)
        normal = np.empty((h, w, 3), np.float32)
        cost = np.empty((h, w), np.float32)
        prior = np.empty((h, w), np.float32)
        o = HpmProblemOpts(int(planar_prior), int(geom), int(multi_geometry), int(seed), int(pyramid_levels),
                           int(fix_quirks))
        self._check(lib().hpm_process_problem(self._h, ctypes.byref(o), _p(depth), _p(normal), _p(cost), _p(prior)),
                    "hpm_process_problem")
        return depth, normal, cost, prior

    def run_scene(self, images, cams, pairs, *, planar_prior=True, geom_iterations=2, seed=0, pyramid_levels=-1,
                  images_are_device=False, outputs=True, extra_maps=False, net=None, batched=False, iterations=0,
                  fix_quirks=False, geom_pass_iterations=0):
        """The reference's main() over a scene.  images: per-view float32 [H, W]
        arrays, or device pointers (ints) with images_are_device; pairs:
        [(ref, [sources])].  outputs: True to return new per-view (depth,
        normal, cost) lists, False for none (the maps stay on the device), or
        a tuple of three caller-owned lists of float32 arrays to fill.
        extra_maps (with outputs=True): also return each view's pass-set-A
        depth and prior depth (hpm_run_scene_ex), five lists in all.
        net: an HpmNetWeights (priornet.Net.weights()) to run the prior-net
        form (hpm_run_scene_net) instead of the plain form.  batched: the
        batched form (hpm_run_scene_batched; with net, the batched prior-net
        form, hpm_run_scene_batched_net).  iterations: with net, PatchMatch
        iterations of each full-scale pass (0: the reference's 3), and
        geom_pass_iterations of each geometric pass (0: as iterations).  fix_quirks:
        HpmSceneOpts.fix_quirks (False keeps the reference's behaviour)."""
        n = len(cams)
        cams = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
        if images_are_device:
            ptrs = [int(p) for p in images]
            keep = None
        else:
            keep = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
            ptrs = [k.ctypes.data for k in keep]
        img_arr = (ctypes.c_void_p * n)(*ptrs)
        refs = np.array([p[0] for p in pairs], np.int32)
        counts = np.array([len(p[1]) for p in pairs], np.int32)
        srcs = np.zeros((len(pairs), MAX_IMAGES - 1), np.int32)
        for i, (_, s) in enumerate(pairs):
            srcs[i, :len(s)] = s
        o = HpmSceneOpts(int(planar_prior), int(geom_iterations), int(seed), int(pyramid_levels), int(iterations),
                         int(fix_quirks), int(geom_pass_iterations))
        outs = None
        if isinstance(outputs, (tuple, list)):
            outs = list(zip(*outputs))
            for v, c in enumerate(cams):
                hw = (int(c["height"]), int(c["width"]))
                for k, shape in enumerate([hw, hw + (3,), hw]):
                    a = outs[v][k]
                    if a.shape != shape or a.dtype != np.float32 or not a.flags.c_contiguous:
                        raise ValueError(f"run_scene: output {k} of view {v} must be float32 {shape}, C order")
            arrs = [(ctypes.c_void_p * n)(*[o_[k].ctypes.data for o_ in outs]) for k in range(3)]
        elif outputs:
            outs = [(np.empty((int(c["height"]), int(c["width"])), np.float32),
                     np.empty((int(c["height"]), int(c["width"]), 3), np.float32),
                     np.empty((int(c["height"]), int(c["width"])), np.float32)) for c in cams]
            arrs = [(ctypes.c_void_p * n)(*[o_[k].ctypes.data for o_ in outs]) for k in range(3)]
        else:
            arrs = [None, None, None]
        if batched:
            if extra_maps:
                raise ValueError("run_scene: the batched form has no extra maps")
            if net is not None:
                self._check(lib().hpm_run_scene_batched_net(self._h, n, img_arr, _p(cams), len(pairs), _p(refs),
                                                            _p(counts), _p(srcs), ctypes.byref(o), ctypes.byref(net),
                                                            arrs[0], arrs[1], arrs[2]), "hpm_run_scene_batched_net")
            else:
                self._check(lib().hpm_run_scene_batched(self._h, n, img_arr, _p(cams), len(pairs), _p(refs),
                                                        _p(counts), _p(srcs), ctypes.byref(o), arrs[0], arrs[1],
                                                        arrs[2]), "hpm_run_scene_batched")
        elif net is not None:
            if extra_maps:
                raise ValueError("run_scene: extra_maps is not available in the prior-net form")
            self._check(lib().hpm_run_scene_net(self._h, n, img_arr, _p(cams), len(pairs), _p(refs), _p(counts),
                                                _p(srcs), ctypes.byref(o), ctypes.byref(net), arrs[0], arrs[1],
                                                arrs[2]), "hpm_run_scene_net")
        elif extra_maps:
            if outputs is not True:
                raise ValueError("run_scene: extra_maps needs outputs=True")
            extra = [[np.empty((int(c["height"]), int(c["width"])), np.float32) for c in cams] for _ in range(2)]
            ex = [(ctypes.c_void_p * n)(*[a.ctypes.data for a in e]) for e in extra]
            self._check(lib().hpm_run_scene_ex(self._h, n, img_arr, _p(cams), len(pairs), _p(refs), _p(counts),
                                               _p(srcs), ctypes.byref(o), arrs[0], arrs[1], arrs[2], ex[0], ex[1]),
                        "hpm_run_scene_ex")
        else:
            self._check(lib().hpm_run_scene(self._h, n, img_arr, _p(cams), len(pairs), _p(refs), _p(counts),
                                            _p(srcs), ctypes.byref(o), arrs[0], arrs[1], arrs[2]), "hpm_run_scene")
        del keep
        if outputs:
            res = [o_[0] for o_ in outs], [o_[1] for o_ in outs], [o_[2] for o_ in outs]
            return res + tuple(extra) if extra_maps else res
        return None

    def run_scene_acmm(self, images, cams, pairs, *, seed=0, geom_iterations=2, size_bound=0, max_iterations=0,
                       geom_max_iterations=0):
        """The ACMM+NESP variant's main() over a scene (hpm_run_scene_acmm):
        coarse-to-fine over an image pyramid whose coarsest scale has every
        longer side at most size_bound (0: the reference's 1000).  images:
        per-view float32 [H, W]; pairs: [(v, [sources])] with pairs[v][0] ==
        v.  Returns per-view (depth, world normal, cost) lists."""
        n = len(cams)
        cams = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
        keep = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
        img_arr = (ctypes.c_void_p * n)(*[k.ctypes.data for k in keep])
        refs = np.array([p[0] for p in pairs], np.int32)
        counts = np.array([len(p[1]) for p in pairs], np.int32)
        srcs = np.zeros((len(pairs), MAX_IMAGES - 1), np.int32)
        for i, (_, s) in enumerate(pairs):
            srcs[i, :len(s)] = s
        o = HpmAcmmOpts(int(geom_iterations), int(seed), int(size_bound), int(max_iterations),
                        int(geom_max_iterations))
        outs = [(np.empty((int(c["height"]), int(c["width"])), np.float32),
                 np.empty((int(c["height"]), int(c["width"]), 3), np.float32),
                 np.empty((int(c["height"]), int(c["width"])), np.float32)) for c in cams]
        arrs = [(ctypes.c_void_p * n)(*[o_[k].ctypes.data for o_ in outs]) for k in range(3)]
        self._check(lib().hpm_run_scene_acmm(self._h, n, img_arr, _p(cams), len(pairs), _p(refs), _p(counts),
                                             _p(srcs), ctypes.byref(o), arrs[0], arrs[1], arrs[2]),
                    "hpm_run_scene_acmm")
        del keep
        return [o_[0] for o_ in outs], [o_[1] for o_ in outs], [o_[2] for o_ in outs]

    def prior_level(self, level, depth, normal, cost):
        """Prior of one pyramid level from given maps: (planes, masks, prior_depth)."""
        h, w = self.shape
        d = np.ascontiguousarray(depth, np.float32)
        n = np.ascontiguousarray(normal, np.float32)
        c = np.ascontiguousarray(cost, np.float32)
        planes = np.empty((h, w, 4), np.float32)
        masks = np.empty((h, w), np.uint32)
        pd = np.empty((h, w), np.float32)
        self._check(lib().hpm_prior_level(self._h, int(level), _p(d), _p(n), _p(c), _p(planes), _p(masks), _p(pd)),
                    "hpm_prior_level")
        return planes, masks, pd

    def prior_stats(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        self._check(lib().hpm_last_prior_stats(self._h, ctypes.byref(a), ctypes.byref(b)), "hpm_last_prior_stats")
        return a.value, b.value

    def get_result(self):
        h, w = self.shape
        planes = np.empty((h, w, 4), np.float32)
        costs = np.empty((h, w), np.float32)
        self._check(lib().hpm_get_result(self._h, _p(planes), _p(costs)), "hpm_get_result")
        return planes, costs

    def get_selected_views(self):
        h, w = self.shape
        v = np.empty((h, w), np.uint32)
        self._check(lib().hpm_get_selected_views(self._h, _p(v)), "hpm_get_selected_views")
        return v

    def cost_vectors(self, planes):
        h, w = self.shape
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        out = np.empty((h, w, self.n - 1), np.float32)
        self._check(lib().hpm_cost_vectors(self._h, _p(planes), _p(out)), "hpm_cost_vectors")
        return out

    def tap_samples(self, planes, pixels):
        """(samples [n][S][36], inside [n][S] bool) of the NCC windows of the
        listed pixels (flat indices)."""
        pl = np.ascontiguousarray(planes, dtype=np.float32)
        px = np.ascontiguousarray(pixels, dtype=np.int32)
        S = self.n - 1
        out = np.zeros((len(px), S, 36), np.float32)
        inside = np.zeros((len(px), S), np.int32)
        self._check(lib().hpm_tap_samples(self._h, _p(pl), _p(px), len(px), _p(out), _p(inside)), "hpm_tap_samples")
        return out, inside.astype(bool)

    def initial_costs(self, planes):
        h, w = self.shape
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        cost = np.empty((h, w), np.float32)
        views = np.empty((h, w), np.uint32)
        self._check(lib().hpm_initial_costs(self._h, _p(planes), _p(cost), _p(views)), "hpm_initial_costs")
        return cost, views

    def geom_costs(self, planes):
        h, w = self.shape
        planes = np.ascontiguousarray(planes, dtype=np.float32)
        out = np.empty((h, w, self.n - 1), np.float32)
        self._check(lib().hpm_geom_costs(self._h, _p(planes), _p(out)), "hpm_geom_costs")
        return out

    def depth_normal_filter(self, planes, costs):
        planes = np.array(planes, dtype=np.float32, copy=True, order="C")
        costs = np.ascontiguousarray(costs, dtype=np.float32)
        self._check(lib().hpm_depth_normal_filter(self._h, _p(planes), _p(costs)), "hpm_depth_normal_filter")
        return planes

    def jbu(self, guide, coarse_depth, coarse_normal):
        guide = np.ascontiguousarray(guide, dtype=np.float32)
        cd = np.ascontiguousarray(coarse_depth, dtype=np.float32)
        cn = np.ascontiguousarray(coarse_normal, dtype=np.float32)
        rows, cols = guide.shape
        s_rows, s_cols = cd.shape
        od = np.zeros((rows, cols), np.float32)
        on = np.zeros((rows, cols, 3), np.float32)
        self._check(lib().hpm_jbu(self._h, _p(guide), cols, rows, _p(cd), _p(cn), s_cols, s_rows, _p(od), _p(on)),
                    "hpm_jbu")
        return od, on

    def profile_enable(self, on: bool = True) -> None:
        self._check(lib().hpm_profile_enable(self._h, int(on)), "hpm_profile_enable")

    def profile_read(self):
        ms = (ctypes.c_float * 4)()
        cnt = (ctypes.c_int * 4)()
        self._check(lib().hpm_profile_read(self._h, ms, cnt), "hpm_profile_read")
        names = ["init", "propagate", "finalize", "jbu"]
        return {n: (float(ms[i]), int(cnt[i])) for i, n in enumerate(names)}

    def count_enable(self, on: bool = True) -> None:
        self._check(lib().hpm_count_enable(self._h, int(on)), "hpm_count_enable")

    def set_scene_workers(self, workers: int) -> None:
        self._check(lib().hpm_set_scene_workers(self._h, int(workers)), "hpm_set_scene_workers")

    def count_read(self):
        a = ctypes.c_uint64()
        b = ctypes.c_uint64()
        self._check(lib().hpm_count_read(self._h, ctypes.byref(a), ctypes.byref(b)), "hpm_count_read")
        return int(a.value), int(b.value)

    def stream(self) -> int:
        return int(lib().hpm_stream(self._h) or 0)


def write_dmb(path: str, data: np.ndarray) -> None:
    a = np.ascontiguousarray(data, dtype=np.float32)
    h, w = a.shape[:2]
    nb = 1 if a.ndim == 2 else a.shape[2]
    rc = lib().hpm_write_dmb(path.encode(), _p(a), h, w, nb)
    if rc != HPM_OK:
        raise HpmError(f"hpm_write_dmb({path}): {STATUS_NAMES.get(rc, rc)}")


def read_dmb(path: str) -> np.ndarray:
    h, w, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = lib().hpm_read_dmb(path.encode(), None, ctypes.c_size_t(0), ctypes.byref(h), ctypes.byref(w),
                            ctypes.byref(nb))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_dmb({path}): {STATUS_NAMES.get(rc, rc)}")
    out = np.empty((h.value, w.value, nb.value), np.float32)
    rc = lib().hpm_read_dmb(path.encode(), _p(out), ctypes.c_size_t(out.size), None, None, None)
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_dmb({path}): {STATUS_NAMES.get(rc, rc)}")
    return out[..., 0] if nb.value == 1 else out


def read_camera(path: str) -> np.ndarray:
    cam = np.zeros(1, CAMERA_DTYPE)
    rc = lib().hpm_read_camera(path.encode(), _p(cam))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_camera({path}): {STATUS_NAMES.get(rc, rc)}")
    return cam[0]


def read_gray8(path: str) -> np.ndarray:
    """images/ file as cv::imread(path, IMREAD_GRAYSCALE) gives it (JPEG, PNG, PGM)."""
    w, h = ctypes.c_int(), ctypes.c_int()
    rc = lib().hpm_read_gray8(path.encode(), None, ctypes.c_size_t(0), ctypes.byref(w), ctypes.byref(h))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_gray8({path}) failed: {rc}")
    out = np.empty((h.value, w.value), np.uint8)
    rc = lib().hpm_read_gray8(path.encode(), _p(out), ctypes.c_size_t(out.nbytes), ctypes.byref(w), ctypes.byref(h))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_gray8({path}) failed: {rc}")
    return out


def read_bgr8(path: str) -> np.ndarray:
    """images/ file as cv::imread(path, IMREAD_COLOR) gives it: uint8 [H, W, 3], B G R."""
    w, h = ctypes.c_int(), ctypes.c_int()
    rc = lib().hpm_read_bgr8(path.encode(), None, ctypes.c_size_t(0), ctypes.byref(w), ctypes.byref(h))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_bgr8({path}) failed: {rc}")
    out = np.empty((h.value, w.value, 3), np.uint8)
    rc = lib().hpm_read_bgr8(path.encode(), _p(out), ctypes.c_size_t(out.nbytes), ctypes.byref(w), ctypes.byref(h))
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_bgr8({path}) failed: {rc}")
    return out


def _fuse_inputs(cams, depths, normals, colors, problems):
    n = len(cams)
    cams = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
    ds = [np.ascontiguousarray(d, dtype=np.float32) for d in depths]
    ns_ = [np.ascontiguousarray(x, dtype=np.float32) for x in normals]
    cs = [np.ascontiguousarray(c, dtype=np.uint8) for c in colors]
    refs = np.array([p[0] for p in problems], np.int32)
    counts = np.array([len(p[1]) for p in problems], np.int32)
    srcs = np.zeros((max(len(problems), 1), MAX_IMAGES - 1), np.int32)
    for i, (_, s) in enumerate(problems):
        srcs[i, :len(s)] = s
    cap = sum(d.size for d in ds)
    return n, cams, ds, ns_, cs, refs, counts, srcs, cap


def fuse_pass(cams, depths, normals, colors, problems, pairs, acmm=False):
    """hpm_fuse_pass: the ordered half of the fusion on the host (no GPU)
    from given pairs, one (pair_src [pixels, ns], pair_w [pixels, ns], points
    [pixels, 3]) per problem.  Returns (xyz, normal, bgr) like fuse()."""
    n, cams, ds, ns_, cs, refs, counts, srcs, cap = _fuse_inputs(cams, depths, normals, colors, problems)
    arr = lambda xs: (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])  # noqa: E731
    ps = [np.ascontiguousarray(p[0], dtype=np.int32) for p in pairs]
    pw = [np.ascontiguousarray(p[1], dtype=np.float32) for p in pairs]
    pt = [np.ascontiguousarray(p[2], dtype=np.float32) for p in pairs]
    xyz = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    bgr = np.empty((cap, 3), np.uint8)
    cnt = ctypes.c_longlong()
    rc = lib().hpm_fuse_pass(int(acmm), n, _p(cams), arr(ds), arr(ns_), arr(cs), len(problems), _p(refs),
                             _p(counts), _p(srcs), arr(ps), arr(pw), arr(pt), _p(xyz), _p(nrm), _p(bgr),
                             ctypes.c_longlong(cap), ctypes.byref(cnt))
    if rc != HPM_OK:
        raise HpmError(f"hpm_fuse_pass: {STATUS_NAMES.get(rc, rc)}")
    k = cnt.value
    return xyz[:k].copy(), nrm[:k].copy(), bgr[:k].copy()


def fuse(cams, depths, normals, colors, problems, device: int = 0, acmm: bool = False):
    """RunFusion (main.cpp:502-633): (xyz [n,3], normal [n,3], bgr [n,3] uint8)
    in the reference's order.  problems: [(ref, [sources])].  acmm: the
    ACMM+NESP variant's RunFusion (hpm_fuse_acmm)."""
    n = len(cams)
    cams = np.ascontiguousarray(cams, dtype=CAMERA_DTYPE)
    ds = [np.ascontiguousarray(d, dtype=np.float32) for d in depths]
    ns_ = [np.ascontiguousarray(x, dtype=np.float32) for x in normals]
    cs = [np.ascontiguousarray(c, dtype=np.uint8) for c in colors]
    arr = lambda xs: (ctypes.c_void_p * n)(*[x.ctypes.data for x in xs])  # noqa: E731
    refs = np.array([p[0] for p in problems], np.int32)
    counts = np.array([len(p[1]) for p in problems], np.int32)
    srcs = np.zeros((max(len(problems), 1), MAX_IMAGES - 1), np.int32)
    for i, (_, s) in enumerate(problems):
        srcs[i, :len(s)] = s
    cap = sum(d.size for d in ds)
    xyz = np.empty((cap, 3), np.float32)
    nrm = np.empty((cap, 3), np.float32)
    bgr = np.empty((cap, 3), np.uint8)
    cnt = ctypes.c_longlong()
    fn = lib().hpm_fuse_acmm if acmm else lib().hpm_fuse
    rc = fn(device, n, _p(cams), arr(ds), arr(ns_), arr(cs), len(problems), _p(refs), _p(counts), _p(srcs), _p(xyz),
            _p(nrm), _p(bgr), ctypes.c_longlong(cap), ctypes.byref(cnt))
    if rc != HPM_OK:
        raise HpmError(f"hpm_fuse{'_acmm' if acmm else ''}: {STATUS_NAMES.get(rc, rc)}")
    k = cnt.value
    return xyz[:k].copy(), nrm[:k].copy(), bgr[:k].copy()


def write_ply(path: str, xyz, normal, bgr) -> None:
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    normal = np.ascontiguousarray(normal, dtype=np.float32)
    bgr = np.ascontiguousarray(bgr, dtype=np.uint8)
    rc = lib().hpm_write_ply(path.encode(), ctypes.c_longlong(len(xyz)), _p(xyz), _p(normal), _p(bgr))
    if rc != HPM_OK:
        raise HpmError(f"hpm_write_ply({path}): {STATUS_NAMES.get(rc, rc)}")


def resize_linear_u8(src: np.ndarray, dw: int, dh: int) -> np.ndarray:
    """cv::resize INTER_LINEAR of a uint8 [H, W] or [H, W, C] image, byte for byte (host)."""
    src = np.ascontiguousarray(src, dtype=np.uint8)
    ch = 1 if src.ndim == 2 else src.shape[2]
    out = np.empty((dh, dw) if src.ndim == 2 else (dh, dw, ch), np.uint8)
    rc = lib().hpm_resize_linear_u8(_p(src), src.shape[1], src.shape[0], ch, _p(out), dw, dh)
    if rc != HPM_OK:
        raise HpmError(f"hpm_resize_linear_u8: {rc}")
    return out


def resize_linear(src: np.ndarray, dw: int, dh: int) -> np.ndarray:
    """cv::resize INTER_LINEAR of a float32 [H, W] or [H, W, C] map (host)."""
    src = np.ascontiguousarray(src, dtype=np.float32)
    ch = 1 if src.ndim == 2 else src.shape[2]
    out = np.empty((dh, dw) if src.ndim == 2 else (dh, dw, ch), np.float32)
    rc = lib().hpm_resize_linear(_p(src), src.shape[1], src.shape[0], ch, _p(out), dw, dh)
    if rc != HPM_OK:
        raise HpmError(f"hpm_resize_linear failed: {rc}")
    return out


def read_pair(path: str):
    n = ctypes.c_int()
    rc = lib().hpm_read_pair(path.encode(), ctypes.byref(n), None, None, None, 0)
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_pair({path}): {STATUS_NAMES.get(rc, rc)}")
    refs = np.zeros(n.value, np.int32)
    counts = np.zeros(n.value, np.int32)
    srcs = np.zeros((n.value, MAX_IMAGES - 1), np.int32)
    rc = lib().hpm_read_pair(path.encode(), ctypes.byref(n), _p(refs), _p(counts), _p(srcs), n.value)
    if rc != HPM_OK:
        raise HpmError(f"hpm_read_pair({path}): {STATUS_NAMES.get(rc, rc)}")
    return [(int(refs[i]), [int(s) for s in srcs[i, :counts[i]]]) for i in range(n.value)]

"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs the reference's HPM-MVS/HPM.cu, compiled unchanged for sm_100a into
oracle/_ref/libhpm_ref.so (recipe: oracle/Makefile), on a B200 and stores its
outputs for small seeded inputs:

  tex_probe.npz   tex2D<float> of the reference's texture set-up at chosen
                  coordinates (bilinear weight quantisation, edge addressing)
  ncc.npz         ComputeMultiViewCostVector / ComputeMultiViewInitialCost-
                  andSelectedViews / ComputeHomography for fixed planes
  geom.npz        ComputeGeomConsistencyCost for fixed planes and depth maps
  jbu.npz         JBU_cu at x2 and x4
  filter.npz      GetDepthandNormal + Black/RedPixelFilter
  pm.npz          whole RunPatchMatch passes (plain; geometric) for the
                  statistical comparison (the reference's RNG is curand
                  XORWOW, so only statistics are comparable)
  cfg1_640x480.npz, cfg2_800x600_s10.npz
                  the same deterministic pieces at the bench's own sizes:
                  config 1 (5 views of 640x480, 4 sources) and an 11-view
                  scene of config 2's recipe at 800x600 (10 sources, the
                  middle level of the bench's pyramid).  The scenes are
                  rebuilt from their seeds by the tests (a SHA-256 of the
                  images guards the generator); outputs are kept at 4096
                  sampled pixels, plus the reference's whole-pass accuracy
                  and kernel times over four seeds.
  acmm_hier.npz   the ACMM+NESP variant's RandomInitialization of a
                  hierarchy pass (ACMM+NESP/windows/ACMM.cu:538-604: JBU
                  average of the previous scale's normals, the threshold
                  pre_costs, the initial cost), from the reference's own
                  ACMM.cu compiled for sm_100a (oracle/_ref/libacmm_ref.so)

Usage (on a GPU machine, from the repository root):
    python tests/golden/make_golden.py [--out tests/golden] [--only small|bench|acmm]
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "hpm-mvs_b200"), os.path.join(ROOT, "oracle")]

import oracle as orc  # noqa: E402
import synthetic as syn  # noqa: E402

W, H, NV = 96, 72, 5


def small_scene(seed=0):
    return syn.make_scene(seed, W, H, NV, n_planes=6, low_texture=0.25)


def test_planes(sc, ref, rng):
    gt = syn.gt_planes_ref_frame(sc, ref)
    H, W = gt.shape[:2]
    pert = gt.copy()
    pert[..., 3] *= rng.uniform(0.97, 1.03, pert.shape[:2]).astype(np.float32)
    # random planes facing the camera at random depths
    n = rng.normal(size=gt.shape[:2] + (3,)).astype(np.float32)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    n[..., 2] = -np.abs(n[..., 2]) - 0.2
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    cam = sc.cams[ref]
    K = cam["K"].reshape(3, 3)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float32)
    d = rng.uniform(1.5, 9.0, gt.shape[:2]).astype(np.float32)
    X = np.stack([d * (xs - K[0, 2]) / K[0, 0], d * (ys - K[1, 2]) / K[1, 1], d], -1)
    rnd = np.concatenate([n, -(n * X).sum(-1, keepdims=True)], -1).astype(np.float32)
    return np.stack([gt, pert, rnd])


def tex_probe():
    # texture A: value 256*x (y-independent); texture B: value 256*y
    w, h = 6, 5
    ta = np.tile(256.0 * np.arange(w, dtype=np.float32), (h, 1))
    tb = np.tile(256.0 * np.arange(h, dtype=np.float32)[:, None], (1, w))
    k = np.arange(4097, dtype=np.float32)
    fine = np.stack([2.5 + k / 4096.0, np.full_like(k, 2.5)], -1)            # fractions along x
    fine_y = np.stack([np.full_like(k, 2.5), 2.5 + k / 4096.0], -1)          # fractions along y
    edge = np.arange(-4.0, w + 4.0, 0.125, dtype=np.float32)
    edges = np.stack([edge, np.full_like(edge, 2.5)], -1)
    edge_y = np.arange(-4.0, h + 4.0, 0.125, dtype=np.float32)
    edges_y = np.stack([np.full_like(edge_y, 2.5), edge_y], -1)
    big = np.array([[1e6, 2.5], [-1e6, 2.5], [2.5, 1e6], [2.5, -1e6], [3.0e9, 2.5]], np.float32)
    rng = np.random.default_rng(7)
    rnd = np.stack([rng.uniform(-1, w + 1, 2000), rng.uniform(-1, h + 1, 2000)], -1).astype(np.float32)
    tr = rng.uniform(0, 255, (h, w)).astype(np.float32).round()
    out = dict(ta=ta, tb=tb, tr=tr, fine=fine, fine_y=fine_y, edges=edges, edges_y=edges_y, big=big, rnd=rnd)
    out["a_fine"] = orc.ref_tex_fetch(ta, fine)
    out["b_fine_y"] = orc.ref_tex_fetch(tb, fine_y)
    out["a_edges"] = orc.ref_tex_fetch(ta, edges)
    out["b_edges_y"] = orc.ref_tex_fetch(tb, edges_y)
    out["a_big"] = orc.ref_tex_fetch(ta, big)
    out["b_big"] = orc.ref_tex_fetch(tb, big)
    out["r_rnd"] = orc.ref_tex_fetch(tr, rnd)
    # single-texel textures: the fetch returns that texel's effective weight
    g = (np.arange(64, dtype=np.float32) - 32.0) / 32.0
    gx, gy = np.meshgrid(g, g)
    dgrid = np.stack([3.5 + gx.ravel(), 2.5 + gy.ravel()], -1).astype(np.float32)
    out["dgrid"] = dgrid
    for val in (1.0, 255.0, 0.7):
        d = np.zeros((h, w), np.float32)
        d[2, 3] = val
        out[f"delta_{val}"] = orc.ref_tex_fetch(d, dgrid)
    # random texture at coordinates on the exact 1/256 grid of both axes
    A, B = np.meshgrid(np.arange(0, 256, 4, dtype=np.float32), np.arange(0, 256, 4, dtype=np.float32))
    grid256 = np.stack([2.5 + A.ravel() / 256.0, 1.5 + B.ravel() / 256.0], -1).astype(np.float32)
    out["grid256"] = grid256
    out["r_grid256"] = orc.ref_tex_fetch(tr, grid256)
    return out


# the bench-size cases: scene recipe, reference view, seed of the inputs
BENCH_CASES = {
    "cfg1_640x480": dict(scene=dict(seed=11, width=640, height=480, n_views=5, n_planes=6, low_texture=0.25), ref=2,
                         seed=501),
    "cfg2_800x600_s10": dict(scene=dict(seed=12, width=800, height=600, n_views=11, n_planes=20, n_spheres=5,
                                        low_texture=0.40), ref=5, seed=502),
}
N_SAMPLES = 4096
STAT_SEEDS = (100, 101, 102, 103)


def acmm_hier_inputs():
    """The ACMM+NESP hierarchy case: 5 views of 128x96; the previous
    scale's world normals (ground truth, perturbed) and costs at 64x48; the
    upsampled depth at 128x96 (ground truth, perturbed).  Returns (scene, ref
    view, images, cameras, planes as the host leaves them ((0, 0, 0, depth)),
    scaled maps (normal, cost))."""
    sc = syn.make_scene(31, 128, 96, 5)
    ref = 2
    imgs, cams = syn.view_set(sc, ref)
    rng = np.random.default_rng(31)
    n = sc.gt_normal[ref][::2, ::2] + rng.normal(0, 0.1, (48, 64, 3))
    n = (n / np.linalg.norm(n, axis=-1, keepdims=True)).astype(np.float32)
    cost = rng.uniform(0, 1, (48, 64)).astype(np.float32)
    scaled = np.concatenate([n, cost[..., None]], -1).astype(np.float32)
    planes = np.zeros((96, 128, 4), np.float32)
    planes[..., 3] = sc.gt_depth[ref] * rng.uniform(0.95, 1.05, (96, 128)).astype(np.float32)
    return sc, ref, imgs, cams, planes, scaled


def acmm_case(out_dir):
    if not orc.acmm_ref_available():
        raise SystemExit("oracle/_ref/libacmm_ref.so is missing: build it with `make -C oracle acmm`")
    sc, ref, imgs, cams, planes, scaled = acmm_hier_inputs()
    op, oc, pre, ov = orc.ref_acmm_hier_init(imgs, cams, planes, scaled)
    np.savez_compressed(os.path.join(out_dir, "acmm_hier.npz"), images_sha256=images_sha256(imgs), planes=op,
                        costs=oc, pre_costs=pre, views=ov)
    print("acmm_hier: finite planes", float(np.isfinite(op).all(-1).mean()), "mean pre", float(np.nanmean(pre)))


def images_sha256(imgs):
    h = hashlib.sha256()
    for i in imgs:
        h.update(np.ascontiguousarray(i, dtype=np.uint8).tobytes())
    return h.hexdigest()


def bench_case_inputs(name):
    """Every input of a bench-size case, rebuilt deterministically from the
    case's seeds: the scene, the problem's images and cameras, three plane
    fields (true, perturbed, random), the geometric depth maps, the JBU
    coarse inputs, the filter's costs and the sampled pixels."""
    case = BENCH_CASES[name]
    kw = dict(case["scene"])
    sc = syn.make_scene(kw.pop("seed"), kw.pop("width"), kw.pop("height"), kw.pop("n_views"), **kw)
    ref = case["ref"]
    imgs, cams = syn.view_set(sc, ref)
    rng = np.random.default_rng(case["seed"])
    planes = test_planes(sc, ref, rng)
    ids = [ref] + list(sc.pairs[ref][1])
    depths = [np.where(rng.random(sc.gt_depth[i].shape) < 0.05, 0.0, sc.gt_depth[i]).astype(np.float32) for i in ids]
    jbu = {}
    for s in (2, 4):
        cd = sc.gt_depth[ref][::s, ::s].copy()
        cd[rng.random(cd.shape) < 0.1] = 0.0
        jbu[s] = (cd, np.ascontiguousarray(sc.gt_normal[ref][::s, ::s]))
    h, w = imgs[0].shape
    costs = rng.uniform(0, 1, (h, w)).astype(np.float32)
    costs[rng.random((h, w)) < 0.1] = 0.0
    pixels = np.sort(rng.choice(h * w, N_SAMPLES, replace=False)).astype(np.int32)
    return dict(sc=sc, ref=ref, imgs=imgs, cams=cams, planes=planes, depths=depths, jbu=jbu, costs=costs,
                pixels=pixels)


def bench_cases(out_dir):
    for name in BENCH_CASES:
        c = bench_case_inputs(name)
        imgs, cams, planes, px = c["imgs"], c["cams"], c["planes"], c["pixels"]
        sc, ref = c["sc"], c["ref"]
        h, w = imgs[0].shape
        S = len(imgs) - 1
        flat = lambda a: a.reshape(h * w, *a.shape[2:])[px]  # noqa: E731
        out = dict(images_sha256=images_sha256(imgs), planes_sha256=hashlib.sha256(planes.tobytes()).hexdigest(),
                   pixels=px, planes=np.stack([flat(p) for p in planes]))
        out["cost_vectors"] = np.stack([flat(orc.ref_cost_vectors(imgs, cams, p)) for p in planes])
        ic = [orc.ref_initial_costs(imgs, cams, p) for p in planes]
        out["init_cost"] = np.stack([flat(a) for a, _ in ic])
        out["init_views"] = np.stack([flat(v) for _, v in ic])
        out["geom_costs"] = np.stack([flat(orc.ref_geom_costs(cams, c["depths"], p)) for p in planes])
        for s, (cd, cn) in c["jbu"].items():
            od, on = orc.ref_jbu(imgs[0], cd, cn)
            out[f"jbu_depth_{s}"] = flat(od)
            out[f"jbu_normal_{s}"] = flat(on)
        out["filter"] = flat(orc.ref_depth_normal_filter(cams[0], planes[1], c["costs"]))
        dmin, dmax = sc.depth_min * 0.6, sc.depth_max * 1.2
        acc, nerr, times = [], [], []
        for seed in STAT_SEEDS:
            pl, _, t = orc.ref_run_patchmatch(imgs, cams, depth_min=dmin, depth_max=dmax, seed=seed, timed=True)
            acc.append(syn.depth_accuracy(pl[..., 3], sc.gt_depth[ref]))
            nerr.append(syn.normal_error_deg(pl[..., :3], sc.gt_normal[ref], sc.gt_depth[ref]))
            times.append([t["init"]] + t["half_steps"] + [t["depth_normal"]] + t["filter"])
        out.update(pass_accuracy=np.array(acc), pass_normal_err_deg=np.array(nerr),
                   pass_kernel_ms=np.array(times, np.float32), sources=S)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **out)
        print(name, "reference pass accuracy", np.round(acc, 4), "normal err", np.round(nerr, 2),
              "half-step ms", np.round(np.mean(np.array(times)[:, 1:7]), 3))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--only", choices=["small", "bench", "acmm"], default=None)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if args.only in (None, "acmm"):
        acmm_case(args.out)
    if args.only == "acmm":
        return
    if not orc.ref_available():
        raise SystemExit("oracle/_ref/libhpm_ref.so is missing: build it with `make -C oracle ref`")
    if args.only != "small":
        bench_cases(args.out)
    if args.only == "bench":
        return
    rng = np.random.default_rng(1234)

    np.savez_compressed(os.path.join(args.out, "tex_probe.npz"), **tex_probe())

    sc = small_scene(0)
    ref = 2
    imgs, cams = syn.view_set(sc, ref)
    planes = test_planes(sc, ref, rng)
    cv = np.stack([orc.ref_cost_vectors(imgs, cams, p) for p in planes])
    ic = [orc.ref_initial_costs(imgs, cams, p) for p in planes]
    homs = np.stack([orc.ref_homography(cams[0], cams[v], planes[2][::7, ::7].reshape(-1, 4)) for v in range(1, NV)])
    np.savez_compressed(os.path.join(args.out, "ncc.npz"), images=np.stack([i.astype(np.uint8) for i in imgs]),
                        cams=cams, planes=planes, cost_vectors=cv, init_cost=np.stack([c for c, _ in ic]),
                        init_views=np.stack([v for _, v in ic]), hom_planes=planes[2][::7, ::7].reshape(-1, 4),
                        homographies=homs)

    depths = [sc.gt_depth[i] for i in [ref] + list(sc.pairs[ref][1])]
    depths = [np.where(rng.random(d.shape) < 0.05, 0.0, d).astype(np.float32) for d in depths]
    gc = np.stack([orc.ref_geom_costs(cams, depths, p) for p in planes])
    np.savez_compressed(os.path.join(args.out, "geom.npz"), cams=cams, depths=np.stack(depths), planes=planes,
                        geom_costs=gc)

    guide = imgs[0]
    jb = {}
    for s in (2, 4):
        cd = sc.gt_depth[ref][::s, ::s].copy()
        cd[rng.random(cd.shape) < 0.1] = 0.0
        cn = sc.gt_normal[ref][::s, ::s].copy()
        od, on = orc.ref_jbu(guide, cd, cn)
        jb[f"coarse_depth_{s}"] = cd
        jb[f"coarse_normal_{s}"] = cn
        jb[f"out_depth_{s}"] = od
        jb[f"out_normal_{s}"] = on
    np.savez_compressed(os.path.join(args.out, "jbu.npz"), guide=guide, **jb)

    costs = rng.uniform(0, 1, (H, W)).astype(np.float32)
    costs[rng.random((H, W)) < 0.1] = 0.0
    filt = orc.ref_depth_normal_filter(cams[0], planes[1], costs)
    np.savez_compressed(os.path.join(args.out, "filter.npz"), cams=cams, planes=planes[1], costs=costs,
                        out=filt)

    dmin, dmax = sc.depth_min * 0.6, sc.depth_max * 1.2
    runs = {}
    for seed in (1, 2):
        pl, co = orc.ref_run_patchmatch(imgs, cams, depth_min=dmin, depth_max=dmax, seed=seed)
        runs[f"plain_planes_{seed}"] = pl
        runs[f"plain_costs_{seed}"] = co
    np.savez_compressed(os.path.join(args.out, "pm.npz"), images=np.stack([i.astype(np.uint8) for i in imgs]),
                        cams=cams, gt_depth=sc.gt_depth[ref], gt_normal=sc.gt_normal[ref], depth_min=dmin,
                        depth_max=dmax, **runs)
    print("golden fixtures written to", args.out)


if __name__ == "__main__":
    main()

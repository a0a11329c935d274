#!/usr/bin/env python
"""main() of HPM-MVS (main.cpp:636-677) from Python, over the same C ABI as
the C++ host (hpm_mvs): images/%08d.jpg (or .png, .pgm) decoded by the
library to the bytes cv::imread gives (HPM.cpp:492, main.cpp:523).

    python hpm-mvs_b200/hpm_mvs.py dense_folder [--seed S] [--levels K]
                                   [--geom-iterations G] [--no-prior] [--device D]
                                   [--no-fusion] [--per-problem] [--resume] [--stop-after N]
                                   [--no-reference-compat] [--log PATH]

Writes HPM/2333_%08d/{depths,depths_geom,normals,costs,depths_prior}.dmb like
the reference's ProcessProblem, then fuses them into HPM/HPM_model.ply
(RunFusion).  Seeds as in the C++ host: problem p of pass
set A uses S + p, of geometric iteration g S + 1000003 (g + 1) + p.

Finished steps are logged in HPM/progress.txt, in the C++ host's format
(Progress): --stop-after N ends the run once N steps have finished, --resume
skips the logged steps.

--acmm runs the ACMM+NESP variant's main() (ACMM+NESP/windows/main.cpp:
299-384) instead: coarse-to-fine over an image pyramid (hpm_run_scene_acmm),
writing ACMM_NESP/2333_%08d/{depths_geom,normals,costs}.dmb and fusing them
into ACMM_NESP/ACMM_NESP_model.ply.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import hpm_b200 as hb  # noqa: E402

MAX_IMAGE_SIZE = 3200  # PatchMatchParams::max_image_size (HPM.h:35)


def load_view(folder: str, vid: int):
    """Gray float image and camera of one view, after the 3200-pixel cap
    (InuputInitialization, HPM.cpp:482-551)."""
    img = None
    for ext in (".jpg", ".png", ".pgm"):
        p = os.path.join(folder, "images", f"{vid:08d}{ext}")
        if os.path.exists(p):
            img = hb.read_gray8(p)
            break
    if img is None:
        raise hb.HpmError(f"no image for view {vid} under {folder}/images")
    img = img.astype(np.float32)
    cam = hb.read_camera(os.path.join(folder, "cams", f"{vid:08d}_cam.txt")).copy()
    h, w = img.shape
    if w > MAX_IMAGE_SIZE or h > MAX_IMAGE_SIZE:
        factor = min(np.float32(MAX_IMAGE_SIZE) / np.float32(w), np.float32(MAX_IMAGE_SIZE) / np.float32(h))
        # std::round of the float product: halves away from zero
        nw = int(np.floor(np.float64(np.float32(w) * factor) + 0.5))
        nh = int(np.floor(np.float64(np.float32(h) * factor) + 0.5))
        img = hb.resize_linear(img, nw, nh)
        sx, sy = np.float32(nw) / np.float32(w), np.float32(nh) / np.float32(h)
        K = cam["K"]
        K[0] *= sx
        K[2] *= sx
        K[4] *= sy
        K[5] *= sy
        w, h = nw, nh
    cam["width"], cam["height"] = w, h
    return img, cam


def process_problem(ctx, folder, ref, srcs, views, *, geom, planar_prior, multi_geometry, seed, levels,
                    fix_quirks=False):
    """ProcessProblem (main.cpp:35-499) for one reference view."""
    out = os.path.join(folder, "HPM", f"2333_{ref:08d}")
    os.makedirs(out, exist_ok=True)
    ids = [ref] + list(srcs)
    ctx.set_views([views[i][0] for i in ids], np.array([views[i][1] for i in ids]))
    if geom:
        suffix = "depths_geom.dmb" if multi_geometry else "depths.dmb"
        depths = [hb.read_dmb(os.path.join(folder, "HPM", f"2333_{i:08d}", suffix)) for i in ids]
        normal = hb.read_dmb(os.path.join(out, "normals.dmb"))
        cost = hb.read_dmb(os.path.join(out, "costs.dmb"))
        ctx.set_geom_depths(depths)
        ctx.set_hypotheses(np.concatenate([normal, depths[0][..., None]], -1), cost)
    d, n, c, pd = ctx.process_problem(planar_prior=planar_prior and not geom, geom=geom,
                                      multi_geometry=multi_geometry, seed=seed, pyramid_levels=levels,
                                      fix_quirks=fix_quirks)
    if planar_prior and not geom:
        hb.write_dmb(os.path.join(out, "depths_prior.dmb"), pd)
    hb.write_dmb(os.path.join(out, "depths_geom.dmb" if geom else "depths.dmb"), d)
    hb.write_dmb(os.path.join(out, "normals.dmb"), n)
    hb.write_dmb(os.path.join(out, "costs.dmb"), c)
    return int(d.size)


def run_scene(ctx, folder, problems, needed, views, *, planar_prior, geom_iterations, seed, levels,
              fix_quirks=False):
    """All passes in one hpm_run_scene_ex call (maps in device memory between
    passes), then the files ProcessProblem leaves for every problem."""
    index = {v: i for i, v in enumerate(needed)}
    pairs = [(index[ref], [index[s] for s in srcs]) for ref, srcs in problems]
    d, n, c, pa, pr = ctx.run_scene([views[v][0] for v in needed], np.array([views[v][1] for v in needed]), pairs,
                                    planar_prior=planar_prior, geom_iterations=geom_iterations, seed=seed,
                                    pyramid_levels=levels, extra_maps=True, fix_quirks=fix_quirks)
    for ref, _ in problems:
        i = index[ref]
        out = os.path.join(folder, "HPM", f"2333_{ref:08d}")
        os.makedirs(out, exist_ok=True)
        if planar_prior:
            hb.write_dmb(os.path.join(out, "depths_prior.dmb"), pr[i])
        hb.write_dmb(os.path.join(out, "depths.dmb"), pa[i])
        if geom_iterations > 0:
            hb.write_dmb(os.path.join(out, "depths_geom.dmb"), d[i])
        hb.write_dmb(os.path.join(out, "normals.dmb"), n[i])
        hb.write_dmb(os.path.join(out, "costs.dmb"), c[i])
    return int(sum(d[index[ref]].size for ref, _ in problems))


def run_scene_acmm(ctx, folder, problems, views, *, geom_iterations, seed):
    """The ACMM+NESP variant's main() minus fusion (hpm_run_scene_acmm), then
    the files its ProcessProblem leaves (main.cpp:96-121)."""
    if [ref for ref, _ in problems] != list(range(len(problems))):
        raise hb.HpmError("the ACMM+NESP variant needs pair.txt to list views 0, 1, ... in order "
                          "(the reference looks a source's scale up by its image id)")
    d, n, c = ctx.run_scene_acmm([views[v][0] for v in range(len(problems))],
                                 np.array([views[v][1] for v in range(len(problems))]),
                                 [(ref, list(srcs)) for ref, srcs in problems], seed=seed,
                                 geom_iterations=geom_iterations)
    for ref, _ in problems:
        out = os.path.join(folder, "ACMM_NESP", f"2333_{ref:08d}")
        os.makedirs(out, exist_ok=True)
        hb.write_dmb(os.path.join(out, "depths_geom.dmb"), d[ref])
        hb.write_dmb(os.path.join(out, "normals.dmb"), n[ref])
        hb.write_dmb(os.path.join(out, "costs.dmb"), c[ref])
    return int(sum(x.size for x in d))


def run_fusion(folder, problems, geom_consistency, device=0, tree="HPM", ply="HPM_model.ply", acmm=False):
    """RunFusion (main.cpp:502-633) with RescaleImageAndCamera
    (HPM.cpp:187-208: OpenCV's 8-bit bilinear, reproduced by
    hpm_resize_linear_u8) over the maps under folder/tree; acmm: the
    ACMM+NESP variant's RunFusion (ACMM+NESP/windows/main.cpp:154-297).
    Returns the point count."""
    cams, depths, normals, colors = [], [], [], []
    for ref, _ in problems:
        out = os.path.join(folder, tree, f"2333_{ref:08d}")
        d = hb.read_dmb(os.path.join(out, "depths_geom.dmb" if geom_consistency else "depths.dmb"))
        n = hb.read_dmb(os.path.join(out, "normals.dmb"))
        cam = hb.read_camera(os.path.join(folder, "cams", f"{ref:08d}_cam.txt")).copy()
        img = None
        for ext in (".jpg", ".png", ".pgm"):
            p = os.path.join(folder, "images", f"{ref:08d}{ext}")
            if os.path.exists(p):
                img = hb.read_bgr8(p)
                break
        if img is None:
            raise hb.HpmError(f"no colour image for view {ref}")
        h, w = d.shape
        if img.shape[:2] != (h, w):
            sx, sy = np.float32(w) / np.float32(img.shape[1]), np.float32(h) / np.float32(img.shape[0])
            img = hb.resize_linear_u8(img, w, h)
            K = cam["K"]
            K[0] *= sx
            K[2] *= sx
            K[4] *= sy
            K[5] *= sy
        cam["width"], cam["height"] = w, h
        cams.append(cam)
        depths.append(d)
        normals.append(n)
        colors.append(img)
    # the reference indexes views by problem order (main.cpp:517-546)
    probs = [(i, list(srcs)) for i, (_, srcs) in enumerate(problems)]
    xyz, nrm, bgr = hb.fuse(np.array(cams), depths, normals, colors, probs, device, acmm=acmm)
    hb.write_ply(os.path.join(folder, tree, ply), xyz, nrm, bgr)
    return len(xyz)


class Progress:
    """The step log of a dense folder, HPM/progress.txt: a settings line,
    then one line per finished step ("A <ref>", "G<g> <ref>", "scene",
    "fusion"), appended after the step's files are written.  Resuming a log
    written with other settings raises."""

    def __init__(self, folder: str, settings: str, resume: bool):
        os.makedirs(os.path.join(folder, "HPM"), exist_ok=True)
        self.path = os.path.join(folder, "HPM", "progress.txt")
        head = "settings " + settings
        self.steps: list[str] = []
        if resume and os.path.exists(self.path):
            with open(self.path) as f:
                lines = f.read().splitlines()
            if lines:
                if lines[0] != head:
                    raise hb.HpmError(f"cannot resume: {self.path} was written with {lines[0]}")
                self.steps = [ln for ln in lines[1:] if ln]
                return
        with open(self.path, "w") as f:
            f.write(head + "\n")

    def done(self, step: str) -> bool:
        return step in self.steps

    def mark(self, step: str) -> None:
        with open(self.path, "a") as f:
            f.write(step + "\n")
            f.flush()
        self.steps.append(step)


class Stopped(Exception):
    pass


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("dense_folder")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--levels", type=int, default=-1)
    ap.add_argument("--geom-iterations", type=int, default=2)
    ap.add_argument("--no-prior", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-fusion", action="store_true")
    ap.add_argument("--per-problem", action="store_true",
                    help="ProcessProblem problem by problem through .dmb files, as the reference runs")
    ap.add_argument("--resume", action="store_true", help="skip the steps HPM/progress.txt lists")
    ap.add_argument("--stop-after", type=int, default=-1, help="stop once this many steps have finished")
    ap.add_argument("--log", default=None,
                    help="append one JSON line per finished step: its wall time and the depth pixels (the fusion: "
                         "points) it wrote")
    ap.add_argument("--no-reference-compat", action="store_true",
                    help="fix the reference's quirks listed at HpmParams in include/hpm_b200.h (default: keep the "
                         "reference's behaviour)")
    ap.add_argument("--acmm", action="store_true",
                    help="run the ACMM+NESP variant (coarse-to-fine image pyramid) into ACMM_NESP/ instead")
    a = ap.parse_args(argv)
    problems = hb.read_pair(os.path.join(a.dense_folder, "pair.txt"))
    print(f"There are {len(problems)} problems needed to be processed!")
    form = "acmm" if a.acmm else ("per-problem" if a.per_problem else "scene")
    settings = (f"seed={a.seed} levels={a.levels} prior={int(not a.no_prior)} geom_iterations={a.geom_iterations} "
                f"form={form}" + (" fix_quirks=1" if a.no_reference_compat else ""))
    fix = a.no_reference_compat
    progress = Progress(a.dense_folder, settings, a.resume)
    count = [0]

    def step(name, work):
        """work() returns the depth pixels it wrote (the fusion: -points)"""
        if progress.done(name):
            return
        if 0 <= a.stop_after <= count[0]:
            raise Stopped
        t0 = time.perf_counter()
        out = work()
        sec = time.perf_counter() - t0
        progress.mark(name)
        count[0] += 1
        if a.log:
            rec = {"step": name, "seconds": sec}
            if out >= 0:
                rec.update(depth_pixels=out, mpix_per_s=out / sec / 1e6 if sec > 0 else 0.0)
            else:
                rec["points"] = -out
            with open(a.log, "a") as f:
                f.write(json.dumps(rec) + "\n")

    state = {}

    def ctx():
        """the views and the context, made on the first step that needs them"""
        if "ctx" not in state:
            needed = sorted({p[0] for p in problems} | {s for p in problems for s in p[1]})
            state["needed"] = needed
            state["views"] = {v: load_view(a.dense_folder, v) for v in needed}
            state["ctx"] = hb.Context(a.device)
        return state["ctx"]

    try:
        if a.acmm:
            step("scene", lambda: run_scene_acmm(ctx(), a.dense_folder, problems, state["views"],
                                                 geom_iterations=a.geom_iterations, seed=a.seed))
        elif a.per_problem:
            for p, (ref, srcs) in enumerate(problems):
                step(f"A {ref}", lambda: process_problem(ctx(), a.dense_folder, ref, srcs, state["views"], geom=False,
                                                         planar_prior=not a.no_prior, multi_geometry=False,
                                                         seed=a.seed + p, levels=a.levels, fix_quirks=fix))
            for g in range(a.geom_iterations):
                for p, (ref, srcs) in enumerate(problems):
                    step(f"G{g} {ref}",
                         lambda: process_problem(ctx(), a.dense_folder, ref, srcs, state["views"], geom=True,
                                                 planar_prior=False, multi_geometry=g > 0,
                                                 seed=a.seed + 1000003 * (g + 1) + p, levels=a.levels,
                                                 fix_quirks=fix))
        else:
            step("scene", lambda: run_scene(ctx(), a.dense_folder, problems, state["needed"], state["views"],
                                            planar_prior=not a.no_prior, geom_iterations=a.geom_iterations,
                                            seed=a.seed, levels=a.levels, fix_quirks=fix))
        if "ctx" in state:
            state.pop("ctx").close()
        if not a.no_fusion:
            def fusion():
                tree, ply = ("ACMM_NESP", "ACMM_NESP_model.ply") if a.acmm else ("HPM", "HPM_model.ply")
                n = run_fusion(a.dense_folder, problems, a.acmm or a.geom_iterations > 0, a.device, tree, ply,
                               acmm=a.acmm)
                print(f"Fused {n} points into {a.dense_folder}/{tree}/{ply}")
                return -n
            step("fusion", fusion)
    except Stopped:
        print(f"Stopped after {count[0]} steps; --resume continues")
    finally:
        if "ctx" in state:
            state.pop("ctx").close()
    return 0


if __name__ == "__main__":
    try:
        sys.exit(main())
    except hb.HpmError as e:
        print(f"hpm_mvs: {e}", file=sys.stderr)
        sys.exit(1)

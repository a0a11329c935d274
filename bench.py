#!/usr/bin/env python
"""Benchmark of the B200-native HPM-MVS depth estimation path.

One JSON line on rank 0.  A *step* is the reference's main() over one scene
(main.cpp:636-677): pass set A (ProcessProblem with the planar + KNN prior on
every pyramid level) for every view, then the geometric-consistency
iterations for every view.  Metric: depth Mpix/s = depth-map pixels of all
views at processed resolution per second.

  value   steps with the images already resident in HBM (hpm_run_scene on
          device pointers, the depth/normal/cost maps stay on the device)
  e2e     the same steps through the public C ABI from pinned host memory:
          images in, every view's depth, normal and cost maps out
  roofline  the dominant kernel pair (one red/black half-step: site/direction
          kernel + selection/refinement kernel) against the measured FP32 FMA
          peak; algorithmic FLOPs = NCC taps x 34 + 80 per (hypothesis,
          source view), + 120 per geometric-consistency term
  cpu_baseline  the CPU oracle (C restatement of the reference, OpenMP over
          all host cores) on one view of the same scene recipe at 320x240

--impl reference times the reference's own HPM.cu kernels (oracle/_ref:
compiled unchanged for sm_100a) through HPM::RunPatchMatch and
JBU::CudaRun, with the host stages (support points, Delaunay via OpenCV,
triangle raster, KNN prior, prior assembly) restated in C, on a bounded
sample of the same scene: one view per step.

Multi-GPU (torchrun): every rank processes its own scene (independent
objects, no data-path collective; weak scaling); the elapsed time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "hpm-mvs_b200")]

METRIC = "depth Mpix/s, plain vs batched prior-net form on 1 B200, at equal %px relerr<1%"
WORKLOAD = dict(width=1600, height=1200, n_views=11, n_planes=20, n_spheres=5, low_texture=0.40, pyramid_levels=2,
                geom_iterations=2, depth_range=(2.0, 8.0), name="full plain HPM scene")
# stress test: 6048x4032 views, which the reference caps to 3200x2133
# (HPM.cpp:525-551, max_image_size 3200): the scene is rendered at the capped
# size directly; its pyramid follows the reference's rule at that size
# (ComputingMultiScaleSettings, HPM.cpp:851-860: 2 levels below full scale)
STRESS = dict(width=3200, height=2133, n_views=20, n_planes=20, n_spheres=5, low_texture=0.50, pyramid_levels=2,
              geom_iterations=2, depth_range=(1.0, 30.0), n_sources=10,
              name="stress scene (6048x4032 capped to 3200x2133 as the reference does)")
# batched form: all 24 reference views of one scene at three sizes, each with
# 10 sources, the pyramid by the reference's rule per view size
BATCHED = dict(width=1920, height=1080, n_views=24, n_planes=20, n_spheres=5, low_texture=0.40, pyramid_levels=-1,
               geom_iterations=2, depth_range=(2.0, 8.0), arc_step_deg=3.0, n_sources=10,
               sizes=[(1920, 1080)] * 8 + [(1600, 1200)] * 8 + [(960, 540)] * 8,
               name="batched scene")

# DRAM traffic of one half-step (k_prop_dirs + k_prop_refine: read + write),
# from an ncu capture of `bench.py --pass-case` (1600x1200, 10 sources), per
# pixel: the hand-off buffers grow with the pixel count
TRAFFIC_BYTES_PER_PX_HALF_STEP = (154.02 + 323.62 + 797.47 + 388.49) * 1e6 / (1600 * 1200)
GEOM_TERM_FLOPS = 120  # two projections (world point + camera, 3x3 each) and the reprojection distance
TAPS, NCC_FLOPS_PER_TAP, FLOPS_PER_HYP_VIEW = 36, 34, 80


def workload_name():
    w = WORKLOAD
    if "sizes" in w:
        sizes = ", ".join(f"{w['sizes'].count(s)} of {s[0]}x{s[1]}" for s in dict.fromkeys(w["sizes"]))
        views = f"{w['n_views']} views ({sizes})"
    else:
        views = f"{w['n_views']} views of {w['width']}x{w['height']}"
    sources = w.get("n_sources", w["n_views"] - 1)
    pyramid = ("a pyramid by the reference's rule per view size" if w["pyramid_levels"] < 0 else
               f"a {w['pyramid_levels'] + 1}-level pyramid")
    return (f"{w['name']}: {views}, {sources} sources each, planar+KNN prior on {pyramid}, "
            f"{w['geom_iterations']} geometric iterations")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", choices=["plain-hpm", "stress", "batched", "acmm"], default="plain-hpm",
                    help="plain-hpm: 11 views of 1600x1200 (the metric's configuration); stress: 20 views of "
                         "6048x4032 capped to 3200x2133, 50%% low texture, depth 1-30 m (one step takes minutes); "
                         "batched: 24 views at three sizes through hpm_run_scene_batched against the per-problem "
                         "driver; acmm: the ACMM+NESP variant (hpm_run_scene_acmm, coarse-to-fine over an image "
                         "pyramid) on the plain-hpm scene beside the plain HPM form")
    ap.add_argument("--size", default=None,
                    help="WxH override of the workload's resolution (profiling captures use a smaller case)")
    ap.add_argument("--views", type=int, default=None, help="override of the scene's view count")
    ap.add_argument("--shard", choices=["scenes", "views"], default="scenes",
                    help="N>1: one scene per rank (weak scaling, no collective) or one scene's views split over the "
                         "ranks with an all-gather of depth maps before each geometric iteration (strong scaling)")
    ap.add_argument("--pass-case", action="store_true",
                    help="kernel-capture case: plain PatchMatch passes of one view of the scene (1 warm-up, then "
                         "--steps passes); prints the half-step time instead of the bench line")
    ap.add_argument("--flow-case", action="store_true",
                    help="kernel-capture case of the problem flow: ProcessProblem of one view of the scene with its "
                         "prior pyramid (initialisation, prior kernels, JBU, filter), then the fusion of the "
                         "scene's ground-truth maps; prints their wall times")
    ap.add_argument("--net-case", action="store_true",
                    help="kernel-capture case of the network's tensor-core convolutions: --steps training steps "
                         "(forward, data and weight gradients, Adam) on a 400x300 input; prints their time")
    args = ap.parse_args()
    if args.config == "stress":
        WORKLOAD.update(STRESS)
    elif args.config == "batched":
        WORKLOAD.update(BATCHED)
    if args.size:
        w, h = (int(x) for x in args.size.lower().split("x"))
        WORKLOAD.update(width=w, height=h)
    if args.views:
        WORKLOAD.update(n_views=args.views)
    return args


class Dist:
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from torchrun).
    Ranks exchange only timing: a barrier around the timed region and the
    max of the elapsed times; the scenes themselves never cross ranks."""

    def __init__(self, n, backend="nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False
        if self.world > 1:
            import torch.distributed as dist

            kw = {"device_id": __import__("torch").device("cuda", self.local)} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 5]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = [n for i, n in enumerate(names) if any(r[2 + i].strip() == "Active" for r in rows)]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def job_mpix_per_s(world, steps, px_per_rank_step, max_ms):
    """Whole-job depth Mpix/s: every rank processed `steps` scenes of
    px_per_rank_step depth pixels; the job took the slowest rank's time."""
    return world * steps * px_per_rank_step / (max_ms * 1e-3) / 1e6


def make_scene(seed, width=None, height=None):
    import synthetic as syn

    w = WORKLOAD
    extra = {k: w[k] for k in ("sizes", "arc_step_deg", "n_sources") if k in w and not (width or height)}
    sc = syn.make_scene(seed, width or w["width"], height or w["height"], w["n_views"], n_planes=w["n_planes"],
                        n_spheres=w["n_spheres"], low_texture=w["low_texture"], depth_range=w["depth_range"], **extra)
    images = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, list(sc.pairs[v][1])) for v in range(w["n_views"])]
    return sc, images, pairs


def passes_per_view():
    w = WORKLOAD
    return 1 + (w["pyramid_levels"] + 1) + w["geom_iterations"]


def scene_accuracy(sc, depths, normals=None):
    import synthetic as syn

    per_view = {int(v): float(syn.depth_accuracy(d, sc.gt_depth[v])) for v, d in sorted(depths.items())}
    out = {"px_relerr_lt_1pct": float(np.mean(list(per_view.values()))), "views": len(depths),
           "per_view": per_view}
    if normals is not None:
        out["median_normal_err_deg"] = float(np.median(
            [syn.normal_error_deg(normals[v], sc.gt_normal[v], sc.gt_depth[v]) for v in normals]))
    return out


def count_launches(fn):
    """Kernels launched by fn(), from the CUDA activity trace (CUPTI)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    counts = {}
    for e in prof.key_averages():
        if e.device_type.name != "CUDA" or e.key.startswith(("Memcpy", "Memset")):
            continue
        counts[e.key] = counts.get(e.key, 0) + e.count
    return counts


def short_kernel_name(k):
    k = k.replace("void ", "").replace("(anonymous namespace)::", "").split("(")[0]
    return k.split("::")[-1] if "::" in k else k


def time_fusion(sc, pairs, depths, normals, with_oracle):
    """RunFusion (main.cpp:502-633) of the last timed step's maps: hpm_fuse
    (consistency tests on the GPU, order-dependent masking on the host),
    wall clock with host maps in and the point list out; beside it the
    oracle's sequential restatement on one host core.  Not part of the
    depth-map metric, as the reference's own timing leaves fusion out."""
    import hpm_b200 as hb

    colors = [np.repeat(g[..., None], 3, -1) for g in sc.images]
    hb.fuse(sc.cams, depths, normals, colors, pairs)  # warm-up
    t0 = time.perf_counter()
    xyz, _, _ = hb.fuse(sc.cams, depths, normals, colors, pairs)
    dt = time.perf_counter() - t0
    npx = sum(d.size for d in depths)
    out = {"ms_per_scene": dt * 1e3, "points": int(len(xyz)), "mpix_per_s": npx / dt / 1e6,
           "what": "hpm_fuse of the scene's final depth/normal maps (11 views), host buffers in and out"}
    if with_oracle:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc

        t0 = time.perf_counter()
        oxyz, _, _ = orc.fuse(sc.cams, depths, normals, colors, pairs)
        odt = time.perf_counter() - t0
        out["cpu_oracle"] = {"ms_per_scene": odt * 1e3, "points": int(len(oxyz)), "mpix_per_s": npx / odt / 1e6,
                             "cores": 1, "kind": "port",
                             "sample": "the same maps through or_fuse (the reference's sequential loop in C)"}
    return out


def cpu_baseline():
    """Oracle on all host cores: one view of a 320x240 scene of the same
    recipe through the whole per-view flow (pass set A with the prior on
    every level, then the geometric passes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import flow as oflow

    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    sc, images, pairs = make_scene(0, 320, 240)
    ref = WORKLOAD["n_views"] // 2
    ids = [ref] + pairs[ref][1]
    imgs, cams = [images[i] for i in ids], sc.cams[ids]
    t0 = time.perf_counter()
    d, n, c, _ = oflow.process_problem(imgs, cams, seed=1, pyramid_levels=WORKLOAD["pyramid_levels"])
    # the sources' depth maps of a geometric pass: the scene's true depths
    # stand in for the sources' own pass-A maps (same per-pixel work)
    dm = [d] + [sc.gt_depth[i].astype(np.float32) for i in ids[1:]]
    for gi in range(WORKLOAD["geom_iterations"]):
        planes = np.concatenate([n, d[..., None]], -1)
        d, n, c, _ = oflow.process_problem(imgs, cams, seed=2 + gi, geom=True, multi_geometry=gi > 0, planes=planes,
                                           costs=c, depth_maps=dm)
        dm[0] = d
    dt = time.perf_counter() - t0
    return {"value": 320 * 240 / dt / 1e6, "unit": "depth Mpix/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port", "seconds": dt,
            "sample": f"one view of a 320x240 scene of the same recipe ({len(ids) - 1} sources): plain pass, "
                      f"{WORKLOAD['pyramid_levels'] + 1} prior levels, {WORKLOAD['geom_iterations']} geometric "
                      "passes, CPU oracle (oracle/hpm_oracle.c, OpenMP; OpenCV resize and Delaunay)"}


def measure_form(args, dist, ctx, sc, images, d_ptrs, pairs, stream, opts, profile=False):
    """One form of the scene step (opts: Context.run_scene keywords) under the
    bench's rules: W untimed warm-up steps; work counters and the kernel
    launch list from untimed re-runs of the first timed step; K timed steps
    with the images resident in HBM (CUDA events on the context's stream,
    max over ranks, SM clocks sampled meanwhile; with `profile`, CUDA events
    around every kernel group as well); K end-to-end steps through the public
    API from pinned host images to every view's depth, normal and cost maps
    in pinned host memory; the accuracy of the last end-to-end step's maps."""
    import torch

    w = WORKLOAD
    nv, W, H = w["n_views"], w["width"], w["height"]

    def step(seed):
        ctx.run_scene(d_ptrs, sc.cams, pairs, seed=seed, images_are_device=True, outputs=False, **opts)

    for i in range(args.warmup):
        step(1000 + i)
    # untimed re-runs of the first timed step: work counters (the counting
    # atomics slow the kernels down) and the kernel launch list
    ctx.count_enable(True)
    step(0)
    n_ncc, n_geom = ctx.count_read()
    ctx.count_enable(False)
    try:
        launches = count_launches(lambda: step(0))
        launch_src = "CUDA activity trace (torch.profiler/CUPTI) of an untimed re-run of one step"
    except Exception as e:  # noqa: BLE001 - the trace is evidence, not a requirement
        launches, launch_src = {}, f"activity trace unavailable: {e!r}"[:200]

    dist.barrier()
    torch.cuda.synchronize()
    with Clocks(dist.local) as clk:
        if profile:
            ctx.profile_enable(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            step(i)
        e1.record(stream)
        e1.synchronize()
        prof = ctx.profile_read() if profile else None
        if profile:
            ctx.profile_enable(False)
    dist.barrier()
    torch.cuda.synchronize()
    ms = dist.max(e0.elapsed_time(e1))

    pin_imgs = [torch.from_numpy(i).pin_memory() for i in images]
    outs = ([torch.empty((H, W), dtype=torch.float32).pin_memory() for _ in range(nv)],
            [torch.empty((H, W, 3), dtype=torch.float32).pin_memory() for _ in range(nv)],
            [torch.empty((H, W), dtype=torch.float32).pin_memory() for _ in range(nv)])
    out_np = tuple([t.numpy() for t in o] for o in outs)
    host_imgs = [p.numpy() for p in pin_imgs]
    dist.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(args.steps):
        ctx.run_scene(host_imgs, sc.cams, pairs, seed=i, outputs=out_np, **opts)
    f1.record(stream)
    f1.synchronize()
    dist.barrier()
    ms_e2e = dist.max(f0.elapsed_time(f1))
    npx = nv * W * H
    return {
        "value": job_mpix_per_s(dist.world, args.steps, npx, ms), "ms_per_step": ms / args.steps,
        "e2e": {"value": job_mpix_per_s(dist.world, args.steps, npx, ms_e2e), "unit": "depth Mpix/s",
                "ms_per_step": ms_e2e / args.steps, "h2d_bytes_per_step": int(sum(i.nbytes for i in images)),
                "d2h_bytes_per_step": int(npx * 4 * 5)},
        "accuracy": scene_accuracy(sc, dict(enumerate(out_np[0])), dict(enumerate(out_np[1]))),
        "clocks": clk.summary(), "ncc_windows": n_ncc, "geom_terms": n_geom, "launches": launches,
        "launch_src": launch_src, "profile": prof, "maps": out_np,
    }


def net_schedule(device):
    """The trained network's weights and the schedule stored with them
    (extra full-scale passes, geometric iterations, planar prior of the
    first full-scale pass, PatchMatch iterations per full-scale pass), or
    None without weights."""
    import priornet

    if not os.path.exists(priornet.WEIGHTS_FILE):
        return None
    net = priornet.Net.load(device=device)
    meta = dict(np.load(priornet.WEIGHTS_FILE))
    get = lambda k, d: int(meta[k]) if k in meta else d  # noqa: E731
    sched = {"pyramid_levels": get("extra_passes", 0), "geom_iterations": get("geom_iterations", 2),
             "planar_prior": get("prior", 1), "iterations": get("iterations", 3)}
    sched["geom_pass_iterations"] = get("geom_pass_iterations", sched["iterations"])
    return net, sched


def form_summary(m):
    """The figures of one measured form for the JSON line."""
    return {k: m[k] for k in ("value", "ms_per_step", "e2e", "accuracy", "clocks")} | {
        "gpu_launches_per_step": sum(m["launches"].values())}


def run_ours(args, dist):
    import torch

    import hpm_b200 as hb

    torch.cuda.set_device(dist.local)
    dev = f"cuda:{dist.local}"
    w = WORKLOAD
    sc, images, pairs = make_scene(seed=dist.rank)
    nv, W, H, S = w["n_views"], w["width"], w["height"], w["n_views"] - 1
    npx = W * H
    peak = hb.fp32_peak(dist.local)
    ctx = hb.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    d_imgs = [torch.from_numpy(i).to(dev) for i in images]
    d_ptrs = [t.data_ptr() for t in d_imgs]
    torch.cuda.synchronize()
    common = (args, dist, ctx, sc, images, d_ptrs, pairs, stream)

    # the plain form: the reference's flow (hpm_run_scene), CUDA events around
    # every kernel group of the timed steps for the roofline
    plain = measure_form(*common, dict(planar_prior=True, geom_iterations=w["geom_iterations"],
                                       pyramid_levels=w["pyramid_levels"]), profile=True)
    # the batched prior-net form with the schedule stored with the weights
    ns = net_schedule(dist.local)
    net = None
    if ns is not None:
        wts, sched = ns[0].weights(), ns[1]
        net = measure_form(*common, dict(sched, net=wts, batched=True))
        net["schedule"] = sched
    ctx.close()
    fusion = time_fusion(sc, pairs, plain["maps"][0], plain["maps"][1], dist.rank == 0 and dist.world == 1)

    # roofline of the dominant kernel pair (one red/black half-step), from the
    # plain form's profiled steps; the batched prior-net form runs the same
    # kernels (with the proposal as one more candidate)
    prof = plain["profile"]
    n_pass = nv * passes_per_view()
    prop_ms, prop_n = prof["propagate"]
    half_steps = prop_n // max(args.steps, 1)
    ncc_half = plain["ncc_windows"] - n_pass * npx * S  # k_init scores one hypothesis per pixel and pass
    flops_step = ncc_half * (TAPS * NCC_FLOPS_PER_TAP + FLOPS_PER_HYP_VIEW) + plain["geom_terms"] * GEOM_TERM_FLOPS
    prop_ms_step = prop_ms / args.steps
    achieved = flops_step / (prop_ms_step * 1e-3) / 1e12

    plain_acc = plain["accuracy"]["px_relerr_lt_1pct"]
    equal = net is not None and net["accuracy"]["px_relerr_lt_1pct"] >= plain_acc - 0.005
    head = net if equal else plain
    plain_step = ("hpm_run_scene: pass set A (plain pass, then one prior pass per pyramid level: support points, "
                  "Delaunay, raster, KNN prior, JBU) for every view, then the geometric iterations for every view; "
                  f"{n_pass} PatchMatch passes of 3 iterations")
    if net is not None:
        sc_ = net["schedule"]
        net_step = ("hpm_run_scene_batched_net: per problem a 1/4-scale plain pass (all problems in one graph), "
                    "the coarse planar prior and the BF16 network's plane proposal; then "
                    f"{1 + sc_['pyramid_levels']} full-scale pass(es) with the proposal as initial hypothesis and "
                    f"as a refinement candidate, then {sc_['geom_iterations']} geometric iteration(s); "
                    f"{sc_['iterations']} PatchMatch iterations per full-scale prior pass, "
                    f"{sc_['geom_pass_iterations']} per geometric pass; every pass of all problems one CUDA "
                    "graph")
        net_out = form_summary(net) | {
            "schedule": sc_, "step": net_step, "speedup_vs_plain": plain["ms_per_step"] / net["ms_per_step"],
            "e2e_speedup_vs_plain": plain["e2e"]["ms_per_step"] / net["e2e"]["ms_per_step"],
            "px_relerr_lt_1pct_minus_plain": net["accuracy"]["px_relerr_lt_1pct"] - plain_acc,
            "equal_accuracy": bool(equal),
            "network": "4 layers of 3x3 conv, 32 channels, BF16 on tcgen05 (FP32 accumulation in TMEM), at "
                       "1/4 scale; weights hpm-mvs_b200/priornet_weights.npz"}
    else:
        net_out = {"unavailable": "no trained weights (hpm-mvs_b200/priornet_weights.npz)"}
    line = {
        "metric": METRIC, "value": head["value"], "unit": "depth Mpix/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene, hpm-mvs_b200/synthetic.py; one scene per rank)",
        "config": {"workload": workload_name(), "width": W, "height": H, "views": nv, "sources": S,
                   "scene": f"{w['n_planes']} planes + {w['n_spheres']} spheres, "
                            f"{int(w['low_texture'] * 100)}% low-texture",
                   "form": "batched prior-net form (its %px within 0.5 pp of the plain form's)" if equal else
                           "plain form (the batched prior-net form is not within 0.5 pp of its %px, or has no "
                           "weights)",
                   "step": net_step if equal else plain_step,
                   "pyramid_levels": w["pyramid_levels"] + 1, "knn_k": 6,
                   "l2": f"inputs larger than L2 ({nv} views x {W}x{H} float images + texture arrays = "
                         f"{2 * nv * npx * 4 / 1e6:.0f} MB, plus the per-view depth/normal/cost maps)",
                   "parallelism": f"one scene per GPU, {dist.world} GPU(s)"},
        "accuracy": head["accuracy"],
        "clocks": head["clocks"],
        "e2e": head["e2e"],
        "gpu_launches": sum(head["launches"].values()) * args.steps,
        "gpu_launches_per_step": {short_kernel_name(k): v
                                  for k, v in sorted(head["launches"].items(), key=lambda x: -x[1])},
        "gpu_launches_source": head["launch_src"],
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "traffic": TRAFFIC_BYTES_PER_PX_HALF_STEP * npx,
                     "traffic_note": "DRAM bytes per half-step (k_prop_dirs + k_prop_refine) from the ncu capture "
                                     "of bench.py --pass-case at 1600x1200 (10 sources), per pixel of the "
                                     "workload",
                     "kernel": "k_prop_dirs + k_prop_refine (one red/black half-step), timed with CUDA events "
                               "in the plain form's timed steps",
                     "peak_source": "measured FP32 FMA probe (hpm_fp32_peak) of measured; "
                                    "MEASURED_PEAKS.json has no FP32 figure",
                     "half_step_ms": prop_ms_step / max(half_steps, 1), "half_steps_per_step": half_steps,
                     "propagate_ms_per_step": prop_ms_step,
                     "propagate_share": prop_ms_step / plain["ms_per_step"],
                     # PM-only rate: the plain form's depth pixels per second of its half-step kernels
                     "pm_only_mpix_per_s": nv * npx / (max(prop_ms_step, 1e-9) * 1e-3) / 1e6,
                     "ncc_windows_per_step": ncc_half, "geom_terms_per_step": plain["geom_terms"],
                     "flops_per_ncc_window": TAPS * NCC_FLOPS_PER_TAP + FLOPS_PER_HYP_VIEW},
        "plain_form": form_summary(plain) | {"step": plain_step},
        "batched_prior_net_form": net_out,
        "fusion": fusion,
        "impl": "ours",
    }
    return line


def run_batched(args, dist):
    """The batched form against the per-problem driver on the same scene of
    uneven view sizes: both device-resident, CUDA events on the context's
    stream, whole-scene steps."""
    import torch

    import hpm_b200 as hb

    torch.cuda.set_device(dist.local)
    dev = f"cuda:{dist.local}"
    w = WORKLOAD
    sc, images, pairs = make_scene(seed=dist.rank)
    npx = sum(i.size for i in images)
    ctx = hb.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    d_imgs = [torch.from_numpy(i).to(dev) for i in images]
    d_ptrs = [t.data_ptr() for t in d_imgs]
    torch.cuda.synchronize()
    opts = dict(geom_iterations=w["geom_iterations"], pyramid_levels=w["pyramid_levels"], images_are_device=True)
    res = {}
    for form, batched in (("batched", True), ("per_problem", False)):
        for i in range(args.warmup):
            ctx.run_scene(d_ptrs, sc.cams, pairs, seed=500 + i, outputs=False, batched=batched, **opts)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(dist.local) as clk:
            e0.record(stream)
            for i in range(args.steps):
                ctx.run_scene(d_ptrs, sc.cams, pairs, seed=i, outputs=False, batched=batched, **opts)
            e1.record(stream)
            e1.synchronize()
        dist.barrier()
        ms = dist.max(e0.elapsed_time(e1)) / args.steps
        d, n, _ = ctx.run_scene(d_ptrs, sc.cams, pairs, seed=0, batched=batched, **opts)
        res[form] = {"ms_per_step": ms, "value": job_mpix_per_s(dist.world, 1, npx, ms),
                     "accuracy": scene_accuracy(sc, dict(enumerate(d)), dict(enumerate(n))), "clocks": clk.summary()}
    ctx.close()
    b = res["batched"]
    return {
        "metric": METRIC, "value": b["value"], "unit": "depth Mpix/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": b["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene of uneven view sizes)",
        "config": {"workload": workload_name(), "views": w["n_views"], "sizes": "8x1920x1080, 8x1600x1200, 8x960x540",
                   "sources": 10, "pyramid": "reference rule per view size", "geom_iterations": w["geom_iterations"],
                   "form": "hpm_run_scene_batched: every pass of all 24 problems one CUDA graph of per-problem "
                           "kernel chains (updated per pass, replayed), half-step tiles tuned per view size"},
        "accuracy": b["accuracy"], "clocks": b["clocks"],
        "per_problem_form": res["per_problem"], "speedup_vs_per_problem": res["per_problem"]["ms_per_step"] /
        b["ms_per_step"], "impl": "ours",
    }


def run_acmm(args, dist):
    """The ACMM+NESP variant (hpm_run_scene_acmm: 800x600, then 1600x1200
    started from the upsampled maps, 2 geometric iterations at each scale)
    beside the plain HPM form (hpm_run_scene) on the same scene: host images
    in and every view's maps out per step, CUDA events on the context's
    stream."""
    import torch

    import hpm_b200 as hb

    torch.cuda.set_device(dist.local)
    dev = f"cuda:{dist.local}"
    w = WORKLOAD
    sc, images, pairs = make_scene(seed=dist.rank)
    npx = sum(i.size for i in images)
    ctx = hb.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    forms = {
        "acmm_nesp": lambda seed: ctx.run_scene_acmm(images, sc.cams, pairs, seed=seed,
                                                     geom_iterations=w["geom_iterations"]),
        "plain_hpm": lambda seed: ctx.run_scene(images, sc.cams, pairs, seed=seed,
                                                geom_iterations=w["geom_iterations"],
                                                pyramid_levels=w["pyramid_levels"]),
    }
    res = {}
    for name, run in forms.items():
        for i in range(args.warmup):
            run(500 + i)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(dist.local) as clk:
            e0.record(stream)
            for i in range(args.steps):
                d, n, _ = run(i)
            e1.record(stream)
            e1.synchronize()
        dist.barrier()
        ms = dist.max(e0.elapsed_time(e1)) / args.steps
        res[name] = {"ms_per_step": ms, "value": job_mpix_per_s(dist.world, 1, npx, ms),
                     "accuracy": scene_accuracy(sc, dict(enumerate(d)), dict(enumerate(n))), "clocks": clk.summary()}
    ctx.close()
    a = res["acmm_nesp"]
    return {
        "metric": "depth Mpix/s of the ACMM+NESP variant on 1 B200", "value": a["value"], "unit": "depth Mpix/s",
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene)",
        "config": {"workload": f"ACMM+NESP variant on {workload_name()}",
                   "scales": "800x600, then 1600x1200 (halvings until the longer side is at most 1000)",
                   "form": "hpm_run_scene_acmm: plain pass and geometric iterations at the coarse scale; JBU of the "
                           "geometric depth and the normals, hierarchy pass and geometric iterations at full scale"},
        "accuracy": a["accuracy"], "clocks": a["clocks"], "plain_hpm_form": res["plain_hpm"],
        "speedup_vs_plain_hpm": res["plain_hpm"]["ms_per_step"] / a["ms_per_step"], "impl": "ours",
    }


def run_view_shards(args, dist):
    """One scene, its problems split over the ranks (scene_dist.py): timed
    from the host images to every rank's final maps on the host."""
    import torch
    import torch.distributed as tdist

    import hpm_b200 as hb
    import scene_dist

    torch.cuda.set_device(dist.local)
    dev = f"cuda:{dist.local}"
    w = WORKLOAD
    sc, images, pairs = make_scene(seed=0)
    nv, W, H = w["n_views"], w["width"], w["height"]
    shapes = {v: (H, W) for v in range(nv)}
    pg = tdist if dist.pg else None
    ctx = hb.Context(dist.local)

    def step(seed):
        solver = scene_dist.GpuSolver(ctx, images, sc.cams, pairs, seed=seed, pyramid_levels=w["pyramid_levels"],
                                      device=dev)
        mine, _ = scene_dist.run_scene_sharded(solver, pairs, shapes, geom_iterations=w["geom_iterations"], dist=pg)
        return {v: m[0].cpu().numpy() for v, m in mine.items()}

    for i in range(args.warmup):
        step(1000 + i)
    dist.barrier()
    torch.cuda.synchronize()
    with Clocks(dist.local) as clk:
        t0 = time.perf_counter()
        for i in range(args.steps):
            out = step(i)
        torch.cuda.synchronize()
        elapsed = (time.perf_counter() - t0) * 1e3
    dist.barrier()
    ms = dist.max(elapsed)
    ctx.close()
    value = args.steps * nv * W * H / (ms * 1e-3) / 1e6
    return {
        "metric": METRIC, "value": value, "unit": "depth Mpix/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, shared by all ranks)",
        "config": {"workload": workload_name(), "width": W, "height": H, "views": nv,
                   "parallelism": f"views of one scene split over {dist.world} GPU(s); all-gather of depth maps "
                                  "(NCCL) before each geometric iteration",
                   "l2": "inputs larger than L2 (see the default mode)"},
        "accuracy": scene_accuracy(sc, out),
        "clocks": clk.summary(),
        "e2e": {"value": value, "unit": "depth Mpix/s", "h2d_bytes_per_step": int(sum(i.nbytes for i in images)),
                "d2h_bytes_per_step": int(len(out) * W * H * 4),
                "note": "host images in, each rank's final depth maps out; timed on the host around whole steps"},
        "impl": "ours",
    }


def run_pass_case(args):
    """Plain passes of reference view n/2 of the bench scene, for ncu captures
    of the half-step kernels."""
    import hpm_b200 as hb
    import synthetic as syn

    sc, images, pairs = make_scene(0)
    ref = WORKLOAD["n_views"] // 2
    ids = [ref] + pairs[ref][1]
    cam = sc.cams[ref]
    dmin, dmax = cam["depth_min"] * np.float32(0.6), cam["depth_max"] * np.float32(1.2)
    with hb.Context() as ctx:
        ctx.set_views([images[i] for i in ids], sc.cams[ids])
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=99))
        ctx.profile_enable(True)
        for i in range(args.steps):
            ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=i))
        prof = ctx.profile_read()
        ctx.profile_enable(False)
        planes, _ = ctx.get_result()
    ms, n = prof["propagate"]
    return {"case": f"plain passes of view {ref}, {WORKLOAD['width']}x{WORKLOAD['height']}, {len(ids) - 1} sources",
            "half_step_ms": ms / max(n, 1), "init_ms": prof["init"][0] / max(prof["init"][1], 1),
            "px_relerr_lt_1pct": float(syn.depth_accuracy(planes[..., 3], sc.gt_depth[ref]))}


def run_flow_case(args):
    """hpm_process_problem of reference view n/2 of the bench scene (plain
    pass, then the prior passes of every pyramid level), then hpm_fuse of
    the scene's ground-truth depth and normal maps, for ncu captures of
    k_init, k_support_blocks, k_tri_planes, k_tri_raster, k_knn_prior,
    k_prior_coarse, k_jbu, k_filter and k_fuse_pairs."""
    import hpm_b200 as hb

    sc, images, pairs = make_scene(0)
    ref = WORKLOAD["n_views"] // 2
    ids = [ref] + pairs[ref][1]
    out = {"case": f"ProcessProblem of view {ref} ({WORKLOAD['width']}x{WORKLOAD['height']}, {len(ids) - 1} "
                   f"sources, {WORKLOAD['pyramid_levels'] + 1}-level prior pyramid), then fusion of "
                   f"{WORKLOAD['n_views']} views"}
    with hb.Context() as ctx:
        ctx.set_views([images[i] for i in ids], sc.cams[ids])
        t0 = time.perf_counter()
        d, _, _, _ = ctx.process_problem(seed=1, pyramid_levels=WORKLOAD["pyramid_levels"])
        out["process_problem_ms"] = (time.perf_counter() - t0) * 1e3
    depths = [g.astype(np.float32) for g in sc.gt_depth]
    normals = [g.astype(np.float32) for g in sc.gt_normal]
    colors = [np.repeat(g[..., None], 3, -1) for g in sc.images]
    t0 = time.perf_counter()
    xyz, _, _ = hb.fuse(sc.cams, depths, normals, colors, pairs)
    out["fuse_ms"] = (time.perf_counter() - t0) * 1e3
    out["points"] = int(len(xyz))
    return out


def run_net_case(args):
    """Training steps of the proposal network on one 400x300 input (the
    coarse size of a 1600x1200 view), for ncu captures of k_conv3x3 and
    k_conv_wgrad: CUDA events around --steps steps after one warm-up."""
    import torch

    import priornet

    net = priornet.Net(0, seed=3)
    tr = priornet.Trainer(net)
    h, w = 300, 400
    g = torch.Generator(device="cuda").manual_seed(5)
    x0 = torch.randn(h, w, 16, device="cuda", generator=g).to(torch.bfloat16)
    td = torch.rand(h, w, device="cuda", generator=g) * 4 + 2
    tn = torch.nn.functional.normalize(torch.randn(h, w, 3, device="cuda", generator=g), dim=-1)
    tm = torch.ones(h, w, dtype=torch.uint8, device="cuda")

    def one():
        tr.accumulate(x0, td, tn, tm, 1.2, 9.6, 1.0 / (h * w))
        tr.apply()

    one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        one()
    e1.record()
    e1.synchronize()
    return {"case": "proposal network training steps at 400x300 (4 layers of 3x3 conv, 32 channels, BF16)",
            "ms_per_training_step": e0.elapsed_time(e1) / args.steps, "loss": float(tr.take_loss())}


def run_reference(args, dist):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    if not orc.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libhpm_ref.so (reference HPM.cu for sm_100a) "
                                                    "was not built: `make -C oracle ref` needs the reference tree"}
    import torch

    import flow as oflow

    torch.cuda.set_device(dist.local)
    w = WORKLOAD
    sc, images, pairs = make_scene(seed=0)
    nv, W, H = w["n_views"], w["width"], w["height"]
    npx = W * H
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))

    def quiet(fn):
        # the reference prints "iteration: i" from RunPatchMatch (HPM.cu:1943)
        sys.stdout.flush()
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        try:
            return fn()
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)

    def problem(v):
        ids = [v] + pairs[v][1]
        return ids, [images[i] for i in ids], sc.cams[ids]

    def pass_a(v, seed):
        ids, imgs, cams = problem(v)
        return oflow.process_problem(imgs, cams, seed=seed, pyramid_levels=w["pyramid_levels"], backend="reference")

    def geom(v, seed, gi, d_src, n, c):
        ids, imgs, cams = problem(v)
        planes = np.concatenate([n, d_src[v][..., None]], -1)
        return oflow.process_problem(imgs, cams, seed=seed, geom=True, multi_geometry=gi > 0, planes=planes,
                                     costs=c, depth_maps=[d_src[i] for i in ids], backend="reference")

    # untimed: pass set A and the first geometric iteration of every view, the
    # maps the sampled views' geometric passes read
    depth_a, normal, cost, depth_g = {}, {}, {}, {}
    for v in range(nv):
        depth_a[v], normal[v], cost[v], _ = quiet(lambda: pass_a(v, 100 + v))
    for v in range(nv):
        depth_g[v], _, _, _ = quiet(lambda: geom(v, 200 + v, 0, depth_a, normal[v], cost[v]))

    def step(i):
        """The whole per-view flow of view i mod n: pass set A, then every
        geometric iteration (the sources' maps from the untimed setup)."""
        v = i % nv
        d, n, c, _ = pass_a(v, 300 + i)
        src = dict(depth_a)
        src[v] = d
        for gi in range(w["geom_iterations"]):
            d, n, c, _ = geom(v, 1000 + i, gi, src, n, c)
            src = dict(depth_g) if gi == 0 else src
            src[v] = d
        return v, d, n

    # the reference's kernels one by one (untimed region): a plain
    # RunPatchMatch of view 0 at the workload's size with CUDA events around
    # each of its launches (the shim's timed copy of HPM.cu:1906-1957)
    ids0, imgs0, cams0 = problem(0)
    cam0 = cams0[0]
    quiet(lambda: orc.ref_run_patchmatch(imgs0, cams0, depth_min=cam0["depth_min"] * 0.6,
                                         depth_max=cam0["depth_max"] * 1.2, seed=5, timed=True))
    _, _, kt = quiet(lambda: orc.ref_run_patchmatch(imgs0, cams0, depth_min=cam0["depth_min"] * 0.6,
                                                   depth_max=cam0["depth_max"] * 1.2, seed=6, timed=True))
    kernel_ms = {"init": kt["init"], "half_step_mean": float(np.mean(kt["half_steps"])),
                 "half_steps": kt["half_steps"], "depth_normal": kt["depth_normal"], "filters": kt["filter"],
                 "what": f"one plain RunPatchMatch of view 0 ({W}x{H}, {len(ids0) - 1} sources), the reference's "
                         "kernels timed one by one with CUDA events"}

    # warm-up on the last views, timed steps from view 0 on (their accuracy
    # compares with the per-view figures of the product's line)
    for i in range(args.warmup):
        quiet(lambda: step(nv - 1 - i % nv))
    torch.cuda.synchronize()
    done, done_n = {}, {}
    with Clocks(dist.local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            v, d, n = quiet(lambda: step(i))
            done[v] = d
            done_n[v] = n
        e1.record()
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    value = args.steps * npx / (ms * 1e-3) / 1e6
    sample = (f"one view per step (timed step i: view i mod {nv}) of the {nv}-view scene: pass set A with the prior on "
              f"{w['pyramid_levels'] + 1} levels, then {w['geom_iterations']} geometric passes; the reference's "
              "HPM.cu kernels (oracle/_ref, compiled unchanged for sm_100a) on the B200 for the PatchMatch passes "
              "and the JBU; host stages on the CPU: OpenCV resize and Delaunay, the oracle's C restatement of the "
              f"support points, raster, KNN prior and prior assembly (OpenMP, {os.environ['OMP_NUM_THREADS']} "
              "threads)")
    return {
        "metric": METRIC, "value": value, "unit": "depth Mpix/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": workload_name(), "width": W, "height": H, "views": nv, "sources": nv - 1,
                   "step": "the reference's per-view flow (main.cpp:35-499 for pass set A, main.cpp:662-674 for the "
                           "geometric iterations) on one view"},
        "accuracy": scene_accuracy(sc, done, done_n),
        "reference_kernel_ms": kernel_ms,
        "clocks": clk.summary(),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "depth Mpix/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "depth Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    dist = Dist(args.gpus)
    try:
        if args.pass_case:
            if dist.rank == 0:
                print(json.dumps(run_pass_case(args)), flush=True)
            return
        if args.flow_case:
            if dist.rank == 0:
                print(json.dumps(run_flow_case(args)), flush=True)
            return
        if args.net_case:
            if dist.rank == 0:
                print(json.dumps(run_net_case(args)), flush=True)
            return
        if args.impl == "reference":
            if dist.rank != 0:
                return
            line = run_reference(args, dist)
        elif args.shard == "views":
            line = run_view_shards(args, dist)
        elif args.config == "batched":
            line = run_batched(args, dist)
        elif args.config == "acmm":
            line = run_acmm(args, dist)
        else:
            line = run_ours(args, dist)
            if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
                line["cpu_baseline"] = cpu_baseline()
        if dist.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark of the B200-native HPM-MVS PatchMatch path.

One JSON line on rank 0.  A *step* is the depth estimation of one reference
view of the workload below through the product's C ABI.  Metric: depth
Mpix/s (reference-view pixels at processed resolution per second).

  value   steps with the views already resident in HBM (hpm_run_patchmatch)
  e2e     the same steps through the public API from pinned host memory:
          hpm_set_views (H2D) + hpm_run_patchmatch + hpm_get_result (D2H)
  roofline  the dominant kernel pair (one red/black half-step: site/direction
          kernel + selection/refinement kernel) against the measured FP32 FMA
          peak; algorithmic FLOPs = NCC taps x 34 + 80 per (hypothesis, view)
  cpu_baseline  the CPU oracle (C restatement of the reference, OpenMP over
          all host cores) on a bounded sample with the same per-pixel work

--impl reference times the reference's own HPM.cu (oracle/_ref: compiled
unchanged for sm_100a) through its HPM::RunPatchMatch on the same workload.

Multi-GPU (torchrun): reference views shard over ranks with no data-path
collective (weak scaling); the elapsed time is the max over ranks.
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
WORKLOAD = dict(name="plain HPM PatchMatch pass, 1600x1200, 10 sources", width=1600, height=1200, n_views=11,
                n_planes=20, n_spheres=5, low_texture=0.40)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--size", default=None,
                    help="WxH override of the workload's resolution (profiling captures use a smaller case)")
    args = ap.parse_args()
    if args.size:
        w, h = (int(x) for x in args.size.lower().split("x"))
        WORKLOAD.update(width=w, height=h, name=f"plain HPM PatchMatch pass, {w}x{h}, 10 sources")
    return args


class Dist:
    def __init__(self, n):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=__import__("torch").device("cuda", self.local))
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

        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local}")
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


def make_workload(seed):
    import synthetic as syn

    w = WORKLOAD
    sc = syn.make_scene(seed, w["width"], w["height"], w["n_views"], n_planes=w["n_planes"],
                        n_spheres=w["n_spheres"], low_texture=w["low_texture"])
    ref = w["n_views"] // 2
    imgs, cams = syn.view_set(sc, ref)
    return sc, ref, imgs, cams, sc.depth_min * 0.6, sc.depth_max * 1.2


def cpu_baseline():
    """Oracle on all host cores over a 320x240 crop of the workload's scene
    geometry with the same number of source views (same per-pixel work)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import synthetic as syn

    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    w = WORKLOAD
    sc = syn.make_scene(0, 320, 240, w["n_views"], n_planes=w["n_planes"], n_spheres=w["n_spheres"],
                        low_texture=w["low_texture"])
    imgs, cams = syn.view_set(sc, w["n_views"] // 2)
    t0 = time.perf_counter()
    orc.run_patchmatch(imgs, cams, depth_min=sc.depth_min * 0.6, depth_max=sc.depth_max * 1.2, seed=1)
    dt = time.perf_counter() - t0
    return {"value": 320 * 240 / dt / 1e6, "unit": "depth Mpix/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port", "seconds": dt,
            "sample": "one full PatchMatch pass of a 320x240 view with 10 sources (same scene recipe, same "
                      "per-pixel work as the 1600x1200 workload), CPU oracle (oracle/hpm_oracle.c), OpenMP"}


def run_ours(args, dist):
    import torch

    import hpm_b200 as hb
    import synthetic as syn

    torch.cuda.set_device(dist.local)
    sc, ref, imgs, cams, dmin, dmax = make_workload(seed=dist.rank)
    W, H, S = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["n_views"] - 1
    npx = W * H
    peak = hb.fp32_peak(dist.local)
    ctx = hb.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dist.local}")
    # pinned host copies of the step inputs and outputs for the end-to-end leg
    pin_imgs = [torch.from_numpy(i).pin_memory() for i in imgs]
    pin_planes = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
    pin_costs = torch.empty((H, W), dtype=torch.float32).pin_memory()
    ctx.set_views([p.numpy() for p in pin_imgs], cams)
    for i in range(args.warmup):
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=1000 + i))
    # cost-vector evaluations of one pass (deterministic per seed), for the roofline
    ctx.count_enable(True)
    ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=0))
    n_cv, n_geom = ctx.count_read()
    ctx.count_enable(False)

    dist.barrier()
    torch.cuda.synchronize()
    with Clocks(dist.local) as clk:
        ctx.profile_enable(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(args.steps):
            ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=i))
        e1.record(stream)
        e1.synchronize()
        prof = ctx.profile_read()
        ctx.profile_enable(False)
    dist.barrier()
    torch.cuda.synchronize()
    ms = dist.max(e0.elapsed_time(e1))
    planes, costs = ctx.get_result()
    acc = syn.depth_accuracy(planes[..., 3], sc.gt_depth[ref])
    nerr = syn.normal_error_deg(planes[..., :3], sc.gt_normal[ref], sc.gt_depth[ref])

    # end to end through the public API, pinned host buffers in and out
    dist.barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for i in range(args.steps):
        ctx.set_views([p.numpy() for p in pin_imgs], cams)
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=i))
        lp, lc = pin_planes.numpy(), pin_costs.numpy()
        rc = hb.lib().hpm_get_result(ctx.handle, hb._p(lp), hb._p(lc))
        if rc != hb.HPM_OK:
            raise hb.HpmError("hpm_get_result failed")
    f1.record(stream)
    f1.synchronize()
    dist.barrier()
    ms_e2e = dist.max(f0.elapsed_time(f1))
    ctx.close()

    launches_per_pass = 1 + 6 * 2 + 3
    prop_ms, prop_n = prof["propagate"]
    half_ms = prop_ms / max(prop_n, 1)
    cv_per_half = (n_cv - npx) / 6.0
    flops_per_cv = S * (36 * 34 + 80)
    achieved = cv_per_half * flops_per_cv / (half_ms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": dist.world * args.steps * npx / (ms * 1e-3) / 1e6, "unit": "depth Mpix/s",
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene, see hpm-mvs_b200/synthetic.py)",
        "config": {"workload": WORKLOAD["name"], "width": W, "height": H, "sources": S,
                   "scene": f"{WORKLOAD['n_planes']} planes + {WORKLOAD['n_spheres']} spheres, "
                            f"{int(WORKLOAD['low_texture'] * 100)}% low-texture",
                   "step": "one plain PatchMatch pass of one reference view: init, 3 red/black iterations, "
                           "depth/normal, checkerboard filter (HPM::RunPatchMatch)",
                   "l2": "inputs larger than L2 (11 views x 1600x1200 float images + texture arrays = 169 MB)",
                   "parallelism": f"views sharded over {dist.world} GPU(s)"},
        "accuracy": {"px_relerr_lt_1pct": acc, "median_normal_err_deg": nerr},
        "clocks": clk.summary(),
        "e2e": {"value": dist.world * args.steps * npx / (ms_e2e * 1e-3) / 1e6, "unit": "depth Mpix/s",
                "h2d_bytes_per_step": int(sum(i.nbytes for i in imgs)), "d2h_bytes_per_step": int(npx * 20)},
        "gpu_launches": launches_per_pass * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "k_prop_dirs + k_prop_refine (one half-step)",
                     "peak_source": "measured FP32 FMA probe (hpm_fp32_peak); MEASURED_PEAKS.json has no FP32 figure",
                     "half_step_ms": half_ms, "cost_vectors_per_half_step": cv_per_half,
                     "flops_per_cost_vector": flops_per_cv},
        "impl": "ours",
    }
    return line


def run_reference(args, dist):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import synthetic as syn

    if not orc.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libhpm_ref.so (reference HPM.cu for sm_100a) "
                                                    "was not built: `make -C oracle ref` needs the reference tree"}
    import torch

    torch.cuda.set_device(dist.local)
    sc, ref, imgs, cams, dmin, dmax = make_workload(seed=dist.rank)
    W, H = WORKLOAD["width"], WORKLOAD["height"]
    npx = W * H

    def call(seed):
        # the reference prints "iteration: i" from RunPatchMatch (HPM.cu:1943)
        sys.stdout.flush()
        saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        try:
            return orc.ref_run_patchmatch(imgs, cams, depth_min=dmin, depth_max=dmax, seed=seed)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
            os.close(devnull)

    for i in range(args.warmup):
        call(1000 + i)
    torch.cuda.synchronize()
    with Clocks(dist.local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            planes, costs = call(i)
        e1.record()
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    value = args.steps * npx / (ms * 1e-3) / 1e6
    acc = syn.depth_accuracy(planes[..., 3], sc.gt_depth[ref])
    return {
        "metric": METRIC, "value": value, "unit": "depth Mpix/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": WORKLOAD["name"], "width": W, "height": H, "sources": WORKLOAD["n_views"] - 1,
                   "step": "the reference's CudaSpaceInitialization-equivalent upload, HPM::RunPatchMatch "
                           "(HPM.cu:1906-1957, with its per-launch device syncs) and result download"},
        "accuracy": {"px_relerr_lt_1pct": acc},
        "clocks": clk.summary(),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "depth Mpix/s", "cores": 1, "kind": "reference",
                         "sample": "the reference's own HPM.cu kernels, compiled unchanged for sm_100a and run on "
                                   "the B200 (the reference has no CPU implementation of this path); one host "
                                   "thread drives it"},
        "e2e": {"value": value, "unit": "depth Mpix/s", "h2d_bytes_per_step": int(sum(i.nbytes for i in imgs)),
                "d2h_bytes_per_step": int(npx * 20)},
    }


def main():
    args = parse_args()
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            if dist.rank != 0:
                return
            line = run_reference(args, dist)
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

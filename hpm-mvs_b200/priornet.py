"""The prior-net form's proposal network: parameters, training, and the
weights the scene driver (hpm_run_scene_net) runs.

Every kernel is the library's own (hpm_net.cu, hpm_priornet.cu): the 3x3
convolutions forward, their data and weight gradients on the tcgen05 tensor
cores, the loss and the Adam step.  PyTorch only holds the device buffers.

Network: 4 layers of 3x3 convolutions, 32 channels, BF16 operands and
activations, FP32 accumulation and master weights.
  input   16 channels at 1/4 scale (hpm_net_coarse_inputs): gray image, the
          coarse plain pass's depth, reference-frame normal and confidence,
          the coarse planar prior's depth and presence
  L1 16->32 ReLU, L2 32->32 ReLU, L3 32->32 ReLU, L4 32->16 linear
  head    depth = dmin + sigmoid(o0) (dmax - dmin), normal = normalise(o1..o3)

Training data: seeded synthetic scenes of config 2's recipe; the targets are
the plain method's final depth and normal maps where the multi-view
consistency test of the reference's fusion passes (hpm_net_targets).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import hpm_b200 as hb

LAYERS = [(16, 32), (32, 32), (32, 32), (32, 16)]
WEIGHTS_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "priornet_weights.npz")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _ok(rc, what):
    if rc != hb.HPM_OK:
        raise hb.HpmError(f"{what}: {hb.STATUS_NAMES.get(rc, rc)}")


class Net:
    """FP32 master parameters on the device, with their packed BF16 images."""

    def __init__(self, device=0, seed=0, weights=None):
        import torch

        self.dev = torch.device("cuda", device)
        g = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for li, (ci, co) in enumerate(LAYERS):
            if weights is not None:
                w = torch.from_numpy(np.asarray(weights[f"w{li}"], np.float32))
                b = torch.from_numpy(np.asarray(weights[f"b{li}"], np.float32))
            else:
                w = torch.randn(co, ci, 3, 3, generator=g) * (2.0 / (9 * ci)) ** 0.5
                b = torch.zeros(co)
                if li == len(LAYERS) - 1:
                    w *= 0.1
            self.w.append(w.to(self.dev).contiguous())
            self.b.append(b.to(self.dev).contiguous())
        self.packed = [torch.empty(9 * ci * co, dtype=torch.bfloat16, device=self.dev) for ci, co in LAYERS]
        self.packed_t = [torch.empty(9 * ci * co, dtype=torch.bfloat16, device=self.dev) for ci, co in LAYERS]
        self.repack()

    @classmethod
    def load(cls, path=WEIGHTS_FILE, device=0):
        return cls(device=device, weights=dict(np.load(path)))

    def save(self, path=WEIGHTS_FILE, **meta):
        arrs = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        arrs.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        arrs.update({k: np.asarray(v) for k, v in meta.items()})
        np.savez_compressed(path, **arrs)

    def repack(self, stream=None):
        for li, (ci, co) in enumerate(LAYERS):
            _ok(hb.lib().hpm_net_pack_weights(_ptr(self.w[li]), co, ci, 0, _ptr(self.packed[li]), stream), "pack")
            if li > 0:
                _ok(hb.lib().hpm_net_pack_weights(_ptr(self.w[li]), co, ci, 1, _ptr(self.packed_t[li]), stream),
                    "pack")

    def weights(self) -> hb.HpmNetWeights:
        """The device pointers hpm_run_scene_net takes (valid while self lives)."""
        wts = hb.HpmNetWeights()
        for li in range(len(LAYERS)):
            wts.packed[li] = self.packed[li].data_ptr()
            wts.bias[li] = self.b[li].data_ptr()
        return wts


class Trainer:
    """Adam on the network with the library's kernels; one step = the summed
    gradients of a batch of views."""

    def __init__(self, net: Net, lr=1e-3, lam=0.5):
        import torch

        self.net, self.lr, self.lam = net, lr, lam
        self.gw = [torch.zeros_like(w) for w in net.w]
        self.gb = [torch.zeros_like(b) for b in net.b]
        self.m = [torch.zeros_like(t) for t in net.w + net.b]
        self.v = [torch.zeros_like(t) for t in net.w + net.b]
        self.step_no = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=net.dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=net.dev)
        self._buf = {}

    def _bufs(self, h, w):
        import torch

        key = (h, w)
        if key not in self._buf:
            d = self.net.dev
            self._buf = {key: dict(a=[torch.empty(h, w, 32, dtype=torch.bfloat16, device=d) for _ in range(3)],
                                   out=torch.empty(h, w, 16, dtype=torch.float32, device=d),
                                   dy=[torch.empty(h, w, c, dtype=torch.bfloat16, device=d) for c in (32, 32, 32, 16)])}
        return self._buf[key]

    def forward(self, x0, h, w, bufs):
        lib, n = hb.lib(), self.net
        src = x0
        for li, (ci, co) in enumerate(LAYERS):
            last = li == len(LAYERS) - 1
            dst = bufs["out"] if last else bufs["a"][li]
            _ok(lib.hpm_net_conv3x3(_ptr(src), h, w, ci, _ptr(n.packed[li]), _ptr(n.b[li]), co, 1 if last else 0,
                                    None, _ptr(dst), 1, _ptr(self.err), None), "conv")
            src = dst
        return bufs["out"]

    def accumulate(self, x0, t_depth, t_normal, t_mask, dmin, dmax, inv_count):
        """Forward, loss and backward of one view (coarse h x w); gradients
        add to the trainer's buffers."""
        lib, n = hb.lib(), self.net
        h, w = x0.shape[:2]
        bufs = self._bufs(h, w)
        out = self.forward(x0, h, w, bufs)
        dy = bufs["dy"][3]
        _ok(lib.hpm_net_loss(_ptr(out), _ptr(t_depth), _ptr(t_normal), _ptr(t_mask), h * w, ctypes.c_float(dmin),
                             ctypes.c_float(dmax), ctypes.c_float(self.lam), ctypes.c_float(inv_count), _ptr(dy),
                             _ptr(self.loss), None), "loss")
        acts = [x0] + bufs["a"]
        for li in range(len(LAYERS) - 1, -1, -1):
            ci, co = LAYERS[li]
            _ok(lib.hpm_net_conv_wgrad(_ptr(acts[li]), _ptr(dy), h, w, ci, co, _ptr(self.gw[li]), _ptr(self.gb[li]),
                                       _ptr(self.err), None), "wgrad")
            if li > 0:
                nxt = bufs["dy"][li - 1]
                _ok(lib.hpm_net_conv3x3(_ptr(dy), h, w, co, _ptr(n.packed_t[li]), None, ci, 2, _ptr(acts[li]),
                                        _ptr(nxt), 1, _ptr(self.err), None), "dgrad")
                dy = nxt

    def apply(self):
        lib = hb.lib()
        self.step_no += 1
        params = self.net.w + self.net.b
        grads = self.gw + self.gb
        for p, g, m, v in zip(params, grads, self.m, self.v):
            _ok(lib.hpm_net_adam(_ptr(p), _ptr(g), _ptr(m), _ptr(v), p.numel(), ctypes.c_float(self.lr),
                                 ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), self.step_no, None),
                "adam")
        self.net.repack()

    def take_loss(self):
        val = float(self.loss.item())
        self.loss.zero_()
        if int(self.err.item()):
            raise hb.HpmError("a tensor-core kernel's bounded wait ran out")
        return val


def view_samples(ctx, images, cams, pairs, depths, normals, seed):
    """Training samples of a scene whose final maps are known: per view the
    network input (hpm_net_coarse_inputs) and the consistency-filtered
    targets (hpm_net_targets), all on the device."""
    import torch

    dev = torch.device("cuda", ctx.device if hasattr(ctx, "device") else 0)
    cams = np.ascontiguousarray(cams, dtype=hb.CAMERA_DTYPE)
    d_depth = [torch.from_numpy(np.ascontiguousarray(d)).to(dev) for d in depths]
    d_normal = [torch.from_numpy(np.ascontiguousarray(n)).to(dev) for n in normals]
    out = []
    for ref, srcs in pairs:
        ids = [ref] + list(srcs)
        h, w = int(cams[ref]["height"]), int(cams[ref]["width"])
        cap = (h // 4 + 2) * (w // 4 + 2)
        x0 = torch.empty(cap * 16, dtype=torch.bfloat16, device=dev)
        keep = [np.ascontiguousarray(images[i], dtype=np.float32) for i in ids]
        arr = (ctypes.c_void_p * len(ids))(*[k.ctypes.data for k in keep])
        pc = np.ascontiguousarray(cams[ids])
        cw, ch = ctypes.c_int(), ctypes.c_int()
        ctx._check(hb.lib().hpm_net_coarse_inputs(ctx.handle, len(ids), arr, hb._p(pc), ctypes.c_uint64(seed + ref),
                                                  _ptr(x0), ctypes.c_size_t(cap), ctypes.byref(cw),
                                                  ctypes.byref(ch)),
                   "hpm_net_coarse_inputs")
        cw, ch = cw.value, ch.value
        x0 = x0[:cw * ch * 16].view(ch, cw, 16)
        td = torch.empty(ch, cw, dtype=torch.float32, device=dev)
        tn = torch.empty(ch, cw, 3, dtype=torch.float32, device=dev)
        tm = torch.empty(ch, cw, dtype=torch.uint8, device=dev)
        sc = np.ascontiguousarray(cams[list(srcs)])
        sd = (ctypes.c_void_p * len(srcs))(*[d_depth[s].data_ptr() for s in srcs])
        sn = (ctypes.c_void_p * len(srcs))(*[d_normal[s].data_ptr() for s in srcs])
        rc = np.ascontiguousarray(cams[ref:ref + 1])
        _ok(hb.lib().hpm_net_targets(0, hb._p(rc), _ptr(d_depth[ref]), _ptr(d_normal[ref]), len(srcs), hb._p(sc), sd,
                                     sn, cw, ch, _ptr(td), _ptr(tn), _ptr(tm), None), "hpm_net_targets")
        dmin = float(cams[ref]["depth_min"]) * 0.6
        dmax = float(cams[ref]["depth_max"]) * 1.2
        out.append(dict(x0=x0.clone(), t_depth=td, t_normal=tn, t_mask=tm, dmin=dmin, dmax=dmax,
                        valid=int(tm.sum().item())))
    return out


def train(samples, net: Net, steps=1500, batch=8, lr=1e-3, lam=0.5, seed=0, log=None):
    """Adam over random batches of views, the learning rate decaying from lr
    to lr / 100 along a half cosine (so that the last weights are not one
    noisy step of a constant rate); returns the loss curve (mean loss per
    valid pixel, per step)."""
    import math

    rng = np.random.default_rng(seed)
    tr = Trainer(net, lr=lr, lam=lam)
    curve = []
    for step in range(steps):
        tr.lr = lr * (0.01 + 0.99 * 0.5 * (1.0 + math.cos(math.pi * step / max(1, steps - 1))))
        idx = rng.choice(len(samples), size=min(batch, len(samples)), replace=False)
        count = sum(samples[i]["valid"] for i in idx)
        if count == 0:
            continue
        for i in idx:
            s = samples[i]
            tr.accumulate(s["x0"], s["t_depth"], s["t_normal"], s["t_mask"], s["dmin"], s["dmax"], 1.0 / count)
        tr.apply()
        curve.append(tr.take_loss() / count)
        if log and (step % 100 == 0 or step == steps - 1):
            log(f"step {step} loss {curve[-1]:.4f}")
    return curve


def evaluate(samples, net: Net):
    """Mean relative depth error, fraction within 1 %, and median normal
    angle (degrees) of the network's head on the samples' valid pixels."""
    import torch

    tr = Trainer(net)
    rel, ang = [], []
    for s in samples:
        h, w = s["x0"].shape[:2]
        out = tr.forward(s["x0"], h, w, tr._bufs(h, w))
        m = s["t_mask"].bool()
        if not m.any():
            continue
        o = out[m]
        d = s["dmin"] + (s["dmax"] - s["dmin"]) * torch.sigmoid(o[:, 0])
        t = s["t_depth"][m]
        rel.append(((d - t).abs() / t).cpu())
        nrm = torch.nn.functional.normalize(o[:, 1:4], dim=1)
        c = (nrm * s["t_normal"][m]).sum(1).clamp(-1, 1)
        ang.append(torch.rad2deg(torch.acos(c)).cpu())
    rel, ang = torch.cat(rel), torch.cat(ang)
    return {"rel_depth_err_mean": float(rel.mean()), "within_1pct": float((rel < 0.01).float().mean()),
            "normal_err_median_deg": float(ang.median()), "pixels": int(len(rel))}


# ---------------------------------------------------------------------------
# Training and evaluation run (on a GPU machine):
#   python hpm-mvs_b200/priornet.py --scenes 200 --eval-scenes 20 --out DIR
# ---------------------------------------------------------------------------

RECIPE = dict(width=1600, height=1200, n_views=11, n_planes=20, n_spheres=5, low_texture=0.40)


def _make_scene(args):
    """(seed, recipe) -> the scene's images, cameras, pairs and ground truth
    (runs in a worker process)."""
    import synthetic as syn

    seed, r = args
    sc = syn.make_scene(seed, r["width"], r["height"], r["n_views"], n_planes=r["n_planes"],
                        n_spheres=r["n_spheres"], low_texture=r["low_texture"])
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(r["n_views"])]
    return dict(seed=seed, images=[i.astype(np.float32) for i in sc.images], cams=sc.cams, pairs=pairs,
                gt_depth=sc.gt_depth, gt_normal=sc.gt_normal)


def _scene_stream(seeds, recipe, workers):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        yield from pool.imap(_make_scene, [(s, recipe) for s in seeds])


def _accuracy(sc, depths, normals):
    import synthetic as syn

    acc = float(np.mean([syn.depth_accuracy(depths[v], sc["gt_depth"][v]) for v in range(len(depths))]))
    ne = float(np.median([syn.normal_error_deg(normals[v], sc["gt_normal"][v], sc["gt_depth"][v])
                          for v in range(len(depths))]))
    return acc, ne


def parse_schedule(text: str):
    """"extra:geom[:prior[:iterations[:geom_pass_iterations]]]" -> the five
    values; prior defaults to 1 (the coarse triangulation), iterations to 3,
    geom_pass_iterations to iterations."""
    v = [int(x) for x in text.split(":")]
    if not 2 <= len(v) <= 5:
        raise ValueError(f"schedule {text!r}: extra:geom[:prior[:iterations[:geom_pass_iterations]]]")
    v += [None, None, 1, 3, None][len(v):]
    if v[4] is None:
        v[4] = v[3]
    return tuple(v)


def main():
    import argparse
    import json
    import sys
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=200)
    ap.add_argument("--eval-scenes", type=int, default=20)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--schedules", default="0:2:2:3,0:2:2:3:2,0:2:2:2,1:2:2:2:1,0:1:2:3,0:2:2:2:1",
                    help="prior-net schedules to evaluate, extra full-scale prior passes:geometric iterations:"
                         "planar prior of the first full-scale pass (1 the coarse triangulation, 2 the proposal):"
                         "PatchMatch iterations per full-scale pass:PatchMatch iterations per geometric pass "
                         "(default: as the full-scale passes)")
    ap.add_argument("--batched", action="store_true", help="evaluate the batched forms (plain and prior-net)")
    ap.add_argument("--weights", default=None,
                    help="evaluate the schedules with these weights instead of generating data and training")
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--size", default=None, help="WxH of the scenes (default 1600x1200)")
    ap.add_argument("--out", default=".")
    args = ap.parse_args()
    recipe = dict(RECIPE)
    if args.size:
        recipe["width"], recipe["height"] = (int(x) for x in args.size.lower().split("x"))
    workers = args.workers or max(1, (os.cpu_count() or 2) * 2 // 3)
    schedules = [parse_schedule(t) for t in args.schedules.split(",")]
    if args.weights:
        args.scenes = 0
    train_seeds = list(range(1000, 1000 + args.scenes))
    eval_seeds = list(range(9000, 9000 + args.eval_scenes))
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    # the pool starts before the first CUDA call
    stream = _scene_stream(train_seeds + eval_seeds, recipe, workers)
    import torch

    torch.cuda.set_device(0)
    summary = dict(recipe=recipe, train_scenes=args.scenes, eval_scenes=args.eval_scenes, workers=workers)
    samples, t_data = [], time.time()
    with hb.Context(0) as ctx:
        for k in range(args.scenes):
            sc = next(stream)
            d, n, _ = ctx.run_scene(sc["images"], sc["cams"], sc["pairs"], seed=sc["seed"])
            samples += view_samples(ctx, sc["images"], sc["cams"], sc["pairs"], d, n, seed=7 * sc["seed"])
            if k % 10 == 0:
                log(f"scene {k}: {len(samples)} views, valid px/view {np.mean([s['valid'] for s in samples]):.0f}")
        summary["data_seconds"] = time.time() - t_data
        summary["train_views"] = len(samples)
        if args.weights:
            net = Net.load(args.weights)
            meta = dict(np.load(args.weights))
            curve = [float(x) for x in meta.get("loss", np.zeros(1))]
            args.scenes, args.steps = int(meta.get("train_scenes", 0)), int(meta.get("steps", 0))
            summary["weights"] = args.weights
        else:
            net = Net(0, seed=1)
            t_train = time.time()
            curve = train(samples, net, steps=args.steps, batch=args.batch, lr=args.lr, log=log)
            torch.cuda.synchronize()
            summary["train_seconds"] = time.time() - t_train
            summary["loss_first_last"] = [curve[0], curve[-1]]
            summary["train_fit"] = evaluate(samples, net)
        del samples
        # held-out scenes: the network's own accuracy, then the plain form and
        # the prior-net form end to end
        rows = []
        for k in range(args.eval_scenes):
            sc = next(stream)
            row = {"seed": sc["seed"]}
            ev = []
            for form, kw in [("plain", dict(geom_iterations=2, batched=args.batched))] + [
                    (f"net_e{e}_g{g}_p{m}_i{i}_j{j}", dict(pyramid_levels=e, geom_iterations=g, planar_prior=m,
                                                           iterations=i, geom_pass_iterations=j, net=net.weights(),
                                                           batched=args.batched))
                    for e, g, m, i, j in schedules]:
                ctx.run_scene(sc["images"], sc["cams"], sc["pairs"], seed=sc["seed"], **kw)  # warm-up
                torch.cuda.synchronize()
                t0 = time.time()
                d, n, _ = ctx.run_scene(sc["images"], sc["cams"], sc["pairs"], seed=sc["seed"] + 1, **kw)
                dt = time.time() - t0
                acc, ne = _accuracy(sc, d, n)
                npx = sum(i.size for i in sc["images"])
                row[form] = dict(seconds=dt, mpix_per_s=npx / dt / 1e6, px_relerr_lt_1pct=acc,
                                 median_normal_err_deg=ne)
                if form == "plain":
                    ev = view_samples(ctx, sc["images"], sc["cams"], sc["pairs"], d, n, seed=7 * sc["seed"])
            row["net_head"] = evaluate(ev, net)
            rows.append(row)
            log(json.dumps(row))
        summary["eval"] = rows
        forms = ["plain"] + [f"net_e{e}_g{g}_p{m}_i{i}_j{j}" for e, g, m, i, j in schedules]
        for form in forms:
            summary[f"eval_{form}"] = {k: float(np.mean([r[form][k] for r in rows]))
                                       for k in ("mpix_per_s", "px_relerr_lt_1pct", "median_normal_err_deg")}
        # the schedule the scene driver uses: the fastest whose accuracy is
        # within 0.5 pp of the plain form's, else the most accurate
        plain_acc = summary["eval_plain"]["px_relerr_lt_1pct"]
        ev = lambda e, g, m, i, j: summary[f"eval_net_e{e}_g{g}_p{m}_i{i}_j{j}"]  # noqa: E731
        ok = [(ev(*t)["mpix_per_s"], t) for t in schedules if ev(*t)["px_relerr_lt_1pct"] >= plain_acc - 0.005]
        if ok:
            _, (e, g, m, i, j) = max(ok)
        else:
            _, (e, g, m, i, j) = max((ev(*t)["px_relerr_lt_1pct"], t) for t in schedules)
        summary["chosen_schedule"] = {"extra_passes": e, "geom_iterations": g, "prior": m, "iterations": i,
                                      "geom_pass_iterations": j}
        net.save(os.path.join(args.out, "priornet_weights.npz"), loss=np.array(curve, np.float32),
                 extra_passes=e, geom_iterations=g, prior=m, iterations=i, geom_pass_iterations=j,
                 train_scenes=args.scenes, steps=args.steps)
    with open(os.path.join(args.out, "priornet_summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps({k: v for k, v in summary.items() if k != "eval"}))


if __name__ == "__main__":
    main()

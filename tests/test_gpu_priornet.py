"""The prior-net form: its training kernels against plain PyTorch fp32
references of the same operations, the training filter against a NumPy
restatement of the reference's fusion test, and the scene driver end to
end (proposals enter PatchMatch only as candidates scored by the NCC)."""
import ctypes

import numpy as np
import pytest

import hpm_b200 as hb
import synthetic as syn

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_loss_gradient_matches_autograd():
    import torch

    n, dmin, dmax, lam = 5000, 1.2, 9.6, 0.5
    g = torch.Generator().manual_seed(3)
    out = (torch.randn(n, 16, generator=g)).cuda()
    td = (torch.rand(n, generator=g) * 6 + 2).cuda()
    tn = torch.nn.functional.normalize(torch.randn(n, 3, generator=g), dim=1).cuda()
    tm = (torch.rand(n, generator=g) < 0.7).to(torch.uint8).cuda()
    dy = torch.empty(n, 16, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(1, device="cuda")
    inv = 1.0 / float(tm.sum())
    assert hb.lib().hpm_net_loss(_ptr(out), _ptr(td), _ptr(tn), _ptr(tm), n, ctypes.c_float(dmin),
                                 ctypes.c_float(dmax), ctypes.c_float(lam), ctypes.c_float(inv), _ptr(dy), _ptr(loss),
                                 None) == hb.HPM_OK
    o = out.clone().requires_grad_(True)
    d = dmin + (dmax - dmin) * torch.sigmoid(o[:, 0])
    nn_ = torch.nn.functional.normalize(o[:, 1:4], dim=1)
    per = (d - td).abs() / td + lam * (1 - (nn_ * tn).sum(1))
    ref_loss = (per * tm).sum()
    (ref_loss * inv).backward()
    torch.cuda.synchronize()
    assert abs(float(loss) - float(ref_loss)) <= 1e-4 * float(ref_loss)
    ref = o.grad
    assert (dy.float()[:, 4:] == 0).all()
    assert (dy.float() - ref).abs().max().item() <= 1e-2 * ref.abs().max().item()


def test_adam_step_matches_torch():
    import torch

    n = 1000
    p = torch.randn(n, device="cuda")
    g = torch.randn(n, device="cuda")
    m = torch.zeros(n, device="cuda")
    v = torch.zeros(n, device="cuda")
    ref = p.clone().requires_grad_(True)
    opt = torch.optim.Adam([ref], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    for step in (1, 2, 3):
        gg = g * step
        ref.grad = gg.clone()
        opt.step()
        g2 = gg.clone()
        assert hb.lib().hpm_net_adam(_ptr(p), _ptr(g2), _ptr(m), _ptr(v), n, ctypes.c_float(1e-3),
                                     ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), step,
                                     None) == hb.HPM_OK
        torch.cuda.synchronize()
        assert (g2 == 0).all()
    assert (p - ref.detach()).abs().max().item() <= 1e-6


def _fusion_mask_numpy(ref_cam, depth, normal, src_cams, src_depths, src_normals):
    """The consistency test of RunFusion (main.cpp:575-612) without its
    masking, vectorised in float64."""
    h, w = depth.shape
    ys, xs = np.mgrid[0:h, 0:w].astype(np.float64)

    def world(c, x, y, d):
        K, R, t = c["K"].reshape(3, 3), c["R"].reshape(3, 3), c["t"]
        X = np.stack([d * (x - K[0, 2]) / K[0, 0], d * (y - K[1, 2]) / K[1, 1], d], -1)
        return (X - t) @ R  # R^T (X - t)

    def project(X, c):
        K, R, t = c["K"].reshape(3, 3), c["R"].reshape(3, 3), c["t"]
        Y = X @ R.T + t
        p = Y @ K.T
        return p[..., 0] / p[..., 2], p[..., 1] / p[..., 2], p[..., 2]

    X = world(ref_cam, xs, ys, depth.astype(np.float64))
    num = np.zeros((h, w), int)
    dyn = np.zeros((h, w))
    for sc, sd, sn in zip(src_cams, src_depths, src_normals):
        px, py, _ = project(X, sc)
        sr, scc = (py + 0.5).astype(int), (px + 0.5).astype(int)
        ok = (scc >= 0) & (scc < sc["width"]) & (sr >= 0) & (sr < sc["height"]) & (depth > 0)
        sr_, sc_ = np.where(ok, sr, 0), np.where(ok, scc, 0)
        dsrc = sd[sr_, sc_]
        ok &= dsrc > 0
        Y = world(sc, sc_.astype(np.float64), sr_.astype(np.float64), dsrc)
        tx, ty, td = project(Y, ref_cam)
        e = np.sqrt((xs - tx) ** 2 + (ys - ty) ** 2)
        rel = np.abs(td - depth) / np.where(depth > 0, depth, 1)
        ang = np.arccos(np.clip((normal * sn[sr_, sc_]).sum(-1), -1, 1))
        good = ok & (e < 2) & (rel < 0.01) & (ang < 0.174533)
        num += good
        dyn += np.where(good, np.exp(-(e + 200 * rel + 10 * ang)), 0)
    return (num >= 1) & (dyn > 0.3 * num)


def test_training_filter_matches_numpy():
    import torch

    sc = syn.make_scene(41, 160, 120, 5, n_planes=5)
    rng = np.random.default_rng(0)
    depths = [(d * rng.uniform(0.995, 1.005, d.shape)).astype(np.float32) for d in sc.gt_depth]
    normals = [n.astype(np.float32) for n in sc.gt_normal]
    ref, srcs = 2, [int(s) for s in sc.pairs[2][1]]
    want = _fusion_mask_numpy(sc.cams[ref], depths[ref], normals[ref], sc.cams[srcs], [depths[s] for s in srcs],
                              [normals[s] for s in srcs])
    dd = [torch.from_numpy(d).cuda() for d in depths]
    dn = [torch.from_numpy(n).cuda() for n in normals]
    h, w = depths[ref].shape
    td = torch.empty(h, w, device="cuda")
    tn = torch.empty(h, w, 3, device="cuda")
    tm = torch.empty(h, w, dtype=torch.uint8, device="cuda")
    cams = np.ascontiguousarray(sc.cams)
    rc = np.ascontiguousarray(cams[ref:ref + 1])
    scs = np.ascontiguousarray(cams[srcs])
    sd = (ctypes.c_void_p * len(srcs))(*[dd[s].data_ptr() for s in srcs])
    sn = (ctypes.c_void_p * len(srcs))(*[dn[s].data_ptr() for s in srcs])
    assert hb.lib().hpm_net_targets(0, hb._p(rc), _ptr(dd[ref]), _ptr(dn[ref]), len(srcs), hb._p(scs), sd, sn, w, h,
                                    _ptr(td), _ptr(tn), _ptr(tm), None) == hb.HPM_OK
    got = tm.cpu().numpy().astype(bool)
    assert want.mean() > 0.3
    # float32 on the device against float64 here: decisions on the thresholds
    # may differ on a few pixels
    assert (got == want).mean() >= 0.998, (got == want).mean()
    np.testing.assert_allclose(td.cpu().numpy(), depths[ref])


def test_prior_net_scene_runs_and_scores_proposals():
    """With a trained network (the committed weights) the prior-net form's
    maps are finite and reach the plain form's accuracy within a stated
    margin on a small scene; with the proposals scored as candidates by the
    unchanged NCC cost, a network that proposes nonsense (zero weights: every
    proposal the far end of the depth range facing the camera) still lets
    PatchMatch find the surfaces."""
    import os

    import priornet

    sc = syn.make_scene(77, 640, 480, 6, n_planes=8, n_spheres=2, low_texture=0.4)
    images = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(6)]
    acc = {}
    with hb.Context() as ctx:
        d, n, _ = ctx.run_scene(images, sc.cams, pairs, seed=5)
        acc["plain"] = np.mean([syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(6)])
        zero = priornet.Net(0, weights={**{f"w{i}": np.zeros((co, ci, 3, 3), np.float32)
                                           for i, (ci, co) in enumerate(priornet.LAYERS)},
                                        **{f"b{i}": np.zeros(co, np.float32)
                                           for i, (ci, co) in enumerate(priornet.LAYERS)}})
        d, n, _ = ctx.run_scene(images, sc.cams, pairs, seed=5, net=zero.weights())
        assert all(np.isfinite(x).mean() > 0.99 for x in d)
        acc["zero_net"] = np.mean([syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(6)])
        if os.path.exists(priornet.WEIGHTS_FILE):
            net = priornet.Net.load()
            d, n, _ = ctx.run_scene(images, sc.cams, pairs, seed=5, net=net.weights())
            acc["net"] = np.mean([syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(6)])
    assert acc["zero_net"] > 0.5 * acc["plain"], acc
    if "net" in acc:
        assert acc["net"] >= acc["plain"] - 0.03, acc

"""The batched form (hpm_run_scene_batched): all problems of a scene in one
persistent launch per kernel and half-step, passes replayed from a CUDA
graph, half-step tiles tuned per view size.

Per-pixel work does not depend on the tile shape or on which CTA does it, so
pass set A must equal hpm_process_problem on a fresh context per problem bit
for bit, on a scene whose views have different sizes."""
import numpy as np
import pytest

import hpm_b200 as hb
import synthetic as syn

pytestmark = pytest.mark.gpu

SIZES = [(160, 120), (128, 96), (96, 72), (160, 120), (128, 96), (96, 72)]


def _scene(seed=61):
    sc = syn.make_scene(seed, 160, 120, len(SIZES), n_planes=6, n_spheres=1, low_texture=0.3, sizes=SIZES,
                        arc_step_deg=6.0)
    imgs = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(len(SIZES))]
    return sc, imgs, pairs


@pytest.mark.parametrize("levels", [0, 1])
def test_batched_pass_set_a_equals_per_problem(levels):
    sc, imgs, pairs = _scene()
    with hb.Context() as ctx:
        d, n, c = ctx.run_scene(imgs, sc.cams, pairs, seed=40, geom_iterations=0, pyramid_levels=levels,
                                batched=True)
        # a second scene on the same context reuses its problem contexts and tuned tiles
        d2, _, _ = ctx.run_scene(imgs, sc.cams, pairs, seed=40, geom_iterations=0, pyramid_levels=levels,
                                 batched=True)
    for p, (ref, srcs) in enumerate(pairs):
        ids = [ref] + srcs
        with hb.Context() as one:
            one.set_views([imgs[i] for i in ids], sc.cams[ids])
            rd, rn, rc, _ = one.process_problem(seed=40 + p, planar_prior=True, pyramid_levels=levels)
        np.testing.assert_array_equal(d[ref], rd)
        np.testing.assert_array_equal(n[ref], rn)
        np.testing.assert_array_equal(c[ref], rc)
        np.testing.assert_array_equal(d2[ref], rd)


def test_batched_scene_keeps_the_accuracy():
    """With the geometric iterations (which read the previous iteration's
    maps of every view) the batched scene reaches the per-problem scene's
    accuracy within 1.5 percentage points."""
    sc, imgs, pairs = _scene(62)
    with hb.Context() as ctx:
        db, _, _ = ctx.run_scene(imgs, sc.cams, pairs, seed=7, pyramid_levels=1, batched=True)
        dp, _, _ = ctx.run_scene(imgs, sc.cams, pairs, seed=7, pyramid_levels=1)
    ab = np.mean([syn.depth_accuracy(db[v], sc.gt_depth[v]) for v in range(len(SIZES))])
    ap = np.mean([syn.depth_accuracy(dp[v], sc.gt_depth[v]) for v in range(len(SIZES))])
    assert ab > 0.3 and abs(ab - ap) <= 0.015, (ab, ap)


@pytest.mark.parametrize("extra,prior", [(0, 1), (1, 2)])
def test_batched_prior_net_pass_set_a_equals_per_problem(extra, prior):
    """The batched prior-net form (hpm_run_scene_batched_net): the coarse
    passes of all problems batched, the full-scale passes batched with each
    problem's proposal candidate.  Its pass set A equals the per-problem
    prior-net form's (hpm_run_scene_net) bit for bit, views of three sizes,
    with and without an extra full-scale pass and for both planar priors
    (the coarse triangulation's, the proposal)."""
    import priornet

    sc, imgs, pairs = _scene(63)
    wts = priornet.Net(0, seed=3).weights()
    opts = dict(seed=40, geom_iterations=0, pyramid_levels=extra, planar_prior=prior, net=wts)
    with hb.Context() as ctx:
        db, nb, cb = ctx.run_scene(imgs, sc.cams, pairs, batched=True, **opts)
        db2, _, _ = ctx.run_scene(imgs, sc.cams, pairs, batched=True, **opts)  # contexts and graphs reused
        dp, np_, cp = ctx.run_scene(imgs, sc.cams, pairs, **opts)
    for ref, _ in pairs:
        np.testing.assert_array_equal(db[ref], dp[ref])
        np.testing.assert_array_equal(nb[ref], np_[ref])
        np.testing.assert_array_equal(cb[ref], cp[ref])
        np.testing.assert_array_equal(db2[ref], dp[ref])
    assert np.mean([syn.depth_accuracy(db[v], sc.gt_depth[v]) for v in range(len(SIZES))]) > 0.2


def test_texture_arrays_are_reused_across_view_sizes():
    """One context alternating between problems whose views differ in size
    (the texture arrays of each size kept per view slot and reused) gives a
    problem the same maps bit for bit each time."""
    sc, imgs, pairs = _scene(64)
    runs = []
    with hb.Context() as ctx:
        for p in (0, 1, 2, 0, 2):
            ref, srcs = pairs[p]
            ids = [ref] + srcs
            ctx.set_views([imgs[i] for i in ids], sc.cams[ids])
            runs.append(ctx.process_problem(seed=9 + p, planar_prior=True, pyramid_levels=1))
    for a, b in ((0, 3), (2, 4)):
        for x, y in zip(runs[a][:3], runs[b][:3]):
            np.testing.assert_array_equal(x, y)

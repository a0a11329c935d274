"""Inputs the reference does not guard against, planted on the host: every
call returns a status and the context stays usable (no fault, no hang).

- zero-variance images: every window is flat, so every NCC is the cost
  ceiling (var < 1e-5, HPM.cu:380-383); then no view can be sampled (every
  sampling probability is 0, and the reference's CDF divides by their zero
  sum, HPM.cu:1591-1612), so the costs are whatever that arithmetic gives
  (NaN, or a stray tiny value) while the planes stay finite and the pass and
  the prior stages complete;
- NaN and Inf planted in the hypotheses, costs, geometric depths and prior
  planes a caller hands in: the pass completes, the planes of pixels that
  were not planted stay finite, and the context runs a clean problem after.
"""
import numpy as np
import pytest

import hpm_b200 as hb
import synthetic as syn

pytestmark = pytest.mark.gpu


def _problem(seed=31, w=96, h=72, n=5):
    """A problem of a small scene: reference view n // 2 and its sources; ids
    are the scene's view numbers in the problem's order."""
    sc = syn.make_scene(seed, w, h, n, n_planes=4, arc_step_deg=4.0)
    ref = n // 2
    imgs, cams = syn.view_set(sc, ref)
    ids = [ref] + [int(s) for s in sc.pairs[ref][1]]
    return sc, ids, imgs, cams, sc.depth_min * 0.6, sc.depth_max * 1.2


def test_zero_variance_images_give_the_cost_ceiling():
    sc, ids, imgs, cams, dmin, dmax = _problem()
    flat = [np.full_like(i, 128.0) for i in imgs]
    with hb.Context() as ctx:
        ctx.set_views(flat, cams)
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=2))
        planes, costs = ctx.get_result()
        assert np.isfinite(planes).all()
        assert ((costs >= 0) & (costs <= 2) | np.isnan(costs)).all()
        d, _, _, _ = ctx.process_problem(seed=3, pyramid_levels=0)  # the prior stages on a flat view
        assert d.shape == imgs[0].shape


def test_planted_nan_and_inf_stay_contained():
    sc, ids, imgs, cams, dmin, dmax = _problem()
    h, w = imgs[0].shape
    rng = np.random.default_rng(4)
    bad = np.zeros((h, w), bool)
    bad[rng.integers(0, h, 40), rng.integers(0, w, 40)] = True
    with hb.Context() as ctx:
        ctx.set_views(imgs, cams)
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=5))
        planes, costs = ctx.get_result()
        planes[bad] = np.array([np.nan, np.inf, -np.inf, np.nan], np.float32)
        costs[bad] = np.nan
        depths = [sc.gt_depth[v].astype(np.float32) for v in ids]
        depths[0][bad] = np.nan
        # geometric pass over the planted state and depths
        ctx.set_geom_depths(depths)
        ctx.set_hypotheses(planes, costs)
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=6, geom=True))
        p2, _ = ctx.get_result()
        # prior pass with planted prior planes
        prior = np.tile(np.array([0, 0, -1, 5.0], np.float32), (h, w, 1))
        prior[bad] = np.array([np.nan, 0, np.inf, np.nan], np.float32)
        ctx.set_prior(prior, np.ones((h, w), np.uint32))
        ctx.run_patchmatch(hb.default_params(dmin, dmax, seed=7, prior=True))
        p3, _ = ctx.get_result()
        for p in (p2, p3):
            assert np.isfinite(p[~bad]).all(-1).mean() > 0.97
        # the context is still good for a clean problem
        ctx.set_views(imgs, cams)
        d, n, c, _ = ctx.process_problem(seed=8, pyramid_levels=0)
        assert np.isfinite(d).mean() > 0.99 and syn.depth_accuracy(d, sc.gt_depth[ids[0]]) > 0.3

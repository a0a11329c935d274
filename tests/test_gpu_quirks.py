"""fix_quirks (HpmParams / HpmProblemOpts / HpmSceneOpts, the front ends'
--no-reference-compat): off by default, so every other test runs the
reference's behaviour; on, it changes the places HpmParams lists."""
import numpy as np
import pytest

import hpm_b200 as hb
import synthetic as syn

pytestmark = pytest.mark.gpu


def test_default_keeps_the_reference_behaviour():
    p = hb.default_params(1.0, 2.0)
    assert p.fix_quirks == 0
    sc = syn.make_scene(5, 96, 72, 4, n_planes=4)
    imgs = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(4)]
    with hb.Context() as ctx:
        a = ctx.run_scene(imgs, sc.cams, pairs, seed=3, pyramid_levels=0)
        b = ctx.run_scene(imgs, sc.cams, pairs, seed=3, pyramid_levels=0, fix_quirks=False)
        c = ctx.run_scene(imgs, sc.cams, pairs, seed=3, pyramid_levels=0, fix_quirks=True)
    for v in range(4):
        np.testing.assert_array_equal(a[0][v], b[0][v])
    assert any((a[0][v] != c[0][v]).mean() > 0.05 for v in range(4))


def test_last_row_of_an_odd_height_is_propagated_only_with_fixed_quirks():
    """The reference's grid covers 2 * ceil(H / 32) * 16 rows (HPM.cu:1926):
    at H = 65 row 64 keeps its initial hypotheses through the half-steps;
    with fix_quirks it is propagated like the others."""
    sc = syn.make_scene(8, 48, 65, 5, n_planes=3, arc_step_deg=4.0)
    imgs, cams = syn.view_set(sc, 2)
    dmin, dmax = sc.depth_min * 0.6, sc.depth_max * 1.2
    rows = {}
    with hb.Context() as ctx:
        for fix in (False, True):
            params = hb.default_params(dmin, dmax, seed=4, fix_quirks=fix)
            ctx.set_views(imgs, cams)
            ctx.run_partial(params, 0, False)
            p0, _ = ctx.get_result()
            ctx.set_views(imgs, cams)
            ctx.run_partial(params, 6, False)
            p6, _ = ctx.get_result()
            rows[fix] = ((p6[64] != p0[64]).any(-1).mean(), (p6[:64] != p0[:64]).any(-1).mean())
    assert rows[False][0] == 0.0 and rows[False][1] > 0.5, rows
    assert rows[True][0] > 0.5, rows


def test_fixed_quirks_keep_the_accuracy():
    """Each fixed place follows what the reference's code evidently intends,
    but the reference's parameters were tuned with its quirks in place: on
    this synthetic scene the fixed form measured 62.2 % of pixels within 1 %
    against 65.7 % (B200).  The test holds the fixed form within 5
    percentage points, a usable pipeline rather than a better one."""
    sc = syn.make_scene(21, 200, 150, 6, n_planes=8, n_spheres=2, low_texture=0.4)
    imgs = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(6)]
    acc = {}
    with hb.Context() as ctx:
        for fix in (False, True):
            d, _, _ = ctx.run_scene(imgs, sc.cams, pairs, seed=11, pyramid_levels=1, fix_quirks=fix)
            acc[fix] = np.mean([syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(6)])
    assert acc[True] >= acc[False] - 0.05, acc

"""The oracle's restatement of the ACMM+NESP variant (CPU): its scale
schedule, its hierarchy acceptance rule and a small coarse-to-fine scene."""
import os
import sys

import numpy as np

import oracle as orc
import synthetic as syn

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import acmm_flow  # noqa: E402


def test_scale_schedule():
    """ComputeMultiScaleSettings (main.cpp:35-71): halvings of the capped
    longer side until it is at most 1000."""
    ms, k, kmax = acmm_flow.multiscale_settings([(1200, 1600), (600, 800), (4032, 6048)])
    assert ms == [1600, 800, 3200] and k == [1, 0, 2] and kmax == 2


def test_scaled_view():
    """InuputInitialization's resize (ACMM.cpp:489-516): fit cur x cur, K
    scaled by the size ratios, views that fit untouched."""
    sc = syn.make_scene(1, 160, 120, 2, n_planes=2)
    img = sc.images[0].astype(np.float32)
    out, cam = acmm_flow.scaled_view(img, sc.cams[0], 80)
    assert out.shape == (60, 80) and (cam["width"], cam["height"]) == (80, 60)
    np.testing.assert_allclose(cam["K"][[0, 2, 4, 5]], sc.cams[0]["K"][[0, 2, 4, 5]] * 0.5)
    same, cam2 = acmm_flow.scaled_view(img, sc.cams[0], 160)
    assert same is img and (cam2["K"] == sc.cams[0]["K"]).all()
    # 161 x 121 to 80: factor 80/161, 121 * 80/161 = 60.12 -> 60
    out3, cam3 = acmm_flow.scaled_view(np.zeros((121, 161), np.float32), sc.cams[0], 80)
    assert out3.shape == (60, 80)


def _case():
    sc = syn.make_scene(11, 64, 48, 4)
    imgs, cams = syn.view_set(sc, 1)
    rng = np.random.default_rng(1)
    gt = sc.gt_depth[1]
    n = sc.gt_normal[1] + rng.normal(0, 0.15, sc.gt_normal[1].shape).astype(np.float32)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    planes0 = np.concatenate([n, (gt * rng.uniform(0.9, 1.1, gt.shape))[..., None]], -1).astype(np.float32)
    return sc, imgs, cams, planes0, sc.depth_min * 0.6, sc.depth_max * 1.2


def test_hierarchy_keeps_only_updates_below_the_threshold():
    sc, imgs, cams, planes0, dmin, dmax = _case()
    kw = dict(depth_min=dmin, depth_max=dmax, seed=9, salt=0, planes=planes0, finalize=False, variant=1)
    pre = np.zeros(planes0.shape[:2], np.float32)
    p0, c0, _ = orc.run_patchmatch(imgs, cams, half_steps=0, hierarchy=1, pre_costs=pre, **kw)
    p2, c2, _ = orc.run_patchmatch(imgs, cams, half_steps=2, hierarchy=1, pre_costs=pre, **kw)
    changed = ~(p2 == p0).all(-1)
    assert 0.02 < changed.mean() < 0.98
    # a changed pixel's cost lies 0.1 below its threshold
    assert (c2[changed] < pre[changed] - 0.1 + 1e-6).all()
    # hierarchy 2 (same size): threshold 0, nothing is kept
    pre2 = np.ones_like(pre)
    q0, _, _ = orc.run_patchmatch(imgs, cams, half_steps=0, hierarchy=2, pre_costs=pre2, **kw)
    q2, _, _ = orc.run_patchmatch(imgs, cams, half_steps=2, hierarchy=2, pre_costs=pre2, **kw)
    assert (pre2 == 0).all()
    np.testing.assert_array_equal(q2, q0)


def test_variant_changes_the_geometric_pass():
    """Weights 0.2 and the cap at 3 change costs against HPM-MVS's 0.1 and 5."""
    sc, imgs, cams, planes0, dmin, dmax = _case()
    ids = [1] + list(sc.pairs[1][1])
    depths = [sc.gt_depth[i] for i in ids]
    kw = dict(depth_min=dmin, depth_max=dmax, seed=2, salt=0, geom=True, planes=planes0, depth_maps=depths,
              half_steps=2, finalize=False)
    pa, ca, _ = orc.run_patchmatch(imgs, cams, variant=1, **kw)
    ph, ch, _ = orc.run_patchmatch(imgs, cams, **kw)
    assert (~np.isclose(ca, ch)).mean() > 0.05


def test_small_scene_two_scales():
    sc = syn.make_scene(6, 96, 72, 4, n_planes=5)
    imgs = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(4)]
    d, n, c, sizes = acmm_flow.run_scene(imgs, sc.cams, pairs, seed=3, size_bound=48)
    assert sizes == [[48] * 4, [96] * 4]
    acc = [syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(4)]
    assert np.mean(acc) > 0.5, acc
    assert all(x.shape == (72, 96) for x in d)


def _hier_golden():
    import pytest

    from conftest import GOLDEN, golden

    path = os.path.join(GOLDEN, "acmm_hier.npz")
    if not os.path.exists(path):
        pytest.skip("acmm_hier.npz not generated yet (tests/golden/make_golden.py --only acmm, on a GPU)")
    sys.path.insert(0, GOLDEN)
    import make_golden as mg

    g = golden("acmm_hier.npz")
    sc, ref, imgs, cams, planes, scaled = mg.acmm_hier_inputs()
    assert mg.images_sha256(imgs) == str(g["images_sha256"]), "scene generator no longer reproduces the fixture"
    return g, imgs, cams, planes, scaled


def test_hierarchy_init_matches_reference():
    """The oracle's hierarchy initialisation against the reference's own
    RandomInitialization (ACMM.cu:538-604, run by oracle/_ref/libacmm_ref.so
    on a B200 for the fixture): the previous scale's normals averaged with
    the JBU's weights, turned to the reference frame with the depth of
    depths.dmb; the threshold pre_costs from the zero-normal plane; the
    initial cost and views.  NCC values within the golden tolerances of the
    HPM-MVS kernels (a tap near a 1/256 weight step may round the other
    way); planes within FP32 rounding of the reference's double-precision
    JBU weights."""
    g, imgs, cams, planes, scaled = _hier_golden()
    _, n_up = orc.jbu_at_scale(imgs[0], scaled[..., 3], scaled[..., :3], 2)
    start = np.concatenate([n_up, planes[..., 3:]], -1).astype(np.float32)
    cam0 = cams[0]
    dmin = np.float32(cam0["depth_min"]) * np.float32(0.6)
    dmax = np.float32(cam0["depth_max"]) * np.float32(1.2)
    pre = np.zeros(planes.shape[:2], np.float32)
    op, oc, ov = orc.run_patchmatch(imgs, cams, depth_min=dmin, depth_max=dmax, planes=start, half_steps=0,
                                    finalize=False, variant=1, hierarchy=1, pre_costs=pre)
    same = np.isclose(op, g["planes"], rtol=1e-4, atol=1e-5).all(-1)
    assert same.mean() >= 0.995, same.mean()
    for got, want in ((oc, g["costs"]), (pre, g["pre_costs"])):
        d = np.abs(got.astype(np.float64) - want)
        d = d[np.isfinite(d)]
        assert d.mean() <= 1e-4 and (d > 1e-3).mean() <= 0.01 and d.max() <= 2e-2, (d.mean(), d.max())
    assert (ov == g["views"]).mean() >= 0.98


def test_three_scales():
    """Two halvings (32, 64, then 128 pixels on the longer side): the
    hierarchy pass runs at two finer scales, each from the previous scale's
    geometric maps."""
    sc = syn.make_scene(7, 128, 96, 4, n_planes=4)
    imgs = [i.astype(np.float32) for i in sc.images]
    pairs = [(v, [int(s) for s in sc.pairs[v][1]]) for v in range(4)]
    d, n, c, sizes = acmm_flow.run_scene(imgs, sc.cams, pairs, seed=2, size_bound=32)
    assert sizes == [[32] * 4, [64] * 4, [128] * 4]
    assert all(x.shape == (96, 128) for x in d)
    acc = [syn.depth_accuracy(d[v], sc.gt_depth[v]) for v in range(4)]
    assert np.mean(acc) > 0.4, acc

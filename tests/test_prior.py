"""Planar-prior stages on the CPU: the product's Delaunay (host C++) against
OpenCV's Subdiv2D, which the reference calls (HPM.cpp:787-809), and the
oracle's restatement of the whole ProcessProblem flow."""
import numpy as np
import pytest

import flow as oflow
import hpm_b200 as hb
import synthetic as syn


def _canon(t):
    return {tuple(sorted([(r[0], r[1]), (r[2], r[3]), (r[4], r[5])])) for r in t}


@pytest.mark.parametrize("w,h,seed", [(160, 120, 0), (400, 300, 1), (1600, 1200, 2)])
def test_delaunay_matches_subdiv2d(w, h, seed):
    """Support-point-like input (at most one point per 5x5 block, in the
    reference's column-major block order): the same set of triangles as
    OpenCV's Subdiv2D, hull slivers included (they depend on the enclosing
    triangle's corners).  The order in which the triangles are listed differs."""
    rng = np.random.default_rng(seed)
    pts = [(cx + rng.integers(0, 5), cy + rng.integers(0, 5)) for cx in range(0, w, 5) for cy in range(0, h, 5)
           if rng.random() < 0.6]
    pts = np.array(pts, np.int32)
    ours, ref = _canon(hb.delaunay(pts, w, h)), _canon(oflow.cv_triangles(pts, w, h))
    assert len(ours) > 0 and ours == ref


def test_delaunay_degenerate_inputs():
    assert len(hb.delaunay(np.zeros((0, 2), np.int32), 10, 10)) == 0
    assert len(hb.delaunay(np.array([[1, 1], [5, 5]], np.int32), 10, 10)) == 0
    line = np.array([[i, 2 * i] for i in range(5)], np.int32)  # collinear: no triangle
    assert len(hb.delaunay(line, 20, 20)) == 0
    sq = np.array([[0, 0], [4, 0], [4, 4], [0, 4]], np.int32)  # co-circular: 2 triangles
    assert len(hb.delaunay(sq, 10, 10)) == 2


def test_scale_levels_rule():
    assert [oflow.scale_levels(*s) for s in [(640, 480), (1000, 900), (1600, 1200), (3200, 2133), (6048, 4032)]] == \
        [0, 0, 1, 2, 3]


def test_oracle_flow_runs():
    """Smoke test of the restated flow on a toy scene (too small for the prior
    to pay off: a handful of support points per level)."""
    sc = syn.make_scene(11, 96, 72, 4, n_planes=4, low_texture=0.4)
    imgs, cams = syn.view_set(sc, 1)
    gt = sc.gt_depth[1]
    d1, n1, c1, pd = oflow.process_problem(imgs, cams, seed=2, planar_prior=True, pyramid_levels=1)
    assert (pd > 0).mean() > 0.3
    assert syn.depth_accuracy(d1, gt) > 0.3


@pytest.mark.parametrize("w,h,seed", [(64, 48, 0), (333, 211, 1), (800, 600, 2)])
def test_knn_grid_search_equals_brute_force(w, h, seed):
    """The oracle's grid neighbour search against its brute-force scan: the
    same six neighbours (ties to the lower index), so the same KNN planes and
    mask, on sparse and clustered support points."""
    import oracle as orc

    rng = np.random.default_rng(seed)
    pts = [(cx + rng.integers(0, 5), cy + rng.integers(0, 5)) for cx in range(0, w - 4, 5)
           for cy in range(0, h - 4, 5) if rng.random() < (0.05 if cx < w // 2 else 0.5)]
    pts = np.array(pts, np.int32)
    sc = syn.make_scene(seed, w, h, 2, n_planes=3)
    cam, depth = sc.cams[0], sc.gt_depth[0].astype(np.float32)
    mask0 = np.where(rng.random((h, w)) < 0.3, 1.0, 0.0).astype(np.float32)
    try:
        orc.set_knn_grid(False)
        pb, mb = orc.knn_supplement(cam, pts, depth, 1.0, sc.depth_min, sc.depth_max, mask0)
    finally:
        orc.set_knn_grid(True)
    pg, mg = orc.knn_supplement(cam, pts, depth, 1.0, sc.depth_min, sc.depth_max, mask0)
    assert (mb < -200).mean() > 0.3
    np.testing.assert_array_equal(mg, mb)
    np.testing.assert_array_equal(pg, pb)

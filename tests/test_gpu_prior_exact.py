"""The integer stages of the planar prior, bit for bit: the triangle-id
raster (main.cpp:96-116) and the 6-nearest-neighbour index sets of
DepthsPredictSupplement (HPM.cpp:939-962), through the C ABI against the
oracle, on identical inputs.  These are the outputs before the float gates
(triangle planes, the kNN depth-range test) that the flow-level tests
compare with a tolerance."""
import numpy as np
import pytest

import hpm_b200 as hb
import oracle as orc

pytestmark = pytest.mark.gpu


def _support_points(seed, w, h, n):
    """Support points as the prior builds them: at most one per 5x5 block,
    with clusters and empty regions."""
    rng = np.random.default_rng(seed)
    bx, by = w // 5, h // 5
    blocks = rng.choice(bx * by, size=min(n, bx * by), replace=False)
    keep = rng.random(len(blocks)) < np.where((blocks % bx) < bx // 3, 0.3, 1.0)  # a sparse third
    blocks = blocks[keep]
    x = (blocks % bx) * 5 + rng.integers(0, 5, len(blocks))
    y = (blocks // bx) * 5 + rng.integers(0, 5, len(blocks))
    return np.stack([x, y], -1).astype(np.int32)


@pytest.mark.parametrize("w,h,n", [(320, 240, 1500), (800, 600, 6000), (1600, 1200, 20000)])
def test_triangle_raster_is_exact(w, h, n):
    pts = _support_points(w + n, w, h, n)
    tris = hb.delaunay(pts, w, h)
    assert len(tris) > n // 3
    ids = hb.raster_triangles(tris, w, h)
    mask, kept = orc.raster_triangles(tris, w, h)
    assert len(kept) == len(tris)
    np.testing.assert_array_equal(ids, mask.astype(np.int32))
    assert (ids > 0).mean() > 0.5


@pytest.mark.parametrize("w,h,n", [(320, 240, 1500), (800, 600, 4000)])
def test_knn_index_sets_are_exact(w, h, n):
    pts = _support_points(7 * w + n, w, h, n)
    tris = hb.delaunay(pts, w, h)
    mask = hb.raster_triangles(tris, w, h).astype(np.float32)
    got = hb.knn6(pts, w, h, mask)
    ref = orc.knn6(pts, w, h, mask)
    np.testing.assert_array_equal(got, ref)
    assert ((got[..., 0] >= 0) == (mask <= 0)).all()


def test_knn_ties_go_to_the_lower_index():
    """A regular lattice puts many support points at equal distances: the
    order of equal distances is the points' order (PCL leaves it open)."""
    w, h = 120, 90
    xs, ys = np.meshgrid(np.arange(2, w, 10), np.arange(2, h, 10))
    pts = np.stack([xs.ravel(), ys.ravel()], -1).astype(np.int32)
    pts = pts[np.random.default_rng(3).permutation(len(pts))]
    got = hb.knn6(pts, w, h)
    np.testing.assert_array_equal(got, orc.knn6(pts, w, h))


def test_knn_with_fewer_than_six_points():
    pts = np.array([[3, 4], [10, 2], [7, 7]], np.int32)
    got = hb.knn6(pts, 16, 12)
    np.testing.assert_array_equal(got, orc.knn6(pts, 16, 12))
    assert (got[..., 3:] == -1).all()

"""hpm_fuse on the GPU against the oracle's sequential RunFusion
(main.cpp:502-633): the same points in the same order.  The consistency
tests use CUDA's acosf/expf, the oracle the host's, so a decision sitting
on a threshold within an ulp may differ; the tests allow a handful."""
import numpy as np
import pytest

import hpm_b200 as hb
import oracle as orc
import synthetic as syn
from test_fusion import fusion_inputs

pytestmark = pytest.mark.gpu


def _compare(prod, ref, max_diff_frac=1e-3):
    xyz, nrm, bgr = prod
    oxyz, onrm, ocol = ref
    assert abs(len(xyz) - len(oxyz)) <= max(2, max_diff_frac * len(oxyz)), (len(xyz), len(oxyz))
    # the sequences agree point for point up to the first decision that differs
    n = min(len(xyz), len(oxyz))
    same = np.all(xyz[:n] == oxyz[:n], axis=1)
    first_diff = n if same.all() else int(np.argmin(same))
    assert first_diff >= (1 - max_diff_frac) * n or len(oxyz) < 100, (first_diff, n)
    k = first_diff
    np.testing.assert_array_equal(nrm[:k], onrm[:k])
    np.testing.assert_array_equal(bgr[:k].astype(np.float32), ocol[:k])


@pytest.mark.parametrize("noise", [0.0, 0.004])
def test_fuse_matches_oracle_on_true_geometry(noise):
    sc, depths, normals, colors, problems = fusion_inputs(3, 160, 120, 5, noise=noise)
    prod = hb.fuse(sc.cams, depths, normals, colors, problems)
    ref = orc.fuse(sc.cams, depths, normals, colors, problems)
    assert len(ref[0]) > 1000
    _compare(prod, ref)


def test_fuse_matches_oracle_on_patchmatch_maps():
    """The maps of a whole scene run (pass set A + two geometric
    iterations), fused by both."""
    nv = 5
    sc = syn.make_scene(4, 200, 150, nv, n_planes=5, low_texture=0.3)
    imgs = [i.astype(np.float32) for i in sc.images]
    problems = [(v, list(sc.pairs[v][1])) for v in range(nv)]
    with hb.Context() as ctx:
        d, n, _ = ctx.run_scene(imgs, sc.cams, problems, seed=5, pyramid_levels=0)
    colors = [np.repeat(g[..., None], 3, -1) for g in sc.images]
    prod = hb.fuse(sc.cams, d, n, colors, problems)
    ref = orc.fuse(sc.cams, d, n, colors, problems)
    assert len(ref[0]) > 0.03 * nv * 200 * 150
    _compare(prod, ref)


def test_fuse_acmm_matches_oracle():
    """hpm_fuse_acmm, the ACMM+NESP variant's RunFusion (at least 2 agreeing
    sources; point, normal and colour averaged), against or_fuse_acmm, which
    tests/test_fusion_reference.py pins to the variant's own code; colour
    bytes truncated as the variant's PLY writer does."""
    sc, depths, normals, colors, problems = fusion_inputs(3, 160, 120, 5, noise=0.004)
    xyz, nrm, bgr = hb.fuse(sc.cams, depths, normals, colors, problems, acmm=True)
    oxyz, onrm, ocol = orc.fuse(sc.cams, depths, normals, colors, problems, acmm=True)
    assert len(oxyz) > 1000
    _compare((xyz, nrm, bgr), (oxyz, onrm, ocol.astype(np.int32).astype(np.float32)))
    # fewer points than the HPM-MVS rule gives on the same maps: two sources needed
    assert len(xyz) < len(hb.fuse(sc.cams, depths, normals, colors, problems)[0])

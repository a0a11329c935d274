"""hpm_jbu_noalloc: joint bilateral upsampling for callers that cannot
allocate device memory while they run (their own pool owns the memory budget,
or a cudaMalloc would stall or upset the host loop).  The caller passes its own
device buffers; the only scratch is the library's fixed device array.

Checked through the C ABI against the context-based hpm_jbu on two calls in a
row with different inputs (so stale scratch from the first call would show),
at the tolerance the other JBU tests use.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden

import hpm_b200 as hb

pytestmark = pytest.mark.gpu


def _noalloc(guide, coarse_depth, coarse_normal):
    import torch

    dev = torch.device("cuda", 0)
    g = torch.from_numpy(np.ascontiguousarray(guide, np.float32)).to(dev)
    cd = torch.from_numpy(np.ascontiguousarray(coarse_depth, np.float32)).to(dev)
    cn = torch.from_numpy(np.ascontiguousarray(coarse_normal, np.float32)).to(dev)
    rows, cols = guide.shape
    s_rows, s_cols = coarse_depth.shape
    od = torch.zeros((rows, cols), dtype=torch.float32, device=dev)
    on = torch.zeros((rows, cols, 3), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = hb.lib().hpm_jbu_noalloc(0, ctypes.c_void_p(g.data_ptr()), cols, rows, ctypes.c_void_p(cd.data_ptr()),
                                  ctypes.c_void_p(cn.data_ptr()), s_cols, s_rows, ctypes.c_void_p(od.data_ptr()),
                                  ctypes.c_void_p(on.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == hb.HPM_OK, rc
    stream.synchronize()
    return od.cpu().numpy(), on.cpu().numpy()


def _cases():
    j = golden("jbu.npz")
    rng = np.random.default_rng(42)
    big_guide = rng.uniform(0, 255, (600, 800)).round().astype(np.float32)
    big_depth = rng.uniform(2, 8, (300, 400)).astype(np.float32)
    big_depth[rng.random(big_depth.shape) < 0.1] = 0
    n = rng.normal(size=(300, 400, 3)).astype(np.float32)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    return [(j["guide"], j["coarse_depth_2"], j["coarse_normal_2"]),
            (j["guide"], j["coarse_depth_4"], j["coarse_normal_4"]),
            (big_guide, big_depth, n)]


def test_noalloc_matches_context_path_on_consecutive_calls():
    cases = _cases()
    with hb.Context(0) as ctx:
        expect = [ctx.jbu(*c) for c in cases]
    # two calls in a row per case, cases back to back on the shared scratch
    for (c, (ed, en)) in list(zip(cases, expect)) * 2:
        od, on = _noalloc(*c)
        np.testing.assert_allclose(od, ed, rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(on, en, rtol=1e-4, atol=1e-5)


def test_noalloc_rejects_coarse_grids_above_the_limit():
    limit = 1 << 20
    s_cols, s_rows = 1025, 1024  # one row more than the fixed scratch holds
    assert s_cols * s_rows > limit
    null = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = hb.lib().hpm_jbu_noalloc(0, null, 2 * s_cols, 2 * s_rows, null, null, s_cols, s_rows, null, null, None)
    assert rc == -1  # HPM_ERR_ARG


def test_noalloc_scale_one_is_a_no_op():
    g = np.ones((8, 8), np.float32)
    od, on = _noalloc(g, np.ones((8, 8), np.float32), np.zeros((8, 8, 3), np.float32))
    assert (od == 0).all() and (on == 0).all()

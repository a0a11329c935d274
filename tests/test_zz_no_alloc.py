"""hpm_jbu_noalloc: joint bilateral upsampling for callers that cannot
allocate device memory while they run (their own pool owns the memory budget,
or a cudaMalloc would stall or upset the host loop).  The caller passes its own
device buffers; the only scratch is the library's fixed device array.

Checked through the C ABI against the context-based hpm_jbu on two calls in a
row with different inputs (so stale scratch from the first call would show),
at the tolerance the other JBU tests use; and that calls after the first one
leave the device's free memory unchanged.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden

import hpm_b200 as hb

pytestmark = pytest.mark.gpu


class _Staged:
    """Inputs and outputs of one call, already in device memory, so that the
    call itself can be checked for allocations."""

    def __init__(self, guide, coarse_depth, coarse_normal):
        import torch

        dev = torch.device("cuda", 0)
        self.g = torch.from_numpy(np.ascontiguousarray(guide, np.float32)).to(dev)
        self.cd = torch.from_numpy(np.ascontiguousarray(coarse_depth, np.float32)).to(dev)
        self.cn = torch.from_numpy(np.ascontiguousarray(coarse_normal, np.float32)).to(dev)
        self.rows, self.cols = guide.shape
        self.s_rows, self.s_cols = coarse_depth.shape
        self.od = torch.zeros((self.rows, self.cols), dtype=torch.float32, device=dev)
        self.on = torch.zeros((self.rows, self.cols, 3), dtype=torch.float32, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self):
        rc = hb.lib().hpm_jbu_noalloc(0, ctypes.c_void_p(self.g.data_ptr()), self.cols, self.rows,
                                      ctypes.c_void_p(self.cd.data_ptr()), ctypes.c_void_p(self.cn.data_ptr()),
                                      self.s_cols, self.s_rows, ctypes.c_void_p(self.od.data_ptr()),
                                      ctypes.c_void_p(self.on.data_ptr()), ctypes.c_void_p(self.stream.cuda_stream))
        assert rc == hb.HPM_OK, rc
        self.stream.synchronize()
        return self.od.cpu().numpy(), self.on.cpu().numpy()


def _noalloc(guide, coarse_depth, coarse_normal):
    return _Staged(guide, coarse_depth, coarse_normal).call()


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


def test_noalloc_calls_after_the_first_allocate_no_device_memory():
    """The first call on a device may load the library's device code (and
    with it the fixed scratch array); every later call must leave the
    device's free memory as it was."""
    import torch

    j = golden("jbu.npz")
    staged = _Staged(j["guide"], j["coarse_depth_4"], j["coarse_normal_4"])
    staged.call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        staged.call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


def test_noalloc_keeps_the_callers_current_device():
    import torch

    before = torch.cuda.current_device()
    g = np.ones((8, 8), np.float32)
    _noalloc(g, np.ones((4, 4), np.float32), np.zeros((4, 4, 3), np.float32))
    assert torch.cuda.current_device() == before


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

"""The proposal network's tensor-core convolutions (hpm_net_conv3x3,
tcgen05 with TMEM accumulators) against a plain PyTorch fp32 reference of
the same operation on the same BF16-rounded inputs and weights.

Tolerances: the accumulation is FP32 in both, so the FP32 epilogue agrees to
1e-4 of the output scale; BF16 outputs carry one BF16 rounding (2^-8
relative), so 1e-2 of the output scale."""
import ctypes

import numpy as np
import pytest

import hpm_b200 as hb

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _pack(w, mode):
    import torch

    cout, cin = w.shape[:2]
    oc, ic = (cin, cout) if mode else (cout, cin)
    out = torch.empty(9 * oc * ic, dtype=torch.bfloat16, device=w.device)
    assert hb.lib().hpm_net_pack_weights(_ptr(w), cout, cin, mode, _ptr(out), None) == hb.HPM_OK
    return out


def _conv(x, packed, bias, cout, epi, aux, tma):
    import torch

    h, w, cin = x.shape
    dt = torch.float32 if epi == 1 else torch.bfloat16
    y = torch.full((h, w, cout), float("nan"), dtype=dt, device=x.device)
    err = torch.zeros(1, dtype=torch.int32, device=x.device)
    rc = hb.lib().hpm_net_conv3x3(_ptr(x), h, w, cin, _ptr(packed), None if bias is None else _ptr(bias), cout, epi,
                                  None if aux is None else _ptr(aux), _ptr(y), int(tma), _ptr(err), None)
    assert rc == hb.HPM_OK, rc
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return y


def _case(h, w, cin, cout, seed):
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(h, w, cin, generator=g).to(torch.bfloat16).cuda()
    wt = (torch.randn(cout, cin, 3, 3, generator=g) / (3 * cin ** 0.5)).cuda()
    b = (torch.randn(cout, generator=g) * 0.1).cuda()
    return x, wt, b


def _ref_forward(x, wt, b):
    import torch

    xf = x.float().permute(2, 0, 1)[None]
    wf = wt.to(torch.bfloat16).float()
    return torch.nn.functional.conv2d(xf, wf, b, padding=1)[0].permute(1, 2, 0)


@pytest.mark.parametrize("tma", [False, True])
@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
@pytest.mark.parametrize("h,w", [(5, 128), (9, 300)])
def test_conv_forward_matches_torch(tma, cin, cout, h, w):
    x, wt, b = _case(h, w, cin, cout, seed=cin * 100 + cout + w)
    ref = _ref_forward(x, wt, b)
    scale = float(ref.abs().max())
    got = _conv(x, _pack(wt, 0), b, cout, 1, None, tma)
    assert (got - ref).abs().max().item() <= 1e-4 * scale
    got = _conv(x, _pack(wt, 0), b, cout, 0, None, tma)
    assert (got.float() - ref.clamp_min(0)).abs().max().item() <= 1e-2 * scale


@pytest.mark.parametrize("tma", [False, True])
@pytest.mark.parametrize("cin,cout", [(32, 32), (16, 32), (32, 16)])
def test_conv_data_gradient_matches_torch(tma, cin, cout):
    """The data gradient through a ReLU: the same kernel with the packed
    weights flipped and transposed, and the ReLU mask of the layer's input
    fused in the epilogue."""
    import torch

    h, w = 7, 200
    x, wt, _ = _case(h, w, cin, cout, seed=7 + cin + cout)
    dy = torch.randn(h, w, cout).to(torch.bfloat16).cuda()
    ref = torch.nn.grad.conv2d_input((1, cin, h, w), wt.to(torch.bfloat16).float(),
                                     dy.float().permute(2, 0, 1)[None], padding=1)[0].permute(1, 2, 0)
    ref = torch.where(x.float() > 0, ref, torch.zeros_like(ref))
    got = _conv(dy, _pack(wt, 1), None, cin, 2, x, tma)
    assert (got.float() - ref).abs().max().item() <= 1e-2 * float(ref.abs().max())


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
@pytest.mark.parametrize("h,w", [(6, 128), (11, 333)])
def test_weight_and_bias_gradients_match_torch(cin, cout, h, w):
    """Weight gradient on the tensor cores (MN-major operands, pixels as K)
    accumulated over many CTAs and tiles, and the bias gradient."""
    import torch

    x, wt, _ = _case(h, w, cin, cout, seed=11 + cin * cout + w)
    dy = torch.randn(h, w, cout).to(torch.bfloat16).cuda()
    ref = torch.nn.grad.conv2d_weight(x.float().permute(2, 0, 1)[None], wt.shape,
                                      dy.float().permute(2, 0, 1)[None], padding=1)
    dw = torch.zeros_like(wt)
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # accumulates
        assert hb.lib().hpm_net_conv_wgrad(_ptr(x), _ptr(dy), h, w, cin, cout, _ptr(dw), _ptr(db), _ptr(err),
                                           None) == hb.HPM_OK
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    scale = float(ref.abs().max())
    assert (dw - 2 * ref).abs().max().item() <= 2e-4 * scale * 2
    dbr = dy.float().sum((0, 1))
    assert (db - 2 * dbr).abs().max().item() <= 1e-3 * float(dbr.abs().max()) * 2


def test_conv_rejects_unsupported_shapes():
    import torch

    x = torch.zeros(4, 4, 8, dtype=torch.bfloat16, device="cuda")
    assert hb.lib().hpm_net_conv3x3(_ptr(x), 4, 4, 8, _ptr(x), _ptr(x), 32, 0, None, _ptr(x), 0, None, None) == -1  # HPM_ERR_ARG

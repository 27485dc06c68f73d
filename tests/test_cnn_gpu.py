"""tcgen05 BF16 convolutions of the sparse-view correction network against the
FP64 oracle: forward, data gradient (the forward kernel on transposed,
tap-flipped weights) and weight gradient."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import ufob

pytestmark = pytest.mark.gpu


def _bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


def _as64(t):
    return t.float().cpu().numpy().astype(np.float64)


def _fwd(x, w, bias=None, relu=0, residual=None):
    L = ufob.lib()
    fn = L.ufob_conv3x3_forward
    fn.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int] * 6 + [ctypes.c_void_p]
    fn.restype = ctypes.c_int
    N, H, W, Ci = x.shape
    Co = w.shape[0]
    out = torch.empty((N, H, W, Co), dtype=torch.float32, device="cuda")
    ufob.check(fn(x.data_ptr(), w.data_ptr(), bias.data_ptr() if bias is not None else None,
                  residual.data_ptr() if residual is not None else None, None, out.data_ptr(), N, H, W, Ci, Co, relu,
                  None))
    torch.cuda.synchronize()
    ufob.device_status()
    return out


@pytest.mark.parametrize("ci,co,hw", [(16, 32, 16), (32, 64, 8), (64, 128, 16), (128, 256, 8), (256, 16, 8),
                                      (16, 16, 23), (64, 32, 5)])
def test_conv_forward(cuda, ci, co, hw):
    rng = np.random.default_rng(ci + co + hw)
    x = rng.standard_normal((2, hw, hw, ci))
    w = rng.standard_normal((co, 9, ci)) / np.sqrt(9 * ci)
    b = rng.standard_normal(co)
    xb, wb = _bf16(x), _bf16(w)
    got = _fwd(xb, wb, torch.from_numpy(b.astype(np.float32)).cuda(), relu=1)
    ref = oracle.conv3x3_nhwc(_as64(xb), _as64(wb), b.astype(np.float32), relu=True)
    assert oracle.rel_l2(got.cpu().numpy(), ref) < 1e-5


def test_conv_residual(cuda):
    rng = np.random.default_rng(5)
    x, w = rng.standard_normal((1, 12, 12, 32)), rng.standard_normal((32, 9, 32)) / 17
    r = rng.standard_normal((1, 12, 12, 32))
    xb, wb, rb = _bf16(x), _bf16(w), _bf16(r)
    got = _fwd(xb, wb, residual=rb)
    ref = oracle.conv3x3_nhwc(_as64(xb), _as64(wb)) + _as64(rb)
    assert oracle.rel_l2(got.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("ci,co", [(32, 16), (64, 128), (16, 256)])
def test_conv_data_gradient(cuda, ci, co):
    """dx = conv(dy, W^T flipped) equals the adjoint of the forward conv."""
    rng = np.random.default_rng(ci * co)
    w = rng.standard_normal((co, 9, ci)) / 10
    dy = rng.standard_normal((2, 10, 10, co))
    wd = oracle.conv3x3_dgrad_weights(w)
    got = _fwd(_bf16(dy), _bf16(wd))
    # adjoint identity <conv(x), dy> = <x, dgrad(dy)> with the FP64 forward conv
    x = rng.standard_normal((2, 10, 10, ci))
    lhs = np.sum(oracle.conv3x3_nhwc(x, _as64(_bf16(w))) * _as64(_bf16(dy)))
    rhs = np.sum(x * got.cpu().numpy().astype(np.float64))
    assert abs(lhs - rhs) < 1e-4 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("ci,co,hw", [(16, 32, 16), (64, 64, 12), (32, 256, 8), (128, 16, 9)])
def test_conv_weight_gradient(cuda, ci, co, hw):
    rng = np.random.default_rng(ci + 7 * co)
    x = rng.standard_normal((2, hw, hw, ci))
    dz = rng.standard_normal((2, hw, hw, co))
    xb, dzb = _bf16(x), _bf16(dz)
    L = ufob.lib()
    fn = L.ufob_conv3x3_wgrad
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 5 + [ctypes.c_void_p]
    fn.restype = ctypes.c_int
    dw = torch.zeros((co, 9, ci), dtype=torch.float32, device="cuda")
    ufob.check(fn(xb.data_ptr(), dzb.data_ptr(), dw.data_ptr(), 2, hw, hw, ci, co, None))
    torch.cuda.synchronize()
    ufob.device_status()
    ref = oracle.conv3x3_wgrad_nhwc(_as64(xb), _as64(dzb))
    assert oracle.rel_l2(dw.cpu().numpy(), ref) < 1e-5

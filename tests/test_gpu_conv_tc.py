"""Tensor-core 3x3x3 convolution (tcgen05.mma, BF16 operands, FP32 accumulation in tensor memory,
channels-last BF16 activations) against the numpy oracle on the same BF16-rounded inputs and
weights, and against the CUDA-core kernel: partial tiles in y and x, z segments and several work
items per CTA, channel counts 16..64, padded output channels (Co = 1, 8, 40), ReLU, both output
layouts."""
import ctypes as C

import numpy as np
import pytest

from grico_b200 import _lib as L
import cnn_oracle as co

pytestmark = pytest.mark.gpu


def _bf16(a):
    import torch

    return torch.tensor(a, dtype=torch.float32).bfloat16().float().numpy()


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _pack(wd, Ci, Co):
    import torch

    nb = L.lib().grico_conv_tc_weight_bytes(Ci, Co)
    assert nb > 0
    wp = torch.empty(nb // 2, dtype=torch.bfloat16, device="cuda")
    L.check(L.lib().grico_conv3d_pack_weights_tc(C.c_void_p(wd.data_ptr()), Ci, Co, C.c_void_p(wp.data_ptr()),
                                                 _stream()), "pack")
    return wp


def _conv_tc(x_cf, w, bias, relu, y_layout):
    """x_cf: FP32 numpy [B, Ci, Z, Y, X]; returns FP32 numpy [B, Co, Z, Y, X]."""
    import torch

    B, Ci, Z, Y, X = x_cf.shape
    Co = w.shape[0]
    xd = torch.tensor(x_cf, device="cuda").permute(0, 2, 3, 4, 1).contiguous().bfloat16()
    wd = torch.tensor(w, device="cuda")
    bd = torch.tensor(bias, device="cuda") if bias is not None else None
    wp = _pack(wd, Ci, Co)
    if y_layout == 0:
        yd = torch.full((B, Z, Y, X, Co), float("nan"), device="cuda", dtype=torch.bfloat16)
    else:
        yd = torch.full((B, Co, Z, Y, X), float("nan"), device="cuda", dtype=torch.float32)
    s = _stream()
    rc = L.lib().grico_conv3d_forward_tc(C.c_void_p(xd.data_ptr()), C.c_void_p(wp.data_ptr()),
                                         C.c_void_p(bd.data_ptr()) if bd is not None else None,
                                         C.c_void_p(yd.data_ptr()), y_layout, B, Ci, Co, Z, Y, X, relu, s)
    L.check(rc, "conv tc")
    L.check(L.lib().grico_conv_tc_status(s), "conv tc status")
    if y_layout == 0:
        yd = yd.float().permute(0, 4, 1, 2, 3)
    return yd.contiguous().cpu().numpy()


@pytest.mark.parametrize("B,Ci,Co,Z,Y,X,relu,layout", [
    (2, 32, 32, 5, 19, 12, 1, 1),
    (1, 16, 64, 3, 16, 8, 0, 1),
    (1, 32, 32, 4, 33, 17, 1, 0),
    (2, 48, 32, 2, 7, 5, 0, 0),
    (1, 64, 32, 3, 9, 9, 1, 1),
    (1, 32, 1, 6, 18, 10, 0, 1),    # the network's last layer: one FP32 output channel
    (1, 16, 8, 2, 5, 20, 1, 0),
    (1, 32, 40, 3, 12, 9, 0, 0),     # N padded to 64, stored channels 0..39
    (2, 32, 32, 40, 35, 20, 1, 0),   # z segments: several work items per CTA
])
def test_conv_tc_matches_oracle(cuda, B, Ci, Co, Z, Y, X, relu, layout):
    rng = np.random.default_rng(B * 1000 + Ci + Co + Z)
    x = _bf16(rng.standard_normal((B, Ci, Z, Y, X)).astype(np.float32))
    w = _bf16((0.2 * rng.standard_normal((Co, Ci, 27))).astype(np.float32))
    bias = rng.standard_normal(Co).astype(np.float32)
    ref = co.conv3d(x, w, bias, relu=bool(relu))
    got = _conv_tc(x, w, bias, relu, layout)
    tol = 1e-2 if layout == 0 else 1e-5  # BF16 output rounding, else FP32 accumulation order
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))


def test_conv_tc_agrees_with_cuda_core_kernel(cuda):
    import torch

    rng = np.random.default_rng(7)
    B, Ci, Co, Z, Y, X = 2, 32, 32, 8, 16, 16
    x = _bf16(rng.standard_normal((B, Ci, Z, Y, X)).astype(np.float32))
    w = _bf16((0.2 * rng.standard_normal((Co, Ci, 27))).astype(np.float32))
    xd, wd = torch.tensor(x, device="cuda"), torch.tensor(w, device="cuda")
    y1 = torch.empty((B, Co, Z, Y, X), device="cuda")
    L.check(L.lib().grico_conv3d_forward(C.c_void_p(xd.data_ptr()), 0, C.c_void_p(wd.data_ptr()), None,
                                         C.c_void_p(y1.data_ptr()), 0, B, Ci, Co, Z, Y, X, 1, _stream()), "conv")
    y2 = _conv_tc(x, w, None, 1, 1)
    y1 = y1.cpu().numpy()
    assert np.max(np.abs(y1 - y2)) <= 1e-5 * np.max(np.abs(y1))


def test_conv_tc_rejects_unsupported_shapes(cuda):
    import torch

    x = torch.zeros(4096, device="cuda")
    p = C.c_void_p(x.data_ptr())
    lib = L.lib()
    assert lib.grico_conv3d_forward_tc(p, p, None, p, 0, 1, 2, 32, 2, 2, 2, 0, None) == L.GRICO_ERR_INVALID  # Ci
    assert lib.grico_conv3d_forward_tc(p, p, None, p, 0, 1, 32, 4, 2, 2, 2, 0, None) == L.GRICO_ERR_INVALID  # Co % 8
    odd = C.c_void_p(x.data_ptr() + 2)
    assert lib.grico_conv3d_forward_tc(odd, p, None, p, 0, 1, 32, 32, 2, 2, 2, 0, None) == L.GRICO_ERR_INVALID
    assert lib.grico_conv3d_pack_weights_tc(p, 2, 32, p, None) == L.GRICO_ERR_INVALID

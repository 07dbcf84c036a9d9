"""Tensor-core 3x3x3 convolution (tcgen05.mma, BF16 operands, FP32 accumulation in tensor memory)
against the numpy oracle on the same BF16-rounded inputs and weights, and against the CUDA-core
kernel; partial tiles in y and x, several channel counts, ReLU, BF16 activations."""
import ctypes as C

import numpy as np
import pytest

from grico_b200 import _lib as L
import cnn_oracle as co

pytestmark = pytest.mark.gpu


def _bf16(a):
    import torch

    return torch.tensor(a, dtype=torch.float32).bfloat16().float().numpy()


@pytest.mark.parametrize("B,Ci,Co,Z,Y,X,relu,xb,yb", [
    (2, 32, 32, 5, 19, 12, 1, 0, 0),
    (1, 16, 64, 3, 16, 8, 0, 0, 0),
    (1, 32, 32, 4, 33, 17, 1, 1, 1),
    (2, 48, 64, 2, 7, 5, 0, 1, 0),
])
def test_conv_tc_matches_oracle(cuda, B, Ci, Co, Z, Y, X, relu, xb, yb):
    import torch

    rng = np.random.default_rng(B * 1000 + Ci + Co)
    x = rng.standard_normal((B, Ci, Z, Y, X)).astype(np.float32)
    w = (0.2 * rng.standard_normal((Co, Ci, 27))).astype(np.float32)
    bias = rng.standard_normal(Co).astype(np.float32)
    ref = co.conv3d(_bf16(x), _bf16(w), bias, relu=bool(relu))
    xd = torch.tensor(x, device="cuda")
    if xb:
        xd = xd.bfloat16()
    wd = torch.tensor(w, device="cuda")
    bd = torch.tensor(bias, device="cuda")
    yd = torch.full((B, Co, Z, Y, X), float("nan"), device="cuda", dtype=torch.bfloat16 if yb else torch.float32)
    s = torch.cuda.current_stream().cuda_stream
    rc = L.lib().grico_conv3d_forward_tc(C.c_void_p(xd.data_ptr()), xb, C.c_void_p(wd.data_ptr()),
                                         C.c_void_p(bd.data_ptr()), C.c_void_p(yd.data_ptr()), yb, B, Ci, Co, Z, Y, X,
                                         relu, C.c_void_p(s))
    L.check(rc, "conv tc")
    L.check(L.lib().grico_conv_tc_status(C.c_void_p(s)), "conv tc status")
    got = yd.float().cpu().numpy()
    tol = 1e-2 if yb else 1e-5  # BF16 output rounding, else FP32 accumulation order
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))


def test_conv_tc_agrees_with_cuda_core_kernel(cuda):
    import torch

    rng = np.random.default_rng(7)
    B, Ci, Co, Z, Y, X = 2, 32, 32, 8, 16, 16
    x = _bf16(rng.standard_normal((B, Ci, Z, Y, X)).astype(np.float32))
    w = _bf16((0.2 * rng.standard_normal((Co, Ci, 27))).astype(np.float32))
    xd, wd = torch.tensor(x, device="cuda"), torch.tensor(w, device="cuda")
    y1 = torch.empty((B, Co, Z, Y, X), device="cuda")
    y2 = torch.empty_like(y1)
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (C.c_void_p(xd.data_ptr()), 0, C.c_void_p(wd.data_ptr()), None)
    L.check(L.lib().grico_conv3d_forward(*args, C.c_void_p(y1.data_ptr()), 0, B, Ci, Co, Z, Y, X, 1, s), "conv")
    L.check(L.lib().grico_conv3d_forward_tc(*args, C.c_void_p(y2.data_ptr()), 0, B, Ci, Co, Z, Y, X, 1, s), "conv tc")
    L.check(L.lib().grico_conv_tc_status(s), "status")
    assert torch.max(torch.abs(y1 - y2)).item() <= 1e-5 * torch.max(torch.abs(y1)).item()


def test_conv_tc_rejects_unsupported_shapes(cuda):
    import torch

    x = torch.zeros(8, device="cuda")
    rc = L.lib().grico_conv3d_forward_tc(C.c_void_p(x.data_ptr()), 0, C.c_void_p(x.data_ptr()), None,
                                         C.c_void_p(x.data_ptr()), 0, 1, 2, 32, 2, 2, 2, 0, None)
    assert rc == L.GRICO_ERR_INVALID

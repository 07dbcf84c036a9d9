"""FP32 apply of uniform cell batches on the tensor cores (tile variant 10: one element matrix
K_e shared by every cell, BF16 hi/lo pieces of x and K_e, FP32 accumulation in tensor memory)
against the CUDA-core FP32 kernels and the FP64 apply, on uniform cubes of degree 1..4 with mass
and diffusion, full and reduced layouts, one and three right-hand sides.

Bounds: the three BF16 products leave ~2^-16 of each term; against the FP64 apply the result
is held to 5e-5 of max|y| for a rough (random) x, and to 1e-4 of max_i sum_j |K_ij x_j| for a
smooth x, where the stiffness rows cancel (the sum-factorised FP32 kernel cancels less)."""
import ctypes as C

import numpy as np
import pytest

import grico_b200 as gb
from grico_b200 import _lib as L
from grico_b200 import batched as bt
from grico_b200.problem import torch_stream_handle

pytestmark = pytest.mark.gpu


def _cube(p, mu, kappa, roots=(2, 2, 2), depth=3):
    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), roots)
    gb.uniform_refine(d, depth)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(mu, kappa))
    for a in (1, 2, 3):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return gb.compile(prob)


def _apply(plan, X, reduced, prec):
    import torch

    k, n = X.shape
    y = torch.empty_like(X)
    fn = L.lib().grico_reduced_apply if reduced else L.lib().grico_apply
    L.check(fn(plan.handle, C.c_void_p(X.data_ptr()), C.c_void_p(y.data_ptr()), k, prec, 0,
               C.c_void_p(torch_stream_handle())), "apply")
    L.check(L.lib().grico_tc_status(C.c_void_p(torch_stream_handle())), "tensor-core status")
    return y.double().cpu().numpy()


@pytest.mark.parametrize("p,mu", [(4, 0.0), (3, 0.7), (2, 0.0), (1, 2.0)])
@pytest.mark.parametrize("reduced", [True, False])
def test_dense_tensor_core_apply(cuda, p, mu, reduced):
    import torch

    plan = _cube(p, mu, 1.3)
    assert len(plan.batches) == 1
    n = plan.n_reduced if reduced else plan.n_full
    rng = np.random.default_rng(p)
    pts = np.linspace(0.0, 1.0, n)
    rough = rng.standard_normal((3, n))
    smooth = np.stack([np.sin(3.0 * pts), np.cos(2.0 * pts) + pts, np.sin(5.0 * pts) * pts])
    for Xh in (rough, smooth):
        y64 = _apply(plan, torch.tensor(Xh, dtype=torch.float64, device="cuda"), reduced, L.GRICO_PREC_FP64)
        a64 = _apply(plan, torch.tensor(np.abs(Xh), dtype=torch.float64, device="cuda"), reduced, L.GRICO_PREC_FP64)
        X32 = torch.tensor(Xh, dtype=torch.float32, device="cuda")
        res = {}
        for var in (10, 1):
            bt.set_tiles(plan, [var], "fp32")
            res[var] = _apply(plan, X32, reduced, L.GRICO_PREC_FP32)
            one = _apply(plan, X32[:1].contiguous(), reduced, L.GRICO_PREC_FP32)
            assert np.max(np.abs(one[0] - res[var][0])) <= 1e-6 * np.max(np.abs(res[var][0]))
        bt.set_tiles(plan, [10], "fp32")
        # |K| |x| scale of each row (diffusion rows cancel on smooth x); the element matrix is
        # not sign-definite, so take the larger of max|y| and the apply to |x| as the scale
        scale = max(np.max(np.abs(y64)), np.max(np.abs(a64)))
        tol = 5e-5 if Xh is rough else 1e-4
        assert np.max(np.abs(res[10] - y64)) <= tol * scale, np.max(np.abs(res[10] - y64)) / scale
        assert np.max(np.abs(res[1] - y64)) <= 2e-5 * scale


def test_autotuner_times_the_tensor_core_variant(cuda):
    plan = _cube(4, 0.0, 1.0)
    tiles = bt.autotune(plan, nrhs=1, precision="fp32", reps=2)
    assert 0 <= int(tiles[0]) < L.TILE_VARIANTS
    L.check(L.lib().grico_tc_status(None), "tensor-core status")

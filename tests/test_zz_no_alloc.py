"""grico_reduced_rhs_static: the reduced right-hand side without any GPU allocation.

It exists for callers that cannot allocate GPU memory during the call (host callbacks,
services with a fixed memory budget); its temporaries live in a static device array instead.
Checked through the C ABI against grico_reduced_rhs on two calls in a row, and the size limit
is checked.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import grico_b200 as gb
from grico_b200 import _lib as L
from cases import CASES, build, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _static_rhs(plan, arrays):
    import torch

    dev = [torch.tensor(a, device="cuda") if a is not None else None for a in arrays]
    ptrs = (C.c_void_p * len(dev))(*[d.data_ptr() if d is not None else None for d in dev])
    out = torch.full((plan.n_reduced,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    rc = L.lib().grico_reduced_rhs_static(plan.handle, ptrs, C.c_void_p(out.data_ptr()),
                                          C.c_void_p(stream.cuda_stream))
    stream.synchronize()
    L.check(rc, "grico_reduced_rhs_static")
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["3d_p4", "3d_p2_hanging", "2d_p4"])
def test_static_rhs_matches_allocating_entry_point(cuda, name):
    D = 2 if name.startswith("2d") else 3
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1) * D * np.pi ** 2 + 0.5 * x[:, 0]
    _, prob = build(name, source=src)
    plan = gb.compile(prob)
    ref = gb.reduced_rhs(plan)
    arrays = gb.problem._source_points(plan)
    first = _static_rhs(plan, arrays)
    second = _static_rhs(plan, arrays)  # the scratch keeps the first call's contents
    assert rel_err(first, ref) <= TOL
    assert rel_err(second, ref) <= TOL


@pytest.mark.parametrize("name", ["3d_p2_hanging", "2d_p4"])
def test_static_rhs_with_dirichlet_shift(cuda, name):
    """Non-zero Dirichlet values make the reduced right-hand side subtract A * shift, which the
    entry point computes in the second half of the static array; two calls in a row also show
    that the second call does not pick up the first call's leftovers there."""
    origin, extent, roots, refine, p, basis, qx, faces = CASES[name]
    D = len(origin)
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1) * D * np.pi ** 2 + 0.5 * x[:, 0]
    d = gb.Domain(origin, extent, roots)
    if refine:
        refine(d.grid)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.5, 1.5))
    gb.add_cell_accumulator(prob, u, gb.Load(src))
    for k, (a, side) in enumerate(faces):
        gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 1.0 + 0.5 * k))
    plan = gb.compile(prob)
    ref = gb.reduced_rhs(plan)
    arrays = gb.problem._source_points(plan)
    homogeneous = _static_rhs(plan, [None] * len(arrays))
    assert np.max(np.abs(homogeneous)) > 0.0  # the shift alone contributes
    first = _static_rhs(plan, arrays)
    second = _static_rhs(plan, arrays)
    assert rel_err(first, ref) <= TOL
    assert rel_err(second, ref) <= TOL


def test_static_rhs_rejects_plans_beyond_the_scratch(cuda):
    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (256, 256))
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(4)))
    assert s.scalar_dof_count > 1 << 20
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    plan = gb.compile(prob)
    import torch

    out = torch.zeros(plan.n_reduced, dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * len(plan.batches))()
    rc = L.lib().grico_reduced_rhs_static(plan.handle, ptrs, C.c_void_p(out.data_ptr()), None)
    assert rc == L.GRICO_ERR_INVALID
    assert b"static scratch holds at most 1048576" in L.lib().grico_last_error()

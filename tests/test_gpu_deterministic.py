"""GRICO_FLAG_DETERMINISTIC: applies without atomic scatter (stored local results summed per dof
in a fixed order).  Results are bitwise identical from call to call and equal the oracle (tensor
cells, hanging nodes, trunk modes), the L-shape's long hanging-node expansions, SIPG interfaces
and finite cells to the same 1e-12 as the default path; FP32 and two right-hand sides too."""
import ctypes as C

import numpy as np
import pytest

import grico_b200 as gb
from grico_b200 import _lib as L
import fc_cases
from cases import build, rel_err, sample_vector
from dg_cases import sipg_case
from test_dg_host import CASES as DG_CASES

pytestmark = pytest.mark.gpu
TOL = 1e-12
DET = L.GRICO_FLAG_HOST_POINTERS | L.GRICO_FLAG_DETERMINISTIC


def _apply(plan, x, reduced=False, flags=DET, nrhs=1):
    x = np.ascontiguousarray(x)
    y = np.empty_like(x)
    prec = L.GRICO_PREC_FP64 if x.dtype == np.float64 else L.GRICO_PREC_FP32
    fn = L.lib().grico_reduced_apply if reduced else L.lib().grico_apply
    L.check(fn(plan.handle, C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), nrhs, prec, flags, None), "apply")
    return y


@pytest.mark.parametrize("name", ["3d_p4", "3d_p2_hanging", "3d_p3_trunk", "2d_p2_hanging", "1d_p3"])
def test_deterministic_apply_matches_oracle_bitwise_repeatable(cuda, name):
    oplan, prob = build(name, mu=0.5, kappa=1.5)
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full)
    y1, y2 = _apply(plan, x), _apply(plan, x)
    assert np.array_equal(y1, y2)
    assert rel_err(y1, oplan.apply(x)) <= TOL
    xr = sample_vector(plan.n_reduced, seed=3)
    r1, r2 = _apply(plan, xr, reduced=True), _apply(plan, xr, reduced=True)
    assert np.array_equal(r1, r2)
    assert rel_err(r1, oplan.reduced_apply(xr)) <= TOL
    # two right-hand sides, and FP32
    X = np.concatenate([x, 2.0 * x])
    Y = _apply(plan, X, nrhs=2)
    assert np.array_equal(Y[: plan.n_full], y1)
    x32 = x.astype(np.float32)
    a, b = _apply(plan, x32), _apply(plan, x32)
    assert np.array_equal(a, b) and rel_err(a, oplan.apply(x)) <= 2e-5


def test_deterministic_apply_with_long_expansions(cuda):
    """Level-5 L-shape: hanging-node expansions of up to 72 terms, the tail buffers of the default
    path are bypassed; the result equals the default path's to rounding and repeats bitwise."""
    from grico_b200 import batched as bt

    plan = gb.compile(bt.lshape_problem(max_level=5))
    xr = sample_vector(plan.n_reduced, seed=5)
    d1, d2 = _apply(plan, xr, reduced=True), _apply(plan, xr, reduced=True)
    assert np.array_equal(d1, d2)
    ref = _apply(plan, xr, reduced=True, flags=L.GRICO_FLAG_HOST_POINTERS)
    assert rel_err(d1, ref) <= TOL


@pytest.mark.parametrize("name", sorted(DG_CASES))
def test_deterministic_sipg_apply(cuda, name):
    oplan, _, plan = sipg_case(**DG_CASES[name])
    x = sample_vector(plan.n_full, seed=11)
    y1, y2 = _apply(plan, x), _apply(plan, x)
    assert np.array_equal(y1, y2)
    assert rel_err(y1, oplan.apply(x)) <= TOL


@pytest.mark.parametrize("builder", ["annulus_hanging", "box_nitsche_3d"])
def test_deterministic_finite_cell_apply(cuda, builder):
    oplan, _, plan, _ = {"annulus_hanging": lambda: fc_cases.annulus(hanging=True, refine=1, depth=2),
                         "box_nitsche_3d": lambda: fc_cases.box_nitsche(dim=3, degree=2, refine=1, mu=0.5)}[builder]()
    x = sample_vector(plan.n_full, seed=11)
    y1, y2 = _apply(plan, x), _apply(plan, x)
    assert np.array_equal(y1, y2)
    assert rel_err(y1, oplan.apply(x)) <= TOL

"""Residual, tangent and Newton on the GPU (residual!, tangent_apply!, solve.jl:277-333) for the
Bratu accumulator of examples/nonlinear_bratu/driver.jl, against the oracle.  FP64 1e-12
relative for residual, tangent and diagonal; Newton solutions within 1e-9."""
import numpy as np
import pytest

import grico_oracle as go
import grico_b200 as gb
from grico_b200 import nonlinear as nl
from bratu_cases import bratu
from cases import rel_err

pytestmark = pytest.mark.gpu


def _state(oplan, seed):
    n = len(oplan.solve_dofs)
    return 0.1 * np.random.default_rng(seed).standard_normal(n)


@pytest.mark.parametrize("cfg", [dict(), dict(roots=(3, 2), degree=4, lam=1.0, amplitude=0.2),
                                 dict(roots=(2, 2, 2), degree=4, lam=1.0, amplitude=0.2)])
def test_residual_tangent_diagonal_match_oracle(cuda, cfg):
    oplan, plan, c = bratu(**cfg)
    ur = _state(oplan, 1)
    x = oplan.expand(ur, include_shift=True)
    r_ref = oplan.project(go.bratu_residual(oplan, x, c["lam"], c["src_scalar"]))
    assert rel_err(nl.reduced_residual(plan, ur), r_ref) <= 1e-12
    d = np.random.default_rng(2).standard_normal(len(ur))
    t_ref = oplan.project(go.bratu_tangent(oplan, x, oplan.expand(d), c["lam"]))
    nl.set_tangent_state(plan, ur)
    try:
        assert rel_err(gb.reduced_apply(plan, d), t_ref) <= 1e-12
        n = len(ur)
        diag_ref = np.array([oplan.project(go.bratu_tangent(oplan, x, oplan.expand(np.eye(n)[j]), c["lam"]))[j]
                             for j in range(n)])
        assert rel_err(gb.reduced_diagonal(plan), diag_ref) <= 1e-12
    finally:
        nl.set_tangent_state(plan, None)
    # clearing the state restores the linear operator
    lin_ref = oplan.reduced_apply(d)
    assert rel_err(gb.reduced_apply(plan, d), lin_ref) <= 1e-12


def test_newton_matches_oracle_and_reference_bound(cuda):
    """test/examples.jl:30-35: L2 error <= 2e-3 on roots (2, 2), degree 2, lam 0.5, A 0.1."""
    oplan, plan, c = bratu()
    state, its = gb.newton_solve(plan, maxiter=10, relative_tolerance=1e-10, absolute_tolerance=1e-10,
                                 linear_relative_tolerance=1e-10)
    ur_ref, its_ref = go.bratu_newton(oplan, c["lam"], c["src_scalar"])
    assert abs(its - its_ref) <= 1
    assert rel_err(state.coefficients, oplan.expand(ur_ref, include_shift=True)) <= 1e-9
    assert gb.l2_error(state, c["exact"]) <= 2.0e-3


def test_newton_example_defaults(cuda):
    """The example's own configuration (driver.jl:27-30: 4 x 4 roots, degree 3, lam 1, A 0.2)."""
    _, plan, c = bratu(roots=(4, 4), degree=3, lam=1.0, amplitude=0.2)
    state, its = gb.newton_solve(plan, maxiter=10, relative_tolerance=1e-10, absolute_tolerance=1e-10,
                                 linear_relative_tolerance=1e-10)
    err = gb.l2_error(state, c["exact"])
    print("Bratu example: Newton iterations", its, "L2 error", err)
    assert its <= 6 and err <= 1e-4

"""GPU parity at the benchmark workloads' full sizes.

* 64^3 cells, p = 4 (16,974,593 dofs): the device's full apply! and reduced apply against the
  oracle's C restatement of the reference's tensor schedule (D + D^2 contractions per cell,
  coloured passes) on the oracle's own uniform numbering, to 1e-12 relative.
* 32 x 32 cells, p = 4 (examples/poisson_matrix_free_gmg/driver.jl at 32 x 32): full apply,
  reduced right-hand side, Jacobi diagonal and the CG + Jacobi solve at relative tolerance
  1e-10 against the literal Python oracle."""
import math

import numpy as np
import pytest

import grico_oracle as go
import grico_b200 as gb
from full_size_cases import (diagnostic_sample_vector, oracle_cell_sum, poisson2d_32, poisson3d_64,
                            uniform_oracle)
from cases import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def poisson64():
    plan = gb.compile(poisson3d_64())
    coords, m, ndofs, fixed = uniform_oracle((64, 64, 64), 4)
    assert plan.n_full == ndofs and np.array_equal(plan.fixed_dofs, fixed)
    return plan, coords, m


def test_poisson64_full_apply_matches_oracle(cuda, poisson64):
    plan, coords, m = poisson64
    x = diagnostic_sample_vector(plan.n_full)
    ref = oracle_cell_sum((64, 64, 64), 4, coords, m, x, 1.0 / 64)
    ref[plan.fixed_dofs] = x[plan.fixed_dofs]  # fixed rows: y = x (assembly.jl:1893-1920)
    assert rel_err(gb.apply(plan, x), ref) <= TOL


def test_poisson64_reduced_apply_matches_oracle(cuda, poisson64):
    plan, coords, m = poisson64
    xr = np.random.default_rng(64).uniform(-1.0, 1.0, plan.n_reduced)
    xf = np.zeros(plan.n_full)
    xf[plan.solve_dofs] = xr
    ref = oracle_cell_sum((64, 64, 64), 4, coords, m, xf, 1.0 / 64)[plan.solve_dofs]
    assert rel_err(gb.reduced_apply(plan, xr), ref) <= TOL


@pytest.fixture(scope="module")
def poisson32():
    od = go.Domain((0.0, 0.0), (1.0, 1.0), (32, 32))
    osp = go.Space(od, 4, basis="full")
    src = lambda x: 2 * math.pi ** 2 * math.sin(math.pi * x[0]) * math.sin(math.pi * x[1])
    oplan = go.Plan(osp, mu=0.0, kappa=1.0, source=src, dirichlet=[(a, s, 0.0) for a in (1, 2) for s in (1, 2)])
    plan = gb.compile(poisson2d_32())
    assert plan.n_full == osp.ndofs == 129 ** 2
    assert plan.n_reduced == len(oplan.solve_dofs) == 127 ** 2
    return oplan, plan


def test_poisson32_apply_rhs_diagonal(cuda, poisson32):
    oplan, plan = poisson32
    x = diagnostic_sample_vector(plan.n_full)
    assert rel_err(gb.apply(plan, x), oplan.apply(x)) <= TOL
    assert rel_err(gb.reduced_rhs(plan), oplan.reduced_rhs()) <= TOL
    assert rel_err(gb.reduced_diagonal(plan), oplan.jacobi_diagonal()) <= TOL


def test_poisson32_cg_jacobi_solve(cuda, poisson32):
    oplan, plan = poisson32
    state = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-10)
    d = oplan.jacobi_diagonal()
    xr, iters = go.cg_solve(oplan.reduced_apply, oplan.reduced_rhs(), precond=lambda r: r / d, rtol=1e-10)
    assert abs(state.report.iterations - iters) <= 1
    assert rel_err(state.coefficients, oplan.expand(xr, include_shift=True)) <= 1e-9
    exact = lambda X: np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1])
    assert gb.l2_error(state, exact) <= 1e-8

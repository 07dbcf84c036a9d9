"""Symmetric interior-penalty DG (interface_apply!, accumulators.jl:1576-1616, with the SIPG
form of benchmark/sine_poisson_sipg.jl) on the GPU against the oracle.

FP64 tolerance 1e-12 relative (atomic scatter order); FP32 2e-5."""
import math

import numpy as np
import pytest

import grico_b200 as gb
from cases import rel_err, sample_vector
from dg_cases import sipg_case
from test_dg_host import CASES, _kat_1d_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("name", sorted(CASES))
def test_sipg_apply_matches_oracle(cuda, name):
    oplan, _, plan = sipg_case(**CASES[name])
    x = sample_vector(plan.n_full, seed=11)
    assert rel_err(gb.apply(plan, x), oplan.apply(x)) <= TOL
    xr = sample_vector(plan.n_reduced, seed=12)
    assert rel_err(gb.reduced_apply(plan, xr), oplan.reduced_apply(xr)) <= TOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_sipg_diagonal_matches_oracle(cuda, name):
    oplan, _, plan = sipg_case(**CASES[name])
    ref = oplan.reduced_diagonal()
    assert ref is not None
    assert rel_err(gb.reduced_diagonal(plan), ref) <= TOL


def test_sipg_two_rhs_and_fp32(cuda):
    oplan, _, plan = sipg_case(**CASES["2d_hp_hanging"])
    xs = np.stack([sample_vector(plan.n_full, seed=s) for s in (1, 2)])
    ys = gb.apply(plan, xs.reshape(-1), nrhs=2).reshape(2, -1)
    for k in range(2):
        assert rel_err(ys[k], oplan.apply(xs[k])) <= TOL
    y32 = gb.apply(plan, xs[0].astype(np.float32))
    assert rel_err(y32, oplan.apply(xs[0])) <= 2e-5


def test_sipg_interface_kat_1d(cuda):
    """The product's interface operator equals the hand-derived 1-D matrix."""
    d = gb.Domain((0.0,), (1.0,), (2,))
    s = gb.HpSpace(d, gb.SpaceOptions(degree=gb.UniformDegree(1), continuity="dg"))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.0, 0.0))
    gb.add_interface(prob, gb.SIPG(3.0))
    plan = gb.compile(prob)
    n = plan.n_full
    A = np.stack([gb.apply(plan, np.eye(n)[j]) for j in range(n)], axis=1)
    order = [int(plan.space.term_index[plan.space.term_offsets[plan.space.box_offsets[li] + m]])
             for li in range(2) for m in range(2)]
    assert np.allclose(A[np.ix_(order, order)], _kat_1d_matrix(3.0), atol=1e-13)


def test_sipg_poisson_manufactured_solution(cuda):
    """-lap u = f on the unit square, u = sin(pi x) sin(pi y), DG p = 3 on an 8 x 8 mesh with a
    hanging refinement, SIPG penalty 10, weak homogeneous Dirichlet: CG + Jacobi converges and
    the L2 error is at the discretisation level."""
    exact = lambda X: np.sin(math.pi * X[:, 0]) * np.sin(math.pi * X[:, 1])
    src = lambda X: 2.0 * math.pi ** 2 * exact(X)
    _, prob, plan = sipg_case(dim=2, degree=3, refine=2, hanging=True, penalty=10.0, source=src)
    state = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-11)
    assert state.report.status == 0
    err = gb.relative_l2_error(state, exact)
    print("SIPG relative L2 error", err, "iterations", state.report.iterations)
    assert err <= 2e-4

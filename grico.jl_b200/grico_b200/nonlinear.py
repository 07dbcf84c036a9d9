"""Residual problems and Newton's method on the device (solve.jl:277-333, assembly.jl:985-1083).

Julia accumulator callbacks cannot run on the GPU, so the residual form is a closed set: the
reaction-diffusion accumulator of examples/nonlinear_bratu/driver.jl,

    residual  R(u; v) = int kappa grad v . grad u + (lam exp(u) - f) v,
    tangent   J(u)[du; v] = int kappa grad v . grad du + lam exp(u) v du.

The plan compiles the linear part (diffusion) as an affine plan.  A residual evaluates u at
the quadrature points (grico_eval_points), forms the load f - lam exp(u) there and subtracts
its projection from the linear apply; the tangent is the same plan with the pointwise mass
lam exp(u(x_q)) (grico_plan_set_mass_points), so the ordinary apply, reduced apply and
diagonal kernels run it.  Newton follows the reference: reduced residual, stop at
max(atol, rtol ||R_0||), correction from CG on the tangent (identity preconditioner, as
default_tangent_linear_solve uses for SPD problems, solve.jl:686-711), damped update.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .problem import (SPD, AffineProblem, AssemblyPlan, Diffusion, Load, State, compile as _compile, expand_reduced,
                      _source_points)


class ExpReaction:
    """The Bratu accumulator (examples/nonlinear_bratu/driver.jl:32-54): value channel
    lam exp(u) - source(x), gradient channel kappa grad u; tangent value channel
    lam exp(u) du."""

    def __init__(self, lam, source=None, kappa=1.0):
        self.lam = float(lam)
        self.source = source
        self.kappa = float(kappa)


class ResidualProblem(AffineProblem):
    """ResidualProblem(u; operator_class) with one ExpReaction accumulator and Dirichlet
    constraints."""

    def __init__(self, field, operator_class=None):
        super().__init__(field, operator_class=operator_class or SPD())
        self.reaction = None


def add_residual_accumulator(problem, test_field, trial_field, op):
    """add_cell_accumulator!(problem::ResidualProblem, test, trial, op) (accumulators.jl:372-411)."""
    if not isinstance(problem, ResidualProblem):
        raise TypeError("residual accumulators need a ResidualProblem")
    if test_field is not problem.field or trial_field is not problem.field:
        raise ValueError("the B200 plan supports one scalar field")
    if not isinstance(op, ExpReaction):
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"residual form {type(op).__name__} is not supported by the GPU plan")
    if problem.reaction is not None:
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "one residual accumulator on the GPU plan")
    problem.reaction = op
    problem.cell_operators = [Diffusion(op.kappa)]
    problem.rhs_operators = [Load(op.source)] if op.source is not None else []
    return problem


def compile(problem):
    """compile(problem::ResidualProblem): the affine plan of the linear part, with the reaction."""
    if not isinstance(problem, ResidualProblem) or problem.reaction is None:
        raise ValueError("compile expects a ResidualProblem with its accumulator")
    plan = _compile(problem)
    if plan.point_batches:
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "residual plans support tensor cells only")
    plan.reaction = problem.reaction
    return plan


def _point_values(plan, u_full):
    """u at the quadrature points of every cell batch: list of [n_cells, nq] arrays."""
    outs = [np.zeros((len(b.cells), b.points.shape[1])) for b in plan.batches]
    ptrs = (L.f64p * len(outs))(*[L.ptr(o, C.c_double) for o in outs])
    u = np.ascontiguousarray(u_full, dtype=np.float64)
    L.check(L.lib().grico_eval_points(plan.handle, L.ptr(u, C.c_double), 0, ptrs, L.GRICO_FLAG_HOST_POINTERS),
            "eval points")
    return outs


def _reduced_load(plan, arrays):
    ptrs = (L.f64p * len(arrays))(*[L.ptr(np.ascontiguousarray(a), C.c_double) for a in arrays])
    out = np.zeros(plan.n_reduced)
    L.check(L.lib().grico_reduced_rhs(plan.handle, ptrs, L.ptr(out, C.c_double), L.GRICO_FLAG_HOST_POINTERS), "rhs")
    return out


def _set_mass_points(plan, arrays):
    if arrays is None:
        L.check(L.lib().grico_plan_set_mass_points(plan.handle, None, 0), "mass points")
        return
    keep = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
    ptrs = (L.f64p * len(keep))(*[L.ptr(a, C.c_double) for a in keep])
    L.check(L.lib().grico_plan_set_mass_points(plan.handle, ptrs, L.GRICO_FLAG_HOST_POINTERS), "mass points")


def reduced_residual(plan, ured):
    """P^T R(shift + P u_red) (assembly.jl:985-1048 on the reduced space)."""
    op = plan.reaction
    uq = _point_values(plan, expand_reduced(plan, ured))
    f = _source_points(plan)
    load = []
    for b, u, fb in zip(plan.batches, uq, f):
        g = -op.lam * np.exp(u)
        if fb is not None:
            g = g + fb.reshape(g.shape)
        load.append(g)
    lin = np.zeros(plan.n_reduced)
    x = np.ascontiguousarray(ured, dtype=np.float64)
    L.check(L.lib().grico_reduced_apply(plan.handle, L.ptr(x, C.c_double), L.ptr(lin, C.c_double), 1,
                                        L.GRICO_PREC_FP64, L.GRICO_FLAG_HOST_POINTERS, None), "apply")
    # reduced_rhs computes P^T (load - K shift): R = P^T K P u_red - that
    return lin - _reduced_load(plan, load)


def set_tangent_state(plan, ured):
    """Make the plan's operator the tangent J(u) at u = shift + P u_red (tangent_apply!,
    assembly.jl:1050-1083); clear with set_tangent_state(plan, None)."""
    if ured is None:
        _set_mass_points(plan, None)
        return
    uq = _point_values(plan, expand_reduced(plan, ured))
    _set_mass_points(plan, [plan.reaction.lam * np.exp(u) for u in uq])


def newton_solve(plan, initial_state=None, maxiter=20, relative_tolerance=None, absolute_tolerance=None,
                 damping=1.0, linear_relative_tolerance=None, linear_absolute_tolerance=0.0, linear_maxiter=None,
                 jacobi=False):
    """solve(plan::ResidualProblem plan; ...) (solve.jl:277-333).  Returns (State, iterations)."""
    eps = math.sqrt(np.finfo(np.float64).eps)
    rtol = eps if relative_tolerance is None else float(relative_tolerance)
    atol = eps if absolute_tolerance is None else float(absolute_tolerance)
    lrtol = eps if linear_relative_tolerance is None else float(linear_relative_tolerance)
    lmax = max(1000, 2 * plan.n_reduced) if linear_maxiter is None else int(linear_maxiter)
    if maxiter < 1 or not damping > 0:
        raise ValueError("maxiter and damping must be positive")
    u = np.zeros(plan.n_reduced)
    if initial_state is not None:
        c = np.asarray(initial_state, dtype=np.float64)
        u = c[plan.solve_dofs].copy() if c.size == plan.n_full else c.copy()
    r0 = None
    try:
        for it in range(maxiter):
            r = reduced_residual(plan, u)
            rn = float(np.linalg.norm(r))
            r0 = rn if r0 is None else r0
            if rn <= max(atol, rtol * r0):
                return State(plan, expand_reduced(plan, u)), it
            set_tangent_state(plan, u)
            du = np.zeros(plan.n_reduced)
            opts = L.GricoSolveOptions(lrtol, float(linear_absolute_tolerance), int(min(lmax, 2 ** 31 - 1)),
                                       L.GRICO_PRECOND_JACOBI if jacobi else L.GRICO_PRECOND_IDENTITY, 30, 0)
            rep = L.GricoSolveReport()
            rhs = np.ascontiguousarray(-r)
            L.check(L.lib().grico_cg_solve(plan.handle, None, L.ptr(rhs, C.c_double), L.ptr(du, C.c_double),
                                           C.byref(opts), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS), "tangent solve")
            set_tangent_state(plan, None)
            u = u + damping * du
        r = reduced_residual(plan, u)
        if float(np.linalg.norm(r)) <= max(atol, rtol * (r0 or 0.0)):
            return State(plan, expand_reduced(plan, u)), maxiter
        raise L.GricoError(L.GRICO_ERR_NOT_CONVERGED, f"Newton solve did not converge in {maxiter} iterations")
    finally:
        set_tangent_state(plan, None)

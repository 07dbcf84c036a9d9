"""GPU parity: the sm_100a cell kernels through the C ABI against the oracle.

FP64 tolerance: max|y - y_oracle| / max|y_oracle| <= 1e-12 (the reference's own test
tolerance for coefficient data is 1e-12; the GPU sums contributions in another order, so
bit equality is not expected for floating point results)."""
import math

import numpy as np
import pytest

import grico_b200 as gb
from cases import CASES, build, rel_err, sample_vector

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_apply_matches_oracle(cuda, name):
    oplan, prob = build(name, mu=0.7, kappa=1.3)
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full)
    y = gb.apply(plan, x)
    assert rel_err(y, oplan.apply(x)) <= TOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_reduced_apply_matches_oracle(cuda, name):
    oplan, prob = build(name)
    plan = gb.compile(prob)
    xr = sample_vector(plan.n_reduced, seed=7)
    assert plan.n_reduced == len(oplan.solve_dofs)
    assert rel_err(gb.reduced_apply(plan, xr), oplan.reduced_apply(xr)) <= TOL


@pytest.mark.parametrize("name", ["2d_p4", "3d_p4", "3d_p1", "3d_p3_trunk", "1d_p3", "2d_p3_over",
                                  "2d_p2_hanging", "3d_p2_hanging"])
def test_reduced_diagonal_matches_oracle(cuda, name):
    """Direct maps: local diagonal kernels (assembly.jl:662-675); hanging maps: the exact
    diagonal against the reference's probing fallback (solve.jl:722-738)."""
    oplan, prob = build(name, mu=0.25, kappa=2.0)
    plan = gb.compile(prob)
    assert rel_err(gb.reduced_diagonal(plan), oplan.jacobi_diagonal()) <= TOL


def test_hanging_diagonal_with_variable_coefficient(cuda):
    kfn = lambda x: 1.0 + x[:, 0] ** 2 + 0.5 * x[:, 1]
    oplan, prob = build("3d_p2_hanging", mu=0.3, kappa_fn=kfn)
    plan = gb.compile(prob)
    assert rel_err(gb.reduced_diagonal(plan), oplan.probe_reduced_diagonal()) <= TOL


def test_variable_coefficient_apply(cuda):
    kfn = lambda x: np.exp(np.sin(3.0 * x[:, 0]) * np.cos(2.0 * x[:, 1]) + 0.3 * x[:, 2])
    oplan, prob = build("3d_p4", kappa_fn=kfn)
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full, seed=3)
    assert rel_err(gb.apply(plan, x), oplan.apply(x)) <= TOL


@pytest.mark.parametrize("name", ["2d_p4", "3d_p4", "2d_p2_hanging", "3d_p2_hanging", "1d_p3"])
def test_reduced_rhs_matches_oracle(cuda, name):
    D = len(CASES[name][0])
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1) * D * np.pi ** 2 + 0.5 * x[:, 0]
    oplan, prob = build(name, source=src)
    plan = gb.compile(prob)
    assert rel_err(gb.reduced_rhs(plan), oplan.reduced_rhs()) <= TOL


@pytest.mark.parametrize("name,value", [("2d_p4", 0.0), ("2d_p4", 1.5), ("3d_p2_hanging", 0.75), ("1d_p3", -2.0)])
def test_full_rhs_matches_oracle(cuda, name, value):
    """rhs! on the full layout (assembly.jl:488-507): load vector, constraint rows carry their
    values (_write_constraint_rhs!, assembly.jl:1876-1891)."""
    D = len(CASES[name][0])
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1) * D * np.pi ** 2 + 0.5 * x[:, 0]
    oplan, prob = build(name, mu=0.4, source=src, dirichlet_value=value)
    plan = gb.compile(prob)
    ref = oplan.rhs_physical()
    for d, v in zip(oplan.fixed, oplan.fixed_values):
        ref[d - 1] = v
    for (pivot, _, _, r) in oplan.rows:
        ref[pivot - 1] = r
    assert rel_err(gb.rhs(plan), ref) <= TOL
    # the reduced right-hand side with the Dirichlet shift, same data
    assert rel_err(gb.reduced_rhs(plan), oplan.reduced_rhs()) <= TOL


def test_mass_kat_1d(cuda):  # test/matrix_free.jl:538-579: apply(mass, ones(2)) ≈ [0.5, 0.5]; rhs ≈ [0.5, 0.5]
    d = gb.Domain((0.0,), (1.0,), (1,))
    s = gb.HpSpace(d, gb.SpaceOptions(degree=gb.UniformDegree(1), continuity="dg"))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Mass(1.0))
    gb.add_cell_accumulator(prob, u, gb.Load(lambda x: np.ones(len(x))))
    plan = gb.compile(prob)
    assert np.allclose(gb.apply(plan, np.ones(2)), [0.5, 0.5], atol=1e-12)
    assert np.allclose(gb.reduced_rhs(plan), [0.5, 0.5], atol=1e-12)


@pytest.mark.parametrize("name", ["2d_p4", "3d_p4", "3d_p2_hanging"])
def test_cg_jacobi_matches_oracle(cuda, name):
    import grico_oracle as go

    D = len(CASES[name][0])
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1) * D * np.pi ** 2
    oplan, prob = build(name, source=src)
    plan = gb.compile(prob)
    state = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-12)
    diag = oplan.jacobi_diagonal()
    pre = lambda r: r / diag
    xr, _ = go.cg_solve(oplan.reduced_apply, oplan.reduced_rhs(), precond=pre, rtol=1e-12)
    ref = oplan.expand(xr, include_shift=True)
    assert rel_err(state.coefficients, ref) <= 1e-9


def test_poisson_example_accuracy(cuda):  # test/examples.jl:6-12: 2x2, p=2, L2 <= 2e-2
    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(2)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    exact = lambda x: np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1])
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(lambda x: 2 * np.pi ** 2 * exact(x)))
    for a in (1, 2):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    state = gb.solve(prob, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-10)
    assert gb.l2_error(state, exact) <= 2e-2


def test_fgmres_matches_cg(cuda):
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1)
    _, prob = build("3d_p4", source=src)
    plan = gb.compile(prob)
    a = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-12)
    b = gb.solve(plan, solver=gb.FGMRESSolver(gb.JacobiPreconditioner(), restart=30), relative_tolerance=1e-12)
    assert rel_err(b.coefficients, a.coefficients) <= 1e-8  # both stop at ||r|| <= 1e-12 ||b||


def test_multi_rhs_equals_single(cuda):
    _, prob = build("3d_p4", mu=0.5)
    plan = gb.compile(prob)
    xs = np.stack([sample_vector(plan.n_full, seed=s) for s in (1, 2, 3)])
    ys = gb.apply(plan, xs.reshape(-1).copy(), nrhs=3).reshape(3, -1)
    for k in range(3):
        assert rel_err(ys[k], gb.apply(plan, xs[k].copy())) <= 1e-14


def test_fp32_apply_close_to_fp64(cuda):
    _, prob = build("3d_p4", mu=0.5)
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full, seed=11)
    y64 = gb.apply(plan, x)
    y32 = gb.apply(plan, x.astype(np.float32))
    assert y32.dtype == np.float32
    assert rel_err(y32, y64) <= 1e-5


def test_device_tensors_and_aliasing(cuda):
    import torch

    _, prob = build("3d_p4")
    plan = gb.compile(prob)
    x = torch.tensor(sample_vector(plan.n_full, seed=5), device="cuda")
    y = gb.apply(plan, x)
    assert rel_err(y.cpu().numpy(), gb.apply(plan, x.cpu().numpy())) <= 1e-14
    with pytest.raises(ValueError):
        gb.apply_(x, plan, x)
    with pytest.raises(ValueError):
        gb.apply(plan, np.zeros(plan.n_full + 1))


def test_cg_not_converged_status(cuda):
    _, prob = build("3d_p4", source=lambda x: np.ones(len(x)))
    plan = gb.compile(prob)
    with pytest.raises(gb.GricoError) as err:
        gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-14, maxiter=2)
    assert err.value.code == -3


@pytest.mark.parametrize("name", ["3d_p4", "3d_p2_hanging", "3d_p3_trunk", "3d_p1", "3d_p4_kappa"])
def test_every_kernel_variant_matches_oracle(cuda, name):
    """All nine 3-D tensor-kernel variants (three cells-per-block sizes; one block per cell group,
    or the persistent pipelined kernel with even-odd or direct contractions) against the oracle:
    mass + diffusion, hanging-node tails,
    trunk (inactive) modes, tabulated coefficients; full and reduced layouts; 2 right-hand sides."""
    from grico_b200 import batched as bt

    kfn = lambda x: np.exp(np.sin(3.0 * x[:, 0]) * np.cos(2.0 * x[:, 1]) + 0.3 * x[:, 2])
    base = name.replace("_kappa", "")
    oplan, prob = build(base, mu=0.7, kappa=1.3, kappa_fn=kfn if name.endswith("_kappa") else None)
    plan = gb.compile(prob)
    xs = np.stack([sample_vector(plan.n_full, seed=s) for s in (5, 6)])
    xr = np.stack([sample_vector(plan.n_reduced, seed=s) for s in (7, 8)])
    ref_full = [oplan.apply(v) for v in xs]
    ref_red = [oplan.reduced_apply(v) for v in xr]
    from grico_b200 import _lib as L

    for var in range(L.TILE_VARIANTS):
        bt.set_tiles(plan, [var] * len(plan.batches))
        yf = gb.apply(plan, xs.reshape(-1), nrhs=2).reshape(2, -1)
        yr = gb.reduced_apply(plan, xr.reshape(-1), nrhs=2).reshape(2, -1)
        for k in range(2):
            assert rel_err(yf[k], ref_full[k]) <= TOL, (var, k)
            assert rel_err(yr[k], ref_red[k]) <= TOL, (var, k)


def test_batch_event_timing(cuda):
    """GRICO_FLAG_TIME_BATCHES records one event pair per batch launch; the query averages them,
    counts the launches, resets the record, and the flag leaves the result unchanged."""
    import ctypes as C
    from grico_b200 import _lib as L

    oplan, prob = build("3d_p2_hanging", mu=0.7, kappa=1.3)
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full, seed=4)
    y0 = gb.apply(plan, x)
    nb = len(plan.batches) + len(plan.point_batches)
    y = np.zeros_like(x)
    for _ in range(3):
        assert L.lib().grico_apply(plan.handle, L.ptr(x, C.c_double), L.ptr(y, C.c_double), 1, L.GRICO_PREC_FP64,
                                   L.GRICO_FLAG_HOST_POINTERS | L.GRICO_FLAG_TIME_BATCHES, None) == 0
    assert rel_err(y, y0) <= TOL
    ms = np.zeros(nb)
    n = np.zeros(nb, dtype=np.int64)
    assert L.lib().grico_plan_batch_times(plan.handle, L.ptr(ms, C.c_double), L.ptr(n, C.c_int64), nb) == 0
    assert (n == 3).all() and (ms > 0).all()
    assert L.lib().grico_plan_batch_times(plan.handle, L.ptr(ms, C.c_double), L.ptr(n, C.c_int64), nb) == 0
    assert (n == 0).all() and (ms == 0).all()
    assert L.lib().grico_plan_batch_times(plan.handle, L.ptr(ms, C.c_double), None, nb + 1) != 0


def test_async_host_pointer_applies(cuda):
    """GRICO_FLAG_ASYNC: three applies with different inputs in flight on two streams (the third
    reuses the first staging slot) give the synchronous results once the streams are drained."""
    import ctypes as C
    import torch
    from grico_b200 import _lib as L

    _, prob = build("3d_p4", mu=0.7, kappa=1.3)
    plan = gb.compile(prob)
    xs = [torch.tensor(sample_vector(plan.n_full, seed=s)).pin_memory() for s in (21, 22, 23)]
    ys = [torch.zeros(plan.n_full, dtype=torch.float64).pin_memory() for _ in range(3)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for k in range(3):
        assert L.lib().grico_apply(plan.handle, xs[k].data_ptr(), ys[k].data_ptr(), 1, L.GRICO_PREC_FP64,
                                   L.GRICO_FLAG_HOST_POINTERS | L.GRICO_FLAG_ASYNC, streams[k % 2].cuda_stream) == 0
    for s in streams:
        s.synchronize()
    for k in range(3):
        assert rel_err(ys[k].numpy(), gb.apply(plan, xs[k].numpy())) <= TOL


@pytest.mark.parametrize("p,extra", [(1, 1), (2, 1), (3, 1), (4, 1), (5, 1), (6, 1), (7, 1), (8, 1),
                                     (1, 2), (2, 2), (3, 2), (4, 2)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_even_odd_pipelined_kernel_matches_oracle(cuda, p, extra, prec):
    """The pipelined kernel with even-odd contractions (variants 3-5) and with direct ones
    (6-8) on plain maps (uniform mesh, homogeneous Dirichlet, constant coefficients) against the
    oracle's C tensor schedule, every isotropic shape q = p + 1 and q = p + 2."""
    from grico_b200 import _lib as L
    from grico_b200 import batched as bt
    from sharded_cases import full_apply

    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (4, 4, 4))
    gb.uniform_refine(d, 1)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p),
                                      quadrature=gb.DegreePlusQuadrature(extra)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.7, 1.3))
    for a in (1, 2, 3):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full, seed=3)
    ref = full_apply(plan, x)
    ref[plan.fixed_dofs] = x[plan.fixed_dofs]
    xv = x.astype(np.float32) if prec == "fp32" else x
    tol = 2e-5 if prec == "fp32" else TOL
    for var in range(3, L.TILE_VARIANTS):
        bt.set_tiles(plan, [var] * len(plan.batches), precision=prec)
        y = gb.apply(plan, xv)
        assert rel_err(y.astype(np.float64), ref) <= tol, var


@pytest.mark.parametrize("roots", [(1, 1, 1), (7, 1, 1), (3, 2, 2), (11, 3, 1)])
@pytest.mark.parametrize("p", [2, 4])
def test_pipelined_kernel_ragged_cell_groups(cuda, roots, p):
    """Cell counts below one group and with a ragged last group (1, 7, 12, 33 cells; groups of
    3..56 cells): every variant against the oracle's C tensor schedule, no constraints (every
    map entry a dof)."""
    from grico_b200 import _lib as L
    from grico_b200 import batched as bt
    from sharded_cases import full_apply

    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 0.5, 2.0), roots)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.3, 1.1))
    plan = gb.compile(prob)
    x = sample_vector(plan.n_full, seed=21)
    ref = full_apply(plan, x)
    for prec, tol in (("fp64", TOL), ("fp32", 2e-5)):
        xv = x.astype(np.float32) if prec == "fp32" else x
        for var in range(L.TILE_VARIANTS):
            bt.set_tiles(plan, [var] * len(plan.batches), precision=prec)
            assert rel_err(gb.apply(plan, xv).astype(np.float64), ref) <= tol, (prec, var)


def test_all_dofs_fixed(cuda):
    """A single p=1 cell with Dirichlet data on every face: no free dof.  The reduced system is
    empty; the full apply writes the constraint rows (y = x) and CG returns at once."""
    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(1)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion(1.0))
    for a in (1, 2, 3):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    plan = gb.compile(prob)
    assert plan.n_reduced == 0 and plan.n_full == 8
    x = sample_vector(8, seed=2)
    assert np.array_equal(gb.apply(plan, x), x)
    state = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()))
    assert state.report.iterations == 0
    assert np.array_equal(state.coefficients, np.zeros(8))

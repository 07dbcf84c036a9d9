"""Sharded plans on the device: several shards held by one process on one GPU (the collective
is then the in-process sum), against the unsharded plan."""
import numpy as np
import pytest

import grico_b200 as gb
from grico_b200.sharded import ShardedOperator, ShardPlan, gather_reduced, sharded_cg
from sharded_cases import poisson

pytestmark = pytest.mark.gpu

CASES = {
    "3d_p4": dict(D=3, roots=(4, 4, 4), p=4, rounds=1),
    "2d_hanging_p3": dict(D=2, roots=(2, 1), p=3, extent=(2.0, 1.0), refine=lambda g: g.refine(2, 2)),
}


def _problem(name, source=None):
    c = dict(CASES[name])
    prob = poisson(c.pop("D"), c.pop("roots"), c.pop("p"), mass=0.25, **c)
    if source is not None:
        gb.add_cell_accumulator(prob, prob.field, gb.Load(source))
    return prob


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("parts", [2, 3])
def test_sharded_apply_matches_unsharded(cuda, name, parts):
    import torch

    plan = gb.compile(_problem(name))
    shards = [ShardPlan(plan, r, parts) for r in range(parts)]
    op = ShardedOperator(shards)
    x = np.random.default_rng(11).standard_normal(plan.n_reduced)
    ref = gb.reduced_apply(plan, x)
    ys = [op.ops.vector(s.n_reduced) for s in shards]
    op.apply([op.ops.upload(s.scatter(x)) for s in shards], ys)
    torch.cuda.synchronize()
    scale = np.max(np.abs(ref))
    for s, y in zip(shards, ys):
        got = y.cpu().numpy()[: s.n_reduced]
        assert np.max(np.abs(got - ref[s.global_reduced])) <= 1e-12 * scale


@pytest.mark.parametrize("name", sorted(CASES))
def test_sharded_rhs_matches_unsharded(cuda, name):
    src = lambda X: np.prod(np.sin(np.pi * X), axis=1) + 1.0
    plan = gb.compile(_problem(name, source=src))
    ref = gb.reduced_rhs(plan)
    shards = [ShardPlan(plan, r, 3) for r in range(3)]
    op = ShardedOperator(shards)
    for s, b in zip(shards, op.rhs()):
        got = b.cpu().numpy()[: s.n_reduced]
        assert np.max(np.abs(got - ref[s.global_reduced])) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("jacobi", [True, False])
def test_sharded_cg_matches_unsharded_cg(cuda, jacobi):
    src = lambda X: np.prod(np.sin(np.pi * X), axis=1)
    plan = gb.compile(_problem("3d_p4", source=src))
    pre = gb.JacobiPreconditioner() if jacobi else gb.IdentityPreconditioner()
    ref = gb.solve(plan, solver=gb.CGSolver(pre), relative_tolerance=1e-10)
    xr = ref.coefficients[plan.solve_dofs]
    shards = [ShardPlan(plan, r, 2) for r in range(2)]
    op = ShardedOperator(shards)
    xs, rep = sharded_cg(op, op.rhs(), 1e-10, maxiter=2000, jacobi=jacobi)
    assert rep.status == 0
    assert abs(rep.iterations - ref.report.iterations) <= 2
    x = gather_reduced(shards, xs, plan.n_reduced, op.ops)
    assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr)
    for s, xv in zip(shards, xs):
        assert np.max(np.abs(xv.cpu().numpy()[: s.n_reduced] - x[s.global_reduced])) <= 1e-13 * np.abs(x).max()


def test_sharded_multigrid_on_the_device_matches_the_device_vcycle(cuda):
    """The sharded V-cycle with the library's device calls (one shard, device ops) against the
    one-GPU device V-cycle of the same hierarchy (damped Jacobi V(2,2), 3-D p = 2), and CG
    preconditioned by it against the device CG + GMG solve."""
    import torch

    from grico_b200.multigrid import GeometricMultigridPreconditioner, build_multigrid
    from grico_b200.sharded import ShardedMultigrid

    # p = 2: damped Jacobi on the modal p = 4 basis stagnates (section on the reference's method)
    prob = poisson(3, (4, 4, 4), 2, mass=0.25, rounds=1)
    gb.add_cell_accumulator(prob, prob.field, gb.Load(lambda x: np.prod(np.sin(np.pi * x), axis=1)))
    plan = gb.compile(prob)
    opts = GeometricMultigridPreconditioner()
    smg = ShardedMultigrid(plan, 0, 1, opts=opts)
    dmg = build_multigrid(plan, opts)
    r = np.random.default_rng(4).standard_normal(plan.n_reduced)
    fine = smg.shards[-1]
    z = smg.apply(smg.ops.upload(fine.scatter(r)))
    zs = gather_reduced([fine], [z], plan.n_reduced, ops=smg.ops)
    zd = dmg.vcycle(r)
    assert np.linalg.norm(zs - zd) <= 1e-11 * np.linalg.norm(zd)
    op = ShardedOperator([fine])
    bs = op.rhs()
    xs, rep = sharded_cg(op, bs, 1e-9, maxiter=3000, preconditioner=smg)
    st = gb.solve(plan, solver=gb.CGSolver(GeometricMultigridPreconditioner()), relative_tolerance=1e-9)
    assert rep.status == 0 and abs(rep.iterations - st.report.iterations) <= max(1, st.report.iterations // 8)
    xg = gather_reduced([fine], xs, plan.n_reduced, ops=op.ops)
    full = gb.expand_reduced(plan, xg)
    assert np.linalg.norm(full - st.coefficients) <= 1e-8 * np.linalg.norm(st.coefficients)
    torch.cuda.synchronize()

"""hp-GMG hierarchy and transfers (host side) against the oracle and the reference's KATs."""
import numpy as np
import pytest

import grico_oracle as go
import grico_b200 as gb
from grico_b200.multigrid import GeometricMultigridPreconditioner, build_hierarchy


def _product_plan(domain, degree, continuity="cg", basis=None, faces=()):
    s = gb.HpSpace(domain, gb.SpaceOptions(basis=basis or gb.FullTensorBasis(), degree=gb.UniformDegree(degree),
                                           continuity=continuity))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(1.0, 1.0))
    for a, side in faces:
        gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return gb.compile(prob, device=False)


def test_level_sizes_h_dg():  # test/multigrid.jl:153-160: [2, 4, 6]
    d = gb.Domain((0.0,), (1.0,), (1,))
    first = d.grid.refine(1, 1)
    d.grid.refine(first + 1, 1)
    plans, _ = build_hierarchy(_product_plan(d, 1, continuity="dg"), GeometricMultigridPreconditioner(), device=False)
    assert [p.n_reduced for p in plans] == [2, 4, 6]


def test_level_sizes_hp_dg():  # test/multigrid.jl:166-171: [2, 4, 8]
    d = gb.Domain((0.0,), (1.0,), (1,))
    d.grid.refine(1, 1)
    plans, _ = build_hierarchy(_product_plan(d, 3, continuity="dg"), GeometricMultigridPreconditioner(), device=False)
    assert [p.n_reduced for p in plans] == [2, 4, 8]


def _oracle_levels(od, degree, faces):
    osp = go.Space(od, degree, basis="full")
    levels = go.hp_multigrid_levels(osp)
    plans = []
    for leaves, degs in levels:
        sp = go.Space(od, lambda leaf, degs=degs: degs[leaf], basis="full", leaves=leaves)
        plans.append(go.Plan(sp, mu=1.0, kappa=1.0, dirichlet=[(a, s, 0.0) for a, s in faces]))
    return plans


def _refine_uniform(grid, depth):
    for _ in range(depth):
        for leaf in list(grid.active_leaves()):
            leaves = [int(leaf)]
            for axis in range(1, grid.D + 1):
                nxt = []
                for c in leaves:
                    f = grid.refine(c, axis)
                    nxt += [f, f + 1]
                leaves = nxt


CASES = {
    "2d_p4": ((0.0, 0.0), (1.0, 1.0), (2, 2), lambda g: _refine_uniform(g, 1), 4, [(1, 1), (2, 2)]),
    "3d_p2": ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (2, 1, 1), lambda g: _refine_uniform(g, 1), 2, [(1, 1)]),
    "2d_hanging_p2": ((0.0, 0.0), (2.0, 1.0), (2, 1), lambda g: g.refine(2, 2), 2, [(1, 1)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_transfers_match_oracle(name):
    origin, extent, roots, refine, p, faces = CASES[name]
    od, pdm = go.Domain(origin, extent, roots), gb.Domain(origin, extent, roots)
    refine(od.grid)
    refine(pdm.grid)
    oplans = _oracle_levels(od, p, faces)
    plans, transfers = build_hierarchy(_product_plan(pdm, p, faces=faces), GeometricMultigridPreconditioner(),
                                       device=False)
    assert [pl.n_reduced for pl in plans] == [len(o.solve_dofs) for o in oplans]
    for i, (off, col, val) in enumerate(transfers):
        ref = go.multigrid_transfer(oplans[i], oplans[i + 1])
        got = {}
        for r in range(len(off) - 1):
            for k in range(off[r], off[r + 1]):
                got[(int(col[k]) + 1, r + 1)] = float(val[k])
        # entries are compared to 1e-12; LU rounding can leave ~1e-17 residues where the
        # oracle's LAPACK produced exact zeros (the reference drops exact zeros only)
        keys = {k for k, v in got.items() if abs(v) > 1e-14} | {k for k, v in ref.items() if abs(v) > 1e-14}
        assert keys, "empty transfer"
        assert max(abs(got.get(k, 0.0) - ref.get(k, 0.0)) for k in keys) <= 1e-12


def test_c2_shape_hierarchy_has_p_then_h_levels():
    """64^3-shaped recipe scaled down: roots 4^3 refined once, p=4 -> p 4,2,1 then 3 single-axis
    h-merges to the roots (multigrid.jl:443-469, 568-586)."""
    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (4, 4, 4))
    gb.uniform_refine(d, 1)
    plans, transfers = build_hierarchy(_product_plan(d, 4, faces=[(a, s) for a in (1, 2, 3) for s in (1, 2)]),
                                       GeometricMultigridPreconditioner(), device=False)
    sizes = [p.n_reduced for p in plans]
    assert len(plans) == 6
    assert sizes[0] == 3 ** 3 and sizes[-1] == 31 ** 3
    assert [p.space.degrees.max() for p in plans] == [1, 1, 1, 1, 2, 4]


def test_smoother_policy():
    """multigrid.jl:347-358: auto -> Jacobi for SPD problems, GMRES otherwise; GMRES needs
    smoother_restart >= max(pre, post); CG refuses the GMRES smoother before any device work."""
    from grico_b200.multigrid import resolved_smoother

    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    plan = _product_plan(d, 2, faces=[(1, 1)])
    assert resolved_smoother(GeometricMultigridPreconditioner(), plan.problem) == "jacobi"
    plan.problem.operator_class = gb.NonsymmetricOperator()
    assert resolved_smoother(GeometricMultigridPreconditioner(), plan.problem) == "gmres"
    with pytest.raises(ValueError):
        resolved_smoother(GeometricMultigridPreconditioner(smoother="gmres", pre_smoothing_steps=9), plan.problem)
    plan.problem.operator_class = gb.SPD()
    with pytest.raises(ValueError):
        gb.solve(plan, solver=gb.CGSolver(GeometricMultigridPreconditioner(smoother="gmres")))
    with pytest.raises(ValueError):
        go.Multigrid([], pre=3, post=1, smoother="gmres", restart=2)


def test_oracle_gmres_smoother_reduces_residual():
    """The oracle's GMRES smoother minimises ||b - A(x + Z y)|| over its Krylov space, so with
    unit damping its residual is never larger than one damped-Jacobi step's."""
    od = go.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    _refine_uniform(od.grid, 1)
    oplans = _oracle_levels(od, 2, [(1, 1), (2, 2)])
    fine = oplans[-1]
    b = np.random.default_rng(1).standard_normal(len(fine.solve_dofs))
    x0 = np.zeros_like(b)
    mg_g = go.Multigrid(oplans, smoother="gmres", restart=4, omega=1.0)
    mg_j = go.Multigrid(oplans, omega=0.8)
    lv = len(oplans) - 1
    for steps in (1, 2, 4):
        xg = mg_g.smooth(lv, x0, b, steps)
        xj = mg_j.smooth(lv, x0, b, 1)
        rg = np.linalg.norm(b - fine.reduced_apply(xg))
        assert rg <= np.linalg.norm(b - fine.reduced_apply(xj)) * (1 + 1e-12)
        assert rg < np.linalg.norm(b)


def test_reference_gmg_fixture_matches_the_product_hierarchy():
    """tests/golden/reference_gmg_8cube_p4.npz (the oracle's reference-method solve at 8^3 cells,
    p = 4): its hierarchy has the level sizes the product builds for the same problem."""
    import os

    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gmg_8cube_p4.npz"))
    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (4, 4, 4))
    _refine_uniform(d.grid, 1)
    plans, _ = build_hierarchy(_product_plan(d, 4, faces=[(a, s) for a in (1, 2, 3) for s in (1, 2)]),
                               GeometricMultigridPreconditioner(), device=False)
    assert [p.n_reduced for p in plans] == fx["level_sizes"].tolist()
    assert fx["vcycle"].size == plans[-1].n_reduced
    for k in fx["cg_iterations"]:
        assert fx[f"cg_iterate_{k}"].size == (plans[-1].n_reduced + 6) // 7  # every 7th dof

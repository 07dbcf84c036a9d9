"""Finite-cell / Nitsche cases built identically in the oracle and in the product.

Shapes: the annulus of examples/annular_nitsche_fcm/driver.jl (2-D, circle surfaces), a small
spherical shell (3-D, sphere surfaces), symmetric Nitsche on the faces of a plain box, an
adaptive annulus with hanging nodes, and an explicit cell-quadrature override."""
import math

import numpy as np

import grico_oracle as go
import grico_b200 as gb

ANNULUS = dict(ri=0.35, ro=1.0, roots=(2, 2), refine=1, degree=2, depth=3, penalty=40.0)
SHELL = dict(center=(1.0, 1.0, 1.0), ri=0.4, ro=0.9, refine=2, degree=2, depth=1)


def annulus_levelset(ri, ro):
    def f(X):
        r = np.hypot(X[:, 0], X[:, 1])
        return np.maximum(r - ro, ri - r)
    return f


def annulus_exact(ri, ro):
    def f(X):
        return np.log(np.hypot(X[:, 0], X[:, 1]) / ro) / math.log(ri / ro)
    return f


def shell_levelset(c, ri, ro):
    c = np.asarray(c)

    def f(X):
        r = np.linalg.norm(X - c[None, :], axis=1)
        return np.maximum(r - ro, ri - r)
    return f


def shell_exact(X):
    return np.sin(2 * X[:, 0]) * np.cos(3 * X[:, 1]) * np.exp(0.5 * X[:, 2])


def _scalar(fn):
    return None if fn is None else (lambda x: float(np.asarray(fn(np.array([x])))[0]))


def _oracle_rules(od, osp, levelset, depth):
    rules = {}
    for li, leaf in enumerate(osp.snapshot.leaves):
        if go.classify_leaf(od, leaf, levelset) != "cut":
            continue
        r = go.finite_cell_candidates(od, leaf, osp.qshape[li], levelset, depth)
        if r is not None:
            rules[leaf] = r
    return rules


def _oracle_surfaces(od, surfaces, penalty, g):
    items = []
    for sq in surfaces:
        w, n = go.physical_surface_data(od, sq.leaf, sq.weights, sq.normals)
        items.append((sq.leaf, sq.points, w, n, penalty, _scalar(g)))
    return items


def annulus(refine=None, degree=None, depth=None, penalty=None, hanging=False, with_rhs=True, device=True):
    """(oracle plan, product problem, product plan) of the annulus with Nitsche circles."""
    o = dict(ANNULUS)
    o.update({k: v for k, v in dict(refine=refine, degree=degree, depth=depth, penalty=penalty).items() if v is not None})
    lev = annulus_levelset(o["ri"], o["ro"])
    exact = annulus_exact(o["ri"], o["ro"])
    od = go.Domain((-o["ro"], -o["ro"]), (2 * o["ro"], 2 * o["ro"]), o["roots"])
    bg = gb.Domain((-o["ro"], -o["ro"]), (2 * o["ro"], 2 * o["ro"]), o["roots"])
    go.uniform_refine(od.grid, o["refine"])
    gb.uniform_refine(bg, o["refine"])
    if hanging:
        # refine the leaves the inner circle cuts once more (hanging nodes on cut cells)
        pd0 = gb.PhysicalDomain(bg, gb.ImplicitRegion(annulus_levelset(o["ri"], 10.0), subdivision_depth=0))
        leaves = bg.grid.active_leaves()
        cls = pd0.classify(leaves)
        for leaf in leaves[cls == 2]:
            for grid in (od.grid, bg.grid):
                fc = grid.refine(int(leaf), 1)
                grid.refine(fc, 2)
                grid.refine(fc + 1, 2)
    pd = gb.PhysicalDomain(bg, gb.ImplicitRegion(lev, subdivision_depth=o["depth"]))
    sp = gb.HpSpace(pd, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(o["degree"])))
    u = gb.ScalarField(sp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    nit = gb.Nitsche(o["penalty"], data=exact if with_rhs else None)
    gb.add_surface_accumulator(prob, u, u, nit)
    if with_rhs:
        gb.add_surface_accumulator(prob, u, nit)
    surfaces = gb.sphere_surface_quadrature(sp, (0.0, 0.0), o["ro"], outward=True) + \
        gb.sphere_surface_quadrature(sp, (0.0, 0.0), o["ri"], outward=False)
    gb.add_surface_quadrature(prob, surfaces)
    osp = go.Space(od, o["degree"], basis="full", leaves=go.physical_active_leaves(od, lev))
    oplan = go.Plan(osp, mu=0.0, kappa=1.0, cell_rules=_oracle_rules(od, osp, lev, o["depth"]),
                    surface_items=_oracle_surfaces(od, surfaces, o["penalty"], exact if with_rhs else None))
    plan = gb.compile(prob, device=device)
    return oplan, prob, plan, exact


def shell(refine=None, degree=None, depth=None, device=True, source=True, oracle=True, tolerance=1e-8,
          cell_measure=None):
    """3-D shell 0.4 < |x - c| < 0.9 in [0, 2]^3 with Nitsche spheres, u = sin 2x cos 3y e^{z/2}."""
    o = dict(SHELL)
    o.update({k: v for k, v in dict(refine=refine, degree=degree, depth=depth).items() if v is not None})
    c = np.array(o["center"])
    lev = shell_levelset(c, o["ri"], o["ro"])
    p = o["degree"]
    penalty = 10.0 * p * p
    f = (lambda X: 12.75 * shell_exact(X)) if source else None
    od = go.Domain((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (1, 1, 1))
    bg = gb.Domain((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (1, 1, 1))
    go.uniform_refine(od.grid, o["refine"])
    gb.uniform_refine(bg, o["refine"])
    pd = gb.PhysicalDomain(bg, gb.ImplicitRegion(lev, subdivision_depth=o["depth"]), cell_measure=cell_measure)
    sp = gb.HpSpace(pd, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(sp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    if f is not None:
        gb.add_cell_accumulator(prob, u, gb.Load(f))
    nit = gb.Nitsche(penalty, data=shell_exact)
    gb.add_surface_accumulator(prob, u, u, nit)
    gb.add_surface_accumulator(prob, u, nit)
    surfaces = gb.sphere_surface_quadrature(sp, c, o["ro"], outward=True, tolerance=tolerance) + \
        gb.sphere_surface_quadrature(sp, c, o["ri"], outward=False, tolerance=tolerance)
    gb.add_surface_quadrature(prob, surfaces)
    oplan = None
    if oracle:
        assert cell_measure is None
        osp = go.Space(od, p, basis="full", leaves=go.physical_active_leaves(od, lev))
        oplan = go.Plan(osp, mu=0.0, kappa=1.0, source=_scalar(f), cell_rules=_oracle_rules(od, osp, lev, o["depth"]),
                        surface_items=_oracle_surfaces(od, surfaces, penalty, shell_exact))
    plan = gb.compile(prob, device=device)
    return oplan, prob, plan, shell_exact


def box_nitsche(dim=2, degree=3, refine=2, penalty=20.0, mu=0.0, device=True):
    """Poisson on the unit box with symmetric Nitsche data on every face (boundary-face items)."""
    roots = (1,) * dim
    od = go.Domain((0.0,) * dim, (1.0,) * dim, roots)
    bg = gb.Domain((0.0,) * dim, (1.0,) * dim, roots)
    go.uniform_refine(od.grid, refine)
    gb.uniform_refine(bg, refine)

    def exact(X):
        out = np.ones(X.shape[0])
        for a in range(dim):
            out = out * np.sin(math.pi * X[:, a] + 0.3)
        return out

    def f(X):
        return (dim * math.pi ** 2 + mu) * exact(X)

    sp = gb.HpSpace(bg, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(degree)))
    u = gb.ScalarField(sp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(mu, 1.0) if mu else gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(f))
    nit = gb.Nitsche(penalty, data=exact)
    osp = go.Space(od, degree, basis="full")
    items = []
    for a in range(1, dim + 1):
        for s in (gb.LOWER, gb.UPPER):
            gb.add_boundary_accumulator(prob, gb.BoundaryFace(a, s), u, u, nit)
            gb.add_boundary_accumulator(prob, gb.BoundaryFace(a, s), u, nit)
    for (leaf, axis, side) in osp.snapshot.boundary:
        li = osp.snapshot.leaf_to_index[leaf]
        q = osp.qshape[li]
        shape = tuple(1 if b == axis - 1 else q[b] for b in range(dim))
        pts, wts = go._tensor_points(shape)
        pts = np.array(pts)
        pts[:, axis - 1] = -1.0 if side == go.LOWER else 1.0
        scale = 1.0
        for b in range(dim):
            if b != axis - 1:
                scale *= od.cell_size(leaf, b)
        scale = math.ldexp(scale, -(dim - 1))
        nrm = np.zeros((len(wts), dim))
        nrm[:, axis - 1] = -1.0 if side == go.LOWER else 1.0
        # face rules carry tangential weights only (integration.jl:2846-2862); the 1-point
        # Gauss rule used for the normal axis above has weight 2
        items.append((leaf, pts, 0.5 * np.array(wts) * scale, nrm, penalty, _scalar(exact)))
    oplan = go.Plan(osp, mu=mu, kappa=1.0, source=_scalar(f), surface_items=items)
    plan = gb.compile(prob, device=device)
    return oplan, prob, plan, exact


def cell_override(device=True):
    """A plain 2-D mesh with explicit cell quadratures on two leaves (add_cell_quadrature!)."""
    od = go.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    bg = gb.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    sp = gb.HpSpace(bg, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(3)))
    u = gb.ScalarField(sp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(0.5, 1.0))
    rng = np.random.default_rng(5)
    rules = {}
    for leaf in (1, 4):
        pts = rng.uniform(-1, 1, size=(23, 2))
        w = rng.uniform(0.05, 0.3, size=23)
        gb.add_cell_quadrature(prob, leaf, pts, w)
        rules[leaf] = (pts, w)
    osp = go.Space(od, 3, basis="full")
    oplan = go.Plan(osp, mu=0.5, kappa=1.0, cell_rules=rules)
    plan = gb.compile(prob, device=device)
    return oplan, prob, plan

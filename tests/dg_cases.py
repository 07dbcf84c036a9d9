"""Symmetric interior-penalty DG cases built identically in the oracle and in the product:
diffusion (+ optional mass) on cells, the SIPG form of benchmark/sine_poisson_sipg.jl on every
interior interface and on every boundary face (homogeneous data imposed weakly)."""
import numpy as np

import grico_oracle as go
import grico_b200 as gb
from cases import refine_uniform


def _hanging(grid, D):
    # refine the first root cell once more along every axis: non-matching interfaces to its
    # neighbours
    leaves = [int(grid.active_leaves()[0])]
    for axis in range(1, D + 1):
        nxt = []
        for c in leaves:
            f = grid.refine(c, axis)
            nxt += [f, f + 1]
        leaves = nxt


def sipg_case(dim=2, degree=2, refine=1, hanging=False, hp=False, penalty=10.0, mu=0.0, continuity="dg",
              source=None, device=True):
    """(oracle plan, product problem, product plan)."""
    roots = (2,) * dim
    od = go.Domain((0.0,) * dim, (1.0,) * dim, roots)
    pd = gb.Domain((0.0,) * dim, (1.0,) * dim, roots)
    for g in (od.grid, pd.grid):
        refine_uniform(g, refine)
        if hanging:
            _hanging(g, dim)
    if hp:
        # degree by leaf: alternate degree and degree + 1 in leaf-id order
        ofn = lambda leaf: tuple([degree + (leaf % 2)] * dim)
        deg = gb.ByLeafDegrees(lambda leaf: degree + (leaf % 2))
        osp = go.Space(od, ofn, basis="full", continuity=continuity)
    else:
        deg = gb.UniformDegree(degree)
        osp = go.Space(od, degree, basis="full", continuity=continuity)
    psp = gb.HpSpace(pd, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=deg, continuity=continuity))
    u = gb.ScalarField(psp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(mu, 1.0) if mu else gb.Diffusion())
    if source is not None:
        gb.add_cell_accumulator(prob, u, gb.Load(source))
    op = gb.SIPG(penalty)
    gb.add_interface(prob, op)
    for a in range(1, dim + 1):
        for s in (gb.LOWER, gb.UPPER):
            gb.add_boundary(prob, gb.BoundaryFace(a, s), op)
    items = []
    snap = osp.snapshot
    for (leaf, axis, side) in snap.boundary:
        li = snap.leaf_to_index[leaf]
        q = osp.qshape[li]
        shape = tuple(1 if b == axis - 1 else q[b] for b in range(dim))
        pts, wts = go._tensor_points(shape)
        pts = np.array(pts)
        pts[:, axis - 1] = -1.0 if side == go.LOWER else 1.0
        scale = 1.0
        for b in range(dim):
            if b != axis - 1:
                scale *= od.cell_size(leaf, b)
        scale = float(np.ldexp(scale, -(dim - 1)))
        nrm = np.zeros((len(wts), dim))
        nrm[:, axis - 1] = -1.0 if side == go.LOWER else 1.0
        h = od.cell_size(leaf, axis - 1)
        eta = penalty * (osp.degrees[li][axis - 1] + 1) ** 2 / h
        items.append((leaf, pts, 0.5 * np.array(wts) * scale, nrm, penalty, None, eta))
    src_scalar = (lambda x: float(source(np.array([x]))[0])) if source else None
    oplan = go.Plan(osp, mu=mu, kappa=1.0, source=src_scalar, surface_items=items, interface_penalty=penalty)
    plan = gb.compile(prob, device=device)
    return oplan, prob, plan

"""The adaptive hp L-shape (Poisson on [-1,1]^3 minus [0,1] x [0,1] x [-1,1], homogeneous
Dirichlet on every boundary face including the re-entrant ones, dyadic refinement toward the
edge x = y = 0, degree min(p_max, 2 + max_level - level)) built identically in the oracle and in
the product, at levels small enough for the oracle."""
import numpy as np

import grico_oracle as go
import grico_b200 as gb
from grico_b200 import batched as bt


def oracle_lshape(max_level=4, start_level=2, p_max=8, mu=0.0, kappa=1.0, source=None):
    od = go.Domain((-1.0, -1.0, -1.0), (2.0, 2.0, 2.0), (2, 2, 2))
    grid = od.grid
    go.uniform_refine(grid, start_level - 1)

    def lo(c, a):
        return od.cell_lower(c, a)

    def hi(c, a):
        return od.cell_lower(c, a) + od.cell_size(c, a)

    def near_edge(c):
        return lo(c, 0) <= 0.0 <= hi(c, 0) and lo(c, 1) <= 0.0 <= hi(c, 1)

    def removed(c):
        return lo(c, 0) >= 0.0 and lo(c, 1) >= 0.0

    for _ in range(start_level, max_level):
        sel = [c for c in grid.active_leaves() if near_edge(c) and not removed(c)]
        for axis in (1, 2, 3):
            nxt = []
            for c in sel:
                f = grid.refine(c, axis)
                nxt += [f, f + 1]
            sel = nxt
    active = [c for c in grid.active_leaves() if not removed(c)]
    degree = lambda leaf: (min(p_max, 2 + max_level - (grid.level(leaf, 0) + 1)),) * 3
    osp = go.Space(od, degree, basis="full", leaves=active)
    src = (lambda x: float(source(np.array([x]))[0])) if source else None
    dirichlet = [(a, s, 0.0) for a in (1, 2, 3) for s in (1, 2)]
    return go.Plan(osp, mu=mu, kappa=kappa, source=src, dirichlet=dirichlet)


def product_lshape(max_level=4, start_level=2, p_max=8, mu=0.0, kappa=1.0, source=None):
    prob = bt.lshape_problem(max_level=max_level, start_level=start_level, p_max=p_max)
    if mu != 0.0 or kappa != 1.0:
        prob.cell_operators = []
        u = prob.field
        gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(mu, kappa))
    if source is not None:
        gb.add_cell_accumulator(prob, prob.field, gb.Load(source))
    return prob

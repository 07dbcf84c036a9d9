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


# the reference's noise pivots (|pivot| ~ 1e-15, amplified by hanging-node coefficients) leave
# its functions off the exact continuous space by ~1e-12 relative; comparisons across the two
# numberings are held to this bound
NOISE = 1e-10


def _box_modes(degs):
    n = [d + 1 for d in degs]
    return [(i, j, k) for k in range(n[2]) for j in range(n[1]) for i in range(n[0])]  # axis 1 fastest


def setup(max_level=4, mu=0.0, kappa=1.0, device=True):
    """Oracle plan, product plan and, per leaf, the product's term lists of every box mode (axis 1
    fastest).  The oracle's leaves may list fewer modes: where its noise pivots eliminated a
    variable, the modes carried only by that variable are gone from its space, while the product
    keeps them."""
    oplan = oracle_lshape(max_level=max_level, mu=mu, kappa=kappa)
    plan = gb.compile(product_lshape(max_level=max_level, mu=mu, kappa=kappa), device=device)
    psp, osp = plan.space, oplan.space
    assert list(osp.snapshot.leaves) == [int(v) for v in psp.leaves]
    terms = []
    for li in range(len(osp.snapshot.leaves)):
        lo_box = psp.box_offsets[li]
        nbox = len(_box_modes(oplan.cells[li]["degs"]))
        assert psp.box_offsets[li + 1] - lo_box == nbox
        terms.append([[(int(psp.term_index[t]) + 1, float(psp.term_coef[t]))
                       for t in range(psp.term_offsets[e], psp.term_offsets[e + 1])]
                      for e in range(lo_box, lo_box + nbox)])  # inactive modes: empty
    return oplan, plan, terms


def box_tables(c):
    """Values and physical gradients of every box mode of the oracle cell `c` at its tensor
    points, from the oracle's 1-D tables (axis 1 fastest in both indices)."""
    V, Gr = c["axis_v"], c["axis_g"]
    vals = np.kron(V[2], np.kron(V[1], V[0]))
    grads = [np.kron(V[2], np.kron(V[1], Gr[0])), np.kron(V[2], np.kron(Gr[1], V[0])),
             np.kron(Gr[2], np.kron(V[1], V[0]))]
    return vals, grads


def box_local_apply(oplan, c, xloc):
    """The oracle's cell operator (accumulators.jl:1022-1054, as Plan.local_apply) on the full
    box of modes."""
    vals, grads = box_tables(c)
    w = c["w"]
    u = vals.T @ xloc
    y = vals @ (w * oplan.mu * u)
    for a in range(3):
        y = y + grads[a] @ (w * oplan.kappa * (grads[a].T @ xloc))
    return y


def expand(plan, xr):
    """u_full = shift + P u_red on the host (assembly.jl:965-970), shift left out."""
    xf = np.zeros(plan.n_full)
    for d in range(plan.n_full):
        lo, hi = plan.red_offsets[d], plan.red_offsets[d + 1]
        xf[d] = plan.red_coef[lo:hi] @ xr[plan.red_index[lo:hi]]
    return xf


def project(plan, yf):
    out = np.zeros(plan.n_reduced)
    for d in range(plan.n_full):
        lo, hi = plan.red_offsets[d], plan.red_offsets[d + 1]
        np.add.at(out, plan.red_index[lo:hi], plan.red_coef[lo:hi] * yf[d])
    return out


def to_product(oplan, plan, terms, u_red):
    """Product reduced coefficients of the function whose oracle reduced coefficients are u_red:
    solve T_product x = the leaf-local mode coefficients (sparse normal equations), restrict to
    the solve dofs and check that the result reproduces the function."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    xo = np.concatenate([[0.0], oplan.expand(u_red)])
    rows, cols, vals, rhs = [], [], [], []
    r = 0
    for li, c in enumerate(oplan.cells):
        local = dict(zip(c["modes"], c["terms"]))
        for mode, t_pr in zip(_box_modes(c["degs"]), terms[li]):
            for (d, cc) in t_pr:
                rows.append(r)
                cols.append(d - 1)
                vals.append(cc)
            rhs.append(sum(cc * xo[d] for (d, cc) in local.get(mode, [])))  # absent mode: 0
            r += 1
    T = sp.csr_matrix((vals, (rows, cols)), shape=(r, plan.n_full))
    rhs = np.array(rhs)
    x = spl.spsolve((T.T @ T).tocsc(), T.T @ rhs)
    xr = x[plan.solve_dofs]
    assert np.max(np.abs(T @ expand(plan, xr) - rhs)) <= NOISE * max(1.0, np.max(np.abs(rhs)))
    return xr


def cell_sum(oplan, plan, terms, x):
    """Sum of the oracle's local cell operators gathered/scattered through the product's maps."""
    y = np.zeros(plan.n_full)
    for li, c in enumerate(oplan.cells):
        xloc = np.array([sum(cc * x[d - 1] for (d, cc) in t) for t in terms[li]])
        yloc = box_local_apply(oplan, c, xloc)
        for t, v in zip(terms[li], yloc):
            for (d, cc) in t:
                y[d - 1] += cc * v
    return y


def full_apply(oplan, plan, terms, x):
    """apply! on the product's layout: cell sum, then the constraint rows (fixed: y = x;
    relation: y_p = x_p - sum c_j x_j), assembly.jl:1893-1920."""
    y = cell_sum(oplan, plan, terms, x)
    y[plan.fixed_dofs] = x[plan.fixed_dofs]
    for (p, idx, co, _) in plan.relations:
        y[p] = x[p] - co @ x[idx]
    return y

"""hp geometric multigrid: hierarchy construction on the host, V-cycle on the device.

Mirrors `GeometricMultigridPreconditioner` (multigrid.jl:66-96) and the hierarchy compile
(`_compile_geometric_multigrid`, multigrid.jl:309-345): p-coarsening first (`:bisect` by
default, multigrid.jl:470-499), then h-coarsening one split frontier per level
(multigrid.jl:514-586); every level is rediscretised with the same forms and constraints;
transfers come from libgrico_b200 (grico_transfer_build); the coarsest level is factorised
by dense Cholesky (at most `coarse_direct_dof_limit` dofs, multigrid.jl:382-398).

Smoothers: damped Jacobi (the reference's SPD smoother, multigrid.jl:943-956), the fixed-step
right-Jacobi GMRES smoother with `smoother_restart` Krylov columns for non-SPD problems
(multigrid.jl:963-1056; `smoother="auto"` picks Jacobi for SPD problems and GMRES otherwise,
multigrid.jl:347-350) and, with `smoother="chebyshev"`, Chebyshev-Jacobi of degree
`chebyshev_degree` on [lambda_max/`chebyshev_range`, 1.2 lambda_max] of D^-1 A (no reference
counterpart).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class GeometricMultigridPreconditioner:
    def __init__(self, min_degree=1, max_levels=16, p_sequence="bisect", pre_smoothing_steps=2,
                 post_smoothing_steps=2, smoother_damping=0.8, smoother="auto", smoother_restart=8,
                 coarse_direct_dof_limit=512, chebyshev_degree=2, chebyshev_range=15.0, precision="fp64"):
        if p_sequence not in ("bisect", "decrease_by_one", "go_to_one"):
            raise ValueError("p_sequence must be :bisect, :decrease_by_one, or :go_to_one")
        if smoother not in ("auto", "jacobi", "gmres", "chebyshev"):
            raise ValueError("smoother must be :auto, :jacobi, :gmres or :chebyshev")
        if max_levels < 1 or pre_smoothing_steps < 0 or post_smoothing_steps < 0 or smoother_damping <= 0:
            raise ValueError("invalid multigrid options")
        if int(smoother_restart) < 1:
            raise ValueError("smoother_restart must be positive")
        self.min_degree = int(min_degree)
        self.max_levels = int(max_levels)
        self.p_sequence = p_sequence
        self.pre_smoothing_steps = int(pre_smoothing_steps)
        self.post_smoothing_steps = int(post_smoothing_steps)
        self.smoother_damping = float(smoother_damping)
        self.smoother = smoother
        self.smoother_restart = int(smoother_restart)
        self.coarse_direct_dof_limit = int(coarse_direct_dof_limit)
        self.chebyshev_degree = int(chebyshev_degree)
        self.chebyshev_range = float(chebyshev_range)
        self.precision = precision


def resolved_smoother(opts, problem=None):
    """multigrid.jl:347-358: `auto` is Jacobi for SPD problems and GMRES otherwise; GMRES needs
    `smoother_restart >= max(pre, post)`."""
    from .problem import SPD

    sm = opts.smoother
    if sm == "auto":
        spd = problem is None or isinstance(getattr(problem, "operator_class", SPD()), SPD)
        sm = "jacobi" if spd else "gmres"
    if sm == "gmres" and max(opts.pre_smoothing_steps, opts.post_smoothing_steps) > opts.smoother_restart:
        raise ValueError("GMRES multigrid smoother requires smoother_restart to be at least "
                         "max(pre_smoothing_steps, post_smoothing_steps)")
    return sm


def _coarsened_degree(degree, lower, sequence):
    """multigrid.jl:470-499"""
    if degree <= lower:
        return degree
    if sequence == "bisect":
        return max(degree // 2, lower)
    if sequence == "decrease_by_one":
        return max(degree - 1, lower)
    return lower


def _coarsened_degrees(degrees, cg, min_degree, sequence):
    """_coarsened_degree on every entry (array form)."""
    degrees = np.asarray(degrees)
    lower = np.minimum(degrees, max(min_degree, 1 if cg else 0))
    if sequence == "bisect":
        c = np.maximum(degrees // 2, lower)
    elif sequence == "decrease_by_one":
        c = np.maximum(degrees - 1, lower)
    else:
        c = lower
    return np.where(degrees <= lower, degrees, c).astype(degrees.dtype)


def h_coarsening(grid, leaves, degrees):
    """Merge every expanded cell whose two children are both active leaves (multigrid.jl:514-586).
    Returns (leaves, degrees) of the coarser level or None.  The merged parent takes the place of
    its first child in the leaf order and the smaller degree of its children per axis."""
    leaves = np.asarray(leaves, dtype=np.int64)
    degrees = np.asarray(degrees)
    parent = np.asarray(grid.parent)[leaves]
    first = np.asarray(grid.first_child)[np.maximum(parent, 0)]
    is_first = (parent > 0) & (leaves == first)
    is_second = (parent > 0) & (leaves == first + 1)
    # a parent merges when both of its children are active leaves
    order = np.argsort(leaves, kind="stable")
    sorted_leaves = leaves[order]

    def position(ids):
        k = np.searchsorted(sorted_leaves, ids)
        k = np.minimum(k, len(sorted_leaves) - 1)
        found = sorted_leaves[k] == ids
        return np.where(found, order[k], -1)

    sib_of_first = position(np.where(is_first, leaves + 1, -1))
    merge_first = is_first & (sib_of_first >= 0)
    if not merge_first.any():
        return None
    sib_of_second = position(np.where(is_second, leaves - 1, -1))
    merge_second = is_second & (sib_of_second >= 0)
    pos_first = np.where(merge_first, np.arange(len(leaves)), np.where(merge_second, sib_of_second, -1))
    merged = pos_first >= 0
    # emit each merged parent once, at the position of whichever child comes first in the order
    emit_pos = np.where(merged, np.minimum(np.arange(len(leaves)), np.where(merge_first, sib_of_first, sib_of_second)),
                        np.arange(len(leaves)))
    keep = (~merged) | (emit_pos == np.arange(len(leaves)))
    new_leaves = np.where(merged, parent, leaves)[keep]
    partner = np.where(merge_first, sib_of_first, np.where(merge_second, sib_of_second, np.arange(len(leaves))))
    new_deg = np.where(merged[:, None], np.minimum(degrees, degrees[partner]), degrees)[keep]
    return new_leaves.astype(np.int64), new_deg.astype(np.int32)


def hp_multigrid_spaces(fine_space, opts):
    """Coarse-to-fine list of (active leaves, per-leaf degrees) (multigrid.jl:443-469)."""
    from .space import HpSpace, SpaceOptions, StoredDegrees

    cg = fine_space.options.continuity == "cg"
    levels = [(fine_space.leaves.copy(), fine_space.degrees.copy())]
    leaves, degrees = levels[0]
    while len(levels) < opts.max_levels:
        nd = _coarsened_degrees(degrees, cg, opts.min_degree, opts.p_sequence)
        if np.array_equal(nd, degrees):
            break
        degrees = nd
        levels.append((leaves, degrees))
    grid = fine_space.domain.grid
    while len(levels) < opts.max_levels:
        nxt = h_coarsening(grid, leaves, degrees)
        if nxt is None:
            break
        leaves, degrees = nxt
        levels.append((leaves, degrees))
    levels.reverse()
    spaces = []
    for i, (lv, dg) in enumerate(levels):
        if i == len(levels) - 1:
            spaces.append(fine_space)
            continue
        o = fine_space.options
        spaces.append(HpSpace(fine_space.domain, SpaceOptions(basis=o.basis, degree=StoredDegrees(lv, dg),
                                                              quadrature=o.quadrature, continuity=o.continuity),
                              active=lv))
    return spaces


def _level_problem(problem, space):
    from .problem import AffineProblem, Dirichlet, ScalarField

    u = ScalarField(space, name=problem.field.name)
    p = AffineProblem(u, operator_class=problem.operator_class)
    p.cell_operators = list(problem.cell_operators)
    p.rhs_operators = list(problem.rhs_operators)
    p.dirichlet = [Dirichlet(u, c.boundary, c.value) for c in problem.dirichlet]
    # face forms carry no field reference, so every level reuses them (multigrid.jl:309-345
    # rediscretises every operator of the problem on each level)
    p.boundary_operators = list(problem.boundary_operators)
    p.boundary_rhs_operators = list(problem.boundary_rhs_operators)
    p.interface_operators = list(getattr(problem, "interface_operators", []))
    return p


def transfer(coarse_plan, fine_plan):
    """Reduced prolongation CSR (fine rows) between consecutive levels."""
    h = C.c_void_p()
    lib = L.lib()
    fine_index = np.ascontiguousarray(fine_plan.reduced_index, dtype=np.int64)
    L.check(lib.grico_transfer_build(coarse_plan.space.handle, fine_plan.space.handle,
                                     L.ptr(coarse_plan.red_offsets, C.c_int64), L.ptr(coarse_plan.red_index, C.c_int64),
                                     L.ptr(coarse_plan.red_coef, C.c_double), coarse_plan.n_reduced,
                                     L.ptr(fine_index, C.c_int64), fine_plan.n_reduced, C.byref(h)), "transfer")
    try:
        nnz = C.c_int64()
        L.check(lib.grico_transfer_export(h, C.byref(nnz), None, None, None))
        off = np.zeros(fine_plan.n_reduced + 1, dtype=np.int64)
        col = np.zeros(nnz.value, dtype=np.int64)
        val = np.zeros(nnz.value, dtype=np.float64)
        L.check(lib.grico_transfer_export(h, None, L.ptr(off, C.c_int64), L.ptr(col, C.c_int64), L.ptr(val, C.c_double)))
    finally:
        lib.grico_transfer_destroy(h)
    return off, col, val


class Multigrid:
    """Device V-cycle over compiled level plans (coarse -> fine)."""

    def __init__(self, plans, transfers, opts):
        self.plans = plans
        self.transfers = transfers
        self.opts = opts
        self.smoother = resolved_smoother(opts, getattr(plans[-1], "problem", None))
        if plans[0].n_reduced > opts.coarse_direct_dof_limit:
            raise L.GricoError(L.GRICO_ERR_INVALID,
                               f"coarse level has {plans[0].n_reduced} dofs > coarse_direct_dof_limit; "
                               "add h-levels or raise the limit")
        handles = (C.c_void_p * len(plans))(*[p.handle.value for p in plans])
        descs = (L.GricoTransferDesc * max(1, len(transfers)))()
        for i, (off, col, val) in enumerate(transfers):
            descs[i].n_fine = plans[i + 1].n_reduced
            descs[i].n_coarse = plans[i].n_reduced
            descs[i].row_offsets = L.ptr(off, C.c_int64)
            descs[i].col_index = L.ptr(col, C.c_int64)
            descs[i].values = L.ptr(val, C.c_double)
        mo = L.GricoMGOptions()
        mo.smoother = {"jacobi": L.GRICO_SMOOTHER_JACOBI, "chebyshev": L.GRICO_SMOOTHER_CHEBYSHEV,
                       "gmres": L.GRICO_SMOOTHER_GMRES}[self.smoother]
        mo.smoother_restart = opts.smoother_restart
        mo.pre_steps = opts.pre_smoothing_steps
        mo.post_steps = opts.post_smoothing_steps
        mo.jacobi_omega = opts.smoother_damping
        mo.chebyshev_degree = opts.chebyshev_degree
        mo.chebyshev_lower = 1.0 / opts.chebyshev_range
        mo.precision = L.GRICO_PREC_FP64 if opts.precision == "fp64" else L.GRICO_PREC_FP32
        h = C.c_void_p()
        L.check(L.lib().grico_mg_create(handles, len(plans), descs, None, C.byref(mo), C.byref(h)), "multigrid")
        self.handle = h

    def level_sizes(self):
        return [p.n_reduced for p in self.plans]

    def lambda_max(self, level):
        """Power-iteration estimate of lambda_max(D^-1 A) on `level` (0 = coarsest) used by the
        Chebyshev smoother; 0 when the smoother is not Chebyshev."""
        return float(L.lib().grico_mg_lambda_max(self.handle, int(level)))

    def vcycle(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        L.check(L.lib().grico_mg_vcycle(self.handle, L.ptr(r, C.c_double), L.ptr(z, C.c_double),
                                        L.GRICO_FLAG_HOST_POINTERS), "vcycle")
        return z

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.lib().grico_mg_destroy(h)
            except Exception:
                pass
            self.handle = None


def build_hierarchy(plan, opts, device=True):
    """Level plans (coarse -> fine) and their transfers for a compiled fine plan."""
    from .problem import compile

    spaces = hp_multigrid_spaces(plan.space, opts)
    if len(spaces) < 2:
        raise L.GricoError(L.GRICO_ERR_INVALID,
                           "GeometricMultigridPreconditioner requires at least one admissible h or p coarsening level")
    plans = [compile(_level_problem(plan.problem, s), device=device) for s in spaces[:-1]] + [plan]
    # coarse levels whose every dof is constrained carry nothing: the coarsest level with free
    # dofs becomes the direct-solve level
    while len(plans) > 2 and plans[0].n_reduced == 0:
        plans.pop(0)
    transfers = [transfer(plans[i], plans[i + 1]) for i in range(len(plans) - 1)]
    return plans, transfers


def build_multigrid(plan, opts):
    plans, transfers = build_hierarchy(plan, opts)
    return Multigrid(plans, transfers, opts)

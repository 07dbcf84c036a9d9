"""Many right-hand sides per solve and the adaptive hp workload they are measured on.

`solve_many` runs grico_cg_solve_multi: nrhs CG iterations in lockstep, one operator apply
for all systems per iteration (all cell batches and right-hand sides in the launches of one
CUDA graph), optionally FP64 iterative refinement around FP32 inner CG.  `autotune` picks the
cells-per-block variant of every tensor-cell batch (grico_plan_autotune).  No reference
counterpart: the reference solves one right-hand side at a time.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def autotune(plan, nrhs=1, precision="fp64", reps=5):
    """Per cell batch: 0 = half, 1 = default, 2 = double cells per block (one block per cell
    group); 3, 4, 5 = the same sizes in the persistent pipelined apply kernel (even-odd
    contractions), 6, 7, 8 = with direct contractions; 9 = one warp per 32 / q cells with one
    thread per cell plane; 10 = FP32 only, uniform batches of degree <= 4: one element matrix on
    the tensor cores (tcgen05, BF16 hi/lo pieces, FP32 accumulation; measured slower than 3..9,
    never the default)."""
    chosen = np.zeros(max(len(plan.batches), 1), dtype=np.int32)
    prec = L.GRICO_PREC_FP64 if precision == "fp64" else L.GRICO_PREC_FP32
    L.check(L.lib().grico_plan_autotune(plan.handle, int(nrhs), prec, int(reps), L.ptr(chosen, C.c_int32)), "autotune")
    return chosen[:len(plan.batches)]


def set_tiles(plan, tiles, precision="fp64"):
    """Replay a kernel-variant choice (as returned by `autotune`) without timing."""
    t = np.ascontiguousarray(tiles, dtype=np.int32)
    prec = L.GRICO_PREC_FP64 if precision == "fp64" else L.GRICO_PREC_FP32
    L.check(L.lib().grico_plan_set_tiles(plan.handle, prec, L.ptr(t, C.c_int32), int(t.size)), "set_tiles")


def solve_many(plan, B, relative_tolerance=1e-10, absolute_tolerance=0.0, maxiter=None, jacobi=True, mixed=False,
               graph=True):
    """X [nrhs, n_reduced] for the stacked reduced right-hand sides B and the per-system reports."""
    B = np.ascontiguousarray(np.atleast_2d(B), dtype=np.float64)
    nrhs, n = B.shape
    if n != plan.n_reduced:
        raise ValueError("right-hand sides must have the reduced length")
    X = np.zeros_like(B)
    maxiter = max(1000, 2 * n) if maxiter is None else int(maxiter)
    opts = L.GricoSolveOptions(float(relative_tolerance), float(absolute_tolerance), int(min(maxiter, 2 ** 31 - 1)),
                               L.GRICO_PRECOND_JACOBI if jacobi else L.GRICO_PRECOND_IDENTITY, 30, 0)
    reps = (L.GricoSolveReport * nrhs)()
    flags = L.GRICO_FLAG_HOST_POINTERS | (L.GRICO_FLAG_MIXED if mixed else 0) | (0 if graph else L.GRICO_FLAG_NO_GRAPH)
    L.check(L.lib().grico_cg_solve_multi(plan.handle, L.ptr(B, C.c_double), L.ptr(X, C.c_double), nrhs,
                                         C.byref(opts), reps, flags), "solve_many")
    return X, list(reps)


def lshape_problem(max_level=7, start_level=2, p_max=8):
    """Poisson on the L-shaped domain [-1,1]^3 minus [0,1] x [0,1] x [-1,1], homogeneous Dirichlet,
    dyadic isotropic refinement toward the re-entrant edge x = y = 0 from level `start_level` to
    `max_level` (a level-l cell has size 2^(1-l)), degree min(p_max, 2 + max_level - level) per
    cell.  Returns the problem (without a load)."""
    from . import mesh, problem as P, space as S

    dom = mesh.Domain((-1.0, -1.0, -1.0), (2.0, 2.0, 2.0), (2, 2, 2))
    grid = dom.grid
    mesh.uniform_refine(dom, start_level - 1)

    def near_edge(leaves):
        lo = dom.cell_lower(leaves)
        hi = lo + dom.cell_size(leaves)
        return (lo[:, 0] <= 0.0) & (hi[:, 0] >= 0.0) & (lo[:, 1] <= 0.0) & (hi[:, 1] >= 0.0)

    def removed(leaves):
        lo = dom.cell_lower(leaves)
        return (lo[:, 0] >= 0.0) & (lo[:, 1] >= 0.0)

    for _ in range(start_level, max_level):
        leaves = grid.active_leaves()
        sel = leaves[near_edge(leaves) & ~removed(leaves)]
        for axis in (1, 2, 3):
            nxt = []
            for c in sel:
                fc = grid.refine(int(c), axis)
                nxt += [fc, fc + 1]
            sel = np.array(nxt, dtype=np.int64)
    leaves = grid.active_leaves()
    active = leaves[~removed(leaves)]
    level_of = {int(l): int(grid.levels[l][0]) + 1 for l in active}
    degree = S.ByLeafDegrees(lambda leaf: min(p_max, 2 + max_level - level_of[leaf]))
    sp = S.HpSpace(dom, S.SpaceOptions(basis=S.FullTensorBasis(), degree=degree), active=active)
    u = P.ScalarField(sp)
    prob = P.AffineProblem(u)
    P.add_cell_accumulator(prob, u, u, P.Diffusion())
    for a in (1, 2, 3):
        for side in (mesh.LOWER, mesh.UPPER):
            P.add_constraint(prob, P.Dirichlet(u, P.BoundaryFace(a, side), 0.0))
    return prob


def gaussian_bumps(nrhs, seed=0):
    """Seeded loads f_k(x) = A_k exp(-|x - c_k|^2 / (2 w_k^2)): centres uniform in the L-shape,
    widths uniform in [0.1, 0.3], amplitudes N(0, 1)."""
    rng = np.random.default_rng(seed)
    loads = []
    while len(loads) < nrhs:
        c = rng.uniform(-1.0, 1.0, 3)
        if c[0] > 0 and c[1] > 0:
            continue
        w = rng.uniform(0.1, 0.3)
        a = rng.standard_normal()
        loads.append((lambda X, c=c, w=w, a=a: a * np.exp(-np.sum((X - c) ** 2, axis=1) / (2 * w * w))))
    return loads


def reduced_rhs_many(plan, loads):
    """Stacked reduced right-hand sides of the plan's problem for each load."""
    from .problem import Load, reduced_rhs

    prob = plan.problem
    saved = list(prob.rhs_operators)
    out = []
    try:
        for f in loads:
            prob.rhs_operators = [Load(f)]
            out.append(reduced_rhs(plan))
    finally:
        prob.rhs_operators = saved
    return np.stack(out)

"""Seeded problem cases built identically in the oracle and in the product."""
import math

import numpy as np

import grico_oracle as go
import grico_b200 as gb


def refine_uniform(grid, depth):
    for _ in range(depth):
        for leaf in list(grid.active_leaves()):
            leaves = [int(leaf)]
            for axis in range(1, grid.D + 1):
                nxt = []
                for c in leaves:
                    fc = grid.refine(c, axis)
                    nxt += [fc, fc + 1]
                leaves = nxt


def hanging_2d(grid):
    grid.refine(2, 2)


def hanging_3d(grid):
    fc = grid.refine(2, 2)
    grid.refine(fc, 3)
    grid.refine(fc + 1, 3)


CASES = {
    # name: (origin, extent, roots, refine, degree, basis, quadrature extra, dirichlet faces)
    "2d_p4": ((0.0, 0.0), (1.0, 1.0), (4, 3), None, 4, "full", 1, [(1, 1), (1, 2), (2, 1), (2, 2)]),
    "2d_p2_hanging": ((0.0, 0.0), (2.0, 1.0), (2, 1), hanging_2d, 2, "full", 1, [(1, 1)]),
    "2d_p3_over": ((0.0, 0.0), (1.0, 2.0), (3, 2), None, 3, "full", 2, [(2, 1)]),
    "3d_p4": ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (2, 2, 2), lambda g: refine_uniform(g, 1), 4, "full", 1,
              [(a, s) for a in (1, 2, 3) for s in (1, 2)]),
    "3d_p2_hanging": ((0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (2, 1, 1), hanging_3d, 2, "full", 1, [(1, 1), (3, 2)]),
    "3d_p3_trunk": ((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (2, 2, 1), None, 3, "trunk", 1, [(1, 1)]),
    "3d_p1": ((0.0, 0.0, 0.0), (1.0, 2.0, 1.0), (3, 2, 2), None, 1, "full", 1, [(2, 2)]),
    "3d_p5_aniso_cells": ((0.0, 0.0, 0.0), (1.0, 0.5, 2.0), (2, 1, 1), None, 5, "full", 1, []),
    "1d_p3": ((0.0,), (1.0,), (4,), None, 3, "full", 1, [(1, 1), (1, 2)]),
}


def build(name, mu=0.0, kappa=1.0, kappa_fn=None, source=None, dirichlet_value=0.0):
    origin, extent, roots, refine, p, basis, qx, faces = CASES[name]
    od = go.Domain(origin, extent, roots)
    pdm = gb.Domain(origin, extent, roots)
    if refine:
        refine(od.grid)
        refine(pdm.grid)
    osp = go.Space(od, p, basis=basis, quadrature_extra=qx)
    kfn_scalar = (lambda x: float(kappa_fn(np.array([x]))[0])) if kappa_fn else None
    src_scalar = (lambda x: float(source(np.array([x]))[0])) if source else None
    oplan = go.Plan(osp, mu=mu, kappa=kappa, kappa_fn=kfn_scalar, source=src_scalar,
                    dirichlet=[(a, s, dirichlet_value) for a, s in faces])
    psp = gb.HpSpace(pdm, gb.SpaceOptions(basis=gb.TrunkBasis() if basis == "trunk" else gb.FullTensorBasis(),
                                           degree=gb.UniformDegree(p), quadrature=gb.DegreePlusQuadrature(qx)))
    u = gb.ScalarField(psp)
    prob = gb.AffineProblem(u)
    if kappa_fn is not None:
        form = gb.VariableDiffusion(kappa_fn, kappa=kappa, mass=mu)
    elif mu == 0.0:
        form = gb.Diffusion(kappa)
    else:
        form = gb.MassDiffusion(mu, kappa)
    gb.add_cell_accumulator(prob, u, u, form)
    if source is not None:
        gb.add_cell_accumulator(prob, u, gb.Load(source))
    for a, s in faces:
        gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, s), dirichlet_value))
    return oplan, prob


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def sample_vector(n, seed=20261203):
    """SplitMix64-seeded values in [-1, 1)."""
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, n)

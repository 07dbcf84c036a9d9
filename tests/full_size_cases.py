"""The benchmark workloads at full size, built through the product's public API, and the
oracle-side data that checks them (uniform numbering, the reference's tensor schedule in C)."""
import math

import numpy as np

import grico_b200 as gb


def poisson3d_64(p=4, roots=(4, 4, 4), depth=4):
    """-Laplace u = f on [0,1]^3, 64^3 cells (4^3 roots refined 4 times, benchmark/hpmg_scaling.jl
    recipe), degree p, Gauss p+1 points per axis, homogeneous Dirichlet on all six faces."""
    d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), roots)
    gb.uniform_refine(d, depth)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(lambda x: 3 * math.pi ** 2 * np.prod(np.sin(np.pi * x), axis=1)))
    for a in (1, 2, 3):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return prob


def poisson2d_32(p=4):
    """examples/poisson_matrix_free_gmg/driver.jl:36-46 at 32 x 32 cells, degree 4: -Laplace u =
    2 pi^2 sin(pi x) sin(pi y), homogeneous Dirichlet on the four faces."""
    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (32, 32))
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(lambda x: 2 * math.pi ** 2 * np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1])))
    for a in (1, 2):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return prob


def uniform_oracle(counts, p):
    """Oracle numbering of a uniform grid (oracle/uniform_maps.py, pinned to the literal
    restatement) with the homogeneous-Dirichlet fixed set on every box face: a mode is on the
    lower face of axis a when its axis-a digit is 0 (the vertex function (1 - x)/2) and the leaf
    touches x_a = 0, on the upper face when the digit is 1 and the leaf touches x_a = 1."""
    import uniform_maps as um

    coords, m, ndofs = um.uniform_space(counts, p)
    D = len(counts)
    n = p + 1
    box = np.arange(n ** D)
    digits = np.stack([(box // n ** a) % n for a in range(D)], axis=1)
    on = np.zeros(m.shape, dtype=bool)
    for a in range(D):
        on |= (coords[:, a] == 0)[:, None] & (digits[:, a] == 0)[None, :]
        on |= (coords[:, a] == counts[a] - 1)[:, None] & (digits[:, a] == 1)[None, :]
    fixed = np.unique(m[on])
    return coords, m, ndofs, fixed


def tensor_tables(p):
    import grico_oracle as go

    pts, W = go.gauss_legendre_rule(p + 1)
    B = np.zeros((p + 1, p + 1))
    G = np.zeros((p + 1, p + 1))
    for j, x in enumerate(pts):
        v, dv = go.integrated_legendre_values_and_derivatives(x, p)
        B[:, j] = v
        G[:, j] = dv
    return B, G, np.array(W)


def oracle_cell_sum(counts, p, coords, m, x, h):
    """Sum over cells of the reference's tensor schedule (oracle/oracle_apply.c) on all threads."""
    import oracle_lib as ol
    import uniform_maps as um

    B, G, W = tensor_tables(p)
    order, off = um.parity_colours(coords)
    y = np.zeros(len(x))
    hh = np.full((len(coords), len(counts)), h)
    ol.tensor_apply(len(counts), p + 1, p + 1, m.astype(np.int32), hh, B, G, W, 0.0, 1.0, None, order, off,
                    np.ascontiguousarray(x, dtype=np.float64), y, threads=ol.max_threads())
    return y


def diagnostic_sample_vector(n):
    """_diagnostic_sample_vector (diagnostics.jl:107-121): sin(0.013 i) + 0.25 cos(0.037 i)."""
    i = np.arange(1, n + 1, dtype=np.float64)
    return np.sin(0.013 * i) + 0.25 * np.cos(0.037 * i)

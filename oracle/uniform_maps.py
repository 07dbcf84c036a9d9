"""Vectorized oracle data for uniform Cartesian grids — TEST INFRASTRUCTURE ONLY.

For a conforming grid whose leaves all share one level per axis and one FullTensor degree,
the reference's continuity compile (continuity.jl phases 1-6) reduces to: every boundary
mode's provisional variable is merged with the same mode of every leaf sharing its vertex /
edge / face (union-find keeps the smallest variable), free roots are numbered in variable
order, then interior modes leaf by leaf in Morton order (continuity.jl:223-252, 934-945,
264-350).  This module computes that numbering with array operations so the CPU baseline can
run at full problem size; tests/test_oracle_kat.py checks it against the literal restatement
in grico_oracle.py.
"""
from __future__ import annotations

import numpy as np


def morton_order(counts):
    """Leaves (lattice coords, axis 1 fastest ids) sorted by Morton code of the lower corner,
    axis D most significant within a bit (topology.jl:451-463)."""
    D = len(counts)
    grids = np.meshgrid(*[np.arange(c, dtype=np.int64) for c in counts], indexing="ij")
    coords = np.stack([g.reshape(-1, order="F") for g in grids], axis=1)  # axis 1 fastest ids
    bits = max(int(c - 1).bit_length() for c in counts)
    code = np.zeros(len(coords), dtype=np.uint64)
    for bit in range(bits - 1, -1, -1):
        for a in range(D - 1, -1, -1):
            code = (code << np.uint64(1)) | ((coords[:, a] >> bit) & 1).astype(np.uint64)
    order = np.argsort(code, kind="stable")
    return coords[order]


def uniform_space(counts, p):
    """Returns (coords [L, D] in Morton order, map [L, (p+1)^D] 0-based dofs, ndofs)."""
    D = len(counts)
    coords = morton_order(counts)
    L = len(coords)
    n = p + 1
    nb = n ** D
    box = np.arange(nb)
    digits = np.stack([(box // n ** a) % n for a in range(D)], axis=1)  # [nb, D]
    boundary = np.any(digits <= 1, axis=1)
    bmodes = np.nonzero(boundary)[0]
    imodes = np.nonzero(~boundary)[0]
    # key per (leaf, boundary mode): per axis (lattice point 2*(i+m) | span 2*i+1, interior index)
    dg = digits[bmodes]  # [nbnd, D]
    key = np.zeros((L, len(bmodes)), dtype=np.int64)
    mult = 1
    for a in range(D):
        ca = coords[:, a][:, None]
        fixed = dg[:, a][None, :] <= 1
        code = np.where(fixed, 2 * (ca + dg[:, a][None, :]), 2 * ca + 1)
        mode = np.where(fixed, 0, dg[:, a][None, :])
        width = 2 * int(counts[a]) + 2
        key = key + code * mult
        mult *= width
        key = key + mode * mult
        mult *= n
    flat = key.reshape(-1)  # variable order = leaf-major, boundary mode order
    _, first, inv = np.unique(flat, return_index=True, return_inverse=True)
    rank = np.empty(len(first), dtype=np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    bdof = rank[inv.reshape(-1)].reshape(L, len(bmodes))
    nfree = len(first)
    m = np.empty((L, nb), dtype=np.int64)
    m[:, bmodes] = bdof
    m[:, imodes] = nfree + np.arange(L * len(imodes)).reshape(L, len(imodes))
    return coords, m, nfree + L * len(imodes)


def parity_colours(coords):
    """Cells with equal coordinate parities share no dof on a uniform grid."""
    D = coords.shape[1]
    colour = np.zeros(len(coords), dtype=np.int64)
    for a in range(D):
        colour += (coords[:, a] & 1) << a
    order = np.argsort(colour, kind="stable")
    offsets = np.concatenate([[0], np.cumsum(np.bincount(colour, minlength=2 ** D))])
    return order, offsets

"""Cartesian refinement tree and affine box domain (host side of the mirror).

Mirrors `CartesianGrid`, `refine!` and `Domain` of Grico.jl (topology.jl:96-163,
refinement.jl:47-76, geometry.jl:134-141, 676-711).  Cell ids are 1-based and children are
appended in blocks of two exactly as the reference does, so cell ids printed here match the
ones the reference's tests use.
"""
from __future__ import annotations

import numpy as np

LOWER, UPPER = 1, 2
NONE = 0


class CartesianGrid:
    """Dyadic midpoint-bisection tree.  Storage arrays carry a dummy entry at index 0."""

    def __init__(self, root_counts, periodic=False):
        if periodic:
            raise ValueError("periodic axes are not supported by the B200 runtime")
        self.D = len(root_counts)
        if not 1 <= self.D <= 3:
            raise ValueError("dimension must be 1, 2 or 3")
        self.root_counts = tuple(int(c) for c in root_counts)
        if any(c < 1 for c in self.root_counts):
            raise ValueError("root_counts must be positive")
        total = int(np.prod(self.root_counts))
        lin = np.arange(total, dtype=np.int64)
        coords = np.zeros((total + 1, self.D), dtype=np.int64)
        stride = 1
        for a in range(self.D):
            coords[1:, a] = (lin // stride) % self.root_counts[a]
            stride *= self.root_counts[a]
        self.levels = np.zeros((total + 1, self.D), dtype=np.int32)
        self.coords = coords
        self.parent = np.zeros(total + 1, dtype=np.int64)
        self.first_child = np.zeros(total + 1, dtype=np.int64)
        self.split_axis = np.zeros(total + 1, dtype=np.int32)
        self.active = np.ones(total + 1, dtype=bool)
        self.active[0] = False
        self.revision = 0

    def stored_cell_count(self):
        return len(self.parent) - 1

    def active_leaves(self):
        return np.nonzero(self.active)[0]

    def _append(self, cells, axis_index, levels, coords):
        self.levels = np.concatenate([self.levels, levels])
        self.coords = np.concatenate([self.coords, coords])
        n = len(levels)
        self.parent = np.concatenate([self.parent, cells])
        self.first_child = np.concatenate([self.first_child, np.zeros(n, dtype=np.int64)])
        self.split_axis = np.concatenate([self.split_axis, np.zeros(n, dtype=np.int32)])
        self.active = np.concatenate([self.active, np.ones(n, dtype=bool)])

    def refine_many(self, cells, axis):
        """Split every cell in `cells` (active leaves) at its midpoint along `axis` (1-based);
        equivalent to calling refine! on each cell in order.  Returns the first-child ids."""
        cells = np.asarray(cells, dtype=np.int64)
        if cells.size == 0:
            return cells
        if not (1 <= axis <= self.D):
            raise ValueError("axis out of range")
        if not np.all(self.active[cells]):
            raise ValueError("only active leaves can be refined")
        a = axis - 1
        first = self.stored_cell_count() + 1 + 2 * np.arange(cells.size, dtype=np.int64)
        lev = np.repeat(self.levels[cells], 2, axis=0)
        crd = np.repeat(self.coords[cells], 2, axis=0)
        lev[:, a] += 1
        crd[:, a] = 2 * crd[:, a] + np.tile(np.array([0, 1], dtype=np.int64), cells.size)
        self._append(np.repeat(cells, 2), a, lev, crd)
        self.first_child[cells] = first
        self.split_axis[cells] = axis
        self.active[cells] = False
        self.revision += 1
        return first

    def refine(self, cell, axis):
        """refine!(grid, cell, axis) — returns the id of the first child (refinement.jl:47-53)."""
        return int(self.refine_many([int(cell)], axis)[0])


def refine(grid, cell, axis):
    return grid.refine(cell, axis)


def uniform_refine(domain, depth):
    """Refine every active leaf on every axis, axis by axis, `depth` times
    (benchmark/hpmg_scaling.jl:122-164).  Child ids follow the reference's per-leaf order."""
    grid = domain.grid
    D = grid.D
    for _ in range(depth):
        leaves = grid.active_leaves()
        # per-leaf blocks: level k of the per-leaf subtree holds 2^k cells; sequential refine!
        # calls allocate each leaf's subtree ids contiguously.
        block = sum(2 ** k for k in range(1, D + 1))
        base = grid.stored_cell_count() + 1
        n = leaves.size
        current = leaves.copy()  # cells to split at this axis, per leaf (n x 2^(axis-1))
        current = current[:, None]
        offset = 0
        new_levels, new_coords, new_parent = [], [], []
        per_axis_first = []
        for a in range(D):
            m = current.shape[1]
            cells = current.reshape(-1)
            # child ids inside each leaf block
            local = offset + 2 * np.arange(m, dtype=np.int64)
            first = (base + block * np.arange(n, dtype=np.int64))[:, None] + local[None, :]
            lev = grid.levels[cells] if a == 0 else lev_prev.reshape(-1, D)
            crd = grid.coords[cells] if a == 0 else crd_prev.reshape(-1, D)
            lev2 = np.repeat(lev, 2, axis=0)
            crd2 = np.repeat(crd, 2, axis=0)
            lev2[:, a] += 1
            crd2[:, a] = 2 * crd2[:, a] + np.tile(np.array([0, 1], dtype=np.int64), cells.size)
            ids = np.stack([first, first + 1], axis=2).reshape(n, 2 * m)
            new_levels.append((ids.reshape(-1), lev2, crd2, np.repeat(cells, 2)))
            per_axis_first.append((cells, first.reshape(-1), a + 1))
            current = ids
            lev_prev, crd_prev = lev2, crd2
            offset += 2 * m
        total_new = n * block
        L = np.zeros((total_new, D), dtype=np.int32)
        Cc = np.zeros((total_new, D), dtype=np.int64)
        Pp = np.zeros(total_new, dtype=np.int64)
        for ids, lev2, crd2, par in new_levels:
            L[ids - base] = lev2
            Cc[ids - base] = crd2
            Pp[ids - base] = par
        grid.levels = np.concatenate([grid.levels, L])
        grid.coords = np.concatenate([grid.coords, Cc])
        grid.parent = np.concatenate([grid.parent, Pp])
        grid.first_child = np.concatenate([grid.first_child, np.zeros(total_new, dtype=np.int64)])
        grid.split_axis = np.concatenate([grid.split_axis, np.zeros(total_new, dtype=np.int32)])
        grid.active = np.concatenate([grid.active, np.zeros(total_new, dtype=bool)])
        for cells, first, axis in per_axis_first:
            grid.first_child[cells] = first
            grid.split_axis[cells] = axis
        last_ids = current.reshape(-1)
        grid.active[leaves] = False
        grid.active[last_ids] = True
        grid.revision += 1
    return domain


class Domain:
    """Domain(origin, extent, root_counts) on a fresh CartesianGrid (geometry.jl:134-141)."""

    def __init__(self, origin, extent, root_counts, periodic=False):
        if not (len(origin) == len(extent) == len(root_counts)):
            raise ValueError("origin, extent and root_counts must have the same dimension")
        self.origin = tuple(float(v) for v in origin)
        self.extent = tuple(float(v) for v in extent)
        if any(e <= 0 for e in self.extent):
            raise ValueError("extent must be positive")
        self.grid = CartesianGrid(root_counts, periodic=periodic)
        self.D = self.grid.D

    def cell_size(self, cells):
        """h per axis: extent/root_count scaled by 2^-level (geometry.jl:683-687)."""
        cells = np.asarray(cells, dtype=np.int64)
        root = np.array(self.extent) / np.array(self.grid.root_counts)
        return np.ldexp(root[None, :], -self.grid.levels[cells].astype(np.int64))

    def cell_lower(self, cells):
        cells = np.asarray(cells, dtype=np.int64)
        h = self.cell_size(cells)
        return np.array(self.origin)[None, :] + h * self.grid.coords[cells]


def grid(domain):
    return domain.grid

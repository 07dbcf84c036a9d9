"""HpSpace on the host: degree policies and the native continuity compile.

Mirrors `HpSpace`, `SpaceOptions`, `FullTensorBasis`/`TrunkBasis`, `UniformDegree`,
`AxisDegrees`, `ByLeafDegrees` and `DegreePlusQuadrature` (space.jl:130-326, basis.jl:60-126).
The continuity algebra runs in libgrico_b200 (grico_space_build); this module only gathers
the active leaves and reads back the compiled term maps.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class FullTensorBasis:
    code = L.GRICO_BASIS_FULL


class TrunkBasis:
    code = L.GRICO_BASIS_TRUNK


class UniformDegree:
    def __init__(self, degree):
        self.degree = int(degree)

    def degrees(self, domain, leaves):
        return np.full((len(leaves), domain.D), self.degree, dtype=np.int32)


class AxisDegrees:
    def __init__(self, degrees):
        self.value = tuple(int(d) for d in degrees)

    def degrees(self, domain, leaves):
        if len(self.value) != domain.D:
            raise ValueError("AxisDegrees length must match the dimension")
        return np.tile(np.array(self.value, dtype=np.int32), (len(leaves), 1))


class ByLeafDegrees:
    """degree_fn(leaf_id) -> int or tuple (space.jl:130)."""

    def __init__(self, fn):
        self.fn = fn

    def degrees(self, domain, leaves):
        out = np.zeros((len(leaves), domain.D), dtype=np.int32)
        for i, leaf in enumerate(leaves):
            v = self.fn(int(leaf))
            out[i] = v if np.ndim(v) else [int(v)] * domain.D
        return out


class StoredDegrees:
    """Explicit per-leaf degrees aligned with an active-leaf list (used by multigrid levels)."""

    def __init__(self, leaves, degrees):
        leaves = np.asarray(leaves, dtype=np.int64)
        order = np.argsort(leaves, kind="stable")
        self.sorted_leaves = leaves[order]
        self.sorted_degrees = np.asarray(degrees, dtype=np.int32).reshape(len(leaves), -1)[order]

    def degrees(self, domain, leaves):
        leaves = np.asarray(leaves, dtype=np.int64)
        k = np.searchsorted(self.sorted_leaves, leaves)
        if np.any(k >= len(self.sorted_leaves)) or np.any(self.sorted_leaves[np.minimum(k, len(self.sorted_leaves) - 1)] != leaves):
            raise KeyError("leaf without a stored degree")
        return self.sorted_degrees[k].astype(np.int32)


class DegreePlusQuadrature:
    def __init__(self, extra_points=1):
        self.extra_points = int(extra_points)


class SpaceOptions:
    """Defaults follow the reference: TrunkBasis, UniformDegree(1), DegreePlusQuadrature(1), :cg
    (space.jl:226-240)."""

    def __init__(self, basis=None, degree=None, quadrature=None, continuity="cg"):
        self.basis = basis if basis is not None else TrunkBasis()
        self.degree = degree if degree is not None else UniformDegree(1)
        if isinstance(self.degree, int):
            self.degree = UniformDegree(self.degree)
        self.quadrature = quadrature if quadrature is not None else DegreePlusQuadrature(1)
        if continuity not in ("cg", "dg", ":cg", ":dg"):
            raise ValueError("continuity must be :cg or :dg")
        self.continuity = continuity.lstrip(":")


class HpSpace:
    """Compiled hp space: Morton-ordered leaves, per-leaf degrees and sparse term maps."""

    def __init__(self, domain, options=None, active=None):
        options = options or SpaceOptions()
        self.domain = domain
        self.options = options
        self.D = domain.D
        grid = domain.grid
        if active is not None:
            leaves = np.asarray(active, dtype=np.int64)
        elif hasattr(domain, "active_leaves"):
            leaves = domain.active_leaves()     # PhysicalDomain: drops :outside leaves
        else:
            leaves = grid.active_leaves()
        self.input_leaves = leaves
        degrees = options.degree.degrees(domain, leaves)
        cg = options.continuity == "cg"
        if cg and np.any(degrees < 1):
            raise ValueError("degree must be at least 1 on :cg axes")
        root = np.array(grid.root_counts, dtype=np.int64)
        lev = np.ascontiguousarray(grid.levels[leaves], dtype=np.int32)
        crd = np.ascontiguousarray(grid.coords[leaves], dtype=np.int64)
        deg = np.ascontiguousarray(degrees, dtype=np.int32)
        handle = C.c_void_p()
        lib = L.lib()
        L.check(lib.grico_space_build(self.D, L.ptr(root, C.c_int64), len(leaves), L.ptr(lev, C.c_int32),
                                      L.ptr(crd, C.c_int64), L.ptr(deg, C.c_int32), options.basis.code,
                                      L.GRICO_CONTINUITY_CG if cg else L.GRICO_CONTINUITY_DG,
                                      options.quadrature.extra_points, C.byref(handle)), "HpSpace")
        self.handle = handle  # kept for multigrid transfers; destroyed with the space
        sizes = [C.c_int64() for _ in range(5)]
        L.check(lib.grico_space_sizes(handle, *[C.byref(s) for s in sizes]))
        ndofs, nterms, nboxes, nbnd, nif = (s.value for s in sizes)
        n = len(leaves)
        order = np.zeros(n, dtype=np.int64)
        box_off = np.zeros(n + 1, dtype=np.int64)
        t_off = np.zeros(nboxes + 1, dtype=np.int64)
        t_idx = np.zeros(nterms, dtype=np.int64)
        t_coef = np.zeros(nterms, dtype=np.float64)
        qshape = np.zeros(n * self.D, dtype=np.int32)
        b_leaf = np.zeros(nbnd, dtype=np.int64)
        b_axis = np.zeros(nbnd, dtype=np.int32)
        b_side = np.zeros(nbnd, dtype=np.int32)
        i_m = np.zeros(nif, dtype=np.int64)
        i_p = np.zeros(nif, dtype=np.int64)
        i_a = np.zeros(nif, dtype=np.int32)
        L.check(lib.grico_space_export(handle, L.ptr(order, C.c_int64), L.ptr(box_off, C.c_int64),
                                       L.ptr(t_off, C.c_int64), L.ptr(t_idx, C.c_int64),
                                       L.ptr(t_coef, C.c_double), L.ptr(qshape, C.c_int32),
                                       L.ptr(b_leaf, C.c_int64), L.ptr(b_axis, C.c_int32),
                                       L.ptr(b_side, C.c_int32), L.ptr(i_m, C.c_int64),
                                       L.ptr(i_p, C.c_int64), L.ptr(i_a, C.c_int32)))
        self.leaves = leaves[order]                      # Morton order, cell ids
        self.degrees = degrees[order]                    # [n, D]
        self.qshape = qshape.reshape(n, self.D)
        self.scalar_dof_count = int(ndofs)
        self.box_offsets = box_off                      # per leaf into the box-mode arrays
        self.term_offsets = t_off                       # CSR over box modes
        self.term_index = t_idx                         # 0-based dofs
        self.term_coef = t_coef
        self.boundary_faces = (b_leaf, b_axis, b_side)  # positions in Morton order, 0-based axis, 0/1 side
        self.interfaces = (i_m, i_p, i_a)
        self.leaf_to_index = {int(l): i for i, l in enumerate(self.leaves)}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.lib().grico_space_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ---- queries mirroring the reference API ----
    def active_leaf_count(self):
        return len(self.leaves)

    def cell_degrees(self, leaf):
        return tuple(int(v) for v in self.degrees[self.leaf_to_index[int(leaf)]])

    def support_shape(self, leaf):
        return tuple(d + 1 for d in self.cell_degrees(leaf))

    def mode_terms(self, leaf, mode):
        """[(dof (1-based), coefficient)] of one local mode (space.jl mode_terms)."""
        i = self.leaf_to_index[int(leaf)]
        shape = self.support_shape(leaf)
        box, stride = 0, 1
        for a, m in enumerate(mode):
            if not 0 <= m < shape[a]:
                raise ValueError("mode outside the degree box")
            box += m * stride
            stride *= shape[a]
        e = self.box_offsets[i] + box
        lo, hi = self.term_offsets[e], self.term_offsets[e + 1]
        if lo == hi:
            raise ValueError(f"mode {mode} is not active on leaf {leaf}")
        return [(int(self.term_index[t]) + 1, float(self.term_coef[t])) for t in range(lo, hi)]

    def local_mode_count(self, leaf):
        i = self.leaf_to_index[int(leaf)]
        lo, hi = self.box_offsets[i], self.box_offsets[i + 1]
        return int(np.count_nonzero(np.diff(self.term_offsets[lo:hi + 1])))


def scalar_dof_count(space):
    return space.scalar_dof_count


def active_leaf_count(space):
    return space.active_leaf_count()

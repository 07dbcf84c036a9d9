"""CPU oracle for the Grico matrix-free hot path — TEST INFRASTRUCTURE ONLY.

This module is a literal, loop-by-loop restatement of the reference algorithms
that produce the data the GPU path consumes (Grico.jl, Julia).  It exists so the
tests can check the product (``grico.jl_b200``) against an independent
derivation.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import it, and only as the checker.

Parity pins (reference known-answer tests restated in ``tests/test_oracle_kat.py``):
  * polynomial values/derivatives      test/core.jl:152-167
  * DOF counts, hanging coefficients   test/space.jl:274-320, 639-700
  * small apply / Dirichlet values     test/matrix_free.jl:305,578,780
  * GMG level sizes                    test/multigrid.jl:160,171

Each function names the reference file:line it follows.  Floating point
operation order follows the reference where the reference fixes it (polynomial
recurrences, Newton, restriction matrices); LAPACK calls use the same drivers
as Julia's LinearAlgebra (getrf/getrs, syevr, geqp3) through scipy.
"""

from __future__ import annotations

import math
from collections import OrderedDict

import numpy as np
import scipy.linalg as sla

EPS = np.finfo(np.float64).eps
LOWER, UPPER = 1, 2
NONE = 0


# ---------------------------------------------------------------------------
# 1-D numerics: src/polynomials.jl, src/quadrature.jl
# ---------------------------------------------------------------------------

def legendre_values(x: float, n: int) -> list:
    """P_0..P_n at x (polynomials.jl:294-306; same operation order)."""
    v = [0.0] * (n + 1)
    v[0] = 1.0
    if n >= 1:
        v[1] = x
    for k in range(2, n + 1):
        inv_k = 1.0 / float(k)
        v[k] = float(2 * k - 1) * inv_k * x * v[k - 1] - float(k - 1) * inv_k * v[k - 2]
    return v


def legendre_values_and_derivatives(x: float, n: int):
    """P and P' (polynomials.jl:308-326)."""
    v = [0.0] * (n + 1)
    d = [0.0] * (n + 1)
    v[0] = 1.0
    d[0] = 0.0
    if n >= 1:
        v[1] = x
        d[1] = 1.0
    for k in range(2, n + 1):
        inv_k = 1.0 / float(k)
        first = float(2 * k - 1) * inv_k
        second = float(k - 1) * inv_k
        v[k] = first * x * v[k - 1] - second * v[k - 2]
        d[k] = first * (v[k - 1] + x * d[k - 1]) - second * d[k - 2]
    return v, d


def integrated_legendre_values_and_derivatives(x: float, n: int):
    """psi_0=(1-x)/2, psi_1=(1+x)/2, psi_k=(P_k-P_{k-2})/sqrt(4k-2); psi_k'=sqrt((2k-1)/2) P_{k-1}
    (polynomials.jl:403-434)."""
    v = legendre_values(x, n)
    d = [0.0] * (n + 1)
    for k in range(n, 1, -1):
        d[k] = math.sqrt(float(2 * k - 1) / 2.0) * v[k - 1]
    d[0] = -0.5
    if n >= 1:
        d[1] = 0.5
    for k in range(n, 1, -1):
        v[k] = (v[k] - v[k - 2]) / math.sqrt(float(4 * k - 2))
    v[0] = 0.5 * (1.0 - x)
    if n >= 1:
        v[1] = 0.5 * (1.0 + x)
    return v, d


def fe_basis_values_and_derivatives(x: float, p: int):
    """Degree 0 is the DG constant, else integrated Legendre (polynomials.jl:238-247)."""
    if p == 0:
        return [1.0], [0.0]
    return integrated_legendre_values_and_derivatives(x, p)


def gauss_legendre_rule(count: int):
    """Newton from cosine guesses, mirrored halves, ascending (quadrature.jl:342-410)."""
    pts = [0.0] * count
    wts = [0.0] * count
    tol = 1.0e3 * EPS
    half = (count + 1) // 2
    for i in range(1, half + 1):
        x = math.cos(math.pi * (float(i) - 0.25) / (float(count) + 0.5))
        converged = False
        for _ in range(32):
            v, d = legendre_values_and_derivatives(x, count)
            delta = v[count] / d[count]
            x -= delta
            if abs(delta) <= tol:
                v, d = legendre_values_and_derivatives(x, count)
                converged = True
                break
        if not converged:
            raise ValueError("Gauss-Legendre root did not converge")
        w = 2.0 / ((1.0 - x * x) * d[count] ** 2)
        pts[i - 1] = -x
        wts[i - 1] = w
        m = count - i
        pts[m] = x
        wts[m] = w
    return pts, wts


# ---------------------------------------------------------------------------
# Modes: src/basis.jl
# ---------------------------------------------------------------------------

def mode_from_linear(index: int, degrees):
    """Mixed radix, axis 1 fastest (basis.jl:351-365)."""
    out = []
    for p in degrees:
        out.append(index % (p + 1))
        index //= (p + 1)
    return tuple(out)


def basis_modes(basis: str, degrees):
    """FullTensor: whole box; Trunk: sum of interior orders <= max degree (basis.jl:97-190)."""
    total = 1
    for p in degrees:
        total *= p + 1
    modes = [mode_from_linear(i, degrees) for i in range(total)]
    if basis == "full":
        return modes
    limit = max(degrees) if degrees else 0
    return [m for m in modes if sum(0 if v <= 1 else v for v in m) <= limit]


def flatten_mode(mode, shape):
    """One-based mixed-radix index (space.jl:941-951)."""
    idx, stride = 1, 1
    for a in range(len(mode)):
        idx += mode[a] * stride
        stride *= shape[a]
    return idx


# ---------------------------------------------------------------------------
# Topology: src/topology.jl, src/refinement.jl, src/geometry.jl
# ---------------------------------------------------------------------------

class Grid:
    """Cartesian refinement tree; cell ids are 1-based like the reference (topology.jl:96-163)."""

    def __init__(self, root_counts):
        self.D = len(root_counts)
        self.root_counts = tuple(int(c) for c in root_counts)
        total = 1
        for c in self.root_counts:
            total *= c
        self.levels = [[0] * (total + 1) for _ in range(self.D)]
        self.coords = [[0] * (total + 1) for _ in range(self.D)]
        self.parent = [NONE] * (total + 1)
        self.first_child = [NONE] * (total + 1)
        self.split_axis = [0] * (total + 1)
        self.active = [False] + [True] * total
        strides = []
        s = 1
        for a in range(self.D):
            strides.append(s)
            s *= self.root_counts[a]
        for cell in range(1, total + 1):
            lin = cell - 1
            for a in range(self.D):
                self.coords[a][cell] = (lin // strides[a]) % self.root_counts[a]

    def stored(self):
        return len(self.parent) - 1

    def refine(self, cell, axis):
        """Append one midpoint child block (refinement.jl:47-76). axis is 1-based."""
        assert self.active[cell]
        a = axis - 1
        first = self.stored() + 1
        for off in range(2):
            for b in range(self.D):
                if b == a:
                    self.levels[b].append(self.levels[b][cell] + 1)
                    self.coords[b].append(2 * self.coords[b][cell] + off)
                else:
                    self.levels[b].append(self.levels[b][cell])
                    self.coords[b].append(self.coords[b][cell])
            self.parent.append(cell)
            self.first_child.append(NONE)
            self.split_axis.append(0)
            self.active.append(True)
        self.first_child[cell] = first
        self.split_axis[cell] = axis
        self.active[cell] = False
        return first

    def active_leaves(self):
        return [c for c in range(1, self.stored() + 1) if self.active[c]]

    def level(self, cell, a):
        return self.levels[a][cell]

    def coord(self, cell, a):
        return self.coords[a][cell]


def uniform_refine(grid: Grid, depth: int):
    """Refine every leaf on every axis, axis by axis (benchmark/hpmg_scaling.jl:122-164)."""
    for _ in range(depth):
        for leaf in list(grid.active_leaves()):
            leaves = [leaf]
            for axis in range(1, grid.D + 1):
                nxt = []
                for cur in leaves:
                    f = grid.refine(cur, axis)
                    nxt += [f, f + 1]
                leaves = nxt


def morton_ordered_leaves(grid: Grid, leaves=None):
    """Sort active leaves by Morton code of the lower corner on the finest lattice; bits high to low,
    axes D..1 within a bit; ties by level tuple then cell id (topology.jl:250-268, 451-463)."""
    leaves = grid.active_leaves() if leaves is None else [int(l) for l in leaves]
    D = grid.D
    max_levels = [max(grid.level(l, a) for l in leaves) for a in range(D)]
    bit_count = 0
    for a in range(D):
        value = (grid.root_counts[a] << max_levels[a]) - 1
        bits = 0
        while value > 0:
            bits += 1
            value >>= 1
        bit_count = max(bit_count, bits)

    def key(leaf):
        lower = [grid.coord(leaf, a) << (max_levels[a] - grid.level(leaf, a)) for a in range(D)]
        code = 0
        for bit in range(bit_count - 1, -1, -1):
            for a in range(D - 1, -1, -1):
                code = (code << 1) | ((lower[a] >> bit) & 1)
        return (code, tuple(grid.level(leaf, a) for a in range(D)), leaf)

    return sorted(leaves, key=key)


class Snapshot:
    """Morton-ordered leaves, boundary faces and interfaces (topology.jl:232-245, 1502-1545).

    Neighbour search is done on the common finest lattice; the enumeration order matches the
    reference: leaves in Morton order, axes ascending, UPPER-side partners sorted by their
    tangential lower corner (axis 1 first)."""

    def __init__(self, grid: Grid, leaves=None):
        self.grid = grid
        D = grid.D
        self.leaves = morton_ordered_leaves(grid, leaves)
        self.leaf_to_index = {leaf: i for i, leaf in enumerate(self.leaves)}
        self.finest = [max(grid.level(l, a) for l in self.leaves) for a in range(D)]
        self.lower = {}
        self.upper = {}
        for l in self.leaves:
            self.lower[l] = tuple(grid.coord(l, a) << (self.finest[a] - grid.level(l, a)) for a in range(D))
            self.upper[l] = tuple((grid.coord(l, a) + 1) << (self.finest[a] - grid.level(l, a)) for a in range(D))
        self.extent = [grid.root_counts[a] << self.finest[a] for a in range(D)]
        # index leaves by their lower/upper face coordinate on each axis
        by_lower = [dict() for _ in range(D)]
        for l in self.leaves:
            for a in range(D):
                by_lower[a].setdefault(self.lower[l][a], []).append(l)
        self.boundary = []  # (leaf, axis(1-based), side)
        self.interfaces = []  # (minus, plus, axis(1-based))
        # tree lookup over the active leaves and all their ancestors (topology.jl:1547-1566)
        self.tree = {}
        for l in self.leaves:
            cur = l
            while cur != NONE:
                self.tree[(tuple(grid.level(cur, a) for a in range(D)), tuple(grid.coord(cur, a) for a in range(D)))] = cur
                cur = grid.parent[cur]
        for l in self.leaves:
            for a in range(D):
                for side in (LOWER, UPPER):
                    if self.covering_neighbor(l, a, side) == NONE:
                        self.boundary.append((l, a + 1, side))
        for l in self.leaves:
            for a in range(D):
                partners = []
                for other in by_lower[a].get(self.upper[l][a], []):
                    ok = True
                    for b in range(D):
                        if b == a:
                            continue
                        if not (max(self.lower[l][b], self.lower[other][b]) < min(self.upper[l][b], self.upper[other][b])):
                            ok = False
                            break
                    if ok:
                        partners.append(other)
                partners.sort(key=lambda o: tuple(0 if b == a else self.lower[o][b] for b in range(D)))
                for o in partners:
                    self.interfaces.append((l, o, a + 1))


    def covering_neighbor(self, cell, a, side):
        """`_snapshot_covering_neighbor` (topology.jl:1590-1608, 1670-1677): the tree cell of the
        same level tuple next to `cell` across side `side` of axis `a` (0-based) if the lookup
        holds it; otherwise retry from the parent while `cell` touches the parent's boundary on
        that side (always when the parent was split along another axis).  NONE: no covering
        neighbour, so the face is a boundary face."""
        grid = self.grid
        D = grid.D
        cur = cell
        while True:
            lev = tuple(grid.level(cur, b) for b in range(D))
            crd = [grid.coord(cur, b) for b in range(D)]
            crd[a] += -1 if side == LOWER else 1
            if 0 <= crd[a] < (grid.root_counts[a] << lev[a]):
                cand = self.tree.get((lev, tuple(crd)), NONE)
                if cand != NONE:
                    return cand
            par = grid.parent[cur]
            if par == NONE:
                return NONE
            if grid.split_axis[par] == a + 1 and (grid.coord(cur, a) & 1) != (0 if side == LOWER else 1):
                return NONE
            cur = par


class Domain:
    """Affine box geometry on a grid (geometry.jl:134-141, 676-711)."""

    def __init__(self, origin, extent, root_counts):
        self.origin = tuple(float(v) for v in origin)
        self.extent = tuple(float(v) for v in extent)
        self.grid = Grid(root_counts)
        self.D = len(root_counts)

    def cell_size(self, cell, a):
        root = self.extent[a] / self.grid.root_counts[a]
        return math.ldexp(root, -self.grid.level(cell, a))

    def cell_lower(self, cell, a):
        return self.origin[a] + self.cell_size(cell, a) * self.grid.coord(cell, a)

    def center_half(self, cell, a):
        size = self.cell_size(cell, a)
        lower = self.origin[a] + size * self.grid.coord(cell, a)
        half = 0.5 * size
        return lower + half, half

    def det_biunit(self, cell):
        prod = 1.0
        for a in range(self.D):
            prod *= self.cell_size(cell, a)
        return math.ldexp(prod, -self.D)


# ---------------------------------------------------------------------------
# Continuity: src/continuity.jl (phases 1-6)
# ---------------------------------------------------------------------------

def _constraint_tolerance(coefs):
    scale = 0.0
    for c in coefs:
        scale = max(scale, abs(c))
    return 4.0 * EPS * max(scale, 1.0)


class Row:
    __slots__ = ("vars", "coefs")

    def __init__(self):
        self.vars = []
        self.coefs = []

    def add(self, var, c):
        """continuity.jl:1000-1010"""
        for i, v in enumerate(self.vars):
            if v == var:
                self.coefs[i] += c
                return
        self.vars.append(var)
        self.coefs.append(c)

    def remove_at(self, i):
        del self.vars[i]
        del self.coefs[i]

    def remove_var(self, var):
        for i, v in enumerate(self.vars):
            if v == var:
                self.remove_at(i)
                return

    def cleanup(self):
        """continuity.jl:681-700"""
        tol = _constraint_tolerance(self.coefs)
        i = 0
        while i < len(self.vars):
            if abs(self.coefs[i]) <= tol:
                self.remove_at(i)
            else:
                i += 1

    def accumulate(self, src, factor=1.0):
        for v, c in zip(src.vars, src.coefs):
            self.add(v, factor * c)


def _uf_root(parent, v):
    root = v
    while parent[root] != root:
        root = parent[root]
    while parent[v] != v:
        nxt = parent[v]
        parent[v] = root
        v = nxt
    return root


def _uf_union(parent, a, b):
    """Smaller root wins (continuity.jl:1053-1065)."""
    ra = _uf_root(parent, a)
    rb = _uf_root(parent, b)
    if ra == rb:
        return ra
    if ra < rb:
        parent[rb] = ra
        return ra
    parent[ra] = rb
    return rb


_RESTRICTION_CACHE = {}


def affine_restriction_matrix(source_degree, target_degree, delta, relative):
    """Collocation on target_degree+1 Gauss points, LU solve (continuity.jl:1158-1198)."""
    key = (source_degree, target_degree, delta, relative)
    if key in _RESTRICTION_CACHE:
        return _RESTRICTION_CACHE[key]
    scale = math.ldexp(1.0, -delta)
    shift = 0.0 if delta == 0 else scale * (2.0 * float(relative) + 1.0) - 1.0
    n = target_degree + 1
    pts, _ = gauss_legendre_rule(n)
    basis = np.zeros((n, n))
    for i in range(n):
        v, _ = fe_basis_values_and_derivatives(pts[i], target_degree)
        basis[i, :] = v
    src = np.zeros((n, source_degree + 1))
    for i in range(n):
        xi = scale * pts[i] + shift
        v, _ = fe_basis_values_and_derivatives(xi, source_degree)
        src[i, :] = v
    lu, piv = sla.lu_factor(basis)
    mat = sla.lu_solve((lu, piv), src)
    _RESTRICTION_CACHE[key] = mat
    return mat


def _interval_level_coord(lower, upper, finest):
    length = upper - lower
    assert length > 0 and (length & (length - 1)) == 0
    shift = length.bit_length() - 1
    return finest - shift, lower >> shift


def _restriction_coefficient(src_lo, src_hi, tgt_lo, tgt_hi, src_index, src_deg, tgt_deg, tgt_index, finest):
    """continuity.jl:1085-1147"""
    sl, sc = _interval_level_coord(src_lo, src_hi, finest)
    tl, tc = _interval_level_coord(tgt_lo, tgt_hi, finest)
    delta = tl - sl
    relative = tc - (sc << delta)
    mat = affine_restriction_matrix(src_deg, tgt_deg, delta, relative)
    return float(mat[tgt_index, src_index])


class Space:
    """HpSpace compile (space.jl:300-326, 742-752; continuity.jl phases 1-6).

    degree_fn(leaf) -> degree tuple; basis 'full' or 'trunk'; continuity 'cg' or 'dg' (all axes);
    quadrature extra points (DegreePlusQuadrature, default 1)."""

    def __init__(self, domain: Domain, degree, basis="trunk", continuity="cg", quadrature_extra=1, leaves=None):
        self.domain = domain
        self.grid = domain.grid
        self.D = domain.D
        self.basis = basis
        self.continuity = continuity
        self.snapshot = Snapshot(self.grid, leaves)
        snap = self.snapshot
        D = self.D
        leaves = snap.leaves
        if callable(degree):
            self.degrees = [tuple(degree(l)) for l in leaves]
        else:
            deg = tuple(degree) if isinstance(degree, (tuple, list)) else (int(degree),) * D
            self.degrees = [deg for _ in leaves]
        self.quadrature_extra = quadrature_extra
        self.qshape = [tuple(max(d + quadrature_extra, 1) for d in degs) for degs in self.degrees]
        self.patterns = []
        for degs in self.degrees:
            modes = basis_modes(basis, degs)
            self.patterns.append((modes, [m for m in modes if any(v <= 1 for v in m)]))
        self.next_dof = 1
        nleaf = len(leaves)
        self.lookup = [dict() for _ in range(nleaf)]
        self.min_pivot = math.inf
        self.noise_pivots = 0
        self.face_modes = {}
        self.boundary_terms = []
        if continuity == "cg":
            self._build_boundary_variables()
            self._compile_boundary_terms()
        # phase 6
        self.leaf_modes = []
        self.leaf_terms = []  # list per leaf: list per mode of [(dof, coef)]
        for li in range(nleaf):
            modes_out, terms_out = [], []
            for mode in self.patterns[li][0]:
                if continuity == "cg" and any(v <= 1 for v in mode):
                    var = self.lookup[li][mode]
                    terms = [(d, c) for (d, c) in self.boundary_terms[var] if c != 0.0]
                else:
                    terms = [(self.next_dof, 1.0)]
                    self.next_dof += 1
                if terms:
                    modes_out.append(mode)
                    terms_out.append(terms)
            self.leaf_modes.append(modes_out)
            self.leaf_terms.append(terms_out)
        self.ndofs = self.next_dof - 1

    # -- phase 3 ---------------------------------------------------------
    def _fm(self, li, axis, side):
        return self.face_modes.setdefault((li, axis, side), [])

    def _build_boundary_variables(self):
        """continuity.jl:223-252"""
        nxt = 1
        for li in range(len(self.snapshot.leaves)):
            for mode in self.patterns[li][1]:
                var = nxt
                self.lookup[li][mode] = var
                for a in range(self.D):
                    if mode[a] <= 1:
                        self._fm(li, a + 1, mode[a] + LOWER).append((var, mode))
                nxt += 1
        self.nvars = nxt - 1
        self.boundary_terms = [None] + [[] for _ in range(self.nvars)]

    # -- phases 4/5 ------------------------------------------------------
    def _matching(self, f, s, axis):
        snap = self.snapshot
        lf, ls = snap.leaves[f], snap.leaves[s]
        for b in range(self.D):
            if b == axis - 1:
                continue
            if snap.lower[lf][b] != snap.lower[ls][b] or snap.upper[lf][b] != snap.upper[ls][b]:
                return False
        return True

    def _same_trace_modes(self, f, s, axis):
        fv = self._fm(f, axis, UPPER)
        sv = self._fm(s, axis, LOWER)
        if len(fv) != len(sv):
            return False
        for (_, mode) in fv:
            m2 = tuple(0 if b == axis - 1 else mode[b] for b in range(self.D))
            if m2 not in self.lookup[s]:
                return False
        return True

    def _compile_boundary_terms(self):
        """continuity.jl:384-422"""
        snap = self.snapshot
        parent = list(range(self.nvars + 1))
        pairs = [(snap.leaf_to_index[m], snap.leaf_to_index[p], ax) for (m, p, ax) in snap.interfaces]
        constraint_pairs = []
        for (f, s, axis) in pairs:
            if self._matching(f, s, axis) and self._same_trace_modes(f, s, axis):
                for (var, mode) in self._fm(f, axis, UPPER):
                    m2 = tuple(0 if b == axis - 1 else mode[b] for b in range(self.D))
                    _uf_union(parent, var, self.lookup[s][m2])
            else:
                constraint_pairs.append((f, s, axis))
        roots = [0] + [_uf_root(parent, v) for v in range(1, self.nvars + 1)]
        rows = self._face_rows(roots, constraint_pairs)
        if not rows:
            free = [0] * (self.nvars + 1)
            for v in range(1, self.nvars + 1):
                if roots[v] == v:
                    free[v] = self.next_dof
                    self.next_dof += 1
            for v in range(1, self.nvars + 1):
                if roots[v] == v:
                    self.boundary_terms[v] = [(free[v], 1.0)]
            for v in range(1, self.nvars + 1):
                if roots[v] != v:
                    self.boundary_terms[v] = self.boundary_terms[roots[v]]
            return
        # components (continuity.jl:809-833)
        cparent = list(range(self.nvars + 1))
        for row in rows:
            if len(row.vars) <= 1:
                continue
            for v in row.vars[1:]:
                _uf_union(cparent, row.vars[0], v)
        comp_rows = {}
        for row in rows:
            if not row.vars:
                continue
            comp_rows.setdefault(_uf_root(cparent, row.vars[0]), []).append(row)
        components = sorted(comp_rows.keys())
        pivots = [None] * (self.nvars + 1)
        orders = []
        self.min_pivot = math.inf
        for comp in components:
            local = {}
            order = []
            for row in comp_rows[comp]:
                while True:
                    changed = False
                    for i, v in enumerate(row.vars):
                        expr = local.get(v)
                        if expr is None:
                            continue
                        factor = row.coefs[i]
                        row.remove_at(i)
                        row.accumulate(expr, factor)
                        changed = True
                        break
                    row.cleanup()
                    if not changed:
                        break
                if not row.vars:
                    continue
                pidx = max(range(len(row.vars)), key=lambda i: row.vars[i])
                pivot, pcoef = row.vars[pidx], row.coefs[pidx]
                self.min_pivot = min(self.min_pivot, abs(pcoef))
                if abs(pcoef) < 1e-10:
                    self.noise_pivots += 1      # diagnostic only: a rounding-residue pivot
                row.remove_var(pivot)
                scale = -(1.0 / pcoef)
                expr = Row()
                expr.accumulate(row, scale)
                expr.cleanup()
                local[pivot] = expr
                pivots[pivot] = expr
                order.append(pivot)
            orders.append(order)
        free = [0] * (self.nvars + 1)
        for v in range(1, self.nvars + 1):
            if roots[v] == v and pivots[v] is None:
                free[v] = self.next_dof
                self.next_dof += 1
        for v in range(1, self.nvars + 1):
            if roots[v] == v:
                self.boundary_terms[v] = [] if pivots[v] is not None else [(free[v], 1.0)]
        for order in orders:
            for pivot in reversed(order):
                expr = pivots[pivot]
                acc = Row()
                for v, factor in zip(expr.vars, expr.coefs):
                    if factor == 0.0:
                        continue
                    terms = self.boundary_terms[v]
                    if not terms:
                        assert free[v] == 0
                        continue
                    for (d, c) in terms:
                        acc.add(d, factor * c)
                acc.cleanup()
                self.boundary_terms[pivot] = sorted(zip(acc.vars, acc.coefs), key=lambda t: t[0])
        for v in range(1, self.nvars + 1):
            if roots[v] != v:
                self.boundary_terms[v] = self.boundary_terms[roots[v]]

    def _face_rows(self, roots, constraint_pairs):
        """continuity.jl:470-530, 566-620"""
        snap = self.snapshot
        D = self.D
        rows = []
        for (f, s, axis) in constraint_pairs:
            a0 = axis - 1
            cdeg = tuple(0 if b == a0 else max(self.degrees[f][b], self.degrees[s][b]) for b in range(D))
            lf, ls = snap.leaves[f], snap.leaves[s]
            face = snap.upper[lf][a0]
            plo = tuple(face if b == a0 else max(snap.lower[lf][b], snap.lower[ls][b]) for b in range(D))
            phi = tuple(face if b == a0 else min(snap.upper[lf][b], snap.upper[ls][b]) for b in range(D))
            for cmode in basis_modes("full", cdeg):
                row = Row()
                for (li, side, sign) in ((f, UPPER, 1.0), (s, LOWER, -1.0)):
                    leaf = snap.leaves[li]
                    for (var, mode) in self._fm(li, axis, side):
                        coef = 1.0
                        for b in range(D):
                            if b == a0:
                                continue
                            coef *= _restriction_coefficient(snap.lower[leaf][b], snap.upper[leaf][b], plo[b], phi[b],
                                                             mode[b], self.degrees[li][b], cdeg[b], cmode[b],
                                                             snap.finest[b])
                            if coef == 0.0:
                                coef = 0.0
                                break
                        if coef == 0.0:
                            continue
                        row.add(roots[var], sign * coef)
                row.cleanup()
                if row.vars:
                    rows.append(row)
        return rows

    # -- queries ---------------------------------------------------------
    def mode_terms(self, leaf, mode):
        li = self.snapshot.leaf_to_index[leaf]
        return self.leaf_terms[li][self.leaf_modes[li].index(tuple(mode))]


# ---------------------------------------------------------------------------
# Plan data: integration tables (integration.jl:2161-2191, 2677-2742), Dirichlet
# (plans.jl:486-972), reduced map (assembly.jl:112-314), colouring (plans.jl:307-396)
# ---------------------------------------------------------------------------

class Plan:
    """A compiled scalar affine problem with cell forms.

    form: ('mass_diffusion', mu, kappa) meaning TestChannels(mu*u, kappa*grad u);
    kappa_fn: optional callable x -> kappa(x) multiplying the gradient channel pointwise.
    dirichlet: list of (axis, side, value) with constant values."""

    def __init__(self, space: Space, mu=0.0, kappa=1.0, kappa_fn=None, source=None, dirichlet=(),
                 cell_rules=None, surface_items=(), interface_penalty=None):
        """cell_rules: {leaf: (reference points [n, D], reference weights [n])} replacing the
        tensor rule of those leaves (finite-cell cut cells, add_cell_quadrature!);
        surface_items: [(leaf, reference points, physical weights, physical unit normals,
        penalty, g[, eta])] symmetric Nitsche items (boundary faces or embedded surfaces); eta
        defaults to penalty / min(h);
        interface_penalty: SIPG interior-penalty terms on every interface of the space
        (benchmark/sine_poisson_sipg.jl:54-95) with this penalty."""
        cell_rules = cell_rules or {}
        self.space = space
        dom = space.domain
        D = space.D
        snap = space.snapshot
        self.mu, self.kappa, self.kappa_fn, self.source = mu, kappa, kappa_fn, source
        self.ndofs = space.ndofs
        self.cells = []
        for li, leaf in enumerate(snap.leaves):
            if leaf in cell_rules:
                ref, wref = cell_rules[leaf]
                c = self._point_item(li, leaf, ref)
                c["w"] = np.asarray(wref, dtype=np.float64) * dom.det_biunit(leaf)
                self.cells.append(c)
                continue
            q = space.qshape[li]
            rules = [gauss_legendre_rule(n) for n in q]
            degs = space.degrees[li]
            modes = space.leaf_modes[li]
            det = dom.det_biunit(leaf)
            ch = [dom.center_half(leaf, a) for a in range(D)]
            inv_j = [1.0 / ch[a][1] for a in range(D)]
            axis_v, axis_g = [], []
            for a in range(D):
                V = np.zeros((degs[a] + 1, q[a]))
                G = np.zeros((degs[a] + 1, q[a]))
                for j in range(q[a]):
                    v, d = fe_basis_values_and_derivatives(rules[a][0][j], degs[a])
                    V[:, j] = v
                    G[:, j] = [inv_j[a] * dd for dd in d]
                axis_v.append(V)
                axis_g.append(G)
            npts = int(np.prod(q))
            pts = np.zeros((npts, D))
            w = np.zeros(npts)
            for p in range(npts):
                idx = mode_from_linear(p, tuple(n - 1 for n in q))
                wt = 1.0
                for a in range(D):
                    wt *= rules[a][1][idx[a]]
                w[p] = wt * det
                for a in range(D):
                    pts[p, a] = ch[a][0] + rules[a][0][idx[a]] * ch[a][1]
            # full shape tables values[mode, point], gradients[axis, mode, point] as tensor
            # products of the 1-D tables (integration.jl:2717-2740)
            mi = np.array(modes, dtype=np.int64).reshape(len(modes), D)
            pi = np.array([mode_from_linear(p, tuple(n - 1 for n in q)) for p in range(npts)],
                          dtype=np.int64).reshape(npts, D)
            fv = [axis_v[a][mi[:, a]][:, pi[:, a]] for a in range(D)]
            fg = [axis_g[a][mi[:, a]][:, pi[:, a]] for a in range(D)]
            vals = np.ones((len(modes), npts))
            for a in range(D):
                vals = vals * fv[a]
            grads = np.ones((D, len(modes), npts))
            for a in range(D):
                for b in range(D):
                    grads[a] = grads[a] * (fg[b] if b == a else fv[b])
            terms = space.leaf_terms[li]
            self.cells.append(dict(leaf=leaf, modes=modes, terms=terms, w=w, pts=pts, vals=vals, grads=grads,
                                   axis_v=axis_v, axis_g=axis_g, q=q, degs=degs))
        self.surfaces = []
        for (leaf, ref, wphys, nphys, penalty, g, *_) in surface_items:
            li = snap.leaf_to_index[leaf]
            c = self._point_item(li, leaf, ref)
            c["w"] = np.asarray(wphys, dtype=np.float64)
            c["normals"] = np.asarray(nphys, dtype=np.float64).reshape(-1, D)
            c["eta"] = penalty / min(dom.cell_size(leaf, a) for a in range(D))
            c["g"] = g
            self.surfaces.append(c)
        for k, it in enumerate(surface_items):
            if len(it) > 6 and it[6] is not None:
                self.surfaces[k]["eta"] = float(it[6])
        self.interfaces = []
        if interface_penalty is not None:
            for (m, pl, ax1) in snap.interfaces:
                self.interfaces.append(self._interface_item(m, pl, ax1 - 1, interface_penalty))
        self.colors = self._colour()
        self.fixed, self.fixed_values, self.rows = self._dirichlet(dirichlet)
        self.fixed_mask = np.zeros(self.ndofs + 1, dtype=bool)
        self.fixed_mask[self.fixed] = True
        self.blocked = np.zeros(self.ndofs + 1, dtype=bool)
        for (pivot, _, _, _) in self.rows:
            self.blocked[pivot] = True
        self._reduced_map()

    def _interface_item(self, m, pl, ax, penalty):
        """Shared tangential patch of the faces of leaves m (its upper face on axis ax) and pl,
        with max(q-, q+) Gauss points per tangential axis (integration.jl:2279-2307, 2800-2841),
        both sides' tables at the patch points, physical weights and the SIPG penalty
        (sine_poisson_sipg.jl:28-40)."""
        space, dom, D = self.space, self.space.domain, self.space.D
        snap = space.snapshot
        lm, lp = snap.leaf_to_index[m], snap.leaf_to_index[pl]
        chm = [dom.center_half(m, a) for a in range(D)]
        chp = [dom.center_half(pl, a) for a in range(D)]
        tang = [a for a in range(D) if a != ax]
        lo = {a: max(chm[a][0] - chm[a][1], chp[a][0] - chp[a][1]) for a in tang}
        hi = {a: min(chm[a][0] + chm[a][1], chp[a][0] + chp[a][1]) for a in tang}
        rules = [gauss_legendre_rule(max(space.qshape[lm][a], space.qshape[lp][a])) for a in tang]
        shape = tuple(len(r[0]) - 1 for r in rules)
        npts = int(np.prod([len(r[0]) for r in rules])) if tang else 1
        ref_m = np.zeros((npts, D))
        ref_p = np.zeros((npts, D))
        w = np.ones(npts)
        for p in range(npts):
            idx = mode_from_linear(p, shape) if tang else ()
            x = [0.0] * D
            for k, a in enumerate(tang):
                half = 0.5 * (hi[a] - lo[a])
                x[a] = lo[a] + half * (1.0 + rules[k][0][idx[k]])
                w[p] *= rules[k][1][idx[k]] * half
            for a in tang:
                ref_m[p, a] = (x[a] - chm[a][0]) / chm[a][1]
                ref_p[p, a] = (x[a] - chp[a][0]) / chp[a][1]
            ref_m[p, ax] = 1.0
            ref_p[p, ax] = -1.0
        hm, hp = dom.cell_size(m, ax), dom.cell_size(pl, ax)
        pmax = max(space.degrees[lm][ax], space.degrees[lp][ax])
        sigma = penalty * (pmax + 1) ** 2 / (2.0 * hm * hp / (hm + hp))
        return dict(minus=self._point_item(lm, m, ref_m), plus=self._point_item(lp, pl, ref_p), w=w, axis=ax,
                    sigma=sigma)

    def interface_local_apply(self, it, xm, xp):
        """-[v]{du/dn} - {dv/dn}[u] + sigma [v][u] at every patch point, [w] = w- - w+,
        n = e_axis from minus to plus (sine_poisson_sipg.jl:54-95)."""
        a = it["axis"]
        mi, pi = it["minus"], it["plus"]
        jump = mi["vals"].T @ xm - pi["vals"].T @ xp
        avg = 0.5 * (mi["grads"][a].T @ xm + pi["grads"][a].T @ xp)
        cv = it["w"] * (it["sigma"] * jump - avg)
        cd = -0.5 * it["w"] * jump
        return mi["vals"] @ cv + mi["grads"][a] @ cd, -(pi["vals"] @ cv) + pi["grads"][a] @ cd

    def _point_item(self, li, leaf, ref):
        """Full value/gradient tables of one leaf's modes at arbitrary reference points
        (_compile_field_values, integration.jl:2527-2560, non-tensor branch)."""
        space, dom, D = self.space, self.space.domain, self.space.D
        degs = space.degrees[li]
        modes = space.leaf_modes[li]
        ref = np.asarray(ref, dtype=np.float64).reshape(-1, D)
        npts = ref.shape[0]
        ch = [dom.center_half(leaf, a) for a in range(D)]
        vals = np.ones((len(modes), npts))
        grads = np.ones((D, len(modes), npts))
        pts = np.zeros((npts, D))
        for p in range(npts):
            tv, tg = [], []
            for a in range(D):
                v, d = fe_basis_values_and_derivatives(ref[p, a], degs[a])
                tv.append(v)
                tg.append([dd / ch[a][1] for dd in d])
                pts[p, a] = ch[a][0] + ref[p, a] * ch[a][1]
            for i, m in enumerate(modes):
                val = 1.0
                for a in range(D):
                    val *= tv[a][m[a]]
                vals[i, p] = val
                for a in range(D):
                    g = 1.0
                    for b in range(D):
                        g *= tg[b][m[b]] if b == a else tv[b][m[b]]
                    grads[a, i, p] = g
        return dict(leaf=leaf, modes=modes, terms=space.leaf_terms[li], pts=pts, vals=vals, grads=grads,
                    q=None, degs=degs)

    def surface_local_apply(self, c, xloc):
        """TestChannels(-du/dn + eta*u, -u*n) at every point (driver.jl:52-62), projected with
        the full tables (_accumulate_one_sided_apply_basis!, accumulators.jl:1133-1161)."""
        D = self.space.D
        u = c["vals"].T @ xloc
        g = np.stack([c["grads"][a].T @ xloc for a in range(D)])
        dn = sum(g[a] * c["normals"][:, a] for a in range(D))
        t0 = c["w"] * (-dn + c["eta"] * u)
        return c["vals"] @ t0 + sum(c["grads"][a] @ (-c["w"] * u * c["normals"][:, a]) for a in range(D))

    def _items(self):
        for c in self.cells:
            yield c, self.local_apply
        for c in self.surfaces:
            yield c, self.surface_local_apply

    # -- colouring (plans.jl:368-424) ------------------------------------------------
    def _colour(self):
        """One batch when all cells share a signature; greedy first-fit colours in batch order."""
        batches = OrderedDict()
        for ci, c in enumerate(self.cells):
            sig = (len(c["w"]), len(c["modes"]), tuple(len(t) for t in c["terms"]))
            batches.setdefault(sig, []).append(ci)
        order = []
        for items in batches.values():
            colour_sets, colour_items = [], []
            for ci in items:
                dofs = {d for t in self.cells[ci]["terms"] for (d, _) in t}
                for k, s in enumerate(colour_sets):
                    if not (s & dofs):
                        s |= dofs
                        colour_items[k].append(ci)
                        break
                else:
                    colour_sets.append(set(dofs))
                    colour_items.append([ci])
            order.append(colour_items)
        return order

    # -- Dirichlet (plans.jl:486-972) -----------------------------------------------
    def _dirichlet(self, dirichlet):
        if not dirichlet:
            return [], [], []
        space = self.space
        dom = space.domain
        D = space.D
        snap = space.snapshot
        faces = []
        for (leaf, axis, side) in snap.boundary:
            for (ax, sd, val) in dirichlet:
                if ax == axis and sd == side:
                    faces.append((leaf, axis, side, val))
        involved = sorted({d for (leaf, _, _, _) in faces
                           for t in space.leaf_terms[snap.leaf_to_index[leaf]] for (d, _) in t})
        pos = {d: i for i, d in enumerate(involved)}
        n = len(involved)
        G = np.zeros((n, n))
        rhs = np.zeros(n)
        for (leaf, axis, side, val) in faces:
            li = snap.leaf_to_index[leaf]
            a0 = axis - 1
            degs = space.degrees[li]
            q = space.qshape[li]
            rules = [gauss_legendre_rule(nq) for nq in q]
            face_q = [1 if b == a0 else q[b] for b in range(D)]
            face_det = 1.0
            for b in range(D):
                if b != a0:
                    face_det *= dom.cell_size(leaf, b)
            face_det = math.ldexp(face_det, -(D - 1))
            modes = space.leaf_modes[li]
            terms = space.leaf_terms[li]
            npts = int(np.prod(face_q))
            phi = np.zeros((npts, len(modes)))
            wts = np.zeros(npts)
            for p in range(npts):
                idx = mode_from_linear(p, tuple(nq - 1 for nq in face_q))
                wt = 1.0
                xi = []
                for b in range(D):
                    if b == a0:
                        xi.append(-1.0 if side == LOWER else 1.0)
                    else:
                        xi.append(rules[b][0][idx[b]])
                        wt *= rules[b][1][idx[b]]
                wts[p] = wt * face_det
                tables = [fe_basis_values_and_derivatives(xi[b], degs[b])[0] for b in range(D)]
                for i, m in enumerate(modes):
                    v = 1.0
                    for b in range(D):
                        v *= tables[b][m[b]]
                    phi[p, i] = v
            # face mass matrix and load, scattered through the term maps (plans.jl:563-612, 668-702)
            local_g = phi.T @ (wts[:, None] * phi)
            local_r = phi.T @ wts * val
            cols = sorted({pos[d] for t in terms for (d, _) in t})
            cpos = {c: k for k, c in enumerate(cols)}
            T = np.zeros((len(modes), len(cols)))
            for i, t in enumerate(terms):
                for (d, c) in t:
                    T[i, cpos[pos[d]]] += c
            ix = np.array(cols)
            G[np.ix_(ix, ix)] += T.T @ local_g @ T
            if val != 0.0:
                rhs[ix] += T.T @ local_r
        evals, evecs = sla.eigh(G, driver="evr")
        order = np.argsort(-evals, kind="stable")
        evals, evecs = evals[order], evecs[:, order]
        scale = np.max(np.abs(evals)) if n else 0.0
        tol = 0.0 if scale == 0 else 1000 * EPS * scale * max(n, 1)
        count = int(np.sum(evals > tol))
        if count == 0:
            return [], [], []
        C = evecs[:, :count].T.copy()
        targets = (evecs.T @ rhs)[:count] / evals[:count]
        _, _, perm = sla.qr(C, pivoting=True, mode="economic")
        pivcols = list(perm[:count])
        freecols = [c for c in range(n) if c not in set(pivcols)]
        P = C[:, pivcols]
        shift = np.linalg.solve(P, targets)
        fixed, fixed_vals, rows = [], [], []
        if freecols:
            coupling = -np.linalg.solve(P, C[:, freecols])
        for r in range(count):
            idx, co = [], []
            for k, fc in enumerate(freecols):
                if abs(coupling[r, k]) > tol:
                    idx.append(involved[fc])
                    co.append(float(coupling[r, k]))
            pivot = involved[pivcols[r]]
            if not idx:
                fixed.append(pivot)
                fixed_vals.append(float(shift[r]))
            else:
                rows.append((pivot, idx, co, float(shift[r])))
        perm2 = np.argsort(fixed, kind="stable")
        fixed = [fixed[i] for i in perm2]
        fixed_vals = [fixed_vals[i] for i in perm2]
        rows.sort(key=lambda r: r[0])
        return fixed, fixed_vals, rows

    # -- reduced map (assembly.jl:112-314) ------------------------------------------
    def _reduced_map(self):
        n = self.ndofs
        constrained = self.fixed_mask | self.blocked
        self.solve_dofs = [d for d in range(1, n + 1) if not constrained[d]]
        self.reduced_index = np.zeros(n + 1, dtype=np.int64)
        for i, d in enumerate(self.solve_dofs):
            self.reduced_index[d] = i + 1
        fixed_val = dict(zip(self.fixed, self.fixed_values))
        rows = {r[0]: r for r in self.rows}
        cache = {}

        def expand(d):
            if d in cache:
                return cache[d]
            if self.reduced_index[d] != 0:
                out = (0.0, {int(self.reduced_index[d]): 1.0})
            elif d in fixed_val:
                out = (fixed_val[d], {})
            elif d in rows:
                _, idx, co, rhs = rows[d]
                shift, red = rhs, {}
                for j, c in zip(idx, co):
                    s2, r2 = expand(j)
                    shift += c * s2
                    for k, v in r2.items():
                        red[k] = red.get(k, 0.0) + c * v
                out = (shift, red)
            else:
                out = (0.0, {})
            cache[d] = out
            return out

        self.shift = np.zeros(n + 1)
        self.P_rows = []
        for d in range(1, n + 1):
            s, red = expand(d)
            self.shift[d] = s
            self.P_rows.append(sorted(red.items()))

    # -- runtime (assembly.jl:540-564, 905-915; accumulators.jl:1022-1054) ----------
    def local_apply(self, c, xloc):
        w = c["w"]
        u = c["vals"].T @ xloc
        g = np.stack([c["grads"][a].T @ xloc for a in range(self.space.D)])
        kap = self.kappa * (np.array([self.kappa_fn(tuple(p)) for p in c["pts"]]) if self.kappa_fn else 1.0)
        t0 = w * self.mu * u
        tg = w * kap * g
        y = c["vals"] @ t0 + sum(c["grads"][a] @ tg[a] for a in range(self.space.D))
        return y

    def apply(self, x):
        """y = A x on the full layout (1-based arrays of length ndofs+1 are used internally)."""
        x1 = np.concatenate([[0.0], np.asarray(x, dtype=np.float64)])
        y1 = np.zeros(self.ndofs + 1)
        for colours in self.colors:
            for items in colours:
                for ci in items:
                    c = self.cells[ci]
                    xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
                    yloc = self.local_apply(c, xloc)
                    for i, t in enumerate(c["terms"]):
                        if yloc[i] == 0.0:
                            continue
                        for (d, cc) in t:
                            if self.fixed_mask[d] or self.blocked[d]:
                                continue
                            y1[d] += cc * yloc[i]
        for c in self.surfaces:
            xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
            yloc = self.surface_local_apply(c, xloc)
            for i, t in enumerate(c["terms"]):
                for (d, cc) in t:
                    if self.fixed_mask[d] or self.blocked[d]:
                        continue
                    y1[d] += cc * yloc[i]
        for it in self.interfaces:
            for side, yloc in zip(("minus", "plus"), self._interface_apply_sides(it, x1)):
                for i, t in enumerate(it[side]["terms"]):
                    for (d, cc) in t:
                        if self.fixed_mask[d] or self.blocked[d]:
                            continue
                        y1[d] += cc * yloc[i]
        for d in self.fixed:
            y1[d] = x1[d]
        for (pivot, idx, co, _) in self.rows:
            v = x1[pivot]
            for j, c in zip(idx, co):
                v -= c * x1[j]
            y1[pivot] = v
        return y1[1:]

    def _interface_apply_sides(self, it, x1):
        xm = np.array([sum(cc * x1[d] for (d, cc) in t) for t in it["minus"]["terms"]])
        xp = np.array([sum(cc * x1[d] for (d, cc) in t) for t in it["plus"]["terms"]])
        return self.interface_local_apply(it, xm, xp)

    def apply_physical(self, x):
        x1 = np.concatenate([[0.0], np.asarray(x, dtype=np.float64)])
        y1 = np.zeros(self.ndofs + 1)
        for c, fn in self._items():
            xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
            yloc = fn(c, xloc)
            for i, t in enumerate(c["terms"]):
                for (d, cc) in t:
                    y1[d] += cc * yloc[i]
        for it in self.interfaces:
            for side, yloc in zip(("minus", "plus"), self._interface_apply_sides(it, x1)):
                for i, t in enumerate(it[side]["terms"]):
                    for (d, cc) in t:
                        y1[d] += cc * yloc[i]
        return y1[1:]

    def expand(self, xr, include_shift=False):
        xf = np.zeros(self.ndofs)
        for d in range(1, self.ndofs + 1):
            v = self.shift[d] if include_shift else 0.0
            for (k, c) in self.P_rows[d - 1]:
                v += c * xr[k - 1]
            xf[d - 1] = v
        return xf

    def project(self, yf):
        yr = np.zeros(len(self.solve_dofs))
        for d in range(1, self.ndofs + 1):
            for (k, c) in self.P_rows[d - 1]:
                yr[k - 1] += c * yf[d - 1]
        return yr

    def reduced_apply(self, xr):
        return self.project(self.apply_physical(self.expand(xr)))

    def physical_diagonal(self):
        """cell_diagonal! basis probe + coefficient-squared scatter (accumulators.jl:1056-1083,
        assembly.jl:1811-1825)."""
        out = np.zeros(self.ndofs + 1)
        D = self.space.D
        for c in self.cells:
            kap = self.kappa * (np.array([self.kappa_fn(tuple(p)) for p in c["pts"]]) if self.kappa_fn else 1.0)
            diag = c["vals"] ** 2 @ (c["w"] * self.mu) + sum((c["grads"][a] ** 2) @ (c["w"] * kap) for a in range(D))
            for i, t in enumerate(c["terms"]):
                for (d, cc) in t:
                    out[d] += cc * cc * diag[i]
        for c in self.surfaces:
            dn = sum(c["grads"][a] * c["normals"][:, a][None, :] for a in range(D))
            diag = (c["eta"] * c["vals"] ** 2 - 2.0 * c["vals"] * dn) @ c["w"]
            for i, t in enumerate(c["terms"]):
                for (d, cc) in t:
                    out[d] += cc * cc * diag[i]
        for it in self.interfaces:  # interface_diagonal!, sine_poisson_sipg.jl:97-123
            a = it["axis"]
            for side, sign in (("minus", 1.0), ("plus", -1.0)):
                c = it[side]
                diag = (it["sigma"] * c["vals"] ** 2 - sign * c["vals"] * c["grads"][a]) @ it["w"]
                for i, t in enumerate(c["terms"]):
                    for (d, cc) in t:
                        out[d] += cc * cc * diag[i]
        return out[1:]

    def reduced_diagonal(self):
        """Direct copy when the map is an injection, else None (assembly.jl:662-726)."""
        for c in self.cells + self.surfaces + [it[s] for it in self.interfaces for s in ("minus", "plus")]:
            for t in c["terms"]:
                if len(t) != 1:
                    return None
        pd = self.physical_diagonal()
        return np.array([pd[d - 1] for d in self.solve_dofs])

    def probe_reduced_diagonal(self):
        """One reduced apply per unit vector (solve.jl:722-738) — the reference's fallback when
        the reduced map is not a direct injection."""
        n = len(self.solve_dofs)
        out = np.zeros(n)
        e = np.zeros(n)
        for i in range(n):
            e[i] = 1.0
            out[i] = self.reduced_apply(e)[i]
            e[i] = 0.0
        return out

    def jacobi_diagonal(self):
        """_jacobi_inverse_diagonal's diagonal (solve.jl:713-720): local kernels, else probing."""
        d = self.reduced_diagonal()
        return d if d is not None else self.probe_reduced_diagonal()

    def rhs_physical(self):
        out = np.zeros(self.ndofs + 1)
        D = self.space.D
        for c in self.cells:
            if self.source is None:
                break
            f = np.array([self.source(tuple(p)) for p in c["pts"]])
            loc = c["vals"] @ (c["w"] * f)
            for i, t in enumerate(c["terms"]):
                if loc[i] == 0.0:
                    continue
                for (d, cc) in t:
                    out[d] += cc * loc[i]
        for c in self.surfaces:
            if c["g"] is None:
                continue
            g = np.array([c["g"](tuple(p)) for p in c["pts"]])
            # TestChannels(eta*g, -g*n) (driver.jl:65-76)
            loc = c["vals"] @ (c["w"] * c["eta"] * g) + sum(c["grads"][a] @ (-c["w"] * g * c["normals"][:, a])
                                                            for a in range(D))
            for i, t in enumerate(c["terms"]):
                for (d, cc) in t:
                    out[d] += cc * loc[i]
        return out[1:]

    def reduced_rhs(self):
        b = self.rhs_physical()
        if np.any(self.shift[1:] != 0.0):
            b = b - self.apply_physical(self.shift[1:])
        return self.project(b)


def cg_solve(apply_fn, b, precond=None, rtol=1e-10, atol=0.0, maxiter=10000, raise_unconverged=True):
    """PCG with the unpreconditioned stop rule (solve.jl:376-431).  After maxiter iterations
    without convergence it raises, as the reference does (solve.jl:430), or with
    raise_unconverged=False returns the last iterate."""
    n = len(b)
    x = np.zeros(n)
    r = b.copy()
    z = precond(r) if precond else r.copy()
    p = z.copy()
    rz = float(np.dot(r, z))
    tol = max(atol, rtol * math.sqrt(float(np.dot(b, b))))
    if float(np.dot(r, r)) <= tol * tol:
        return x, 0
    for it in range(1, maxiter + 1):
        ap = apply_fn(p)
        den = float(np.dot(p, ap))
        if not den > 0:
            raise ValueError("CG encountered a non-positive operator direction")
        alpha = rz / den
        x += alpha * p
        r -= alpha * ap
        if float(np.dot(r, r)) <= tol * tol:
            return x, it
        z = precond(r) if precond else r.copy()
        rz_new = float(np.dot(r, z))
        beta = rz_new / rz
        p = z + beta * p
        rz = rz_new
    if not raise_unconverged:
        return x, maxiter
    raise ValueError("CG did not converge")


def fgmres_solve(apply_fn, b, precond=None, restart=30, rtol=1e-10, atol=0.0, maxiter=10000, raise_unconverged=True):
    """Right-preconditioned flexible GMRES(restart) with modified Gram-Schmidt, restated from
    `_fgmres_solve` (solve.jl:433-542): Givens rotations on each new Hessenberg column
    (`_apply_previous_givens_rotations!`, `_givens_rotation`, `_apply_givens_rotation!`,
    solve.jl:544-576), the cycle ends when |g[j+1]| <= tol or the Arnoldi norm is zero, and
    `_finish_fgmres_cycle!` (solve.jl:578-589) back-substitutes (`_upper_triangular_solve!`,
    solve.jl:591-614), adds Z y to x and recomputes the true residual b - A x.
    Returns (x, total inner iterations); after maxiter without convergence it raises, as the
    reference does (solve.jl:541), or with raise_unconverged=False returns the last iterate."""
    n = len(b)
    x = np.zeros(n)
    r = np.array(b, dtype=np.float64, copy=True)
    bnorm = math.sqrt(float(np.dot(b, b)))
    tol = max(atol, rtol * bnorm)
    if math.sqrt(float(np.dot(r, r))) <= tol:
        return x, 0
    m = min(restart, n)
    total = 0

    def finish(H, g, Z, count):
        y = np.zeros(count)
        for row in range(count - 1, -1, -1):
            v = g[row]
            for col in range(row + 1, count):
                v -= H[row, col] * y[col]
            d = H[row, row]
            if not math.isfinite(d):
                raise ValueError("FGMRES encountered a non-finite Krylov least-squares diagonal")
            if d == 0.0:
                raise ValueError("FGMRES encountered a singular Krylov least-squares problem")
            y[row] = v / d
        xn = x
        for col in range(count):
            if y[col] != 0.0:
                xn = xn + y[col] * Z[:, col]
        return xn, b - apply_fn(xn)

    while total < maxiter:
        V = np.zeros((n, m + 1))
        Z = np.zeros((n, m))
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        cs = np.zeros(m)
        sn = np.zeros(m)
        beta = math.sqrt(float(np.dot(r, r)))
        if beta <= tol:
            return x, total
        V[:, 0] = r / beta
        g[0] = beta
        inner_limit = min(m, maxiter - total)
        inner = 0
        updated = False
        for j in range(inner_limit):
            total += 1
            inner = j + 1
            Z[:, j] = precond(V[:, j]) if precond else V[:, j]
            w = apply_fn(Z[:, j])
            for i in range(j + 1):
                H[i, j] = float(np.dot(w, V[:, i]))
                w = w - H[i, j] * V[:, i]
            nrm = math.sqrt(float(np.dot(w, w)))
            H[j + 1, j] = nrm
            if nrm > 0.0:
                V[:, j + 1] = w / nrm
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j] = cs[i] * a + sn[i] * c
                H[i + 1, j] = -sn[i] * a + cs[i] * c
            scale = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if scale == 0.0 else (H[j, j] / scale, H[j + 1, j] / scale)
            a, c = H[j, j], H[j + 1, j]
            H[j, j] = cs[j] * a + sn[j] * c
            H[j + 1, j] = -sn[j] * a + cs[j] * c
            a, c = g[j], g[j + 1]
            g[j] = cs[j] * a + sn[j] * c
            g[j + 1] = -sn[j] * a + cs[j] * c
            if abs(g[j + 1]) <= tol or nrm == 0.0:
                x, r = finish(H, g, Z, j + 1)
                if math.sqrt(float(np.dot(r, r))) <= tol:
                    return x, total
                updated = True
                break
        if inner == 0:
            raise ValueError("FGMRES failed to build a Krylov update")
        if not updated:
            x, r = finish(H, g, Z, inner)
        if math.sqrt(float(np.dot(r, r))) <= tol:
            return x, total
    if not raise_unconverged:
        return x, total
    raise ValueError("FGMRES did not converge")


def power_iteration_start(n, level):
    """Start vector of the lambda_max(D^-1 A) estimate used for the Chebyshev smoother: a
    xorshift64 stream seeded with 0x9e3779b97f4a7c15 + level, v_i = 0.5 + (s mod 1000003) /
    1000003.  Project-defined (the reference has no Chebyshev smoother)."""
    mask = (1 << 64) - 1
    s = (0x9E3779B97F4A7C15 + level) & mask
    v = np.empty(n)
    for i in range(n):
        s ^= (s << 13) & mask
        s ^= s >> 7
        s ^= (s << 17) & mask
        v[i] = 0.5 + float(s % 1000003) / 1000003.0
    return v


def estimate_lambda_max(apply_fn, dinv, level, iterations=20):
    """Power iteration on D^-1 A: x_0 from `power_iteration_start`, t = D^-1 A x,
    lambda = ||t|| / ||x||, x = t / ||t||; 20 steps.  Project-defined estimate."""
    x = power_iteration_start(len(dinv), level)
    lam = 0.0
    for _ in range(iterations):
        t = dinv * apply_fn(x)
        tn, xn = math.sqrt(float(np.dot(t, t))), math.sqrt(float(np.dot(x, x)))
        if not (tn > 0.0 and xn > 0.0):
            break
        lam = tn / xn
        x = t / tn
    return lam


def bratu_residual(plan: Plan, x_full, lam, source=None):
    """Full-layout residual of the accumulator of examples/nonlinear_bratu/driver.jl:39-45:
    value channel lam exp(u) - f, gradient channel kappa grad u, on every cell rule; constraint
    rows are not written (the reduced residual projects them away)."""
    D = plan.space.D
    x1 = np.concatenate([[0.0], np.asarray(x_full, dtype=np.float64)])
    y1 = np.zeros(plan.ndofs + 1)
    for c in plan.cells:
        xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
        u = c["vals"].T @ xloc
        g = [c["grads"][a].T @ xloc for a in range(D)]
        f = np.array([source(tuple(p)) for p in c["pts"]]) if source else 0.0
        yloc = c["vals"] @ (c["w"] * (lam * np.exp(u) - f)) + sum(c["grads"][a] @ (c["w"] * plan.kappa * g[a])
                                                                for a in range(D))
        for i, t in enumerate(c["terms"]):
            for (d, cc) in t:
                y1[d] += cc * yloc[i]
    return y1[1:]


def bratu_tangent(plan: Plan, x_full, dx_full, lam):
    """Tangent action of the same accumulator (driver.jl:48-54): value channel lam exp(u) du,
    gradient channel kappa grad du."""
    D = plan.space.D
    x1 = np.concatenate([[0.0], np.asarray(x_full, dtype=np.float64)])
    d1 = np.concatenate([[0.0], np.asarray(dx_full, dtype=np.float64)])
    y1 = np.zeros(plan.ndofs + 1)
    for c in plan.cells:
        xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
        dloc = np.array([sum(cc * d1[d] for (d, cc) in t) for t in c["terms"]])
        u = c["vals"].T @ xloc
        du = c["vals"].T @ dloc
        g = [c["grads"][a].T @ dloc for a in range(D)]
        yloc = c["vals"] @ (c["w"] * lam * np.exp(u) * du) + sum(c["grads"][a] @ (c["w"] * plan.kappa * g[a])
                                                                  for a in range(D))
        for i, t in enumerate(c["terms"]):
            for (d, cc) in t:
                y1[d] += cc * yloc[i]
    return y1[1:]


def bratu_newton(plan: Plan, lam, source=None, rtol=1e-10, atol=1e-10, maxiter=10):
    """Newton on the reduced space with exact (dense) tangent solves (solve.jl:277-333)."""
    n = len(plan.solve_dofs)
    ur = np.zeros(n)
    r0 = None
    for it in range(maxiter + 1):
        x = plan.expand(ur, include_shift=True)
        r = plan.project(bratu_residual(plan, x, lam, source))
        rn = float(np.linalg.norm(r))
        r0 = rn if r0 is None else r0
        if rn <= max(atol, rtol * r0):
            return ur, it
        if it == maxiter:
            break
        J = np.zeros((n, n))
        for j in range(n):
            e = np.zeros(n)
            e[j] = 1.0
            J[:, j] = plan.project(bratu_tangent(plan, x, plan.expand(e), lam))
        ur = ur + np.linalg.solve(J, -r)
    raise ValueError("Newton solve did not converge")


def l2_error(plan: Plan, full_values, exact):
    """Cell quadrature L2 error (verification.jl:201-230)."""
    x1 = np.concatenate([[0.0], np.asarray(full_values)])
    err2 = 0.0
    for c in plan.cells:
        xloc = np.array([sum(cc * x1[d] for (d, cc) in t) for t in c["terms"]])
        u = c["vals"].T @ xloc
        ex = np.array([exact(tuple(p)) for p in c["pts"]])
        err2 += float(np.sum(c["w"] * (u - ex) ** 2))
    return math.sqrt(err2)


# ---------------------------------------------------------------------------
# hp geometric multigrid: src/multigrid.jl
# ---------------------------------------------------------------------------

def coarsened_degree(degree, lower, sequence="bisect"):
    """multigrid.jl:470-499"""
    if degree <= lower:
        return degree
    if sequence == "bisect":
        return max(degree // 2, lower)
    if sequence == "decrease_by_one":
        return max(degree - 1, lower)
    return lower


def hp_multigrid_levels(space: Space, min_degree=1, max_levels=16, sequence="bisect"):
    """Coarse-to-fine list of (leaves, {leaf: degrees}) (multigrid.jl:443-469, 514-586)."""
    cg = space.continuity == "cg"
    grid = space.grid
    leaves = list(space.snapshot.leaves)
    degs = {leaf: tuple(space.degrees[i]) for i, leaf in enumerate(leaves)}
    levels = [(leaves, dict(degs))]
    while len(levels) < max_levels:
        nd = {}
        for leaf, d in degs.items():
            nd[leaf] = tuple(coarsened_degree(v, min(v, max(min_degree, 1 if cg else 0)), sequence) for v in d)
        if nd == degs:
            break
        degs = nd
        levels.append((leaves, dict(degs)))
    while len(levels) < max_levels:
        active = set(leaves)
        cands = []
        for cell in range(1, grid.stored() + 1):
            f = grid.first_child[cell]
            if f and f in active and (f + 1) in active:
                cands.append(cell)
        if not cands:
            break
        child_to_parent = {}
        for c in cands:
            f = grid.first_child[c]
            child_to_parent[f] = c
            child_to_parent[f + 1] = c
            degs[c] = tuple(min(a, b) for a, b in zip(degs[f], degs[f + 1]))
            del degs[f]
            del degs[f + 1]
        new, emitted = [], set()
        for leaf in leaves:
            p = child_to_parent.get(leaf)
            if p is None:
                new.append(leaf)
            elif p not in emitted:
                emitted.add(p)
                new.append(p)
        leaves = morton_ordered_leaves(grid, new)
        levels.append((leaves, dict(degs)))
    levels.reverse()
    return levels


def multigrid_transfer(coarse: Plan, fine: Plan):
    """Reduced prolongation entries {(coarse_red, fine_red): value}, 1-based reduced indices
    (multigrid.jl:614-848)."""
    cs, fs = coarse.space, fine.space
    grid = cs.grid
    D = cs.D
    fine_index = fs.snapshot.leaf_to_index
    entries = {}
    cred = {d: coarse.P_rows[d - 1] for d in range(1, coarse.ndofs + 1)}
    for ci, cleaf in enumerate(cs.snapshot.leaves):
        if cleaf in fine_index:
            fines = [cleaf]
        else:
            f = grid.first_child[cleaf]
            fines = [f, f + 1]
        for fleaf in fines:
            fi = fine_index[fleaf]
            mats = []
            for a in range(D):
                delta = grid.level(fleaf, a) - grid.level(cleaf, a)
                rel = grid.coord(fleaf, a) - (grid.coord(cleaf, a) << delta)
                mats.append(affine_restriction_matrix(cs.degrees[ci][a], fs.degrees[fi][a], delta, rel))
            target = {}
            for cm, cterms in zip(cs.leaf_modes[ci], cs.leaf_terms[ci]):
                source = {}
                for (d, c) in cterms:
                    for (r, pc) in cred[d]:
                        source[r] = source.get(r, 0.0) + c * pc
                for fm in fs.leaf_modes[fi]:
                    coef = 1.0
                    for a in range(D):
                        coef *= mats[a][fm[a], cm[a]]
                    if coef == 0.0:
                        continue
                    tv = target.setdefault(fm, {})
                    for r, v in source.items():
                        if coef * v != 0.0:
                            tv[r] = tv.get(r, 0.0) + coef * v
            for fm, tv in target.items():
                terms = fs.leaf_terms[fi][fs.leaf_modes[fi].index(fm)]
                if len(terms) != 1:
                    continue
                d, c = terms[0]
                rf = int(fine.reduced_index[d])
                if rf == 0:
                    continue
                for r, v in tv.items():
                    val = (1.0 / c) * v
                    if val == 0.0:
                        continue
                    key = (r, rf)
                    if key in entries:
                        old = entries[key]
                        assert abs(old - val) <= 10000 * EPS * max(1.0, abs(old), abs(val))
                    else:
                        entries[key] = val
    return entries


class Multigrid:
    """V-cycle with damped Jacobi smoothing and a dense Cholesky coarse solve
    (multigrid.jl:858-956, common.jl:272-330).  `smoother="chebyshev"` adds the project's
    Chebyshev-Jacobi smoother (no reference counterpart): `chebyshev_degree` steps of the
    Chebyshev semi-iteration for D^-1 A (Y. Saad, Iterative Methods for Sparse Linear Systems,
    2nd ed., Algorithm 12.1) on [lambda_max / chebyshev_range, 1.2 lambda_max], lambda_max from
    `estimate_lambda_max` on every level above the coarsest."""

    def __init__(self, plans, pre=2, post=2, omega=0.8, smoother="jacobi", restart=8, chebyshev_degree=2,
                 chebyshev_range=15.0):
        self.plans = plans
        self.pre, self.post, self.omega = pre, post, omega
        if smoother not in ("jacobi", "gmres", "chebyshev"):
            raise ValueError("smoother must be jacobi, gmres or chebyshev")
        self.chebyshev_degree, self.chebyshev_lower = chebyshev_degree, 1.0 / chebyshev_range
        if smoother == "gmres" and max(pre, post) > restart:
            raise ValueError("GMRES smoother requires restart >= max(pre, post)")  # multigrid.jl:352-358
        self.smoother, self.restart = smoother, restart
        self.transfers = [multigrid_transfer(plans[i], plans[i + 1]) for i in range(len(plans) - 1)]
        self.P = []
        for i, ent in enumerate(self.transfers):
            M = np.zeros((len(plans[i + 1].solve_dofs), len(plans[i].solve_dofs)))
            for (rc, rf), v in ent.items():
                M[rf - 1, rc - 1] = v
            self.P.append(M)
        self.dinv = [1.0 / p.jacobi_diagonal() for p in plans]
        c = plans[0]
        n0 = len(c.solve_dofs)
        A0 = np.zeros((n0, n0))
        for j in range(n0):
            e = np.zeros(n0)
            e[j] = 1.0
            A0[:, j] = c.reduced_apply(e)
        self.L0 = np.linalg.cholesky(A0)
        self.lmax = [0.0] * len(plans)
        if smoother == "chebyshev":
            for lv in range(1, len(plans)):
                self.lmax[lv] = estimate_lambda_max(plans[lv].reduced_apply, self.dinv[lv], lv)

    def smooth_chebyshev(self, level, x, b, steps):
        """Saad's Algorithm 12.1 with the Jacobi preconditioner: theta, delta the centre and
        half width of [lmin, lmax]; d_0 = D^-1 r / theta, d_k = rho_k rho_{k-1} d_{k-1} +
        (2 rho_k / delta) D^-1 r, rho_k = 1 / (2 theta/delta - rho_{k-1}); x += d_k."""
        p = self.plans[level]
        lmax = 1.2 * self.lmax[level]
        lmin = lmax * self.chebyshev_lower
        theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sigma = theta / delta
        d = np.zeros_like(x)
        for _ in range(steps):
            rho_old = 1.0 / sigma
            for k in range(self.chebyshev_degree):
                z = self.dinv[level] * (b - p.reduced_apply(x))
                if k == 0:
                    d = (1.0 / theta) * z
                else:
                    rho = 1.0 / (2.0 * sigma - rho_old)
                    d = (rho * rho_old) * d + (2.0 * rho / delta) * z
                    rho_old = rho
                x = x + d
        return x

    def smooth(self, level, x, b, steps):
        p = self.plans[level]
        if self.smoother == "gmres":
            return self.smooth_gmres(level, x, b, steps)
        if self.smoother == "chebyshev":
            return self.smooth_chebyshev(level, x, b, steps)
        for _ in range(steps):
            r = b - p.reduced_apply(x)
            x = x + self.omega * self.dinv[level] * r
        return x

    def smooth_gmres(self, level, x, b, steps):
        """Fixed-step right-Jacobi-preconditioned GMRES smoother (multigrid.jl:963-1056):
        `count` Arnoldi steps with modified Gram-Schmidt, Givens rotations on the Hessenberg
        columns (solve.jl:544-576), back substitution, x += omega * Z y."""
        if steps == 0:
            return x
        p = self.plans[level]
        r = b - p.reduced_apply(x)
        beta = math.sqrt(float(np.dot(r, r)))
        if beta == 0.0:
            return x
        n = len(b)
        count = min(steps, self.restart, n)
        if count == 0:
            return x
        V = np.zeros((n, count + 1))
        Z = np.zeros((n, count))
        H = np.zeros((count + 1, count))
        g = np.zeros(count + 1)
        cs = np.zeros(count)
        sn = np.zeros(count)
        V[:, 0] = r / beta
        g[0] = beta
        inner = 0
        for j in range(count):
            inner = j + 1
            Z[:, j] = self.dinv[level] * V[:, j]
            w = p.reduced_apply(Z[:, j])
            for i in range(j + 1):
                H[i, j] = float(np.dot(w, V[:, i]))
                w = w - H[i, j] * V[:, i]
            nrm = math.sqrt(float(np.dot(w, w)))
            H[j + 1, j] = nrm
            if nrm > 0.0:
                V[:, j + 1] = w / nrm
            for i in range(j):
                a, c = H[i, j], H[i + 1, j]
                H[i, j] = cs[i] * a + sn[i] * c
                H[i + 1, j] = -sn[i] * a + cs[i] * c
            scale = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if scale == 0.0 else (H[j, j] / scale, H[j + 1, j] / scale)
            a, c = H[j, j], H[j + 1, j]
            H[j, j] = cs[j] * a + sn[j] * c
            H[j + 1, j] = -sn[j] * a + cs[j] * c
            a, c = g[j], g[j + 1]
            g[j] = cs[j] * a + sn[j] * c
            g[j + 1] = -sn[j] * a + cs[j] * c
            if nrm == 0.0:
                break
        y = np.zeros(inner)
        for row in range(inner - 1, -1, -1):
            v = g[row] - sum(H[row, col] * y[col] for col in range(row + 1, inner))
            if not math.isfinite(H[row, row]) or H[row, row] == 0.0:
                raise ValueError("GMRES smoother: singular Krylov least-squares problem")
            y[row] = v / H[row, row]
        for j in range(inner):
            if self.omega * y[j] != 0.0:
                x = x + (self.omega * y[j]) * Z[:, j]
        return x

    def vcycle(self, level, b):
        if level == 0:
            y = np.linalg.solve(self.L0, b)
            return np.linalg.solve(self.L0.T, y)
        x = np.zeros_like(b)
        x = self.smooth(level, x, b, self.pre)
        r = b - self.plans[level].reduced_apply(x)
        bc = self.P[level - 1].T @ r
        xc = self.vcycle(level - 1, bc)
        x = x + self.P[level - 1] @ xc
        return self.smooth(level, x, b, self.post)

    def apply(self, r):
        return self.vcycle(len(self.plans) - 1, r)


# ---------------------------------------------------------------------------
# Finite cells and embedded surfaces: src/regions.jl, src/embedded.jl
# ---------------------------------------------------------------------------

def classifier_value(classifier, x):
    """regions.jl:819-830; `classifier` takes an [n, D] array (one row here)."""
    v = classifier(np.asarray(x, dtype=np.float64).reshape(1, -1))
    v = np.asarray(v).reshape(-1)[0]
    if isinstance(v, (bool, np.bool_)):
        return -1.0 if v else 1.0
    v = float(v)
    if not math.isfinite(v):
        raise ValueError("finite-cell classifier values must be finite")
    return v


def map_from_biunit_cube(dom: Domain, leaf, xi):
    """center + xi * half per axis (geometry.jl:571-578)."""
    out = []
    for a in range(dom.D):
        c, h = dom.center_half(leaf, a)
        out.append(c + xi[a] * h)
    return out


def _subcell_corner(lower, upper, mask):
    """regions.jl:424-427"""
    return [upper[a] if (mask >> a) & 1 else lower[a] for a in range(len(lower))]


def classify_subcell(dom: Domain, leaf, classifier, lower, upper):
    """regions.jl:736-757: corners then centre; 'outside' / 'inside' / 'cut'."""
    D = dom.D
    neg = pos = False
    for mask in range(1 << D):
        v = classifier_value(classifier, map_from_biunit_cube(dom, leaf, _subcell_corner(lower, upper, mask)))
        neg |= v < 0.0
        pos |= v > 0.0
    center = [0.5 * (lower[a] + upper[a]) for a in range(D)]
    v = classifier_value(classifier, map_from_biunit_cube(dom, leaf, center))
    neg |= v < 0.0
    pos |= v > 0.0
    if not neg:
        return "outside"
    if not pos:
        return "inside"
    return "cut"


def classify_leaf(dom: Domain, leaf, classifier):
    D = dom.D
    return classify_subcell(dom, leaf, classifier, [-1.0] * D, [1.0] * D)


def physical_active_leaves(dom: Domain, classifier):
    """regions.jl:267-279"""
    leaves = [l for l in dom.grid.active_leaves() if classify_leaf(dom, l, classifier) != "outside"]
    if not leaves:
        raise ValueError("physical domains must contain at least one active physical leaf")
    return leaves


def _tensor_points(qshape):
    """TensorQuadrature points and weights, axis 1 fastest (quadrature.jl:219-226)."""
    D = len(qshape)
    rules = [gauss_legendre_rule(q) for q in qshape]
    pts, wts = [], []
    for p in range(int(np.prod(qshape))):
        idx = mode_from_linear(p, tuple(q - 1 for q in qshape))
        pts.append([rules[a][0][idx[a]] for a in range(D)])
        w = 1.0
        for a in range(D):
            w *= rules[a][1][idx[a]]
        wts.append(w)
    return pts, wts


def _append_subcell_quadrature(points, weights, dom, leaf, classifier, base, lower, upper, filter_points):
    """regions.jl:759-792 plus the sliver fallback of regions.jl:794-817."""
    D = dom.D
    center = [0.5 * (lower[a] + upper[a]) for a in range(D)]
    half = [0.5 * (upper[a] - lower[a]) for a in range(D)]
    scale = 1.0
    for a in range(D):
        scale *= half[a]
    appended = False
    for eta, w in zip(*base):
        xi = [center[a] + half[a] * eta[a] for a in range(D)]
        if filter_points and not classifier_value(classifier, map_from_biunit_cube(dom, leaf, xi)) < 0.0:
            continue
        points.append(xi)
        weights.append(w * scale)
        appended = True
    if filter_points and not appended:
        total = (1 << D) + 1
        vol = 1.0
        for a in range(D):
            vol *= upper[a] - lower[a]
        sw = vol / total
        if classifier_value(classifier, map_from_biunit_cube(dom, leaf, center)) < 0.0:
            points.append(center)
            weights.append(sw)
        for mask in range(1 << D):
            xi = _subcell_corner(lower, upper, mask)
            if classifier_value(classifier, map_from_biunit_cube(dom, leaf, xi)) < 0.0:
                points.append(xi)
                weights.append(sw)


def _collect_candidates(points, weights, dom, leaf, classifier, base, lower, upper, depth, max_depth):
    """regions.jl:477-510 (depth-first, child masks in increasing order)."""
    cls = classify_subcell(dom, leaf, classifier, lower, upper)
    if cls == "inside":
        _append_subcell_quadrature(points, weights, dom, leaf, classifier, base, lower, upper, False)
        return
    if cls == "outside":
        return
    if depth >= max_depth:
        _append_subcell_quadrature(points, weights, dom, leaf, classifier, base, lower, upper, True)
        return
    D = dom.D
    mid = [0.5 * (lower[a] + upper[a]) for a in range(D)]
    for mask in range(1 << D):
        cl = [mid[a] if (mask >> a) & 1 else lower[a] for a in range(D)]
        cu = [upper[a] if (mask >> a) & 1 else mid[a] for a in range(D)]
        _collect_candidates(points, weights, dom, leaf, classifier, base, cl, cu, depth + 1, max_depth)


def finite_cell_candidates(dom: Domain, leaf, qshape, classifier, max_depth):
    """Unfitted candidate rule of one leaf: None outside, the tensor rule inside, the octree
    candidates when cut (regions.jl:297-322 before the moment fit)."""
    D = dom.D
    cls = classify_leaf(dom, leaf, classifier)
    if cls == "outside":
        return None
    base = _tensor_points(qshape)
    if cls == "inside":
        return np.array(base[0]), np.array(base[1])
    points, weights = [], []
    _collect_candidates(points, weights, dom, leaf, classifier, base, [-1.0] * D, [1.0] * D, 0, max_depth)
    if not points:
        return None
    return np.array(points), np.array(weights)


def physical_surface_data(dom: Domain, leaf, ref_weights, ref_normals):
    """integration.jl:2501-2516: w * det(J) / |J n|, J^-1 n / |J^-1 n| for diagonal J."""
    D = dom.D
    J = [0.5 * dom.cell_size(leaf, a) for a in range(D)]
    det = 1.0
    for a in range(D):
        det *= J[a]
    ws, ns = [], []
    for w, n in zip(ref_weights, ref_normals):
        mapped = math.sqrt(sum((J[a] * n[a]) ** 2 for a in range(D)))
        ws.append(w * det / mapped)
        t = [n[a] / J[a] for a in range(D)]
        mag = math.sqrt(sum(v * v for v in t))
        ns.append([v / mag for v in t])
    return np.array(ws), np.array(ns)

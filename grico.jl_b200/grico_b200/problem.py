"""Problems, accumulator forms, compile and the runtime calls (host side of the mirror).

Mirrors `ScalarField`, `AffineProblem`, `add_cell_accumulator!`, `Dirichlet`/`BoundaryFace`,
`add_constraint!`, `compile`, `apply`/`apply!`, `rhs` and `solve` (problem.jl:47-612,
plans.jl:170-231, assembly.jl:456-564, solve.jl:219-266).

Julia accumulator callbacks cannot run on the GPU, so cell operators are a closed set of form
descriptors: `Diffusion`, `MassDiffusion`, `Mass`, `VariableDiffusion` (pointwise coefficient
tabulated at the quadrature points) and `Load` (right-hand side f(x)).  Any other operator
object raises GricoError(GRICO_ERR_UNSUPPORTED_FORM), like the reference raises ArgumentError.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from .mesh import LOWER, UPPER


# ---------------------------------------------------------------------------------------
# forms
# ---------------------------------------------------------------------------------------

class Diffusion:
    """TestChannels(0, kappa*grad u) — examples/poisson_matrix_free_gmg/driver.jl:36-38."""

    def __init__(self, kappa=1.0):
        self.mass, self.kappa, self.coefficient = 0.0, float(kappa), None


class MassDiffusion:
    """TestChannels(mass*u, kappa*grad u) — benchmark/hpmg_scaling.jl:23-25."""

    def __init__(self, mass=1.0, kappa=1.0):
        self.mass, self.kappa, self.coefficient = float(mass), float(kappa), None


class Mass:
    def __init__(self, mass=1.0):
        self.mass, self.kappa, self.coefficient = float(mass), 0.0, None


class VariableDiffusion:
    """TestChannels(mass*u, kappa*a(x) grad u) with a(x) tabulated at the quadrature points.
    `coefficient(points)` receives an [n, D] array and returns [n] values."""

    def __init__(self, coefficient, kappa=1.0, mass=0.0):
        self.mass, self.kappa, self.coefficient = float(mass), float(kappa), coefficient


class Load:
    """cell_rhs_accumulate returning f(x) — `source(points)` on an [n, D] array."""

    def __init__(self, source):
        self.source = source


class SIPG:
    """Symmetric interior-penalty DG Poisson terms (benchmark/sine_poisson_sipg.jl:24-157), as an
    interface operator (`add_interface`) and as a boundary operator (`add_boundary`):
    interior  -{du/dn}[v] - {dv/dn}[u] + sigma [u][v],  [w] = w- - w+, n from minus to plus,
              sigma = penalty (max(p-, p+) + 1)^2 / (2 h- h+ / (h- + h+)) along the face axis;
    boundary  -v du/dn - u dv/dn + sigma u v,  sigma = penalty (p + 1)^2 / h, with the load
              TestChannels(sigma g, -g n) when `data` is given (g = 0 otherwise)."""

    def __init__(self, penalty, data=None):
        self.penalty = float(penalty)
        if not self.penalty >= 0.0:
            raise ValueError("penalty must be non-negative")
        self.data = data


class Nitsche:
    """Symmetric Nitsche Dirichlet data u = g on boundary faces or embedded surfaces
    (examples/annular_nitsche_fcm/driver.jl:45-76): bilinear TestChannels(-du/dn + eta*u, -u*n),
    right-hand side TestChannels(eta*g, -g*n), eta = penalty / min(cell_size).  `data(points)`
    returns g on an [n, D] array (None: g = 0)."""

    def __init__(self, penalty, data=None):
        self.penalty = float(penalty)
        if not self.penalty >= 0.0:
            raise ValueError("penalty must be non-negative")
        self.data = data


# ---------------------------------------------------------------------------------------
# fields, constraints, problems
# ---------------------------------------------------------------------------------------

class ScalarField:
    def __init__(self, space, name="u"):
        self.space = space
        self.name = name


class BoundaryFace:
    def __init__(self, axis, side):
        if side not in (LOWER, UPPER):
            raise ValueError("side must be LOWER or UPPER")
        self.axis, self.side = int(axis), int(side)


class Dirichlet:
    """Strong Dirichlet data on one boundary face; constant values only on the GPU path."""

    def __init__(self, field, boundary, data):
        self.field, self.boundary = field, boundary
        if callable(data):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "Dirichlet data must be a constant on the B200 path")
        self.value = float(data)


class SPD:
    pass


class NonsymmetricOperator:
    pass


class AffineProblem:
    def __init__(self, field, operator_class=None):
        self.field = field
        self.operator_class = operator_class or SPD()
        self.cell_operators = []
        self.rhs_operators = []
        self.dirichlet = []
        self.surface_operators = []        # bilinear Nitsche forms on embedded surfaces
        self.surface_rhs_operators = []
        self.boundary_operators = []       # (BoundaryFace, Nitsche or SIPG)
        self.interface_operators = []      # SIPG on every interior interface
        self.boundary_rhs_operators = []
        self.surfaces = []                 # SurfaceQuadrature attachments
        self.cell_quadratures = {}         # leaf -> (reference points, reference weights)


def add_cell_accumulator(problem, test_field, *args):
    """add_cell_accumulator!(problem, test, trial, op) or (problem, test, load) (accumulators.jl:356-370)."""
    if len(args) == 2:
        trial, op = args
        if trial is not test_field or test_field is not problem.field:
            raise ValueError("the B200 plan supports one scalar field")
        if not isinstance(op, (Diffusion, MassDiffusion, Mass, VariableDiffusion)):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"accumulator form {type(op).__name__} is not supported by the GPU plan")
        problem.cell_operators.append(op)
    elif len(args) == 1:
        (op,) = args
        if not isinstance(op, Load):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"rhs form {type(op).__name__} is not supported by the GPU plan")
        problem.rhs_operators.append(op)
    else:
        raise TypeError("add_cell_accumulator(problem, test, trial, op) or (problem, test, load)")
    return problem


def add_surface_accumulator(problem, test_field, *args):
    """add_surface_accumulator!(problem, test, trial, op) or (problem, test, op)
    (accumulators.jl:435-466); the B200 plan recognises the symmetric Nitsche form."""
    if test_field is not problem.field:
        raise ValueError("the B200 plan supports one scalar field")
    if len(args) == 2:
        trial, op = args
        if trial is not test_field:
            raise ValueError("the B200 plan supports one scalar field")
        if not isinstance(op, Nitsche):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"surface form {type(op).__name__} is not supported by the GPU plan")
        problem.surface_operators.append(op)
    elif len(args) == 1:
        (op,) = args
        if not isinstance(op, Nitsche):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"surface rhs form {type(op).__name__} is not supported by the GPU plan")
        problem.surface_rhs_operators.append(op)
    else:
        raise TypeError("add_surface_accumulator(problem, test, trial, op) or (problem, test, op)")
    return problem


def add_boundary_accumulator(problem, boundary, test_field, *args):
    """add_boundary_accumulator!(problem, boundary, test, trial, op) or (problem, boundary, test, op)
    (accumulators.jl:396-411) with the symmetric Nitsche form."""
    if not isinstance(boundary, BoundaryFace):
        raise TypeError("boundary must be a BoundaryFace")
    if test_field is not problem.field:
        raise ValueError("the B200 plan supports one scalar field")
    if len(args) == 2:
        trial, op = args
        if trial is not test_field:
            raise ValueError("the B200 plan supports one scalar field")
        if not isinstance(op, Nitsche):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"boundary form {type(op).__name__} is not supported by the GPU plan")
        problem.boundary_operators.append((boundary, op))
    elif len(args) == 1:
        (op,) = args
        if not isinstance(op, Nitsche):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"boundary rhs form {type(op).__name__} is not supported by the GPU plan")
        problem.boundary_rhs_operators.append((boundary, op))
    else:
        raise TypeError("add_boundary_accumulator(problem, boundary, test, trial, op) or (problem, boundary, test, op)")
    return problem


def add_interface(problem, op):
    """add_interface!(problem, operator) (problem.jl): an operator on every interior interface of
    the space (matching and hanging); the B200 plan supports the SIPG form."""
    if not isinstance(op, SIPG):
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"interface form {type(op).__name__} is not supported by the GPU plan")
    if problem.interface_operators:
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "one interface form on the GPU plan")
    problem.interface_operators.append(op)
    return problem


def add_boundary(problem, boundary, op):
    """add_boundary!(problem, boundary, operator): the SIPG boundary operator (with its load when
    op.data is given) or the symmetric Nitsche form on the boundary faces of `boundary`."""
    if not isinstance(boundary, BoundaryFace):
        raise TypeError("boundary must be a BoundaryFace")
    if not isinstance(op, (SIPG, Nitsche)):
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, f"boundary form {type(op).__name__} is not supported by the GPU plan")
    problem.boundary_operators.append((boundary, op))
    if op.data is not None:
        problem.boundary_rhs_operators.append((boundary, op))
    return problem


def add_surface_quadrature(problem, surface):
    """add_surface_quadrature!(problem, surface) (embedded.jl:181-184); also accepts a list."""
    from .regions import SurfaceQuadrature

    items = surface if isinstance(surface, (list, tuple)) else [surface]
    for it in items:
        if not isinstance(it, SurfaceQuadrature):
            raise TypeError("expected SurfaceQuadrature items")
        problem.surfaces.append(it)
    return problem


def add_cell_quadrature(problem, leaf, points, weights):
    """add_cell_quadrature!(problem, leaf, quadrature) (embedded.jl:203-207): override one leaf's
    cell rule with explicit biunit reference points and reference weights."""
    pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
    w = np.asarray(weights, dtype=np.float64).reshape(-1)
    if pts.shape != (w.size, problem.field.space.D):
        raise ValueError("cell quadrature points and weights must match the dimension")
    if np.any(np.abs(pts) > 1.0 + 1e-12):
        raise ValueError("cell quadrature points must lie in the biunit cell")
    problem.cell_quadratures[int(leaf)] = (pts, w)
    return problem


def add_constraint(problem, constraint):
    if not isinstance(constraint, Dirichlet):
        raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "only Dirichlet constraints are supported")
    problem.dirichlet.append(constraint)
    return problem


# ---------------------------------------------------------------------------------------
# compile
# ---------------------------------------------------------------------------------------

class _Batch:
    """A tensor-cell batch of the host plan.  `points` (physical quadrature points, n_cells x nq x
    D) is built on first use: only right-hand sides, tabulated coefficients and error norms read
    it, and at 64^3 cells, p = 4 it is 0.8 GB."""

    def __getattr__(self, name):
        if name == "points":
            D = self.lower.shape[1]
            grids = np.meshgrid(*[self.rules[a][0] for a in range(D)], indexing="ij")
            # axis 1 fastest: flatten in Fortran order
            ref = np.stack([g.reshape(-1, order="F") for g in grids], axis=1)  # [nq, D]
            half = 0.5 * self.h
            pts = (self.lower + half)[:, None, :] + ref[None, :, :] * half[:, None, :]
            self.points = pts
            return pts
        raise AttributeError(name)


def _gauss(n):
    pts = np.zeros(n)
    wts = np.zeros(n)
    L.check(L.lib().grico_gauss_legendre(n, L.ptr(pts, C.c_double), L.ptr(wts, C.c_double)))
    return pts, wts


def _fe_basis(x, p):
    v = np.zeros(p + 2)
    d = np.zeros(p + 2)
    L.check(L.lib().grico_fe_basis(float(x), p, L.ptr(v, C.c_double), L.ptr(d, C.c_double)))
    return v[: p + 1], d[: p + 1]


def _tables(p, q):
    """B[i, j] = psi_i(xi_j) on q Gauss points."""
    pts, wts = _gauss(q)
    B = np.zeros((p + 1, q))
    G = np.zeros((p + 1, q))
    for j in range(q):
        v, d = _fe_basis(pts[j], p)
        B[:, j] = v
        G[:, j] = d
    return pts, wts, B, G


def _item_maps(space, cells, b):
    """Box-mode maps of the leaves at Morton positions `cells` (single terms inline, multi-term
    expansions into a tail CSR), stored on `b` as map_index/map_coef/tail_*/nbox."""
    degree = tuple(int(v) for v in space.degrees[cells[0]]) if len(cells) else ()
    nb = int(np.prod([d + 1 for d in degree])) if len(cells) else 0
    b.nbox = nb
    starts = space.box_offsets[cells]
    ent = (starts[:, None] + np.arange(nb)[None, :]).reshape(-1)
    lo = space.term_offsets[ent]
    hi = space.term_offsets[ent + 1]
    cnt = hi - lo
    mp = np.full(ent.size, -1, dtype=np.int32)
    single = cnt == 1
    mp[single] = space.term_index[lo[single]].astype(np.int32)
    coef = np.ones(ent.size)
    coef[single] = space.term_coef[lo[single]]
    multi = np.nonzero(cnt > 1)[0]
    if multi.size:
        mp[multi] = -(np.arange(multi.size, dtype=np.int32) + 2)
        tcnt = cnt[multi]
        b.tail_offsets = np.concatenate([[0], np.cumsum(tcnt)]).astype(np.int64)
        tsrc = np.concatenate([np.arange(l, h) for l, h in zip(lo[multi], hi[multi])])
        b.tail_index = space.term_index[tsrc].astype(np.int32)
        b.tail_coef = space.term_coef[tsrc].astype(np.float64)
    else:
        b.tail_offsets = b.tail_index = b.tail_coef = None
    b.map_index = np.ascontiguousarray(mp)
    b.map_coef = None if np.all(coef == 1.0) else np.ascontiguousarray(coef)


def _concat_item_maps(a, b):
    """a's item maps become [a's box modes, b's box modes] per item (interface items), with b's
    tail expansions appended to a's tail table."""
    n = len(a.map_index) // max(a.nbox, 1) if a.nbox else 0
    ma = a.map_index.reshape(n, a.nbox)
    mb = b.map_index.reshape(n, b.nbox).copy()
    na_tail = 0 if a.tail_offsets is None else len(a.tail_offsets) - 1
    tails = mb <= -2
    mb[tails] -= na_tail  # tail k of b becomes tail na_tail + k: code -(k + 2) - na_tail
    a.map_index = np.ascontiguousarray(np.concatenate([ma, mb], axis=1).reshape(-1).astype(np.int32))
    ca = np.ones(ma.shape) if a.map_coef is None else a.map_coef.reshape(n, a.nbox)
    cb = np.ones(mb.shape) if b.map_coef is None else b.map_coef.reshape(n, b.nbox)
    coef = np.concatenate([ca, cb], axis=1).reshape(-1)
    a.map_coef = None if np.all(coef == 1.0) else np.ascontiguousarray(coef)
    if b.tail_offsets is not None:
        if a.tail_offsets is None:
            a.tail_offsets, a.tail_index, a.tail_coef = b.tail_offsets, b.tail_index, b.tail_coef
        else:
            base = a.tail_offsets[-1]
            a.tail_offsets = np.concatenate([a.tail_offsets, base + b.tail_offsets[1:]]).astype(np.int64)
            a.tail_index = np.concatenate([a.tail_index, b.tail_index]).astype(np.int32)
            a.tail_coef = np.concatenate([a.tail_coef, b.tail_coef])
    a.nbox_minus, a.nbox = a.nbox, a.nbox + b.nbox


def fe_basis_table(x, p):
    """psi_0..psi_p and derivatives at every entry of x: ([n, p+1], [n, p+1])
    (polynomials.jl:403-434, vectorised)."""
    x = np.asarray(x, dtype=np.float64)
    v = np.zeros((x.size, p + 1))
    d = np.zeros((x.size, p + 1))
    if p == 0:
        v[:, 0] = 1.0
        return v, d
    v[:, 0] = 0.5 * (1.0 - x)
    v[:, 1] = 0.5 * (1.0 + x)
    d[:, 0] = -0.5
    d[:, 1] = 0.5
    pm2, pm1 = np.ones_like(x), x.copy()
    for k in range(2, p + 1):
        pk = ((2 * k - 1) * x * pm1 - (k - 1) * pm2) / k
        v[:, k] = (pk - pm2) / math.sqrt(4 * k - 2)
        d[:, k] = math.sqrt((2 * k - 1) / 2.0) * pm1
        pm2, pm1 = pm1, pk
    return v, d


class _PointBatch:
    pass


def _subcell_supported(D, degree, qshape):
    if D not in L.SUBCELL_SHAPES or len(set(degree)) != 1 or len(set(qshape)) != 1:
        return False
    return (degree[0] + 1, qshape[0]) in L.SUBCELL_SHAPES[D] and int(np.prod(qshape)) <= 64


def _subcell_point_chunks(b, chunk=65536):
    """(physical points [m*qp, D], weights [m*qp] incl. det and the keep mask, item index [m*qp],
    reference points [m*qp, D]) of the subcell points of a GRICO_ITEM_SUBCELLS batch, `chunk`
    subcells at a time, in the order of the kernel's source arrays (subcell-major, tensor point
    minor, axis 1 fastest)."""
    D = b.h.shape[1]
    q = b.q[0]
    pts, wts = _gauss(q)
    grids = np.meshgrid(*([pts] * D), indexing="ij")
    eta = np.stack([g.reshape(-1, order="F") for g in grids], axis=1)       # [qp, D]
    wg = np.meshgrid(*([wts] * D), indexing="ij")
    W = np.ones(eta.shape[0])
    for a in range(D):
        W = W * wg[a].reshape(-1, order="F")
    qp = eta.shape[0]
    bitpos = np.arange(qp, dtype=np.uint64)
    nsub = len(b.subcell_level)
    item_of = np.repeat(np.arange(len(b.cells)), np.diff(b.subcell_offsets))
    det = np.prod(0.5 * b.h, axis=1)
    for s0 in range(0, nsub, chunk):
        s1 = min(nsub, s0 + chunk)
        half = np.ldexp(1.0, -b.subcell_level[s0:s1].astype(np.int64))[:, None]
        c = -1.0 + (2.0 * b.subcell_pos[s0:s1] + 1.0) * half                  # [m, D]
        xi = c[:, None, :] + half[:, :, None] * eta[None, :, :]                # [m, qp, D]
        it = item_of[s0:s1]
        hh = 0.5 * b.h[it]
        X = (b.lower[it] + hh)[:, None, :] + xi * hh[:, None, :]
        keep = ((b.subcell_mask[s0:s1, None] >> bitpos[None, :]) & np.uint64(1)).astype(bool)
        w = W[None, :] * (b.subcell_weight[s0:s1] * det[it])[:, None] * keep
        yield X.reshape(-1, D), w.reshape(-1), np.repeat(it, qp), xi.reshape(-1, D)


class AssemblyPlan:
    """Compiled plan: descriptor arrays built here, device data owned by libgrico_b200."""

    def __init__(self, problem, device=True):
        if not problem.cell_operators:
            raise ValueError("problem has no cell operator")
        if len(problem.cell_operators) > 1:
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "the GPU plan accepts one cell operator form")
        self.problem = problem
        self.form = problem.cell_operators[0]
        space = problem.field.space
        self.space = space
        domain = space.domain
        self.D = D = space.D
        n_full = space.scalar_dof_count
        self.n_full = n_full
        from .regions import FiniteCellExtension, PhysicalDomain

        physical = isinstance(domain, PhysicalDomain)
        if physical and (problem.dirichlet or problem.boundary_operators or problem.boundary_rhs_operators):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM,
                               "boundary-face constraints and forms on a PhysicalDomain are not supported by the GPU plan")
        # --- which leaves integrate on point rules: cut cells and explicit cell quadratures ---
        point_rule = {}
        for leaf, rule in problem.cell_quadratures.items():
            if leaf not in space.leaf_to_index:
                raise ValueError(f"cell quadrature leaf {leaf} is not an active leaf")
            point_rule[space.leaf_to_index[leaf]] = rule
        self.n_cut = 0
        sub_groups = []      # (Morton positions, degree, qshape) integrated as octree subcells
        if physical and not (isinstance(domain.cell_measure, FiniteCellExtension) and domain.cell_measure.alpha == 1.0):
            cls = domain.classify(space.leaves)
            cut = np.nonzero(cls == 2)[0]
            cut = np.array([c for c in cut if int(c) not in point_rule], dtype=np.int64)
            self.n_cut = int(cut.size)
            if cut.size:
                sig_cut = np.concatenate([space.degrees[cut], space.qshape[cut]], axis=1)
                for sg in np.unique(sig_cut, axis=0):
                    sel = cut[np.all(sig_cut == sg, axis=1)]
                    deg, qsig = tuple(int(v) for v in sg[:D]), tuple(int(v) for v in sg[D:])
                    if domain.quadrature == "candidates" and _subcell_supported(D, deg, qsig):
                        sub_groups.append((sel, deg, qsig))
                        continue
                    rules = domain.cut_cell_quadrature(space.leaves[sel], qsig, _gauss)
                    for c, r in zip(sel, rules):
                        if r is not None:        # no candidate at all: the tensor rule stays
                            point_rule[int(c)] = r
        tensor_mask = np.ones(len(space.leaves), dtype=bool)
        tensor_mask[list(point_rule)] = False
        for sel, _, _ in sub_groups:
            tensor_mask[sel] = False
        # --- tensor batches by (degrees, quadrature shape), first appearance in Morton order ---
        sig = np.concatenate([space.degrees, space.qshape], axis=1)
        self.batches = []
        tensor_cells = np.nonzero(tensor_mask)[0]
        if tensor_cells.size:
            _, first, inv = np.unique(sig[tensor_cells], axis=0, return_index=True, return_inverse=True)
            inv = inv.reshape(-1)
            for g in np.argsort(first, kind="stable"):
                cells = tensor_cells[inv == g]
                b = _Batch()
                b.cells = cells                                      # Morton positions
                b.leaves = space.leaves[cells]
                b.degree = tuple(int(v) for v in space.degrees[cells[0]])
                b.q = tuple(int(v) for v in space.qshape[cells[0]])
                _item_maps(space, cells, b)
                b.h = np.ascontiguousarray(domain.cell_size(b.leaves))
                b.lower = domain.cell_lower(b.leaves)
                # reference points of the tensor rule, axis 1 fastest
                b.rules = [_tables(b.degree[a], b.q[a]) for a in range(D)]
                b.kappa_points = None
                if self.form.coefficient is not None:
                    vals = np.asarray(self.form.coefficient(b.points.reshape(-1, D)), dtype=np.float64)
                    b.kappa_points = np.ascontiguousarray(vals.reshape(len(cells), -1))
                self.batches.append(b)
        # --- point-quadrature items: cut cells, faces, embedded surfaces ---
        self.point_batches = []
        extra = self._build_subcell_items(sub_groups)
        self._build_cell_items(point_rule, extra)
        self._build_nitsche_items(problem)
        self._build_interface_items(problem)
        # --- Dirichlet: fixed dofs are the dofs with a trace on a selected boundary face ---
        self._compile_dirichlet(problem)
        # --- reduced map u_full = shift + P u_red (assembly.jl:112-314): free dofs are neither
        # fixed nor relation pivots, numbered in dof order; a pivot's row expands its relation
        # (whose dofs are free: fixed dofs were substituted before the relations were formed) ---
        free = np.ones(n_full, dtype=bool)
        free[self.fixed_dofs] = False
        for (pivot, _, _, _) in self.relations:
            free[pivot] = False
        self.solve_dofs = np.nonzero(free)[0]
        self.n_reduced = int(self.solve_dofs.size)
        reduced_index = np.full(n_full, -1, dtype=np.int64)
        reduced_index[self.solve_dofs] = np.arange(self.n_reduced)
        self.reduced_index = reduced_index
        self.shift = np.zeros(n_full)
        self.shift[self.fixed_dofs] = self.fixed_values
        counts = free.astype(np.int64)
        extra = {}
        for (pivot, idx, co, rhs) in self.relations:
            if np.any(reduced_index[idx] < 0):
                raise ValueError("a Dirichlet relation couples to a constrained dof")
            extra[pivot] = (reduced_index[idx], co)
            counts[pivot] = idx.size
            self.shift[pivot] = rhs
        self.red_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        if extra:
            self.red_index = np.zeros(int(self.red_offsets[-1]), dtype=np.int64)
            self.red_coef = np.ones(int(self.red_offsets[-1]))
            self.red_index[self.red_offsets[self.solve_dofs]] = np.arange(self.n_reduced)
            for pivot, (ri, co) in extra.items():
                lo = self.red_offsets[pivot]
                order = np.argsort(ri, kind="stable")
                self.red_index[lo:lo + ri.size] = ri[order]
                self.red_coef[lo:lo + ri.size] = co[order]
        else:
            self.red_index = np.arange(self.n_reduced, dtype=np.int64)
            self.red_coef = np.ones(self.n_reduced)
        self.handle = None
        if device:
            self._create_device_plan()

    def _new_point_batch(self, kind, positions, degree):
        space, domain, D = self.space, self.space.domain, self.D
        pb = _PointBatch()
        pb.kind = kind
        pb.cells = np.asarray(positions, dtype=np.int64)
        pb.leaves = space.leaves[pb.cells]
        pb.degree = degree
        _item_maps(space, pb.cells, pb)
        pb.h = np.ascontiguousarray(domain.cell_size(pb.leaves))
        pb.lower = domain.cell_lower(pb.leaves)
        return pb

    def _finish_point_batch(self, pb, refs, weights, normals=None, eta=None):
        D = self.D
        counts = np.array([len(w) for w in weights], dtype=np.int64)
        pb.point_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        pb.ref_points = np.ascontiguousarray(np.concatenate(refs).reshape(-1, D)) if len(refs) else np.zeros((0, D))
        pb.weights = np.ascontiguousarray(np.concatenate(weights)) if len(weights) else np.zeros(0)
        pb.normals = None if normals is None else np.ascontiguousarray(np.concatenate(normals).reshape(-1, D))
        pb.eta = None if eta is None else np.ascontiguousarray(eta, dtype=np.float64)
        item = np.repeat(np.arange(len(pb.cells)), counts)
        half = 0.5 * pb.h[item]
        pb.points = (pb.lower[item] + half) + pb.ref_points * half           # physical points [P, D]
        pb.kappa_points = None
        if pb.kind == L.GRICO_ITEM_CELL and self.form.coefficient is not None:
            pb.kappa_points = np.ascontiguousarray(
                np.asarray(self.form.coefficient(pb.points), dtype=np.float64).reshape(-1))
        self.point_batches.append(pb)

    def _build_cell_items(self, point_rule, extra=()):
        """Cells on explicit point rules (moment-fitted cut cells, add_cell_quadrature!, sliver
        points of subcell cut cells): kind-1 items grouped by degree (Morton order)."""
        space, D = self.space, self.D
        items = sorted([(int(c), r[0], r[1]) for c, r in point_rule.items()] + list(extra), key=lambda t: t[0])
        if not items:
            return
        pos = np.array([t[0] for t in items], dtype=np.int64)
        degs = space.degrees[pos]
        for dsig in np.unique(degs, axis=0):
            idx = [i for i in range(len(items)) if np.all(degs[i] == dsig)]
            sel = pos[idx]
            pb = self._new_point_batch(L.GRICO_ITEM_CELL, sel, tuple(int(v) for v in dsig))
            det = np.prod(0.5 * pb.h, axis=1)
            refs = [items[i][1] for i in idx]
            wts = [items[i][2] * det[k] for k, i in enumerate(idx)]
            self._finish_point_batch(pb, refs, wts)

    def _build_subcell_items(self, groups):
        """Cut cells of the candidate rule as octree subcells (GRICO_ITEM_SUBCELLS), one batch per
        (degree, quadrature shape).  Returns the sliver fallback points as extra point rules."""
        from .regions import FiniteCellExtension

        space, domain, D = self.space, self.space.domain, self.D
        extra = []
        if not groups:
            return extra
        alpha = domain.cell_measure.alpha if isinstance(domain.cell_measure, FiniteCellExtension) else 0.0
        for sel, deg, qsig in groups:
            off, lev, pos, mask, ws, slivers = domain.subcell_quadrature(space.leaves[sel], qsig, _gauss)
            nq = int(np.prod(qsig))
            if alpha > 0.0:
                # (1 - alpha) * physical + alpha * the full cell as one level-0 subcell per cell
                counts = np.diff(off) + 1
                first = np.concatenate([[0], np.cumsum(counts)])[:-1]
                tot = int(counts.sum())
                full = np.uint64((1 << nq) - 1) if nq < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
                lev2 = np.zeros(tot, dtype=np.int32)
                pos2 = np.zeros((tot, D), dtype=np.int32)
                mask2 = np.full(tot, full, dtype=np.uint64)
                ws2 = np.full(tot, alpha)
                rest = np.ones(tot, dtype=bool)
                rest[first] = False
                lev2[rest], pos2[rest], mask2[rest], ws2[rest] = lev, pos, mask, (1.0 - alpha) * ws
                off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
                lev, pos, mask, ws = lev2, pos2, mask2, ws2
                slivers = {c: (p, (1.0 - alpha) * w) for c, (p, w) in slivers.items()}
            pb = self._new_point_batch(L.GRICO_ITEM_SUBCELLS, sel, deg)
            pb.q = qsig
            pb.subcell_offsets = off
            pb.subcell_level = np.ascontiguousarray(lev, dtype=np.int32)
            pb.subcell_pos = np.ascontiguousarray(pos, dtype=np.int32)
            pb.subcell_mask = np.ascontiguousarray(mask, dtype=np.uint64)
            pb.subcell_weight = np.ascontiguousarray(ws, dtype=np.float64)
            pb.point_offsets = None
            pb.ref_points = pb.weights = pb.normals = pb.eta = None
            pb.kappa_points = None
            if self.form.coefficient is not None and len(lev):
                pb.kappa_points = np.ascontiguousarray(np.concatenate([
                    np.asarray(self.form.coefficient(X), dtype=np.float64).reshape(-1)
                    for X, _, _, _ in _subcell_point_chunks(pb)]))
            self.point_batches.append(pb)
            for c, (p, w) in slivers.items():
                extra.append((int(sel[c]), p, w))
        return extra

    def _build_nitsche_items(self, problem):
        """Boundary-face items (integration.jl:2230-2256) and embedded-surface items
        (integration.jl:2338-2357) of the Nitsche forms, grouped by degree."""
        from .regions import physical_surface_data

        space, D = self.space, self.D
        domain = space.domain
        bil = problem.surface_operators
        rhs = problem.surface_rhs_operators
        if len(bil) > 1 or len(rhs) > 1:
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "the GPU plan accepts one surface form and one surface load")
        if rhs and not bil:
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "a Nitsche surface load needs the matching Nitsche surface form")
        if bil and rhs and bil[0].penalty != rhs[0].penalty:
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "Nitsche surface form and load must share the penalty")
        items = []   # (position, ref pts, phys weights, phys normals, penalty, data, src tag)
        if bil and problem.surfaces:
            op = bil[0]
            g = rhs[0].data if rhs else None
            for sq in sorted(problem.surfaces, key=lambda s: s.leaf):
                if sq.leaf not in space.leaf_to_index:
                    raise ValueError(f"surface quadrature leaf {sq.leaf} is not an active leaf")
                w, n = physical_surface_data(domain, sq.leaf, sq)
                items.append((space.leaf_to_index[sq.leaf], sq.points, w, n, op.penalty, g))
        # boundary faces: one bilinear and at most one load per face
        bops = {}
        for bf, op in problem.boundary_operators:
            key = (bf.axis - 1, bf.side - 1)
            if key in bops:
                raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "one boundary form per face on the GPU plan")
            bops[key] = [op, None]
        for bf, op in problem.boundary_rhs_operators:
            key = (bf.axis - 1, bf.side - 1)
            if key not in bops or bops[key][1] is not None or bops[key][0].penalty != op.penalty or \
                    type(bops[key][0]) is not type(op):
                raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM,
                                   "a Nitsche boundary load needs the matching Nitsche boundary form")
            bops[key][1] = op.data
        if bops:
            b_leaf, b_axis, b_side = space.boundary_faces
            for pos, ax, sd in zip(b_leaf, b_axis, b_side):
                key = (int(ax), int(sd))
                if key not in bops:
                    continue
                op, g = bops[key]
                q = space.qshape[pos]
                rules = [_gauss(int(q[a])) if a != ax else (np.array([-1.0 if sd == 0 else 1.0]), np.array([1.0]))
                         for a in range(D)]
                grids = np.meshgrid(*[r[0] for r in rules], indexing="ij")
                wg = np.meshgrid(*[r[1] for r in rules], indexing="ij")
                ref = np.stack([gg.reshape(-1, order="F") for gg in grids], axis=1)
                wref = np.ones(ref.shape[0])
                for a in range(D):
                    wref = wref * wg[a].reshape(-1, order="F")
                h = domain.cell_size(space.leaves[[pos]])[0]
                scale = 1.0 if D == 1 else math.ldexp(float(np.prod([h[a] for a in range(D) if a != ax])), -(D - 1))
                nrm = np.zeros((ref.shape[0], D))
                nrm[:, ax] = -1.0 if sd == 0 else 1.0
                # SIPG boundary penalty (sine_poisson_sipg.jl:42-46); Nitsche: penalty / min(h)
                eta = (op.penalty * (int(space.degrees[pos][ax]) + 1) ** 2 / float(h[ax])
                       if isinstance(op, SIPG) else None)
                items.append((int(pos), ref, wref * scale, nrm, op.penalty, g, eta))
        if not items:
            return
        degs = np.array([space.degrees[it[0]] for it in items]).reshape(len(items), D)
        for dsig in np.unique(degs, axis=0):
            sel = [i for i in range(len(items)) if np.all(degs[i] == dsig)]
            pb = self._new_point_batch(L.GRICO_ITEM_NITSCHE, [items[i][0] for i in sel], tuple(int(v) for v in dsig))
            eta = np.array([items[i][6] if len(items[i]) > 6 and items[i][6] is not None
                            else items[i][4] / float(np.min(pb.h[k])) for k, i in enumerate(sel)])
            pb.data = [items[i][5] for i in sel]
            self._finish_point_batch(pb, [items[i][1] for i in sel], [items[i][2] for i in sel],
                                     [items[i][3] for i in sel], eta)

    def _build_interface_items(self, problem):
        """Two-sided SIPG items on every interior interface (integration.jl:2262-2307): the shared
        tangential patch is the intersection of the two faces with max(q-, q+) Gauss points per
        tangential axis (integration.jl:2800-2841); one batch per (minus degree, plus degree,
        point count) in enumeration order."""
        if not problem.interface_operators:
            return
        op = problem.interface_operators[0]
        space, domain, D = self.space, self.space.domain, self.D
        i_m, i_p, i_a = space.interfaces
        if len(i_m) == 0:
            return
        lower = domain.cell_lower(space.leaves)
        size = domain.cell_size(space.leaves)
        items = []
        for m, pl, ax in zip(i_m.tolist(), i_p.tolist(), i_a.tolist()):
            tang = [a for a in range(D) if a != ax]
            lo = np.maximum(lower[m], lower[pl])
            hi = np.minimum(lower[m] + size[m], lower[pl] + size[pl])
            rules = [_gauss(int(max(space.qshape[m][a], space.qshape[pl][a]))) for a in tang]
            npts = int(np.prod([len(r[0]) for r in rules])) if tang else 1
            phys = np.zeros((npts, D))
            w = np.ones(npts)
            if tang:
                grids = np.meshgrid(*[r[0] for r in rules], indexing="ij")
                wg = np.meshgrid(*[r[1] for r in rules], indexing="ij")
                for k, a in enumerate(tang):
                    half = 0.5 * (hi[a] - lo[a])
                    phys[:, a] = lo[a] + half * (1.0 + grids[k].reshape(-1, order="F"))
                    w = w * wg[k].reshape(-1, order="F") * half
            phys[:, ax] = lower[m][ax] + size[m][ax]
            ref_m = (phys - (lower[m] + 0.5 * size[m])) / (0.5 * size[m])
            ref_p = (phys - (lower[pl] + 0.5 * size[pl])) / (0.5 * size[pl])
            ref_m[:, ax] = 1.0
            ref_p[:, ax] = -1.0
            hm, hp = float(size[m][ax]), float(size[pl][ax])
            pmax = max(int(space.degrees[m][ax]), int(space.degrees[pl][ax]))
            sigma = op.penalty * (pmax + 1) ** 2 / (2.0 * hm * hp / (hm + hp))
            items.append((m, pl, ax, ref_m, ref_p, w, sigma))
        sig = {}
        for it in items:
            key = (tuple(int(v) for v in space.degrees[it[0]]), tuple(int(v) for v in space.degrees[it[1]]), len(it[5]))
            sig.setdefault(key, []).append(it)
        for (dm, dp, _), its in sig.items():
            pb = self._new_point_batch(L.GRICO_ITEM_INTERFACE, [it[0] for it in its], dm)
            plus = _PointBatch()
            _item_maps(space, np.array([it[1] for it in its], dtype=np.int64), plus)
            _concat_item_maps(pb, plus)
            pb.degree_plus = dp
            pb.plus_cells = np.array([it[1] for it in its], dtype=np.int64)
            pb.h_plus = np.ascontiguousarray(domain.cell_size(space.leaves[pb.plus_cells]))
            pb.face_axis = np.array([it[2] for it in its], dtype=np.int32)
            pb.ref_points_plus = np.ascontiguousarray(np.concatenate([it[4] for it in its]).reshape(-1, D))
            self._finish_point_batch(pb, [it[3] for it in its], [it[5] for it in its],
                                     eta=np.array([it[6] for it in its]))

    def _points(self, b):
        D = self.D
        grids = np.meshgrid(*[b.rules[a][0] for a in range(D)], indexing="ij")
        # axis 1 fastest: flatten in Fortran order
        ref = np.stack([g.reshape(-1, order="F") for g in grids], axis=1)  # [nq, D]
        half = 0.5 * b.h
        center = b.lower + half
        return center[:, None, :] + ref[None, :, :] * half[:, None, :]

    def _compile_dirichlet(self, problem):
        """Dirichlet data as fixed dofs and affine relation rows (plans.jl:486-972).

        The reference projects the data onto the trace space in L2: a Gram system over every
        dof with a term on a selected boundary face, its rank from an eigen decomposition, pivot
        dofs from QR with column pivoting and, for pivots that couple to free dofs, relation
        rows x_p - sum c_j x_j = rhs (plans.jl:884-943).  Its row space is that of the trace
        rows: one row per trace mode of each selected face, sum_t c_t x_{d_t} = target (the
        constant on vertex modes, 0 on the others: a constant is exact in the trace basis).
        Here a row with one term fixes its dof (target / coefficient; where faces with
        different constants meet, the last face in enumeration order wins); rows with several
        terms (hanging-node expansions on a Dirichlet face) have their fixed dofs substituted
        and are solved per connected component by the reference's steps (`_dirichlet_system`).
        Vectorised per (degrees, axis, side) group of boundary faces."""
        space = self.space
        D = self.D
        self.fixed_dofs = np.zeros(0, dtype=np.int64)
        self.fixed_values = np.zeros(0, dtype=np.float64)
        self.relations = []
        if not problem.dirichlet:
            return
        b_leaf, b_axis, b_side = space.boundary_faces
        sel = {}
        for con in problem.dirichlet:
            key = (con.boundary.axis - 1, con.boundary.side - 1)
            if key in sel and sel[key] != con.value:
                raise ValueError("multiple Dirichlet constraints target the same boundary face")
            sel[key] = con.value
        b_leaf = np.asarray(b_leaf, dtype=np.int64)
        b_axis = np.asarray(b_axis, dtype=np.int64)
        b_side = np.asarray(b_side, dtype=np.int64)
        face_ids = np.arange(len(b_leaf), dtype=np.int64)
        t_entry, t_dof, t_coef = [], [], []          # per term: row, dof, coefficient
        e_target, e_cnt, e_order = [], [], []        # per row (face trace mode)
        base = 0
        matched = set()
        degs = space.degrees[b_leaf] if len(b_leaf) else np.zeros((0, D), dtype=np.int64)
        for (ax, sd), val in sel.items():
            mask = (b_axis == ax) & (b_side == sd)
            if not mask.any():
                continue
            matched.add((ax, sd))
            fsel = face_ids[mask]
            for dsig in np.unique(degs[fsel], axis=0):
                g = fsel[np.all(degs[fsel] == dsig, axis=1)]
                shape = dsig + 1
                nb = int(np.prod(shape))
                box = np.arange(nb)
                digits = np.stack([(box // int(np.prod(shape[:a]))) % shape[a] for a in range(D)], axis=1)
                modes = np.nonzero(digits[:, ax] == sd)[0]
                vertex = np.all(digits[modes] <= 1, axis=1)
                e = (space.box_offsets[b_leaf[g]][:, None] + modes[None, :]).reshape(-1)
                lo = space.term_offsets[e]
                cnt = space.term_offsets[e + 1] - lo
                rep = np.repeat(np.arange(e.size), cnt)
                t = np.repeat(lo - np.concatenate([[0], np.cumsum(cnt)[:-1]]), cnt) + np.arange(int(cnt.sum()))
                t_entry.append(base + rep)
                t_dof.append(space.term_index[t].astype(np.int64))
                t_coef.append(np.asarray(space.term_coef[t], dtype=np.float64))
                e_target.append(np.where(np.tile(vertex, len(g)), float(val), 0.0))
                e_cnt.append(cnt.astype(np.int64))
                # enumeration order: boundary face, then mode
                e_order.append(np.repeat(g, len(modes)) * (1 << 32) + np.tile(np.arange(len(modes)), len(g)))
                base += e.size
        for key in sel:
            if key not in matched:
                raise ValueError("Dirichlet constraint does not match any boundary face")
        if base == 0:
            return
        t_entry, t_dof, t_coef = np.concatenate(t_entry), np.concatenate(t_dof), np.concatenate(t_coef)
        e_target, e_cnt, e_order = np.concatenate(e_target), np.concatenate(e_cnt), np.concatenate(e_order)
        single_t = e_cnt[t_entry] == 1
        fixed = np.unique(t_dof[single_t])
        values = np.zeros(fixed.size)
        sv_t = single_t & (e_target[t_entry] != 0.0)
        if sv_t.any():
            sd_ = t_dof[sv_t]
            sv = e_target[t_entry[sv_t]] / t_coef[sv_t]
            so = e_order[t_entry[sv_t]]
            last = np.lexsort((so, sd_))          # by dof, then enumeration order
            sd_, sv = sd_[last], sv[last]
            keep = np.ones(sd_.size, dtype=bool)
            keep[:-1] = sd_[1:] != sd_[:-1]        # last assignment per dof
            values[np.searchsorted(fixed, sd_[keep])] = sv[keep]
        multi_t = ~single_t
        rel = []
        if multi_t.any():
            fixed_val = np.zeros(self.n_full)
            is_fixed = np.zeros(self.n_full, dtype=bool)
            is_fixed[fixed] = True
            fixed_val[fixed] = values
            me, md, mc = t_entry[multi_t], t_dof[multi_t], t_coef[multi_t]
            target = e_target.copy()
            np.subtract.at(target, me[is_fixed[md]], mc[is_fixed[md]] * fixed_val[md[is_fixed[md]]])
            keep = ~is_fixed[md]
            me, md, mc = me[keep], md[keep], mc[keep]
            if me.size:
                fx, fv, rel = _dirichlet_components(me, md, mc, target)
                if fx.size:
                    fixed = np.concatenate([fixed, fx])
                    values = np.concatenate([values, fv])
                    order = np.argsort(fixed, kind="stable")
                    fixed, values = fixed[order], values[order]
        self.fixed_dofs = fixed.astype(np.int64)
        self.fixed_values = values
        self.relations = sorted(rel, key=lambda r: r[0])

    def _create_device_plan(self):
        descs = (L.GricoCellBatchDesc * len(self.batches))()
        for i, b in enumerate(self.batches):
            d = descs[i]
            d.n_cells = len(b.cells)
            for a in range(3):
                d.degree[a] = b.degree[a] if a < self.D else 0
                d.qpoints[a] = b.q[a] if a < self.D else 1
            d.map_index = L.ptr(b.map_index, C.c_int32)
            d.map_coef = L.ptr(b.map_coef, C.c_double)
            d.n_tail = 0 if b.tail_offsets is None else len(b.tail_offsets) - 1
            d.tail_offsets = L.ptr(b.tail_offsets, C.c_int64)
            d.tail_index = L.ptr(b.tail_index, C.c_int32)
            d.tail_coef = L.ptr(b.tail_coef, C.c_double)
            d.cell_size = L.ptr(b.h, C.c_double)
            d.kappa_points = L.ptr(b.kappa_points, C.c_double)
        pdescs = (L.GricoPointBatchDesc * max(1, len(self.point_batches)))()
        for i, b in enumerate(self.point_batches):
            d = pdescs[i]
            d.n_items = len(b.cells)
            d.kind = b.kind
            for a in range(3):
                d.degree[a] = b.degree[a] if a < self.D else 0
            d.map_index = L.ptr(b.map_index, C.c_int32)
            d.map_coef = L.ptr(b.map_coef, C.c_double)
            d.n_tail = 0 if b.tail_offsets is None else len(b.tail_offsets) - 1
            d.tail_offsets = L.ptr(b.tail_offsets, C.c_int64)
            d.tail_index = L.ptr(b.tail_index, C.c_int32)
            d.tail_coef = L.ptr(b.tail_coef, C.c_double)
            d.cell_size = L.ptr(b.h, C.c_double)
            if b.kind == L.GRICO_ITEM_SUBCELLS:
                for a in range(3):
                    d.qpoints[a] = b.q[a] if a < self.D else 1
                d.subcell_offsets = L.ptr(b.subcell_offsets, C.c_int64)
                d.subcell_level = L.ptr(b.subcell_level, C.c_int32)
                d.subcell_pos = L.ptr(b.subcell_pos, C.c_int32)
                d.subcell_mask = L.ptr(b.subcell_mask, C.c_uint64)
                d.subcell_weight = L.ptr(b.subcell_weight, C.c_double)
            if b.kind == L.GRICO_ITEM_INTERFACE:
                for a in range(3):
                    d.degree_plus[a] = b.degree_plus[a] if a < self.D else 0
                d.ref_points_plus = L.ptr(b.ref_points_plus, C.c_double)
                d.cell_size_plus = L.ptr(b.h_plus, C.c_double)
                d.face_axis = L.ptr(b.face_axis, C.c_int32)
            d.point_offsets = L.ptr(b.point_offsets, C.c_int64)
            d.ref_points = L.ptr(b.ref_points, C.c_double)
            d.weights = L.ptr(b.weights, C.c_double)
            d.normals = L.ptr(b.normals, C.c_double)
            d.eta = L.ptr(b.eta, C.c_double)
            d.kappa_points = L.ptr(b.kappa_points, C.c_double)
        pd = L.GricoPlanDesc()
        pd.n_point_batches = len(self.point_batches)
        pd.point_batches = pdescs
        pd.dim = self.D
        pd.form = L.GRICO_FORM_MASS_DIFFUSION
        pd.mass = self.form.mass
        pd.kappa = self.form.kappa
        pd.n_full = self.n_full
        pd.n_batches = len(self.batches)
        pd.batches = descs
        pd.n_fixed = len(self.fixed_dofs)
        pd.fixed_dofs = L.ptr(self.fixed_dofs, C.c_int64)
        pd.fixed_values = L.ptr(self.fixed_values, C.c_double)
        rels = self.relations
        pd.n_relations = len(rels)
        if rels:
            self._rel_pivot = np.array([r[0] for r in rels], dtype=np.int64)
            self._rel_offsets = np.concatenate([[0], np.cumsum([r[1].size for r in rels])]).astype(np.int64)
            self._rel_index = np.ascontiguousarray(np.concatenate([r[1] for r in rels]), dtype=np.int64)
            self._rel_coef = np.ascontiguousarray(np.concatenate([r[2] for r in rels]), dtype=np.float64)
            self._rel_rhs = np.array([r[3] for r in rels], dtype=np.float64)
            pd.rel_pivot = L.ptr(self._rel_pivot, C.c_int64)
            pd.rel_offsets = L.ptr(self._rel_offsets, C.c_int64)
            pd.rel_index = L.ptr(self._rel_index, C.c_int64)
            pd.rel_coef = L.ptr(self._rel_coef, C.c_double)
            pd.rel_rhs = L.ptr(self._rel_rhs, C.c_double)
        pd.n_reduced = self.n_reduced
        pd.red_offsets = L.ptr(self.red_offsets, C.c_int64)
        pd.red_index = L.ptr(self.red_index, C.c_int64)
        pd.red_coef = L.ptr(self.red_coef, C.c_double)
        pd.red_shift = L.ptr(self.shift, C.c_double)
        handle = C.c_void_p()
        L.check(L.lib().grico_plan_create(C.byref(pd), C.byref(handle)), "compile")
        self.handle = handle

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                L.lib().grico_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ---- sizes ----
    def dof_count(self):
        return self.n_full

    def reduced_dof_count(self):
        return self.n_reduced


def compile(problem, device=True):
    """compile(problem) -> AssemblyPlan (plans.jl:170-231).  device=False builds only the host
    descriptor (no CUDA call), which the CPU tests compare with the oracle."""
    return AssemblyPlan(problem, device=device)


# ---------------------------------------------------------------------------------------
# runtime
# ---------------------------------------------------------------------------------------

def _vector_call(fn, plan, x, y, n, nrhs=1):
    """Dispatch host numpy arrays (copied by the library) or torch CUDA tensors (device
    pointers, current torch stream)."""
    if isinstance(x, np.ndarray):
        x = np.ascontiguousarray(x)
        prec = L.GRICO_PREC_FP64 if x.dtype == np.float64 else L.GRICO_PREC_FP32
        if x.size != n * nrhs:
            raise ValueError(f"coefficient vector must have length {n * nrhs}")
        if y is None:
            y = np.zeros_like(x)
        L.check(fn(plan.handle, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), nrhs, prec,
                   L.GRICO_FLAG_HOST_POINTERS, None), "apply")
        return y
    import torch  # device tensors

    if not (isinstance(x, torch.Tensor) and x.is_cuda):
        raise TypeError("vectors must be numpy arrays or CUDA tensors")
    if x.numel() != n * nrhs:
        raise ValueError(f"coefficient vector must have length {n * nrhs}")
    prec = L.GRICO_PREC_FP64 if x.dtype == torch.float64 else L.GRICO_PREC_FP32
    if y is None:
        y = torch.empty_like(x)
    if y.data_ptr() == x.data_ptr():
        raise ValueError("result and coefficient vector must not alias")
    L.check(fn(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), nrhs, prec, 0,
               C.c_void_p(torch_stream_handle())), "apply")
    return y


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the library reads a NULL stream as "the plan's stream"


def torch_stream_handle():
    """Handle of torch's current stream as the library expects it (legacy default stream -> 0x1)."""
    import torch

    h = torch.cuda.current_stream().cuda_stream
    return h if h else CUDA_STREAM_LEGACY


def apply(plan, x, nrhs=1):
    """apply(plan, x) on the full layout (assembly.jl:517-530)."""
    return _vector_call(L.lib().grico_apply, plan, x, None, plan.n_full, nrhs)


def apply_(y, plan, x, nrhs=1):
    """apply!(y, plan, x)."""
    return _vector_call(L.lib().grico_apply, plan, x, y, plan.n_full, nrhs)


def reduced_apply(plan, x, nrhs=1):
    """_reduced_apply! (assembly.jl:905-915)."""
    return _vector_call(L.lib().grico_reduced_apply, plan, x, None, plan.n_reduced, nrhs)


def _dirichlet_components(entry, dof, coef, target, rank_tol=1e-8, noise_tol=1e-11):
    """Fixed dofs and relation rows from the multi-term trace rows left after substituting the
    fixed dofs, per connected component of the row-dof graph.  The reference's steps
    (`_dirichlet_constraint_system` and `_dirichlet_relations`, plans.jl:884-972: rank of the
    trace system, pivot dofs by QR with column pivoting, coupling -P^-1 C_free, a pivot without
    coupling becomes a fixed dof) are taken on the trace rows themselves rather than on their
    Gram matrix: hanging-node expansions on deep hp meshes reach coefficients of 1e5-1e6, whose
    squares would push a Gram rank tolerance above genuine constraints.  Rows are scaled to unit
    max norm; the rank is the count of |R_kk| > rank_tol |R_00| of the pivoted QR (on the hp
    L-shape dependent rows stay below 1e-12 and genuine ones above 1e-5); row terms below
    noise_tol of the row's largest, and rows below noise_tol of the component's largest, are
    rounding residue and are dropped first; coupling entries
    below 1e-14 of their row's largest are dropped.  The affine space is the one the reference's
    projection defines.  Returns (fixed dofs, values, [(pivot, dofs, coefs, rhs)])."""
    import scipy.linalg as sla
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    rows_u, row_inv = np.unique(entry, return_inverse=True)
    dofs_u, dof_inv = np.unique(dof, return_inverse=True)
    nr, nd = rows_u.size, dofs_u.size
    graph = coo_matrix((np.ones(row_inv.size), (row_inv, nr + dof_inv)), shape=(nr + nd, nr + nd))
    _, label = connected_components(graph, directed=False)
    fixed, values, rel = [], [], []
    row_lab, dof_lab = label[:nr], label[nr:]
    term_lab = row_lab[row_inv]
    for comp in np.unique(dof_lab):
        r_idx = np.nonzero(row_lab == comp)[0]
        d_idx = np.nonzero(dof_lab == comp)[0]          # ascending dof order
        rpos = np.full(nr, -1, dtype=np.int64)
        rpos[r_idx] = np.arange(r_idx.size)
        dpos = np.full(nd, -1, dtype=np.int64)
        dpos[d_idx] = np.arange(d_idx.size)
        sel = term_lab == comp
        A = np.zeros((r_idx.size, d_idx.size))
        np.add.at(A, (rpos[row_inv[sel]], dpos[dof_inv[sel]]), coef[sel])
        b = target[rows_u[r_idx]].astype(np.float64)
        scale = np.max(np.abs(A), axis=1)
        # rounding residue of long hanging-node elimination chains: terms ~1e-14 of their row's
        # largest, and whole rows whose terms all cancelled to that level (e.g. 1e-15 against
        # coefficients of order 1 elsewhere); scaled to unit norm they would pose as constraints
        A[np.abs(A) <= noise_tol * scale[:, None]] = 0.0
        keep = scale > noise_tol * (float(scale.max()) if scale.size else 0.0)
        A, b, scale = A[keep], b[keep], scale[keep]
        if not A.size:
            continue
        A /= scale[:, None]
        b = b / scale
        Qm, R, perm = sla.qr(A, pivoting=True, mode="economic")
        diag = np.abs(np.diag(R))
        count = int(np.sum(diag > rank_tol * diag[0])) if diag.size and diag[0] > 0 else 0
        if count == 0:
            continue
        tb = Qm.T @ b
        if np.any(np.abs(tb[count:]) > 1e-8 * max(float(np.linalg.norm(b)), 1.0)):
            raise ValueError("Dirichlet data is inconsistent on the selected boundary faces")
        piv = perm[:count]
        rest = perm[count:]
        order = np.argsort(rest, kind="stable")
        free = rest[order]                              # free columns in dof order
        R11 = R[:count, :count]
        shift = sla.solve_triangular(R11, tb[:count])
        coupling = (-sla.solve_triangular(R11, R[:count, count:][:, order]) if free.size
                    else np.zeros((count, 0)))
        gdofs = dofs_u[d_idx]
        for k in range(count):
            row = coupling[k]
            big = np.abs(row) > 1e-14 * max(1.0, float(np.max(np.abs(row))) if row.size else 1.0)
            pivot = int(gdofs[piv[k]])
            if not big.any():
                fixed.append(pivot)
                values.append(float(shift[k]))
            else:
                rel.append((pivot, gdofs[free[big]].astype(np.int64), row[big].astype(np.float64), float(shift[k])))
    return np.array(fixed, dtype=np.int64), np.array(values, dtype=np.float64), rel


def _source_points(plan, problem=None):
    """Per-point source values: f at the cell points of every tensor batch, then per point
    batch f at cell-item points or the Nitsche data g at face/surface points."""
    problem = problem or plan.problem
    arrays = []
    for b in plan.batches:
        if problem.rhs_operators:
            f = np.zeros(b.points.shape[:2])
            for op in problem.rhs_operators:
                f += np.asarray(op.source(b.points.reshape(-1, plan.D)), dtype=np.float64).reshape(f.shape)
            arrays.append(np.ascontiguousarray(f))
        else:
            arrays.append(None)
    for b in plan.point_batches:
        if b.kind == L.GRICO_ITEM_SUBCELLS:
            if problem.rhs_operators:
                parts = []
                for X, _, _, _ in _subcell_point_chunks(b):
                    f = np.zeros(X.shape[0])
                    for op in problem.rhs_operators:
                        f += np.asarray(op.source(X), dtype=np.float64).reshape(-1)
                    parts.append(f)
                arrays.append(np.ascontiguousarray(np.concatenate(parts)) if parts else None)
            else:
                arrays.append(None)
        elif b.kind == L.GRICO_ITEM_CELL:
            if problem.rhs_operators:
                f = np.zeros(b.points.shape[0])
                for op in problem.rhs_operators:
                    f += np.asarray(op.source(b.points), dtype=np.float64).reshape(-1)
                arrays.append(np.ascontiguousarray(f))
            else:
                arrays.append(None)
        elif b.kind == L.GRICO_ITEM_INTERFACE:
            arrays.append(None)  # interior interfaces carry no load
        else:
            g = np.zeros(b.points.shape[0])
            any_data = False
            for k, fn in enumerate(b.data):
                if fn is None:
                    continue
                lo, hi = b.point_offsets[k], b.point_offsets[k + 1]
                if hi > lo:
                    g[lo:hi] = np.asarray(fn(b.points[lo:hi]), dtype=np.float64).reshape(-1)
                any_data = True
            arrays.append(np.ascontiguousarray(g) if any_data else None)
    return arrays


def rhs(plan):
    """Full-layout right-hand side rhs! (assembly.jl:488-507): the load vector with the
    constraint rows' right-hand sides written in (fixed values, relation rhs)."""
    if isinstance(plan, AffineProblem):
        plan = compile(plan)
    arrays = _source_points(plan)
    ptrs = (L.f64p * len(arrays))(*[L.ptr(a, C.c_double) if a is not None else None for a in arrays])
    out = np.zeros(plan.n_full)
    L.check(L.lib().grico_rhs(plan.handle, ptrs, L.ptr(out, C.c_double), L.GRICO_FLAG_HOST_POINTERS), "rhs")
    return out


def reduced_rhs(plan):
    """Reduced right-hand side P^T (b - A shift) (assembly.jl:917-933)."""
    arrays = _source_points(plan)
    ptrs = (L.f64p * len(arrays))(*[L.ptr(a, C.c_double) if a is not None else None for a in arrays])
    out = np.zeros(plan.n_reduced)
    L.check(L.lib().grico_reduced_rhs(plan.handle, ptrs, L.ptr(out, C.c_double), L.GRICO_FLAG_HOST_POINTERS), "rhs")
    return out


def reduced_diagonal(plan):
    out = np.zeros(plan.n_reduced)
    L.check(L.lib().grico_reduced_diagonal(plan.handle, L.ptr(out, C.c_double), L.GRICO_FLAG_HOST_POINTERS), "diagonal")
    return out


def expand_reduced(plan, ured):
    ured = np.ascontiguousarray(ured, dtype=np.float64)
    out = np.zeros(plan.n_full)
    L.check(L.lib().grico_expand_reduced(plan.handle, L.ptr(ured, C.c_double), L.ptr(out, C.c_double),
                                         L.GRICO_FLAG_HOST_POINTERS), "expand")
    return out


class IdentityPreconditioner:
    code = L.GRICO_PRECOND_IDENTITY


class JacobiPreconditioner:
    code = L.GRICO_PRECOND_JACOBI


class CGSolver:
    def __init__(self, preconditioner=None):
        self.preconditioner = preconditioner or IdentityPreconditioner()


class FGMRESSolver:
    def __init__(self, preconditioner=None, restart=30):
        self.preconditioner = preconditioner or IdentityPreconditioner()
        self.restart = int(restart)


class State:
    def __init__(self, plan, coefficients, report=None):
        self.plan = plan
        self.coefficients = coefficients
        self.report = report


def solve(plan_or_problem, solver=None, relative_tolerance=None, absolute_tolerance=0.0, maxiter=None,
          initial_solution=None, graph=True):
    """solve(plan; solver=CGSolver(...)) on the reduced system (solve.jl:229-276).  `graph=False`
    launches each CG iteration op by op instead of replaying it as a CUDA graph."""
    from .multigrid import GeometricMultigridPreconditioner, build_multigrid

    plan = plan_or_problem if isinstance(plan_or_problem, AssemblyPlan) else compile(plan_or_problem)
    solver = solver or CGSolver(JacobiPreconditioner())
    rtol = math.sqrt(np.finfo(np.float64).eps) if relative_tolerance is None else float(relative_tolerance)
    maxiter = max(1000, 2 * plan.n_reduced) if maxiter is None else int(maxiter)
    b = reduced_rhs(plan)
    x = np.zeros(plan.n_reduced) if initial_solution is None else np.array(initial_solution, dtype=np.float64)
    mg = None
    pre = solver.preconditioner
    if isinstance(pre, GeometricMultigridPreconditioner):
        from .multigrid import resolved_smoother

        if isinstance(solver, CGSolver):
            if not isinstance(plan.problem.operator_class, SPD):
                raise ValueError("CG with GeometricMultigridPreconditioner requires an SPD affine problem; "
                                 "use FGMRESSolver")  # multigrid.jl:248-251
            if resolved_smoother(pre, plan.problem) == "gmres":
                raise ValueError("CG with GeometricMultigridPreconditioner requires the Jacobi smoother; "
                                 "use FGMRESSolver for nonsymmetric smoother policies")  # multigrid.jl:253-255
        mg = build_multigrid(plan, pre)
        code = L.GRICO_PRECOND_MULTIGRID
    else:
        code = pre.code
    opts = L.GricoSolveOptions(rtol, float(absolute_tolerance), int(min(maxiter, 2**31 - 1)), code,
                               getattr(solver, "restart", 30), 0 if initial_solution is None else 1)
    rep = L.GricoSolveReport()
    fn = L.lib().grico_cg_solve if isinstance(solver, CGSolver) else L.lib().grico_fgmres_solve
    L.check(fn(plan.handle, mg.handle if mg is not None else None, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
               C.byref(opts), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS | (0 if graph else L.GRICO_FLAG_NO_GRAPH)),
            "solve")
    return State(plan, expand_reduced(plan, x), rep)


def _quadrature_chunks(plan, full_values=None):
    """(weights, physical points, u at the points or None) over every cell rule: tensor batches,
    cell point items and subcell items (verification.jl:201-230 integrates over the same rules)."""
    x = None if full_values is None else np.asarray(full_values, dtype=np.float64)
    D = plan.D
    vals = _point_values(plan, x) if x is not None else [None] * len(plan.batches)
    for b, u in zip(plan.batches, vals):
        yield _point_weights(plan, b).reshape(-1), b.points.reshape(-1, D), None if u is None else u.reshape(-1)
    for b in plan.point_batches:
        if b.kind == L.GRICO_ITEM_CELL:
            u = None
            if x is not None:
                loc = _local_coefficients(b, x)
                item = np.repeat(np.arange(len(b.cells)), np.diff(b.point_offsets))
                u = _eval_at(b, loc, item, b.ref_points)
            yield b.weights, b.points, u
        elif b.kind == L.GRICO_ITEM_SUBCELLS:
            loc = _local_coefficients(b, x) if x is not None else None
            for X, w, item, xi in _subcell_point_chunks(b):
                yield w, X, (_eval_at(b, loc, item, xi) if loc is not None else None)


def _eval_at(b, loc, item, ref):
    """u at reference points `ref` of the items `item` from their local coefficients."""
    D = ref.shape[1]
    phi = np.ones((ref.shape[0], 1))
    for a in range(D):
        va, _ = fe_basis_table(ref[:, a], b.degree[a])
        # box index axis 1 fastest: new = old + stride * m_a
        phi = (va[:, :, None] * phi[:, None, :]).reshape(phi.shape[0], -1)
    return np.einsum("pm,pm->p", phi, loc[item])


def _quadrature_sets(plan):
    """(weights, physical points) of every cell rule."""
    return [(w, X) for w, X, _ in _quadrature_chunks(plan)]


def l2_error(state, exact):
    """Quadrature L2 error on the cell rules, cut-cell rules included (verification.jl:201-230,
    270-275)."""
    err2 = 0.0
    for w, X, u in _quadrature_chunks(state.plan, state.coefficients):
        ex = np.asarray(exact(X), dtype=np.float64).reshape(-1)
        err2 += float(np.sum(w * (u - ex) ** 2))
    return math.sqrt(err2)


def relative_l2_error(state, exact):
    num = l2_error(state, exact)
    den2 = 0.0
    for w, X, _ in _quadrature_chunks(state.plan):
        ex = np.asarray(exact(X), dtype=np.float64).reshape(-1)
        den2 += float(np.sum(w * ex ** 2))
    return num / math.sqrt(den2) if den2 > 0 else num


def _local_coefficients(b, x):
    n = len(b.cells)
    mp = b.map_index.reshape(n, b.nbox)
    loc = np.where(mp >= 0, x[np.maximum(mp, 0)], 0.0)
    if b.map_coef is not None:
        loc = loc * b.map_coef.reshape(n, b.nbox)
    if b.tail_offsets is not None:
        rows, cols = np.nonzero(mp <= -2)
        for r, c in zip(rows, cols):
            k = -(int(mp[r, c]) + 2)
            lo, hi = b.tail_offsets[k], b.tail_offsets[k + 1]
            loc[r, c] = float(np.dot(b.tail_coef[lo:hi], x[b.tail_index[lo:hi]]))
    return loc


def _point_weights(plan, b):
    D = plan.D
    w1 = [b.rules[a][1] for a in range(D)]
    grids = np.meshgrid(*w1, indexing="ij")
    ref = np.prod(np.stack([g.reshape(-1, order="F") for g in grids], axis=1), axis=1)
    det = np.prod(0.5 * b.h, axis=1)
    return det[:, None] * ref[None, :]


def _point_values(plan, full_values):
    """u at the quadrature points, [n_cells, nq] per batch with points axis 1 fastest."""
    x = np.asarray(full_values, dtype=np.float64)
    D = plan.D
    out = []
    for b in plan.batches:
        n = len(b.cells)
        loc = _local_coefficients(b, x)
        # box index is axis 1 fastest: t axes are [cell, mD, ..., m1]; contract m_a with B_a
        t = loc.reshape([n] + [b.degree[a] + 1 for a in reversed(range(D))])
        for a in range(D):
            ax = D - a  # position of axis a
            t = np.moveaxis(np.tensordot(t, b.rules[a][2], axes=([ax], [0])), -1, ax)
        # now axes [cell, qD, ..., q1] -> flatten with q1 fastest (C order on reversed axes)
        out.append(t.reshape(n, -1))
    return out

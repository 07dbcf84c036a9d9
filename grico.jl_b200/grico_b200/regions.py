"""Finite-cell physical domains and embedded surfaces (host side of the mirror).

Mirrors `ImplicitRegion`, `PhysicalDomain`, `FiniteCellExtension`, `finite_cell_quadrature`
and the cut-cell quadrature of regions.jl:

* classification samples the classifier at the 2^D corners and the centre of a (sub)cell
  (regions.jl:736-757): no negative sample = outside, no positive sample = inside, else cut;
  Bool classifiers read true as inside (regions.jl:819-830);
* `:outside` leaves leave the space (regions.jl:267-279);
* cut leaves get the octree candidate rule of regions.jl:466-510 and 759-817 in the same
  depth-first order: inside subcells contribute the mapped tensor rule, cut subcells split until
  `subdivision_depth`, terminal cut subcells keep their points with negative classifier value
  and fall back to the negative corner/centre samples when none is left;
* `quadrature="moment_fitted"` then reduces the candidates with the reference's non-negative
  moment fit (regions.jl:519-708: Legendre moments up to the quadrature shape, Lawson-Hanson
  NNLS on SVD subproblems, greedy point elimination); the default `"candidates"` keeps the
  unfitted candidate set.

All classification and candidate generation is vectorised over every cut cell (and every
subcell of one depth) at once.  Classifiers receive an [n, D] array of physical points and
return n values.
"""
from __future__ import annotations

import numpy as np

from .mesh import Domain

MAX_TERMINAL_SUBCELLS = 1 << 20        # regions.jl:451
MOMENT_TOLERANCE = 1.0e3 * np.finfo(np.float64).eps   # regions.jl:513-517
WEIGHT_PRUNE_RATIO = 1.0e-8
MAX_ELIMINATION_ITERATIONS = 1024


def classifier_values(classifier, X):
    """regions.jl:819-830 on an [n, D] array of physical points."""
    v = np.asarray(classifier(X))
    if v.dtype == bool:
        return np.where(v, -1.0, 1.0)
    if not np.issubdtype(v.dtype, np.number):
        raise ValueError("finite-cell classifiers must return Bool or Real values")
    v = v.astype(np.float64).reshape(-1)
    if not np.all(np.isfinite(v)):
        raise ValueError("finite-cell classifier values must be finite")
    return v


def _check_depth(depth, D):
    if not isinstance(depth, (int, np.integer)) or depth < 0:
        raise ValueError("subdivision_depth must be a non-negative integer")
    terminal = 1
    for _ in range(int(depth)):
        if terminal > MAX_TERMINAL_SUBCELLS // (1 << D):
            raise ValueError("subdivision_depth creates too many finite-cell subcells")
        terminal *= 1 << D


class ImplicitRegion:
    def __init__(self, classifier, subdivision_depth=2):
        if not isinstance(subdivision_depth, (int, np.integer)) or subdivision_depth < 0 \
                or subdivision_depth > 60:
            raise ValueError("subdivision_depth must be a non-negative integer")
        self.classifier = classifier
        self.subdivision_depth = int(subdivision_depth)


class PhysicalMeasure:
    pass


class FiniteCellExtension:
    """Cut cells integrate (1 - alpha) * physical + alpha * full cell (regions.jl:57-81, 352-381)."""

    def __init__(self, alpha):
        alpha = float(alpha)
        if not 0.0 <= alpha <= 1.0:
            raise ValueError("alpha must lie in [0, 1]")
        self.alpha = alpha


def _corner_bits(D):
    return np.array([[(m >> a) & 1 for a in range(D)] for m in range(1 << D)], dtype=bool)


def _tensor_rule(qshape, gauss):
    """Tensor points [nq, D] (axis 1 fastest) and weights [nq] on [-1, 1]^D."""
    D = len(qshape)
    rules = [gauss(int(q)) for q in qshape]
    grids = np.meshgrid(*[r[0] for r in rules], indexing="ij")
    wgrid = np.meshgrid(*[r[1] for r in rules], indexing="ij")
    pts = np.stack([g.reshape(-1, order="F") for g in grids], axis=1)
    w = np.ones(pts.shape[0])
    for a in range(D):
        w = w * wgrid[a].reshape(-1, order="F")
    return pts, w


class PhysicalDomain:
    """Background Domain plus an implicit region (regions.jl:125-196)."""

    def __init__(self, background: Domain, region: ImplicitRegion, cell_measure=None,
                 quadrature="candidates"):
        if quadrature not in ("candidates", "moment_fitted"):
            raise ValueError("quadrature must be 'candidates' or 'moment_fitted'")
        cell_measure = cell_measure if cell_measure is not None else PhysicalMeasure()
        if not isinstance(cell_measure, (PhysicalMeasure, FiniteCellExtension)):
            raise ValueError("cell_measure must be an AbstractCellMeasure")
        _check_depth(region.subdivision_depth, background.D)
        self.background = background
        self.region = region
        self.cell_measure = cell_measure
        self.quadrature = quadrature
        self.grid = background.grid
        self.D = background.D
        self.origin, self.extent = background.origin, background.extent

    def cell_size(self, cells):
        return self.background.cell_size(cells)

    def cell_lower(self, cells):
        return self.background.cell_lower(cells)

    def map_from_biunit(self, cells, xi):
        """center + xi * half per axis (geometry.jl:571-578, 706-711)."""
        h = self.cell_size(cells)
        half = 0.5 * h
        return (self.cell_lower(cells) + half) + xi * half

    def classify(self, cells, lower=None, upper=None):
        """0 outside, 1 inside, 2 cut for each (cell, reference subcell [lower, upper])."""
        cells = np.asarray(cells, dtype=np.int64)
        n, D = len(cells), self.D
        if n == 0:
            return np.zeros(0, dtype=np.int64)
        lower = -np.ones((n, D)) if lower is None else lower
        upper = np.ones((n, D)) if upper is None else upper
        bits = _corner_bits(D)
        xi = np.where(bits[None, :, :], upper[:, None, :], lower[:, None, :])      # [n, 2^D, D]
        mid = 0.5 * (lower + upper)
        xi = np.concatenate([xi, mid[:, None, :]], axis=1)
        S = xi.shape[1]
        X = self.map_from_biunit(np.repeat(cells, S), xi.reshape(-1, D))
        v = classifier_values(self.region.classifier, X).reshape(n, S)
        neg = np.any(v < 0.0, axis=1)
        pos = np.any(v > 0.0, axis=1)
        return np.where(~neg, 0, np.where(~pos, 1, 2)).astype(np.int64)

    def active_leaves(self):
        leaves = self.grid.active_leaves()
        cls = self.classify(leaves)
        keep = leaves[cls != 0]
        if keep.size == 0:
            raise ValueError("physical domains must contain at least one active physical leaf")
        return keep

    # ------------------------------------------------------------------------------------
    def candidate_quadrature(self, cells, qshape, gauss, chunk=4096):
        """Unfitted candidate rules of cut cells sharing one quadrature shape.

        Returns (offsets [n+1], xi [P, D], w [P]) with each cell's points in the depth-first
        order of regions.jl:477-510."""
        cells = np.asarray(cells, dtype=np.int64)
        offs = [np.zeros(1, dtype=np.int64)]
        pts, wts = [], []
        base = 0
        for s in range(0, len(cells), chunk):
            o, x, w = self._candidates_chunk(cells[s:s + chunk], qshape, gauss)
            offs.append(o[1:] + base)
            base += int(o[-1])
            pts.append(x)
            wts.append(w)
        return (np.concatenate(offs), np.concatenate(pts) if pts else np.zeros((0, self.D)),
                np.concatenate(wts) if wts else np.zeros(0))

    def _candidates_chunk(self, cells, qshape, gauss):
        D = self.D
        B = 1 << D
        maxd = self.region.subdivision_depth
        eta, ew = _tensor_rule(qshape, gauss)
        nq = len(ew)
        bits = _corner_bits(D)
        n = len(cells)
        cid = np.arange(n)
        lower = -np.ones((n, D))
        upper = np.ones((n, D))
        key = np.zeros(n, dtype=np.int64)
        blocks = []   # (cid [m], key [m], order [m], xi [m, D], w [m])
        for depth in range(maxd + 1):
            if cid.size == 0:
                break
            cls = self.classify(cells[cid], lower, upper)
            terminal = depth >= maxd
            center = 0.5 * (lower + upper)
            half = 0.5 * (upper - lower)
            scale = np.prod(half, axis=1)
            emit = np.nonzero((cls == 1) | ((cls == 2) & terminal))[0]
            if emit.size:
                xi = center[emit, None, :] + half[emit, None, :] * eta[None, :, :]     # [m, nq, D]
                w = (ew[None, :] * scale[emit, None])
                keep = np.ones((emit.size, nq), dtype=bool)
                cut = cls[emit] == 2
                if np.any(cut):
                    ci = np.nonzero(cut)[0]
                    X = self.map_from_biunit(np.repeat(cells[cid[emit[ci]]], nq), xi[ci].reshape(-1, D))
                    keep[ci] = (classifier_values(self.region.classifier, X) < 0.0).reshape(len(ci), nq)
                order = np.broadcast_to(np.arange(nq)[None, :], (emit.size, nq))
                blocks.append((np.repeat(cid[emit], nq)[keep.reshape(-1)], np.repeat(key[emit], nq)[keep.reshape(-1)],
                               order[keep], xi[keep], w[keep]))
                empty = np.nonzero(cut & ~np.any(keep, axis=1))[0]
                if empty.size:
                    self._sliver_fallback(blocks, cells, cid[emit[empty]], key[emit[empty]],
                                          lower[emit[empty]], upper[emit[empty]])
            split = np.nonzero((cls == 2) & (not terminal))[0]
            if split.size == 0:
                break
            mid = center[split]
            weight = B ** (maxd - depth - 1)
            lo = np.where(bits[None, :, :], mid[:, None, :], lower[split, None, :]).reshape(-1, D)
            hi = np.where(bits[None, :, :], upper[split, None, :], mid[:, None, :]).reshape(-1, D)
            key = (key[split, None] + np.arange(B)[None, :] * weight).reshape(-1)
            cid = np.repeat(cid[split], B)
            lower, upper = lo, hi
        if not blocks:
            return np.zeros(n + 1, dtype=np.int64), np.zeros((0, D)), np.zeros(0)
        c = np.concatenate([b[0] for b in blocks])
        k = np.concatenate([b[1] for b in blocks])
        o = np.concatenate([b[2] for b in blocks])
        x = np.concatenate([b[3] for b in blocks])
        w = np.concatenate([b[4] for b in blocks])
        perm = np.lexsort((o, k, c))
        counts = np.bincount(c, minlength=n)
        return np.concatenate([[0], np.cumsum(counts)]).astype(np.int64), x[perm], w[perm]

    def subcell_quadrature(self, cells, qshape, gauss, chunk=8192):
        """The candidate rule of cut cells as octree subcells (the representation the subcell
        kernel integrates by sum factorisation): per cell, in depth-first order, the inside
        subcells and the terminal cut subcells with a keep mask over the qshape tensor points
        (bit p, axis 1 fastest).  Returns (offsets [n+1], level [S], pos [S, D], mask [S] uint64,
        weight factor [S] = 2^(-D level), slivers) where slivers maps a cell index to the
        explicit (points, weights) of the sliver fallback (regions.jl:794-817)."""
        cells = np.asarray(cells, dtype=np.int64)
        D = self.D
        nq = int(np.prod(qshape))
        if nq > 64:
            raise ValueError("subcell masks hold at most 64 points")
        maxd = self.region.subdivision_depth
        B = 1 << D
        eta, _ = _tensor_rule(qshape, gauss)
        bits = _corner_bits(D)
        pw = (np.uint64(1) << np.arange(nq, dtype=np.uint64))
        out_c, out_k, out_lev, out_pos, out_mask = [], [], [], [], []
        slivers = {}
        for s0 in range(0, len(cells), chunk):
            cc = cells[s0:s0 + chunk]
            n = len(cc)
            cid = np.arange(n)
            lower = -np.ones((n, D))
            upper = np.ones((n, D))
            key = np.zeros(n, dtype=np.int64)
            for depth in range(maxd + 1):
                if cid.size == 0:
                    break
                cls = self.classify(cc[cid], lower, upper)
                terminal = depth >= maxd
                center = 0.5 * (lower + upper)
                half = 0.5 * (upper - lower)
                emit = np.nonzero((cls == 1) | ((cls == 2) & terminal))[0]
                if emit.size:
                    keep = np.ones((emit.size, nq), dtype=bool)
                    cut = np.nonzero(cls[emit] == 2)[0]
                    if cut.size:
                        xi = center[emit[cut], None, :] + half[emit[cut], None, :] * eta[None, :, :]
                        X = self.map_from_biunit(np.repeat(cc[cid[emit[cut]]], nq), xi.reshape(-1, D))
                        keep[cut] = (classifier_values(self.region.classifier, X) < 0.0).reshape(cut.size, nq)
                    has = np.any(keep, axis=1)
                    e2 = emit[has]
                    out_c.append(cid[e2] + s0)
                    out_k.append(key[e2])
                    out_lev.append(np.full(e2.size, depth, dtype=np.int32))
                    out_pos.append(np.rint((lower[e2] + 1.0) * (2.0 ** (depth - 1))).astype(np.int32))
                    out_mask.append((keep[has].astype(np.uint64) * pw[None, :]).sum(axis=1, dtype=np.uint64))
                    empty = emit[~has]
                    if empty.size:
                        blocks = []
                        self._sliver_fallback(blocks, cc, cid[empty], key[empty], lower[empty], upper[empty])
                        bc, _, _, bx, bw = blocks[0]
                        for c in np.unique(bc):
                            sel = bc == c
                            prev = slivers.get(int(c) + s0)
                            pts, wts = bx[sel], bw[sel]
                            if prev is not None:
                                pts, wts = np.concatenate([prev[0], pts]), np.concatenate([prev[1], wts])
                            slivers[int(c) + s0] = (pts, wts)
                split = np.nonzero((cls == 2) & (not terminal))[0]
                if split.size == 0:
                    break
                mid = center[split]
                weight = B ** (maxd - depth - 1)
                lo = np.where(bits[None, :, :], mid[:, None, :], lower[split, None, :]).reshape(-1, D)
                hi = np.where(bits[None, :, :], upper[split, None, :], mid[:, None, :]).reshape(-1, D)
                key = (key[split, None] + np.arange(B)[None, :] * weight).reshape(-1)
                cid = np.repeat(cid[split], B)
                lower, upper = lo, hi
        if out_c:
            c = np.concatenate(out_c)
            k = np.concatenate(out_k)
            perm = np.lexsort((k, c))
            lev = np.concatenate(out_lev)[perm]
            pos = np.concatenate(out_pos)[perm].reshape(-1, D)
            mask = np.concatenate(out_mask)[perm]
            counts = np.bincount(c, minlength=len(cells))
        else:
            lev = np.zeros(0, dtype=np.int32)
            pos = np.zeros((0, D), dtype=np.int32)
            mask = np.zeros(0, dtype=np.uint64)
            counts = np.zeros(len(cells), dtype=np.int64)
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        ws = np.ldexp(1.0, -D * lev.astype(np.int64))
        return off, lev, np.ascontiguousarray(pos, dtype=np.int32), mask, ws, slivers

    def _sliver_fallback(self, blocks, cells, cid, key, lower, upper):
        """regions.jl:794-817: centre then corners with negative values, weight vol/(2^D+1)."""
        D = self.D
        bits = _corner_bits(D)
        m = len(cid)
        center = 0.5 * (lower + upper)
        corners = np.where(bits[None, :, :], upper[:, None, :], lower[:, None, :])
        samples = np.concatenate([center[:, None, :], corners], axis=1)   # [m, S, D]
        S = samples.shape[1]
        X = self.map_from_biunit(np.repeat(cells[cid], S), samples.reshape(-1, D))
        neg = (classifier_values(self.region.classifier, X) < 0.0).reshape(m, S)
        sw = np.prod(upper - lower, axis=1) / S
        order = np.broadcast_to(np.arange(S)[None, :], (m, S))
        blocks.append((np.repeat(cid, S)[neg.reshape(-1)], np.repeat(key, S)[neg.reshape(-1)], order[neg],
                       samples[neg], np.repeat(sw, S)[neg.reshape(-1)]))

    def cut_cell_quadrature(self, cells, qshape, gauss):
        """Per-cell (xi, w) of the assembly rule of cut cells (regions.jl:297-381)."""
        off, xi, w = self.candidate_quadrature(cells, qshape, gauss)
        out = []
        meas = self.cell_measure
        if isinstance(meas, FiniteCellExtension) and meas.alpha == 1.0:
            raise ValueError("cells with alpha = 1 use the tensor rule")
        full = _tensor_rule(qshape, gauss) if isinstance(meas, FiniteCellExtension) else None
        for i in range(len(cells)):
            p, q = xi[off[i]:off[i + 1]], w[off[i]:off[i + 1]]
            if p.shape[0] == 0:
                out.append(None)
                continue
            if self.quadrature == "moment_fitted":
                p, q = moment_fit(p, q, qshape)
            if full is not None and meas.alpha > 0.0:
                p = np.concatenate([p, full[0]])
                q = np.concatenate([(1.0 - meas.alpha) * q, meas.alpha * full[1]])
            out.append((p, q))
        return out


def finite_cell_quadrature(domain: Domain, leaf, qshape, classifier, subdivision_depth=2):
    """finite_cell_quadrature(domain, leaf, quadrature_shape, classifier) (regions.jl:407-413):
    None when outside, the tensor rule (as points, weights) when inside, else the moment-fitted
    cut rule."""
    from .problem import _gauss

    region = ImplicitRegion(classifier, subdivision_depth=subdivision_depth)
    pd = PhysicalDomain(domain, region, quadrature="moment_fitted")
    leaf = np.array([int(leaf)])
    cls = int(pd.classify(leaf)[0])
    if cls == 0:
        return None
    if cls == 1:
        return _tensor_rule(qshape, _gauss)
    return pd.cut_cell_quadrature(leaf, qshape, _gauss)[0]


# ----------------------------------------------------------------------------------------
# moment fitting (regions.jl:519-708)
# ----------------------------------------------------------------------------------------

def _legendre_table(x, n):
    """P_0..P_n at points x: [len(x), n+1] by the three-term recurrence."""
    out = np.ones((len(x), n + 1))
    if n >= 1:
        out[:, 1] = x
    for k in range(2, n + 1):
        out[:, k] = ((2 * k - 1) * x * out[:, k - 1] - (k - 1) * out[:, k - 2]) / k
    return out


def moment_matrix(points, degrees):
    """[prod(degrees+1), n] full-tensor Legendre products, axis 1 fastest in the mode index."""
    D = points.shape[1]
    tabs = [_legendre_table(points[:, a], degrees[a]) for a in range(D)]
    mat = np.ones((1, points.shape[0]))
    for a in range(D):
        # new index = old + stride * m_a with axis 1 fastest
        mat = (tabs[a].T[:, None, :] * mat[None, :, :]).reshape(-1, points.shape[0])
    return mat


def _lstsq_min_norm(A, b, tol):
    if A.size == 0:
        return np.zeros(A.shape[1])
    U, S, Vt = np.linalg.svd(A, full_matrices=False)
    if S.size == 0:
        return np.zeros(A.shape[1])
    cut = tol * S[0]
    r = U.T @ b
    scaled = np.where(S > cut, r / np.where(S > cut, S, 1.0), 0.0)
    return Vt.T @ scaled


def nnls(A, b, tol):
    """Active-set NNLS as regions.jl:605-683; returns (x, relative residual)."""
    n = A.shape[1]
    x = np.zeros(n)
    passive = np.zeros(n, dtype=bool)
    grad = A.T @ b
    it = 0
    while it < max(8 * n, 32):
        cand = -1
        best = 0.0
        for i in range(n):
            if not passive[i] and grad[i] > best:
                best = grad[i]
                cand = i
        if cand < 0 or not grad[cand] > tol:
            break
        passive[cand] = True
        while True:
            idx = np.nonzero(passive)[0]
            sol = _lstsq_min_norm(A[:, idx], b, tol)
            trial = np.zeros(n)
            trial[idx] = sol
            if np.all(sol > tol):
                x = trial
                break
            alpha = 1.0
            for i in idx:
                if trial[i] > tol:
                    continue
                den = x[i] - trial[i]
                if abs(den) <= tol:
                    continue
                alpha = min(alpha, x[i] / den)
            x = x + alpha * (trial - x)
            for i in idx:
                if x[i] <= tol:
                    x[i] = 0.0
                    passive[i] = False
            if not np.any(passive):
                break
        grad = A.T @ (b - A @ x)
        it += 1
    res = b - A @ x
    return x, np.linalg.norm(res) / max(np.linalg.norm(b), 1.0)


def moment_fit(points, weights, qshape):
    """Reduce a candidate rule to at most prod(qshape) points when the moments allow it."""
    qshape = tuple(int(q) for q in qshape)
    min_count = int(np.prod(qshape))
    if len(points) <= min_count:
        return points, weights
    A = moment_matrix(points, qshape)
    if A.shape[0] <= 1:
        return points, weights
    b = A @ weights
    tol = MOMENT_TOLERANCE
    full, res = nnls(A, b, tol)
    if not res <= tol:
        return points, weights
    cur = np.nonzero(full > tol)[0]
    if cur.size == 0:
        return points, weights
    cw = full[cur]
    if cur.size > A.shape[0]:
        order = np.argsort(-cw, kind="stable")
        cur = cur[order[:A.shape[0]]]
        cw, res = nnls(A[:, cur], b, tol)
        if not res <= tol:
            return points, weights
    prev, prev_w = cur.copy(), cw.copy()
    for _ in range(MAX_ELIMINATION_ITERATIONS):
        if len(cur) <= min_count:
            break
        thr = max(tol, WEIGHT_PRUNE_RATIO * np.max(cw))
        removable = np.nonzero(cw <= thr)[0]
        removable = [int(np.argmin(cw))] if removable.size == 0 else sorted(removable, key=lambda i: cw[i])
        accepted = False
        for li in removable:
            trial = np.delete(cur, li)
            if len(trial) < min_count:
                continue
            tw, r = nnls(A[:, trial], b, tol)
            if not r <= tol:
                continue
            cur, cw = trial, tw
            prev, prev_w = cur.copy(), cw.copy()
            accepted = True
            break
        if not accepted:
            break
    return points[prev], prev_w


# ----------------------------------------------------------------------------------------
# embedded surfaces
# ----------------------------------------------------------------------------------------

class SurfaceQuadrature:
    """SurfaceQuadrature(leaf, points, weights, normals) (embedded.jl:33-46, 97-106): biunit
    reference points, reference-surface weights and reference normals of one leaf.  Compilation
    maps them to physical weights det(J)/|J n| w and unit normals J^-1 n / |J^-1 n|
    (integration.jl:2338-2357, 2501-2516)."""

    def __init__(self, leaf, points, weights, normals):
        leaf = int(leaf)
        if leaf < 1:
            raise ValueError("leaf must be positive")
        pts = np.atleast_2d(np.asarray(points, dtype=np.float64))
        w = np.asarray(weights, dtype=np.float64).reshape(-1)
        nrm = np.asarray(normals, dtype=np.float64)
        if nrm.ndim == 1:
            nrm = np.tile(nrm, (pts.shape[0], 1))
        if pts.shape[0] != w.size or nrm.shape != pts.shape:
            raise ValueError("surface quadrature points, weights and normals must match")
        if np.any(~np.isfinite(w)) or np.any(w < 0):
            raise ValueError("surface quadrature weights must be finite and non-negative")
        if np.any(np.abs(pts) > 1.0 + 1e-12):
            raise ValueError("surface quadrature points must lie in the biunit cell")
        nn = np.linalg.norm(nrm, axis=1)
        if np.any(~(nn > 0)):
            raise ValueError("surface normals must be nonzero")
        self.leaf = leaf
        self.points = pts
        self.weights = w
        self.normals = nrm / nn[:, None]


def physical_surface_data(domain, leaf, surface):
    """(physical weights, physical unit normals) of one surface quadrature."""
    h = domain.cell_size(np.array([leaf]))[0]
    J = 0.5 * h
    detj = float(np.prod(J))
    mapped = surface.normals * J[None, :]
    w = surface.weights * (detj / np.sqrt(np.sum(mapped ** 2, axis=1)))
    t = surface.normals / J[None, :]
    n = t / np.sqrt(np.sum(t ** 2, axis=1))[:, None]
    return w, n


def _box_sphere_pieces(lo, hi, c, R, min_normal=0.3, max_depth=12):
    """Boxes covering [lo, hi] on which |x - c| is monotone along every axis and some axis k
    keeps |n_k| >= min_normal on the sphere (so the height function over the other axes has a
    bounded Jacobian): split at the planes x_a = c_a crossing the box, then bisect boxes that
    have no such axis.  Returns (lo, hi, k) triples; boxes the sphere misses are dropped."""
    boxes = [(lo.copy(), hi.copy())]
    for a in range(len(lo)):
        nxt = []
        for l, u in boxes:
            if l[a] < c[a] < u[a]:
                u1 = u.copy()
                u1[a] = c[a]
                l2 = l.copy()
                l2[a] = c[a]
                nxt += [(l, u1), (l2, u)]
            else:
                nxt.append((l, u))
        boxes = nxt
    out = []
    stack = [(l, u, 0) for l, u in boxes]
    D = len(lo)
    while stack:
        l, u, depth = stack.pop()
        near = np.clip(c, l, u)
        far = np.maximum(np.abs(l - c), np.abs(u - c))
        if np.linalg.norm(near - c) > R or np.linalg.norm(far) < R:
            continue
        mind = np.minimum(np.abs(l - c), np.abs(u - c))      # box does not straddle c_a
        k = int(np.argmax(mind))
        if mind[k] >= min_normal * R or depth >= max_depth:
            out.append((l, u, k))
            continue
        mid = 0.5 * (l + u)
        for mask in range(1 << D):
            bits = np.array([(mask >> a) & 1 for a in range(D)], dtype=bool)
            stack.append((np.where(bits, mid, l), np.where(bits, u, mid), depth + 1))
    return out


def _gauss_segments(a, b, breaks, gx, gw):
    """Composite Gauss points on [a, b] split at the interior breakpoints."""
    cuts = sorted(float(t) for t in breaks if a < t < b)
    edges = [a] + cuts + [b]
    xs, ws = [], []
    for s, e in zip(edges[:-1], edges[1:]):
        if e <= s:
            continue
        xs.append(0.5 * (s + e) + 0.5 * (e - s) * gx)
        ws.append(0.5 * (e - s) * gw)
    if not xs:
        return np.zeros(0), np.zeros(0)
    return np.concatenate(xs), np.concatenate(ws)


def _root(c, rho2, lo, hi):
    """x in [lo, hi] with (x - c)^2 = rho2 on the side of c that the interval lies on."""
    if rho2 < 0:
        return None
    r = np.sqrt(rho2)
    x = c + r if lo >= c else c - r
    return x if lo <= x <= hi else None


def _sphere_piece_3d(lo, hi, k, c, R, gx, gw):
    """Physical points and weights of the sphere inside one box on which |x - c| is monotone
    along every axis, as a height function along axis k over the other two axes.  Cartesian
    inner/outer Gauss rules unless the box touches both centre planes x_j = c_j and x_m = c_m
    (a box at the pole of axis k) and a circle x_k = const crosses it: there the boundary
    circles would be tangent to the box faces, so the polar rule is used."""
    rest = [a for a in range(3) if a != k]
    mind = np.minimum(np.abs(lo - c), np.abs(hi - c))
    if mind[rest[0]] > 0 or mind[rest[1]] > 0:
        return _sphere_piece_cartesian(lo, hi, k, c, R, gx, gw)
    dk = sorted((abs(lo[k] - c[k]), abs(hi[k] - c[k])))
    far = np.maximum(np.abs(lo - c), np.abs(hi - c))
    rho_big2 = R * R - dk[0] ** 2
    rho_small2 = R * R - dk[1] ** 2
    if rho_small2 <= 0 and rho_big2 >= far[rest[0]] ** 2 + far[rest[1]] ** 2:
        return _sphere_piece_cartesian(lo, hi, k, c, R, gx, gw)
    return _sphere_piece_polar(lo, hi, k, c, R, gx, gw)


def _sphere_piece_polar(lo, hi, k, c, R, gx, gw):
    """The pole-box case of _sphere_piece_3d, integrated in
    polar coordinates (r, phi) about the centre's projection.  In those coordinates the box
    faces x_k = lo_k, hi_k become circles r = const and the other faces become smooth graphs
    r(phi), so composite Gauss rules split at the few phi where a limit switches are exact up
    to the Gauss order (a closed-form instance of dimension reduction with height functions,
    R. I. Saye, SIAM J. Sci. Comput. 37 (2015) A993-A1019)."""
    j, m = [a for a in range(3) if a != k]
    sj = 1.0 if lo[j] >= c[j] else -1.0
    sm = 1.0 if lo[m] >= c[m] else -1.0
    sk = 1.0 if lo[k] >= c[k] else -1.0
    uj = sorted((sj * (lo[j] - c[j]), sj * (hi[j] - c[j])))
    um = sorted((sm * (lo[m] - c[m]), sm * (hi[m] - c[m])))
    dk = sorted((abs(lo[k] - c[k]), abs(hi[k] - c[k])))
    R2 = R * R
    if R2 - dk[0] ** 2 < 0:
        return np.zeros((0, 3)), np.zeros(0)
    rho_big = np.sqrt(R2 - dk[0] ** 2)
    rho_small = np.sqrt(max(R2 - dk[1] ** 2, 0.0))
    phi0 = np.arctan2(um[0], uj[1])
    phi1 = np.arctan2(um[1], uj[0])
    breaks = [np.arctan2(um[0], uj[0]), np.arctan2(um[1], uj[1])]
    for rho in (rho_small, rho_big):
        if rho <= 0:
            continue
        for e in uj:
            if e <= rho:
                breaks.append(np.arccos(e / rho))
        for e in um:
            if e <= rho:
                breaks.append(np.arcsin(e / rho))
    ph, wph = _gauss_segments(phi0, phi1, breaks, gx, gw)
    if ph.size == 0:
        return np.zeros((0, 3)), np.zeros(0)
    cs, sn = np.cos(ph), np.sin(ph)
    with np.errstate(divide="ignore", invalid="ignore"):
        lo_j = np.where(uj[0] > 0, uj[0] / cs, 0.0)
        lo_m = np.where(um[0] > 0, um[0] / sn, 0.0)
        hi_j = np.where(cs > 0, uj[1] / cs, np.inf)
        hi_m = np.where(sn > 0, um[1] / sn, np.inf)
    r_lo = np.maximum(rho_small, np.maximum(lo_j, lo_m))
    r_hi = np.minimum(rho_big, np.minimum(hi_j, hi_m))
    ok = r_hi > r_lo
    if not np.any(ok):
        return np.zeros((0, 3)), np.zeros(0)
    ph, wph, cs, sn, r_lo, r_hi = ph[ok], wph[ok], cs[ok], sn[ok], r_lo[ok], r_hi[ok]
    half = 0.5 * (r_hi - r_lo)
    r = (0.5 * (r_lo + r_hi))[:, None] + half[:, None] * gx[None, :]          # [nphi, q]
    hgt = np.sqrt(np.maximum(R2 - r * r, 0.0))
    w = (wph * half)[:, None] * gw[None, :] * r * (R / hgt)
    pts = np.zeros(r.shape + (3,))
    pts[..., j] = c[j] + sj * r * cs[:, None]
    pts[..., m] = c[m] + sm * r * sn[:, None]
    pts[..., k] = c[k] + sk * hgt
    return pts.reshape(-1, 3), w.reshape(-1)


def _sphere_piece_cartesian(lo, hi, k, c, R, gx, gw):
    """Height function t(x_j, x_m) along axis k: outer Gauss rule over x_m split where a
    boundary curve leaves the box through an x_j face, inner rule over x_j split at the
    circles x_k = lo_k, hi_k.  The inner axis j is the one farther from its centre plane."""
    rest = [a for a in range(3) if a != k]
    mind = np.minimum(np.abs(lo - c), np.abs(hi - c))
    j = rest[0] if mind[rest[0]] >= mind[rest[1]] else rest[1]
    m = rest[1] if j == rest[0] else rest[0]
    sk = 1.0 if lo[k] >= c[k] else -1.0
    R2 = R * R

    def rho2(t):  # squared radius of the circle cut from the sphere by x_k = t
        return R2 - (t - c[k]) ** 2

    breaks = []
    for tk in (lo[k], hi[k]):
        for tj in (lo[j], hi[j]):
            r = _root(c[m], rho2(tk) - (tj - c[j]) ** 2, lo[m], hi[m])
            if r is not None:
                breaks.append(r)
    xm, wm = _gauss_segments(lo[m], hi[m], breaks, gx, gw)
    P, W = [], []
    for xmv, wmv in zip(xm, wm):
        ib = []
        for tk in (lo[k], hi[k]):
            r = _root(c[j], rho2(tk) - (xmv - c[m]) ** 2, lo[j], hi[j])
            if r is not None:
                ib.append(r)
        xj, wj = _gauss_segments(lo[j], hi[j], ib, gx, gw)
        if xj.size == 0:
            continue
        r2 = R2 - (xj - c[j]) ** 2 - (xmv - c[m]) ** 2
        ok = r2 >= 0
        t = c[k] + sk * np.sqrt(np.where(ok, r2, 0.0))
        ok &= (t >= lo[k]) & (t <= hi[k])
        if not np.any(ok):
            continue
        xj, wj, t = xj[ok], wj[ok], t[ok]
        pts = np.zeros((xj.size, 3))
        pts[:, j] = xj
        pts[:, m] = xmv
        pts[:, k] = t
        P.append(pts)
        W.append(wmv * wj * R / np.abs(t - c[k]))       # |grad phi| / |d phi / d x_k|
    if not P:
        return np.zeros((0, 3)), np.zeros(0)
    return np.concatenate(P), np.concatenate(W)


def _circle_piece_2d(lo, hi, k, c, R, gx, gw):
    j = 1 - k
    sk = 1.0 if lo[k] >= c[k] else -1.0
    R2 = R * R
    breaks = []
    for tk in (lo[k], hi[k]):
        r = _root(c[j], R2 - (tk - c[k]) ** 2, lo[j], hi[j])
        if r is not None:
            breaks.append(r)
    xj, wj = _gauss_segments(lo[j], hi[j], breaks, gx, gw)
    rho2 = R2 - (xj - c[j]) ** 2
    ok = rho2 >= 0
    t = c[k] + sk * np.sqrt(np.where(ok, rho2, 0.0))
    ok &= (t >= lo[k]) & (t <= hi[k])
    pts = np.zeros((int(ok.sum()), 2))
    pts[:, j] = xj[ok]
    pts[:, k] = t[ok]
    return pts, wj[ok] * R / np.abs(t[ok] - c[k])


def _box_sphere_pieces_split(lo, hi, c, R):
    mid = 0.5 * (lo + hi)
    D = len(lo)
    out = []
    for mask in range(1 << D):
        bits = np.array([(mask >> a) & 1 for a in range(D)], dtype=bool)
        out += _box_sphere_pieces(np.where(bits, mid, lo), np.where(bits, hi, mid), c, R)
    return out


def sphere_surface_quadrature(space, center, radius, outward=True, points_per_axis=None, tolerance=1e-11,
                              max_depth=8):
    """SurfaceQuadrature items for the sphere (3-D) or circle (2-D) |x - center| = radius on
    every active leaf of `space` it crosses.  Each leaf's piece is integrated by composite
    Gauss rules (`points_per_axis` points per segment, default max degree + 2) on the height-
    function parametrisation of the surface, split at the points where the surface leaves the
    box, so that the rule is exact up to the Gauss order on each smooth piece; pieces whose
    area still changes by more than `tolerance` (relative) with 4 more points per segment (a
    boundary curve tangent to the box, near the poles) are bisected.  Normals point
    away from the centre when `outward` (the outer boundary of a ball), towards it otherwise
    (the inner boundary of a shell)."""
    from .problem import _gauss

    dom = space.domain
    D = dom.D
    if D not in (2, 3):
        raise ValueError("sphere_surface_quadrature supports dimensions 2 and 3")
    c = np.asarray(center, dtype=np.float64)
    R = float(radius)
    if c.shape != (D,) or not R > 0:
        raise ValueError("center must have the domain dimension and radius must be positive")
    q = int(points_per_axis) if points_per_axis else int(space.degrees.max()) + 2
    gx, gw = _gauss(q)
    leaves = space.leaves
    lower = dom.cell_lower(leaves)
    size = dom.cell_size(leaves)
    upper = lower + size
    nearest = np.clip(c[None, :], lower, upper)
    dmin = np.sqrt(np.sum((nearest - c[None, :]) ** 2, axis=1))
    far = np.maximum(np.abs(lower - c[None, :]), np.abs(upper - c[None, :]))
    dmax = np.sqrt(np.sum(far ** 2, axis=1))
    hits = np.nonzero((dmin <= R) & (dmax >= R))[0]
    piece = _sphere_piece_3d if D == 3 else _circle_piece_2d
    gx2, gw2 = _gauss(q + 4)
    out = []
    for i in hits:
        P, W = [], []
        stack = [(lo, hi, k, 0) for lo, hi, k in _box_sphere_pieces(lower[i], upper[i], c, R)]
        while stack:
            lo, hi, k, depth = stack.pop()
            p, w = piece(lo, hi, k, c, R, gx, gw)
            # accept when a rule with 4 more points per segment agrees (no tangency left inside)
            a2 = piece(lo, hi, k, c, R, gx2, gw2)[1].sum()
            if abs(w.sum() - a2) > tolerance * max(a2, np.prod(hi - lo) ** ((D - 1) / D)) and depth < max_depth:
                for sl, su, sk in _box_sphere_pieces_split(lo, hi, c, R):
                    stack.append((sl, su, sk, depth + 1))
                continue
            if p.shape[0]:
                P.append(p)
                W.append(w)
        if not P:
            continue
        X = np.concatenate(P)
        w_phys = np.concatenate(W)
        n_phys = (X - c[None, :]) / R
        if not outward:
            n_phys = -n_phys
        half = 0.5 * size[i]
        xi = np.clip((X - (lower[i] + half)) / half, -1.0, 1.0)
        # reference normal and weight that the compile maps back to (w_phys, n_phys)
        nr = n_phys * half[None, :]
        nr /= np.linalg.norm(nr, axis=1)[:, None]
        w_ref = w_phys * np.linalg.norm(nr * half[None, :], axis=1) / np.prod(half)
        out.append(SurfaceQuadrature(int(leaves[i]), xi, w_ref, nr))
    return out

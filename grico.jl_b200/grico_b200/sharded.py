"""Sharded plans: the cells of one compiled plan split over ranks, with the partition-surface
halo sum of every apply.

The reference runs in one shared-memory process (its backend seam, `src/common.jl:8-18`, has
the single `_SharedMemoryCPUBackend`); here a job spread over several GPUs splits the cells.
They are cut into contiguous ranges of the Morton order (the active-leaf order of
`topology.jl:250-268`), balanced by the work of a cell, prod(p+1) * prod(q).  A rank compiles
the plan of its cells over a local numbering of the dofs they touch.  A reduced dof touched by
several ranks is shared: the lowest of them owns it, the others hold it as a ghost.  The local
reduced vector lists owned dofs first and ghosts after them, so a sum over owned entries (a dot
product) is a sum over a prefix.

One sharded apply is the local reduced apply followed by the halo sum.  With one shard per
process, each rank sends its contributions to the dofs it shares with a neighbouring rank to
that rank and receives the neighbour's (point-to-point, `ShardGroup.exchange`), then adds the
contributions in rank order; otherwise each shard packs its contributions into a buffer indexed
by global halo slot, the buffers are summed over all shards (one all-reduce), and each shard
unpacks the sums.  Vectors stay consistent: every rank holds the same value of a shared dof.  CG (`solve.jl:376-431`) then needs two more
all-reduces per iteration: p.Ap, and (r.r, r.z) together.

`ShardGroup` is the collective: `torch.distributed` across processes (NCCL between GPUs) and,
for several shards held by one process, a sum over them first.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

import numpy as np

from . import _lib as L
from .problem import AssemblyPlan, reduced_rhs


def cell_ranks(plan, parts):
    """Part of every active leaf (Morton position): contiguous ranges balanced by the per-cell
    work prod(p+1) * prod(q); each leaf goes to the part holding the middle of its share."""
    if parts < 1:
        raise ValueError("parts must be positive")
    space = plan.space
    w = np.prod(space.degrees.astype(np.float64) + 1.0, axis=1) * np.prod(space.qshape.astype(np.float64), axis=1)
    if len(w) < parts:
        raise ValueError(f"{len(w)} cells cannot be split into {parts} parts")
    c = np.cumsum(w)
    mid = (c - 0.5 * w) / c[-1]
    rank = np.minimum((mid * parts).astype(np.int64), parts - 1)
    if np.unique(rank).size != parts:
        raise ValueError(f"a part of the {parts}-way split holds no cell")
    return rank.astype(np.int32)


def _entry_dofs(b, sel):
    """Full dofs touched by the cells `sel` of batch b: single-term entries and tail rows."""
    nb = b.nbox
    m = b.map_index.reshape(-1, nb)[sel].reshape(-1)
    out = [m[m >= 0]]
    if b.tail_offsets is not None:
        k = -m[m <= -2] - 2
        if k.size:
            lo, hi = b.tail_offsets[k], b.tail_offsets[k + 1]
            out.append(b.tail_index[np.concatenate([np.arange(a, z) for a, z in zip(lo, hi)])])
    return np.concatenate(out)


def _touched(plan, rank, r):
    t = np.zeros(plan.n_full, dtype=bool)
    for b in plan.batches:
        sel = np.nonzero(rank[b.cells] == r)[0]
        if sel.size:
            t[_entry_dofs(b, sel)] = True
    return t


def _local_batch(b, sel, glob):
    """Batch b restricted to its cells `sel`, map entries renumbered to local full dofs (glob:
    sorted global ids of the local dofs) and tail rows renumbered in order of use."""
    lb = copy.copy(b)
    nb = b.nbox
    lb.__dict__.pop("points", None)
    lb.cells = b.cells[sel]
    lb.leaves = b.leaves[sel]
    lb.h = np.ascontiguousarray(b.h[sel])
    lb.lower = b.lower[sel]
    lb.kappa_points = None if b.kappa_points is None else np.ascontiguousarray(b.kappa_points[sel])
    m = b.map_index.reshape(-1, nb)[sel].reshape(-1).copy()
    single = m >= 0
    m[single] = np.searchsorted(glob, m[single]).astype(np.int32)
    lb.map_coef = None if b.map_coef is None else np.ascontiguousarray(b.map_coef.reshape(-1, nb)[sel].reshape(-1))
    multi = np.nonzero(m <= -2)[0]
    if multi.size:
        k = -m[multi] - 2
        lo, hi = b.tail_offsets[k], b.tail_offsets[k + 1]
        cnt = hi - lo
        src = np.concatenate([np.arange(a, z) for a, z in zip(lo, hi)])
        lb.tail_offsets = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
        lb.tail_index = np.searchsorted(glob, b.tail_index[src]).astype(np.int32)
        lb.tail_coef = np.ascontiguousarray(b.tail_coef[src])
        m[multi] = -(np.arange(multi.size, dtype=np.int32) + 2)
    else:
        lb.tail_offsets = lb.tail_index = lb.tail_coef = None
    lb.map_index = np.ascontiguousarray(m.astype(np.int32))
    return lb


class ShardPlan:
    """Rank r's share of `plan` split `parts` ways.

    Attributes: `plan` (an AssemblyPlan over the local dofs: apply, rhs and diagonal work on it
    unchanged), `n_owned` (owned reduced dofs: local reduced ids 0..n_owned-1), `global_reduced`
    (global reduced id of every local reduced dof), `halo_local` / `halo_slot` (the local reduced
    ids of shared dofs and their global halo slots), `n_halo` (global halo slots) and
    `neighbours` (a list of (rank, positions in the halo list of the dofs shared with it))."""

    def __init__(self, plan, rank, parts, device=True, cell_rank=None):
        if plan.point_batches:
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM, "sharded plans support tensor cells only")
        if getattr(plan, "relations", None):
            raise L.GricoError(L.GRICO_ERR_UNSUPPORTED_FORM,
                               "sharded plans need Dirichlet data that fixes single dofs (no relation rows)")
        if not 0 <= rank < parts:
            raise ValueError("rank out of range")
        self.rank, self.parts = int(rank), int(parts)
        cr = cell_ranks(plan, parts) if cell_rank is None else cell_rank
        self.cell_rank = cr
        # ranks touching every full dof: how many, and the lowest
        count = np.zeros(plan.n_full, dtype=np.int32)
        first = np.full(plan.n_full, -1, dtype=np.int32)
        free = plan.reduced_index >= 0
        mine = _touched(plan, cr, rank)
        common = []   # (rank q, full ids of the free dofs both ranks touch, ascending)
        for r in range(parts):
            t = mine if r == rank else _touched(plan, cr, r)
            count += t
            first[(first < 0) & t] = r
            if r != rank:
                both = np.nonzero(mine & t & free)[0]
                if both.size:
                    common.append((r, both))
        shared = free & (count >= 2)
        halo_global = np.nonzero(shared)[0]                      # full ids, sorted: slot order
        self.n_halo = int(halo_global.size)
        # local numbering
        glob = np.nonzero(mine)[0]
        lfree = free[glob]
        owned = lfree & (first[glob] == rank)
        ghost = lfree & ~owned
        order = np.concatenate([np.nonzero(owned)[0], np.nonzero(ghost)[0]])   # local full ids
        self.n_owned = int(owned.sum())
        n_red = int(order.size)
        red_of_local = np.full(glob.size, -1, dtype=np.int64)
        red_of_local[order] = np.arange(n_red)
        self.global_full = glob
        self.global_reduced = plan.reduced_index[glob[order]]
        sh = shared[glob[order]]
        self.halo_local = np.ascontiguousarray(np.nonzero(sh)[0].astype(np.int32))
        self.halo_slot = np.ascontiguousarray(np.searchsorted(halo_global, glob[order][sh]).astype(np.int32))
        # neighbours: every rank sharing a dof with this one, with the positions of the shared
        # dofs in this rank's halo list, in ascending global order (the order both sides use)
        halo_full = glob[order][sh]
        by_full = np.argsort(halo_full, kind="stable")
        self.neighbours = [(q, np.ascontiguousarray(by_full[np.searchsorted(halo_full[by_full], ids)].astype(np.int64)))
                           for q, ids in common]
        # the local plan: same problem and form, local cells and dofs
        lp = object.__new__(AssemblyPlan)
        lp.problem, lp.form, lp.space, lp.D = plan.problem, plan.form, plan.space, plan.D
        lp.n_full = int(glob.size)
        lp.n_cut = 0
        lp.point_batches = []
        lp.batches = []
        for b in plan.batches:
            sel = np.nonzero(cr[b.cells] == rank)[0]
            if sel.size:
                lp.batches.append(_local_batch(b, sel, glob))
        fixed_local = np.nonzero(~lfree)[0]
        lp.fixed_dofs = fixed_local.astype(np.int64)
        lp.fixed_values = np.ascontiguousarray(plan.shift[glob[fixed_local]])
        lp.relations = []
        lp.solve_dofs = order.astype(np.int64)
        lp.n_reduced = n_red
        lp.reduced_index = red_of_local
        lp.red_offsets = np.concatenate([[0], np.cumsum(lfree.astype(np.int64))]).astype(np.int64)
        lp.red_index = np.ascontiguousarray(red_of_local[np.nonzero(lfree)[0]])
        lp.red_coef = np.ones(n_red)
        lp.shift = np.ascontiguousarray(plan.shift[glob])
        lp.handle = None
        if device:
            lp._create_device_plan()
        self.plan = lp

    @property
    def n_reduced(self):
        return self.plan.n_reduced

    def scatter(self, global_reduced_vector):
        """This rank's local reduced vector from a global one."""
        return np.ascontiguousarray(np.asarray(global_reduced_vector)[self.global_reduced])


class ShardGroup:
    """Sum over all shards of a job: first over the shards this process holds (a list; one in a
    job with one process per GPU), then across processes with torch.distributed (`group`, or
    the default group when it is initialised with more than one rank).

    `halo`: how a job with one shard per process sums the halo of an apply.  "neighbours"
    (default): each rank exchanges its contributions with the ranks it shares dofs with
    (point-to-point, one send and one receive per neighbour) and adds them in rank order;
    "allreduce": one all-reduce over every halo slot of the job."""

    def __init__(self, group=None, halo="neighbours"):
        import torch.distributed as dist

        if halo not in ("neighbours", "allreduce"):
            raise ValueError("halo must be 'neighbours' or 'allreduce'")
        self.group = group
        self.halo = halo
        self.dist = dist if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1 else None

    def peer(self, q):
        """Global rank of rank q of the group."""
        return q if self.group is None else self.dist.get_global_rank(self.group, q)

    def exchange(self, sends, recvs):
        """Point-to-point: sends[k] = (rank, tensor) goes to that rank, recvs[k] = (rank, tensor)
        is filled from it (the two lists may name different ranks); returns when all have
        completed.  Every pair of ranks must agree on what it exchanges."""
        d = self.dist
        ops = [d.P2POp(d.isend, sb, self.peer(q), self.group) for q, sb in sends]
        ops += [d.P2POp(d.irecv, rb, self.peer(q), self.group) for q, rb in recvs]
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()

    def allreduce(self, views):
        """Sum the same-shaped tensors `views` (one per local shard) over every shard of the job;
        every view receives the sum."""
        head = views[0]
        for v in views[1:]:
            head.add_(v)
        if self.dist is not None:
            self.dist.all_reduce(head, group=self.group)
        for v in views[1:]:
            v.copy_(head)


def _ptr(t, offset=0):
    return C.c_void_p(t.data_ptr() + 8 * offset)


class _DeviceOps:
    """The sharded path's device work: libgrico_b200 calls on torch CUDA tensors (FP64), all on
    torch's current stream, so the collectives order behind them."""

    def __init__(self):
        import torch

        from .problem import torch_stream_handle

        self.torch = torch
        self.stream = C.c_void_p(torch_stream_handle())

    def vector(self, n):
        return self.torch.zeros(max(int(n), 1), dtype=self.torch.float64, device="cuda")

    def upload(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")

    def index(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32)).to("cuda")

    def apply(self, shard, x, y):
        L.check(L.lib().grico_reduced_apply(shard.plan.handle, _ptr(x), _ptr(y), 1, L.GRICO_PREC_FP64, 0,
                                            self.stream), "sharded apply")

    def pack(self, shard, idx, y, buf):
        loc, slot = idx
        L.check(L.lib().grico_halo_pack(_ptr(y), _ptr(loc), _ptr(slot), int(shard.halo_local.size), _ptr(buf),
                                        int(shard.n_halo), self.stream), "halo pack")

    def unpack(self, shard, idx, buf, y):
        loc, slot = idx
        L.check(L.lib().grico_halo_unpack(_ptr(y), _ptr(loc), _ptr(slot), int(shard.halo_local.size), _ptr(buf),
                                          self.stream), "halo unpack")

    def dot(self, n, x, y, out, slot, partial):
        L.check(L.lib().grico_vec_dot(int(n), _ptr(x), _ptr(y), _ptr(out, slot), _ptr(partial), self.stream), "dot")

    def diagonal(self, shard, d):
        self.torch.cuda.current_stream().synchronize()
        L.check(L.lib().grico_reduced_diagonal(shard.plan.handle, C.cast(_ptr(d), L.f64p), 0), "diagonal")

    def invert(self, n, d, dinv):
        L.check(L.lib().grico_vec_invert(int(n), _ptr(d), _ptr(dinv), self.stream), "Jacobi")

    def update_xr(self, n, n_sum, x, r, p, q, s, partial):
        L.check(L.lib().grico_cg_update_xr(int(n), int(n_sum), _ptr(x), _ptr(r), _ptr(p), _ptr(q), _ptr(s),
                                           _ptr(partial), self.stream), "cg update")

    def precondition(self, n, n_sum, dinv, r, z, s, partial):
        L.check(L.lib().grico_cg_precondition(int(n), int(n_sum), None if dinv is None else _ptr(dinv), _ptr(r),
                                              _ptr(z), _ptr(s), _ptr(partial), self.stream), "cg precondition")

    def direction(self, n, p, z, s):
        L.check(L.lib().grico_cg_direction(int(n), _ptr(p), _ptr(z), _ptr(s), self.stream), "cg direction")

    def copy(self, src, dst):
        L.check(L.lib().grico_vec_axpby(int(src.numel()), 1.0, _ptr(src), 0.0, _ptr(dst), self.stream), "copy")

    def host(self, t):
        return t.cpu().numpy()


class ShardedOperator:
    """The sharded reduced operator of the shards this process holds (one per process in a
    multi-GPU job; several on one device to run a split on a single GPU)."""

    def __init__(self, shards, group=None, ops=None):
        self.shards = list(shards)
        self.group = group or ShardGroup()
        self.ops = ops or _DeviceOps()
        o = self.ops
        self._idx = [(o.index(s.halo_local), o.index(s.halo_slot)) for s in self.shards]
        self._nbr = None
        if self.group.dist is not None and self.group.halo == "neighbours" and len(self.shards) == 1:
            self._setup_neighbours(o.vector(1).device)
        else:
            self._buf = [o.vector(s.n_halo) for s in self.shards]

    def _setup_neighbours(self, device):
        import torch

        s = self.shards[0]
        h = int(s.halo_local.size)
        rows = sorted([s.rank] + [q for q, _ in s.neighbours])
        self._loc = torch.as_tensor(s.halo_local.astype(np.int64), device=device)
        self._rows = torch.zeros((len(rows), max(h, 1)), dtype=torch.float64, device=device)
        self._me = rows.index(s.rank)
        self._nbr = [(q, rows.index(q), torch.as_tensor(pos, device=device),
                      torch.zeros(pos.size, dtype=torch.float64, device=device),
                      torch.zeros(pos.size, dtype=torch.float64, device=device)) for q, pos in s.neighbours]
        # a first collective over the whole group, so that the point-to-point calls that follow
        # only ever involve neighbours
        self.group.dist.all_reduce(torch.zeros(1, dtype=torch.float64, device=device), group=self.group.group)

    def _halo_neighbours(self, y):
        """Neighbour halo sum: this rank's contributions to its shared dofs go to the ranks that
        share them, theirs come back into one row per rank, and the rows are added in rank order,
        so every rank forms the same sum, bit for bit, for a dof it shares."""
        h = int(self.shards[0].halo_local.size)
        if h == 0:
            return
        rows = self._rows[:, :h]
        rows.zero_()
        mine = rows[self._me]
        mine.copy_(y.index_select(0, self._loc))
        for _, _, pos, sb, _ in self._nbr:
            sb.copy_(mine.index_select(0, pos))
        self.group.exchange([(q, sb) for q, _, _, sb, _ in self._nbr], [(q, rb) for q, _, _, _, rb in self._nbr])
        for _, row, pos, _, rb in self._nbr:
            rows[row].index_copy_(0, pos, rb)
        acc = rows[0].clone()
        for i in range(1, rows.shape[0]):
            acc.add_(rows[i])
        y.index_copy_(0, self._loc, acc)

    def halo_sum(self, ys):
        """Sum the shards' contributions to every shared dof; each shard's entries become the sums."""
        o = self.ops
        if self._nbr is not None:
            self._halo_neighbours(ys[0])
            return
        if self.shards[0].n_halo == 0:
            return
        for s, idx, y, buf in zip(self.shards, self._idx, ys, self._buf):
            o.pack(s, idx, y, buf)
        self.group.allreduce([b[: self.shards[0].n_halo] for b in self._buf])
        for s, idx, y, buf in zip(self.shards, self._idx, ys, self._buf):
            o.unpack(s, idx, buf, y)

    def apply(self, xs, ys):
        """ys[k] = (A x)_local of shard k, consistent on shared dofs."""
        for s, x, y in zip(self.shards, xs, ys):
            self.ops.apply(s, x, y)
        self.halo_sum(ys)

    def rhs(self):
        """Local reduced right-hand sides, consistent on shared dofs."""
        bs = [self.ops.upload(reduced_rhs(s.plan)) if s.n_reduced else self.ops.vector(0) for s in self.shards]
        self.halo_sum(bs)
        return bs

    def inverse_diagonal(self):
        o = self.ops
        ds = [o.vector(s.n_reduced) for s in self.shards]
        for s, d in zip(self.shards, ds):
            o.diagonal(s, d)
        self.halo_sum(ds)
        out = [o.vector(s.n_reduced) for s in self.shards]
        for s, d, di in zip(self.shards, ds, out):
            o.invert(s.n_reduced, d, di)
        return out


class ShardedReport:
    def __init__(self, iterations, status, initial_residual, final_residual):
        self.iterations = iterations
        self.status = status
        self.initial_residual = initial_residual
        self.final_residual = final_residual


def sharded_cg(op, bs, relative_tolerance=None, absolute_tolerance=0.0, maxiter=1000, jacobi=True,
               preconditioner=None):
    """Preconditioned CG on the sharded reduced system (solve.jl:376-431: stop when
    ||r|| <= max(atol, rtol ||b||), Jacobi or identity preconditioner, or `preconditioner`, an
    object whose apply(r) returns the consistent local z, e.g. ShardedMultigrid; one shard per
    process then).  `bs`: consistent local right-hand sides (ShardedOperator.rhs).  Returns
    (local solutions, report)."""
    o = op.ops
    shards = op.shards
    if preconditioner is not None:
        if len(shards) != 1:
            raise ValueError("a V-cycle preconditioner needs one shard per process")
        jacobi = False
    rtol = math.sqrt(np.finfo(np.float64).eps) if relative_tolerance is None else float(relative_tolerance)
    n = [s.n_reduced for s in shards]
    no = [s.n_owned for s in shards]
    dinv = op.inverse_diagonal() if jacobi else [None] * len(shards)
    xs = [o.vector(k) for k in n]
    rs = [o.vector(k) for k in n]
    zs = [o.vector(k) for k in n]
    ps = [o.vector(k) for k in n]
    qs = [o.vector(k) for k in n]
    ss = [o.vector(8) for _ in shards]      # rz, pAp, rr, rz_new, bb
    part = [o.vector(592) for _ in shards]

    def precondition(k):
        if preconditioner is None:
            o.precondition(n[k], no[k], dinv[k], rs[k], zs[k], ss[k], part[k])
            return
        z = preconditioner.apply(rs[k])
        zs[k][: n[k]] = z[: n[k]]
        o.dot(no[k], rs[k], zs[k], ss[k], 3, part[k])

    for k in range(len(shards)):
        o.copy(bs[k], rs[k])
        o.dot(no[k], bs[k], bs[k], ss[k], 4, part[k])
        precondition(k)                                                      # s3 = r.z
        o.copy(zs[k], ps[k])
    op.group.allreduce([s[3:5] for s in ss])                                  # r.z, b.b
    for s in ss:
        s[0:1].copy_(s[3:4])
        s[2:3].copy_(s[4:5])                                                   # r = b: r.r = b.b
    h = o.host(ss[0])
    bnorm = math.sqrt(h[4])
    tol = max(float(absolute_tolerance), rtol * bnorm)
    rr = h[2]
    init = math.sqrt(rr)
    it = 0
    status = L.GRICO_OK
    converged = rr <= tol * tol
    while not converged and it < maxiter:
        it += 1
        op.apply(ps, qs)
        for k in range(len(shards)):
            o.dot(no[k], ps[k], qs[k], ss[k], 1, part[k])
        op.group.allreduce([s[1:2] for s in ss])                               # p.Ap
        for k in range(len(shards)):
            o.update_xr(n[k], no[k], xs[k], rs[k], ps[k], qs[k], ss[k], part[k])
            precondition(k)
        op.group.allreduce([s[2:4] for s in ss])                               # r.r, r.z
        h = o.host(ss[0])
        pap, rr = h[1], h[2]
        if not pap > 0.0:
            status = L.GRICO_ERR_BREAKDOWN if math.isfinite(pap) else L.GRICO_ERR_NONFINITE
            break
        if not math.isfinite(rr):
            status = L.GRICO_ERR_NONFINITE
            break
        if rr <= tol * tol:
            converged = True
            break
        for k in range(len(shards)):
            o.direction(n[k], ps[k], zs[k], ss[k])
    if status == L.GRICO_OK and not converged:
        status = L.GRICO_ERR_NOT_CONVERGED
    return xs, ShardedReport(it, status, init, math.sqrt(rr) if math.isfinite(rr) else rr)


def _csr_take(off, rows):
    """Entry positions of the CSR rows `rows`, row by row."""
    rows = np.asarray(rows, dtype=np.int64)
    cnt = off[rows + 1] - off[rows]
    if cnt.sum() == 0:
        return np.zeros(0, dtype=np.int64)
    return np.repeat(off[rows] - (np.cumsum(cnt) - cnt), cnt) + np.arange(int(cnt.sum()), dtype=np.int64)


def _reduced_sets(plan, cell_rank, parts):
    """Per rank, the sorted global reduced ids of the free dofs its cells touch (a rank's local
    reduced dofs), and per reduced dof the lowest rank holding it (its owner)."""
    sets = []
    for r in range(parts):
        g = plan.reduced_index[np.nonzero(_touched(plan, cell_rank, r))[0]]
        sets.append(np.unique(g[g >= 0]).astype(np.int64))
    owner = np.full(plan.n_reduced, parts, dtype=np.int64)
    for r in reversed(range(parts)):
        owner[sets[r]] = r
    return sets, owner


class _TransferLinks:
    """Point-to-point restriction and prolongation between a sharded coarse level and the fine
    level above it, for rank `me`; every list is computed from the global hierarchy on every
    rank, so both ends of a send agree on it.

    Restriction: this rank sums P^T over its owned fine rows into the coarse dofs they reach
    (`cols_own`, sorted global ids), keeps the entries it holds and sends the others' share to
    each rank holding them; every holder adds the contributions in rank order.  Prolongation:
    the coarse values this rank's fine rows need but it does not hold come from their owners."""

    def __init__(self, me, parts, off, col, coarse_sets, coarse_owner, fine_sets, fine_owner, coarse_local, device):
        import torch

        self.me = me
        nc = coarse_owner.size
        holds = []
        for r in range(parts):
            m = np.zeros(nc, dtype=bool)
            m[coarse_sets[r]] = True
            holds.append(m)
        lpos = np.full(nc, -1, dtype=np.int64)
        lpos[coarse_local] = np.arange(coarse_local.size)
        cols = [np.unique(col[_csr_take(off, np.nonzero(fine_owner == r)[0])]) for r in range(parts)]
        need = [np.unique(col[_csr_take(off, fine_sets[r])]) for r in range(parts)]
        own = cols[me]
        self.cols_own = own
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=device)
        f = lambda n: torch.zeros(int(n), dtype=torch.float64, device=device)
        # restriction
        mine = holds[me][own]
        self.r_keep = (t(np.nonzero(mine)[0]), t(lpos[own[mine]]))
        self.r_send = []
        for q in range(parts):
            if q != me:
                sel = np.nonzero(holds[q][own])[0]
                if sel.size:
                    self.r_send.append((q, t(sel), f(sel.size)))
        self.r_recv = []
        for q in range(parts):
            if q != me:
                ids = cols[q][holds[me][cols[q]]]
                if ids.size:
                    self.r_recv.append((q, t(lpos[ids]), f(ids.size)))
        rows = sorted({me} | {q for q, _, _ in self.r_recv})
        self.r_rows = f(len(rows) * max(coarse_local.size, 1)).reshape(len(rows), -1)
        self.r_me = rows.index(me)
        self.r_row = {q: rows.index(q) for q, _, _ in self.r_recv}
        # prolongation
        nd = need[me]
        here = holds[me][nd]
        self.need = nd
        self.p_here = (t(np.nonzero(here)[0]), t(lpos[nd[here]]))
        self.p_recv = []
        miss = nd[~here]
        for q in range(parts):
            ids = miss[coarse_owner[miss] == q]
            if q != me and ids.size:
                self.p_recv.append((q, t(np.searchsorted(nd, ids)), f(ids.size)))
        self.p_send = []
        for q in range(parts):
            if q != me:
                mq = need[q][~holds[q][need[q]]]
                ids = mq[coarse_owner[mq] == me]
                if ids.size:
                    self.p_send.append((q, t(lpos[ids]), f(ids.size)))

    def restrict(self, group, partial, n_local):
        """Local coarse right-hand side from this rank's partial sums over `cols_own`."""
        rows = self.r_rows[:, : max(n_local, 1)]
        rows.zero_()
        sel, pos = self.r_keep
        rows[self.r_me].index_copy_(0, pos, partial.index_select(0, sel))
        for _, sel, sb in self.r_send:
            sb.copy_(partial.index_select(0, sel))
        group.exchange([(q, sb) for q, _, sb in self.r_send], [(q, rb) for q, _, rb in self.r_recv])
        for q, pos, rb in self.r_recv:
            rows[self.r_row[q]].index_copy_(0, pos, rb)
        acc = rows[0].clone()
        for i in range(1, rows.shape[0]):
            acc.add_(rows[i])
        return acc

    def needed_values(self, group, xc, out):
        """out[k] = the coarse value of global id need[k], from xc (local coarse vector) and the
        owners of the ones this rank does not hold."""
        k, pos = self.p_here
        out.index_copy_(0, k, xc.index_select(0, pos))
        for _, pos, sb in self.p_send:
            sb.copy_(xc.index_select(0, pos))
        group.exchange([(q, sb) for q, _, sb in self.p_send], [(q, rb) for q, _, rb in self.p_recv])
        for _, k, rb in self.p_recv:
            out.index_copy_(0, k, rb)
        return out


def gather_reduced(shards, xs, n_reduced, ops=None):
    """Global reduced vector from the owned entries of the shards (host arrays; for one process
    holding every shard, or rank 0 after gathering)."""
    out = np.zeros(n_reduced)
    for s, x in zip(shards, xs):
        hx = ops.host(x) if ops is not None else np.asarray(x)
        out[s.global_reduced[: s.n_owned]] = hx[: s.n_owned]
    return out


class ShardedMultigrid:
    """hp-multigrid V-cycle over sharded levels: `_vcycle!` (multigrid.jl:858-889) with damped
    Jacobi smoothing (`_smooth_jacobi!`, multigrid.jl:943-956) and the dense coarse solve
    (multigrid.jl:891-924, common.jl:272-330).

    Every level of the hierarchy (`build_hierarchy`: the same h/p coarsening as the one-GPU
    V-cycle) is split over the ranks by its own Morton ranges (`ShardPlan`, one shard per
    process), so a level apply is the sharded apply with its halo sum.  Transfers between
    levels, in a job of several processes with neighbour halos: restriction sums P^T over each
    rank's owned fine rows and sends each rank holding a reached coarse dof its share, the
    holders adding the shares in rank order; prolongation fetches the coarse values a rank's fine
    rows need but it does not hold from their owners, then applies the rank's rows of P
    (`_TransferLinks`, all point to point).  Otherwise they use global vectors: restriction into
    a global coarse vector (one all-reduce of the coarse length), prolongation from the owned
    entries of all ranks (one all-reduce).  The coarsest level is solved redundantly on every rank from the same
    gathered right-hand side (Cholesky of the coarse matrix, assembled at set-up from sharded
    applies of unit vectors).  Vectors stay consistent on shared dofs throughout, so the
    V-cycle is that of the unsharded hierarchy up to the order of floating-point sums."""

    def __init__(self, plan, rank, parts, opts=None, group=None, ops=None, device=True):
        import torch

        from .multigrid import GeometricMultigridPreconditioner, build_hierarchy, resolved_smoother

        self.opts = opts or GeometricMultigridPreconditioner()
        if resolved_smoother(self.opts, plan.problem) != "jacobi":
            raise L.GricoError(L.GRICO_ERR_INVALID, "the sharded V-cycle smooths with damped Jacobi")
        self.torch = torch
        self.group = group or ShardGroup()
        self.ops = ops or _DeviceOps()
        plans, transfers = build_hierarchy(plan, self.opts, device=device)
        self.shards = [ShardPlan(p, rank, parts, device=device) for p in plans]
        self.levels = [ShardedOperator([s], group=self.group, ops=self.ops) for s in self.shards]
        self.n_global = [p.n_reduced for p in plans]
        self.dinv = [None] + [lv.inverse_diagonal()[0] for lv in self.levels[1:]]
        dev = self.dinv[-1].device if len(self.dinv) > 1 else torch.device("cpu")
        self.device = dev
        self._owned = [torch.as_tensor(s.global_reduced[: s.n_owned].astype(np.int64), device=dev) for s in self.shards]
        self._local = [torch.as_tensor(s.global_reduced.astype(np.int64), device=dev) for s in self.shards]
        # prolongation rows of this rank's fine dofs as (local row, global column, value) triples;
        # restriction sums P^T over the rows of its owned fine dofs (a prefix of the local rows)
        self._P = []
        for i, (off, col, val) in enumerate(transfers):
            rows = np.asarray(self.shards[i + 1].global_reduced, dtype=np.int64)
            cnt = off[rows + 1] - off[rows]
            take = np.concatenate([np.arange(off[g], off[g + 1]) for g in rows]) if rows.size else np.zeros(0, np.int64)
            loc = np.repeat(np.arange(rows.size, dtype=np.int64), cnt)
            self._P.append((torch.as_tensor(loc, device=dev), torch.as_tensor(col[take].astype(np.int64), device=dev),
                            torch.as_tensor(val[take].astype(np.float64), device=dev)))
        # with one shard per process and neighbour halos, the transfers exchange only the coarse
        # entries a rank's rows reach or need, point to point (`_TransferLinks`); otherwise they
        # go through global coarse vectors and all-reduces
        self._links = None
        if self.group.dist is not None and self.group.halo == "neighbours":
            parts = self.shards[0].parts
            sets = [_reduced_sets(p, s.cell_rank, parts) for p, s in zip(plans, self.shards)]
            self._links = []
            for i, (off, col, _) in enumerate(transfers):
                lk = _TransferLinks(rank, parts, off, col, sets[i][0], sets[i][1], sets[i + 1][0], sets[i + 1][1],
                                    np.asarray(self.shards[i].global_reduced, dtype=np.int64), dev)
                loc, colg, v = self._P[i]
                cg = colg.cpu().numpy()
                own = (loc < self.shards[i + 1].n_owned).cpu().numpy()
                lk.pos_need = torch.as_tensor(np.searchsorted(lk.need, cg), device=dev)
                lk.own = torch.as_tensor(np.nonzero(own)[0], device=dev)
                lk.pos_own = torch.as_tensor(np.searchsorted(lk.cols_own, cg[own]), device=dev)
                self._links.append(lk)
        # coarse matrix from sharded applies of unit vectors (the same sequence on every rank)
        n0 = self.n_global[0]
        A0 = np.zeros((n0, n0))
        e = np.zeros(n0)
        for j in range(n0):
            e[j] = 1.0
            x = self._upload(e[self.shards[0].global_reduced])
            y = self.ops.vector(self.shards[0].n_reduced)
            self.levels[0].apply([x], [y])
            A0[:, j] = self._gather(0, y).cpu().numpy()
            e[j] = 0.0
        self.coarse_factor = np.linalg.cholesky(0.5 * (A0 + A0.T)) if n0 else np.zeros((0, 0))

    def _upload(self, a):
        return self.torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.device)

    def _gather(self, level, x):
        """Global vector of `level` from the owned entries of every rank (one all-reduce)."""
        g = self.torch.zeros(max(self.n_global[level], 1), dtype=self.torch.float64, device=self.device)
        no = self.shards[level].n_owned
        g.index_copy_(0, self._owned[level], x[:no])
        self.group.allreduce([g])
        return g[: self.n_global[level]]

    def _apply(self, level, x):
        y = self.ops.vector(self.shards[level].n_reduced)
        self.levels[level].apply([x], [y])
        return y

    def _smooth(self, level, x, b, steps):
        n = self.shards[level].n_reduced
        w = self.opts.smoother_damping
        for _ in range(steps):
            y = self._apply(level, x)
            x[:n] += w * self.dinv[level][:n] * (b[:n] - y[:n])
        return x

    def vcycle(self, level, b):
        """Local correction of `level` for the consistent local right-hand side b."""
        n = self.shards[level].n_reduced
        if level == 0:
            bg = self._gather(0, b).cpu().numpy()
            xg = np.linalg.solve(self.coarse_factor.T, np.linalg.solve(self.coarse_factor, bg)) if bg.size else bg
            x = self.ops.vector(n)
            if n:
                x[:n] = self._upload(xg[self.shards[0].global_reduced])
            return x
        x = self._smooth(level, self.ops.vector(n), b, self.opts.pre_smoothing_steps)
        r = self.ops.vector(n)
        r[:n] = b[:n] - self._apply(level, x)[:n]
        nc = self.shards[level - 1].n_reduced
        fo = self.shards[level].n_owned
        loc, col, val = self._P[level - 1]
        bc = self.ops.vector(nc)
        if self._links is not None:
            lk = self._links[level - 1]
            torch = self.torch
            pc = torch.zeros(lk.cols_own.size, dtype=torch.float64, device=self.device)
            pc.index_add_(0, lk.pos_own, val[lk.own] * r[loc[lk.own]])
            bl = lk.restrict(self.group, pc, nc)
            if nc:
                bc[:nc] = bl[:nc]
            xc = self.vcycle(level - 1, bc)
            xn = lk.needed_values(self.group, xc, torch.zeros(lk.need.size, dtype=torch.float64, device=self.device))
            if n:
                x.index_add_(0, loc, val * xn[lk.pos_need])
            return self._smooth(level, x, b, self.opts.post_smoothing_steps)
        own = loc < fo
        rc = self.torch.zeros(max(self.n_global[level - 1], 1), dtype=self.torch.float64, device=self.device)
        rc.index_add_(0, col[own], val[own] * r[loc[own]])
        self.group.allreduce([rc])
        if nc:
            bc[:nc] = rc[self._local[level - 1]]
        xc = self.vcycle(level - 1, bc)
        xg = self._gather(level - 1, xc)
        if n:
            x.index_add_(0, loc, val * xg[col])
        return self._smooth(level, x, b, self.opts.post_smoothing_steps)

    def apply(self, r):
        """z = V-cycle(r) on the finest level (local, consistent)."""
        return self.vcycle(len(self.shards) - 1, r)

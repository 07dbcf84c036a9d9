"""Problems and a host restatement of the sharded path's device steps for the sharded tests.

`HostOps` stands in for the library's device calls on CPU: the local reduced apply runs the
oracle's C tensor schedule on the shard's own maps, the Jacobi diagonal probes that apply, and
the CG steps restate the kernels of csrc/grico_shard.cu in numpy.  What the tests exercise is
the product's host logic around them: the partition, the local numbering, the halo slots, the
collective and the sharded CG loop."""
import numpy as np
import torch

import grico_b200 as gb
import grico_oracle as go
import oracle_lib as ol


def poisson(D, roots, p, rounds=0, extent=None, refine=None, mass=0.0):
    """-div grad u (+ mass u) on a box with homogeneous Dirichlet on every face; `rounds` uniform
    refinements, then `refine(grid)` (local refinement: hanging nodes)."""
    d = gb.Domain((0.0,) * D, extent or (1.0,) * D, roots)
    if rounds:
        gb.uniform_refine(d, rounds)
    if refine is not None:
        refine(d.grid)
    s = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(s)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.MassDiffusion(mass, 1.0))
    for a in range(1, D + 1):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return prob


def tables(p, q):
    pts, W = go.gauss_legendre_rule(q)
    B = np.zeros((p + 1, q))
    G = np.zeros((p + 1, q))
    for j, x in enumerate(pts):
        v, d = go.integrated_legendre_values_and_derivatives(x, p)
        B[:, j] = v[: p + 1]
        G[:, j] = d[: p + 1]
    return B, G, np.array(W)


def full_apply(plan, xf):
    """Cell operator on the full layout through the oracle's tensor schedule (single-term maps,
    one degree per axis per batch)."""
    yf = np.zeros(plan.n_full)
    for b in plan.batches:
        p, q = b.degree[0], b.q[0]
        assert all(v == p for v in b.degree) and all(v == q for v in b.q) and b.tail_offsets is None
        B, G, W = tables(p, q)
        nc = len(b.cells)
        ol.tensor_apply(plan.D, p + 1, q, b.map_index, b.h, B, G, W, plan.form.mass, plan.form.kappa, None,
                        np.arange(nc, dtype=np.int64), np.array([0, nc], dtype=np.int64), xf, yf, threads=1)
    return yf


def reduced_apply(plan, x):
    xf = np.zeros(plan.n_full)
    xf[plan.solve_dofs] = x
    return full_apply(plan, xf)[plan.solve_dofs]


def reduced_diagonal(plan):
    n = plan.n_reduced
    d = np.zeros(n)
    e = np.zeros(n)
    for i in range(n):
        e[i] = 1.0
        d[i] = reduced_apply(plan, e)[i]
        e[i] = 0.0
    return d


class HostOps:
    """CPU stand-in for the sharded path's device calls (torch CPU tensors as vectors)."""

    def vector(self, n):
        return torch.zeros(max(int(n), 1), dtype=torch.float64)

    def upload(self, a):
        return torch.from_numpy(np.array(a, dtype=np.float64))

    def index(self, a):
        return np.asarray(a, dtype=np.int64)

    def apply(self, shard, x, y):
        n = shard.n_reduced
        y.numpy()[:n] = reduced_apply(shard.plan, x.numpy()[:n])

    def pack(self, shard, idx, y, buf):
        loc, slot = idx
        b = buf.numpy()
        b[: shard.n_halo] = 0.0
        b[slot] = y.numpy()[loc]

    def unpack(self, shard, idx, buf, y):
        loc, slot = idx
        y.numpy()[loc] = buf.numpy()[slot]

    def dot(self, n, x, y, out, slot, partial):
        out.numpy()[slot] = float(np.dot(x.numpy()[:n], y.numpy()[:n]))

    def diagonal(self, shard, d):
        d.numpy()[: shard.n_reduced] = reduced_diagonal(shard.plan)

    def invert(self, n, d, dinv):
        dinv.numpy()[:n] = 1.0 / d.numpy()[:n]

    def update_xr(self, n, n_sum, x, r, p, q, s, partial):
        sv, xv, rv, pv, qv = s.numpy(), x.numpy(), r.numpy(), p.numpy(), q.numpy()
        if sv[1] > 0.0:
            a = sv[0] / sv[1]
            xv[:n] += a * pv[:n]
            rv[:n] -= a * qv[:n]
        sv[2] = float(np.dot(rv[:n_sum], rv[:n_sum]))

    def precondition(self, n, n_sum, dinv, r, z, s, partial):
        rv, zv = r.numpy(), z.numpy()
        zv[:n] = rv[:n] if dinv is None else dinv.numpy()[:n] * rv[:n]
        s.numpy()[3] = float(np.dot(rv[:n_sum], zv[:n_sum]))

    def direction(self, n, p, z, s):
        sv = s.numpy()
        p.numpy()[:n] = z.numpy()[:n] + (sv[3] / sv[0]) * p.numpy()[:n]
        sv[0] = sv[3]

    def copy(self, src, dst):
        dst.numpy()[: src.numel()] = src.numpy()

    def host(self, t):
        return t.numpy().copy()


def global_cg(plan, b, rtol, jacobi=True):
    """The oracle's PCG (solve.jl:376-431) on the unsharded plan."""
    dinv = 1.0 / reduced_diagonal(plan) if jacobi else None
    return go.cg_solve(lambda v: reduced_apply(plan, v), b, precond=(lambda r: dinv * r) if jacobi else None,
                       rtol=rtol)

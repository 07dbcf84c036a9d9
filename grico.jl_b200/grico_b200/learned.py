"""Learned smoother: a small 3-D convolutional network that maps D^-1-scaled residuals on the
degree-1 level of a uniform hex mesh (plus the log coefficient) to corrections, trained on the
GPU by this library's own convolution, ReLU, loss and Adam kernels, and used as one smoothing
sweep of the hp-GMG V-cycle (grico_mg_set_learned).  No reference counterpart.

Training objective (unsupervised in the error): for residuals r drawn from plain GMG
iterations, the correction c = sigma * N(D^-1 r / sigma, log a) should solve A c = r, so the
loss is ||r - A c||^2_{D^-1} / ||r||^2_{D^-1}, whose gradient with respect to c is
-2 A D^-1 (r - A c) / ||r||^2_{D^-1} (A symmetric); it is scattered back to the network output
grid and back-propagated through the convolutions.  torch is used only for device memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .grf import GaussianRandomField


def _p(t):
    return C.c_void_p(t.data_ptr())


def _check(rc, what):
    L.check(rc, what)


class SmootherNet:
    """4 convolutions 3x3x3 (2 -> 32 -> 32 -> 32 -> 1), ReLU between them, FP32 weights."""

    def __init__(self, channels=(2, 32, 32, 32, 1), seed=0):
        import torch

        self.channels = tuple(int(c) for c in channels)
        rng = np.random.default_rng(seed)
        self.w, self.b = [], []
        for k in range(len(self.channels) - 1):
            ci, co = self.channels[k], self.channels[k + 1]
            std = np.sqrt(2.0 / (ci * 27)) * (0.1 if k == len(self.channels) - 2 else 1.0)
            self.w.append(torch.tensor(rng.standard_normal((co, ci, 27)) * std, dtype=torch.float32, device="cuda"))
            self.b.append(torch.zeros(co, dtype=torch.float32, device="cuda"))

    @property
    def n_layers(self):
        return len(self.w)

    def host_arrays(self):
        return ([w.detach().cpu().numpy().astype(np.float32) for w in self.w],
                [b.detach().cpu().numpy().astype(np.float32) for b in self.b])

    def save(self, path):
        ws, bs = self.host_arrays()
        np.savez(path, channels=np.array(self.channels), **{f"w{k}": w for k, w in enumerate(ws)},
                 **{f"b{k}": b for k, b in enumerate(bs)})

    @classmethod
    def load(cls, path):
        import torch

        d = np.load(path)
        net = cls(tuple(int(c) for c in d["channels"]))
        for k in range(net.n_layers):
            net.w[k] = torch.tensor(d[f"w{k}"], dtype=torch.float32, device="cuda")
            net.b[k] = torch.tensor(d[f"b{k}"], dtype=torch.float32, device="cuda")
        return net

    # ---- forward / backward on [B][C][Z][Y][X] FP32 tensors -------------------------------
    def forward(self, x, stream=None):
        """Activations [x, a1, ..., out]."""
        import torch

        acts = [x]
        B, _, Z, Y, X = x.shape
        lib = L.lib()
        for k in range(self.n_layers):
            co = self.channels[k + 1]
            y = torch.empty((B, co, Z, Y, X), dtype=torch.float32, device="cuda")
            _check(lib.grico_conv3d_forward(_p(acts[-1]), 0, _p(self.w[k]), _p(self.b[k]), _p(y), 0, B,
                                            self.channels[k], co, Z, Y, X, int(k + 1 < self.n_layers), stream),
                   "conv forward")
            acts.append(y)
        return acts

    def backward(self, acts, gout, stream=None):
        """Weight and bias gradients for the output gradient gout (same shape as the output)."""
        import torch

        B, _, Z, Y, X = acts[0].shape
        lib = L.lib()
        gw = [torch.empty_like(w) for w in self.w]
        gb = [torch.empty_like(b) for b in self.b]
        g = gout.contiguous()
        for k in reversed(range(self.n_layers)):
            ci, co = self.channels[k], self.channels[k + 1]
            if k + 1 < self.n_layers:
                _check(lib.grico_relu_backward(_p(acts[k + 1]), _p(g), g.numel(), stream), "relu backward")
            _check(lib.grico_conv3d_backward_weight(_p(acts[k]), _p(g), _p(gw[k]), _p(gb[k]), B, ci, co, Z, Y, X,
                                                    stream), "conv backward weight")
            if k > 0:
                gx = torch.empty_like(acts[k])
                wt = torch.empty_like(self.w[k])
                _check(lib.grico_conv3d_backward_data(_p(g), _p(self.w[k]), _p(wt), _p(gx), B, ci, co, Z, Y, X,
                                                      stream), "conv backward data")
                g = gx
        return gw, gb


# ---- the degree-1 level as a vertex grid -----------------------------------------------------

def vertex_grid(plan):
    """(grid_index [nz*ny*nx], (nx, ny, nz)) of a degree-1 plan on a uniform 3-D mesh: every
    reduced dof is the value at one vertex; -1 marks constrained or absent vertices."""
    space = plan.space
    if space.D != 3 or np.any(space.degrees != 1):
        raise ValueError("the learned smoother runs on the degree-1 level of a uniform 3-D mesh")
    grid = space.domain.grid
    lev = grid.levels[space.leaves]
    if np.any(lev != lev[0]):
        raise ValueError("the learned smoother needs a uniform mesh")
    counts = np.array(grid.root_counts) << lev[0]
    nx, ny, nz = (int(c) + 1 for c in counts)
    crd = grid.coords[space.leaves]
    idx = np.full(nx * ny * nz, -1, dtype=np.int64)
    for box in range(8):
        m = np.array([(box >> a) & 1 for a in range(3)])
        e = space.box_offsets[:-1] + box
        lo, hi = space.term_offsets[e], space.term_offsets[e + 1]
        ok = (hi - lo) == 1
        dof = space.term_index[lo[ok]]
        red = plan.reduced_index[dof]
        v = crd[ok] + m[None, :]
        g = (v[:, 2] * ny + v[:, 1]) * nx + v[:, 0]
        idx[g[red >= 0]] = red[red >= 0]
    return idx, (nx, ny, nz)


def vertex_points(dims, origin, extent):
    nx, ny, nz = dims
    ax = [origin[a] + extent[a] * np.arange(n) / (n - 1) for a, n in enumerate((nx, ny, nz))]
    Z, Yg, Xg = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return np.stack([Xg.reshape(-1), Yg.reshape(-1), Z.reshape(-1)], axis=1)


# ---- training ---------------------------------------------------------------------------------

class TrainingSample:
    """One degree-1 problem: its device plan, D^-1, grid map and log coefficient on the grid."""

    def __init__(self, plan, log_coef_grid):
        import torch

        self.plan = plan
        self.idx_host, self.dims = vertex_grid(plan)
        self.idx = torch.tensor(self.idx_host, device="cuda")
        d = plan_reduced_diagonal(plan)
        self.dinv = torch.tensor(1.0 / d, dtype=torch.float32, device="cuda")
        self.logc = torch.tensor(np.asarray(log_coef_grid, dtype=np.float32), device="cuda")
        self.residuals = []    # FP32 device vectors from plain GMG iterations


def plan_reduced_diagonal(plan):
    from .problem import reduced_diagonal

    return reduced_diagonal(plan)


def gmg_residuals(plan, mg, rhs_list, iterations=(1, 2, 3, 4)):
    """Residuals b - A x_k after k plain CG+GMG iterations from x_0 = 0 for every right-hand side."""
    from .problem import reduced_apply

    out = []
    for b in rhs_list:
        for k in iterations:
            x = np.zeros(plan.n_reduced)
            so = L.GricoSolveOptions(0.0, 0.0, int(k), L.GRICO_PRECOND_MULTIGRID, 30, 0)
            rep = L.GricoSolveReport()
            L.lib().grico_cg_solve(plan.handle, mg.handle, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
                                   C.byref(so), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS)
            r = b - reduced_apply(plan, x)
            if np.linalg.norm(r) > 0:
                out.append(r)
    return out


class Trainer:
    """Adam on the smoother network over TrainingSamples (all kernels from libgrico_b200)."""

    def __init__(self, net, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        import torch

        self.net, self.lr, self.beta1, self.beta2, self.eps = net, lr, beta1, beta2, eps
        self.m = [torch.zeros_like(t) for t in net.w + net.b]
        self.v = [torch.zeros_like(t) for t in net.w + net.b]
        self.step_count = 0
        self.partial = torch.zeros(600, dtype=torch.float64, device="cuda")
        self.sums = torch.zeros(64, dtype=torch.float64, device="cuda")

    def loss_and_grad(self, sample, residuals):
        """Mean over the residuals of ||r - A c||^2_{D^-1} / ||r||^2_{D^-1} and the output-grid
        gradient; residuals: list of FP32 device vectors."""
        import torch

        lib = L.lib()
        nx, ny, nz = sample.dims
        ng = nx * ny * nz
        n = sample.plan.n_reduced
        B = len(residuals)
        x = torch.empty((B, 2, nz, ny, nx), dtype=torch.float32, device="cuda")
        sig, den = [], []
        z = torch.empty(n, dtype=torch.float32, device="cuda")
        for k, r in enumerate(residuals):
            torch.mul(sample.dinv, r, out=z)
            dd = float(torch.dot(z.double(), r.double()))
            s = float(np.sqrt(dd / max(n, 1)))
            sig.append(s)
            den.append(dd)
            _check(lib.grico_grid_gather(_p(sample.idx), ng, _p(z), 1.0 / s, _p(x[k, 0]), None), "gather")
            x[k, 1].copy_(sample.logc.view(nz, ny, nx))
        acts = self.net.forward(x)
        out = acts[-1]
        c = torch.zeros((B, n), dtype=torch.float32, device="cuda")
        for k in range(B):
            _check(lib.grico_grid_scatter_add(_p(sample.idx), ng, _p(out[k, 0]), sig[k], _p(c[k]), None), "scatter")
        ac = torch.empty_like(c)
        _check(lib.grico_reduced_apply(sample.plan.handle, _p(c), _p(ac), B, L.GRICO_PREC_FP32, 0,
                                       C.c_void_p(1)), "apply")
        w = torch.empty_like(c)
        for k in range(B):
            _check(lib.grico_weighted_residual(_p(residuals[k]), _p(ac[k]), _p(sample.dinv), _p(w[k]), n,
                                               _p(self.partial), C.c_void_p(self.sums.data_ptr() + 8 * k), None),
                   "weighted residual")
        aw = torch.empty_like(w)
        _check(lib.grico_reduced_apply(sample.plan.handle, _p(w), _p(aw), B, L.GRICO_PREC_FP32, 0,
                                       C.c_void_p(1)), "apply")
        gout = torch.zeros_like(out)
        for k in range(B):
            _check(lib.grico_grid_gather(_p(sample.idx), ng, _p(aw[k]), -2.0 * sig[k] / (den[k] * B),
                                         _p(gout[k, 0]), None), "gather")
        loss = float(sum(self.sums[k].item() / den[k] for k in range(B)) / B)
        return loss, acts, gout

    def step(self, sample, residuals):
        loss, acts, gout = self.loss_and_grad(sample, residuals)
        gw, gb = self.net.backward(acts, gout)
        self.step_count += 1
        lib = L.lib()
        for t, g, m, v in zip(self.net.w + self.net.b, gw + gb, self.m, self.v):
            _check(lib.grico_adam_step(_p(t), _p(g), _p(m), _p(v), t.numel(), self.lr, self.beta1, self.beta2,
                                       self.step_count, self.eps, None), "adam")
        return loss


def attach(mg, level_plan, level, net, log_coef_grid, omega=1.0):
    """Install the trained network as the learned sweep of multigrid `mg` on `level`."""
    idx, (nx, ny, nz) = vertex_grid(level_plan)
    ws, bs = net.host_arrays()
    chans = np.array(net.channels, dtype=np.int32)
    wp = (C.POINTER(C.c_float) * len(ws))(*[w.ctypes.data_as(C.POINTER(C.c_float)) for w in ws])
    bp = (C.POINTER(C.c_float) * len(bs))(*[b.ctypes.data_as(C.POINTER(C.c_float)) for b in bs])
    logc = np.ascontiguousarray(log_coef_grid, dtype=np.float32)
    d = L.GricoLearnedDesc(int(level), nx, ny, nz, L.ptr(idx, C.c_int64), logc.ctypes.data_as(C.POINTER(C.c_float)),
                           net.n_layers, L.ptr(chans, C.c_int32), wp, bp, float(omega))
    _check(L.lib().grico_mg_set_learned(mg.handle, C.byref(d)), "set learned")
    mg._learned_keepalive = (idx, ws, bs, chans, logc)


# ---- the variable-coefficient workload --------------------------------------------------------

def grf_diffusion_problem(refine, degree=2, seed=0, corr_length=0.05, variance=2.0, points_per_length=4.0):
    """-div(a grad u) = 1 on [0,1]^3, a = exp(g) with g a Gaussian random field, homogeneous
    Dirichlet, 2^refine cells per axis.  Returns (problem, field)."""
    from . import mesh, problem as P, space as S

    g = GaussianRandomField(seed, corr_length=corr_length, variance=variance, points_per_length=points_per_length)
    dom = mesh.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    mesh.uniform_refine(dom, refine)
    sp = S.HpSpace(dom, S.SpaceOptions(basis=S.FullTensorBasis(), degree=S.UniformDegree(degree)))
    u = P.ScalarField(sp)
    prob = P.AffineProblem(u)
    P.add_cell_accumulator(prob, u, u, P.VariableDiffusion(g.coefficient()))
    P.add_cell_accumulator(prob, u, P.Load(lambda X: np.ones(X.shape[0])))
    for a in (1, 2, 3):
        for side in (mesh.LOWER, mesh.UPPER):
            P.add_constraint(prob, P.Dirichlet(u, P.BoundaryFace(a, side), 0.0))
    return prob, g


def level_log_coefficient(level_plan, field):
    """log a at the vertices of a degree-1 level (the network's second input channel)."""
    _, dims = vertex_grid(level_plan)
    return field(vertex_points(dims, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))).astype(np.float32)


def learned_stats(mg):
    """(sweeps run, sweeps kept) of the learned sweep of `mg`."""
    a, b = C.c_int64(), C.c_int64()
    _check(L.lib().grico_mg_learned_stats(mg.handle, C.byref(a), C.byref(b)), "learned stats")
    return a.value, b.value

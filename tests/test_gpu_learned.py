"""Learned smoother on the GPU: the convolution kernels against the numpy oracle, training
through the library's own kernels, and the learned sweep inside FGMRES + V-cycle.

Tolerances: FP32 convolutions within 1e-4 relative of the float64 oracle (FP32 accumulation
over at most 27 * 32 terms); BF16 outputs within 1e-2."""
import numpy as np
import pytest

import cnn_oracle as co
import grico_b200 as gb
from grico_b200 import _lib as L
from grico_b200 import learned as lr
from grico_b200.multigrid import GeometricMultigridPreconditioner, build_hierarchy, Multigrid

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def test_conv_kernels_match_oracle(cuda):
    import torch

    rng = np.random.default_rng(2)
    B, Ci, Co, Z, Y, X = 2, 3, 11, 9, 7, 10
    x = rng.standard_normal((B, Ci, Z, Y, X)).astype(np.float32)
    w = (rng.standard_normal((Co, Ci, 27)) * 0.2).astype(np.float32)
    b = rng.standard_normal(Co).astype(np.float32)
    gy = rng.standard_normal((B, Co, Z, Y, X)).astype(np.float32)
    tx, tw, tb, tgy = (torch.tensor(a, device="cuda") for a in (x, w, b, gy))
    ty = torch.empty((B, Co, Z, Y, X), dtype=torch.float32, device="cuda")
    lib = L.lib()
    p = lambda t: t.data_ptr()
    assert lib.grico_conv3d_forward(p(tx), 0, p(tw), p(tb), p(ty), 0, B, Ci, Co, Z, Y, X, 1, None) == 0
    ref = co.conv3d(x, w, b, relu=True)
    assert _rel(ty.cpu().numpy(), ref) <= 1e-4
    tyb = torch.empty((B, Co, Z, Y, X), dtype=torch.bfloat16, device="cuda")
    assert lib.grico_conv3d_forward(p(tx), 0, p(tw), p(tb), p(tyb), 1, B, Ci, Co, Z, Y, X, 1, None) == 0
    assert _rel(tyb.float().cpu().numpy(), ref) <= 1e-2
    gx, gw, gbias = co.conv3d_backward(x, w, gy)
    tgx = torch.empty_like(tx)
    twt = torch.empty_like(tw)
    tgw = torch.empty_like(tw)
    tgb = torch.empty_like(tb)
    assert lib.grico_conv3d_backward_data(p(tgy), p(tw), p(twt), p(tgx), B, Ci, Co, Z, Y, X, None) == 0
    assert lib.grico_conv3d_backward_weight(p(tx), p(tgy), p(tgw), p(tgb), B, Ci, Co, Z, Y, X, None) == 0
    assert _rel(tgx.cpu().numpy(), gx) <= 1e-4
    assert _rel(tgw.cpu().numpy(), gw) <= 1e-4
    assert _rel(tgb.cpu().numpy(), gbias) <= 1e-4


def test_network_gradients_match_oracle(cuda):
    """Full back-propagation (ReLU masks, masked MSE, every layer) against the oracle."""
    import torch

    rng = np.random.default_rng(3)
    net = lr.SmootherNet((2, 8, 8, 1), seed=4)
    ws, bs = net.host_arrays()
    onet = co.Net([(w.astype(np.float64), b.astype(np.float64)) for w, b in zip(ws, bs)])
    x = rng.standard_normal((2, 2, 6, 5, 7)).astype(np.float32)
    t = rng.standard_normal((2, 1, 6, 5, 7)).astype(np.float32)
    loss_ref, grads_ref = onet.gradients(x.astype(np.float64), t.astype(np.float64))
    acts = net.forward(torch.tensor(x, device="cuda"))
    tt = torch.tensor(t, device="cuda")
    g = torch.empty_like(acts[-1])
    partial = torch.zeros(600, dtype=torch.float64, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.lib().grico_mse_grad(acts[-1].data_ptr(), tt.data_ptr(), None, g.data_ptr(), g.numel(), float(g.numel()),
                                  partial.data_ptr(), loss.data_ptr(), None) == 0
    assert abs(loss.item() - loss_ref) <= 1e-5 * abs(loss_ref)
    gw, gbias = net.backward(acts, g)
    for k in range(len(gw)):
        assert _rel(gw[k].cpu().numpy(), grads_ref[k][0]) <= 1e-4
        assert _rel(gbias[k].cpu().numpy(), grads_ref[k][1]) <= 1e-4


def _level1_sample(refine, seed):
    """A degree-1 GRF problem with its own multigrid, as a training sample with GMG residuals."""
    import torch

    prob, field = lr.grf_diffusion_problem(refine, degree=1, seed=seed)
    plan = gb.compile(prob)
    mg = Multigrid(*build_hierarchy(plan, GeometricMultigridPreconditioner(smoother="chebyshev")),
                   GeometricMultigridPreconditioner(smoother="chebyshev"))
    sample = lr.TrainingSample(plan, lr.level_log_coefficient(plan, field))
    rng = np.random.default_rng(seed)
    rhs = [gb.reduced_rhs(plan)] + [rng.standard_normal(plan.n_reduced) for _ in range(2)]
    sample.residuals = [torch.tensor(r, dtype=torch.float32, device="cuda")
                        for r in lr.gmg_residuals(plan, mg, rhs, iterations=(1, 2, 3))]
    return sample


def _train(samples, steps, batch=4, seed=0):
    net = lr.SmootherNet(seed=seed)
    tr = lr.Trainer(net, lr=2e-3)
    rng = np.random.default_rng(seed)
    losses = []
    for s in range(steps):
        smp = samples[s % len(samples)]
        pick = rng.choice(len(smp.residuals), size=min(batch, len(smp.residuals)), replace=False)
        losses.append(tr.step(smp, [smp.residuals[i] for i in pick]))
    return net, losses


def test_training_reduces_the_residual_loss(cuda):
    samples = [_level1_sample(3, seed) for seed in (11, 12)]
    net, losses = _train(samples, 60)
    first, last = np.mean(losses[:6]), np.mean(losses[-6:])
    print("training loss", first, "->", last)
    assert np.isfinite(last) and last < 0.9 * first


def test_learned_sweep_inside_fgmres_vcycle(cuda):
    """FGMRES(30) + V-cycle on -div(exp(g) grad u) = 1 with and without the learned sweep on the
    degree-1 level; the sweep is judged by the true residual, so it can only be kept when it
    helps, and the solve reaches the same tolerance."""
    samples = [_level1_sample(4, seed) for seed in (21, 22)]
    net, _ = _train(samples, 80)
    prob, field = lr.grf_diffusion_problem(4, degree=2, seed=5)
    plan = gb.compile(prob)
    opts = GeometricMultigridPreconditioner(smoother="chebyshev", pre_smoothing_steps=2, post_smoothing_steps=2)
    plans, transfers = build_hierarchy(plan, opts)
    b = gb.reduced_rhs(plan)
    iters = {}
    for name in ("plain", "learned"):
        mg = Multigrid(plans, transfers, opts)
        if name == "learned":
            level = len(plans) - 2
            lr.attach(mg, plans[level], level, net, lr.level_log_coefficient(plans[level], field))
        import ctypes as C
        x = np.zeros(plan.n_reduced)
        so = L.GricoSolveOptions(1e-8, 0.0, 500, L.GRICO_PRECOND_MULTIGRID, 30, 0)
        rep = L.GricoSolveReport()
        rc = L.lib().grico_fgmres_solve(plan.handle, mg.handle, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
                                        C.byref(so), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS)
        assert rc == 0
        iters[name] = rep.iterations
        if name == "learned":
            sweeps, kept = lr.learned_stats(mg)
            print("learned sweeps", sweeps, "kept", kept)
            assert sweeps > 0
    print("FGMRES iterations", iters)
    assert iters["learned"] <= 1.5 * iters["plain"] + 1

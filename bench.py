#!/usr/bin/env python
"""Benchmark: FP64 matrix-free apply DOFs/s on the 3-D Poisson workload (64^3 cells, p = 4,
Gauss 5^3, homogeneous Dirichlet: 16,974,593 dofs), one step = one full-layout apply!.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs (torchrun) are independent replicas per rank (weak scaling, no data-path
collective); the job value is the sum over ranks with the max time over ranks.
The reference arm times the CPU restatement of Grico's tensor-product apply (the oracle's C
kernel, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grico.jl_b200"))

WORKLOAD = {"workload": "poisson3d_64cube_p4_dirichlet", "cells": "64x64x64", "degree": 4,
            "quadrature": "gauss 5x5x5", "dofs": 16974593, "form": "TestChannels(0, grad u)",
            "layout": "full (apply!)"}
METRIC = "DOFs/s matrix-free apply; time-to-1e-8 L² error (learned+mixed vs plain GPU)"
UNIT = "DOFs/s"
# flops per cell of the collocation schedule (2 q n (n^2 + q n + q^2) + 2 D q^(D+1)) * 2 + pointwise
N1 = Q1 = 5
FLOPS_PER_CELL = 2 * (2 * Q1 * N1 * (N1 * N1 + Q1 * N1 + Q1 * Q1) + 2 * 3 * Q1 ** 4) + 9 * Q1 ** 3


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# DRAM bytes of one subcell_apply launch per subcell (ncu, 32^3 shell: 19,729,664 B read, 0 B
# written, 469,928 subcells)
FCM_SUBCELL_TRAFFIC_PER_SUBCELL = 19729664.0 / 469928.0


def load_bf16_peak():
    """Measured dense BF16 TFLOP/s (burst, cuBLAS) of this pool's B200s, else the fallback 1590."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f).get("bf16_tflops", 1590.0))
    return 1590.0


def sample_vector(n):
    """_diagnostic_sample_vector (diagnostics.jl:107-121): sin(0.013 i) + 0.25 cos(0.037 i)."""
    i = np.arange(1, n + 1, dtype=np.float64)
    return np.sin(0.013 * i) + 0.25 * np.cos(0.037 * i)


class ClockSampler:
    """nvidia-smi clocks during the timed region (SM MHz, max, throttle reasons)."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_problem(gb):
    domain = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (4, 4, 4))
    gb.uniform_refine(domain, 4)
    space = gb.HpSpace(domain, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(4)))
    u = gb.ScalarField(space)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    for a in (1, 2, 3):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    return prob


FCM_WORKLOAD = {"workload": "fcm_shell_64cube_p3_nitsche", "cells": "64x64x64 background on [0,2]^3",
                "region": "0.4 < |x - (1,1,1)| < 0.9", "degree": 3, "basis": "full tensor",
                "quadrature": "gauss 4x4x4; cut cells: unfitted octree candidates, depth 3 (as subcells)",
                "surfaces": "sphere quadratures r = 0.9 (outward), r = 0.4 (inward)",
                "form": "TestChannels(0, grad u) + symmetric Nitsche, penalty 10 p^2 / h",
                "layout": "full (apply!)"}


def build_fcm_problem(gb, refine=6, p=3):
    """Finite-cell shell with Nitsche spheres, u = sin 2x cos 3y e^{z/2} (f = 12.75 u)."""
    c = np.array([1.0, 1.0, 1.0])

    def shell(X):
        r = np.linalg.norm(X - c[None, :], axis=1)
        return np.maximum(r - 0.9, 0.4 - r)

    exact = lambda X: np.sin(2 * X[:, 0]) * np.cos(3 * X[:, 1]) * np.exp(0.5 * X[:, 2])
    dom = gb.Domain((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (1, 1, 1))
    gb.uniform_refine(dom, refine)
    pdm = gb.PhysicalDomain(dom, gb.ImplicitRegion(shell, subdivision_depth=3))
    space = gb.HpSpace(pdm, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(p)))
    u = gb.ScalarField(space)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(lambda X: 12.75 * exact(X)))
    nit = gb.Nitsche(10.0 * p * p, data=exact)
    gb.add_surface_accumulator(prob, u, u, nit)
    gb.add_surface_accumulator(prob, u, nit)
    gb.add_surface_quadrature(prob, gb.sphere_surface_quadrature(space, c, 0.9, outward=True) +
                              gb.sphere_surface_quadrature(space, c, 0.4, outward=False))
    return prob


def cpu_reference_run(steps, warmup, budget_s=20.0):
    """Time the oracle's C restatement of the reference tensor apply on the full workload with
    every host thread.  Returns (DOFs/s, seconds per apply, threads, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import grico_oracle as go
    import oracle_lib as ol
    import uniform_maps as um

    counts, p = (64, 64, 64), 4
    coords, m, ndofs = um.uniform_space(counts, p)
    order, off = um.parity_colours(coords)
    pts, W = go.gauss_legendre_rule(p + 1)
    B = np.zeros((p + 1, p + 1))
    G = np.zeros((p + 1, p + 1))
    for j, x in enumerate(pts):
        v, d = go.integrated_legendre_values_and_derivatives(x, p)
        B[:, j] = v
        G[:, j] = d
    h = np.full((len(coords), 3), 1.0 / 64)
    x = sample_vector(ndofs)
    y = np.zeros(ndofs)
    threads = ol.max_threads()
    args = (3, p + 1, p + 1, m.astype(np.int32), h, B, G, np.array(W), 0.0, 1.0, None, order, off)
    t0 = time.perf_counter()
    ol.tensor_apply(*args, x, y, threads=threads)  # warm-up, also sizes the sample
    one = time.perf_counter() - t0
    reps = max(1, min(steps, int(budget_s / max(one, 1e-6))))
    times = []
    for _ in range(reps):
        y[:] = 0.0
        t0 = time.perf_counter()
        ol.tensor_apply(*args, x, y, threads=threads)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    sample = f"{reps} full applies of the 64^3 p=4 workload ({ndofs} dofs), median"
    return ndofs / sec, sec, threads, sample


def run_reference(args, rank, world):
    if rank != 0:
        return
    value, sec, threads, sample = cpu_reference_run(args.steps, args.warmup)
    probe = probe_julia()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (diagnostic sample vector)",
            "config": dict(WORKLOAD, parallelism="host threads"), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "reference_probe": probe},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def solve_legs(gb, L, plan, prob, target=1e-8, only=None):
    """Time to relative L2 error <= `target` on the same workload with f = 3 pi^2 prod sin(pi x_i)
    (exact u = prod sin): each method solves with ||r|| <= rtol ||b|| for rtol = 1e-6, 1e-7, ...
    and reports the first solve whose relative L2 error (verification.jl:297-304) meets the
    target.  Times are device seconds of the Krylov solve (CUDA events inside grico_cg_solve);
    the hierarchy set-up is reported separately."""
    import ctypes as C

    from grico_b200.multigrid import GeometricMultigridPreconditioner, build_multigrid

    exact = lambda X: np.prod(np.sin(np.pi * X), axis=1)
    prob.rhs_operators = [gb.Load(lambda X: 3.0 * np.pi ** 2 * exact(X))]
    b = gb.reduced_rhs(plan)
    cheb = lambda deg, steps, prec="fp64": GeometricMultigridPreconditioner(
        smoother="chebyshev", chebyshev_degree=deg, pre_smoothing_steps=steps, post_smoothing_steps=steps,
        precision=prec)
    # name: (short id, preconditioner, maxiter); every solve of a leg runs inside an NVTX range
    # named by the short id (profilers filter on it)
    legs = {
        "fp64_cg_gmg_jacobi_v22 (reference method)": ("ref_jacobi", GeometricMultigridPreconditioner(), 2000),
        "fp64_cg_gmg_chebyshev2_v22 (plain FP64 GPU, no CUDA graph)": ("fp64_nograph", cheb(2, 2), 500),
        "fp64_cg_gmg_chebyshev2_v22 (plain FP64 GPU)": ("fp64", cheb(2, 2), 500),
        "mixed_cg_fp64_gmg_chebyshev2_v22_fp32": ("mixed2", cheb(2, 2, "fp32"), 500),
        "mixed_cg_fp64_gmg_chebyshev3_v22_fp32": ("mixed3", cheb(3, 2, "fp32"), 500),
    }
    import torch

    out = {}
    for name, (sid, opts, maxiter) in legs.items():
        if only and sid not in only:
            continue
        t0 = time.perf_counter()
        mg = build_multigrid(plan, opts)
        setup = time.perf_counter() - t0
        # one loose solve first: it captures the iteration graph that the plan keeps for the
        # timed solves with this hierarchy; its time (capture included) is reported beside them
        x = np.zeros(plan.n_reduced)
        so = L.GricoSolveOptions(1e-2, 0.0, maxiter, L.GRICO_PRECOND_MULTIGRID, 30, 0)
        rep = L.GricoSolveReport()
        flags = L.GRICO_FLAG_HOST_POINTERS | (L.GRICO_FLAG_NO_GRAPH if "no CUDA graph" in name else 0)
        L.lib().grico_cg_solve(plan.handle, mg.handle, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
                               C.byref(so), C.byref(rep), flags)
        first = {"rtol": 1e-2, "iterations": int(rep.iterations), "solve_seconds": float(rep.seconds)}
        tries = []
        hit = None
        for rtol in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9, 1e-10):
            x = np.zeros(plan.n_reduced)
            so = L.GricoSolveOptions(rtol, 0.0, maxiter, L.GRICO_PRECOND_MULTIGRID, 30, 0)
            rep = L.GricoSolveReport()
            flags = L.GRICO_FLAG_HOST_POINTERS | (L.GRICO_FLAG_NO_GRAPH if "no CUDA graph" in name else 0)
            torch.cuda.nvtx.range_push(sid)
            rc = L.lib().grico_cg_solve(plan.handle, mg.handle, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
                                        C.byref(so), C.byref(rep), flags)
            torch.cuda.nvtx.range_pop()
            err = gb.relative_l2_error(gb.State(plan, gb.expand_reduced(plan, x), rep), exact)
            tries.append({"rtol": rtol, "status": int(rc), "iterations": int(rep.iterations),
                          "solve_seconds": float(rep.seconds), "relative_l2_error": err})
            if rc == 0 and err <= target:
                hit = tries[-1]
                break
            if rc != 0:
                break
        out[name] = {"time_to_target_seconds": hit["solve_seconds"] if hit else None,
                     "iterations": hit["iterations"] if hit else None, "target_relative_l2": target,
                     "host_setup_seconds": setup, "levels": len(mg.plans), "first_solve": first,
                     "tries": tries}
        del mg
    return out


def learned_legs(gb, L, refine=7, train_refine=5, train_fields=6, train_steps=200, target=1e-8):
    """Variable-coefficient workload: -div(exp(g) grad u) = 1, g a Gaussian random field
    (correlation length 0.05, variance 2), 2^refine cells per axis, p = 2, FGMRES(30) + hp-GMG
    V(2,2) Chebyshev(3).  Legs: plain FP64, FP32 V-cycle, learned sweep (FP64), learned sweep +
    FP32 V-cycle, and the reference's own method in FP64 (damped Jacobi V(2,2), the SPD default
    of multigrid.jl:66-96); each reports the device time of the first FGMRES solve (rtol 1e-4,
    1e-5, ...) whose relative L2 distance to a converged FP64 state is <= target."""
    import ctypes as C

    import torch

    from grico_b200 import learned as lr
    from grico_b200.multigrid import GeometricMultigridPreconditioner, Multigrid, build_hierarchy

    t0 = time.perf_counter()
    samples = []
    for seed in range(100, 100 + train_fields):
        prob1, f1 = lr.grf_diffusion_problem(train_refine, degree=1, seed=seed)
        plan1 = gb.compile(prob1)
        o1 = GeometricMultigridPreconditioner(smoother="chebyshev")
        mg1 = Multigrid(*build_hierarchy(plan1, o1), o1)
        smp = lr.TrainingSample(plan1, lr.level_log_coefficient(plan1, f1))
        rng = np.random.default_rng(seed)
        rhs = [gb.reduced_rhs(plan1)] + [rng.standard_normal(plan1.n_reduced) for _ in range(3)]
        smp.residuals = [torch.tensor(r, dtype=torch.float32, device="cuda")
                         for r in lr.gmg_residuals(plan1, mg1, rhs, iterations=(1, 2, 3, 4))]
        samples.append(smp)
        del mg1
    net = lr.SmootherNet(seed=0)
    tr = lr.Trainer(net, lr=2e-3)
    rng = np.random.default_rng(0)
    losses = []
    torch.cuda.synchronize()
    t_train = time.perf_counter()
    for step in range(train_steps):
        smp = samples[step % len(samples)]
        pick = rng.choice(len(smp.residuals), size=min(4, len(smp.residuals)), replace=False)
        losses.append(tr.step(smp, [smp.residuals[i] for i in pick]))
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t_train
    data_s = t_train - t0

    prob, field = lr.grf_diffusion_problem(refine, degree=2, seed=0)
    plan = gb.compile(prob)
    b = gb.reduced_rhs(plan)

    def fgmres(mg, rtol, maxiter=1000):
        x = np.zeros(plan.n_reduced)
        so = L.GricoSolveOptions(rtol, 0.0, maxiter, L.GRICO_PRECOND_MULTIGRID, 30, 0)
        rep = L.GricoSolveReport()
        rc = L.lib().grico_fgmres_solve(plan.handle, mg.handle, L.ptr(b, C.c_double), L.ptr(x, C.c_double),
                                        C.byref(so), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS)
        return rc, rep, x

    results = {}
    ref = None
    for prec in ("fp64", "fp32"):
        opts = GeometricMultigridPreconditioner(smoother="chebyshev", pre_smoothing_steps=2, post_smoothing_steps=2,
                                                precision=prec)
        plans, transfers = build_hierarchy(plan, opts)
        for learned in (False, True):
            mg = Multigrid(plans, transfers, opts)
            level = len(plans) - 2
            if learned:
                lr.attach(mg, plans[level], level, net, lr.level_log_coefficient(plans[level], field))
            if ref is None:
                rc, rep, ref = fgmres(mg, 1e-12, 3000)
                ref_state = gb.State(plan, gb.expand_reduced(plan, ref), rep)
                ref_norm = gb.l2_error(ref_state, lambda X: np.zeros(X.shape[0]))
                if rc != 0 or not ref_norm > 0:
                    raise RuntimeError(f"reference solve failed: status {rc}, iterations {rep.iterations}, "
                                       f"|b| {np.linalg.norm(b)}, |x| {np.linalg.norm(ref)}, "
                                       f"{L.lib().grico_last_error().decode()}")
            tries, hit = [], None
            for rtol in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9):
                rc, rep, x = fgmres(mg, rtol)
                diff = gb.State(plan, gb.expand_reduced(plan, x - ref), rep)
                err = gb.l2_error(diff, lambda X: np.zeros(X.shape[0])) / ref_norm
                tries.append({"rtol": rtol, "status": int(rc), "iterations": int(rep.iterations),
                              "solve_seconds": float(rep.seconds), "relative_l2_error": err})
                if rc == 0 and err <= target:
                    hit = tries[-1]
                    break
            name = ("learned+" if learned else "") + ("mixed_fp32_vcycle" if prec == "fp32" else "fp64")
            entry = {"time_to_target_seconds": hit["solve_seconds"] if hit else None,
                     "iterations": hit["iterations"] if hit else None, "tries": tries}
            if learned:
                entry["learned_sweeps"], entry["learned_kept"] = lr.learned_stats(mg)
            results[name] = entry
            del mg
    # the reference's method on the GPU: FP64, damped Jacobi (omega 0.8) V(2,2), without and with
    # the learned sweep (the same V-cycle; the sweep replaces the last pre-smoothing step)
    opts = GeometricMultigridPreconditioner()
    plans, transfers = build_hierarchy(plan, opts)
    for learned in (False, True):
        mg = Multigrid(plans, transfers, opts)
        level = len(plans) - 2
        if learned:
            lr.attach(mg, plans[level], level, net, lr.level_log_coefficient(plans[level], field))
        tries, hit = [], None
        for rtol in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9):
            rc, rep, x = fgmres(mg, rtol, 3000)
            diff = gb.State(plan, gb.expand_reduced(plan, x - ref), rep)
            err = gb.l2_error(diff, lambda X: np.zeros(X.shape[0])) / ref_norm
            tries.append({"rtol": rtol, "status": int(rc), "iterations": int(rep.iterations),
                          "solve_seconds": float(rep.seconds), "relative_l2_error": err})
            if rc == 0 and err <= target:
                hit = tries[-1]
                break
            if rc != 0:
                break
        name = ("learned+" if learned else "") + "fp64_reference_jacobi_v22"
        results[name] = {"time_to_target_seconds": hit["solve_seconds"] if hit else None,
                         "iterations": hit["iterations"] if hit else None, "tries": tries}
        if learned:
            results[name]["learned_sweeps"], results[name]["learned_kept"] = lr.learned_stats(mg)
        del mg
    return {"dofs": plan.n_full, "levels": len(plans), "train": {
        "fields": train_fields, "field_cells": f"{2 ** train_refine}^3 (degree 1)", "residual_grids":
        sum(len(s.residuals) for s in samples), "steps": train_steps, "train_seconds": train_s,
        "data_seconds": data_s, "loss_first": float(np.mean(losses[:10])), "loss_last": float(np.mean(losses[-10:]))},
        "legs": results, "target_relative_l2": target}


def batched_legs(gb, L, max_level=7, nrhs=32, rtol=1e-10):
    """Adaptive hp L-shape (hanging nodes, degrees 2..7) with 32 Gaussian-bump loads: 32 single
    CG solves one after another vs one lockstep solve (FP64, and FP32 inside FP64 refinement);
    device seconds of the solves, tiles autotuned per batch first."""
    import ctypes as C

    import torch

    from grico_b200 import batched as bt

    t0 = time.perf_counter()
    plan = gb.compile(bt.lshape_problem(max_level=max_level))
    setup = time.perf_counter() - t0
    tiles = {p: bt.autotune(plan, nrhs=nrhs, precision=p, reps=5).tolist() for p in ("fp64", "fp32")}
    B = bt.reduced_rhs_many(plan, bt.gaussian_bumps(nrhs, seed=0))
    # single-right-hand-side solves, one after another
    single_s, single_it = 0.0, []
    for s in range(nrhs):
        x = np.zeros(plan.n_reduced)
        so = L.GricoSolveOptions(rtol, 0.0, 100000, L.GRICO_PRECOND_JACOBI, 30, 0)
        rep = L.GricoSolveReport()
        L.check(L.lib().grico_cg_solve(plan.handle, None, L.ptr(B[s], C.c_double), L.ptr(x, C.c_double),
                                       C.byref(so), C.byref(rep), L.GRICO_FLAG_HOST_POINTERS), "cg")
        single_s += rep.seconds
        single_it.append(rep.iterations)
    out = {"dofs": plan.n_full, "reduced_dofs": plan.n_reduced, "cells": int(len(plan.space.leaves)),
           "batches": [[int(b.degree[0]), len(b.cells)] for b in plan.batches], "nrhs": nrhs, "rtol": rtol,
           "host_setup_seconds": setup, "tiles": tiles,
           "single_cg_fp64": {"seconds": single_s, "iterations_max": max(single_it)}}
    # three repeats of each lockstep solve (each captures its iteration graph; the first call on
    # the plan also allocates the solver's work buffers): the median is the leg's time, all
    # repeats are reported with their iteration counts
    for name, mixed in (("lockstep_cg_fp64", False), ("lockstep_cg_fp32_in_fp64_refinement", True)):
        times, its = [], []
        for _ in range(3):
            X, reps = bt.solve_many(plan, B, relative_tolerance=rtol, mixed=mixed)
            times.append(float(reps[0].seconds))
            its.append(int(max(r.iterations for r in reps)))
        out[name] = {"seconds": float(np.median(times)), "repeats_seconds": times, "repeats_iterations_max": its,
                     "iterations_max": max(r.iterations for r in reps),
                     "status": sorted({int(r.status) for r in reps})}
    # operator throughput, 1 vs nrhs right-hand sides (FP64 and FP32)
    for prec, dt in ((L.GRICO_PREC_FP64, torch.float64), (L.GRICO_PREC_FP32, torch.float32)):
        for k in (1, nrhs):
            xv = torch.ones(k * plan.n_reduced, dtype=dt, device="cuda")
            yv = torch.empty_like(xv)
            st = torch.cuda.Stream()
            for _ in range(3):
                L.lib().grico_reduced_apply(plan.handle, xv.data_ptr(), yv.data_ptr(), k, prec, 0, st.cuda_stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(20):
                L.lib().grico_reduced_apply(plan.handle, xv.data_ptr(), yv.data_ptr(), k, prec, 0, st.cuda_stream)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 20
            out[f"apply_{'fp64' if prec == L.GRICO_PREC_FP64 else 'fp32'}_nrhs{k}"] = {
                "ms": ms, "dofs_per_s": k * plan.n_reduced / (ms * 1e-3)}
    return out


def probe_julia():
    """The reference itself is Julia: record whether this host can run it."""
    import shutil

    exe = shutil.which("julia")
    if exe is None:
        return "julia: not found on PATH (reference CPU path unavailable on this host)"
    try:
        r = subprocess.run([exe, "--version"], capture_output=True, text=True, timeout=30)
        return (r.stdout or r.stderr).strip()
    except Exception as exc:  # noqa: BLE001
        return f"julia present but --version failed: {exc}"


def _timed_device(fn, reps, stream):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def c1_leg(gb, L, peak):
    """2-D Poisson, 32 x 32 cells, p = 4, q = 5 (16,641 dofs), homogeneous Dirichlet: 100
    matrix-free applies (direct launches, and replayed as one CUDA graph) and the CG + Jacobi
    solve to relative residual 1e-10, checked against the exact solution."""
    import torch

    d = gb.Domain((0.0, 0.0), (1.0, 1.0), (32, 32))
    sp = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(4)))
    u = gb.ScalarField(sp)
    prob = gb.AffineProblem(u)
    gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
    gb.add_cell_accumulator(prob, u, gb.Load(lambda X: 2 * np.pi ** 2 * np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1])))
    for a in (1, 2):
        for side in (gb.LOWER, gb.UPPER):
            gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, side), 0.0))
    t0 = time.perf_counter()
    plan = gb.compile(prob)
    setup = time.perf_counter() - t0
    n = plan.n_full
    x = torch.tensor(sample_vector(n), device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    st = torch.cuda.Stream()

    def apply():
        L.lib().grico_apply(plan.handle, x.data_ptr(), y.data_ptr(), 1, L.GRICO_PREC_FP64, 0, st.cuda_stream)

    for _ in range(10):
        apply()
    torch.cuda.synchronize()
    ms_direct = _timed_device(apply, 100, st)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(st):
        with torch.cuda.graph(g, stream=st):
            for _ in range(100):
                apply()
    with torch.cuda.stream(st):  # replay() launches on the current stream: the timed one
        g.replay()
        torch.cuda.synchronize()
        ms_graph = _timed_device(g.replay, 5, st) / 100
    del g
    exact = lambda X: np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1])
    gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-10)  # warm
    t0 = time.perf_counter()
    state = gb.solve(plan, solver=gb.CGSolver(gb.JacobiPreconditioner()), relative_tolerance=1e-10)
    wall = time.perf_counter() - t0
    alg = 2 * 8 * n
    best = min(ms_direct, ms_graph)
    # the oracle's C port of the reference tensor schedule (2-D), all host threads, 100 applies
    cpu = None
    try:
        for sub in ("oracle", "tests"):
            sys.path.insert(0, os.path.join(ROOT, sub))
        from full_size_cases import oracle_cell_sum, uniform_oracle
        import oracle_lib as ol

        coords, m, ndofs, _ = uniform_oracle((32, 32), 4)
        xs = sample_vector(ndofs)
        oracle_cell_sum((32, 32), 4, coords, m, xs, 1.0 / 32)
        t0 = time.perf_counter()
        for _ in range(100):
            oracle_cell_sum((32, 32), 4, coords, m, xs, 1.0 / 32)
        sec = (time.perf_counter() - t0) / 100
        cpu = {"value": ndofs / sec, "unit": "DOFs/s", "cores": ol.max_threads(), "kind": "port",
               "sample": "100 applies of the 32x32 p=4 workload (oracle C restatement, all threads)"}
    except Exception as exc:  # noqa: BLE001
        cpu = {"value": None, "error": str(exc)[:200]}
    return {"metric": "DOFs/s matrix-free apply (100 applies) and CG+Jacobi time to rtol 1e-10",
            "config": {"workload": "poisson2d_32x32_p4_dirichlet", "cells": "32x32", "degree": 4,
                       "quadrature": "gauss 5x5", "dofs": n, "reduced_dofs": plan.n_reduced},
            "value": n / (best * 1e-3), "unit": "DOFs/s", "dtype": "f64",
            "apply_ms_direct": ms_direct, "apply_ms_graph": ms_graph, "applies_100_ms": 100 * best,
            "solve": {"iterations": int(state.report.iterations), "device_seconds": float(state.report.seconds),
                      "wall_seconds_with_host_copies": wall, "l2_error": gb.l2_error(state, exact)},
            "host_setup_seconds": setup,
            "roofline": {"bound": "hbm", "achieved": alg / (best * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (best * 1e-3) / 1e9 / peak, "traffic": None,
                         "note": "266 KB per apply stay in L2: launch latency, not HBM, bounds this size"},
            "cpu_baseline": cpu}


def c3_leg(gb, L, peak):
    out = batched_legs(gb, L)
    a = out["apply_fp64_nrhs32"]
    alg = 2 * 8 * out["reduced_dofs"] * 32
    return {"metric": "time to rtol 1e-10 for 32 right-hand sides (adaptive hp L-shape)",
            "value": out["lockstep_cg_fp64"]["seconds"], "unit": "s", "higher_is_better": False,
            "config": {"workload": "lshape_hp32", "levels": "2..7", "degrees": "2..7", "nrhs": 32},
            "batched": out,
            "roofline": {"bound": "hbm", "achieved": alg / (a["ms"] * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (a["ms"] * 1e-3) / 1e9 / peak, "traffic": None,
                         "note": "FP64 reduced apply for 32 right-hand sides: 2*8*n_reduced*32 bytes per apply"},
            "cpu_baseline": {"value": None, "reason": "the oracle's C port covers single-term (conforming) maps only; "
                                                      "this mesh has hanging-node expansions"}}


def conv_legs(L, peak_tf):
    """The network's 3x3x3 convolutions, CUDA-core kernel (FP32 arithmetic, channel-first) vs the
    tcgen05 tensor-core kernel (BF16 operands, channels-last): device time per call (CUDA
    events, 20 calls after 3), on the 65^3 vertex grid of the 64^3-cell learned level and on a
    batch of four 64^3 grids."""
    import ctypes as C

    import torch

    lib = L.lib()
    st = torch.cuda.Stream()
    out = []
    P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    for (B, Ci, Co, Z, Y, X) in ((4, 32, 32, 64, 64, 64), (1, 32, 32, 65, 65, 65), (1, 16, 32, 65, 65, 65),
                                 (1, 32, 1, 65, 65, 65)):
        g = torch.Generator(device="cuda").manual_seed(B * 100 + Ci + Co)
        with torch.cuda.stream(st):
            x = torch.randn(B, Ci, Z, Y, X, device="cuda", generator=g).bfloat16()
            xcl = x.permute(0, 2, 3, 4, 1).contiguous()
            w = 0.2 * torch.randn(Co, Ci, 27, device="cuda", generator=g)
            b = torch.randn(Co, device="cuda", generator=g)
            y = torch.empty(B, Co, Z, Y, X, device="cuda", dtype=torch.bfloat16)
            lay = 1 if Co % 8 else 0
            ytc = (torch.empty(B, Co, Z, Y, X, device="cuda") if lay else
                   torch.empty(B, Z, Y, X, Co, device="cuda", dtype=torch.bfloat16))
            wp = torch.empty(lib.grico_conv_tc_weight_bytes(Ci, Co) // 2, device="cuda", dtype=torch.bfloat16)
        torch.cuda.synchronize()
        sh = C.c_void_p(st.cuda_stream)
        L.check(lib.grico_conv3d_pack_weights_tc(P(w), Ci, Co, P(wp), sh), "pack")
        calls = {"cuda_core_fp32": lambda: lib.grico_conv3d_forward(P(x), 1, P(w), P(b), P(y), 1, B, Ci, Co, Z, Y, X,
                                                                    1, sh),
                 "tcgen05_bf16": lambda: lib.grico_conv3d_forward_tc(P(xcl), P(wp), P(b), P(ytc), lay, B, Ci, Co, Z, Y,
                                                                     X, 1, sh)}
        row = {"batch": B, "ci": Ci, "co": Co, "grid": [Z, Y, X]}
        flops = 2.0 * B * Z * Y * X * Co * Ci * 27
        for name, fn in calls.items():
            for _ in range(3):
                L.check(fn(), name)
            torch.cuda.synchronize()
            ms = _timed_device(fn, 20, st)
            row[name] = {"us": ms * 1e3, "tflops": flops / (ms * 1e-3) / 1e12}
        L.check(lib.grico_conv_tc_status(sh), "conv tc status")
        ref = y.float()
        got = ytc.float() if lay else ytc.float().permute(0, 4, 1, 2, 3)
        row["max_rel_diff"] = float((ref - got).abs().max() / ref.abs().max())
        row["speedup"] = row["cuda_core_fp32"]["us"] / row["tcgen05_bf16"]["us"]
        row["tcgen05_frac_of_bf16_peak"] = row["tcgen05_bf16"]["tflops"] / peak_tf
        out.append(row)
    return out


def c4_leg(gb, L):
    out = learned_legs(gb, L, refine=6)
    leg = out["legs"]
    return {"metric": "time to relative L2 error 1e-8 (learned + mixed vs plain FP64 GPU)",
            "value": leg["learned+mixed_fp32_vcycle"]["time_to_target_seconds"], "unit": "s",
            "higher_is_better": False,
            "config": {"workload": "grf_learned64", "cells": "64^3", "degree": 2,
                       "solver": "FGMRES(30) + hp-GMG V(2,2)",
                       "note": "64^3 cells in the default run; --workload grf_learned128 runs 128^3"},
            "plain_fp64_seconds": leg["fp64"]["time_to_target_seconds"], "learned": out,
            "network_convolutions": conv_legs(L, load_bf16_peak()),
            "cpu_baseline": {"value": None, "reason": "no CPU port of the FGMRES + GMG solve at this size"}}


def c5_leg(gb, L, peak):
    """Finite-cell shell, 64^3 background cells, p = 3: FP64 and FP32 full applies."""
    import torch

    t0 = time.perf_counter()
    plan = gb.compile(build_fcm_problem(gb, refine=6))
    setup = time.perf_counter() - t0
    n = plan.n_full
    res = {}
    for prec, dt, name in ((L.GRICO_PREC_FP64, torch.float64, "fp64"), (L.GRICO_PREC_FP32, torch.float32, "fp32")):
        x = torch.tensor(sample_vector(n), device="cuda", dtype=dt)
        y = torch.empty_like(x)
        st = torch.cuda.Stream()
        fn = lambda: L.lib().grico_apply(plan.handle, x.data_ptr(), y.data_ptr(), 1, prec, 0, st.cuda_stream)
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        ms = _timed_device(fn, 20, st)
        res[name] = {"ms": ms, "dofs_per_s": n / (ms * 1e-3)}
    alg = 2 * 8 * n
    sub = [b for b in plan.point_batches if b.kind == L.GRICO_ITEM_SUBCELLS]
    return {"metric": "DOFs/s finite-cell matrix-free apply", "value": res["fp64"]["dofs_per_s"], "unit": "DOFs/s",
            "config": dict(FCM_WORKLOAD, dofs=n, cut_cells=plan.n_cut,
                           subcells=int(sum(len(b.subcell_level) for b in sub))),
            "apply": res, "host_setup_seconds": setup,
            "roofline": {"bound": "hbm", "achieved": alg / (res["fp64"]["ms"] * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg / (res["fp64"]["ms"] * 1e-3) / 1e9 / peak,
                         "traffic": FCM_SUBCELL_TRAFFIC_PER_SUBCELL * sum(len(b.subcell_level) for b in sub),
                         "traffic_note": "subcell kernel DRAM bytes per launch, scaled by the subcells from an ncu "
                                         "capture on the 32^3 shell (19,729,664 B for 469,928 subcells)",
                         "note": "whole FP64 apply (all batches); the cut-cell subcell kernel dominates"},
            "cpu_baseline": {"value": None, "reason": "the oracle's C port covers tensor cells only; the cut-cell "
                                                      "oracle is the pure-Python restatement (test sizes)"}}


def config_legs(gb, L, only=None):
    """Every benchmark configuration besides the headline one, each in its own try block."""
    import traceback

    peak, _ = load_peaks()
    legs = {"c1_poisson2d_32_p4": lambda: c1_leg(gb, L, peak), "c3_lshape_hp32": lambda: c3_leg(gb, L, peak),
            "c4_grf_learned64": lambda: c4_leg(gb, L), "c5_fcm_shell64": lambda: c5_leg(gb, L, peak)}
    out = {}
    for name, fn in legs.items():
        if only and name not in only:
            continue
        t0 = time.perf_counter()
        try:
            out[name] = fn()
        except Exception as exc:  # noqa: BLE001
            out[name] = {"error": f"{type(exc).__name__}: {exc}"[:300], "trace": traceback.format_exc()[-600:]}
        out[name]["leg_wall_seconds"] = time.perf_counter() - t0
    return out


def sharded_leg(gb, plan, rank, world, steps, warmup):
    """The same mesh split over the ranks (strong scaling): each rank applies the reduced
    operator of its Morton range of cells and the partition-surface halo is summed, either by
    point-to-point exchange with the ranks sharing dofs (NCCL send/receive, the default) or by
    one NCCL all-reduce over every halo slot.  Device time with CUDA events, max over ranks; the
    result is checked against the unsharded reduced apply on this rank's dofs."""
    import torch
    import torch.distributed as dist

    from grico_b200.sharded import ShardedOperator, ShardGroup, ShardPlan

    t0 = time.perf_counter()
    shard = ShardPlan(plan, rank, world)
    setup = time.perf_counter() - t0
    xg = sample_vector(plan.n_reduced)
    ref = gb.reduced_apply(plan, xg)[shard.global_reduced]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    res = []
    for mode in ("neighbours", "allreduce"):
        op = ShardedOperator([shard], ShardGroup(halo=mode))
        x = op.ops.upload(shard.scatter(xg))
        y = op.ops.vector(shard.n_reduced)
        for _ in range(warmup):
            op.apply([x], [y])
        res.append(timed(lambda: op.apply([x], [y])))
        res.append(float(np.max(np.abs(y.cpu().numpy()[: shard.n_reduced] - ref)) / np.max(np.abs(ref))))
    yl = op.ops.vector(shard.n_reduced)
    res.append(timed(lambda: op.ops.apply(shard, x, yl)))  # the local apply alone
    t = torch.tensor(res, device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, err, ms_ar, err_ar, ms_local = (float(v) for v in t.cpu())
    return {"metric": "sharded reduced apply throughput (one 64^3 p=4 mesh split over the GPUs)",
            "value": plan.n_reduced / (ms * 1e-3), "unit": "DOFs/s", "scaling": "strong",
            "ms_per_apply": ms, "allreduce_halo_ms_per_apply": ms_ar, "local_apply_ms_max": ms_local,
            "halo_slots": shard.n_halo, "neighbours_rank0": [q for q, _ in shard.neighbours],
            "halo_bytes_per_apply_rank0": 16 * sum(int(pos.size) for _, pos in shard.neighbours),
            "cells_rank0": int(sum(len(b.cells) for b in shard.plan.batches)),
            "partition": "contiguous Morton ranges balanced by (p+1)^3 q^3",
            "collective": "NCCL send/receive with the neighbouring ranks (ms_per_apply); NCCL all-reduce of every "
                          "halo slot (allreduce_halo_ms_per_apply)",
            "max_rel_err_vs_unsharded": max(err, err_ar), "shard_setup_seconds": setup}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--soak", type=float, default=1.5, help="seconds of untimed load while clocks are sampled")
    ap.add_argument("--no-solve", action="store_true", help="skip the CG+GMG time-to-tolerance legs")
    ap.add_argument("--solve-legs", default="", help="comma-separated short ids of the solve legs to run "
                    "(ref_jacobi, fp64_nograph, fp64, mixed2, mixed3); default: all")
    ap.add_argument("--workload", default="poisson64",
                    choices=["poisson64", "fcm_shell64", "fcm_shell32", "grf_learned128", "grf_learned64",
                             "lshape_hp32", "lshape_apply32", "conv_tc", "sipg3d", "dense_tc64"],
                    help="poisson64: 3-D Poisson 64^3 p=4 (default); fcm_shell*: finite-cell shell with Nitsche")
    ap.add_argument("--fp32", action="store_true", help="time the FP32 apply instead of FP64")
    ap.add_argument("--train-fields", type=int, default=6, help="grf_learned*: training fields (32^3 cells each)")
    ap.add_argument("--train-steps", type=int, default=200, help="grf_learned*: Adam steps")
    ap.add_argument("--no-configs", action="store_true", help="skip the other benchmark configurations")
    ap.add_argument("--configs", default="", help="comma-separated config legs to run (c1_poisson2d_32_p4, "
                    "c3_lshape_hp32, c4_grf_learned64, c5_fcm_shell64); default: all")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import grico_b200 as gb
    from grico_b200 import _lib as L

    if args.workload == "conv_tc":
        # the network's convolutions alone (CUDA-core vs tensor-core kernels), for profiling
        rows = conv_legs(L, load_bf16_peak())
        if rank == 0:
            print(json.dumps({"metric": "3x3x3 convolution device time", "unit": "us", "n_gpus": world,
                              "higher_is_better": False, "data": "synthetic (seeded normal activations)",
                              "config": {"workload": "conv_tc"}, "convolutions": rows}), flush=True)
        return
    if args.workload == "sipg3d":
        # DG (SIPG) Poisson on the unit cube, 16^3 cells of degree 3: FP64 full apply
        import torch

        d = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (16, 16, 16))
        sp = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(3), continuity="dg"))
        u = gb.ScalarField(sp)
        prob = gb.AffineProblem(u)
        gb.add_cell_accumulator(prob, u, u, gb.Diffusion())
        gb.add_interface(prob, gb.SIPG(10.0))
        plan = gb.compile(prob)
        st = torch.cuda.Stream()
        xv = torch.tensor(sample_vector(plan.n_full), dtype=torch.float64, device="cuda")
        yv = torch.empty_like(xv)
        fn = lambda: L.lib().grico_apply(plan.handle, xv.data_ptr(), yv.data_ptr(), 1, L.GRICO_PREC_FP64, 0,
                                         st.cuda_stream)
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = _timed_device(fn, args.steps, st)
        if rank == 0:
            print(json.dumps({"metric": "DG (SIPG) FP64 apply device time", "value": ms, "unit": "ms",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                              "data": "synthetic", "config": {"workload": "sipg3d", "cells": "16^3", "degree": 3,
                                                               "dofs": plan.n_full,
                                                               "interfaces": int(sum(len(b.cells) for b in plan.point_batches))},
                              "checksum": float(yv.double().sum().item())}), flush=True)
        return
    if args.workload == "dense_tc64":
        # the 64^3 p = 4 reduced FP32 apply with every 3-D kernel variant, the tensor-core
        # element-matrix variant (10) among them, against the FP64 apply
        import torch

        from grico_b200 import batched as bt

        prob = build_problem(gb)
        plan = gb.compile(prob)
        st = torch.cuda.Stream()
        nr = plan.n_reduced
        x64 = torch.tensor(sample_vector(nr), dtype=torch.float64, device="cuda")
        y64 = torch.empty_like(x64)
        x32, y32 = x64.float(), torch.empty(nr, dtype=torch.float32, device="cuda")
        f64 = lambda: L.lib().grico_reduced_apply(plan.handle, x64.data_ptr(), y64.data_ptr(), 1, L.GRICO_PREC_FP64, 0,
                                                  st.cuda_stream)
        for _ in range(args.warmup):
            f64()
        torch.cuda.synchronize()
        res = {"fp64_ms": _timed_device(f64, args.steps, st)}
        ref = y64.double()
        f32 = lambda: L.lib().grico_reduced_apply(plan.handle, x32.data_ptr(), y32.data_ptr(), 1, L.GRICO_PREC_FP32, 0,
                                                  st.cuda_stream)
        for var in (10, 3, 9, 1):
            bt.set_tiles(plan, [var] * len(plan.batches), "fp32")
            for _ in range(args.warmup):
                f32()
            torch.cuda.synchronize()
            ms = _timed_device(f32, args.steps, st)
            res[f"fp32_variant{var}"] = {"ms": ms, "rel_err_vs_fp64": float((y32.double() - ref).abs().max() / ref.abs().max())}
        L.check(L.lib().grico_tc_status(C.c_void_p(st.cuda_stream)), "tensor-core status")
        if rank == 0:
            print(json.dumps({"metric": "64^3 p=4 reduced apply device time per kernel variant", "unit": "ms",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                              "data": "synthetic", "config": {"workload": "dense_tc64", "reduced_dofs": nr}, **res}),
                  flush=True)
        return
    if args.workload == "lshape_apply32":
        # the hp L-shape's reduced FP64 apply, 1 and 32 right-hand sides, W untimed then K timed
        import torch

        from grico_b200 import batched as bt

        plan = gb.compile(bt.lshape_problem(max_level=7))
        res = {}
        st = torch.cuda.Stream()
        for k in (1, 32):
            xv = torch.ones(k * plan.n_reduced, dtype=torch.float64, device="cuda")
            yv = torch.empty_like(xv)
            fn = lambda: L.lib().grico_reduced_apply(plan.handle, xv.data_ptr(), yv.data_ptr(), k, L.GRICO_PREC_FP64,
                                                     0, st.cuda_stream)
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            res[f"nrhs{k}_ms"] = _timed_device(fn, args.steps, st)
        if rank == 0:
            print(json.dumps({"metric": "reduced FP64 apply device time (adaptive hp L-shape)", "unit": "ms",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
                              "data": "synthetic", "config": {"workload": "lshape_apply32", "dofs": plan.n_full,
                                                               "reduced_dofs": plan.n_reduced}, **res}), flush=True)
        return
    if args.workload == "lshape_hp32":
        out = batched_legs(gb, L)
        if rank == 0:
            print(json.dumps({"metric": "time to rtol 1e-10 for 32 right-hand sides (adaptive hp L-shape)",
                              "value": out["lockstep_cg_fp32_in_fp64_refinement"]["seconds"], "unit": "s",
                              "n_gpus": world, "steps": 1, "warmup": 0, "higher_is_better": False,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32",
                              "data": "synthetic (seeded Gaussian bumps)",
                              "config": {"workload": "lshape_hp32", "levels": "2..7", "degrees": "2..7"},
                              "batched": out}), flush=True)
        return
    if args.workload.startswith("grf_learned"):
        out = learned_legs(gb, L, refine=7 if args.workload.endswith("128") else 6, train_fields=args.train_fields,
                           train_steps=args.train_steps)
        leg = out["legs"]
        value = leg["learned+mixed_fp32_vcycle"]["time_to_target_seconds"]
        if rank == 0:
            print(json.dumps({"metric": "time to relative L2 error 1e-8 (learned + mixed vs plain FP64 GPU)",
                              "value": value, "unit": "s", "n_gpus": world, "steps": 1, "warmup": 0,
                              "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32",
                              "data": "synthetic (seeded Gaussian random fields)",
                              "config": {"workload": args.workload, "degree": 2, "solver": "FGMRES(30) + hp-GMG V(2,2)"},
                              "plain_fp64_seconds": leg["fp64"]["time_to_target_seconds"],
                              "reference_method_fp64_seconds": leg["fp64_reference_jacobi_v22"]["time_to_target_seconds"],
                              "learned": out}), flush=True)
        return
    fcm = args.workload.startswith("fcm")
    if fcm:
        args.no_solve = True
        prob = build_fcm_problem(gb, refine=6 if args.workload == "fcm_shell64" else 5)
    else:
        prob = build_problem(gb)
    plan = gb.compile(prob)
    n = plan.n_full
    prec = L.GRICO_PREC_FP32 if args.fp32 else L.GRICO_PREC_FP64
    vdtype = torch.float32 if args.fp32 else torch.float64
    x = torch.tensor(sample_vector(n), device="cuda", dtype=vdtype)
    y = torch.empty_like(x)
    stream = torch.cuda.Stream()  # explicit stream: the kernels and the timing events share it
    torch.cuda.synchronize()

    def step(flags=0):
        L.check(L.lib().grico_apply(plan.handle, x.data_ptr(), y.data_ptr(), 1, prec, flags,
                                    stream.cuda_stream), "apply")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        # untimed soak of identical steps so the clock samples cover a loaded GPU
        t_soak = time.perf_counter()
        while time.perf_counter() - t_soak < args.soak:
            for _ in range(50):
                step()
            torch.cuda.synchronize()
        nbt = len(plan.batches) + len(plan.point_batches)
        ms_b = np.zeros(nbt)
        L.check(L.lib().grico_plan_batch_times(plan.handle, L.ptr(ms_b, C.c_double), None, nbt), "batch times")
        start.record(stream)
        for _ in range(args.steps):
            # CUDA events around every batch kernel, recorded on the launching stream in order
            step(L.GRICO_FLAG_TIME_BATCHES)
        end.record(stream)
        torch.cuda.synchronize()
        n_b = np.zeros(nbt, dtype=np.int64)
        L.check(L.lib().grico_plan_batch_times(plan.handle, L.ptr(ms_b, C.c_double), L.ptr(n_b, C.c_int64), nbt),
                "batch times")
        # keep the sampler running for at least a few samples on short regions
        time.sleep(0.3)
    ms = start.elapsed_time(end) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    dofs_per_s = n / (ms * 1e-3) * world

    # ---- end to end through the C ABI with pinned host buffers (copies inside the timed region) ----
    # Every step copies its input from pinned host memory and its result back.  Steps alternate
    # between two streams and two result buffers (GRICO_FLAG_ASYNC), so step k's copy out
    # overlaps step k+1's copy in on the full-duplex link; the clock stops after the last result
    # is on the host.
    hx = torch.tensor(sample_vector(n), dtype=vdtype).pin_memory()
    hys = [torch.empty(n, dtype=vdtype).pin_memory() for _ in range(2)]
    e2e_streams = [torch.cuda.Stream(), torch.cuda.Stream()]

    def e2e_step(k):
        L.check(L.lib().grico_apply(plan.handle, hx.data_ptr(), hys[k % 2].data_ptr(), 1, prec,
                                    L.GRICO_FLAG_HOST_POINTERS | L.GRICO_FLAG_ASYNC,
                                    e2e_streams[k % 2].cuda_stream), "apply")

    for k in range(2):
        e2e_step(k)
    torch.cuda.synchronize()
    e2e_steps = max(3, min(args.steps, 20))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        e2e_step(k)
    for st_ in e2e_streams:
        st_.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    hy = hys[(e2e_steps - 1) % 2]
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = n / e2e_s * world
    # check the e2e result equals the device result
    torch.cuda.synchronize()
    assert torch.allclose(hy.cuda(), y, rtol=0, atol=(1e-5 if args.fp32 else 1e-12) * float(y.abs().max()))

    # the same apply with GRICO_FLAG_DETERMINISTIC (stored local results summed per dof in a fixed
    # order): device time per apply and a bitwise repeat check, outside the timed region
    det_info = None
    if world == 1:
        try:
            yd1, yd2 = torch.empty_like(y), torch.empty_like(y)
            det = lambda out: L.check(L.lib().grico_apply(plan.handle, x.data_ptr(), out.data_ptr(), 1, prec,
                                                          L.GRICO_FLAG_DETERMINISTIC, stream.cuda_stream), "det apply")
            det(yd1)
            torch.cuda.synchronize()
            det_ms = _timed_device(lambda: det(yd2), 5, stream)
            det_info = {"ms": det_ms, "bitwise_repeatable": bool(torch.equal(yd1, yd2)),
                        "max_rel_diff_vs_atomic": float((yd1 - y).abs().max() / y.abs().max())}
            del yd1, yd2
        except Exception as exc:  # noqa: BLE001
            det_info = {"error": f"{type(exc).__name__}: {exc}"[:200]}

    sharded_info = None
    if world > 1 and not fcm:
        try:
            sharded_info = sharded_leg(gb, plan, rank, world, args.steps, args.warmup)
        except Exception as exc:  # noqa: BLE001  (the headline line is printed either way)
            sharded_info = {"error": f"{type(exc).__name__}: {exc}"[:200]}

    solve_info = None
    if not args.no_solve:
        solve_info = solve_legs(gb, L, plan, prob, only=[v for v in args.solve_legs.split(",") if v])
    configs_info = None
    if not fcm and world == 1 and not args.no_configs and not args.fp32:
        configs_info = config_legs(gb, L, only=[v for v in args.configs.split(",") if v])

    if rank == 0:
        peak, peak_kind = load_peaks()
        vbytes = 4 if args.fp32 else 8
        alg_bytes = 2 * vbytes * n
        # dominant kernel: the batch with the largest device time per apply
        top = int(np.argmax(ms_b))
        kernel_ms = float(ms_b[top])
        achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
        launches = len(plan.batches) + len(plan.point_batches) + (1 if len(plan.fixed_dofs) else 0)
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "subcell_apply_fcm_shell64.txt" if fcm else
                             "cell_apply_3d_pipe_p4_poisson64.txt")
        if os.path.exists(tpath):
            for line in open(tpath):
                if line.startswith("traffic_bytes_per_full_apply:") and not args.fp32:
                    field = line.split(":", 1)[1].split()
                    try:  # a summary without a capture of this launch says "null (why)"
                        traffic = float(field[0]) if field else None
                    except ValueError:
                        traffic = None
        cpu = None
        if not args.no_cpu_baseline and world == 1 and not fcm:
            value, sec, threads, sample = cpu_reference_run(3, 1, budget_s=15.0)
            cpu = {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
        if fcm:
            sub = [b for b in plan.point_batches if b.kind == L.GRICO_ITEM_SUBCELLS]
            config = dict(FCM_WORKLOAD, dofs=n, full_cells=int(sum(len(b.cells) for b in plan.batches)),
                          cut_cells=plan.n_cut, subcells=int(sum(len(b.subcell_level) for b in sub)),
                          surface_points=int(sum(b.weights.size for b in plan.point_batches
                                                 if b.kind == L.GRICO_ITEM_NITSCHE)))
            if traffic is None:
                traffic = FCM_SUBCELL_TRAFFIC_PER_SUBCELL * config["subcells"]
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "peak_kind": peak_kind,
                    "traffic_note": "subcell kernel DRAM bytes per launch, scaled by the subcells from an ncu capture "
                                    "on the 32^3 shell (19,729,664 B for 469,928 subcells)",
                    "kernel_ms": kernel_ms, "kernel_share_of_apply": kernel_ms / ms,
                    "note": "achieved = 2*bytes(value)*n_full / average launch time of the dominant kernel "
                            "(CUDA events around each launch inside the timed region); the cut-cell subcell kernel "
                            "(FP64 pipe / shared memory) dominates"}
        else:
            config = dict(WORKLOAD)
            fp64_tflops = FLOPS_PER_CELL * 64 ** 3 / (kernel_ms * 1e-3) / 1e12
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "peak_kind": peak_kind,
                    "kernel": "cell_apply_3d_pipe<5,5,5>", "kernel_ms": kernel_ms,
                    "kernel_share_of_apply": kernel_ms / ms,
                    "note": "achieved = 2*bytes(value)*n_full / average launch time of the dominant kernel "
                            "(CUDA events around each launch inside the timed region); the FP64 pipe and shared "
                            "memory, not HBM, bound it (see fp64_tflops)",
                    "flops_per_cell": FLOPS_PER_CELL,
                    ("fp32_tflops" if args.fp32 else "fp64_tflops"): fp64_tflops}
        config.update(parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                      l2="inputs larger than L2 (x, y and cell maps each above 126 MB)" if not fcm else
                      "x, y 22 MB; subcell records 45 MB; maps and surface data above L2")
        out = {
            "metric": METRIC, "value": dofs_per_s, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.fp32 else "f64",
            "data": "synthetic (diagnostic sample vector)", "config": config,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": vbytes * n,
                    "d2h_bytes_per_step": vbytes * n},
            "gpu_launches": launches * args.steps,
            "roofline": roof,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "solve": solve_info,
        }
        if det_info is not None:
            out["deterministic_apply"] = det_info
        if sharded_info is not None:
            out["sharded"] = sharded_info
        if configs_info is not None:
            out["configs"] = configs_info
        out["reference_probe"] = probe_julia()
        if fcm:
            out["cpu_baseline_note"] = ("the oracle's C kernel covers tensor cells only; the finite-cell parity "
                                        "oracle is a pure-Python restatement (test sizes)")
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""The oracle's FGMRES and Chebyshev restatements pinned on the CPU.

FGMRES against the reference's own known answers: a 1x1 system scaled by 1e-14 solves to 1.0
(test/feature_stability.jl:178-181) and a nonsymmetric system matches a direct solve to 1e-8 at
relative tolerance 1e-12 (test/multigrid.jl:143-147).  Chebyshev: k steps of the recurrence from
x = 0 equal the closed-form Chebyshev polynomial of D^-1 A (error factor
T_k((theta - lambda)/delta) / T_k(theta/delta), Saad, Algorithm 12.1)."""
import types

import numpy as np
import pytest

import grico_oracle as go
from cases import build, rel_err


def test_fgmres_tiny_scaled_system():  # test/feature_stability.jl:178-181
    x, iters = go.fgmres_solve(lambda v: 1.0e-14 * v, np.array([1.0e-14]), rtol=1e-10)
    assert x[0] == pytest.approx(1.0)
    assert iters == 1


@pytest.mark.parametrize("restart", [30, 3])
def test_fgmres_nonsymmetric_matches_direct_solve(restart):  # test/multigrid.jl:143-147
    rng = np.random.default_rng(5)
    n = 24
    A = np.eye(n) * 4.0 + 0.6 * rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    dinv = 1.0 / np.diag(A)
    x, _ = go.fgmres_solve(lambda v: A @ v, b, precond=lambda r: dinv * r, restart=restart, rtol=1e-12)
    assert np.allclose(x, np.linalg.solve(A, b), atol=1e-8)


def test_fgmres_matches_cg_on_spd_plan():
    src = lambda x: np.prod(np.sin(np.pi * x), axis=1)
    oplan, _ = build("2d_p4", mu=0.3, source=src)
    b = oplan.reduced_rhs()
    diag = oplan.jacobi_diagonal()
    xc, _ = go.cg_solve(oplan.reduced_apply, b, precond=lambda r: r / diag, rtol=1e-12)
    xf, iters = go.fgmres_solve(oplan.reduced_apply, b, precond=lambda r: r / diag, restart=7, rtol=1e-12)
    assert rel_err(xf, xc) <= 1e-9
    assert iters > 7  # at least one restart


def test_fgmres_restart_equals_full_gmres_within_one_cycle():
    """With restart >= the iteration count the method is plain right-preconditioned GMRES: the
    residual after k steps is the minimum over the k-dimensional Krylov space."""
    rng = np.random.default_rng(8)
    n = 12
    A = np.eye(n) * 3.0 + 0.4 * rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    x, iters = go.fgmres_solve(lambda v: A @ v, b, restart=50, rtol=1e-13)
    assert iters <= n
    K = np.stack([np.linalg.matrix_power(A, k) @ b for k in range(iters)], axis=1)
    c, *_ = np.linalg.lstsq(A @ K, b, rcond=None)
    assert np.allclose(x, K @ c, atol=1e-8)


def _dense_level(A):
    plan = types.SimpleNamespace(reduced_apply=lambda v: A @ v)
    return plan


@pytest.mark.parametrize("degree", [1, 2, 3, 5])
def test_chebyshev_recurrence_equals_polynomial(degree):
    rng = np.random.default_rng(degree)
    n = 30
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(np.linspace(0.5, 40.0, n)) @ Q.T
    A = 0.5 * (A + A.T)
    dinv = 1.0 / np.diag(A)
    lam = go.estimate_lambda_max(lambda v: A @ v, dinv, 1, iterations=200)
    M = dinv[:, None] * A
    assert lam == pytest.approx(max(abs(np.linalg.eigvals(M))), rel=1e-6)
    fake = types.SimpleNamespace(plans=[None, _dense_level(A)], dinv=[None, dinv], lmax=[0.0, lam],
                                 chebyshev_lower=1.0 / 15.0, chebyshev_degree=degree)
    b = rng.standard_normal(n)
    x = go.Multigrid.smooth_chebyshev(fake, 1, np.zeros(n), b, 1)
    # closed form: e_k = p_k(D^-1 A) e_0 with e_0 = -A^-1 b
    lmax = 1.2 * lam
    lmin = lmax / 15.0
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    # D^-1 A is similar to the symmetric S = D^-1/2 A D^-1/2
    s = np.sqrt(dinv)
    S = s[:, None] * A * s[None, :]
    w, U = np.linalg.eigh(S)
    Tk = np.polynomial.chebyshev.Chebyshev.basis(degree)
    pk = Tk((theta - w) / delta) / Tk(theta / delta)
    e0 = -np.linalg.solve(A, b)
    # e_k = D^-1/2 U diag(pk) U^T D^1/2 e0
    ek = (U @ (pk * (U.T @ (e0 / s)))) * s
    assert rel_err(x - np.linalg.solve(A, b), ek) <= 1e-10


def _three_term_sweeps(A, dinv, lam, degree, x, b, steps, x_zero):
    """The device smoother's even-degree form (`chebyshev3_step` in csrc/grico_mg.cu), written
    out with its two buffers: x_{k+1} = x_k + c1 (x_k - x_{k-1}) + c2 D^-1 (b - A x_k), iterates
    alternating between `x` and `d`; with x_zero the first iterate is zero and not applied."""
    lmax = 1.2 * lam
    lmin = lmax / 15.0
    theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
    sigma = theta / delta
    bufs = {"x": np.full_like(b, np.nan) if x_zero else x.copy(), "d": np.full_like(b, np.nan)}
    for s in range(steps):
        rho_old = 1.0 / sigma
        for k in range(degree):
            cur, nxt = ("x", "d") if k % 2 == 0 else ("d", "x")
            cur_zero = s == 0 and k == 0 and x_zero
            prev_zero = s == 0 and k == 1 and x_zero
            xk = np.zeros_like(b) if cur_zero else bufs[cur]
            r = b if cur_zero else b - A @ xk
            c1, c2 = 0.0, 1.0 / theta
            if k > 0:
                rho = 1.0 / (2.0 * sigma - rho_old)
                c1, c2 = rho * rho_old, 2.0 * rho / delta
                rho_old = rho
            prev = np.zeros_like(b) if (c1 == 0.0 or prev_zero) else bufs[nxt]
            bufs[nxt] = xk + (c1 * (xk - prev) if c1 != 0.0 else 0.0) + c2 * dinv * r
    return bufs["x"]


@pytest.mark.parametrize("degree,steps,x_zero", [(2, 1, True), (2, 2, True), (4, 2, False), (2, 2, False)])
def test_three_term_chebyshev_equals_update_form(degree, steps, x_zero):
    """The even-degree three-term form of the device smoother gives the oracle's update-form
    Chebyshev sweeps (Saad, Algorithm 12.1), from a zero or a given start, to rounding."""
    rng = np.random.default_rng(3 + degree)
    n = 40
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(np.linspace(0.3, 25.0, n)) @ Q.T
    A = 0.5 * (A + A.T)
    dinv = 1.0 / np.diag(A)
    lam = go.estimate_lambda_max(lambda v: A @ v, dinv, 1, iterations=100)
    fake = types.SimpleNamespace(plans=[None, _dense_level(A)], dinv=[None, dinv], lmax=[0.0, lam],
                                 chebyshev_lower=1.0 / 15.0, chebyshev_degree=degree)
    b = rng.standard_normal(n)
    x0 = np.zeros(n) if x_zero else rng.standard_normal(n)
    ref = go.Multigrid.smooth_chebyshev(fake, 1, x0.copy(), b, steps)
    got = _three_term_sweeps(A, dinv, lam, degree, x0, b, steps, x_zero)
    assert np.all(np.isfinite(got))  # no NaN of the never-written buffers was read
    assert rel_err(got, ref) <= 1e-13


def test_power_iteration_start_is_deterministic():
    v = go.power_iteration_start(5, 3)
    assert np.all((v >= 0.5) & (v < 1.5))
    assert np.array_equal(v, go.power_iteration_start(5, 3))
    assert not np.array_equal(v, go.power_iteration_start(5, 4))

"""The oracle's Newton restatement on the reference's Bratu test configuration
(test/examples.jl:30-35: roots (2, 2), degree 2, lam 0.5, amplitude 0.1, L2 error <= 2e-3)."""
import numpy as np

import grico_oracle as go
from bratu_cases import bratu


def test_oracle_newton_meets_reference_bound():
    oplan, _, c = bratu(device=False)
    ur, its = go.bratu_newton(oplan, c["lam"], c["src_scalar"])
    err = go.l2_error(oplan, oplan.expand(ur, include_shift=True), c["ex_scalar"])
    assert its <= 10 and err <= 2.0e-3


def test_oracle_tangent_is_the_residual_derivative():
    oplan, _, c = bratu(device=False)
    rng = np.random.default_rng(0)
    n = len(oplan.solve_dofs)
    u = oplan.expand(0.1 * rng.standard_normal(n), include_shift=True)
    d = oplan.expand(rng.standard_normal(n))
    h = 1e-6
    fd = (go.bratu_residual(oplan, u + h * d, c["lam"], c["src_scalar"]) -
          go.bratu_residual(oplan, u - h * d, c["lam"], c["src_scalar"])) / (2 * h)
    t = go.bratu_tangent(oplan, u, d, c["lam"])
    assert np.max(np.abs(fd - t)) <= 1e-7 * np.max(np.abs(t))

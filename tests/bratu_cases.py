"""The manufactured Bratu problem of examples/nonlinear_bratu/driver.jl built identically in the
oracle and in the product: -lap u + lam exp(u) = f on (0, 1)^2, u = 0 on the boundary,
u_e = A sin(pi x) sin(pi y), f = 2 pi^2 u_e + lam exp(u_e)."""
import math

import numpy as np

import grico_oracle as go
import grico_b200 as gb


def bratu(roots=(2, 2), degree=2, lam=0.5, amplitude=0.1, device=True):
    """The example in 2-D (len(roots) = 2) or its 3-D analogue u_e = A prod sin(pi x_i)."""
    D = len(roots)
    exact = lambda X: amplitude * np.prod(np.sin(math.pi * X[:, :D]), axis=1)
    source = lambda X: D * math.pi ** 2 * exact(X) + lam * np.exp(exact(X))
    od = go.Domain((0.0,) * D, (1.0,) * D, roots)
    osp = go.Space(od, degree, basis="full")
    faces = [(a, s) for a in range(1, D + 1) for s in (go.LOWER, go.UPPER)]
    oplan = go.Plan(osp, mu=0.0, kappa=1.0, dirichlet=[(a, s, 0.0) for a, s in faces])
    d = gb.Domain((0.0,) * D, (1.0,) * D, roots)
    sp = gb.HpSpace(d, gb.SpaceOptions(basis=gb.FullTensorBasis(), degree=gb.UniformDegree(degree)))
    u = gb.ScalarField(sp)
    prob = gb.ResidualProblem(u)
    gb.add_residual_accumulator(prob, u, u, gb.ExpReaction(lam, source))
    for a, s in faces:
        gb.add_constraint(prob, gb.Dirichlet(u, gb.BoundaryFace(a, s), 0.0))
    plan = gb.compile_residual(prob) if device else None
    src_scalar = lambda x: float(source(np.array([x]))[0])
    ex_scalar = lambda x: float(exact(np.array([x]))[0])
    return oplan, plan, dict(lam=lam, source=source, src_scalar=src_scalar, exact=exact, ex_scalar=ex_scalar)

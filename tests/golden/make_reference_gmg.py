"""Writes reference_gmg_8cube_p4.npz (python tests/golden/make_reference_gmg.py; about 15 minutes
on one core, most of it the oracle's hierarchy set-up).

The reference's own solver at an intermediate size: the unit cube, 4^3 roots refined once (8^3
cells), degree 4, full tensor basis, mass + diffusion (1, 1), homogeneous Dirichlet on all six
faces; the oracle's hp hierarchy (p 4 -> 2 -> 1, then h-merges to the roots) and V(2,2) with
damped Jacobi (omega 0.8, multigrid.jl:858-889, 943-956).  Stored: the V-cycle of a seeded
right-hand side b (numpy default_rng(7) standard normal over the reduced dofs), and CG with that
V-cycle (solve.jl:376-431) stopped after K = 5, 10, 20 and 40 iterations: the iterates and the
residual norm after 40 (the method diverges on this modal p = 4 basis: the residual grows)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("tests", "grico.jl_b200", "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import grico_oracle as go  # noqa: E402
from test_multigrid_host import _oracle_levels, _refine_uniform  # noqa: E402

KS = (5, 10, 20, 40)
SAMPLE = slice(0, None, 7)


def main():
    od = go.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (4, 4, 4))
    _refine_uniform(od.grid, 1)
    faces = [(a, s) for a in (1, 2, 3) for s in (1, 2)]
    oplans = _oracle_levels(od, 4, faces)
    omg = go.Multigrid(oplans)
    fine = oplans[-1]
    n = len(fine.solve_dofs)
    b = np.random.default_rng(7).standard_normal(n)
    z = omg.apply(b)
    out = {}
    for k in KS:
        x, iters = go.cg_solve(fine.reduced_apply, b, precond=omg.apply, rtol=1e-14, maxiter=k,
                               raise_unconverged=False)
        assert iters == k
        out[f"cg_iterate_{k}"] = x[SAMPLE]  # every 7th reduced dof keeps the fixture small
    r = b - fine.reduced_apply(out[f"cg_iterate_{KS[-1]}"])
    np.savez(os.path.join(HERE, "reference_gmg_8cube_p4.npz"), level_sizes=np.array([len(o.solve_dofs) for o in oplans]),
             b_sum=np.array([b.sum()]), vcycle=z, cg_iterations=np.array(KS),
             cg_residual_norm=np.array([np.linalg.norm(r)]), b_norm=np.array([np.linalg.norm(b)]), **out)


if __name__ == "__main__":
    main()

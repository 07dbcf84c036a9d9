"""The adaptive hp L-shape (mixed degrees 2..4, hanging nodes, re-entrant Dirichlet faces) on the
device against the oracle.

On this mesh the reference's continuity compile meets redundant constraint rows that cancel to
rounding level; their pivots are noise (|pivot| ~ 1e-15) and eliminate a genuine free variable,
so the reference's dof numbering depends on the last bits of its LU.  The product drops those
rows and keeps the extra dofs.  The checks therefore do not compare dof by dof:

* bilinear form: for random functions u_i of the oracle's reduced space (which is contained in
  the product's), the Gram matrix G_ij = a(u_i, u_j) from the oracle's reduced apply equals the
  one from the device's reduced apply on the same functions written in the product's
  coefficients (leaf-local mode coefficients are numbering independent);
* operator on the product's maps: the oracle's cell kernel (accumulators.jl:1022-1054) on the full
  box of modes, gathered and scattered through the product's term maps (hanging-node expansions
  included) and with the
  product's constraint rows (fixed dofs and Dirichlet relations, assembly.jl:1893-1920), equals
  the device's full apply, reduced apply and exact reduced diagonal (the probe of
  solve.jl:722-738) to 1e-12."""
import numpy as np
import pytest

import grico_b200 as gb
from cases import rel_err
from lshape_cases import NOISE, box_local_apply, cell_sum, expand, full_apply, project, setup, to_product

pytestmark = pytest.mark.gpu
TOL = 1e-12
MU, KAPPA = 0.3, 1.7


@pytest.fixture(scope="module")
def lshape():
    return setup(mu=MU, kappa=KAPPA)


def test_lshape_has_dirichlet_relations(cuda, lshape):
    _, plan, _ = lshape
    assert len(plan.relations) > 0  # hanging-node traces on Dirichlet faces


def test_lshape_bilinear_form_matches_oracle(cuda, lshape):
    oplan, plan, terms = lshape
    rng = np.random.default_rng(3)
    U = rng.standard_normal((6, len(oplan.solve_dofs)))
    G_or = np.array([[uj @ oplan.reduced_apply(ui) for uj in U] for ui in U])
    X = np.stack([to_product(oplan, plan, terms, u) for u in U])
    Y = np.stack([gb.reduced_apply(plan, x.copy()) for x in X])
    assert rel_err(X @ Y.T, G_or) <= NOISE


def test_lshape_full_and_reduced_apply(cuda, lshape):
    oplan, plan, terms = lshape
    x = np.random.default_rng(5).uniform(-1.0, 1.0, plan.n_full)
    assert rel_err(gb.apply(plan, x.copy()), full_apply(oplan, plan, terms, x)) <= TOL
    xr = np.random.default_rng(6).uniform(-1.0, 1.0, plan.n_reduced)
    ref = project(plan, cell_sum(oplan, plan, terms, expand(plan, xr)))
    assert rel_err(gb.reduced_apply(plan, xr), ref) <= TOL


def test_lshape_exact_diagonal(cuda, lshape):
    oplan, plan, terms = lshape
    diag = np.zeros(plan.n_reduced)
    for li, c in enumerate(oplan.cells):
        nloc = len(terms[li])
        K = np.stack([box_local_apply(oplan, c, e) for e in np.eye(nloc)], axis=1)
        # local mode -> reduced dofs: product terms composed with the reduced map
        R = {}
        for i, t in enumerate(terms[li]):
            for (d, cc) in t:
                lo, hi = plan.red_offsets[d - 1], plan.red_offsets[d]
                for k, rc in zip(plan.red_index[lo:hi], plan.red_coef[lo:hi]):
                    R.setdefault(int(k), {}).setdefault(i, 0.0)
                    R[int(k)][i] += cc * rc
        for k, ent in R.items():
            diag[k] += sum(ci * K[i, j] * cj for i, ci in ent.items() for j, cj in ent.items())
    assert rel_err(gb.reduced_diagonal(plan), diag) <= TOL


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_buffered_tails_match_the_per_thread_walk(cuda, precision):
    """Level-5 L-shape (hanging-node expansions up to 72 terms, buffered): the reduced apply of 32
    right-hand sides (tails summed by one warp each before the cell kernel and spread after it)
    equals the apply of 33 (above the buffer's width: each cell-kernel thread walks its own
    expansions) on the same columns, and the single-column apply equals column 0."""
    import ctypes as C

    import torch

    from grico_b200 import _lib as L
    from grico_b200 import batched as bt
    from grico_b200.problem import torch_stream_handle

    plan = gb.compile(bt.lshape_problem(max_level=5))
    n = plan.n_reduced
    dt, prec = (torch.float64, L.GRICO_PREC_FP64) if precision == "fp64" else (torch.float32, L.GRICO_PREC_FP32)
    rng = np.random.default_rng(3)
    X = torch.tensor(rng.standard_normal((33, n)), dtype=dt, device="cuda")
    Y = {}
    for k in (1, 32, 33):
        y = torch.empty((k, n), dtype=dt, device="cuda")
        # torch's stream as the library reads it (a NULL stream would mean the plan's own stream)
        L.check(L.lib().grico_reduced_apply(plan.handle, C.c_void_p(X.data_ptr()), C.c_void_p(y.data_ptr()), k, prec, 0,
                                            C.c_void_p(torch_stream_handle())), "apply")
        Y[k] = y.double().cpu().numpy()
    tol = 1e-12 if precision == "fp64" else 2e-5
    scale = np.max(np.abs(Y[33]))
    assert np.max(np.abs(Y[32] - Y[33][:32])) <= tol * scale
    assert np.max(np.abs(Y[1][0] - Y[33][0])) <= tol * scale

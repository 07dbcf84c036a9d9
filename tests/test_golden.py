"""Committed golden fixtures (tests/golden, written by tests/golden/make_golden.py): the oracle
against the reference's known-answer values and against its own stored outputs; the GPU path
against the stored outputs at the parity tolerance."""
import json
import os

import numpy as np
import pytest

import grico_oracle as go
from cases import build, rel_err

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(HERE, "kats.json")))
FIX = np.load(os.path.join(HERE, "oracle_cases.npz"))
CASE_NAMES = sorted({k.split("/")[0] for k in FIX.files})
MU, KAPPA = 0.7, 1.3
TOL = 1e-12


def source(x):
    return np.prod(np.sin(np.pi * x), axis=1) + 0.5


def test_oracle_matches_reference_kats():
    assert np.allclose(go.legendre_values(0.5, 2), KATS["legendre_values_0.5_deg2"], atol=TOL)
    assert np.allclose(go.legendre_values_and_derivatives(0.5, 2)[1], KATS["legendre_derivatives_0.5_deg2"], atol=TOL)
    assert np.allclose(go.integrated_legendre_values_and_derivatives(-1.0, 4)[0], KATS["integrated_values_-1_deg4"],
                       atol=TOL)
    assert np.allclose(go.integrated_legendre_values_and_derivatives(1.0, 4)[0], KATS["integrated_values_+1_deg4"],
                       atol=TOL)
    assert np.allclose(go.integrated_legendre_values_and_derivatives(0.0, 1)[1], KATS["integrated_derivatives_0_deg1"],
                       atol=TOL)
    assert np.allclose(go.integrated_legendre_values_and_derivatives(0.0, 2)[1], KATS["integrated_derivatives_0_deg2"],
                       atol=TOL)
    assert go.Space(go.Domain((0.0, 0.0), (1.0, 1.0), (1, 1)), (2, 1), basis="full").ndofs == \
        KATS["single_cell_full_p21_dofs"]
    d = go.Domain((0.0, 0.0), (2.0, 1.0), (2, 1))
    d.grid.refine(2, 2)
    s = go.Space(d, 2)
    assert s.ndofs == KATS["hanging_2d_p2_dofs"]
    t = s.mode_terms(3, (0, 1))
    assert [i for i, _ in t] == KATS["hanging_2d_p2_terms_dofs"]
    assert np.allclose([c for _, c in t], KATS["hanging_2d_p2_terms_coefficients"], atol=TOL)
    d3 = go.Domain((0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (2, 1, 1))
    fc = d3.grid.refine(2, 2)
    d3.grid.refine(fc, 3)
    d3.grid.refine(fc + 1, 3)
    assert go.Space(d3, 2).ndofs == KATS["hanging_3d_p2_dofs"]
    assert go.Space(go.Domain((0.0,), (1.0,), (2,)), 3, basis="full", continuity="dg").ndofs == \
        KATS["dg_1d_p3_two_cells_dofs"]
    plan = go.Plan(go.Space(go.Domain((0.0,), (1.0,), (1,)), 1, continuity="dg"), mu=1.0, kappa=0.0,
                   source=lambda x: 1.0)
    assert np.allclose(plan.apply(np.ones(2)), KATS["mass_1d_p1_dg_apply_ones"], atol=TOL)
    assert np.allclose(plan.rhs_physical(), KATS["mass_1d_p1_dg_rhs_source_one"], atol=TOL)


@pytest.mark.parametrize("name", CASE_NAMES)
def test_oracle_reproduces_its_fixtures(name):
    """The oracle still computes what the fixtures hold (a change to the oracle shows here)."""
    oplan, _ = build(name, mu=MU, kappa=KAPPA, source=source)
    assert rel_err(oplan.apply(FIX[f"{name}/x"]), FIX[f"{name}/apply"]) <= 1e-14
    assert rel_err(oplan.reduced_apply(FIX[f"{name}/xr"]), FIX[f"{name}/reduced_apply"]) <= 1e-14
    assert rel_err(oplan.reduced_rhs(), FIX[f"{name}/reduced_rhs"]) <= 1e-14
    diag = oplan.reduced_diagonal()
    diag = diag if diag is not None else oplan.probe_reduced_diagonal()
    assert rel_err(diag, FIX[f"{name}/reduced_diagonal"]) <= 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASE_NAMES)
def test_gpu_path_matches_golden_fixtures(cuda, name):
    import grico_b200 as gb

    _, prob = build(name, mu=MU, kappa=KAPPA, source=source)
    plan = gb.compile(prob)
    assert rel_err(gb.apply(plan, FIX[f"{name}/x"]), FIX[f"{name}/apply"]) <= TOL
    assert rel_err(gb.reduced_apply(plan, FIX[f"{name}/xr"]), FIX[f"{name}/reduced_apply"]) <= TOL
    assert rel_err(gb.reduced_rhs(plan), FIX[f"{name}/reduced_rhs"]) <= TOL
    assert rel_err(gb.reduced_diagonal(plan), FIX[f"{name}/reduced_diagonal"]) <= TOL

"""SIPG interface items on the host: the product's interface batches (patch points, weights,
penalties, maps) against the oracle's restatement (integration.jl:2262-2307, 2800-2841;
benchmark/sine_poisson_sipg.jl), and properties of the oracle's SIPG operator."""
import numpy as np
import pytest

import grico_b200 as gb
from grico_b200 import _lib as L
from dg_cases import sipg_case

CASES = {
    "2d_p2": dict(dim=2, degree=2, refine=1),
    "2d_p3_hanging": dict(dim=2, degree=3, refine=1, hanging=True),
    "2d_hp_hanging": dict(dim=2, degree=2, refine=1, hanging=True, hp=True),
    "3d_p2_hanging": dict(dim=3, degree=2, refine=0, hanging=True),
}


def _product_items(plan):
    out = {}
    for b in plan.point_batches:
        if b.kind != L.GRICO_ITEM_INTERFACE:
            continue
        for k in range(len(b.cells)):
            lo, hi = b.point_offsets[k], b.point_offsets[k + 1]
            key = (int(b.leaves[k]), int(plan.space.leaves[b.plus_cells[k]]), int(b.face_axis[k]))
            out[key] = dict(w=b.weights[lo:hi], rm=b.ref_points[lo:hi], rp=b.ref_points_plus[lo:hi],
                            sigma=float(b.eta[k]))
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_interface_items_match_oracle(name):
    oplan, _, plan = sipg_case(**CASES[name], device=False)
    prod = _product_items(plan)
    assert len(prod) == len(oplan.interfaces) > 0
    for it in oplan.interfaces:
        key = (it["minus"]["leaf"], it["plus"]["leaf"], it["axis"])
        p = prod[key]
        assert p["sigma"] == pytest.approx(it["sigma"], rel=1e-15)
        # same tensor patch rule; compare as point sets (tangential axis order may differ)
        assert np.isclose(p["w"].sum(), it["w"].sum(), rtol=1e-14)
        assert np.allclose(np.sort(p["w"]), np.sort(it["w"]), rtol=1e-14, atol=0)
        assert np.all(np.abs(p["rm"][:, it["axis"]] - 1.0) == 0) and np.all(np.abs(p["rp"][:, it["axis"]] + 1.0) == 0)


@pytest.mark.parametrize("name", ["2d_p2", "2d_hp_hanging"])
def test_boundary_penalties_match_oracle(name):
    oplan, _, plan = sipg_case(**CASES[name], device=False)
    prod = sorted(float(e) for b in plan.point_batches if b.kind == L.GRICO_ITEM_NITSCHE for e in b.eta)
    orac = sorted(float(c["eta"]) for c in oplan.surfaces)
    assert np.allclose(prod, orac, rtol=1e-15)


@pytest.mark.parametrize("name", ["2d_p2", "2d_hp_hanging"])
def test_oracle_sipg_operator_is_symmetric_positive(name):
    """The SIPG form is symmetric; with penalty 10 it is positive definite on these meshes."""
    oplan, _, _ = sipg_case(**CASES[name], device=False)
    n = oplan.ndofs
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = oplan.apply_physical(e)
    assert np.max(np.abs(A - A.T)) <= 1e-12 * np.max(np.abs(A))
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).min() > 0


def test_interface_form_refused_outside_the_closed_set():
    d = gb.Domain((0.0,), (1.0,), (2,))
    s = gb.HpSpace(d, gb.SpaceOptions(degree=gb.UniformDegree(1), continuity="dg"))
    prob = gb.AffineProblem(gb.ScalarField(s))
    with pytest.raises(gb.GricoError):
        gb.add_interface(prob, gb.Nitsche(1.0))


def _kat_1d_matrix(penalty):
    """Interface matrix of the SIPG form on [0, 1] split at 0.5, DG p = 1 (modes (1-xi)/2,
    (1+xi)/2 per cell), derived by hand from benchmark/sine_poisson_sipg.jl:54-95:
    [u] = m1 - p0, {u'} = (m1 - m0) + (p1 - p0), sigma = penalty (1 + 1)^2 / (2 h h / 2h) = 8 penalty;
    rows/columns (m0, m1, p0, p1)."""
    s = 8.0 * penalty
    return np.array([[0.0, 1.0, -1.0, 0.0],
                     [1.0, s - 2.0, 2.0 - s, -1.0],
                     [-1.0, 2.0 - s, s - 2.0, 1.0],
                     [0.0, -1.0, 1.0, 0.0]])


def test_oracle_sipg_interface_kat_1d():
    import grico_oracle as go

    od = go.Domain((0.0,), (1.0,), (2,))
    osp = go.Space(od, 1, basis="full", continuity="dg")
    oplan = go.Plan(osp, mu=0.0, kappa=0.0, interface_penalty=3.0)
    n = oplan.ndofs
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = oplan.apply_physical(e)
    # local (leaf, mode) -> dof from the space's term maps
    order = [t[0][0] - 1 for li in range(2) for t in osp.leaf_terms[li]]
    assert np.allclose(A[np.ix_(order, order)], _kat_1d_matrix(3.0), atol=1e-13)

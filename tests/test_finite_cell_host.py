"""Finite-cell classification, candidate quadrature, moment fit and surface quadratures on the
host: oracle pinned to the reference's known answers, product checked against the oracle."""
import math

import numpy as np
import pytest

import grico_oracle as go
import grico_b200 as gb
from grico_b200 import regions as rg
from grico_b200.problem import _gauss

import fc_cases


# ---- oracle pins: test/embedded_geometry.jl ------------------------------------------------

def test_oracle_physical_active_leaves_kat():
    """embedded_geometry.jl:20-38: x - 0.5 on (0,1) with two roots keeps leaf 1 only; the shifted
    background has no physical leaf."""
    lev = lambda X: X[:, 0] - 0.5
    od = go.Domain((0.0,), (1.0,), (2,))
    assert go.physical_active_leaves(od, lev) == [1]
    with pytest.raises(ValueError):
        go.physical_active_leaves(go.Domain((2.0,), (1.0,), (2,)), lev)
    pd = gb.PhysicalDomain(gb.Domain((0.0,), (1.0,), (2,)), gb.ImplicitRegion(lev, subdivision_depth=1))
    assert pd.active_leaves().tolist() == [1]
    with pytest.raises(ValueError):
        gb.PhysicalDomain(gb.Domain((2.0,), (1.0,), (2,)), gb.ImplicitRegion(lev, subdivision_depth=1)).active_leaves()


def test_oracle_finite_cell_robustness_kat():
    """embedded_geometry.jl:40-58: outside -> nothing, inside -> tensor rule, sliver keeps a
    positive weight, the half cube has reference volume 4."""
    od = go.Domain((0.0,), (1.0,), (1,))
    assert go.finite_cell_candidates(od, 1, (2,), lambda X: np.ones(len(X)), 2) is None
    assert go.finite_cell_candidates(od, 1, (2,), lambda X: X[:, 0], 2) is None
    pts, w = go.finite_cell_candidates(od, 1, (2,), lambda X: -np.ones(len(X)), 2)
    assert pts.shape == (2, 1) and abs(w.sum() - 2.0) < 1e-15
    pts, w = go.finite_cell_candidates(od, 1, (1,), lambda X: X[:, 0] - 1.0e-6, 0)
    assert len(w) >= 1 and w.sum() > 0.0
    od3 = go.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    pts, w = go.finite_cell_candidates(od3, 1, (2, 2, 2), lambda X: X[:, 0] - 0.5, 1)
    assert abs(w.sum() - 4.0) <= 1e-10


def test_product_finite_cell_quadrature_kat():
    """The same known answers through the product's finite_cell_quadrature (moment fitted)."""
    dom = gb.Domain((0.0,), (1.0,), (1,))
    assert gb.finite_cell_quadrature(dom, 1, (2,), lambda X: np.ones(len(X))) is None
    assert gb.finite_cell_quadrature(dom, 1, (2,), lambda X: X[:, 0]) is None
    pts, w = gb.finite_cell_quadrature(dom, 1, (2,), lambda X: -np.ones(len(X)))
    assert pts.shape == (2, 1)
    pts, w = gb.finite_cell_quadrature(dom, 1, (1,), lambda X: X[:, 0] - 1.0e-6, subdivision_depth=0)
    assert len(w) >= 1 and w.sum() > 0.0
    dom3 = gb.Domain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (1, 1, 1))
    pts, w = gb.finite_cell_quadrature(dom3, 1, (2, 2, 2), lambda X: X[:, 0] - 0.5, subdivision_depth=1)
    assert abs(w.sum() - 4.0) <= 1e-10
    with pytest.raises(ValueError, match="subdivision_depth"):
        gb.ImplicitRegion(lambda X: X[:, 0], subdivision_depth=1.5)
    with pytest.raises(ValueError, match="subdivision_depth"):
        gb.PhysicalDomain(dom, gb.ImplicitRegion(lambda X: X[:, 0], subdivision_depth=21))


def test_bool_classifier_reads_true_as_inside():
    dom = gb.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    pd = gb.PhysicalDomain(dom, gb.ImplicitRegion(lambda X: X[:, 0] < 0.6, subdivision_depth=1))
    od = go.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    cls = pd.classify(dom.grid.active_leaves())
    ocls = [go.classify_leaf(od, l, lambda X: X[:, 0] < 0.6) for l in od.grid.active_leaves()]
    assert [{0: "outside", 1: "inside", 2: "cut"}[int(c)] for c in cls] == ocls


# ---- product vs oracle ----------------------------------------------------------------------

@pytest.mark.parametrize("dim", [2, 3])
def test_candidate_quadrature_matches_oracle_bitwise(dim):
    if dim == 2:
        lev = fc_cases.annulus_levelset(0.35, 1.0)
        origin, extent, roots, refine, depth = (-1.0, -1.0), (2.0, 2.0), (2, 2), 1, 3
    else:
        lev = fc_cases.shell_levelset((1.0, 1.0, 1.0), 0.4, 0.9)
        origin, extent, roots, refine, depth = (0.0,) * 3, (2.0,) * 3, (1, 1, 1), 1, 2
    od = go.Domain(origin, extent, roots)
    go.uniform_refine(od.grid, refine)
    bg = gb.Domain(origin, extent, roots)
    gb.uniform_refine(bg, refine)
    pd = gb.PhysicalDomain(bg, gb.ImplicitRegion(lev, subdivision_depth=depth))
    assert sorted(pd.active_leaves().tolist()) == sorted(go.physical_active_leaves(od, lev))
    leaves = bg.grid.active_leaves()
    cut = leaves[pd.classify(leaves) == 2]
    assert cut.size > 0
    q = (3,) * dim
    off, xi, w = pd.candidate_quadrature(cut, q, _gauss)
    for i, leaf in enumerate(cut):
        pts, wts = go.finite_cell_candidates(od, int(leaf), q, lev, depth)
        assert np.array_equal(pts, xi[off[i]:off[i + 1]])
        assert np.array_equal(wts, w[off[i]:off[i + 1]])


def test_moment_fit_reproduces_moments():
    lev = fc_cases.annulus_levelset(0.35, 1.0)
    bg = gb.Domain((-1.0, -1.0), (2.0, 2.0), (2, 2))
    gb.uniform_refine(bg, 1)
    pd = gb.PhysicalDomain(bg, gb.ImplicitRegion(lev, subdivision_depth=3))
    leaves = bg.grid.active_leaves()
    cut = leaves[pd.classify(leaves) == 2][:4]
    off, xi, w = pd.candidate_quadrature(cut, (3, 3), _gauss)
    for i in range(len(cut)):
        P, W = xi[off[i]:off[i + 1]], w[off[i]:off[i + 1]]
        fp, fw = rg.moment_fit(P, W, (3, 3))
        assert len(fw) <= len(W)
        assert np.all(fw >= 0)
        A = rg.moment_matrix(P, (3, 3))
        Af = rg.moment_matrix(fp, (3, 3))
        m = A @ W
        assert np.linalg.norm(Af @ fw - m) <= 1e-12 * max(np.linalg.norm(m), 1.0)


# ---- surface quadratures ----------------------------------------------------------------------

@pytest.mark.parametrize("refine", [1, 3])
def test_sphere_quadrature_exact_moments(refine):
    c = np.array([1.0, 1.0, 1.0])
    dom = gb.Domain((0.0, 0.0, 0.0), (2.0, 2.0, 2.0), (1, 1, 1))
    gb.uniform_refine(dom, refine)
    sp = gb.HpSpace(dom, gb.SpaceOptions(degree=gb.UniformDegree(3)))
    for R in (0.9, 0.4):
        area = m2 = 0.0
        for sq in gb.sphere_surface_quadrature(sp, c, R):
            w, n = rg.physical_surface_data(dom, sq.leaf, sq)
            h = dom.cell_size(np.array([sq.leaf]))[0]
            X = dom.cell_lower(np.array([sq.leaf]))[0] + 0.5 * h * (sq.points + 1.0)
            assert np.allclose(n, (X - c) / R, atol=1e-12)
            area += w.sum()
            m2 += (w * (X[:, 0] - c[0]) ** 2 * (X[:, 1] - c[1]) ** 2).sum()
        assert abs(area / (4 * math.pi * R * R) - 1) < 1e-11
        assert abs(m2 / (4 * math.pi * R ** 6 / 15) - 1) < 1e-11


def test_circle_quadrature_exact_and_oracle_mapping():
    dom = gb.Domain((-1.0, -1.0), (2.0, 2.0), (2, 2))
    gb.uniform_refine(dom, 2)
    od = go.Domain((-1.0, -1.0), (2.0, 2.0), (2, 2))
    go.uniform_refine(od.grid, 2)
    sp = gb.HpSpace(dom, gb.SpaceOptions(degree=gb.UniformDegree(2)))
    length = 0.0
    for sq in gb.sphere_surface_quadrature(sp, (0.0, 0.0), 0.35, outward=False):
        w, n = rg.physical_surface_data(dom, sq.leaf, sq)
        ow, on = go.physical_surface_data(od, sq.leaf, sq.weights, sq.normals)
        assert np.allclose(w, ow, rtol=1e-14, atol=0) and np.allclose(n, on, rtol=0, atol=1e-15)
        length += w.sum()
    assert abs(length / (2 * math.pi * 0.35) - 1) < 1e-11


# ---- host plan structure -----------------------------------------------------------------------

def test_annulus_plan_structure():
    oplan, prob, plan, _ = fc_cases.annulus(device=False)
    kinds = {b.kind for b in plan.point_batches}
    assert gb._lib.GRICO_ITEM_SUBCELLS in kinds and gb._lib.GRICO_ITEM_NITSCHE in kinds
    n_cut = sum(len(b.cells) for b in plan.point_batches if b.kind == gb._lib.GRICO_ITEM_SUBCELLS)
    assert n_cut == plan.n_cut == len([c for c in oplan.cells if c["q"] is None])
    n_tensor = sum(len(b.cells) for b in plan.batches)
    assert n_tensor + n_cut == len(plan.space.leaves)
    # cut-cell volume plus full cells approximates the annulus area to the octree accuracy
    vol = sum(float(np.sum(w)) for w, _ in gb.problem._quadrature_sets(plan))
    assert abs(vol / (math.pi * (1 - 0.35 ** 2)) - 1) < 2e-2


def test_unsupported_surface_forms():
    oplan, prob, plan, _ = fc_cases.annulus(device=False)
    with pytest.raises(gb.GricoError):
        gb.add_surface_accumulator(prob, prob.field, prob.field, gb.Diffusion())
    u = prob.field
    prob.surface_rhs_operators.append(gb.Nitsche(1.0))
    with pytest.raises(gb.GricoError):
        gb.compile(prob, device=False)


@pytest.mark.parametrize("dim", [2, 3])
def test_subcell_representation_equals_candidate_rule(dim):
    """The subcell records (inside subcells, masked terminal subcells, sliver points) list
    exactly the candidate points and weights of regions.jl:477-510, bit for bit."""
    if dim == 2:
        lev = fc_cases.annulus_levelset(0.35, 1.0)
        origin, extent, roots, refine, depth, q = (-1.0, -1.0), (2.0, 2.0), (2, 2), 1, 3, (3, 3)
    else:
        lev = fc_cases.shell_levelset((1.0, 1.0, 1.0), 0.4, 0.9)
        origin, extent, roots, refine, depth, q = (0.0,) * 3, (2.0,) * 3, (1, 1, 1), 1, 2, (4, 4, 4)
    bg = gb.Domain(origin, extent, roots)
    gb.uniform_refine(bg, refine)
    pd = gb.PhysicalDomain(bg, gb.ImplicitRegion(lev, subdivision_depth=depth))
    leaves = bg.grid.active_leaves()
    cut = leaves[pd.classify(leaves) == 2]
    off, xi, w = pd.candidate_quadrature(cut, q, _gauss)
    soff, slev, spos, smask, sws, slivers = pd.subcell_quadrature(cut, q, _gauss)
    eta, ew = rg._tensor_rule(q, _gauss)
    for i in range(len(cut)):
        pts, wts = [], []
        for s in range(soff[i], soff[i + 1]):
            half = np.ldexp(1.0, -int(slev[s]))
            c = -1.0 + (2.0 * spos[s] + 1.0) * half
            keep = [(int(smask[s]) >> p) & 1 for p in range(len(ew))]
            for p in range(len(ew)):
                if keep[p]:
                    pts.append(c + half * eta[p])
                    wts.append(ew[p] * sws[s])
        if i in slivers:
            pts += list(slivers[i][0])
            wts += list(slivers[i][1])
        P = np.array(pts).reshape(-1, dim)
        Wt = np.array(wts)
        ref_p, ref_w = xi[off[i]:off[i + 1]], w[off[i]:off[i + 1]]
        assert P.shape == ref_p.shape
        o1 = np.lexsort(P.T[::-1])
        o2 = np.lexsort(ref_p.T[::-1])
        assert np.array_equal(P[o1], ref_p[o2])
        assert np.array_equal(Wt[o1], ref_w[o2])

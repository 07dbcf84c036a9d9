"""The oracle against the reference's own known-answer tests (test/core.jl, test/space.jl,
test/matrix_free.jl).  Coefficients use the reference's tolerance SPACE_TOL = 1e-12; dof
indices must match exactly."""
import math

import numpy as np
import pytest

import grico_oracle as go

TOL = 1e-12


def test_polynomial_core():  # test/core.jl:152-156
    assert np.allclose(go.legendre_values(0.5, 2), [1.0, 0.5, -0.125], atol=TOL)
    _, d = go.legendre_values_and_derivatives(0.5, 2)
    assert np.allclose(d, [0.0, 1.0, 1.5], atol=TOL)
    v, _ = go.integrated_legendre_values_and_derivatives(-1.0, 4)
    assert np.allclose(v, [1, 0, 0, 0, 0], atol=TOL)
    v, _ = go.integrated_legendre_values_and_derivatives(1.0, 4)
    assert np.allclose(v, [0, 1, 0, 0, 0], atol=TOL)
    _, d = go.integrated_legendre_values_and_derivatives(0.0, 1)
    assert np.allclose(d, [-0.5, 0.5], atol=TOL)
    _, d = go.integrated_legendre_values_and_derivatives(0.0, 2)
    assert np.allclose(d, [-0.5, 0.5, 0.0], atol=TOL)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 12])
def test_gauss_legendre_exactness(n):  # test/core.jl:271+
    pts, wts = go.gauss_legendre_rule(n)
    assert all(a < b for a, b in zip(pts, pts[1:]))
    for k in range(2 * n):
        exact = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(sum(w * x ** k for x, w in zip(pts, wts)) - exact) < 1e-13


def test_single_cell_space():  # test/space.jl:274-304
    d = go.Domain((0.0, 0.0), (1.0, 1.0), (1, 1))
    s = go.Space(d, (2, 1), basis="full")
    assert s.ndofs == 6
    for k, m in enumerate([(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (2, 1)]):
        assert s.mode_terms(1, m) == [(k + 1, 1.0)]


def _hanging_2d():
    d = go.Domain((0.0, 0.0), (2.0, 1.0), (2, 1))
    d.grid.refine(2, 2)
    return d


def test_hanging_2d_coefficients():  # test/space.jl:306-319
    s = go.Space(_hanging_2d(), 2)
    assert s.ndofs == 16
    for leaf, mode in ((3, (0, 1)), (4, (0, 0))):
        t = s.mode_terms(leaf, mode)
        assert [i for i, _ in t] == [2, 5, 8]
        assert np.allclose([c for _, c in t], [0.5, 0.5, -0.6123724356957945], atol=TOL)


def test_hanging_3d_count():  # test/space.jl:672-700
    d = go.Domain((0.0, 0.0, 0.0), (2.0, 1.0, 1.0), (2, 1, 1))
    g = d.grid
    fc = g.refine(2, 2)
    g.refine(fc, 3)
    g.refine(fc + 1, 3)
    assert go.Space(d, 2).ndofs == 50


def test_dg_space():  # test/space.jl:321-332
    s = go.Space(go.Domain((0.0,), (1.0,), (2,)), 3, basis="full", continuity="dg")
    assert s.ndofs == 8
    assert s.mode_terms(1, (1,)) == [(2, 1.0)]
    assert s.mode_terms(2, (0,)) == [(5, 1.0)]


def _space_value(space, leaf, xi, coeffs):
    li = space.snapshot.leaf_to_index[leaf]
    val = 0.0
    for mode, terms in zip(space.leaf_modes[li], space.leaf_terms[li]):
        phi = 1.0
        for a, x in enumerate(xi):
            v, _ = go.fe_basis_values_and_derivatives(x, space.degrees[li][a])
            phi *= v[mode[a]]
        val += phi * sum(c * coeffs[d - 1] for d, c in terms)
    return val


def test_hanging_trace_continuity_2d():  # test/space.jl:633-660
    d = _hanging_2d()
    s = go.Space(d, 2)
    first_child = 3
    for dof in range(s.ndofs):
        unit = np.zeros(s.ndofs)
        unit[dof] = 1.0
        for y in (-0.75, -0.25, 0.25, 0.75):
            right = (_space_value(s, first_child, (-1.0, 2 * y + 1), unit) if y < 0
                     else _space_value(s, first_child + 1, (-1.0, 2 * y - 1), unit))
            assert abs(_space_value(s, 1, (1.0, y), unit) - right) < TOL


def test_mass_apply_and_rhs_1d():  # test/matrix_free.jl:538-579
    d = go.Domain((0.0,), (1.0,), (1,))
    s = go.Space(d, 1, continuity="dg")
    plan = go.Plan(s, mu=1.0, kappa=0.0, source=lambda x: 1.0)
    assert np.allclose(plan.apply(np.ones(2)), [0.5, 0.5], atol=TOL)
    assert np.allclose(plan.rhs_physical(), [0.5, 0.5], atol=TOL)


def test_poisson_2x2_accuracy():  # test/examples.jl:6-12 (Poisson GMG example, 2x2 p=2, L2 <= 2e-2)
    d = go.Domain((0.0, 0.0), (1.0, 1.0), (2, 2))
    s = go.Space(d, 2, basis="full")
    exact = lambda x: math.sin(math.pi * x[0]) * math.sin(math.pi * x[1])
    plan = go.Plan(s, mu=0.0, kappa=1.0, source=lambda x: 2 * math.pi ** 2 * exact(x),
                   dirichlet=[(a, sd, 0.0) for a in (1, 2) for sd in (1, 2)])
    b = plan.reduced_rhs()
    xr, _ = go.cg_solve(plan.reduced_apply, b, rtol=1e-12)
    err = go.l2_error(plan, plan.expand(xr, include_shift=True), exact)
    assert err <= 2e-2


@pytest.mark.parametrize("counts,p", [((3, 2), 2), ((4, 4), 4), ((2, 3, 2), 2), ((4, 4, 4), 3)])
def test_uniform_numbering_matches_literal_oracle(counts, p):
    """The array-based numbering used by the CPU baseline equals the union-find restatement."""
    import uniform_maps as um

    D = len(counts)
    d = go.Domain((0.0,) * D, (1.0,) * D, counts)
    s = go.Space(d, p, basis="full")
    coords, m, ndofs = um.uniform_space(counts, p)
    assert ndofs == s.ndofs
    for li, leaf in enumerate(s.snapshot.leaves):
        assert [d.grid.coord(leaf, a) for a in range(D)] == list(coords[li])
        got = [int(v) + 1 for v in m[li]]
        want = [t[0][0] for t in s.leaf_terms[li]]
        assert got == want


@pytest.mark.parametrize("counts,p", [((4, 3), 4), ((2, 2, 3), 3), ((3, 3, 3), 4)])
def test_c_tensor_apply_matches_basis_loop(counts, p):
    """The C restatement of the tensor schedule equals the basis-loop oracle (no constraints)."""
    import oracle_lib as ol
    import uniform_maps as um

    D = len(counts)
    d = go.Domain((0.0,) * D, (1.0, 2.0, 0.5)[:D], counts)
    s = go.Space(d, p, basis="full")
    plan = go.Plan(s, mu=0.6, kappa=1.7)
    coords, m, ndofs = um.uniform_space(counts, p)
    c0 = plan.cells[0]
    B = c0["axis_v"][0]
    G = c0["axis_g"][0] / (2.0 / d.cell_size(c0["leaf"], 0))
    pts, W = go.gauss_legendre_rule(p + 1)
    h = np.array([[d.cell_size(leaf, a) for a in range(D)] for leaf in s.snapshot.leaves])
    order, off = um.parity_colours(coords)
    x = np.random.default_rng(0).standard_normal(ndofs)
    y = np.zeros(ndofs)
    ol.tensor_apply(D, p + 1, p + 1, m, h, B, G, np.array(W), 0.6, 1.7, None, order, off, x, y, threads=2)
    ref = plan.apply_physical(x)
    assert np.max(np.abs(y - ref)) <= 1e-12 * np.max(np.abs(ref))

"""The adaptive hp L-shape space (levels 2..4, degrees 2..4, hanging nodes, re-entrant boundary
faces) against the oracle on the CPU.

Bit-exact: Morton order, boundary faces including the faces next to the removed quadrant
(covering-neighbour rule, topology.jl:1509-1521, 1596-1608) and interfaces.  The continuity
compile meets noise pivots on this mesh (redundant rows cancelling to ~1e-15 that the reference
pivots on), so the product keeps one dof per noise pivot and the dof maps are compared as
function spaces: the product's Dirichlet-constrained space contains the oracle's, and its
functions vanish on every Dirichlet face (plans.jl:486-972, relation rows where hanging-node
traces couple several dofs)."""
import numpy as np
import pytest

import grico_oracle as go
import grico_b200 as gb
from lshape_cases import expand, setup, to_product


@pytest.fixture(scope="module")
def pair():
    return setup(device=False)


def test_lshape_topology_matches_oracle(pair):
    oplan, plan, _ = pair
    osp, psp = oplan.space, plan.space
    assert list(osp.snapshot.leaves) == [int(v) for v in psp.leaves]
    b_leaf, b_axis, b_side = psp.boundary_faces
    got = [(int(psp.leaves[l]), int(a) + 1, int(s) + 1) for l, a, s in zip(b_leaf, b_axis, b_side)]
    assert got == osp.snapshot.boundary
    od = osp.domain
    reentrant = [l for l, a, s in osp.snapshot.boundary
                 if a == 1 and s == 2 and od.cell_lower(l, 0) + od.cell_size(l, 0) == 0.0 and od.cell_lower(l, 1) >= 0.0]
    assert reentrant
    i_m, i_p, i_a = psp.interfaces
    got = [(int(psp.leaves[m]), int(q), int(a) + 1) for m, q, a in zip(i_m, psp.leaves[i_p], i_a)]
    assert got == osp.snapshot.interfaces


def test_lshape_dof_count_and_noise_pivots(pair):
    oplan, plan, _ = pair
    osp = oplan.space
    assert osp.min_pivot < 1e-10
    assert plan.n_full == osp.ndofs + osp.noise_pivots


def test_lshape_dirichlet_space_contains_oracle_space(pair):
    oplan, plan, terms = pair
    u = np.random.default_rng(0).standard_normal(len(oplan.solve_dofs))
    xr = to_product(oplan, plan, terms, u)  # checks that the product reproduces the function
    x = expand(plan, xr)
    assert np.max(np.abs(x[plan.fixed_dofs])) <= 1e-10
    assert len(plan.relations) > 0
    for (p, idx, co, rhs_p) in plan.relations:
        assert abs(x[p] - co @ x[idx] - rhs_p) <= 1e-10
    assert plan.n_reduced >= len(oplan.solve_dofs)


def test_lshape_product_functions_vanish_on_dirichlet_faces(pair):
    oplan, plan, terms = pair
    osp = oplan.space
    xr = np.random.default_rng(1).standard_normal(plan.n_reduced)
    xf = np.zeros(plan.n_full + 1)
    for d in range(plan.n_full):
        lo, hi = plan.red_offsets[d], plan.red_offsets[d + 1]
        xf[d + 1] = plan.shift[d] + plan.red_coef[lo:hi] @ xr[plan.red_index[lo:hi]]
    pts, _ = go.gauss_legendre_rule(5)
    worst = 0.0
    for (leaf, axis, side) in osp.snapshot.boundary:
        li = osp.snapshot.leaf_to_index[leaf]
        c = oplan.cells[li]
        m = np.array([sum(cc * xf[d] for (d, cc) in t) for t in terms[li]])
        n = [dg + 1 for dg in c["degs"]]
        modes = [(i, j, k) for k in range(n[2]) for j in range(n[1]) for i in range(n[0])]
        a = axis - 1
        tang = [b for b in range(3) if b != a]
        for p1 in pts:
            for p2 in pts:
                ref = [0.0, 0.0, 0.0]
                ref[a] = -1.0 if side == 1 else 1.0
                ref[tang[0]], ref[tang[1]] = p1, p2
                tab = [go.fe_basis_values_and_derivatives(ref[b], c["degs"][b])[0] for b in range(3)]
                v = sum(m[k] * tab[0][md[0]] * tab[1][md[1]] * tab[2][md[2]] for k, md in enumerate(modes))
                worst = max(worst, abs(v))
    assert worst <= 1e-9

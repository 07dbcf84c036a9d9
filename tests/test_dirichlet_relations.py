"""Dirichlet relation rows from multi-term trace rows (plans.jl:884-972 restated on the trace
rows): every vector built from the relations satisfies the rows, the count of constrained dofs
is the rank, and rows that cancelled to rounding level pose no constraint."""
import numpy as np

from grico_b200.problem import _dirichlet_components


def _rows(A, base=100):
    ent, dof, coef = [], [], []
    for i in range(A.shape[0]):
        for j in range(A.shape[1]):
            if A[i, j] != 0.0:
                ent.append(i)
                dof.append(base + j)
                coef.append(A[i, j])
    return np.array(ent), np.array(dof), np.array(coef)


def _complete(A, fixed, values, rel, rng, base=100):
    x = np.zeros(base + A.shape[1])
    constrained = set(fixed.tolist()) | {r[0] for r in rel}
    free = [base + j for j in range(A.shape[1]) if base + j not in constrained]
    x[free] = rng.standard_normal(len(free))
    x[fixed] = values
    for p, idx, c, rhs in rel:
        x[p] = rhs + c @ x[idx]
    return x[base:]


def test_relations_satisfy_the_trace_rows():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((6, 10)) * np.array([1e5, 1, 1e-3, 1, 300, 1])[:, None]
    A[4] = A[0] / 1e5 + 2 * A[1]          # dependent row
    b = np.zeros(6)
    fixed, values, rel = _dirichlet_components(*_rows(A), b)
    assert len(fixed) + len(rel) == np.linalg.matrix_rank(A) == 5
    x = _complete(A, fixed, values, rel, rng)
    assert np.max(np.abs(A @ x)) <= 1e-10 * np.max(np.abs(A))


def test_rounding_residue_rows_are_no_constraint():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((3, 6))
    noise = np.zeros((1, 6))
    noise[0, 2:5] = [1.7e-15, -4.0e-16, 9.0e-16]  # a row whose terms cancelled to rounding level
    A = np.vstack([A, noise])
    fixed, values, rel = _dirichlet_components(*_rows(A), np.zeros(4))
    assert len(fixed) + len(rel) == 3

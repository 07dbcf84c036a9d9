"""Writes the golden fixtures of this folder (python tests/golden/make_golden.py).

kats.json: the reference's own known-answer values, copied from its test suite
(test/core.jl:152-156, test/space.jl:274-332 and 672-700, test/matrix_free.jl:538-579).
oracle_cases.npz: for small seeded problems of tests/cases.py, the seeded inputs and the oracle's
outputs (full apply, reduced apply, reduced right-hand side, reduced diagonal).  The oracle is
pinned to kats.json by tests/test_golden.py and tests/test_oracle_kat.py; the GPU path is checked
against oracle_cases.npz at the parity tolerance 1e-12 relative."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ("tests", "grico.jl_b200", "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

KATS = {
    "legendre_values_0.5_deg2": [1.0, 0.5, -0.125],
    "legendre_derivatives_0.5_deg2": [0.0, 1.0, 1.5],
    "integrated_values_-1_deg4": [1.0, 0.0, 0.0, 0.0, 0.0],
    "integrated_values_+1_deg4": [0.0, 1.0, 0.0, 0.0, 0.0],
    "integrated_derivatives_0_deg1": [-0.5, 0.5],
    "integrated_derivatives_0_deg2": [-0.5, 0.5, 0.0],
    "single_cell_full_p21_dofs": 6,
    "hanging_2d_p2_dofs": 16,
    "hanging_2d_p2_terms_dofs": [2, 5, 8],
    "hanging_2d_p2_terms_coefficients": [0.5, 0.5, -0.6123724356957945],
    "hanging_3d_p2_dofs": 50,
    "dg_1d_p3_two_cells_dofs": 8,
    "mass_1d_p1_dg_apply_ones": [0.5, 0.5],
    "mass_1d_p1_dg_rhs_source_one": [0.5, 0.5],
}

CASE_NAMES = ["1d_p3", "2d_p4", "2d_p2_hanging", "2d_p3_over", "3d_p2_hanging", "3d_p3_trunk", "3d_p1"]
MU, KAPPA = 0.7, 1.3


def source(x):
    return np.prod(np.sin(np.pi * x), axis=1) + 0.5


def main():
    from cases import build, sample_vector

    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(KATS, f, indent=1)
    arrays = {}
    for name in CASE_NAMES:
        oplan, _ = build(name, mu=MU, kappa=KAPPA, source=source)
        n_full, n_red = oplan.space.ndofs, len(oplan.solve_dofs)
        x = sample_vector(n_full, seed=11)
        xr = sample_vector(n_red, seed=12)
        arrays[f"{name}/x"] = x
        arrays[f"{name}/apply"] = oplan.apply(x)
        arrays[f"{name}/xr"] = xr
        arrays[f"{name}/reduced_apply"] = oplan.reduced_apply(xr)
        arrays[f"{name}/reduced_rhs"] = oplan.reduced_rhs()
        diag = oplan.reduced_diagonal()
        # multi-term (hanging) maps: the reference probes with unit vectors (solve.jl:722-738)
        arrays[f"{name}/reduced_diagonal"] = diag if diag is not None else oplan.probe_reduced_diagonal()
    np.savez_compressed(os.path.join(HERE, "oracle_cases.npz"), **arrays)


if __name__ == "__main__":
    main()

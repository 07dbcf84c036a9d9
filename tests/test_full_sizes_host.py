"""The 64^3, p = 4 workload's dof maps and Dirichlet set at full size (16,974,593 dofs) are
bit-identical to the oracle's uniform numbering (oracle/uniform_maps.py, itself pinned to the
literal restatement of continuity.jl in test_oracle_kat.py)."""
import numpy as np

import grico_b200 as gb
from full_size_cases import poisson3d_64, uniform_oracle


def test_poisson64_maps_and_fixed_set_bit_exact():
    plan = gb.compile(poisson3d_64(), device=False)
    coords, m, ndofs, fixed = uniform_oracle((64, 64, 64), 4)
    assert plan.n_full == ndofs == 257 ** 3
    assert len(plan.batches) == 1
    b = plan.batches[0]
    assert b.tail_offsets is None and b.map_coef is None
    assert np.array_equal(b.map_index.reshape(len(coords), -1), m.astype(np.int32))
    assert np.array_equal(plan.fixed_dofs, fixed)
    assert not plan.relations
    assert plan.n_reduced == 255 ** 3

"""o2f_residual_norm_noalloc (scratch in a static device array, no device
allocation on the call, for hosts that may not allocate during a call)
against the existing entry point o2f_residual.

The file name sorts last, so in a full run the no-alloc call comes after
every other GPU test; it also passes alone."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, developed_state, small_mesh

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # the two reductions sum the same squares in different orders


@pytest.mark.parametrize("n_surface,n_layers", [(48, 12), (200, 60)])
def test_residual_norm_noalloc_matches_o2f_residual(n_surface, n_layers):
    from optimisation2forme_b200 import SimulationParams, Solver
    m = small_mesh(triangles=True, n_surface=n_surface, n_layers=n_layers, seed=3)
    p = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, limiter_k=5.0, final_time=1.0, cfl_number=0.5,
                         verbosity=0)
    with Solver(p, desc=desc_of(m)) as s:
        U = developed_state(s, 60)
        s.set_state(U)
        R = s.compute_residual()
        ref = float(np.sqrt(np.sum(R.reshape(-1, 4)[:, 0] ** 2)))
        assert ref > 0.0
        first = s.residual_norm_noalloc()
        second = s.residual_norm_noalloc()  # the completion ticket was reset by the first call
        for got in (first, second):
            assert abs(got - ref) <= REL_TOL * ref
        assert first == second
        # the interface states it leaves are the ones o2f_residual leaves
        np.testing.assert_array_equal(s.compute_residual(), R)

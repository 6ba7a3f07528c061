"""o2f_residual_norm_noalloc (scratch in a static device array, no device
allocation on the call, for hosts that may not allocate during a call)
against the existing entry point o2f_residual.

The file name sorts last, so in a full run the no-alloc call comes after
every other GPU test; it also passes alone."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import desc_of, developed_state, small_mesh

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # the two reductions sum the same squares in different orders


def _free_bytes() -> int:
    import torch
    torch.cuda.synchronize()
    return int(torch.cuda.mem_get_info()[0])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n_surface,n_layers", [(48, 12), (200, 60)])
def test_residual_norm_noalloc_matches_o2f_residual(n_surface, n_layers, precision):
    from optimisation2forme_b200 import SimulationParams, Solver
    m = small_mesh(triangles=True, n_surface=n_surface, n_layers=n_layers, seed=3)
    p = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, limiter_k=5.0, final_time=1.0, cfl_number=0.5,
                         verbosity=0)
    with Solver(p, desc=desc_of(m)) as s:
        U = developed_state(s, 60)
        s.set_params(dataclasses.replace(p, precision=precision))
        s.set_state(U)
        R = s.compute_residual()  # an FP32 context allocates its FP32 buffers here
        ref = float(np.sqrt(np.sum(R.reshape(-1, 4)[:, 0] ** 2)))
        assert ref > 0.0
        first = s.residual_norm_noalloc()  # may look up the scratch address (set-up)
        free0 = _free_bytes()
        launches0 = s.timing()["kernel_launches"]
        second = s.residual_norm_noalloc()  # the completion ticket was reset by the first call
        free1 = _free_bytes()
        for got in (first, second):
            assert abs(got - ref) <= REL_TOL * ref
        assert first == second
        # no device memory taken by the call, and only the residual + norm kernels launched
        assert free1 == free0
        assert s.timing()["kernel_launches"] - launches0 == 6
        # the interface states it leaves are the ones o2f_residual leaves
        np.testing.assert_array_equal(s.compute_residual(), R)


def test_residual_norm_noalloc_fp32_context_needs_its_buffers():
    from optimisation2forme_b200 import O2FError, SimulationParams, Solver
    m = small_mesh(triangles=True, n_surface=48, n_layers=12, seed=3)
    p = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, limiter_k=5.0, final_time=1.0, cfl_number=0.5,
                         verbosity=0, precision="fp32")
    with Solver(p, desc=desc_of(m)) as s:
        s.initialize_freestream()
        with pytest.raises(O2FError, match="STATE"):
            s.residual_norm_noalloc()
        R = s.compute_residual()
        got = s.residual_norm_noalloc()
        ref = float(np.sqrt(np.sum(R.reshape(-1, 4)[:, 0] ** 2)))
        assert got == ref or abs(got - ref) <= REL_TOL * ref

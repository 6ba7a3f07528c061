"""Failure detection on the GPU without a GPU fault: every error is a status
returned to the host, caused by host-made inputs (a NaN state, an iteration
cap, a call out of order).  No kernel traps or hangs: the device-driven loops
carry step / iteration caps and stop flags that the host reads."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, max_rel, perturbed_freestream, small_mesh
from oracle import cpu

pytestmark = pytest.mark.gpu


def _solver():
    from optimisation2forme_b200 import SimulationParams, Solver
    m = small_mesh(triangles=True, n_surface=48, n_layers=12, seed=0)
    p = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, limiter_k=5.0, final_time=1.0, cfl_number=0.5,
                         verbosity=0)
    return Solver(p, desc=desc_of(m)), p


def test_nonfinite_state_stops_the_time_loop_with_a_status():
    from optimisation2forme_b200 import O2FError
    s, p = _solver()
    with s:
        U = perturbed_freestream(s.n_cells, p, seed=1, amp=1e-3)
        U[4 * 7] = np.nan
        s.set_state(U)
        with pytest.raises(O2FError) as e:
            s.time_loop(50)
        assert e.value.status == "O2F_ERR_NONFINITE"
        # the context stays usable
        s.initialize_freestream()
        assert s.time_loop(3)["steps"] == 3


def test_negative_density_follows_the_reference():
    """A cell with negative density makes that cell's wave speed NaN; the
    reference's std::max skips it (src/simulation.cpp:96), so the loop goes
    on while the residual stays finite and stops with a status (never a
    trap) once it does not -- exactly where the oracle's state turns
    non-finite."""
    from optimisation2forme_b200 import HostMesh
    s, p = _solver()
    with s:
        U = perturbed_freestream(s.n_cells, p, seed=1, amp=1e-3)
        U[4 * 3] = -1.0
        s.set_state(U)
        U0 = s.get_state()
        o = cpu.Oracle(HostMesh(desc=desc_of(small_mesh(triangles=True, n_surface=48, n_layers=12, seed=0))), p)
        for n in (1, 20):
            s.set_state(U0)
            r = s.time_loop(n, raise_on_failure=False)
            ro = o.march(U0, n)
            if np.all(np.isfinite(ro["U"])):
                assert r["status"] == "OK" and r["steps"] == n
                assert max_rel(s.get_state(), ro["U"]) <= 1e-8
            else:
                assert r["status"] == "O2F_ERR_NONFINITE"


def test_adjoint_iteration_cap_returns_not_converged():
    s, p = _solver()
    with s:
        s.initialize_freestream()
        s.time_loop(50)
        s.compute_residual()
        res = s.solve_adjoint_system(beta=0.1, tol=1e-15, max_iter=3, restart=2, raise_on_failure=False)
        assert res["status"] == "O2F_ERR_NOT_CONVERGED"
        assert res["iters"] == 3
        assert np.isfinite(res["relres"])


def test_call_order_is_checked():
    from optimisation2forme_b200 import O2FError
    s, p = _solver()
    with s:
        with pytest.raises(O2FError) as e:
            s.lift_drag()
        assert e.value.status == "O2F_ERR_STATE"
        with pytest.raises(O2FError) as e:
            s.solve_adjoint_system()
        assert e.value.status == "O2F_ERR_STATE"
        with pytest.raises(ValueError):
            s.set_state(np.zeros(5))


def test_ilu_sweep_wait_that_runs_out_returns_a_status():
    """The ILU(0) sweeps wait, bounded, on the ready flags of the rows they
    depend on.  A row made never to signal (test hook) lets its dependants'
    waits run out: the solve returns O2F_ERR_CUDA instead of hanging, and
    after the hook is cleared the same context solves to the same lambda as
    before."""
    from optimisation2forme_b200 import O2FError
    s, p = _solver()
    with s:
        s.initialize_freestream()
        s.time_loop(50)
        s.compute_residual()
        ref = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=2000, restart=500)
        s.debug_ilu_stall(True, spin_limit=1 << 12)
        with pytest.raises(O2FError) as e:
            s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=20, restart=10)
        assert e.value.status == "O2F_ERR_CUDA"
        assert "dependency wait" in str(e.value)
        s.debug_ilu_stall(False)
        again = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=2000, restart=500)
        assert again["iters"] == ref["iters"]
        np.testing.assert_array_equal(again["lambda"], ref["lambda"])


def test_block_sweeps_and_waiting_sweeps_give_the_same_solution():
    """The two ways of sweeping the ILU triangles -- one thread block walking
    the dependency levels, or persistent warps waiting on their rows'
    dependencies -- compute every row with the same arithmetic: the adjoint
    solves agree bit for bit, and switching back and forth on one context
    keeps them so."""
    s, p = _solver()
    with s:
        s.initialize_freestream()
        s.time_loop(50)
        s.compute_residual()
        a = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=2000, restart=500)
        s.debug_ilu_stall(False, spin_limit=1 << 22)  # the waiting sweeps
        b = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=2000, restart=500)
        s.debug_ilu_stall(False)
        c = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=2000, restart=500)
        assert a["iters"] == b["iters"] == c["iters"]
        np.testing.assert_array_equal(a["lambda"], b["lambda"])
        np.testing.assert_array_equal(a["lambda"], c["lambda"])

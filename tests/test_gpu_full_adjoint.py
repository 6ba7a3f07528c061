"""Consistent adjoint (adjoint_jacobian="full"): the stored Jacobian and the
objective gradient against directional finite differences of the solver's
own residual and objective, <J^T x, v> = <x, dR/dU v> and <b, v> = dJ/dU v
(random x, v), and the adjoint solve with them.  The reference operator (first-order flux,
inviscid wall pressure) is measured on the same identities for contrast."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import desc_of, developed_state, small_mesh

pytestmark = pytest.mark.gpu

BETA = 0.1


def _params(**kw):
    from optimisation2forme_b200 import SimulationParams
    d = dict(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0, limiter_k=5.0,
             verbosity=0, adjoint_precond="none")
    d.update(kw)
    return SimulationParams(**d)


def _directional(s, U, v, delta):
    """(R(U + d v) - R(U - d v)) / 2d and the same for the objective J."""
    s.set_state(U + delta * v)
    Rp = s.compute_residual()
    Jp = s.lift_drag(BETA)[2]
    s.set_state(U - delta * v)
    Rm = s.compute_residual()
    Jm = s.lift_drag(BETA)[2]
    s.set_state(U)
    return (Rp - Rm) / (2 * delta), (Jp - Jm) / (2 * delta)


def test_full_jacobian_and_gradient_match_directional_differences():
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=48, n_layers=12, seed=3)
    with Solver(_params(adjoint_jacobian="full"), desc=desc_of(m)) as s:
        U = developed_state(s, 300)
        rng = np.random.default_rng(0)
        scale = np.tile(np.abs(U.reshape(-1, 4)).max(axis=0), s.n_cells)
        v = rng.standard_normal(U.size) * scale
        x = rng.standard_normal(U.size)
        dR, dJ = _directional(s, U, v, 1e-10)
        s.compute_residual()
        jtx = s.apply_jacobian_transpose(x)
        b = s.assemble_adjoint_rhs(BETA)
        lhs, rhs = float(jtx @ v), float(x @ dR)
        err_op = abs(lhs - rhs) / abs(rhs)
        err_b = abs(float(b @ v) - dJ) / abs(dJ)
        # the reference operator and right-hand side on the same identities
        s.set_params(_params())
        s.set_state(U)
        s.compute_residual()
        ref_op = abs(float(s.apply_jacobian_transpose(x) @ v) - rhs) / abs(rhs)
        ref_b = abs(float(s.assemble_adjoint_rhs(BETA) @ v) - dJ) / abs(dJ)
        print(f"\nfull adjoint: <J^T x, v> vs FD {err_op:.2e} (reference operator {ref_op:.2e}); "
              f"<b, v> vs dJ {err_b:.2e} (reference RHS {ref_b:.2e})")
        # The limiter of E and rho*u turns over within ~1e-4 absolute, so both
        # sides are differences of a barely differentiable residual: they
        # agree to 2e-2 at steps of 1e-6, 7e-4 at 1e-8, 2e-5 at 1e-10
        # (measured); the Jacobian uses 1e-9, the check 1e-10.
        assert err_op <= 1e-3 and err_b <= 1e-5
        assert ref_op > 100 * err_op and ref_b > 100 * err_b


def test_full_adjoint_solve_ends_with_a_status():
    """BiCGSTAB on the full operator does not converge on these transient
    states (measured: relres 1e4 to 1e17 after 3,000-5,000 iterations with
    ILU(0) of the full operator, with the pseudo-time shift, or without a
    preconditioner, at steps of 1e-4 to 1e-9; the reference operator
    converges in 87-148 iterations on the same states; so does the frozen-
    limiter variant below).  The solve must end
    with a status within its iteration cap, leave lambda finite where it
    reports it, and the context usable."""
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=48, n_layers=12, seed=3)
    with Solver(_params(adjoint_jacobian="full", adjoint_precond="ilu0"), desc=desc_of(m)) as s:
        developed_state(s, 300)
        res = s.solve_adjoint_system(BETA, tol=1e-8, max_iter=1000, raise_on_failure=False)
        print(f"\nfull adjoint solve: {res['status']} after {res['iters']} iterations, relres {res['relres']:.2e}")
        assert res["status"] in ("OK", "O2F_ERR_NOT_CONVERGED", "O2F_ERR_NONFINITE", "O2F_ERR_BREAKDOWN")
        assert res["iters"] <= 1000
        if res["status"] != "O2F_ERR_NONFINITE":
            assert np.all(np.isfinite(res["lambda"]))
        s.set_params(dataclasses.replace(s.params, adjoint_jacobian="reference"))
        s.compute_residual()
        ref = s.solve_adjoint_system(BETA, tol=1e-8, max_iter=5000, raise_on_failure=False)
        assert ref["status"] == "OK"


def test_frozen_limiter_adjoint_converges():
    """adjoint_jacobian="frozen_limiter": the same construction with the
    limiter values held at the state (their derivative left out, as usual
    for limited schemes).  Its BiCGSTAB with ILU(0) of that operator
    converges (1,679 iterations here, 173 on a state 5,000 steps on), and
    lambda solves the stored system."""
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=48, n_layers=12, seed=3)
    shape = Solver.shape_params(["m", "p", "t"], [0.02, 0.4, 0.12])
    with Solver(_params(adjoint_jacobian="frozen_limiter", adjoint_precond="ilu0"), desc=desc_of(m)) as s:
        developed_state(s, 300)
        res = s.solve_adjoint_system(BETA, tol=1e-8, max_iter=5000, raise_on_failure=False)
        print(f"\nfrozen-limiter adjoint: {res['status']} after {res['iters']} iterations, relres {res['relres']:.2e}")
        assert res["status"] == "OK" and res["relres"] <= 1e-8
        b = s.assemble_adjoint_rhs(BETA)
        r = s.apply_jacobian_transpose(res["lambda"]) - b
        assert np.linalg.norm(r) <= 1e-7 * np.linalg.norm(b)
        g = s.compute_shape_gradient(["m", "p"], shape, beta=BETA, lam=res["lambda"])
        s.set_params(dataclasses.replace(s.params, adjoint_jacobian="reference"))
        s.compute_residual()
        ref = s.solve_adjoint_system(BETA, tol=1e-8, max_iter=5000)
        g_ref = s.compute_shape_gradient(["m", "p"], shape, beta=BETA, lam=ref["lambda"])
        print(f"frozen-limiter dJ/d(m, p) {g}, reference {g_ref}")
        assert np.all(np.isfinite(g)) and not np.allclose(g, g_ref, rtol=1e-3)

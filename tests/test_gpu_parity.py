"""CUDA path against the oracle and the reference's golden outputs.

Bit-exact (SHA-256 of float64 bytes / array_equal of the bits) wherever the
operation order is the reference's: residual and its stages, J^T x, adjoint
right-hand side, perturbed geometry.  Tolerances where the GPU legitimately
reduces in another order or uses CUDA's libm:
  * forces C_L, C_D, J: parallel reduction                   rel 1e-12
  * time loop (dt via CUDA hypot):                           rel 1e-10
  * adjoint lambda vs a direct sparse solve (tol 1e-10):     rel 1e-6
  * shape gradient (CUDA acos/tan weights of the perturbed
    meshes, reduction of lambda . dR):                       rel 1e-6 (bar: 1e-4)
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import (GOLDEN, assemble_jt, bits_equal, desc_of, developed_state, max_rel, perturbed_freestream, sha,
                      small_mesh)
from oracle import cpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fixture_solver(fixture_params, fixture_state):
    from optimisation2forme_b200 import Solver
    s = Solver(fixture_params, fixture_params.mesh_name)
    s.set_state(fixture_state)
    yield s
    s.close()


def test_residual_is_bit_exact_on_the_reference_fixture(fixture_solver, golden):
    R = fixture_solver.compute_residual()
    assert sha(R) == golden["residual"]["R"]["sha256"]
    for k in ("grad", "edge_LR", "edge_tau"):
        assert sha(fixture_solver.debug(k)) == golden["residual"][k]["sha256"], k


def test_forces_on_the_reference_fixture(fixture_solver, golden):
    fixture_solver.compute_residual()
    cl, cd, J = fixture_solver.lift_drag(50.0)
    assert max_rel([cl, cd, J], golden["forces"][:3]) < 1e-12


def test_jt_and_rhs_are_bit_exact_on_the_reference_fixture(fixture_solver, golden):
    fixture_solver.compute_residual()
    nc = fixture_solver.n_cells
    x = np.random.default_rng(0).standard_normal(4 * nc)
    assert sha(fixture_solver.apply_jacobian_transpose(x)) == golden["jt"]["sha256"]
    assert sha(fixture_solver.assemble_adjoint_rhs(50.0)) == golden["rhs"]["sha256"]


def test_shape_gradient_on_the_reference_fixture(fixture_solver, fixture_state, golden):
    from optimisation2forme_b200 import Solver, load_params_generic
    names, vals, opt = load_params_generic(GOLDEN / "naca_2D_shape_params_0.txt")
    lam = 1e-3 * np.random.default_rng(1).standard_normal(4 * fixture_solver.n_cells)
    fixture_solver.set_state(fixture_state)
    g = fixture_solver.compute_shape_gradient(opt, Solver.shape_params(names, vals), beta=50.0, lam=lam)
    ref = np.array(golden["shape_grad"])
    assert np.all(np.abs(g - ref) <= 1e-6 * np.abs(ref).max())


def test_perturbed_geometry_matches_oracle(fixture_solver, fixture_params, fixture_mesh):
    from optimisation2forme_b200 import Solver, load_params_generic
    names, vals, _ = load_params_generic(GOLDEN / "naca_2D_shape_params_0.txt")
    sh = Solver.shape_params(names, vals)
    o = cpu.Oracle(fixture_mesh, fixture_params)
    for name, pid in (("m", 0), ("p", 1), ("t", 2)):
        ref = o.perturbed(sh, pid, 1e-6)
        for k in ("vert_xy", "cell_vol", "cell_ctr", "edge_len", "edge_n", "edge_ctr"):
            assert bits_equal(fixture_solver.perturbed_geometry(sh, name, 1e-6, k), ref[k]), (name, k)


@pytest.mark.parametrize("triangles,aoa,limiter", [(False, 0.0, "venkatakrishnan"), (True, 2.0, "venkatakrishnan"),
                                                   (True, 1.25, "barth_jespersen")])
def test_residual_jt_rhs_bit_exact_vs_oracle_on_generated_meshes(triangles, aoa, limiter):
    from optimisation2forme_b200 import HostMesh, SimulationParams, Solver
    m = small_mesh(triangles=triangles, n_surface=96, n_layers=24, seed=7)
    p = SimulationParams(viscosity=0.05, inflow_velocity=0.6, aoa_deg=aoa, limiter=limiter, limiter_k=5.0,
                         verbosity=0)
    o = cpu.Oracle(HostMesh(desc=desc_of(m)), p)
    with Solver(p, desc=desc_of(m)) as s:
        U = perturbed_freestream(s.n_cells, p, seed=3)
        s.set_state(U)
        R = s.compute_residual()
        r = o.residual(U)
        assert bits_equal(R, r["R"])
        assert bits_equal(s.debug("edge_LR"), r["edge_LR"])
        assert bits_equal(s.debug("vertex_U"), r["vertex_U"])
        x = np.random.default_rng(4).standard_normal(4 * s.n_cells)
        assert bits_equal(s.apply_jacobian_transpose(x), o.jt(r["edge_LR"], x))
        assert bits_equal(s.assemble_adjoint_rhs(0.1), o.rhs(r["edge_LR"], 0.1))
        f = s.lift_drag(0.1)
        assert max_rel(f, o.forces(r["edge_LR"], r["edge_tau"], 0.1)) < 1e-12


def _stable(**kw):
    """Reference physics at the reference's own viscosity: stable with the
    reference's explicit time step on these meshes."""
    from optimisation2forme_b200 import SimulationParams
    d = dict(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0, limiter_k=5.0,
             verbosity=0)
    d.update(kw)
    return SimulationParams(**d)


def test_time_loop_matches_oracle():
    from optimisation2forme_b200 import HostMesh, Solver
    m = small_mesh(triangles=True, n_surface=96, n_layers=24, seed=2)
    p = _stable()
    o = cpu.Oracle(HostMesh(desc=desc_of(m)), p)
    with Solver(p, desc=desc_of(m)) as s:
        s.initialize_freestream()
        U0 = s.get_state()
        res = s.time_loop(40)
        ref = o.march(U0, 40)
        assert res["steps"] == ref["steps"] == 40
        assert np.isfinite(ref["U"]).all()
        assert max_rel(s.get_state(), ref["U"]) < 1e-10
        assert max_rel(res["history"], ref["history"]) < 1e-10
        assert abs(res["t"] - ref["t"]) <= 1e-10 * ref["t"]


def test_time_loop_stops_at_final_time_and_on_residual_drop():
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=2)
    p = _stable(final_time=2e-5)
    with Solver(p, desc=desc_of(m)) as s:
        res = s.time_loop(100000)
        assert 0 < res["steps"] < 100000
        assert res["t"] >= 2e-5
        assert res["t"] - 2e-5 < 2e-5 / res["steps"] * 2
        s.set_params(dataclasses.replace(p, final_time=1e9))
        s.initialize_freestream()
        res2 = s.time_loop(20000, residual_drop=0.5)
        h = res2["history"]
        assert res2["steps"] < 20000
        assert h[-1] <= 0.5 * h[0]
        assert np.all(h[:-1] > 0.5 * h[0])


@pytest.mark.parametrize("triangles", [False, True])
def test_adjoint_solve_matches_direct_solve_of_the_oracle_operator(triangles):
    import scipy.sparse.linalg as sla
    from optimisation2forme_b200 import HostMesh, Solver
    m = small_mesh(triangles=triangles, n_surface=64, n_layers=16, seed=4)
    p = _stable()
    hm = HostMesh(desc=desc_of(m))
    o = cpu.Oracle(hm, p)
    with Solver(p, desc=desc_of(m)) as s:
        U = developed_state(s, 300)
        s.compute_residual()
        res = s.solve_adjoint_system(beta=0.1, tol=1e-10, max_iter=5000)
        assert res["relres"] <= 1e-10
        r = o.residual(U)
        b = o.rhs(r["edge_LR"], 0.1)
        true_rel = np.linalg.norm(b - o.jt(r["edge_LR"], res["lambda"])) / np.linalg.norm(b)
        assert true_rel <= 2e-10
        lam = sla.spsolve(assemble_jt(o, hm, r["edge_LR"]).tocsc(), b)
        assert max_rel(res["lambda"], lam) < 1e-6


def test_reference_krylov_path_gives_the_same_adjoint():
    """Identity preconditioner (the reference's solver) and block ILU(0)
    converge to the same lambda; the identity path needs far more iterations."""
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=False, n_surface=48, n_layers=12, seed=4)
    p = _stable()
    with Solver(p, desc=desc_of(m)) as s:
        developed_state(s, 300)
        s.compute_residual()
        a = s.solve_adjoint_system(beta=0.1, tol=1e-9, max_iter=200000)
        s.set_params(dataclasses.replace(p, adjoint_precond="none"))
        s.compute_residual()
        b = s.solve_adjoint_system(beta=0.1, tol=1e-9, max_iter=200000)
        assert a["relres"] <= 1e-9 and b["relres"] <= 1e-9
        assert b["iters"] > 5 * a["iters"]
        assert max_rel(a["lambda"], b["lambda"]) < 1e-5


def test_shape_gradient_with_own_adjoint_matches_oracle():
    from optimisation2forme_b200 import HostMesh, Solver
    m = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=4, m=0.02, p=0.4, t=0.12)
    p = _stable()
    o = cpu.Oracle(HostMesh(desc=desc_of(m)), p)
    sh = Solver.shape_params(["m", "p", "t", "pos_x"], [0.02, 0.4, 0.12, 0.355])
    with Solver(p, desc=desc_of(m)) as s:
        U = developed_state(s, 300)
        s.compute_residual()
        out = s.optimize_shape(["m", "p", "t"], sh, beta=0.1, tol=1e-10)
        lam = s.solve_adjoint_system(beta=0.1, tol=1e-10)["lambda"]
        g_ref = o.shape_gradient(U, lam, sh, [0, 1, 2], 0.1)
        assert np.all(np.abs(out["grad"] - g_ref) <= 1e-6 * np.abs(g_ref).max())
        assert out["relres"] <= 1e-10


def test_profile_kernels_reports_every_class():
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=1)
    with Solver(_stable(), desc=desc_of(m)) as s:
        prof = s.profile_kernels(3)
        assert set(prof) == {"vertex_state", "cell_gradient", "vertex_visc", "edge_flux", "cell_residual",
                             "jt_apply", "jt_blocks"}
        assert all(v > 0 for v in prof.values())

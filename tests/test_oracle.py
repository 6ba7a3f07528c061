"""The CPU oracle (oracle/o2f_oracle.c) pinned against the reference.

1. Against the golden digests of the reference's own outputs on the shipped
   fixture (tests/golden/golden.json): bit-for-bit (SHA-256 of the float64
   bytes).
2. Live against the compiled reference (oracle/_ref) on seeded quad O-grids,
   when that build is present.
3. Properties of the extensions the reference does not have (angle of attack,
   valence >= 5): zero angle reproduces the reference path exactly.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import GOLDEN, bits_equal, desc_of, max_rel, perturbed_freestream, sha, small_mesh
from oracle import cpu, ref


@pytest.fixture(scope="module")
def fixture_oracle(fixture_mesh, fixture_params):
    return cpu.Oracle(fixture_mesh, fixture_params)


@pytest.fixture(scope="module")
def fixture_residual(fixture_oracle, fixture_state):
    return fixture_oracle.residual(fixture_state)


def test_residual_matches_reference_digests(fixture_residual, golden):
    for k in ("R", "grad", "edge_LR", "edge_tau"):
        assert sha(fixture_residual[k]) == golden["residual"][k]["sha256"], k


def test_known_answers_of_the_fixture(fixture_residual, fixture_oracle, golden):
    # RMS(R_rho) ~ 0.101 and C_L ~ 0 on the symmetric airfoil (m = 0).
    R = fixture_residual["R"]
    assert abs(np.sqrt(np.mean(R[0::4] ** 2)) - 0.10146) < 1e-4
    f = fixture_oracle.forces(fixture_residual["edge_LR"], fixture_residual["edge_tau"], 50.0)
    assert abs(f[0]) < 2e-3
    assert bits_equal(f, golden["forces"][:3])


def test_jt_rhs_and_gradient_match_reference_digests(fixture_oracle, fixture_residual, fixture_state, golden):
    from optimisation2forme_b200 import Solver, load_params_generic
    LR = fixture_residual["edge_LR"]
    nc = fixture_oracle.nc
    x = np.random.default_rng(0).standard_normal(4 * nc)
    assert sha(fixture_oracle.jt(LR, x)) == golden["jt"]["sha256"]
    names, vals, opt = load_params_generic(GOLDEN / "naca_2D_shape_params_0.txt")
    beta = dict(zip(names, vals))["beta"]
    assert sha(fixture_oracle.rhs(LR, beta)) == golden["rhs"]["sha256"]
    lam = 1e-3 * np.random.default_rng(1).standard_normal(4 * nc)
    g = fixture_oracle.shape_gradient(fixture_state, lam, Solver.shape_params(names, vals), [0, 1], beta)
    assert bits_equal(g, golden["shape_grad"])


def test_topology_matches_reference_digests(fixture_mesh, golden):
    for k, d in golden["topology"].items():
        assert sha(fixture_mesh.array(k)) == d["sha256"], k


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("n_surface,n_layers,seed", [(48, 12, 0), (96, 30, 3)])
def test_oracle_equals_reference_on_generated_quads(tmp_path, n_surface, n_layers, seed):
    """Seeded quad O-grids (every interior vertex has 4 cells): the oracle and
    the reference agree bit for bit on every stage and on J^T x."""
    from optimisation2forme_b200 import HostMesh, SimulationParams, save_cell_states
    from optimisation2forme_b200.meshgen import write_msh2
    m = small_mesh(triangles=False, n_surface=n_surface, n_layers=n_layers, seed=seed, m=0.03, p=0.45)
    msh = tmp_path / "g.msh"
    write_msh2(msh, m)
    p = SimulationParams(mesh_name=str(msh), viscosity=0.05, inflow_velocity=0.6)
    hm = HostMesh(msh)
    o = cpu.Oracle(hm, p)
    U = perturbed_freestream(o.nc, p, seed=seed)
    st = tmp_path / "state"
    save_cell_states(st, U)
    cfg = ref.write_config(tmp_path / "cfg.txt", mesh=str(msh), state=str(st), viscosity=0.05,
                           inflow_velocity=0.6)
    topo = ref.run("topo", cfg)
    for k in ("edge_v", "edge_c", "edge_bc", "cell_edges", "vert_cells", "vert_cells_ord"):
        assert np.array_equal(hm.array(k), topo[k]), k
    r1 = ref.run("residual", cfg)
    r2 = o.residual(np.loadtxt(st, skiprows=1).reshape(-1))
    for k in ("R", "grad", "edge_LR", "edge_tau"):
        assert bits_equal(r2[k], r1[k]), k
    x = np.random.default_rng(seed).standard_normal(4 * o.nc)
    x.tofile(tmp_path / "x.f64")
    assert bits_equal(o.jt(r2["edge_LR"], x), ref.run("jt", cfg, tmp_path / "x.f64")["jt_y"])


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
def test_oracle_time_loop_equals_reference(tmp_path):
    """A few SSP-RK3 steps of the restated time loop against the reference
    functions driven by the harness: identical states, dt and residual history."""
    from optimisation2forme_b200 import HostMesh, SimulationParams, save_cell_states
    from optimisation2forme_b200.meshgen import write_msh2
    m = small_mesh(triangles=False, n_surface=48, n_layers=12, seed=5)
    msh = tmp_path / "g.msh"
    write_msh2(msh, m)
    p = SimulationParams(mesh_name=str(msh), viscosity=0.05, inflow_velocity=0.6, cfl_number=0.5, final_time=1.0)
    o = cpu.Oracle(HostMesh(msh), p)
    U = perturbed_freestream(o.nc, p, seed=2)
    save_cell_states(tmp_path / "s", U)
    cfg = ref.write_config(tmp_path / "cfg.txt", mesh=str(msh), state=str(tmp_path / "s"), viscosity=0.05,
                           inflow_velocity=0.6, final_time=1.0)
    r1 = ref.run("march", cfg, 5)
    r2 = o.march(np.loadtxt(tmp_path / "s", skiprows=1).reshape(-1), 5)
    assert bits_equal(r2["U"], r1["U"])
    assert bits_equal(r2["dt"], r1["march_dt"])
    assert bits_equal(r2["history"], r1["march_rnorm"])


def test_zero_angle_of_attack_is_the_reference_path(fixture_mesh, fixture_params, fixture_state, fixture_residual):
    p = dataclasses.replace(fixture_params, aoa_deg=0.0)
    r = cpu.Oracle(fixture_mesh, p).residual(fixture_state)
    assert bits_equal(r["R"], fixture_residual["R"])
    p2 = dataclasses.replace(fixture_params, aoa_deg=2.0)
    r2 = cpu.Oracle(fixture_mesh, p2).residual(fixture_state)
    assert not bits_equal(r2["R"], fixture_residual["R"])


def test_triangle_mesh_interpolation_is_consistent():
    """Valence >= 5 vertices (no reference counterpart): the weights of every
    vertex sum to one and a uniform state is reproduced at interior vertices."""
    from optimisation2forme_b200 import HostMesh, SimulationParams
    m = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=1)
    hm = HostMesh(desc=desc_of(m))
    assert np.diff(hm.array("vert_cells_off")).max() >= 6
    w = hm.array("vert_w")
    off = hm.array("vert_cells_off")
    sums = np.add.reduceat(w, off[:-1])
    assert np.allclose(sums, 1.0, atol=1e-12)
    p = SimulationParams(viscosity=0.05, inflow_velocity=0.5)
    o = cpu.Oracle(hm, p)
    rho, pr = p.rho_ref, p.p_ref
    u = 0.5 * np.sqrt(1.4 * pr / rho)
    U = np.tile([rho, rho * u, 0.0, pr / 0.4 + 0.5 * rho * u * u], o.nc)
    r = o.residual(U)
    vU = r["vertex_U"].reshape(-1, 4)
    interior = hm.array("vert_bc") == 0
    assert max_rel(vU[interior], np.broadcast_to(U[:4], vU[interior].shape)) < 1e-12

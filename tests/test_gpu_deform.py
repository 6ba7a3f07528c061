"""Moving a live context to a new shape without re-meshing: new vertex
coordinates (o2f_set_vertex_coords) give exactly the context a fresh build on
those coordinates gives, and the GPU deformation (o2f_deform_shape) moves the
wall by the reference's perturbation formula, keeps the outer boundary and
carries the interior along without folding a cell."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import bits_equal, desc_of, developed_state, small_mesh

pytestmark = pytest.mark.gpu

KW = dict(triangles=True, n_surface=48, n_layers=12, seed=11)


def _params():
    from optimisation2forme_b200 import SimulationParams
    return SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0,
                            limiter_k=5.0, verbosity=0)


def _shape(m, p, t):
    from optimisation2forme_b200 import Solver
    return Solver.shape_params(["pos_x", "c", "m", "p", "t"], [0.355, 1.0, m, p, t])


def test_new_coordinates_give_the_context_of_a_fresh_build():
    from optimisation2forme_b200 import Solver
    from optimisation2forme_b200._lib import O2FError
    a = small_mesh(m=0.02, p=0.4, t=0.12, **KW)
    b = small_mesh(m=0.04, p=0.35, t=0.11, **KW)
    with Solver(_params(), desc=desc_of(a)) as moved, Solver(_params(), desc=desc_of(b)) as fresh:
        U = developed_state(moved, 200)
        moved.set_vertex_coords(b["node_xy"])
        with pytest.raises(O2FError) as e:
            moved.lift_drag(0.1)  # the interface states belong to the old geometry
        assert e.value.status == "O2F_ERR_STATE"
        assert bits_equal(moved.get_state(), U)  # the state is kept
        fresh.set_state(U)
        assert bits_equal(moved.compute_residual(), fresh.compute_residual())
        assert moved.lift_drag(0.1) == fresh.lift_drag(0.1)
        x = np.random.default_rng(1).standard_normal(4 * moved.n_cells)
        assert bits_equal(moved.apply_jacobian_transpose(x), fresh.apply_jacobian_transpose(x))
        assert bits_equal(moved.assemble_adjoint_rhs(0.1), fresh.assemble_adjoint_rhs(0.1))
        ra, rb = moved.time_loop(50), fresh.time_loop(50)
        assert ra["t"] == rb["t"] and bits_equal(moved.get_state(), fresh.get_state())


def test_deformation_moves_the_wall_by_the_perturbation_formula():
    from optimisation2forme_b200 import HostMesh, Solver
    a = small_mesh(m=0.02, p=0.4, t=0.12, **KW)
    with Solver(_params(), desc=desc_of(a)) as s:
        developed_state(s, 50)
        frm = _shape(0.02, 0.4, 0.12)
        # the wall as the shape gradient perturbs it: m + 0.01
        wall_ref = s.perturbed_geometry(frm, "m", 0.01, "vert_xy").reshape(-1, 2)
        xy0 = s.mesh_array("vert_xy").reshape(-1, 2)
        s.deform_shape(frm, _shape(0.03, 0.4, 0.12), power=4)
        xy1 = s.mesh_array("vert_xy").reshape(-1, 2)
        vbc = s.mesh_array("vert_bc")
        wall, outer = vbc == ord("w"), (vbc != 0) & (vbc != ord("w"))
        assert bits_equal(xy1[wall], wall_ref[wall])
        assert bits_equal(xy1[outer], xy0[outer])
        dwall = np.linalg.norm(xy1[wall] - xy0[wall], axis=1).max()
        dint = np.linalg.norm(xy1[vbc == 0] - xy0[vbc == 0], axis=1)
        assert dwall > 0 and 0 < dint.max() <= dwall * (1 + 1e-12)
        # the interior against inverse distance weighting restated in numpy:
        # all boundary vertices are sources, weights |r|^-4
        src = vbc != 0
        d_src = np.where(wall[src][:, None], wall_ref[src] - xy0[src], 0.0)
        inner = np.nonzero(vbc == 0)[0]
        r2 = ((xy0[inner][:, None, :] - xy0[src][None, :, :]) ** 2).sum(-1)
        w = 1.0 / (r2 * r2)
        want = xy0[inner] + (w @ d_src) / w.sum(axis=1)[:, None]
        assert np.abs(xy1[inner] - want).max() <= 1e-12 * dwall
        # the context's geometry is the host build on the moved coordinates
        h = HostMesh(desc=desc_of(dict(a, node_xy=xy1.reshape(-1))))
        for name in ("cell_vol", "edge_n", "vert_w"):
            assert bits_equal(s.mesh_array(name), h.array(name)), name
        assert np.all(h.array("cell_vol") > 0)
        r = s.time_loop(20)
        assert r["status"] == "OK" and np.all(np.isfinite(s.get_state()))


def test_outer_loop_on_a_deformed_mesh():
    from optimisation2forme_b200.meshgen import OGridSpec
    from optimisation2forme_b200.optimize import SignDescent, optimise
    spec = OGridSpec(m=0.02, p=0.4, t=0.12, n_surface=48, n_layers=12, triangles=True, seed=2)
    dfm = optimise(spec, _params(), iterations=3, rk_steps=100, beta=0.1, tol=1e-8, mesh_update="deform")
    reg = optimise(spec, _params(), iterations=1, rk_steps=100, beta=0.1, tol=1e-8)
    rule = SignDescent()
    for a, b in zip(dfm, dfm[1:]):
        assert (b["m"], b["p"]) == rule.step(a["m"], a["p"], a["dJ_dm"], a["dJ_dp"])
    assert all(h["adjoint_status"] == "OK" for h in dfm)
    # the first iteration runs on the generated mesh in both modes
    assert (dfm[0]["J"], dfm[0]["dJ_dm"], dfm[0]["dJ_dp"]) == (reg[0]["J"], reg[0]["dJ_dm"], reg[0]["dJ_dp"])
    print(f"\ndeformed-mesh loop: J {[round(h['J'], 6) for h in dfm]}, m {[h['m'] for h in dfm]}, "
          f"p {[h['p'] for h in dfm]}, adjoint iterations {[h['adjoint_iters'] for h in dfm]}")

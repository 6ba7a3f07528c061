"""Headless field images (o2f_render_field) against the numpy restatement of
the reference's view (oracle/render_ref.py): the same bytes for every cell
field, both colour maps, triangles and quadrilaterals, a non-square image,
the pressure range rule, a given range, and an all-black image when the
field is uniform."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, developed_state, small_mesh
from oracle import render_ref as rr

pytestmark = pytest.mark.gpu


def _params():
    from optimisation2forme_b200 import SimulationParams
    return SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0,
                            limiter_k=5.0, verbosity=0)


@pytest.mark.parametrize("triangles", [True, False])
def test_images_match_the_oracle(triangles):
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=triangles, n_surface=48, n_layers=12, seed=5)
    with Solver(_params(), desc=desc_of(m)) as s:
        U = developed_state(s, 150)
        nx, ny = 96, 72
        for field in ("rho", "rho_u", "rho_v", "E", "u", "v", "p", "div", "u_y"):
            for cmap in ("", "schlieren"):
                img, rng = s.render_field(field, nx, ny, cmap)
                grad = s.debug("grad") if field in ("div", "u_y") else None
                sc = rr.cell_scalar(U, field, s.params.gamma, grad)
                lo, hi = rr.colour_range(sc, field)
                assert rng == (lo, hi), field
                want = rr.render(m["node_xy"], m["cell_offsets"], m["cell_nodes"], sc, nx, ny, lo, hi, cmap)
                bad = np.argwhere(np.any(img != want, axis=-1))
                assert bad.size == 0, f"{field} {cmap}: {len(bad)} pixels differ, first {bad[:3].tolist()}"
        assert rng[0] < rng[1]
        # a given range; black outside the mesh (the airfoil) and colour inside
        img, rng = s.render_field("p", nx, ny, vrange=(90_000.0, 110_000.0))
        assert rng == (90_000.0, 110_000.0)
        sc = rr.cell_scalar(U, "p", s.params.gamma)
        assert np.array_equal(img, rr.render(m["node_xy"], m["cell_offsets"], m["cell_nodes"], sc, nx, ny,
                                             90_000.0, 110_000.0))
        assert np.any(img.sum(axis=-1) == 0) and np.any(img.sum(axis=-1) > 0)


def test_uniform_field_draws_nothing():
    from optimisation2forme_b200 import Solver
    m = small_mesh(triangles=True, n_surface=32, n_layers=8, seed=1)
    with Solver(_params(), desc=desc_of(m)) as s:
        s.initialize_freestream()
        img, rng = s.render_field("rho", 40, 30)
        assert rng[0] == rng[1] and not img.any()

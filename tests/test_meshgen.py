"""The seeded O-grid generator that stands in for Gmsh: counter-clockwise
cells, closed wall and far-field loops, boundary vertices with 2 or 4 cells
(the reference's barycentric weights extrapolate at 3), and the workload
sizes."""
from __future__ import annotations

import numpy as np
import pytest

from optimisation2forme_b200.meshgen import OGridSpec, config_mesh, naca4_surface, naca_ogrid, viscosity_for


def _signed_areas(m):
    xy = m["node_xy"].reshape(-1, 2)
    offs, cn = m["cell_offsets"], m["cell_nodes"]
    out = []
    for c in range(len(offs) - 1):
        v = xy[cn[offs[c]:offs[c + 1]]]
        x, y = v[:, 0], v[:, 1]
        out.append(0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))
    return np.array(out)


@pytest.mark.parametrize("triangles", [True, False])
def test_cells_are_counter_clockwise_and_tile_the_annulus(triangles):
    spec = OGridSpec(n_surface=40, n_layers=10, triangles=triangles, seed=3)
    m = naca_ogrid(spec)
    a = _signed_areas(m)
    assert np.all(a > 0)
    # the cells fill the disc of radius r_far minus the airfoil
    S = naca4_surface(spec.m, spec.p, spec.t, spec.n_surface, spec.chord, spec.pos_x)
    airfoil = 0.5 * np.sum(S[:, 0] * np.roll(S[:, 1], -1) - np.roll(S[:, 0], -1) * S[:, 1])
    far_loop = m["node_xy"].reshape(-1, 2)[m["segments"][m["segment_bc"] == ord("f")][:, 0]]
    disc = 0.5 * np.sum(far_loop[:, 0] * np.roll(far_loop[:, 1], -1) - np.roll(far_loop[:, 0], -1) * far_loop[:, 1])
    assert a.sum() == pytest.approx(disc - airfoil, rel=1e-9)


def test_boundary_vertices_have_two_or_four_cells():
    m = naca_ogrid(OGridSpec(n_surface=40, n_layers=10, triangles=True, seed=5))
    nv = m["node_xy"].size // 2
    count = np.bincount(m["cell_nodes"], minlength=nv)
    bverts = np.unique(m["segments"])
    assert set(np.unique(count[bverts])) <= {2, 4}


def test_segments_close_both_loops():
    m = naca_ogrid(OGridSpec(n_surface=30, n_layers=6, seed=1))
    for code in (ord("f"), ord("w")):
        seg = m["segments"][m["segment_bc"] == code]
        assert np.array_equal(np.sort(seg[:, 0]), np.sort(seg[:, 1]))  # every vertex starts and ends one segment


def test_generator_is_seeded():
    a = naca_ogrid(OGridSpec(n_surface=30, n_layers=6, seed=7))
    b = naca_ogrid(OGridSpec(n_surface=30, n_layers=6, seed=7))
    c = naca_ogrid(OGridSpec(n_surface=30, n_layers=6, seed=8))
    assert np.array_equal(a["cell_nodes"], b["cell_nodes"]) and np.array_equal(a["node_xy"], b["node_xy"])
    assert not np.array_equal(a["cell_nodes"], c["cell_nodes"])


def test_workload_sizes_and_viscosity():
    spec, flow = config_mesh("large")
    cells = 2 * (spec.n_surface + 3 + 1) * spec.n_layers  # 2 triangles per quad; +3 base points, +1 LE
    assert 1.9e6 < cells < 2.1e6 and spec.first_height == 1e-4 and flow["mach"] == 0.85
    mu = viscosity_for(1e4, 0.6)
    assert mu == pytest.approx(1.225 * 0.6 * np.sqrt(1.4 * 101325 / 1.225) / 1e4)

"""The image oracle (oracle/render_ref.py) on the CPU: colour-map values
worked out by hand from the reference's formulas
(include/renderer_colormap.hpp:16-95), the pressure range rule of
Simulator::output_step, and the pixel map on a mesh small enough to check
cell by cell."""
from __future__ import annotations

import numpy as np

from oracle import render_ref as rr


def test_colour_maps_at_their_breakpoints():
    t = np.array([0.0, 0.25, 0.5, 1.0, -3.0, 7.0, np.nan])
    got = rr.colormap_bwr(t)
    # b(0) = float(0.3) * 255 + 0.5 -> 77; white at 0.5; r(1) = 0.5 -> 128
    want = [[0, 0, 77], [0, 0, 255], [255, 255, 255], [128, 0, 0], [0, 0, 77], [128, 0, 0], [128, 0, 0]]
    assert got.tolist() == want
    got = rr.colormap_schlieren(np.array([0.0, 0.35, 0.7, 1.0]))
    assert got.tolist() == [[0, 0, 0], [0, 0, 128], [0, 0, 255], [255, 255, 255]]


def test_pressure_range_is_rounded_to_5000():
    s = np.array([99_999.0, 101_325.0, 112_000.5])
    assert rr.colour_range(s, "p") == (95_000.0, 115_000.0)
    assert rr.colour_range(s, "rho") == (99_999.0, 112_000.5)


def test_pixel_map_of_two_triangles():
    # unit square split along the diagonal (0,0)-(1,1): cell 0 below, cell 1 above
    xy = np.array([0.0, 0.0, 1.0, 0.0, 1.0, 1.0, 0.0, 1.0])
    offs = np.array([0, 3, 6])
    nodes = np.array([0, 1, 2, 0, 2, 3])
    m = rr.pixel_cells(xy, offs, nodes, 4, 4)
    j, i = np.mgrid[0:4, 0:4]
    # pixel centres on the diagonal belong to both cells: the lower number wins
    assert np.array_equal(m, np.where(i >= j, 0, 1))
    img = rr.render(xy, offs, nodes, np.array([0.0, 1.0]), 4, 4, 0.0, 1.0)
    # top image row = pixel row j = 3 (y = 3.5/4): cell 1 (t = 1, dark red) left of the diagonal
    assert img[0].tolist() == [[128, 0, 0]] * 3 + [[0, 0, 77]]
    assert img[3].tolist() == [[0, 0, 77]] * 4  # bottom row: cell 0 (t = 0)

"""New vertex coordinates for a built mesh (o2f_host_mesh_set_coords), on the
CPU: a mesh moved onto the coordinates of another O-grid of the same topology
must export exactly the arrays of a mesh built from those coordinates, since
the device geometry of o2f_set_vertex_coords is uploaded from them."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, small_mesh

ARRAYS = ["vert_xy", "cell_vol", "cell_ctr", "edge_len", "edge_n", "edge_ctr", "vert_cells_ord", "vert_wcells",
          "vert_w", "min_h", "edge_v", "edge_c", "edge_bc", "vert_bc", "cell_edges", "vert_cells", "cell_nbrs"]


def _bits(a):
    return a.view(np.int64) if a.dtype == np.float64 else a


def _pair(triangles):
    kw = dict(triangles=triangles, n_surface=48, n_layers=12, seed=11)
    a = small_mesh(m=0.02, p=0.4, t=0.12, **kw)
    b = small_mesh(m=0.04, p=0.35, t=0.11, **kw)  # (the generator folds cells at m=0.05, p=0.3, t=0.10 here)
    assert np.array_equal(a["cell_nodes"], b["cell_nodes"]) and np.array_equal(a["segments"], b["segments"])
    return a, b


@pytest.mark.parametrize("triangles", [True, False])
def test_moved_mesh_equals_a_mesh_built_on_the_new_coordinates(triangles):
    from optimisation2forme_b200 import HostMesh
    a, b = _pair(triangles)
    moved, fresh = HostMesh(desc=desc_of(a)), HostMesh(desc=desc_of(b))
    moved.set_coords(b["node_xy"])
    for name in ARRAYS:
        assert np.array_equal(_bits(moved.array(name)), _bits(fresh.array(name))), name
    # and back
    moved.set_coords(a["node_xy"])
    orig = HostMesh(desc=desc_of(a))
    for name in ARRAYS:
        assert np.array_equal(_bits(moved.array(name)), _bits(orig.array(name))), name


def test_collapsed_or_folded_cells_are_rejected_and_the_mesh_is_kept():
    from optimisation2forme_b200 import HostMesh
    from optimisation2forme_b200._lib import O2FError
    a, _ = _pair(True)
    h = HostMesh(desc=desc_of(a))
    before = {n: h.array(n) for n in ARRAYS}
    xy = a["node_xy"].reshape(-1, 2).copy()
    c0 = a["cell_nodes"][a["cell_offsets"][0]:a["cell_offsets"][1]]
    collapsed = xy.copy()
    collapsed[c0] = collapsed[c0[0]]  # every vertex of cell 0 on one point
    with pytest.raises(O2FError) as e:
        h.set_coords(collapsed)
    assert e.value.status == "O2F_ERR_MESH"
    folded = xy.copy()
    folded[:, 1] = -folded[:, 1]  # mirror image: every cell changes orientation
    with pytest.raises(O2FError) as e:
        h.set_coords(folded)
    assert e.value.status == "O2F_ERR_MESH"
    bad = xy.copy()
    bad[3, 0] = np.nan
    with pytest.raises(O2FError) as e:
        h.set_coords(bad)
    assert e.value.status == "O2F_ERR_ARG"
    for name in ARRAYS:
        assert np.array_equal(_bits(h.array(name)), _bits(before[name])), name

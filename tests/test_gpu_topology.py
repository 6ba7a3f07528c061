"""Mesh topology built on the GPU (o2f_host_mesh_create_gpu) against the host
build that reproduces the reference's std::map / std::unordered_set orders:
every exported array identical, on O-grids of triangles and quads, on a
shuffled numbering (irregular insertion sequences), on a fan whose centre
vertex has 40 cells (the emulated sets rehash), and the same error statuses
on broken meshes."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, small_mesh

pytestmark = pytest.mark.gpu

ARRAYS = ["edge_v", "edge_c", "edge_bc", "vert_bc", "cell_edges_off", "cell_edges", "vert_cells_off", "vert_cells",
          "vert_cells_ord", "vert_wcells", "cell_verts_off", "cell_verts", "cell_nbrs_off", "cell_nbrs", "vert_xy",
          "edge_len", "edge_n", "edge_ctr", "cell_vol", "cell_ctr", "vert_w", "min_h"]


def _same(m):
    from optimisation2forme_b200 import HostMesh
    a, b = HostMesh(desc=desc_of(m)), HostMesh(desc=desc_of(m), gpu=True)
    for name in ARRAYS:
        x, y = a.array(name), b.array(name)
        if x.dtype == np.float64:
            x, y = x.view(np.int64), y.view(np.int64)
        assert np.array_equal(x, y), name


def _shuffled(m, seed):
    """Same mesh, vertices and cells renumbered at random."""
    rng = np.random.default_rng(seed)
    nv = m["node_xy"].size // 2
    pv = rng.permutation(nv)  # new id of old vertex
    inv = np.argsort(pv)
    xy = m["node_xy"].reshape(-1, 2)[inv].reshape(-1)
    offs, nodes = m["cell_offsets"], m["cell_nodes"]
    cells = [pv[nodes[offs[c]:offs[c + 1]]] for c in range(len(offs) - 1)]
    order = rng.permutation(len(cells))
    cells = [cells[i] for i in order]
    new_offs = np.concatenate([[0], np.cumsum([len(c) for c in cells])])
    return dict(node_xy=xy, segments=pv[m["segments"]], segment_bc=m["segment_bc"], cell_offsets=new_offs,
                cell_nodes=np.concatenate(cells))


def _fan(n=40, r=1.0):
    t = np.linspace(0.0, 2 * np.pi, n, endpoint=False)
    xy = np.concatenate([[[0.0, 0.0]], np.stack([r * np.cos(t), r * np.sin(t)], axis=1)]).reshape(-1)
    cells = np.array([[0, 1 + i, 1 + (i + 1) % n] for i in range(n)])
    segs = np.array([[1 + i, 1 + (i + 1) % n] for i in range(n)])
    return dict(node_xy=xy, segments=segs, segment_bc=np.full(n, ord("f"), dtype=np.uint8),
                cell_offsets=np.arange(0, 3 * n + 1, 3), cell_nodes=cells.reshape(-1))


@pytest.mark.parametrize("triangles", [True, False])
def test_gpu_build_equals_host_build(triangles):
    m = small_mesh(triangles=triangles, n_surface=64, n_layers=16, seed=3)
    _same(m)
    _same(_shuffled(m, 7))


def test_high_valence_vertex():
    _same(_fan(40))
    _same(_shuffled(_fan(40), 2))


def test_broken_meshes_give_the_host_errors():
    from optimisation2forme_b200 import HostMesh, O2FError
    m = small_mesh(triangles=True, n_surface=32, n_layers=8, seed=1)
    no_bc = dict(m, segments=m["segments"][1:], segment_bc=m["segment_bc"][1:])
    # the edge between the second and third vertex of cell 0 is interior
    bc_inside = dict(m, segments=np.concatenate([m["segments"], [m["cell_nodes"][1:3]]]),
                     segment_bc=np.concatenate([m["segment_bc"], [ord("w")]]).astype(np.uint8))
    c0 = m["cell_nodes"][:3]
    shared3 = dict(m, cell_offsets=np.concatenate([m["cell_offsets"], [m["cell_offsets"][-1] + 3]]),
                   cell_nodes=np.concatenate([m["cell_nodes"], c0]))
    out_of_range = dict(m, cell_nodes=np.where(np.arange(m["cell_nodes"].size) == 4, 10 ** 7, m["cell_nodes"]))
    for bad in (no_bc, bc_inside, shared3, out_of_range):
        statuses = []
        for gpu in (False, True):
            with pytest.raises(O2FError) as e:
                HostMesh(desc=desc_of(bad), gpu=gpu)
            statuses.append(e.value.status)
        assert statuses[0] == statuses[1] == "O2F_ERR_MESH", statuses


def test_large_context_uses_the_same_mesh():
    """From 100,000 cells a context builds its topology on the GPU; its mesh
    is the host build's."""
    from optimisation2forme_b200 import HostMesh, Solver, SimulationParams
    m = small_mesh(triangles=True, n_surface=400, n_layers=130, seed=9)
    assert m["cell_offsets"].size - 1 >= 100_000
    host = HostMesh(desc=desc_of(m))
    with Solver(SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, verbosity=0), desc=desc_of(m)) as s:
        for name in ARRAYS:
            x, y = host.array(name), s.mesh_array(name)
            if x.dtype == np.float64:
                x, y = x.view(np.int64), y.view(np.int64)
            assert np.array_equal(x, y), name

"""The msh2 reader's two paths, on the CPU: files from 1 MB are parsed by all
host threads (node and element lines at once), anything else -- or any
irregular layout -- by the stream reader.  Both must give the mesh the
generator wrote; the reference's own fixture (2.1 MB) goes through the
parallel path in the oracle tests."""
from __future__ import annotations

import numpy as np

from conftest import desc_of, small_mesh

ARRAYS = ["vert_xy", "edge_v", "edge_c", "edge_bc", "cell_edges", "vert_cells", "cell_vol", "vert_w"]


def _bits(a):
    return a.view(np.int64) if a.dtype == np.float64 else a


def test_parallel_and_stream_readers_give_the_written_mesh(tmp_path):
    from optimisation2forme_b200 import HostMesh
    from optimisation2forme_b200.meshgen import write_msh2
    m = small_mesh(triangles=True, n_surface=200, n_layers=60, seed=6)
    big = tmp_path / "big.msh"
    write_msh2(big, m)
    assert big.stat().st_size >= 1 << 20  # the parallel path
    text = big.read_text()
    # two node entries on one line: legal for the stream reader only
    k = text.index("\n", text.index("\n", text.index("$Nodes\n") + 7) + 1)
    joined = tmp_path / "joined.msh"
    joined.write_text(text[:k] + " " + text[k + 1:])
    # CRLF line ends and a '+' sign: both readers accept them
    crlf = tmp_path / "crlf.msh"
    crlf.write_bytes(text.replace("\n", "\r\n").replace("\n1 ", "\n+1 ", 1).encode())
    want = HostMesh(desc=desc_of(m))
    for path in (big, joined, crlf):
        got = HostMesh(path)
        for name in ARRAYS:
            assert np.array_equal(_bits(got.array(name)), _bits(want.array(name))), (path.name, name)

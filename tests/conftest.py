"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device; everything else
runs on the CPU (the oracle, host mesh build, I/O, ABI symbol table, gloo
ranks).  The golden fixtures in tests/golden/ travel with the repository, so
no test needs the reference checkout at run time; tests that run the
reference's own compiled code (oracle/_ref) skip when it is absent."""
from __future__ import annotations

import lzma
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built() -> None:
    from optimisation2forme_b200 import build as b
    b.build()


_ensure_built()


@pytest.fixture(scope="session")
def golden_dir(tmp_path_factory) -> Path:
    """Decompressed copies of the reference fixtures."""
    d = tmp_path_factory.mktemp("golden")
    for f in GOLDEN.glob("*.xz"):
        with lzma.open(f, "rb") as src, open(d / f.stem, "wb") as dst:
            shutil.copyfileobj(src, dst)
    shutil.copy(GOLDEN / "naca_2D_shape_params_0.txt", d / "naca_2D_shape_params_0.txt")
    return d


@pytest.fixture(scope="session")
def fixture_params(golden_dir):
    """Reference physics of the shipped fixtures (mesh_opti/config.txt:14-61:
    mu = 1.8e-5, M = 0.3, CFL 0.5, final_time 0.005, later keys win)."""
    from optimisation2forme_b200 import SimulationParams
    return SimulationParams(mesh_name=str(golden_dir / "naca_2D_shape_0.msh"), viscosity=1.8e-5, Pr=0.71,
                            cfl_number=0.5, final_time=0.005, inflow_velocity=0.3,
                            boundary_conditions="inflow_outflow_x", initial_condition="one_x",
                            state_load_path=str(golden_dir / "naca_2D_flow_1"),
                            shape_param_file=str(golden_dir / "naca_2D_shape_params_0.txt"), verbosity=0)


@pytest.fixture(scope="session")
def fixture_mesh(fixture_params):
    from optimisation2forme_b200 import HostMesh
    return HostMesh(fixture_params.mesh_name)


@pytest.fixture(scope="session")
def fixture_state(fixture_params, fixture_mesh):
    from optimisation2forme_b200 import load_cell_states
    return load_cell_states(fixture_params.state_load_path, fixture_mesh.array("cell_vol").size)


@pytest.fixture(scope="session")
def golden():
    import json
    return json.loads((GOLDEN / "golden.json").read_text())


def small_mesh(triangles=True, n_surface=64, n_layers=20, seed=0, **kw):
    """A small seeded NACA O-grid description (quads: reference-valid)."""
    from optimisation2forme_b200.meshgen import OGridSpec, naca_ogrid
    return naca_ogrid(OGridSpec(n_surface=n_surface, n_layers=n_layers, triangles=triangles, seed=seed, **kw))


def desc_of(m):
    from optimisation2forme_b200 import mesh_desc
    return mesh_desc(m["node_xy"], m["segments"], m["segment_bc"], m["cell_offsets"], m["cell_nodes"])


def perturbed_freestream(n_cells, params, seed=0, amp=0.02):
    """A seeded non-uniform state around the freestream (positive rho, p)."""
    rng = np.random.default_rng(seed)
    g, rho, p = params.gamma, params.rho_ref, params.p_ref
    a = np.sqrt(g * p / rho)
    u = params.inflow_velocity * a
    r = rho * (1 + amp * rng.standard_normal(n_cells))
    uu = u * (1 + amp * rng.standard_normal(n_cells))
    vv = u * amp * rng.standard_normal(n_cells)
    pp = p * (1 + amp * rng.standard_normal(n_cells))
    E = pp / (g - 1) + 0.5 * r * (uu * uu + vv * vv)
    return np.stack([r, r * uu, r * vv, E], axis=1).reshape(-1)


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def max_rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def sha(a) -> str:
    import hashlib
    a = np.asarray(a)
    return hashlib.sha256(np.ascontiguousarray(a).astype("<f8" if a.dtype.kind == "f" else "<i8").tobytes()).hexdigest()


def developed_state(solver, steps=300):
    """A flow marched from the freestream (smooth, physically reachable)."""
    solver.initialize_freestream()
    solver.time_loop(steps)
    return solver.get_state()


def assemble_jt(oracle, host_mesh, LR):
    """J^T as a scipy sparse matrix, probed column by column through the
    oracle's matrix-free product (distance-2 colouring of the cells)."""
    import scipy.sparse as sp
    nc = oracle.nc
    ec = host_mesh.array("edge_c").reshape(-1, 2)
    nbr = [set() for _ in range(nc)]
    for a, c in ec:
        if c >= 0:
            nbr[a].add(c)
            nbr[c].add(a)
    col = -np.ones(nc, dtype=np.int64)
    for c in range(nc):
        used = set()
        for n in nbr[c]:
            used.add(col[n])
            used.update(col[m] for m in nbr[n])
        k = 0
        while k in used:
            k += 1
        col[c] = k
    rows, cols, vals = [], [], []
    for k in range(col.max() + 1):
        idx = np.where(col == k)[0]
        for j in range(4):
            x = np.zeros(4 * nc)
            x[4 * idx + j] = 1.0
            y = oracle.jt(LR, x).reshape(-1, 4)
            for i in idx:
                for r in [i] + list(nbr[i]):
                    for q in range(4):
                        if y[r, q] != 0.0:
                            rows.append(4 * r + q)
                            cols.append(4 * i + j)
                            vals.append(y[r, q])
    return sp.csr_matrix((vals, (rows, cols)), shape=(4 * nc, 4 * nc))

"""Host-side mirror of the reference's call surface over the C ABI.

The reference exposes free functions on a mutable ``Mesh&``
(include/advection.hpp:16-19, include/diffusion.hpp:16, include/compute.hpp:18,
include/shape_optimization.hpp:24-29).  ``Solver`` is the device-resident
counterpart: one object per mesh, holding the state and the interface states
of the last residual, with methods named after the reference functions.
Arrays at this boundary are numpy, in reference cell / edge order, with
per-cell 4-vectors interleaved ``4*i+k`` (rho, rho_u, rho_v, E).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import O2FError, check, lib

__all__ = [
    "SimulationParams", "load_config", "load_params_generic", "load_cell_states", "save_cell_states",
    "HostMesh", "Solver", "O2FError", "mesh_desc",
]


@dataclasses.dataclass
class SimulationParams:
    """Fields of the reference's SimulationParams (include/params.hpp:15-81)
    that the hot path reads, plus the keys the reference hard-codes."""

    mesh_name: str = "naca_2D.msh"
    cfl_number: float = 0.1
    final_time: float = 5.0
    gamma: float = 1.4
    viscosity: float = 1e-6
    Pr: float = 0.71
    cp: float = 1005.0
    inflow_velocity: float = 1.0
    rho_ref: float = 1.225
    p_ref: float = 101325.0
    boundary_conditions: str = "periodic"
    initial_condition: str = "one"
    state_load_path: str = ""
    state_save_path: str = ""
    shape_opt_enable: bool = False
    shape_param_file: str = ""
    shape_log_file: str = ""
    verbosity: int = 1
    # keys without a reference counterpart (defaults reproduce the reference)
    aoa_deg: float = 0.0
    limiter_k: float = 1e-2
    limiter: str = "venkatakrishnan"
    precision: str = "fp64"
    adjoint_precond: str = "ilu0"
    dt_mode: str = "reference"
    adjoint_shift: float = 0.0
    adjoint_jacobian: str = "reference"
    adjoint_fd_step: float = 1e-9
    adjoint_precision: str = "fp64"
    adjoint_sweeps: str = "auto"
    max_steps: int = 2**62
    residual_drop: float = 0.0
    adjoint_tol: float = 1e-6
    adjoint_restart: int = 500
    adjoint_max_iter: int = 100000

    def to_c(self) -> _lib.Params:
        p = _lib.Params()
        lib().o2f_params_default(C.byref(p))
        for f in ("gamma", "viscosity", "Pr", "cp", "cfl_number", "final_time", "inflow_velocity", "rho_ref",
                  "p_ref", "aoa_deg", "limiter_k", "adjoint_shift", "adjoint_fd_step"):
            setattr(p, f, float(getattr(self, f)))
        lim = self.limiter.lower()
        if lim in ("venkatakrishnan", "venkat"):
            p.limiter = _lib.LIMITER_VENKAT
        elif lim in ("barth_jespersen", "bj"):
            p.limiter = _lib.LIMITER_BARTH_JESPERSEN
        else:
            raise ValueError(f"unknown limiter {self.limiter!r}")
        p.precision = {"fp64": _lib.PREC_F64, "fp32": _lib.PREC_F32}[self.precision.lower()]
        p.adjoint_precision = {"fp64": _lib.PREC_F64, "fp32": _lib.PREC_F32}[self.adjoint_precision.lower()]
        p.adjoint_sweeps = {"auto": 0, "block": 1, "waiting": 2}[self.adjoint_sweeps.lower()]
        p.adjoint_precond = {"none": 0, "identity": 0, "ilu0": 1}[self.adjoint_precond.lower()]
        p.dt_mode = {"reference": 0, "thermal": 1}[self.dt_mode.lower()]
        p.adjoint_jacobian = {"reference": 0, "first_order": 0, "full": 1,
                              "frozen_limiter": 2}[self.adjoint_jacobian.lower()]
        p.verbosity = int(self.verbosity)
        return p


_FLOAT_KEYS = {"cfl_number", "final_time", "gamma", "viscosity", "Pr", "cp", "inflow_velocity", "rho_ref", "p_ref",
               "aoa_deg", "limiter_k", "residual_drop", "adjoint_tol", "adjoint_shift", "adjoint_fd_step"}
_INT_KEYS = {"verbosity", "max_steps", "adjoint_restart", "adjoint_max_iter"}
_STR_KEYS = {"mesh_name", "boundary_conditions", "initial_condition", "state_load_path", "state_save_path",
             "shape_param_file", "shape_log_file", "limiter", "precision", "adjoint_precond", "dt_mode",
             "adjoint_jacobian", "adjoint_precision", "adjoint_sweeps"}


def load_config(path: str | os.PathLike, params: SimulationParams | None = None) -> SimulationParams:
    """Read a reference config file: ``key = value`` lines, ``#`` comments,
    later keys override earlier ones (load_config, src/params.cpp:18-83).
    Keys the hot path does not use are ignored, as the reference ignores
    unknown keys."""
    p = params or SimulationParams()
    with open(path, "r", encoding="utf-8", errors="replace") as fh:
        for line in fh:
            t = line.strip()
            if not t or t.startswith("#") or "=" not in t:
                continue
            key, val = (s.strip() for s in t.split("=", 1))
            if key in _FLOAT_KEYS:
                setattr(p, key, float(val.split()[0]))
            elif key in _INT_KEYS:
                setattr(p, key, int(float(val.split()[0])))
            elif key == "shape_opt_enable":
                p.shape_opt_enable = bool(int(val.split()[0]))
            elif key in _STR_KEYS:
                setattr(p, key, val)
    if p.boundary_conditions not in ("inflow_outflow_x", "periodic"):
        raise ValueError(f"Unknown boundary condition: {p.boundary_conditions}")
    return p


def load_params_generic(path: str | os.PathLike) -> tuple[list[str], list[float], list[str]]:
    """``key = v`` / ``key *= v`` parameter file (loadParamsGeneric,
    src/shape_optimization.cpp:19-98): returns (names_all, values_all,
    optimised names in order of first appearance)."""
    names_all: list[str] = []
    values_all: list[float] = []
    is_opt: set[str] = set()
    if not path or str(path) == "none":
        return names_all, values_all, []
    with open(path, "r", encoding="utf-8") as fh:
        for line in fh:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            mark = False
            if "*=" in line:
                mark = True
                key, sval = line.split("*=", 1)
            elif "=" in line:
                key, sval = line.split("=", 1)
            else:
                parts = line.split()
                key, sval = (parts + ["", ""])[:2]
            key, sval = key.strip(), sval.strip()
            if not key or not sval:
                continue
            v = float(sval.split()[0])
            if key in names_all:
                values_all[names_all.index(key)] = v
            else:
                names_all.append(key)
                values_all.append(v)
            if mark:
                is_opt.add(key)
            else:
                is_opt.discard(key)
    return names_all, values_all, [k for k in names_all if k in is_opt]


def load_cell_states(path: str | os.PathLike, n_cells: int) -> np.ndarray:
    """State file: ``N`` then N lines ``rho rho_u rho_v E`` (loadCellStates,
    src/utils.cpp:29-67).  Raises on a size mismatch, as the reference does."""
    with open(path, "r") as fh:
        head = fh.readline().split()
        if not head:
            raise ValueError(f"corrupt state file ({path}): cannot read the number of cells")
        n = int(head[0])
        if n != n_cells:
            raise ValueError(f"size mismatch ({path}): file={n} vs mesh={n_cells}")
        data = np.loadtxt(fh, dtype=np.float64, ndmin=2)
    if data.shape != (n, 4):
        raise ValueError(f"truncated state file ({path}): {data.shape[0]} of {n} cells")
    return np.ascontiguousarray(data.reshape(-1))


def save_cell_states(path: str | os.PathLike, U: np.ndarray) -> None:
    """Write the reference state format with 17 significant digits
    (saveCellStates, src/utils.cpp:70-107)."""
    U = np.asarray(U, dtype=np.float64).reshape(-1, 4)
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f"{U.shape[0]}\n")
        np.savetxt(fh, U, fmt="%.17e")


def _ptr(a: np.ndarray, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def write_image(path: str | os.PathLike, img: np.ndarray) -> None:
    """An RGB uint8 image [h, w, 3] as binary PPM (".ppm") or PNG (other
    suffixes; zlib, no other dependency)."""
    import struct
    import zlib
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    if path.suffix.lower() == ".ppm":
        path.write_bytes(f"P6\n{w} {h}\n255\n".encode() + img.tobytes())
        return

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    raw = b"".join(b"\x00" + img[r].tobytes() for r in range(h))
    path.write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
                     chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def save_state_binary(path: str | os.PathLike, U: np.ndarray, time: float = 0.0, steps: int = 0) -> None:
    """Binary checkpoint of a state (o2f_checkpoint_write): the values of the
    reference's text state file, bit for bit, as four float64 arrays."""
    U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
    if U.size == 0 or U.size % 4:
        raise ValueError("state must hold 4 values per cell")
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    check(lib().o2f_checkpoint_write(str(path).encode(), U.size // 4, _ptr(U), float(time), int(steps)))


def load_state_binary(path: str | os.PathLike, n_cells: int) -> tuple[np.ndarray, float, int]:
    """(state, time, steps) from a binary checkpoint (o2f_checkpoint_read);
    raises O2FError(O2F_ERR_IO) on a foreign, damaged or mismatched file."""
    U = np.empty(4 * int(n_cells))
    t = C.c_double()
    steps = C.c_int64()
    check(lib().o2f_checkpoint_read(str(path).encode(), int(n_cells), _ptr(U), C.byref(t), C.byref(steps)))
    return U, t.value, steps.value


def mesh_desc(node_xy, segments, segment_bc, cell_offsets, cell_nodes):
    """Build an o2f_mesh_desc; returns (desc, keepalive)."""
    keep = [np.ascontiguousarray(node_xy, dtype=np.float64).reshape(-1),
            np.ascontiguousarray(segments, dtype=np.int64).reshape(-1),
            np.ascontiguousarray(segment_bc, dtype=np.uint8).reshape(-1),
            np.ascontiguousarray(cell_offsets, dtype=np.int64).reshape(-1),
            np.ascontiguousarray(cell_nodes, dtype=np.int64).reshape(-1)]
    d = _lib.MeshDesc()
    d.n_nodes = keep[0].size // 2
    d.node_xy = _ptr(keep[0])
    d.n_segments = keep[2].size
    d.segments = _ptr(keep[1], C.c_int64)
    d.segment_bc = _ptr(keep[2], C.c_uint8)
    d.n_cells = keep[3].size - 1
    d.cell_offsets = _ptr(keep[3], C.c_int64)
    d.cell_nodes = _ptr(keep[4], C.c_int64)
    return d, keep


_INT_ARRAYS = {"edge_v", "edge_c", "edge_bc", "vert_bc", "cell_edges_off", "cell_edges", "vert_cells_off",
               "vert_cells", "vert_cells_ord", "vert_wcells", "cell_verts_off", "cell_verts", "cell_nbrs_off",
               "cell_nbrs"}


class HostMesh:
    """Host-only mesh build (topology, geometry, interpolation weights) in
    reference order; needs no GPU."""

    def __init__(self, msh: str | os.PathLike | None = None, *, desc=None, gpu: bool = False,
                 stream: int | None = None):
        """gpu=True builds the integer topology on the GPU
        (o2f_host_mesh_create_gpu); the result is the same mesh."""
        h = C.c_void_p()
        if msh is not None:
            check(lib().o2f_host_mesh_from_msh(str(msh).encode(), C.byref(h)))
        elif gpu:
            d, self._keep = desc
            check(lib().o2f_host_mesh_create_gpu(C.byref(d), C.c_void_p(stream) if stream else None, C.byref(h)))
        else:
            d, self._keep = desc
            check(lib().o2f_host_mesh_create(C.byref(d), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().o2f_host_mesh_destroy(self._h)
            self._h = None

    def array(self, name: str) -> np.ndarray:
        n = C.c_int64()
        check(lib().o2f_host_mesh_export(self._h, name.encode(), None, C.byref(n)))
        out = np.empty(n.value, dtype=np.int64 if name in _INT_ARRAYS else np.float64)
        check(lib().o2f_host_mesh_export(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), C.byref(n)))
        return out

    def set_coords(self, node_xy: np.ndarray) -> None:
        """New vertex coordinates, same topology (o2f_host_mesh_set_coords)."""
        xy = np.ascontiguousarray(node_xy, dtype=np.float64).reshape(-1)
        if xy.size != self.array("vert_xy").size:
            raise ValueError("node_xy must hold 2 values per vertex")
        check(lib().o2f_host_mesh_set_coords(self._h, _ptr(xy)))


class Solver:
    """A device-resident mesh + state: the counterpart of the reference's
    ``Mesh&`` as seen by the hot-path functions."""

    def __init__(self, params: SimulationParams, msh: str | os.PathLike | None = None, *, desc=None,
                 stream: int | None = None):
        self.params = params
        h = C.c_void_p()
        cp = params.to_c()
        s = C.c_void_p(stream) if stream else None
        if msh is not None:
            check(lib().o2f_create_from_msh(str(msh).encode(), C.byref(cp), s, C.byref(h)))
        else:
            d, self._keep = desc
            check(lib().o2f_create(C.byref(d), C.byref(cp), s, C.byref(h)))
        self._h = h
        info = _lib.MeshInfo()
        check(lib().o2f_get_info(h, C.byref(info)))
        self.n_cells = info.n_cells
        self.n_edges = info.n_edges
        self.n_vertices = info.n_vertices
        self.n_wall_edges = info.n_wall_edges
        self.min_h = info.min_h
        self.device_bytes = info.device_bytes
        self.max_vertex_valence = info.max_vertex_valence

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().o2f_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- configuration / state ------------------------------------------------
    def set_params(self, params: SimulationParams) -> None:
        self.params = params
        cp = params.to_c()
        check(lib().o2f_set_params(self._h, C.byref(cp)))

    def set_state(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
        if U.size != 4 * self.n_cells:
            raise ValueError("state must hold 4 values per cell")
        check(lib().o2f_state_set(self._h, _ptr(U)))

    def set_vertex_coords(self, node_xy: np.ndarray) -> None:
        """New vertex coordinates for the same topology (o2f_set_vertex_coords):
        geometry as a fresh context on them would have, state kept."""
        xy = np.ascontiguousarray(node_xy, dtype=np.float64).reshape(-1)
        if xy.size != 2 * self.n_vertices:
            raise ValueError("node_xy must hold 2 values per vertex")
        check(lib().o2f_set_vertex_coords(self._h, _ptr(xy)))

    def deform_shape(self, frm: _lib.ShapeParams, to: _lib.ShapeParams, power: int = 4) -> None:
        """Move the mesh from shape `frm` to shape `to` (o2f_deform_shape): wall
        by the reference's perturbation formula, interior by inverse distance
        weighting with weights |r|^-power."""
        check(lib().o2f_deform_shape(self._h, C.byref(frm), C.byref(to), int(power)))

    def render_field(self, field: str = "p", nx: int = 512, ny: int = 512, cmap: str = "",
                     vrange: tuple[float, float] | None = None) -> tuple[np.ndarray, tuple[float, float]]:
        """Headless image of a cell field (o2f_render_field): uint8 [ny, nx, 3],
        top row first, and the colour range used."""
        img = np.zeros((int(ny), int(nx), 3), dtype=np.uint8)
        rng_out = np.zeros(2)
        rng_in = None if vrange is None else np.asarray(vrange, dtype=np.float64)
        check(lib().o2f_render_field(self._h, field.encode(), int(nx), int(ny), cmap.encode(),
                                     None if rng_in is None else _ptr(rng_in), _ptr(img, C.c_uint8), _ptr(rng_out)))
        return img, (float(rng_out[0]), float(rng_out[1]))

    def get_state(self) -> np.ndarray:
        U = np.empty(4 * self.n_cells)
        check(lib().o2f_state_get(self._h, _ptr(U)))
        return U

    def initialize_freestream(self) -> None:
        """init_one_x (src/init.cpp:57-81)."""
        check(lib().o2f_state_freestream(self._h))

    def mesh_array(self, name: str) -> np.ndarray:
        n = C.c_int64()
        check(lib().o2f_mesh_export(self._h, name.encode(), None, C.byref(n)))
        out = np.empty(n.value, dtype=np.int64 if name in _INT_ARRAYS else np.float64)
        check(lib().o2f_mesh_export(self._h, name.encode(), out.ctypes.data_as(C.c_void_p), C.byref(n)))
        return out

    # -- hot path -----------------------------------------------------------------
    def compute_residual(self) -> np.ndarray:
        """computeResidual (src/shape_optimization.cpp:171-189)."""
        R = np.empty(4 * self.n_cells)
        check(lib().o2f_residual(self._h, _ptr(R)))
        return R

    def debug(self, name: str) -> np.ndarray:
        sizes = {"R": 4 * self.n_cells, "grad": 8 * self.n_cells, "edge_LR": 8 * self.n_edges,
                 "edge_tau": 3 * self.n_edges, "edge_F": 4 * self.n_edges, "vertex_U": 4 * self.n_vertices}
        out = np.empty(sizes[name])
        check(lib().o2f_debug_get(self._h, name.encode(), _ptr(out)))
        return out

    def time_loop(self, max_steps: int, residual_drop: float = 0.0, raise_on_failure: bool = True) -> dict:
        """Simulator::time_loop (src/simulation.cpp:68-126).  On a non-finite
        state the loop stops; with raise_on_failure=False the steps done and
        the history up to that point are returned with the status."""
        hist = np.zeros(max(int(max_steps), 1))
        steps = C.c_int64()
        t = C.c_double()
        code = lib().o2f_rk3_run(self._h, int(max_steps), float(residual_drop), _ptr(hist), C.byref(steps),
                                 C.byref(t))
        if raise_on_failure:
            check(code)
        return {"steps": steps.value, "t": t.value, "history": hist[: min(steps.value, hist.size)],
                "status": _lib.STATUS.get(code, "OK")}

    def lift_drag(self, beta: float = 1.0) -> tuple[float, float, float]:
        """(C_L, C_D, J): computeLiftDragCoefficients (src/compute.cpp:92-132)
        and computeDirectObjectiveTerm (src/shape_optimization.cpp:893-939)."""
        out = np.empty(3)
        check(lib().o2f_forces(self._h, float(beta), _ptr(out)))
        return float(out[0]), float(out[1]), float(out[2])

    def apply_jacobian_transpose(self, x: np.ndarray) -> np.ndarray:
        """applyJacobianTranspose (src/shape_optimization.cpp:237-484)."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        y = np.empty(4 * self.n_cells)
        check(lib().o2f_jt_apply(self._h, _ptr(x), _ptr(y)))
        return y

    def assemble_adjoint_rhs(self, beta: float = 1.0) -> np.ndarray:
        """assembleAdjointRHS (src/shape_optimization.cpp:491-554)."""
        b = np.empty(4 * self.n_cells)
        check(lib().o2f_adjoint_rhs(self._h, float(beta), _ptr(b)))
        return b

    def solve_adjoint_system(self, beta: float = 1.0, tol: float = 1e-6, max_iter: int = 100000,
                             restart: int = 500, raise_on_failure: bool = True, guess: np.ndarray | None = None) -> dict:
        """solveAdjointSystem (src/shape_optimization.cpp:658-740); `guess`
        (reference order, 4 per cell) replaces the zero initial lambda."""
        lam = np.empty(4 * self.n_cells)
        it = C.c_int64()
        rr = C.c_double()
        if guess is None:
            code = lib().o2f_adjoint_solve(self._h, float(beta), float(tol), int(max_iter), int(restart), _ptr(lam),
                                           C.byref(it), C.byref(rr))
        else:
            g = np.ascontiguousarray(guess, dtype=np.float64).reshape(-1)
            if g.size != 4 * self.n_cells:
                raise ValueError("guess must hold 4 values per cell")
            code = lib().o2f_adjoint_solve_guess(self._h, float(beta), float(tol), int(max_iter), int(restart),
                                                 _ptr(g), _ptr(lam), C.byref(it), C.byref(rr))
        res = {"lambda": lam, "iters": it.value, "relres": rr.value, "status": _lib.STATUS.get(code, "OK")}
        if code != 0 and raise_on_failure:
            check(code)
        return res

    def solve_adjoint_rhs(self, rhs: np.ndarray, tol: float = 1e-6, max_iter: int = 100000, restart: int = 500,
                          guess: np.ndarray | None = None, raise_on_failure: bool = True) -> dict:
        """J^T lambda = rhs with the context's operator (o2f_adjoint_solve_rhs)."""
        b = np.ascontiguousarray(rhs, dtype=np.float64).reshape(-1)
        if b.size != 4 * self.n_cells:
            raise ValueError("rhs must hold 4 values per cell")
        g = None if guess is None else np.ascontiguousarray(guess, dtype=np.float64).reshape(-1)
        lam = np.empty(4 * self.n_cells)
        it = C.c_int64()
        rr = C.c_double()
        code = lib().o2f_adjoint_solve_rhs(self._h, _ptr(b), float(tol), int(max_iter), int(restart),
                                           None if g is None else _ptr(g), _ptr(lam), C.byref(it), C.byref(rr))
        res = {"lambda": lam, "iters": it.value, "relres": rr.value, "status": _lib.STATUS.get(code, "OK")}
        if code != 0 and raise_on_failure:
            check(code)
        return res

    @staticmethod
    def shape_params(names_all: Sequence[str] = (), values_all: Sequence[float] = ()) -> _lib.ShapeParams:
        """Defaults of applyShapePerturbationNACA12 (src/shape_optimization.cpp:830-834)."""
        d = dict(zip(names_all, values_all))
        return _lib.ShapeParams(d.get("pos_x", 0.355), d.get("c", 1.0), d.get("m", 0.02), d.get("p", 0.4),
                                d.get("t", 0.12))

    @staticmethod
    def param_ids(names: Iterable[str]) -> list[int]:
        ids = []
        for n in names:
            if n in ("m", "cambrure"):
                ids.append(_lib.PARAM_M)
            elif n in ("p", "position_cambrure"):
                ids.append(_lib.PARAM_P)
            elif n in ("t", "epaisseur"):
                ids.append(_lib.PARAM_T)
            else:
                raise ValueError(f"shape parameter {n!r} is not handled")
        return ids

    def compute_shape_gradient(self, names: Sequence[str], shape: _lib.ShapeParams, beta: float = 1.0,
                               eps: float = 1e-6, lam: np.ndarray | None = None) -> np.ndarray:
        """computeShapeGradient (src/shape_optimization.cpp:942-1016)."""
        ids = (C.c_int * max(len(names), 1))(*self.param_ids(names))
        g = np.zeros(max(len(names), 1))
        lp = None
        if lam is not None:
            lam = np.ascontiguousarray(lam, dtype=np.float64).reshape(-1)
            lp = _ptr(lam)
        check(lib().o2f_shape_gradient(self._h, C.byref(shape), ids, len(names), float(beta), float(eps), lp,
                                       _ptr(g)))
        return g[: len(names)]

    def optimize_shape(self, names: Sequence[str], shape: _lib.ShapeParams, beta: float = 1.0, eps: float = 1e-6,
                       tol: float = 1e-6) -> dict:
        """optimizeShape (src/shape_optimization.cpp:1022-1067) minus the
        printing and the log file (see write_shape_log)."""
        ids = (C.c_int * max(len(names), 1))(*self.param_ids(names))
        g = np.zeros(max(len(names), 1))
        out = np.zeros(3)
        check(lib().o2f_optimize_shape(self._h, C.byref(shape), ids, len(names), float(beta), float(eps),
                                       float(tol), _ptr(g), _ptr(out)))
        return {"J": float(out[0]), "iters": int(out[1]), "relres": float(out[2]), "grad": g[: len(names)]}

    def perturbed_geometry(self, shape: _lib.ShapeParams, name: str, eps: float, which: str) -> np.ndarray:
        sizes = {"vert_xy": 2 * self.n_vertices, "edge_len": self.n_edges, "edge_n": 2 * self.n_edges,
                 "edge_ctr": 2 * self.n_edges, "cell_vol": self.n_cells, "cell_ctr": 2 * self.n_cells,
                 "vert_w": int(self.mesh_array("vert_w").size)}
        out = np.empty(sizes[which])
        check(lib().o2f_debug_perturbed(self._h, C.byref(shape), self.param_ids([name])[0], float(eps),
                                        which.encode(), _ptr(out)))
        return out

    def profile_kernels(self, reps: int = 20) -> dict:
        """Mean duration (ms) of one launch of each kernel class, CUDA events
        on the context stream."""
        ms = np.zeros(len(_lib.KERNEL_CLASSES))
        check(lib().o2f_profile_kernels(self._h, int(reps), _ptr(ms)))
        return dict(zip(_lib.KERNEL_CLASSES, ms.tolist()))

    def residual_norm_noalloc(self) -> float:
        """||R_rho||_2 of the current state through o2f_residual_norm_noalloc
        (no device allocation on the call; one call at a time per device)."""
        out = C.c_double()
        check(lib().o2f_residual_norm_noalloc(self._h, C.byref(out)))
        return out.value

    def debug_ilu_stall(self, stall: bool, spin_limit: int = 0) -> None:
        """Test hook (o2f_debug_ilu_stall): the solves started afterwards run
        their ILU sweeps with one row that never signals and `spin_limit`
        polls per wait, so a bounded wait runs out; False / 0 restore."""
        check(lib().o2f_debug_ilu_stall(self._h, int(bool(stall)), int(spin_limit)))

    def timing(self) -> dict:
        t = _lib.Timing()
        check(lib().o2f_get_timing(self._h, C.byref(t)))
        return {"residual_ms": t.residual_ms, "kernel_launches": t.kernel_launches}


class Batch:
    """Several Solver contexts of one precision (all FP64 or all FP32)
    advanced together by the batched time loop (o2f_batch_*): one grouped
    launch per phase of each SSP-RK3 step for all candidates, each candidate
    with its own mesh, flow parameters, dt and stop condition, and the same
    states as its own Solver.time_loop.  The contexts must outlive the
    batch."""

    PHASES = ("vertex_state", "cell_gradient", "vertex_visc", "edge_flux", "cell_residual", "wave_speed")

    def __init__(self, solvers: Sequence[Solver]):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        check(lib().o2f_batch_create(arr, len(self.solvers), C.byref(h)))
        self._h = h

    def tune(self, reps: int = 5) -> dict:
        """Autotune block size and entities per thread of every phase."""
        cfg = (C.c_int * (2 * len(self.PHASES)))()
        check(lib().o2f_batch_tune(self._h, int(reps), cfg))
        return {p: (cfg[2 * i], cfg[2 * i + 1]) for i, p in enumerate(self.PHASES)}

    def time_loop(self, max_steps: int, residual_drop: float = 0.0) -> list[dict]:
        n = len(self.solvers)
        steps = (C.c_int64 * n)()
        t = np.zeros(n)
        st = (C.c_int * n)()
        check(lib().o2f_batch_rk3_run(self._h, int(max_steps), float(residual_drop), steps, _ptr(t), st))
        return [{"steps": steps[i], "t": float(t[i]), "status": _lib.STATUS.get(st[i], "OK")} for i in range(n)]

    def launches(self) -> int:
        n = C.c_int64()
        check(lib().o2f_batch_launches(self._h, C.byref(n)))
        return n.value

    def history(self, index: int, count: int) -> np.ndarray:
        out = np.empty(max(int(count), 1))
        check(lib().o2f_batch_history(self._h, int(index), _ptr(out), int(count)))
        return out[: int(count)]

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().o2f_batch_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_shape_log(path: str | os.PathLike, names: Sequence[str], J: float, grad: Sequence[float]) -> None:
    """appendShapeOptLog (src/shape_optimization.cpp:112-145): the file is
    truncated and holds one line `` J=<%.8f> name=<%.6e> ...``."""
    if not path or str(path) == "none":
        return
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as fh:
        fh.write(f" J={J:.8f}" + "".join(f" {n}={g:.6e}" for n, g in zip(names, grad)) + "\n")

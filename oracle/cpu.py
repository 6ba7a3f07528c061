"""Test infrastructure only: ctypes binding of the C oracle (oracle/o2f_oracle.c).

The oracle consumes the mesh in reference order as exported by the product's
host mesh build (whose integer topology the tests pin against the
reference's own Mesh).  All arithmetic is sequential FP64 on the CPU.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "o2f_oracle.c"
LIB = HERE / "_build" / "libo2f_oracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)


class Mesh(C.Structure):
    _fields_ = [("nv", C.c_int64), ("nc", C.c_int64), ("ne", C.c_int64), ("vxy", _dp), ("vbc", _ip),
                ("vert_coff", _ip), ("vert_cells", _ip), ("vert_cells_ord", _ip), ("cell_eoff", _ip),
                ("cell_edges", _ip), ("cell_voff", _ip), ("cell_verts", _ip), ("cvol", _dp), ("cctr", _dp),
                ("edge_v", _ip), ("edge_c", _ip), ("edge_bc", _ip), ("elen", _dp), ("en", _dp), ("ectr", _dp)]


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("viscosity", C.c_double), ("Pr", C.c_double), ("cp", C.c_double),
                ("cfl_number", C.c_double), ("final_time", C.c_double), ("inflow_velocity", C.c_double),
                ("rho_ref", C.c_double), ("p_ref", C.c_double), ("aoa_deg", C.c_double),
                ("limiter_k", C.c_double), ("limiter", C.c_int), ("dt_mode", C.c_int)]


class Shape(C.Structure):
    _fields_ = [("pos_x", C.c_double), ("c", C.c_double), ("m", C.c_double), ("p", C.c_double),
                ("t", C.c_double)]


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc (no FMA contraction, no -march)."""
    if force or not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime,
                                                               (HERE / "o2f_oracle.h").stat().st_mtime):
        LIB.parent.mkdir(exist_ok=True)
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-o", str(LIB),
                        str(SRC), "-lm"], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        h = C.CDLL(str(build()))
        h.o2fo_residual.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, _dp, _dp, _dp, _dp, _dp]
        h.o2fo_forces.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, _dp, C.c_double, _dp]
        h.o2fo_jt.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, _dp, _dp]
        h.o2fo_rhs.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, C.c_double, _dp]
        h.o2fo_march.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, C.c_int64, C.c_double, _dp, _dp, _dp]
        h.o2fo_march.restype = C.c_int64
        h.o2fo_perturb.argtypes = [C.POINTER(Mesh), C.POINTER(Params), C.POINTER(Shape), C.c_int, C.c_double,
                                   C.POINTER(Mesh)]
        h.o2fo_shape_gradient.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, _dp, C.POINTER(Shape),
                                          C.POINTER(C.c_int), C.c_int, C.c_double, C.c_double, _dp]
        h.o2fo_bicgstab.argtypes = [C.POINTER(Mesh), C.POINTER(Params), _dp, _dp, C.c_double, C.c_int64, C.c_int64,
                                    _dp, _ip, _dp]
        h.o2fo_bicgstab.restype = C.c_int
        _lib = h
    return _lib


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """The C oracle bound to one mesh (arrays from a product HostMesh)."""

    def __init__(self, host_mesh, params):
        g = host_mesh.array
        self.arr = {k: np.ascontiguousarray(g(k)) for k in (
            "vert_xy", "vert_bc", "vert_cells_off", "vert_cells", "vert_cells_ord", "cell_edges_off", "cell_edges",
            "cell_verts_off", "cell_verts", "cell_vol", "cell_ctr", "edge_v", "edge_c", "edge_bc", "edge_len",
            "edge_n", "edge_ctr")}
        a = self.arr
        self.nv, self.nc, self.ne = a["vert_xy"].size // 2, a["cell_vol"].size, a["edge_len"].size
        self.m = Mesh(self.nv, self.nc, self.ne, _p(a["vert_xy"]), _p(a["vert_bc"], C.c_int64),
                      _p(a["vert_cells_off"], C.c_int64), _p(a["vert_cells"], C.c_int64),
                      _p(a["vert_cells_ord"], C.c_int64), _p(a["cell_edges_off"], C.c_int64),
                      _p(a["cell_edges"], C.c_int64), _p(a["cell_verts_off"], C.c_int64),
                      _p(a["cell_verts"], C.c_int64), _p(a["cell_vol"]), _p(a["cell_ctr"]),
                      _p(a["edge_v"], C.c_int64), _p(a["edge_c"], C.c_int64), _p(a["edge_bc"], C.c_int64),
                      _p(a["edge_len"]), _p(a["edge_n"]), _p(a["edge_ctr"]))
        self.set_params(params)

    def set_params(self, params) -> None:
        self.p = Params(params.gamma, params.viscosity, params.Pr, params.cp, params.cfl_number, params.final_time,
                        params.inflow_velocity, params.rho_ref, params.p_ref, params.aoa_deg, params.limiter_k,
                        0 if params.limiter.lower() in ("venkatakrishnan", "venkat") else 1,
                        1 if params.dt_mode == "thermal" else 0)

    def residual(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        out = {"R": np.empty(4 * self.nc), "grad": np.empty(8 * self.nc), "edge_LR": np.empty(8 * self.ne),
               "edge_tau": np.empty(3 * self.ne), "vertex_U": np.empty(4 * self.nv)}
        lib().o2fo_residual(C.byref(self.m), C.byref(self.p), _p(U), _p(out["R"]), _p(out["grad"]),
                            _p(out["edge_LR"]), _p(out["edge_tau"]), _p(out["vertex_U"]))
        return out

    def forces(self, LR, tau, beta):
        out = np.empty(3)
        lib().o2fo_forces(C.byref(self.m), C.byref(self.p), _p(LR), _p(tau), float(beta), _p(out))
        return out

    def jt(self, LR, x):
        y = np.empty(4 * self.nc)
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib().o2fo_jt(C.byref(self.m), C.byref(self.p), _p(LR), _p(x), _p(y))
        return y

    def rhs(self, LR, beta):
        b = np.empty(4 * self.nc)
        lib().o2fo_rhs(C.byref(self.m), C.byref(self.p), _p(LR), float(beta), _p(b))
        return b

    def march(self, U, max_steps, drop_tol=0.0):
        U = np.array(U, dtype=np.float64, copy=True)
        dts = np.zeros(max(max_steps, 1))
        hist = np.zeros(max(max_steps, 1))
        t = C.c_double()
        n = lib().o2fo_march(C.byref(self.m), C.byref(self.p), _p(U), int(max_steps), float(drop_tol), _p(dts),
                             _p(hist), C.byref(t))
        return {"U": U, "steps": n, "dt": dts[:n], "history": hist[:n], "t": t.value}

    def perturbed(self, shape, param, eps):
        a = {k: self.arr[k].copy() for k in ("vert_xy", "cell_vol", "cell_ctr", "edge_len", "edge_n", "edge_ctr")}
        out = Mesh.from_buffer_copy(self.m)
        out.vxy, out.cvol, out.cctr = _p(a["vert_xy"]), _p(a["cell_vol"]), _p(a["cell_ctr"])
        out.elen, out.en, out.ectr = _p(a["edge_len"]), _p(a["edge_n"]), _p(a["edge_ctr"])
        s = Shape(shape.pos_x, shape.c, shape.m, shape.p, shape.t)
        lib().o2fo_perturb(C.byref(self.m), C.byref(self.p), C.byref(s), int(param), float(eps), C.byref(out))
        return a

    def shape_gradient(self, U, lam, shape, params, beta, eps=1e-6):
        ids = (C.c_int * len(params))(*params)
        g = np.empty(len(params))
        s = Shape(shape.pos_x, shape.c, shape.m, shape.p, shape.t)
        lib().o2fo_shape_gradient(C.byref(self.m), C.byref(self.p), _p(np.ascontiguousarray(U)),
                                  _p(np.ascontiguousarray(lam)), C.byref(s), ids, len(params), float(beta),
                                  float(eps), _p(g))
        return g

    def bicgstab(self, LR, b, tol, max_iter=100000, restart=500):
        x = np.empty(4 * self.nc)
        it = C.c_int64()
        rr = C.c_double()
        rc = lib().o2fo_bicgstab(C.byref(self.m), C.byref(self.p), _p(LR), _p(b), float(tol), int(max_iter),
                                 int(restart), _p(x), C.byref(it), C.byref(rr))
        return {"lambda": x, "iters": it.value, "relres": rr.value, "converged": rc == 0}

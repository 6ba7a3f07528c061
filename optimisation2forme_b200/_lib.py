"""ctypes binding of ``libo2f.so`` (the C ABI declared in include/o2f.h).

Loading fails loudly when the native library is missing: there is no
Python or CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libo2f.so"

O2F_OK = 0
STATUS = {
    -1: "O2F_ERR_ARG",
    -2: "O2F_ERR_IO",
    -3: "O2F_ERR_MESH",
    -4: "O2F_ERR_CUDA",
    -5: "O2F_ERR_NONFINITE",
    -6: "O2F_ERR_NOT_CONVERGED",
    -7: "O2F_ERR_BREAKDOWN",
    -8: "O2F_ERR_STATE",
    -9: "O2F_ERR_INTERNAL",
}

PREC_F64 = 0
PREC_F32 = 1
LIMITER_VENKAT = 0
LIMITER_BARTH_JESPERSEN = 1
PARAM_M, PARAM_P, PARAM_T = 0, 1, 2


class O2FError(RuntimeError):
    """A non-zero o2f_status, with the library's message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code
        self.status = STATUS.get(code, str(code))


class Params(C.Structure):
    _fields_ = [
        ("gamma", C.c_double),
        ("viscosity", C.c_double),
        ("Pr", C.c_double),
        ("cp", C.c_double),
        ("cfl_number", C.c_double),
        ("final_time", C.c_double),
        ("inflow_velocity", C.c_double),
        ("rho_ref", C.c_double),
        ("p_ref", C.c_double),
        ("aoa_deg", C.c_double),
        ("limiter_k", C.c_double),
        ("adjoint_shift", C.c_double),
        ("limiter", C.c_int),
        ("precision", C.c_int),
        ("adjoint_precond", C.c_int),
        ("dt_mode", C.c_int),
        ("verbosity", C.c_int),
        ("adjoint_jacobian", C.c_int),
        ("adjoint_fd_step", C.c_double),
        ("adjoint_precision", C.c_int),
        ("adjoint_sweeps", C.c_int),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int64),
        ("node_xy", C.POINTER(C.c_double)),
        ("n_segments", C.c_int64),
        ("segments", C.POINTER(C.c_int64)),
        ("segment_bc", C.POINTER(C.c_uint8)),
        ("n_cells", C.c_int64),
        ("cell_offsets", C.POINTER(C.c_int64)),
        ("cell_nodes", C.POINTER(C.c_int64)),
    ]


class MeshInfo(C.Structure):
    _fields_ = [
        ("n_cells", C.c_int64),
        ("n_edges", C.c_int64),
        ("n_vertices", C.c_int64),
        ("n_wall_edges", C.c_int64),
        ("n_boundary_edges", C.c_int64),
        ("max_vertex_valence", C.c_int64),
        ("min_h", C.c_double),
        ("device_bytes", C.c_size_t),
    ]


class ShapeParams(C.Structure):
    _fields_ = [("pos_x", C.c_double), ("c", C.c_double), ("m", C.c_double), ("p", C.c_double),
                ("t", C.c_double)]


class Timing(C.Structure):
    _fields_ = [("residual_ms", C.c_double), ("kernel_launches", C.c_int64)]


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int64)
_vp = C.c_void_p
_fp = C.POINTER(C.c_float)

# name -> (argtypes); every function returns int except noted.
SIGNATURES = {
    "o2f_last_error": ([], C.c_char_p),
    "o2f_version": ([], C.c_char_p),
    "o2f_params_default": ([C.POINTER(Params)], None),
    "o2f_host_mesh_create": ([C.POINTER(MeshDesc), C.POINTER(_vp)], C.c_int),
    "o2f_host_mesh_from_msh": ([C.c_char_p, C.POINTER(_vp)], C.c_int),
    "o2f_host_mesh_create_gpu": ([C.POINTER(MeshDesc), _vp, C.POINTER(_vp)], C.c_int),
    "o2f_host_mesh_export": ([_vp, C.c_char_p, _vp, _ip], C.c_int),
    "o2f_host_mesh_destroy": ([_vp], C.c_int),
    "o2f_create": ([C.POINTER(MeshDesc), C.POINTER(Params), _vp, C.POINTER(_vp)], C.c_int),
    "o2f_create_from_msh": ([C.c_char_p, C.POINTER(Params), _vp, C.POINTER(_vp)], C.c_int),
    "o2f_destroy": ([_vp], C.c_int),
    "o2f_set_params": ([_vp, C.POINTER(Params)], C.c_int),
    "o2f_get_info": ([_vp, C.POINTER(MeshInfo)], C.c_int),
    "o2f_mesh_export": ([_vp, C.c_char_p, _vp, _ip], C.c_int),
    "o2f_state_set": ([_vp, _dp], C.c_int),
    "o2f_state_get": ([_vp, _dp], C.c_int),
    "o2f_state_freestream": ([_vp], C.c_int),
    "o2f_residual": ([_vp, _dp], C.c_int),
    "o2f_debug_get": ([_vp, C.c_char_p, _dp], C.c_int),
    "o2f_rk3_run": ([_vp, C.c_int64, C.c_double, _dp, _ip, _dp], C.c_int),
    "o2f_forces": ([_vp, C.c_double, _dp], C.c_int),
    "o2f_jt_apply": ([_vp, _dp, _dp], C.c_int),
    "o2f_adjoint_rhs": ([_vp, C.c_double, _dp], C.c_int),
    "o2f_adjoint_solve": ([_vp, C.c_double, C.c_double, C.c_int64, C.c_int64, _dp, _ip, _dp], C.c_int),
    "o2f_shape_gradient": ([_vp, C.POINTER(ShapeParams), C.POINTER(C.c_int), C.c_int, C.c_double, C.c_double, _dp,
                            _dp], C.c_int),
    "o2f_optimize_shape": ([_vp, C.POINTER(ShapeParams), C.POINTER(C.c_int), C.c_int, C.c_double, C.c_double,
                            C.c_double, _dp, _dp], C.c_int),
    "o2f_debug_perturbed": ([_vp, C.POINTER(ShapeParams), C.c_int, C.c_double, C.c_char_p, _dp], C.c_int),
    "o2f_state_device": ([_vp, C.POINTER(_dp)], C.c_int),
    "o2f_cell_permutation": ([_vp, _ip], C.c_int),
    "o2f_get_timing": ([_vp, C.POINTER(Timing)], C.c_int),
    "o2f_profile_kernels": ([_vp, C.c_int, _dp], C.c_int),
    "o2f_residual_norm_noalloc": ([_vp, _dp], C.c_int),
    "o2f_debug_ilu_stall": ([_vp, C.c_int, C.c_int64], C.c_int),
    "o2f_hllc_flux": ([C.c_int64, _dp, _dp, C.c_double, _dp], C.c_int),
    "o2f_bc_states": ([C.POINTER(Params), C.c_int64, C.POINTER(C.c_uint8), _dp], C.c_int),
    "o2f_bc_ghosts": ([C.POINTER(Params), C.c_int64, C.POINTER(C.c_uint8), _dp, _dp], C.c_int),
    "o2f_bc_diffusion": ([C.c_int64, C.POINTER(C.c_uint8), _dp], C.c_int),
    "o2f_host_mesh_set_coords": ([_vp, _dp], C.c_int),
    "o2f_checkpoint_write": ([C.c_char_p, C.c_int64, _dp, C.c_double, C.c_int64], C.c_int),
    "o2f_checkpoint_read": ([C.c_char_p, C.c_int64, _dp, _dp, C.POINTER(C.c_int64)], C.c_int),
    "o2f_set_vertex_coords": ([_vp, _dp], C.c_int),
    "o2f_deform_shape": ([_vp, C.POINTER(ShapeParams), C.POINTER(ShapeParams), C.c_int], C.c_int),
    "o2f_render_field": ([_vp, C.c_char_p, C.c_int, C.c_int, C.c_char_p, _dp, C.POINTER(C.c_uint8), _dp], C.c_int),
    "o2f_batch_create": ([C.POINTER(_vp), C.c_int, C.POINTER(_vp)], C.c_int),
    "o2f_adjoint_solve_rhs": ([_vp, _dp, C.c_double, C.c_int64, C.c_int64, _dp, _dp, C.POINTER(C.c_int64), _dp],
                              C.c_int),
    "o2f_adjoint_solve_guess": ([_vp, C.c_double, C.c_double, C.c_int64, C.c_int64, _dp, _dp, C.POINTER(C.c_int64),
                                 _dp], C.c_int),
    "o2f_mlp_create": ([C.c_int, C.c_float, C.c_uint64, _vp, C.POINTER(_vp)], C.c_int),
    "o2f_mlp_destroy": ([_vp], C.c_int),
    "o2f_mlp_n_params": ([_vp, C.POINTER(C.c_int64)], C.c_int),
    "o2f_mlp_set_data": ([_vp, _fp, _fp, C.c_int64], C.c_int),
    "o2f_mlp_train": ([_vp, C.c_int, C.c_int, C.c_float, C.c_uint64, _fp], C.c_int),
    "o2f_mlp_predict": ([_vp, _fp, C.c_int64, _fp], C.c_int),
    "o2f_mlp_gradients": ([_vp, _fp, _fp, C.c_int, _fp, _fp], C.c_int),
    "o2f_mlp_get_params": ([_vp, _fp, _fp], C.c_int),
    "o2f_mlp_set_params": ([_vp, _fp], C.c_int),
    "o2f_batch_destroy": ([_vp], C.c_int),
    "o2f_batch_tune": ([_vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "o2f_batch_rk3_run": ([_vp, C.c_int64, C.c_double, C.POINTER(C.c_int64), _dp, C.POINTER(C.c_int)], C.c_int),
    "o2f_batch_history": ([_vp, C.c_int, _dp, C.c_int64], C.c_int),
    "o2f_batch_launches": ([_vp, C.POINTER(C.c_int64)], C.c_int),
}

KERNEL_CLASSES = ["vertex_state", "cell_gradient", "vertex_visc", "edge_flux", "cell_residual", "jt_apply",
                  "jt_blocks"]

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"native library {LIB_PATH} is missing: run `python -m optimisation2forme_b200.build`")
        h = C.CDLL(str(LIB_PATH))
        for name, (args, res) in SIGNATURES.items():
            f = getattr(h, name)
            f.argtypes = args
            f.restype = res
        _lib = h
    return _lib


def check(code: int) -> None:
    if code != O2F_OK:
        raise O2FError(code, lib().o2f_last_error().decode(errors="replace"))

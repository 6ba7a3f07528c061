"""B200 implementation of the shape-gradient hot path of a 2-D compressible
Navier-Stokes adjoint shape optimiser (ThibaultMaurelOujia/Optimisation2Forme).

The compute lives in the native library ``libo2f.so`` (C ABI in
``include/o2f.h``, CUDA kernels for sm_100a); this package is the host-side
binding.  Importing works without a GPU; creating a ``Solver`` needs one.
"""
from ._lib import LIB_PATH, O2FError, lib
from .solver import (Batch, HostMesh, SimulationParams, Solver, load_cell_states, load_config, load_params_generic,
                     load_state_binary, mesh_desc, save_cell_states, save_state_binary, write_image,
                     write_shape_log)

__all__ = ["LIB_PATH", "O2FError", "lib", "Batch", "HostMesh", "SimulationParams", "Solver", "load_cell_states",
           "load_config", "load_params_generic", "load_state_binary", "mesh_desc", "save_cell_states",
           "save_state_binary", "write_image", "write_shape_log"]

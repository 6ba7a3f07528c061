"""Array entry points of the reference's per-edge / per-state functions:
o2f_hllc_flux on the interface states a residual left reproduces that
residual's edge fluxes bit for bit; o2f_bc_states / o2f_bc_ghosts /
o2f_bc_diffusion against a restatement of src/boundary.cpp:7-127."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import bits_equal, desc_of, perturbed_freestream, small_mesh

pytestmark = pytest.mark.gpu

CODES = np.array([ord("i"), ord("o"), ord("f"), ord("w"), 0, ord("x")], dtype=np.uint8)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _bp(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def test_hllc_flux_array_equals_the_residual_fluxes():
    from optimisation2forme_b200 import SimulationParams, Solver
    from optimisation2forme_b200._lib import check, lib
    p = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, limiter_k=5.0, verbosity=0)
    with Solver(p, desc=desc_of(small_mesh(triangles=True, n_surface=64, n_layers=16, seed=5))) as s:
        s.set_state(perturbed_freestream(s.n_cells, p, seed=2))
        s.compute_residual()
        LR = np.ascontiguousarray(s.debug("edge_LR"))
        F = s.debug("edge_F")
        n = np.ascontiguousarray(s.mesh_array("edge_n"))
        out = np.empty(4 * s.n_edges)
        check(lib().o2f_hllc_flux(s.n_edges, _dp(LR), _dp(n), p.gamma, _dp(out)))
        assert bits_equal(out, F)


def _reference_bc(code, q, fs):
    rho, ru, rv, E = q
    if code in (ord("i"), ord("f")):
        return list(fs)
    if code == ord("w"):
        kinetic_old = 0.5 * (ru * ru + rv * rv) / rho
        return [rho, 0.0, 0.0, E - kinetic_old]
    return [rho, ru, rv, E]


def test_boundary_function_arrays_against_the_reference_formulas():
    from optimisation2forme_b200 import SimulationParams
    from optimisation2forme_b200._lib import check, lib
    p = SimulationParams(inflow_velocity=0.6)
    cp = p.to_c()
    g, rho0, p0 = p.gamma, p.rho_ref, p.p_ref
    u0 = p.inflow_velocity * np.sqrt(g * p0 / rho0)
    fs = [rho0, rho0 * u0, rho0 * 0.0, p0 / (g - 1.0) + 0.5 * rho0 * (u0 * u0 + 0.0 * 0.0)]
    n = CODES.size
    U = np.tile([1.1, 250.0, -12.0, 2.6e5], n).astype(np.float64)
    got = U.copy()
    check(lib().o2f_bc_states(C.byref(cp), n, _bp(CODES), _dp(got)))
    ref = np.array([_reference_bc(int(c), U[4 * k:4 * k + 4], fs) for k, c in enumerate(CODES)]).reshape(-1)
    assert bits_equal(got, ref)
    R = np.empty(4 * n)
    check(lib().o2f_bc_ghosts(C.byref(cp), n, _bp(CODES), _dp(U), _dp(R)))
    for k, c in enumerate(CODES):
        L = U[4 * k:4 * k + 4]
        if c in (ord("i"), ord("o"), ord("f")):
            exp = _reference_bc(int(c), L, fs)
        elif c == ord("w"):
            exp = [L[0], -L[1], -L[2], L[3]]
        else:
            exp = list(L)
        assert bits_equal(R[4 * k:4 * k + 4], np.array(exp)), chr(c) if c else "0"
    T = np.tile([1.5, -2.5, 3.5, -4.5, 5.5], n).astype(np.float64)
    check(lib().o2f_bc_diffusion(n, _bp(CODES), _dp(T)))
    for k, c in enumerate(CODES):
        exp = np.zeros(5) if c in (ord("f"), ord("w")) else np.array([1.5, -2.5, 3.5, -4.5, 5.5])
        assert bits_equal(T[5 * k:5 * k + 5], exp)

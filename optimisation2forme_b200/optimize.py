"""In-process shape-optimisation loop: the reference's outer loop
(mesh_opti/run_opti.sh) without restarting the solver or re-meshing with
Gmsh between iterations.

Per iteration, as in the reference: march the flow of the current shape from
the previous iteration's state (run_opti.sh rewrites state_load_path to the
last saved flow), compute J, the adjoint and dJ/d(m, p), then move m and p by
fixed steps against the sign of their gradients, clamped
(run_opti.sh:6-14, 114-131).  The mesh of the new shape has the topology of
the first one, so the state and the adjoint carry over cell by cell; the
adjoint of each iteration starts from the previous lambda (a warm start that
the plain BiCGSTAB then converges from, to the same tolerance).  The mesh of
the new shape comes either from the seeded O-grid generator (regenerate: a
new context per iteration) or from moving the current mesh on the GPU
(deform: one context for the whole loop, wall by the perturbation formula,
interior by inverse distance weighting; the state never leaves the device).
"""
from __future__ import annotations

import dataclasses
from typing import Sequence

import numpy as np

from .meshgen import OGridSpec, naca_ogrid
from .solver import SimulationParams, Solver, mesh_desc


@dataclasses.dataclass
class SignDescent:
    """The reference's update rule (run_opti.sh:6-14)."""
    step_m: float = 0.002
    step_p: float = 0.01
    m_min: float = 0.0
    m_max: float = 0.12
    p_min: float = 1e-3
    p_max: float = 0.999

    def step(self, m: float, p: float, grad_m: float, grad_p: float) -> tuple[float, float]:
        """dJ/dtheta < 0 -> increase theta, otherwise decrease it (a zero
        gradient decreases it too, as in run_opti.sh:116-117); clamp; keep 8
        decimals as the reference's printf("%.8f")."""
        s_m = 1.0 if grad_m < 0 else -1.0
        s_p = 1.0 if grad_p < 0 else -1.0
        m_new = min(max(m + s_m * self.step_m, self.m_min), self.m_max)
        p_new = min(max(p + s_p * self.step_p, self.p_min), self.p_max)
        return float(f"{m_new:.8f}"), float(f"{p_new:.8f}")


def optimise(spec: OGridSpec, params: SimulationParams, iterations: int, rk_steps: int, beta: float = 50.0,
             rule: SignDescent | None = None, warm_adjoint: bool = True, tol: float = 1e-6,
             max_iter: int = 100000, stream: int | None = None, mesh_update: str = "regenerate",
             idw_power: int = 4) -> list[dict]:
    """Run `iterations` steps of the loop from spec's (m, p); returns one
    record per iteration: m, p, J, C_L, C_D, dJ/dm, dJ/dp, adjoint
    iterations and relres, time-loop steps.  mesh_update: "regenerate" or
    "deform" (see the module docstring)."""
    if mesh_update == "deform":
        return _optimise_deform(spec, params, iterations, rk_steps, beta, rule or SignDescent(), warm_adjoint, tol,
                                max_iter, stream, idw_power)
    if mesh_update != "regenerate":
        raise ValueError("mesh_update must be 'regenerate' or 'deform'")
    rule = rule or SignDescent()
    m, p = spec.m, spec.p
    U = lam = None
    cells = None
    history = []
    for k in range(iterations):
        mesh = naca_ogrid(dataclasses.replace(spec, m=m, p=p))
        with Solver(params, desc=mesh_desc(mesh["node_xy"], mesh["segments"], mesh["segment_bc"],
                                           mesh["cell_offsets"], mesh["cell_nodes"]), stream=stream) as s:
            if cells is not None and s.n_cells != cells:
                raise RuntimeError("the mesh topology changed between iterations")
            cells = s.n_cells
            if U is None:
                s.initialize_freestream()
            else:
                s.set_state(U)
            run = s.time_loop(rk_steps)
            C_L, C_D, J = s.lift_drag(beta)
            adj = s.solve_adjoint_system(beta, tol=tol, max_iter=max_iter, raise_on_failure=False,
                                         guess=lam if (warm_adjoint and lam is not None) else None)
            shape = Solver.shape_params(["pos_x", "c", "m", "p", "t"], [spec.pos_x, spec.chord, m, p, spec.t])
            g = s.compute_shape_gradient(["m", "p"], shape, beta=beta, lam=adj["lambda"])
            U = s.get_state()
            lam = adj["lambda"] if adj["status"] == "OK" else None
        history.append({"iteration": k, "m": m, "p": p, "J": J, "C_L": C_L, "C_D": C_D, "dJ_dm": float(g[0]),
                        "dJ_dp": float(g[1]), "adjoint_iters": adj["iters"], "adjoint_relres": adj["relres"],
                        "adjoint_status": adj["status"], "steps": run["steps"]})
        m, p = rule.step(m, p, float(g[0]), float(g[1]))
    return history


def _optimise_deform(spec, params, iterations, rk_steps, beta, rule, warm_adjoint, tol, max_iter, stream,
                     idw_power) -> list[dict]:
    m, p = spec.m, spec.p
    mesh = naca_ogrid(spec)
    history = []
    lam = None

    def shape(m_, p_):
        return Solver.shape_params(["pos_x", "c", "m", "p", "t"], [spec.pos_x, spec.chord, m_, p_, spec.t])

    with Solver(params, desc=mesh_desc(mesh["node_xy"], mesh["segments"], mesh["segment_bc"],
                                       mesh["cell_offsets"], mesh["cell_nodes"]), stream=stream) as s:
        s.initialize_freestream()
        for k in range(iterations):
            run = s.time_loop(rk_steps)
            C_L, C_D, J = s.lift_drag(beta)
            adj = s.solve_adjoint_system(beta, tol=tol, max_iter=max_iter, raise_on_failure=False,
                                         guess=lam if (warm_adjoint and lam is not None) else None)
            g = s.compute_shape_gradient(["m", "p"], shape(m, p), beta=beta, lam=adj["lambda"])
            lam = adj["lambda"] if adj["status"] == "OK" else None
            history.append({"iteration": k, "m": m, "p": p, "J": J, "C_L": C_L, "C_D": C_D, "dJ_dm": float(g[0]),
                            "dJ_dp": float(g[1]), "adjoint_iters": adj["iters"], "adjoint_relres": adj["relres"],
                            "adjoint_status": adj["status"], "steps": run["steps"]})
            m_new, p_new = rule.step(m, p, float(g[0]), float(g[1]))
            if k + 1 < iterations:
                s.deform_shape(shape(m, p), shape(m_new, p_new), power=idw_power)
            m, p = m_new, p_new
    return history


def write_history(path, history: Sequence[dict]) -> None:
    """One line per iteration, in the spirit of the reference's shape logs."""
    with open(path, "w") as fh:
        for h in history:
            fh.write(f"{h['iteration']} m={h['m']:.8f} p={h['p']:.8f} J={h['J']:.8f} dJ/dm={h['dJ_dm']:.6e} "
                     f"dJ/dp={h['dJ_dp']:.6e} adjoint_iters={h['adjoint_iters']}\n")

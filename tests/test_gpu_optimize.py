"""The in-process shape-optimisation loop on the GPU: the reference's update
rule applied to the computed gradients, converged adjoints, and the warm
start from the previous iteration's lambda changing nothing but the
iteration count."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sign_descent_loop_with_carried_state_and_adjoint():
    from optimisation2forme_b200 import SimulationParams
    from optimisation2forme_b200.meshgen import OGridSpec
    from optimisation2forme_b200.optimize import SignDescent, optimise
    spec = OGridSpec(m=0.02, p=0.4, t=0.12, n_surface=48, n_layers=12, triangles=True, seed=2)
    params = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0,
                              limiter_k=5.0, verbosity=0)
    warm = optimise(spec, params, iterations=4, rk_steps=100, beta=0.1, tol=1e-8)
    cold = optimise(spec, params, iterations=4, rk_steps=100, beta=0.1, tol=1e-8, warm_adjoint=False)
    rule = SignDescent()
    for a, b in zip(warm, warm[1:]):
        assert (b["m"], b["p"]) == rule.step(a["m"], a["p"], a["dJ_dm"], a["dJ_dp"])
    for w, c in zip(warm, cold):
        assert w["adjoint_status"] == "OK" and c["adjoint_status"] == "OK"
        assert (w["m"], w["p"], w["J"]) == (c["m"], c["p"], c["J"])  # same shapes, same states
        for key in ("dJ_dm", "dJ_dp"):
            assert abs(w[key] - c[key]) <= 1e-5 * max(abs(c[key]), 1e-12)
    wi, ci = [h["adjoint_iters"] for h in warm], [h["adjoint_iters"] for h in cold]
    print(f"\nouter loop: J {[round(h['J'], 6) for h in warm]}; adjoint iterations warm {wi} cold {ci}")
    assert wi[0] == ci[0]
    assert np.all(np.isfinite([h["J"] for h in warm]))

"""The outer loop's update rule, the reference's fixed-step sign descent
(mesh_opti/run_opti.sh:6-14, 114-131)."""
from __future__ import annotations

from optimisation2forme_b200.optimize import SignDescent


def test_steps_against_the_gradient_sign():
    r = SignDescent()
    assert r.step(0.02, 0.4, -1.0, 2.0) == (0.022, 0.39)
    assert r.step(0.02, 0.4, 3.0, -0.5) == (0.018, 0.41)


def test_zero_gradient_decreases_like_the_reference():
    # m = 0 makes dJ/dp exactly zero (no camber): the reference then lowers p
    assert SignDescent().step(0.0, 0.4, -1.0, 0.0) == (0.002, 0.39)


def test_clamps_and_eight_decimals():
    r = SignDescent()
    assert r.step(0.0, 0.0015, 1.0, 1.0) == (0.0, 0.001)
    assert r.step(0.1195, 0.995, -1.0, -1.0) == (0.12, 0.999)
    m, p = r.step(0.0123456789, 0.5, -1.0, 1.0)
    assert m == 0.01434568 and p == 0.49

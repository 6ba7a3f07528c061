"""Host logic of bench.py (no GPU): the seeded candidate set, the byte
models of the roofline and the projection of the reference's reduced
evaluation."""
from __future__ import annotations

import numpy as np


def test_candidate_set_is_seeded_and_sized():
    import bench
    a = bench.candidate_set(4, 7, 20_000, 60_000, 1e-3)
    b = bench.candidate_set(4, 7, 20_000, 60_000, 1e-3)
    for x, y in zip(a, b):
        assert x.spec == y.spec and x.mach == y.mach and x.aoa == y.aoa
        np.testing.assert_array_equal(x.mesh["node_xy"], y.mesh["node_xy"])
    for c in a:
        cells = c.mesh["cell_offsets"].size - 1
        assert 0.8 * 20_000 <= cells <= 1.2 * 60_000
        assert 0.0 <= c.spec.m <= 0.06 and 0.2 <= c.spec.p <= 0.6 and 0.08 <= c.spec.t <= 0.18
        assert 0.5 <= c.mach <= 0.8 and 0.0 <= c.aoa <= 4.0


def test_byte_models():
    import bench
    nc, ne, nv, nnz = 2007720, 3012984, 1003860, 6023160
    kb = bench.kernel_bytes(nc, ne, nv, nnz)
    assert kb["cell_gradient"] == nc * 120 + ne * 129 + nv * 32
    assert bench.residual_bytes(nc, ne, nv, nnz) == nc * 88 + ne * 56 + nv * 4 + nnz * 12
    assert bench.residual_bytes(nc, ne, nv, nnz, w=4) < bench.residual_bytes(nc, ne, nv, nnz)


def test_reference_projection():
    import bench
    r = {"steps": 20, "steps_s": 2.0, "iters": 10, "bicgstab_s": 0.5, "objective_s": 0.01, "gradient_s": 0.3}
    assert abs(bench.projected_eval_s(r, 2000, 400) - (200.0 + 20.0 + 0.31)) < 1e-9

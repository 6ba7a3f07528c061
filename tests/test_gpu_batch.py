"""Batched time loop (o2f_batch_*): several candidates with uneven meshes and
their own flow parameters advanced by grouped launches.  Each candidate's FP64
state must be bit-identical to the same context advanced alone."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import bits_equal, desc_of, small_mesh

pytestmark = pytest.mark.gpu


def _params(**kw):
    from optimisation2forme_b200 import SimulationParams
    d = dict(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0, limiter_k=5.0,
             verbosity=0)
    d.update(kw)
    return SimulationParams(**d)


CANDIDATES = [
    (dict(triangles=True, n_surface=48, n_layers=12, seed=1, m=0.0, p=0.4, t=0.12), dict(inflow_velocity=0.5)),
    (dict(triangles=False, n_surface=64, n_layers=16, seed=2, m=0.02, p=0.4, t=0.10),
     dict(inflow_velocity=0.7, aoa_deg=3.0)),
    (dict(triangles=True, n_surface=96, n_layers=24, seed=3, m=0.04, p=0.3, t=0.15),
     dict(inflow_velocity=0.6, aoa_deg=0.5, limiter="barth_jespersen")),
]


def _contexts():
    from optimisation2forme_b200 import Solver
    return [Solver(_params(**pk), desc=desc_of(small_mesh(**mk))) for mk, pk in CANDIDATES]


def _single_runs(steps, **override):
    out = []
    for s in _contexts():
        with s:
            if override:
                s.set_params(dataclasses.replace(s.params, **override))
            s.initialize_freestream()
            r = s.time_loop(steps)
            out.append((s.get_state(), r, s.lift_drag(0.1)))
    return out


def test_batched_time_loop_is_bit_identical_to_single_contexts():
    from optimisation2forme_b200 import Batch
    ref = _single_runs(40)
    ctxs = _contexts()
    try:
        for s in ctxs:
            s.initialize_freestream()
        with Batch(ctxs) as b:
            res = b.time_loop(40)
            for i, s in enumerate(ctxs):
                U, r, forces = ref[i]
                assert res[i]["status"] == "OK" and res[i]["steps"] == r["steps"] == 40
                assert res[i]["t"] == r["t"]
                assert bits_equal(s.get_state(), U)
                # interface states of the last stage are left in the context
                assert s.lift_drag(0.1) == forces
                h = b.history(i, 40)
                np.testing.assert_allclose(h, r["history"], rtol=1e-13)
    finally:
        for s in ctxs:
            s.close()


def test_tuned_batch_keeps_the_states():
    from optimisation2forme_b200 import Batch
    ref = _single_runs(25)
    ctxs = _contexts()
    try:
        with Batch(ctxs) as b:
            cfg = b.tune(reps=3)
            assert set(cfg) == set(Batch.PHASES)
            for block, tile in cfg.values():
                assert block in (128, 256, 512) and tile in (1, 2, 4)
            for s in ctxs:
                s.initialize_freestream()
            res = b.time_loop(25)
            for i, s in enumerate(ctxs):
                assert res[i]["steps"] == 25
                assert bits_equal(s.get_state(), ref[i][0])
    finally:
        for s in ctxs:
            s.close()


def test_candidates_stop_independently():
    from optimisation2forme_b200 import Batch
    ctxs = _contexts()
    try:
        # the second candidate reaches its final time after a few steps
        s1 = ctxs[1]
        s1.initialize_freestream()
        probe = s1.time_loop(1)
        s1.set_params(dataclasses.replace(s1.params, final_time=3.5 * probe["t"]))
        for s in ctxs:
            s.initialize_freestream()
        with Batch(ctxs) as b:
            res = b.time_loop(30)
        single = _contexts()[1]
        with single:
            single.set_params(dataclasses.replace(single.params, final_time=3.5 * probe["t"]))
            single.initialize_freestream()
            r = single.time_loop(30)
            assert 2 <= r["steps"] < 30
            assert [x["steps"] for x in res] == [30, r["steps"], 30]
            assert bits_equal(single.get_state(), s1.get_state())
    finally:
        for s in ctxs:
            s.close()


def test_poisoned_candidate_fails_alone():
    """A non-finite state in one candidate stops that candidate with
    O2F_ERR_NONFINITE; the others run their steps, bit-identical to their
    own single-context runs, and the batch stays usable."""
    from optimisation2forme_b200 import Batch
    ref = _single_runs(30)
    ctxs = _contexts()
    try:
        for s in ctxs:
            s.initialize_freestream()
        U = ctxs[1].get_state()
        U[4 * 5 + 1] = np.nan
        ctxs[1].set_state(U)
        with Batch(ctxs) as b:
            res = b.time_loop(30)
            assert res[1]["status"] == "O2F_ERR_NONFINITE" and res[1]["steps"] < 30
            for i in (0, 2):
                assert res[i]["status"] == "OK" and res[i]["steps"] == 30
                assert bits_equal(ctxs[i].get_state(), ref[i][0])
            # the batch runs again once the candidate has a finite state
            ctxs[1].initialize_freestream()
            for i in (0, 2):
                ctxs[i].initialize_freestream()
            again = b.time_loop(30)
            assert all(r["status"] == "OK" and r["steps"] == 30 for r in again)
            assert bits_equal(ctxs[1].get_state(), ref[1][0])
    finally:
        for s in ctxs:
            s.close()


def test_batched_mixed_precision_is_bit_identical_to_single_fp32_contexts():
    """A batch of FP32 (mixed-precision) contexts: the grouped FP32 residual
    phases advance every candidate exactly as its own context's FP32 time
    loop, and leave the same FP64 linearisation (forces, adjoint RHS)."""
    from optimisation2forme_b200 import Batch, Solver
    ref = []
    for mk, pk in CANDIDATES:
        with Solver(_params(precision="fp32", **pk), desc=desc_of(small_mesh(**mk))) as s:
            s.initialize_freestream()
            r = s.time_loop(30)
            ref.append((s.get_state(), r, s.lift_drag(0.1), s.assemble_adjoint_rhs(0.1)))
    ctxs = [Solver(_params(precision="fp32", **pk), desc=desc_of(small_mesh(**mk))) for mk, pk in CANDIDATES]
    try:
        for s in ctxs:
            s.initialize_freestream()
        with Batch(ctxs) as b:
            b.tune(reps=2)
            for s in ctxs:
                s.initialize_freestream()
            res = b.time_loop(30)
            assert b.launches() > 0
            for i, s in enumerate(ctxs):
                U, r, forces, rhs = ref[i]
                assert res[i]["status"] == "OK" and res[i]["steps"] == r["steps"] == 30
                assert res[i]["t"] == r["t"]
                assert bits_equal(s.get_state(), U)
                assert s.lift_drag(0.1) == forces
                assert bits_equal(s.assemble_adjoint_rhs(0.1), rhs)
    finally:
        for s in ctxs:
            s.close()


def test_batch_rejects_mixed_precisions():
    from optimisation2forme_b200 import Batch, O2FError, Solver
    (mk0, pk0), (mk1, pk1) = CANDIDATES[0], CANDIDATES[1]
    with Solver(_params(**pk0), desc=desc_of(small_mesh(**mk0))) as a, \
            Solver(_params(precision="fp32", **pk1), desc=desc_of(small_mesh(**mk1))) as b:
        with pytest.raises(O2FError):
            Batch([a, b])


def test_concurrent_adjoints_on_own_streams_equal_sequential_ones():
    """Adjoint solves and shape gradients of several contexts run at once
    from host threads, each context on its own stream (as the fast path runs
    its candidates' adjoints): every result equals the same context's solve
    run alone, bit for bit."""
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from optimisation2forme_b200 import Solver
    streams = [torch.cuda.Stream() for _ in CANDIDATES]
    ctxs = [Solver(_params(adjoint_precision="fp32", **pk), desc=desc_of(small_mesh(**mk)), stream=st.cuda_stream)
            for (mk, pk), st in zip(CANDIDATES, streams)]

    def run(s):
        s.initialize_freestream()
        s.time_loop(40)
        a = s.solve_adjoint_system(0.1, tol=1e-9, max_iter=5000, restart=500)
        g = s.compute_shape_gradient(["m", "p", "t"], Solver.shape_params(), beta=0.1)
        return a["lambda"], a["iters"], g

    try:
        alone = [run(s) for s in ctxs]
        with ThreadPoolExecutor(max_workers=len(ctxs)) as ex:
            together = list(ex.map(run, ctxs))
        for (l0, i0, g0), (l1, i1, g1) in zip(alone, together):
            assert i0 == i1
            assert bits_equal(l0, l1)
            assert bits_equal(g0, g1)
    finally:
        for s in ctxs:
            s.close()

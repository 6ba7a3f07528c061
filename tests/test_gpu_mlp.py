"""Warm-start network on the tensor cores (tcgen05 GEMMs, BF16 operands, FP32
accumulation) against the numpy oracle, its training, and the warm start:
BiCGSTAB started from the predicted adjoint reaches the same true-residual
tolerance and the same lambda as from zero (the plain solver checks the
prediction), and the test reports both iteration counts."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import desc_of, small_mesh
from oracle import mlp_ref

pytestmark = pytest.mark.gpu

TOL_FORWARD = 2e-2   # ||y_gpu - y_oracle|| / ||y_oracle||: BF16 ties, FP32 vs FP64 accumulation
TOL_GRAD = 3e-2      # per layer, same norm


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.empty((n, 7), dtype=np.float32)
    x[:, 0] = rng.uniform(-2, 3, n)
    x[:, 1] = rng.uniform(-2, 2, n)
    x[:, 2] = rng.uniform(0, 0.06, n)
    x[:, 3] = rng.uniform(0.2, 0.6, n)
    x[:, 4] = rng.uniform(0.08, 0.18, n)
    x[:, 5] = rng.uniform(0.5, 0.8, n)
    x[:, 6] = rng.uniform(0, 4, n)
    return x


def _layer_slices():
    ins, outs = mlp_ref.dims()
    off, out = 0, []
    for i, o in zip(ins, outs):
        out.append(slice(off, off + o * i))
        off += o * i
        out.append(slice(off, off + o))
        off += o
    return out


def test_forward_matches_oracle():
    from optimisation2forme_b200.warmstart import Network
    with Network(max_batch=1024, seed=3) as net:
        x = _inputs(300, 0)  # not a multiple of the 128-row tile
        y = net.predict(x)
        p, f = net.params()
        yo, _ = mlp_ref.forward(p, f, x)
        err = np.linalg.norm(y - yo) / np.linalg.norm(yo)
        print(f"\nmlp forward rel err {err:.2e}")
        assert err <= TOL_FORWARD


def test_gradients_match_oracle():
    from optimisation2forme_b200.warmstart import Network
    with Network(max_batch=2048, seed=5) as net:
        x = _inputs(1000, 1)
        t = np.random.default_rng(2).standard_normal((1000, 8)).astype(np.float32)
        loss, g = net.gradients(x, t)
        p, f = net.params()
        lo, go = mlp_ref.gradients(p, f, x, t)
        assert abs(loss - lo) <= 1e-3 * lo
        errs = []
        for s in _layer_slices():
            den = np.linalg.norm(go[s])
            errs.append(np.linalg.norm(g[s] - go[s]) / den if den > 0 else np.linalg.norm(g[s]))
        print(f"\nmlp gradient rel err per tensor {np.array(errs)}")
        assert max(errs) <= TOL_GRAD


def test_training_fits_a_smooth_field():
    from optimisation2forme_b200.warmstart import Network
    x = _inputs(20000, 4)
    r = np.hypot(x[:, 0] - 0.5, x[:, 1])
    t = np.stack([np.sin(2 * x[:, 0]) * x[:, 5], np.cos(3 * x[:, 1]) + x[:, 2] * 10, np.exp(-r) * x[:, 6],
                  x[:, 3] * x[:, 4] * 10, np.tanh(x[:, 1] - x[:, 0]), r / 3, x[:, 5] ** 2, np.sin(r * 4)],
                 axis=1).astype(np.float32)
    with Network(max_batch=4096, seed=7) as net:
        net.set_data(x, t)
        hist = net.train(400, batch=2048, lr=2e-3, seed=1)
        print(f"\nmlp training loss {hist[0]:.3e} -> {hist[-20:].mean():.3e}")
        assert np.all(np.isfinite(hist))
        assert hist[-20:].mean() < 0.05 * hist[:5].mean()


def test_warm_start_cuts_adjoint_iterations():
    """Train on the solver's own (state, adjoint) fields over a family of
    shapes, then start the adjoint of an unseen shape from the prediction:
    BiCGSTAB reaches the same true-residual tolerance and the same lambda in
    fewer iterations than from zero.  The inputs are standardised, the
    adjoint target is lambda / sqrt(V), and fields from near-singular states
    (adjoint peaks 40-150x the family's) are left out of the training set."""
    from optimisation2forme_b200 import SimulationParams, Solver
    from optimisation2forme_b200.warmstart import (InputScaler, Network, Normaliser, adjoint_guess, sample,
                                                   select_fields)
    p0 = SimulationParams(viscosity=1.8e-5, inflow_velocity=0.6, aoa_deg=2.0, cfl_number=0.5, final_time=10.0,
                          limiter_k=5.0, verbosity=0)
    # 200 RK3 steps stay finite for every shape of the family except
    # (0.04, 0.5, 0.10), whose state develops a negative-pressure cell
    shapes = [(m, p, t) for m in (0.0, 0.02, 0.04) for p in (0.3, 0.5) for t in (0.10, 0.14)
              if (m, p, t) != (0.04, 0.5, 0.10)]
    xs, ys = [], []
    for (m, p, t) in shapes:
        mesh = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=11, m=m, p=p, t=t)
        with Solver(p0, desc=desc_of(mesh)) as s:
            x, y = sample(s, m, p, t, steps=200)
            xs.append(x)
            ys.append(y)
    keep = select_fields(ys)
    assert 6 <= len(keep) < len(shapes)  # the near-singular fields are dropped
    X, Y = np.concatenate([xs[i] for i in keep]), np.concatenate([ys[i] for i in keep])
    scaler, norm = InputScaler.fit(X), Normaliser.fit(Y)
    with Network(max_batch=8192, freq_scale=4.0, seed=1) as net:
        net.set_data(scaler.apply(X), norm.to_net(Y))
        hist = net.train(2000, batch=4096, lr=1e-3, seed=3)
        held = (0.03, 0.4, 0.12)  # inside the family, not one of its members
        mesh = small_mesh(triangles=True, n_surface=64, n_layers=16, seed=11, m=held[0], p=held[1], t=held[2])
        with Solver(p0, desc=desc_of(mesh)) as s:
            s.initialize_freestream()
            s.time_loop(200)
            cold = s.solve_adjoint_system(beta=0.1, tol=1e-10)
            guess = adjoint_guess(net, norm, s, *held, beta=0.1, scaler=scaler)
            warm = s.solve_adjoint_system(beta=0.1, tol=1e-10, guess=guess)
            err0 = np.linalg.norm(guess - cold["lambda"]) / np.linalg.norm(cold["lambda"])
            print(f"\nwarm start: kept {len(keep)}/{len(shapes)} fields; training loss {hist[0]:.3e} -> "
                  f"{hist[-20:].mean():.3e}; guess rel err {err0:.2e}; iterations {cold['iters']} -> {warm['iters']}")
            assert warm["relres"] <= 1e-10 and cold["relres"] <= 1e-10
            assert np.linalg.norm(warm["lambda"] - cold["lambda"]) <= 1e-6 * np.linalg.norm(cold["lambda"])
            assert err0 < 0.6
            assert warm["iters"] < cold["iters"]

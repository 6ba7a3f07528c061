"""The warm-start network's CPU oracle (oracle/mlp_ref.py): BF16 rounding,
and its backward pass against central finite differences of its own
forward pass with the rounding switched off."""
from __future__ import annotations

import numpy as np

from oracle import mlp_ref


def _random_net(seed=0, scale=0.05):
    rng = np.random.default_rng(seed)
    ins, outs = mlp_ref.dims()
    parts = []
    for i, o in zip(ins, outs):
        W = rng.standard_normal((o, i)) * np.sqrt(2.0 / i)
        if o == mlp_ref.N_OUT_PAD:
            W[mlp_ref.N_OUT:] = 0.0
        parts += [W.reshape(-1), rng.standard_normal(o) * scale]
    return np.concatenate(parts), rng.standard_normal(64) * 0.5


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.14159265, 0.0], dtype=np.float32)
    y = mlp_ref.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0            # tie to even
    assert y[2] == 1.0 + 2.0 ** -6                # tie rounds up to the even neighbour
    assert y[3] == -2.5 and y[5] == 0.0
    assert abs(y[4] - 3.140625) < 1e-12


def test_oracle_backward_matches_finite_differences():
    params, freq = _random_net(1)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((16, mlp_ref.N_IN)).astype(np.float32)
    t = rng.standard_normal((16, mlp_ref.N_OUT))
    mlp_ref.EXACT = True
    try:
        _, g = mlp_ref.gradients(params, freq, x, t)
        idx = rng.choice(np.flatnonzero(np.abs(g) > 1e-6), 40, replace=False)
        h = 1e-6
        for i in idx:
            pp, pm = params.copy(), params.copy()
            pp[i] += h
            pm[i] -= h
            lp = np.mean((mlp_ref.forward(pp, freq, x)[0] - t) ** 2)
            lm = np.mean((mlp_ref.forward(pm, freq, x)[0] - t) ** 2)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])
    finally:
        mlp_ref.EXACT = False

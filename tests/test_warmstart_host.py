"""Host side of the warm start: the target normaliser round-trips, compresses
the heavy-tailed adjoint channels and clamps predictions to the training
range before the exponential expansion."""
from __future__ import annotations

import numpy as np

from optimisation2forme_b200.warmstart import Normaliser


def test_normaliser_round_trip_and_standardisation():
    rng = np.random.default_rng(0)
    t = np.concatenate([rng.normal(1e5, 10.0, (500, 4)), rng.standard_cauchy((500, 4)) * 1e-3], axis=1)
    n = Normaliser.fit(t)
    z = n.to_net(t)
    assert np.allclose(z.mean(axis=0), 0.0, atol=1e-5) and np.allclose(z.std(axis=0), 1.0, atol=1e-4)
    back = n.from_net(z)
    assert np.allclose(back, t, rtol=1e-4, atol=1e-9)


def test_predictions_outside_the_training_range_are_clamped():
    rng = np.random.default_rng(1)
    t = rng.standard_normal((200, 8))
    n = Normaliser.fit(t)
    huge = np.full((1, 8), 1e3, dtype=np.float32)
    out = n.from_net(huge)
    assert np.all(np.isfinite(out))
    assert np.all(out[:, 4:] <= np.abs(t[:, 4:]).max(axis=0) * (1 + 1e-6))

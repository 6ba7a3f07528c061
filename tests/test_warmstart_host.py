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


def test_wall_disc_coords_on_a_circle():
    """A unit-circle wall (256 segments, listed from an arbitrary one):
    points at angle th and wall distance d map to s = th / 2 pi (arc from
    the rightmost point) and rho = 1 + log1p(d/h) / log1p(far/h), with
    h = 1e-3 x chord (chord 2), up to the polygon's sag."""
    from optimisation2forme_b200.warmstart import wall_disc_coords
    m = 256
    ang = 2 * np.pi * np.arange(m) / m
    pts = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    a, b = np.roll(pts, 77, axis=0), np.roll(np.roll(pts, -1, axis=0), 77, axis=0)
    rng = np.random.default_rng(3)
    th = rng.uniform(0.05, 2 * np.pi - 0.05, 500)
    d = 10 ** rng.uniform(-4, -1, 500)
    ctr = np.stack([(1 + d) * np.cos(th), (1 + d) * np.sin(th)], axis=1)
    uv = wall_disc_coords(ctr, a, b, h_rel=1e-3, far=20.0)
    rho = np.hypot(uv[:, 0], uv[:, 1])
    s = np.mod(np.arctan2(uv[:, 1], uv[:, 0]), 2 * np.pi) / (2 * np.pi)
    h = 2e-3
    # the polygon lies within 1 - cos(pi/256) < 7.6e-5 inside the circle
    sag = 7.6e-5 / (h + d) / np.log1p(20 / h)
    assert np.all(np.abs(rho - (1 + np.log1p(d / h) / np.log1p(20 / h))) <= sag + 1e-9)
    assert np.allclose(s, th / (2 * np.pi), atol=2e-4)

"""Learned warm start: a network trained on this solver's own state/adjoint
fields predicts, for a new NACA shape and flow, the state and the adjoint
field per cell; the adjoint prediction seeds BiCGSTAB, which still converges
to the same true-residual tolerance (the plain solve is the fallback and
the check on the network's error).

The network (4 x 256 SiLU, Fourier features of the cell centre plus
(m, p, t, Mach, AoA), BF16 weights/activations, FP32 accumulation) is trained
and run by the native library's tensor-core kernels (o2f_mlp_*).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check, lib

N_IN, N_OUT = 7, 8


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Network:
    """Host handle of the native network (o2f_mlp_*)."""

    def __init__(self, max_batch: int = 16384, freq_scale: float = 1.0, seed: int = 0, stream: int | None = None):
        h = C.c_void_p()
        check(lib().o2f_mlp_create(int(max_batch), float(freq_scale), int(seed), C.c_void_p(stream) if stream else None,
                                   C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib().o2f_mlp_n_params(h, C.byref(n)))
        self.n_params = n.value
        self.max_batch = int(max_batch)

    def set_data(self, inputs: np.ndarray, targets: np.ndarray) -> None:
        x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, N_IN)
        y = np.ascontiguousarray(targets, dtype=np.float32).reshape(-1, N_OUT)
        if x.shape[0] != y.shape[0]:
            raise ValueError("inputs and targets differ in length")
        check(lib().o2f_mlp_set_data(self._h, _fptr(x), _fptr(y), x.shape[0]))

    def train(self, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        hist = np.zeros(int(steps), dtype=np.float32)
        check(lib().o2f_mlp_train(self._h, int(steps), int(batch), float(lr), int(seed), _fptr(hist)))
        return hist

    def predict(self, inputs: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, N_IN)
        out = np.empty((x.shape[0], N_OUT), dtype=np.float32)
        check(lib().o2f_mlp_predict(self._h, _fptr(x), x.shape[0], _fptr(out)))
        return out

    def gradients(self, inputs: np.ndarray, targets: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, N_IN)
        y = np.ascontiguousarray(targets, dtype=np.float32).reshape(-1, N_OUT)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        check(lib().o2f_mlp_gradients(self._h, _fptr(x), _fptr(y), x.shape[0], _fptr(g), _fptr(loss)))
        return float(loss[0]), g

    def params(self) -> tuple[np.ndarray, np.ndarray]:
        p = np.empty(self.n_params, dtype=np.float32)
        f = np.empty(64, dtype=np.float32)
        check(lib().o2f_mlp_get_params(self._h, _fptr(p), _fptr(f)))
        return p, f

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError("parameter vector of the wrong size")
        check(lib().o2f_mlp_set_params(self._h, _fptr(p)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            check(lib().o2f_mlp_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclasses.dataclass
class Normaliser:
    """Maps of the 8 targets to the network's outputs: the adjoint channels
    (heavy-tailed: large at the wall, near zero elsewhere) are compressed by
    asinh(lambda / a) with a = their median magnitude, then every channel is
    standardised."""
    mean: np.ndarray
    scale: np.ndarray
    asinh_scale: np.ndarray  # [4], the adjoint channels
    lo: np.ndarray  # range of the standardised training targets: predictions
    hi: np.ndarray  # are clamped to it before the (exponential) sinh expansion

    @staticmethod
    def _compress(t, a):
        y = np.array(t, dtype=np.float64).reshape(-1, N_OUT)
        y[:, 4:] = np.arcsinh(y[:, 4:] / a)
        return y

    @classmethod
    def fit(cls, targets: np.ndarray) -> "Normaliser":
        t = np.asarray(targets, dtype=np.float64).reshape(-1, N_OUT)
        a = np.median(np.abs(t[:, 4:]), axis=0)
        a = np.where(a > 0, a, 1.0)
        y = cls._compress(t, a)
        mu, s = y.mean(axis=0), y.std(axis=0)
        s = np.where(s > 0, s, 1.0)
        z = (y - mu) / s
        return cls(mu, s, a, z.min(axis=0), z.max(axis=0))

    def to_net(self, t):
        return ((self._compress(t, self.asinh_scale) - self.mean) / self.scale).astype(np.float32)

    def from_net(self, y):
        z = np.clip(np.asarray(y, dtype=np.float64).reshape(-1, N_OUT), self.lo, self.hi)
        t = z * self.scale + self.mean
        t[:, 4:] = np.sinh(t[:, 4:]) * self.asinh_scale
        return t


@dataclasses.dataclass
class InputScaler:
    """Standardisation of the 7 inputs: the shape and flow parameters (order
    0.01-1) would otherwise be drowned by the coordinates (up to the far
    field, 20 chords); the Fourier features then act on standardised (x, y)."""
    mean: np.ndarray
    std: np.ndarray

    @classmethod
    def fit(cls, inputs: np.ndarray) -> "InputScaler":
        x = np.asarray(inputs, dtype=np.float64).reshape(-1, N_IN)
        s = x.std(axis=0)
        return cls(x.mean(axis=0), np.where(s > 0, s, 1.0))

    def apply(self, inputs: np.ndarray) -> np.ndarray:
        return ((np.asarray(inputs, dtype=np.float64).reshape(-1, N_IN) - self.mean) / self.std).astype(np.float32)


def select_fields(targets: Sequence[np.ndarray], factor: float = 10.0) -> list[int]:
    """Indices of the training fields to keep: a field whose largest adjoint
    magnitude exceeds `factor` times the median of the fields' maxima comes
    from a near-singular state (a cell at the edge of positivity) and would
    dominate the fit; it is left out."""
    peaks = np.array([np.abs(np.asarray(y).reshape(-1, N_OUT)[:, 4:]).max() for y in targets])
    ref = np.median(peaks)
    return [i for i, v in enumerate(peaks) if v <= factor * ref]


def wall_disc_coords(ctr: np.ndarray, seg_a: np.ndarray, seg_b: np.ndarray, h_rel: float = 1e-3,
                     far: float = 20.0) -> np.ndarray:
    """[n, 2] body-fitted coordinates of the points `ctr` [n, 2] about a wall
    given as segments seg_a -> seg_b ([m, 2] end points, chained head to
    tail into closed loops): the nearest wall point's arc-length fraction s
    (from the rightmost wall point of its loop) and the wall distance d,
    mapped to the disc rho (cos 2 pi s, sin 2 pi s) with
    rho = 1 + log(1 + d/h) / log(1 + far/h) and h = h_rel x chord (the
    wall's x extent).  The wall maps to the unit circle and the far field to
    about radius 2, the boundary layer (d ~ h to 100 h) to rho in
    [1.07, 1.5]: the fields the network learns vary over the disc at one
    scale instead of at 1e-3 and at 20 chords in (x, y)."""
    from scipy.spatial import cKDTree
    ctr = np.asarray(ctr, dtype=np.float64).reshape(-1, 2)
    a = np.asarray(seg_a, dtype=np.float64).reshape(-1, 2)
    b = np.asarray(seg_b, dtype=np.float64).reshape(-1, 2)
    m = a.shape[0]
    # chain the segments into loops by shared end points; arc length per loop
    key = lambda p: (round(p[0], 12), round(p[1], 12))
    starts = {}
    for k in range(m):
        starts.setdefault(key(a[k]), []).append(k)
    s0 = np.zeros(m)
    total = np.ones(m)
    seen = np.zeros(m, dtype=bool)
    seglen = np.hypot(*(b - a).T)
    for first in np.argsort(-a[:, 0], kind="stable"):  # a loop starts at its rightmost point
        if seen[first]:
            continue
        loop, k = [], int(first)
        while k is not None and not seen[k]:
            seen[k] = True
            loop.append(k)
            nxt = [j for j in starts.get(key(b[k]), []) if not seen[j]]
            k = nxt[0] if nxt else None
        cum = np.concatenate([[0.0], np.cumsum(seglen[loop])])
        s0[loop], total[loop] = cum[:-1], max(cum[-1], 1e-300)
    xs = np.concatenate([a[:, 0], b[:, 0]])
    h = h_rel * max(float(xs.max() - xs.min()), 1e-300)
    kq = min(8, m)
    _, idx = cKDTree(0.5 * (a + b)).query(ctr, k=kq)
    idx = idx.reshape(ctr.shape[0], kq)
    ab = b[idx] - a[idx]  # [n, k, 2]
    ap = ctr[:, None, :] - a[idx]
    t = np.clip(np.sum(ap * ab, axis=2) / np.maximum(np.sum(ab * ab, axis=2), 1e-300), 0.0, 1.0)
    q = a[idx] + t[..., None] * ab
    d2 = np.sum((ctr[:, None, :] - q) ** 2, axis=2)
    j = np.argmin(d2, axis=1)
    r = np.arange(ctr.shape[0])
    seg = idx[r, j]
    d = np.sqrt(d2[r, j])
    s = (s0[seg] + t[r, j] * seglen[seg]) / total[seg]
    rho = 1.0 + np.log1p(d / h) / np.log1p(far / h)
    ang = 2.0 * np.pi * s
    return np.stack([rho * np.cos(ang), rho * np.sin(ang)], axis=1)


def wall_segments(solver) -> tuple[np.ndarray, np.ndarray]:
    """End points ([m, 2] each) of a context's wall edges, oriented so that
    the segments chain into loops (each segment's end starts the next one)."""
    xy = solver.mesh_array("vert_xy").reshape(-1, 2)
    ev = solver.mesh_array("edge_v").reshape(-1, 2)
    wall = ev[solver.mesh_array("edge_bc") == ord("w")]
    adj = {}
    for k, (u, v) in enumerate(wall):
        adj.setdefault(int(u), []).append(k)
        adj.setdefault(int(v), []).append(k)
    used = np.zeros(len(wall), dtype=bool)
    A, B = [], []
    for k0 in range(len(wall)):
        if used[k0]:
            continue
        u, v = int(wall[k0][0]), int(wall[k0][1])
        k = k0
        while True:
            used[k] = True
            A.append(u)
            B.append(v)
            nxt = [j for j in adj[v] if not used[j]]
            if not nxt:
                break
            k = nxt[0]
            u, v = v, int(wall[k][1]) if int(wall[k][0]) == v else int(wall[k][0])
    return xy[np.array(A, dtype=np.int64)], xy[np.array(B, dtype=np.int64)]


def cell_inputs(solver, m: float, p: float, t: float, coords: str = "xy") -> np.ndarray:
    """[n_cells, 7] network inputs of a context: cell centres (reference
    order) -- as (x, y), or with coords="wall" as the body-fitted disc
    coordinates of wall_disc_coords -- with the shape and the flow (Mach,
    AoA) of its parameters."""
    ctr = solver.mesh_array("cell_ctr").reshape(-1, 2)
    n = ctr.shape[0]
    x = np.empty((n, N_IN), dtype=np.float32)
    if coords == "wall":
        x[:, 0:2] = wall_disc_coords(ctr, *wall_segments(solver))
    elif coords == "xy":
        x[:, 0:2] = ctr
    else:
        raise ValueError(f"coords must be 'xy' or 'wall', not {coords!r}")
    x[:, 2], x[:, 3], x[:, 4] = m, p, t
    x[:, 5] = solver.params.inflow_velocity
    x[:, 6] = solver.params.aoa_deg
    return x


def _size(solver) -> np.ndarray:
    """sqrt(cell volume) per cell, reference order: the adjoint of the
    finite-volume residual (J^T carries 1/V, the wall right-hand side does
    not) scales with the local cell size, so lambda / sqrt(V) is the smooth
    field the network learns."""
    return np.sqrt(solver.mesh_array("cell_vol")).reshape(-1, 1)


def sample(solver, m: float, p: float, t: float, steps: int, beta: float = 0.1, tol: float = 1e-10,
           coords: str = "xy"):
    """One training sample set: march `steps` RK3 steps from the freestream,
    solve the adjoint, return (inputs, targets [state, lambda/sqrt(V)] per
    cell)."""
    solver.initialize_freestream()
    solver.time_loop(steps)
    U = solver.get_state().reshape(-1, 4)
    lam = solver.solve_adjoint_system(beta=beta, tol=tol)["lambda"].reshape(-1, 4)
    return cell_inputs(solver, m, p, t, coords), np.concatenate([U, lam / _size(solver)], axis=1)


def adjoint_guess(net: Network, norm: Normaliser, solver, m: float, p: float, t: float,
                  beta: float = 0.1, residual_scaled: bool = False, scaler: InputScaler | None = None,
                  coords: str = "xy") -> np.ndarray:
    """Predicted lambda (reference order, interleaved 4 per cell).  With
    residual_scaled, it is multiplied by the alpha minimising
    ||b - J^T (alpha lambda0)|| (one J^T product), which bounds the initial
    residual by ||b||; J^T weighs the guess's cell-scale error by 1/h, so
    that alpha can vanish for a guess that is close in L2.  Needs the
    interface states of the current state.  `scaler`: the input
    standardisation the network was trained with; `coords`: its input
    coordinates (cell_inputs)."""
    x = cell_inputs(solver, m, p, t, coords)
    y = norm.from_net(net.predict(scaler.apply(x) if scaler else x))
    lam0 = np.ascontiguousarray((y[:, 4:8] * _size(solver)).reshape(-1))
    if not residual_scaled:
        return lam0
    b = solver.assemble_adjoint_rhs(beta)
    a0 = solver.apply_jacobian_transpose(lam0)
    den = float(a0 @ a0)
    alpha = float(b @ a0) / den if den > 0 else 0.0
    return alpha * lam0


def state_guess(net: Network, norm: Normaliser, solver, m: float, p: float, t: float,
                scaler: InputScaler | None = None, coords: str = "xy") -> np.ndarray:
    x = cell_inputs(solver, m, p, t, coords)
    y = norm.from_net(net.predict(scaler.apply(x) if scaler else x))
    return np.ascontiguousarray(y[:, 0:4].reshape(-1))

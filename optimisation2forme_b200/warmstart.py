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


def cell_inputs(solver, m: float, p: float, t: float) -> np.ndarray:
    """[n_cells, 7] network inputs of a context: cell centres (reference
    order) with the shape and the flow (Mach, AoA) of its parameters."""
    ctr = solver.mesh_array("cell_ctr").reshape(-1, 2)
    n = ctr.shape[0]
    x = np.empty((n, N_IN), dtype=np.float32)
    x[:, 0:2] = ctr
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


def sample(solver, m: float, p: float, t: float, steps: int, beta: float = 0.1, tol: float = 1e-10):
    """One training sample set: march `steps` RK3 steps from the freestream,
    solve the adjoint, return (inputs, targets [state, lambda/sqrt(V)] per
    cell)."""
    solver.initialize_freestream()
    solver.time_loop(steps)
    U = solver.get_state().reshape(-1, 4)
    lam = solver.solve_adjoint_system(beta=beta, tol=tol)["lambda"].reshape(-1, 4)
    return cell_inputs(solver, m, p, t), np.concatenate([U, lam / _size(solver)], axis=1)


def adjoint_guess(net: Network, norm: Normaliser, solver, m: float, p: float, t: float,
                  beta: float = 0.1, residual_scaled: bool = False, scaler: InputScaler | None = None) -> np.ndarray:
    """Predicted lambda (reference order, interleaved 4 per cell).  With
    residual_scaled, it is multiplied by the alpha minimising
    ||b - J^T (alpha lambda0)|| (one J^T product), which bounds the initial
    residual by ||b||; J^T weighs the guess's cell-scale error by 1/h, so
    that alpha can vanish for a guess that is close in L2.  Needs the
    interface states of the current state.  `scaler`: the input
    standardisation the network was trained with."""
    x = cell_inputs(solver, m, p, t)
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
                scaler: InputScaler | None = None) -> np.ndarray:
    x = cell_inputs(solver, m, p, t)
    y = norm.from_net(net.predict(scaler.apply(x) if scaler else x))
    return np.ascontiguousarray(y[:, 0:4].reshape(-1))

"""Test infrastructure only: numpy restatement of the warm-start network's
forward and backward passes (optimisation2forme_b200/csrc/mlp.cu), the
checker of its tcgen05 kernels.

The network has no counterpart in the reference.  The oracle rounds to BF16
(round to nearest even) at exactly the points where the kernels store BF16
-- features, weights, activations, pre-activations, output and hidden
gradients -- and computes everything else in FP64, so its results differ
from the kernels' only by the FP32 accumulation order and by BF16 ties that
FP32 and FP64 intermediates round differently.
"""
from __future__ import annotations

import numpy as np

N_IN, N_FREQ, N_FEAT, WIDTH, HIDDEN, N_OUT, N_OUT_PAD = 7, 32, 128, 256, 4, 8, 16


EXACT = False  # True: no BF16 rounding (FP64 network, for finite-difference checks of the formulas)


def bf16(x) -> np.ndarray:
    """Round float values to BF16 (nearest even), returned as float64."""
    if EXACT:
        return np.asarray(x, dtype=np.float64)
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    out = r.view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    out[nan] = np.nan
    return out


def dims():
    ins = [N_FEAT] + [WIDTH] * HIDDEN
    outs = [WIDTH] * HIDDEN + [N_OUT_PAD]
    return ins, outs


def unpack(params: np.ndarray):
    """[(W_l [out][in], b_l)] from the flat parameter vector."""
    ins, outs = dims()
    layers, off = [], 0
    for i, o in zip(ins, outs):
        W = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        layers.append((W.astype(np.float64), b.astype(np.float64)))
    assert off == params.size
    return layers


def features(inputs: np.ndarray, freq: np.ndarray) -> np.ndarray:
    x = np.asarray(inputs, dtype=np.float32)
    f = np.asarray(freq, dtype=np.float32).reshape(N_FREQ, 2)
    arg = 2.0 * np.pi * (x[:, :1] * f[:, 0][None, :] + x[:, 1:2] * f[:, 1][None, :]).astype(np.float64)
    X = np.zeros((x.shape[0], N_FEAT))
    X[:, :N_FREQ] = np.sin(arg)
    X[:, N_FREQ:2 * N_FREQ] = np.cos(arg)
    X[:, 2 * N_FREQ:2 * N_FREQ + N_IN] = x
    return bf16(X)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, freq, inputs):
    layers = unpack(params)
    a = features(inputs, freq)
    cache = [a]
    for l, (W, b) in enumerate(layers):
        z = a @ bf16(W).T + b
        if l < HIDDEN:
            cache.append(bf16(z))          # stored pre-activation
            a = bf16(silu(z))              # activation from the unrounded z
            cache.append(a)
        else:
            return z[:, :N_OUT], cache


def gradients(params, freq, inputs, targets):
    """(loss, flat gradient) of the mean squared error over the 8 outputs."""
    layers = unpack(params)
    n = inputs.shape[0]
    y, cache = forward(params, freq, inputs)
    d = y - np.asarray(targets, dtype=np.float64)
    loss = float(np.mean(d * d))
    g = np.zeros((n, N_OUT_PAD))
    g[:, :N_OUT] = bf16(2.0 * d / (n * N_OUT))
    grads = []
    for l in range(HIDDEN, -1, -1):
        W, _ = layers[l]
        below = cache[2 * l]               # features (l = 0) or the activation of layer l-1
        grads.append((g.T @ below, g.sum(axis=0)))
        if l == 0:
            break
        zprev = cache[2 * l - 1]
        g = bf16((g @ bf16(W)) * silu_grad(zprev))
    flat = []
    for dW, db in reversed(grads):
        flat.append(dW.reshape(-1))
        flat.append(db)
    return loss, np.concatenate(flat)

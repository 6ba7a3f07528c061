"""Test infrastructure only: numpy restatement of the reference's field view,
the checker of the headless image kernels (optimisation2forme_b200/csrc/
render.cuh).

  * computeCellScalar (src/compute.cpp:6-60): the cell scalar;
  * Simulator::output_step (src/simulation.cpp:186-193): the colour range,
    pressure rounded outward to multiples of 5000;
  * Mesh::pixelToPhysical and pointInTriangle (src/mesh.cpp:349-353,
    401-411; quadrilaterals as the triangles (A,B,C), (A,C,D), :446-452):
    the pixel -> cell map, here the lowest cell number among the cells that
    contain the pixel centre, -1 outside the mesh;
  * render_scalar_field_unstructured, colormap_B_W_R and
    colormap_schlieren_bluewhite (src/renderer_colormap.cpp:10-47,
    include/renderer_colormap.hpp:16-95): the colours, with the reference's
    float interpolation (lerp(float, float, float)) done in float32.

Everything else is float64 numpy arithmetic, which rounds each operation
like the reference's scalar C++ does (no fused multiply-add).
"""
from __future__ import annotations

import numpy as np

FIELDS = ("rho", "rho_u", "rho_v", "E", "u", "v", "u_x", "u_y", "v_x", "v_y", "div", "p", "pressure")


def cell_scalar(U: np.ndarray, field: str, gamma: float, grad: np.ndarray | None = None) -> np.ndarray:
    """U: [n, 4] conserved states; grad: [n, 2, 4] (x- and y-gradients of
    rho, rho_u, rho_v, E) for the gradient fields."""
    U = np.asarray(U, dtype=np.float64).reshape(-1, 4)
    rho, ru, rv, E = U.T
    nz = rho != 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.where(nz, ru / np.where(nz, rho, 1.0), 0.0)
        v = np.where(nz, rv / np.where(nz, rho, 1.0), 0.0)
        rho_div = np.where(nz, rho, 1.0)
        if field == "rho":
            return rho.copy()
        if field == "rho_u":
            return ru.copy()
        if field == "rho_v":
            return rv.copy()
        if field == "E":
            return E.copy()
        if field == "u":
            return u
        if field == "v":
            return v
        if field in ("p", "pressure"):
            kinetic = 0.5 * (ru * ru + rv * rv) / rho
            return (gamma - 1.0) * (E - kinetic)
        g = np.asarray(grad, dtype=np.float64).reshape(-1, 2, 4)
        gx, gy = g[:, 0, :], g[:, 1, :]
        u_x = (gx[:, 1] - u * gx[:, 0]) / rho_div
        u_y = (gy[:, 1] - u * gy[:, 0]) / rho_div
        v_x = (gx[:, 2] - v * gx[:, 0]) / rho_div
        v_y = (gy[:, 2] - v * gy[:, 0]) / rho_div
    return {"u_x": u_x, "u_y": u_y, "v_x": v_x, "v_y": v_y, "div": u_x + v_y}[field]


def colour_range(s: np.ndarray, field: str) -> tuple[float, float]:
    lo, hi = float(np.min(s)), float(np.max(s))
    if field in ("p", "pressure"):
        step = 5000.0
        return float(np.floor(lo / step) * step), float(np.ceil(hi / step) * step)
    return lo, hi


def _in_triangle(x, y, v0, v1, v2):
    dX, dY = x - v2[0], y - v2[1]
    dX21, dY12 = v2[0] - v1[0], v1[1] - v2[1]
    D = dY12 * (v0[0] - v2[0]) + dX21 * (v0[1] - v2[1])
    s = dY12 * dX + dX21 * dY
    t = (v2[1] - v0[1]) * dX + (v0[0] - v2[0]) * dY
    flip = D < 0
    s, t, D = np.where(flip, -s, s), np.where(flip, -t, t), np.where(flip, -D, D)
    return (s >= 0) & (t >= 0) & ((s + t) <= D)


def pixel_cells(node_xy, cell_offsets, cell_nodes, nx: int, ny: int) -> np.ndarray:
    """[ny, nx] cell number (mesh-file order) per pixel row j (y up), -1 outside."""
    xy = np.asarray(node_xy, dtype=np.float64).reshape(-1, 2)
    x_min, x_max = xy[:, 0].min(), xy[:, 0].max()
    y_min, y_max = xy[:, 1].min(), xy[:, 1].max()
    Lx, Ly = abs(x_max - x_min), abs(y_max - y_min)
    px = x_min + (np.arange(nx) + 0.5) * Lx / nx
    py = y_min + (np.arange(ny) + 0.5) * Ly / ny
    X, Y = np.meshgrid(px, py)  # [ny, nx]
    out = np.full((ny, nx), -1, dtype=np.int64)
    for c in range(len(cell_offsets) - 1):  # ascending: the first hit is the lowest number
        vs = xy[cell_nodes[cell_offsets[c]:cell_offsets[c + 1]]]
        lo, hi = vs.min(axis=0), vs.max(axis=0)
        jx = np.nonzero((px >= lo[0]) & (px <= hi[0]))[0]
        jy = np.nonzero((py >= lo[1]) & (py <= hi[1]))[0]
        if jx.size == 0 or jy.size == 0:
            continue
        sub_x, sub_y = X[np.ix_(jy, jx)], Y[np.ix_(jy, jx)]
        inside = _in_triangle(sub_x, sub_y, vs[0], vs[1], vs[2])
        if len(vs) == 4:
            inside |= _in_triangle(sub_x, sub_y, vs[0], vs[2], vs[3])
        blk = out[np.ix_(jy, jx)]
        blk[(blk < 0) & inside] = c
        out[np.ix_(jy, jx)] = blk
    return out


def _lerp(a, b, t):
    a, b, t = np.float32(a), np.float32(b), np.asarray(t, dtype=np.float32)
    return a + (b - a) * t


def _clamp01(x):
    """std::max(0.0, std::min(1.0, x)): a NaN becomes 1."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(np.isnan(x), 1.0, np.clip(x, 0.0, 1.0))


def _to8(x):
    return (_clamp01(x) * 255.0 + 0.5).astype(np.uint8)


def colormap_bwr(t: np.ndarray) -> np.ndarray:
    t = _clamp01(t)
    q0, q1, q2 = t < 0.25, t < 0.5, t < 0.75
    b = np.where(q0, _lerp(0.3, 1.0, t / 0.25), np.where(q1, 1.0, np.where(q2, _lerp(1.0, 0.0, (t - 0.5) / 0.25), 0.0)))
    g = np.where(q0, 0.0, np.where(q1, _lerp(0.0, 1.0, (t - 0.25) / 0.25),
                                   np.where(q2, _lerp(1.0, 0.0, (t - 0.5) / 0.25), 0.0)))
    r = np.where(q0, 0.0, np.where(q1, _lerp(0.0, 1.0, (t - 0.25) / 0.25),
                                   np.where(q2, 1.0, _lerp(1.0, 0.5, (t - 0.75) / 0.25))))
    return np.stack([_to8(r), _to8(g), _to8(b)], axis=-1)


def colormap_schlieren(t: np.ndarray) -> np.ndarray:
    t = _clamp01(t)
    low = t < 0.7
    s_low, s_high = t / 0.7, (t - 0.7) / 0.3
    blue_low = (_lerp(0.0, 255.0, s_low).astype(np.float64) + 0.5).astype(np.uint8)
    white = (_lerp(0.0, 255.0, s_high).astype(np.float64) + 0.5).astype(np.uint8)
    r = np.where(low, 0, white).astype(np.uint8)
    b = np.where(low, blue_low, 255).astype(np.uint8)
    return np.stack([r, r.copy(), b], axis=-1)


def render(node_xy, cell_offsets, cell_nodes, scalar: np.ndarray, nx: int, ny: int, fmin: float, fmax: float,
           cmap: str = "") -> np.ndarray:
    """[ny, nx, 3] uint8, top row first (image row ny-1-j holds pixel row j)."""
    img = np.zeros((ny, nx, 3), dtype=np.uint8)
    span = fmax - fmin
    if not span > 0.0:
        return img
    cells = pixel_cells(node_xy, cell_offsets, cell_nodes, nx, ny)
    hit = cells >= 0
    with np.errstate(invalid="ignore"):
        t = (np.asarray(scalar, dtype=np.float64)[np.where(hit, cells, 0)] - fmin) / span
    if cmap == "schlieren":
        col = colormap_schlieren(np.sqrt(np.fmax(0.0, t)))  # std::max(0.0, NaN) is 0
    else:
        col = colormap_bwr(t)
    col[~hit] = 0
    return col[::-1].copy()

"""Seeded NACA 4-digit airfoil meshes (Gmsh is not available here).

``naca_ogrid`` builds an O-grid around the airfoil: cosine-clustered surface
points, wall-normal layers with a first height and a geometric growth, then a
smooth geometric blend out to a far-field circle.  Quads can be kept (every
interior vertex has 4 cells, the reference's supported case) or split into
triangles along seeded random diagonals (vertex valence 4..8, the unstructured
case).  Boundaries: ``Airfoil`` (wall) on the surface loop, ``FreeStream``
(far field) on the outer loop, as in the reference's .geo templates.

The result is an o2f mesh description in construction order; ``write_msh2``
writes the same mesh as an ASCII MSH 2.2 file that the reference's own mesh
import reads in the same order.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


def naca4_surface(m: float, p: float, t: float, n: int, chord: float = 1.0, pos_x: float = 0.355,
                  n_te: int = 3, cluster: float = 1.0) -> np.ndarray:
    """Closed surface loop, counter-clockwise from the upper trailing edge over
    the leading edge to the lower trailing edge, then across the blunt base.
    Camber/thickness: the yc/yt formulas of the reference
    (src/shape_optimization.cpp:807-826).  ``cluster`` blends cosine
    clustering (1) with uniform spacing (0) along the chord."""
    k = n // 2
    s = np.linspace(0.0, 1.0, k + 1)
    xr = cluster * 0.5 * (1.0 - np.cos(math.pi * s)) + (1.0 - cluster) * s  # 0 .. 1

    def yc(x):
        if m == 0.0:
            return np.zeros_like(x)
        return np.where(x <= p, m / (p * p) * (2 * p * x - x * x),
                        m / ((1 - p) ** 2) * ((1 - 2 * p) + 2 * p * x - x * x))

    def yt(x):
        return 5 * t * chord * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3
                                - 0.1015 * x ** 4)

    x_up = xr[::-1]  # TE -> LE
    upper = np.stack([pos_x + x_up * chord, yc(x_up) + yt(x_up)], axis=1)
    x_lo = xr[1:]  # LE -> TE (LE shared)
    lower = np.stack([pos_x + x_lo * chord, yc(x_lo) - yt(x_lo)], axis=1)
    pts = [upper, lower]
    if n_te > 0:  # blunt base, lower TE -> upper TE (exclusive of both)
        a, b = lower[-1], upper[0]
        s = np.linspace(0, 1, n_te + 2)[1:-1, None]
        pts.append(a + (b - a) * s)
    return np.concatenate(pts, axis=0)


@dataclasses.dataclass
class OGridSpec:
    m: float = 0.02
    p: float = 0.4
    t: float = 0.12
    n_surface: int = 160
    n_layers: int = 60
    first_height: float = 1e-3
    growth: float = 1.1
    r_far: float = 20.0
    triangles: bool = True
    seed: int = 0
    pos_x: float = 0.355
    chord: float = 1.0
    jitter: float = 0.1
    cluster: float = 1.0


def _normals(S: np.ndarray) -> np.ndarray:
    """Outward unit normals of a counter-clockwise closed loop (vertex average
    of the two adjacent edge normals)."""
    d_next = np.roll(S, -1, axis=0) - S
    d_prev = S - np.roll(S, 1, axis=0)
    n1 = np.stack([d_next[:, 1], -d_next[:, 0]], axis=1)
    n0 = np.stack([d_prev[:, 1], -d_prev[:, 0]], axis=1)
    n1 /= np.linalg.norm(n1, axis=1, keepdims=True)
    n0 /= np.linalg.norm(n0, axis=1, keepdims=True)
    n = n0 + n1
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def naca_ogrid(spec: OGridSpec):
    """Returns dict(node_xy, segments, segment_bc, cell_offsets, cell_nodes):
    an o2f mesh description in construction order."""
    rng = np.random.default_rng(spec.seed)
    S = naca4_surface(spec.m, spec.p, spec.t, spec.n_surface, spec.chord, spec.pos_x, cluster=spec.cluster)
    # The loop runs TE(upper) -> LE -> TE(lower) -> base: counter-clockwise,
    # so the outward normals are (dy, -dx).
    ni = S.shape[0]
    N = _normals(S)
    # Radial distances: one smooth sequence of layer spacings -- geometric
    # growth from the first cell until the cells are about isotropic (mean
    # tangential spacing), then a geometric ratio solved so that the last
    # layer lands on the far field.
    nl = spec.n_layers
    chord = spec.chord
    centre = np.array([spec.pos_x + 0.5 * chord, 0.0])
    h_iso = 2.05 * chord / max(ni // 2, 1)
    d = [0.0]
    h = spec.first_height
    while h < h_iso and len(d) < nl // 2:
        d.append(d[-1] + h)
        h *= spec.growth
    j1 = len(d) - 1
    rest = nl - j1
    span = spec.r_far - d[-1]
    lo, hi = 1.0 + 1e-12, 4.0
    if h * rest >= span:
        q = 1.0 + 1e-12
    else:
        for _ in range(200):  # h (q^rest - 1) / (q - 1) = span
            q = 0.5 * (lo + hi)
            if h * (q ** rest - 1.0) / (q - 1.0) > span:
                hi = q
            else:
                lo = q
    steps = h * np.power(q, np.arange(rest))
    dist = np.cumsum(steps)
    f = dist / dist[-1] if rest > 0 else np.zeros(0)
    A = S + d[-1] * N  # edge of the wall-layer region
    theta = np.arctan2(A[:, 1] - centre[1], A[:, 0] - centre[0])
    F = centre + spec.r_far * np.stack([np.cos(theta), np.sin(theta)], axis=1)
    layers = [S + dj * N for dj in d]
    for fj in f:
        layers.append(A + (F - A) * fj)
    P = np.stack(layers, axis=0)  # [nl+1, ni, 2]
    if spec.jitter > 0 and rest > 2:
        # Seeded jitter of interior far-field points along the radial line.
        u = (F - A) / np.linalg.norm(F - A, axis=1, keepdims=True)
        for j in range(j1 + 1, nl):
            dj = np.linalg.norm(P[j + 1] - P[j - 1], axis=1, keepdims=True) * 0.5
            P[j] += u * dj * spec.jitter * rng.uniform(-1, 1, size=(ni, 1))
    nodes = P.reshape(-1, 2)
    vid = np.arange((nl + 1) * ni).reshape(nl + 1, ni)
    cells = []
    for j in range(nl):
        for i in range(ni):
            i1 = (i + 1) % ni
            # (a, b, c, dd) runs clockwise (i counter-clockwise along the
            # surface, j outward); cells are stored counter-clockwise.
            a, b, c, dd = vid[j, i], vid[j, i1], vid[j + 1, i1], vid[j + 1, i]
            # In the first and last layers the diagonals alternate, so every
            # wall and far-field vertex has 2 or 4 cells: 3 cells would make
            # the reference's barycentric vertex weights extrapolate from the
            # thin triangle of cell centres (weights far outside [0, 1]).
            edge_layer = j == 0 or j == nl - 1
            split_ac = (i % 2 == 0) if edge_layer else rng.random() < 0.5
            if not spec.triangles:
                cells.append((a, dd, c, b))
            elif split_ac:
                cells.append((a, c, b))
                cells.append((a, dd, c))
            else:
                cells.append((a, dd, b))
                cells.append((b, dd, c))
    offs = np.zeros(len(cells) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(c) for c in cells])
    cn = np.fromiter((v for c in cells for v in c), dtype=np.int64, count=int(offs[-1]))
    # Boundary segments: far field first, then the wall (physical group order).
    far = [(vid[nl, i], vid[nl, (i + 1) % ni]) for i in range(ni)]
    wall = [(vid[0, i], vid[0, (i + 1) % ni]) for i in range(ni)]
    seg = np.array(far + wall, dtype=np.int64)
    bc = np.array([ord("f")] * len(far) + [ord("w")] * len(wall), dtype=np.uint8)
    return {"node_xy": nodes.astype(np.float64), "segments": seg, "segment_bc": bc, "cell_offsets": offs,
            "cell_nodes": cn}


def write_msh2(path, mesh: dict) -> None:
    """ASCII MSH 2.2 with physical groups FreeStream (1-D, tag 1), Airfoil
    (1-D, tag 2) and Fluid (2-D, tag 3); nodes tagged 1..N in order, so the
    reference's Gmsh import sees the same vertex, segment and cell orders."""
    xy = mesh["node_xy"].reshape(-1, 2)
    seg = mesh["segments"].reshape(-1, 2)
    bc = mesh["segment_bc"]
    offs, cn = mesh["cell_offsets"], mesh["cell_nodes"]
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "3", '1 1 "FreeStream"',
             '1 2 "Airfoil"', '2 3 "Fluid"', "$EndPhysicalNames", "$Nodes", str(len(xy))]
    lines += [f"{i + 1} {x:.17g} {y:.17g} 0" for i, (x, y) in enumerate(xy)]
    lines += ["$EndNodes", "$Elements"]
    els = []
    eid = 1
    for (a, b), code in zip(seg, bc):
        tag = 1 if code == ord("f") else 2
        els.append(f"{eid} 1 2 {tag} {tag} {a + 1} {b + 1}")
        eid += 1
    for c in range(len(offs) - 1):
        vs = cn[offs[c]:offs[c + 1]]
        typ = 2 if len(vs) == 3 else 3
        els.append(f"{eid} {typ} 2 3 3 " + " ".join(str(v + 1) for v in vs))
        eid += 1
    lines += [str(len(els))] + els + ["$EndElements"]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def config_mesh(name: str, seed: int = 0) -> tuple[OGridSpec, dict]:
    """Mesh specs and flow settings of the named workloads.

    * ``small``  -- NACA 2412, ~20k triangles, M=0.6, AoA=2 deg, Re=5000.
    * ``large``  -- NACA 0012, ~2M triangles, first cell 1e-4 chord, growth
      1.1, M=0.85, AoA=1.25 deg, Re=1e4 (the transonic case).
    * ``medium`` -- the same case at ~1M triangles (kernel profiles).
    * ``mixed``  -- ~500k triangles, seeded (m, p, t, M, AoA).
    """
    if name == "small":
        spec = OGridSpec(m=0.02, p=0.4, t=0.12, n_surface=200, n_layers=50, first_height=2e-3, growth=1.1,
                         seed=seed)
        flow = dict(mach=0.6, aoa=2.0, reynolds=5000.0)
    elif name == "large":
        spec = OGridSpec(m=0.0, p=0.4, t=0.12, n_surface=1400, n_layers=715, first_height=1e-4, growth=1.1,
                         seed=seed)
        flow = dict(mach=0.85, aoa=1.25, reynolds=1e4)
    elif name == "medium":
        spec = OGridSpec(m=0.0, p=0.4, t=0.12, n_surface=1000, n_layers=505, first_height=1e-4, growth=1.1,
                         seed=seed)
        flow = dict(mach=0.85, aoa=1.25, reynolds=1e4)
    elif name == "mixed":
        rng = np.random.default_rng(seed)
        spec = OGridSpec(m=float(rng.uniform(0, 0.06)), p=float(rng.uniform(0.2, 0.6)),
                         t=float(rng.uniform(0.08, 0.18)), n_surface=700, n_layers=357, first_height=1e-4,
                         growth=1.1, seed=seed)
        flow = dict(mach=float(rng.uniform(0.5, 0.8)), aoa=float(rng.uniform(0.0, 4.0)), reynolds=1e4)
    else:
        raise ValueError(name)
    return spec, flow


def viscosity_for(reynolds: float, mach: float, gamma=1.4, rho=1.225, p=101325.0, chord=1.0) -> float:
    """mu = rho U c / Re with the reference's freestream (src/boundary.cpp:10-14)."""
    return rho * mach * math.sqrt(gamma * p / rho) * chord / reynolds

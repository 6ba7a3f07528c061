"""Generates the golden fixtures in tests/golden/ from the reference.

Inputs copied (xz-compressed) from the reference repository's own fixtures:
  naca_2D_shape_0.msh   mesh of optimisation iteration 0 (25,274 quads)
  naca_2D_flow_0/1      cell states before / after iteration 0's time loop
  naca_2D_shape_params_0.txt

Outputs: golden.json -- SHA-256 digests (of the little-endian float64 bytes),
norms and sample values of the arrays that the reference's OWN code
(compiled by oracle/build_ref.sh) produces on (shape_0, flow_1), one thread,
no FMA contraction:
  residual: R, grad, edge_LR, edge_tau, forces
  jt:   y = J^T x with x ~ N(0,1), numpy default_rng(0)
  rhs:  assembleAdjointRHS with beta from the params file
  grad: computeShapeGradient with lambda = 1e-3 * N(0,1), default_rng(1)
and the topology arrays of the reference Mesh.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import lzma
import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402

REF = ref.REF_DIR / "mesh_opti"
FILES = ["naca_2D_shape_0.msh", "naca_2D_flow_0", "naca_2D_flow_1"]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).astype("<f8" if a.dtype.kind == "f" else "<i8").tobytes()).hexdigest()


def summary(a: np.ndarray) -> dict:
    a = np.asarray(a)
    d = {"sha256": digest(a), "size": int(a.size)}
    if a.dtype.kind == "f":
        d.update(l2=float(np.sqrt(np.sum(a * a))), head=[float(x) for x in a[:6]])
    return d


def main() -> None:
    if not ref.available():
        ref.build()
    for f in FILES:
        with open(REF / f, "rb") as src, lzma.open(HERE / (f + ".xz"), "wb", preset=9) as dst:
            shutil.copyfileobj(src, dst)
    shutil.copyfile(REF / "naca_2D_shape_params_0.txt", HERE / "naca_2D_shape_params_0.txt")
    os.chmod(HERE / "naca_2D_shape_params_0.txt", 0o644)
    out: dict = {"source": "reference src/*.cpp compiled by oracle/build_ref.sh (o2f_ref_exact, 1 thread)"}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        cfg = ref.write_config(td / "cfg.txt", mesh=str(REF / "naca_2D_shape_0.msh"),
                               state=str(REF / "naca_2D_flow_1"),
                               params_file=str(REF / "naca_2D_shape_params_0.txt"))
        topo = ref.run("topo", cfg)
        out["topology"] = {k: summary(v) for k, v in sorted(topo.items())}
        res = ref.run("residual", cfg)
        out["residual"] = {k: summary(v) for k, v in sorted(res.items())}
        out["forces"] = [float(x) for x in res["forces"]]
        nc = res["R"].size // 4
        x = np.random.default_rng(0).standard_normal(4 * nc)
        x.tofile(td / "x.f64")
        out["jt"] = summary(ref.run("jt", cfg, td / "x.f64")["jt_y"])
        out["rhs"] = summary(ref.run("rhs", cfg)["rhs_b"])
        lam = 1e-3 * np.random.default_rng(1).standard_normal(4 * nc)
        lam.tofile(td / "lam.f64")
        g = ref.run("grad", cfg, td / "lam.f64")
        out["shape_grad"] = [float(v) for v in g["shape_grad"]]
        out["rms_R_rho"] = float(np.sqrt(np.mean(res["R"][0::4] ** 2)))
    (HERE / "golden.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "golden.json")


if __name__ == "__main__":
    main()

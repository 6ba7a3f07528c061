"""Test infrastructure only: runs the reference solver's own code (built by
oracle/build_ref.sh into oracle/_ref/) as a subprocess and reads its dumps.

One process per call, because the reference sizes function-static scratch
buffers on its first residual (src/advection.cpp:9-23, src/diffusion.cpp:9-25).
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# The reference checkout: $O2F_REFERENCE_DIR, else a directory named
# "reference" beside this repository's checkout.
REF_DIR = Path(os.environ.get("O2F_REFERENCE_DIR", str(HERE.parent.parent / "reference")))
EXE_EXACT = HERE / "_ref" / "o2f_ref_exact"
EXE_FAST = HERE / "_ref" / "o2f_ref_fast"


EXE_ADAPTER = HERE / "_ref" / "o2f_adapter_check"


def available() -> bool:
    return EXE_EXACT.exists() and EXE_ADAPTER.exists()


def stale() -> bool:
    """True when a built binary is missing or older than a source it is built
    from here (the harness, the adapter check, the adapter and the C ABI
    header it compiles in)."""
    if not available():
        return True
    root = HERE.parent
    deps = [HERE / "ref_harness.cpp", HERE / "adapter_check.cpp", HERE / "build_ref.sh", root / "include" / "o2f.h",
            root / "optimisation2forme_b200" / "adapters" / "navier_stokes_o2f.cpp"]
    t = min(EXE_EXACT.stat().st_mtime, EXE_ADAPTER.stat().st_mtime)
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build() -> bool:
    """Compile the reference from its sources when they are present."""
    if (REF_DIR / "src" / "advection.cpp").exists():
        subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True, env={**os.environ, "REF_DIR": str(REF_DIR)},
                       capture_output=True)
        return True
    return False


def write_binary_mesh(path: Path, mesh: dict) -> Path:
    """The binary model variant read by oracle/shims/gmsh.h: the same groups
    as meshgen.write_msh2 (FreeStream 1, Airfoil 2, Fluid 3), same orders."""
    xy = np.asarray(mesh["node_xy"], dtype=np.float64).reshape(-1, 2)
    seg = np.asarray(mesh["segments"], dtype=np.int64).reshape(-1, 2)
    bc = np.asarray(mesh["segment_bc"])
    offs = np.asarray(mesh["cell_offsets"], dtype=np.int64)
    cn = np.asarray(mesh["cell_nodes"], dtype=np.int64)
    sizes = np.diff(offs)
    with open(path, "wb") as fh:
        fh.write(b"O2FMSHB1")
        fh.write(np.int64(len(xy)).tobytes())
        fh.write(np.concatenate([xy, np.zeros((len(xy), 1))], axis=1).astype("<f8").tobytes())
        names = [(1, 1, b"FreeStream"), (1, 2, b"Airfoil"), (2, 3, b"Fluid")]
        fh.write(np.int64(len(names)).tobytes())
        for d, t, n in names:
            fh.write(np.array([d, t, len(n)], dtype="<i4").tobytes() + n)
        fh.write(np.int64(len(seg) + len(sizes)).tobytes())
        tag = np.where(bc == ord("f"), 1, 2)
        hdr_seg = np.stack([np.ones(len(seg), dtype=np.int64), tag, tag], axis=1)
        hdr_cell = np.stack([np.where(sizes == 3, 2, 3), np.full(len(sizes), 3), np.full(len(sizes), 3)], axis=1)
        fh.write(np.concatenate([hdr_seg, hdr_cell]).astype("<i4").tobytes())
        fh.write((np.concatenate([seg.reshape(-1), cn]) + 1).astype("<i8").tobytes())
    return Path(path)


def write_config(path: Path, *, mesh: str, state: str = "", params_file: str = "", viscosity=1.8e-5,
                 inflow_velocity=0.3, cfl=0.5, final_time=0.005, Pr=0.71, extra: str = "") -> Path:
    """A reference config file (keys of src/params.cpp:35-77)."""
    txt = (f"viscosity = {viscosity!r}\nPr = {Pr!r}\ncfl_number = {cfl!r}\nfinal_time = {final_time!r}\n"
           f"verbosity = 0\nreload_config = 0\ninitial_condition = one_x\nboundary_conditions = inflow_outflow_x\n"
           f"noise_level = 0\ninflow_velocity = {inflow_velocity!r}\nmesh_name = {mesh}\n")
    if state:
        txt += f"state_load_path = {state}\n"
    if params_file:
        txt += f"shape_param_file = {params_file}\n"
    Path(path).write_text(txt + extra)
    return Path(path)


def run(mode: str, config: Path, *args: str, exact: bool = True, threads: int = 1, capture=False) -> dict:
    """Run one harness mode; returns {name: array} of its dumps (or stdout)."""
    exe = EXE_EXACT if exact else EXE_FAST
    with tempfile.TemporaryDirectory() as td:
        env = {**os.environ, "OMP_NUM_THREADS": str(threads)}
        r = subprocess.run([str(exe), mode, str(config), td, *map(str, args)], cwd=td, env=env, capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({mode}): {r.stderr.strip()}")
        if capture:
            return {"stdout": r.stdout}
        out = {}
        for f in Path(td).iterdir():
            if f.suffix == ".f64":
                out[f.stem] = np.fromfile(f, dtype=np.float64)
            elif f.suffix == ".i64":
                out[f.stem] = np.fromfile(f, dtype=np.int64)
        return out

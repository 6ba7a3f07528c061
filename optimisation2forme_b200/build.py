"""Build recipe for the native library ``optimisation2forme_b200/libo2f.so``.

The library is compiled in-tree with nvcc for sm_100a only.  Device code that
runs in FP64 is compiled with ``-fmad=false`` so that no multiply-add is
contracted: the FP64 residual then rounds exactly like the reference's x86-64
build.  Host C++ is compiled with ``-ffp-contract=off`` for the same reason
(interpolation weights and geometry are computed on the host).

Usage: ``python -m optimisation2forme_b200.build`` (or ``build()`` from Python).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libo2f.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libo2f.so")


def _cutlass_include() -> str:
    """CUTLASS/CuTe headers (the tcgen05 descriptor layouts of the warm-start
    GEMM): $O2F_CUTLASS_INCLUDE, else the copy vendored with flashinfer."""
    import importlib.util
    env = os.environ.get("O2F_CUTLASS_INCLUDE")
    if env and (Path(env) / "cute").is_dir():
        return env
    spec = importlib.util.find_spec("flashinfer")
    for loc in (spec.submodule_search_locations or []) if spec else []:
        cand = Path(loc) / "data" / "cutlass" / "include"
        if (cand / "cute" / "arch" / "mma_sm100_desc.hpp").exists():
            return str(cand)
    raise RuntimeError("CUTLASS headers not found: set O2F_CUTLASS_INCLUDE to a CUTLASS include directory")


def _deps(src: Path) -> list[Path]:
    return [src] + sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "o2f.h"]


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... ({r.returncode})")


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every translation unit that is out of date and link libo2f.so."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    inc = [f"-I{INCLUDE}", f"-I{CSRC}"]
    host_flags = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp", "-Wall", "-Wno-unused-function"]
    cuda_inc = ["-I/usr/local/cuda/include"]
    objs = []
    jobs = []
    for src in sorted(CSRC.glob("*.cpp")):
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, _deps(src)):
            jobs.append(["g++", *host_flags, *inc, *cuda_inc, "-c", str(src), "-o", str(obj)])
    for src in sorted(CSRC.glob("*.cu")):
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        # FP64 parity code: no FMA contraction.  Mixed-precision and network
        # code: contraction on; the network also needs the CUTLASS headers.
        learned = src.stem.startswith("mlp")
        fmad = "-fmad=true" if src.stem.endswith("_f32") or learned else "-fmad=false"
        extra = [f"-I{_cutlass_include()}"] if learned else []
        if src.stem.endswith("_f32"):
            # FP32 residual: approximate division and square root, FP32
            # denormals flushed (FP64 code in the unit is unaffected)
            extra += ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
        if force or _stale(obj, _deps(src)):
            jobs.append([nvcc, *ARCH, "-O3", "-std=c++17", "-lineinfo", fmad, "--expt-relaxed-constexpr",
                         "-Xcompiler", "-fPIC,-ffp-contract=off", *inc, *extra, "-c", str(src), "-o", str(obj)])
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(out)
        elif verbose and out.strip():
            sys.stderr.write(out)
    if failed:
        raise RuntimeError("compilation of libo2f failed")
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl",
              "-lpthread", "-lgomp"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)

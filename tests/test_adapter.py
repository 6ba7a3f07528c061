"""The C++ adapter with the reference's own signatures compiles against the
reference's headers (compile only; the reference tree is present where the
reference is vendored for the oracle, absent elsewhere)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

from oracle import ref

ROOT = Path(__file__).resolve().parents[1]
REF = Path(ref.REF_DIR)


@pytest.mark.skipif(not (REF / "include" / "shape_optimization.hpp").exists() or shutil.which("g++") is None,
                    reason="reference headers or g++ absent")
def test_adapter_compiles_against_the_reference_headers():
    src = ROOT / "optimisation2forme_b200" / "adapters" / "navier_stokes_o2f.cpp"
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-Wall", f"-I{ROOT / 'include'}", f"-I{REF / 'include'}",
           f"-I{ROOT / 'oracle' / 'shims'}", str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

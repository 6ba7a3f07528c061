"""Host part of the consistent adjoint on the CPU: the Jacobian stencil is the
two-vertex-ring neighbourhood, symmetric, and its colouring leaves no two
cells of a colour in any stencil (tests/stencil_check.cpp, compiled with the
library's mesh_host.cpp)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is needed to compile the check")
def test_stencil_and_colouring(tmp_path):
    exe = tmp_path / "stencil_check"
    csrc = ROOT / "optimisation2forme_b200" / "csrc"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", f"-I{ROOT / 'include'}", f"-I{csrc}",
                    str(ROOT / "tests" / "stencil_check.cpp"), str(csrc / "mesh_host.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr

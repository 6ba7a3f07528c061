"""The residual kernels' shared-reciprocal quotients (csrc/qdiv.h) against IEEE
division, on the CPU: the header is host/device code, compiled here with g++
into tests/qdiv_check.cpp.  Random operands, the quotients closest to a
rounding midpoint that 53-bit operands allow, and special values must all
give the bits of a/b, which is what keeps the FP64 residual bit-identical to
the reference's."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is needed to compile the check")
def test_qdiv_equals_ieee_division(tmp_path):
    exe = tmp_path / "qdiv_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{ROOT / 'optimisation2forme_b200' / 'csrc'}",
                    str(ROOT / "tests" / "qdiv_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "2000000", "40000", "7"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout

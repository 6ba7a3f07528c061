"""The std::unordered_set iteration-order emulation used by the GPU mesh
build (csrc/uset_order.h) against the container itself, on the CPU: random
and ascending insertion sequences of every length up to the emulation's
limit (tests/uset_order_check.cpp)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ is needed to compile the check")
def test_emulated_order_equals_std_unordered_set(tmp_path):
    exe = tmp_path / "uset_order_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{ROOT / 'optimisation2forme_b200' / 'csrc'}",
                    str(ROOT / "tests" / "uset_order_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), "300000", "5"], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout

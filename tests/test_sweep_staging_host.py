"""Index arithmetic of the block ILU sweep's shared-memory staging
(optimisation2forme_b200/csrc/ilu.cuh: sweep_stage_chunks, sweep_stage_level,
sweep_cta_row), restated on the host: for random partitions of n positions
into levels, every staged copy reads inside the packed factor copy and writes
inside its buffer, every staged read of a row lands on what was copied for
it, and the shared-memory total stays within the per-block limit."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

ILU = Path(__file__).resolve().parents[1] / "optimisation2forme_b200" / "csrc" / "ilu.cuh"


def _const(name: str, env: dict) -> int:
    m = re.search(rf"constexpr\s+(?:int|size_t)\s+{name}\s*=\s*([^;]+);", ILU.read_text())
    assert m, name
    expr = m.group(1).replace("sizeof(Vec4<double>)", "32").replace("sizeof(double)", "8")
    return int(eval(expr, {}, env))  # the header's own constant expressions


def _consts() -> dict:
    env: dict = {}
    for name in ("kSweepWindow", "kStageSlots", "kStageChunkDoubles", "kStageChunksFwd", "kStageChunksBwd",
                 "kStageBwdD", "kStageDoubles", "kSweepSmem"):
        env[name] = _const(name, env)
    return env


def stage_chunks(b: int, e: int, cap: int) -> int:
    if b >= e:
        return 0
    return min(((e - 1) >> 5) - (b >> 5) + 1, cap)


@pytest.mark.parametrize("forward", [True, False])
@pytest.mark.parametrize("seed", range(6))
def test_staged_copies_and_reads_stay_in_bounds(forward: bool, seed: int):
    k = _consts()
    assert k["kSweepSmem"] <= 227 * 1024
    assert k["kStageBwdD"] + k["kStageChunksBwd"] * 512 <= k["kStageDoubles"]
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 5000))
    n32 = (n + 31) // 32 * 32
    pack_len = n32 * 144  # doubles, as allocated for the block sweeps
    dir_base = 0 if forward else n32 * 64
    cap = k["kStageChunksFwd"] if forward else k["kStageChunksBwd"]
    cd = k["kStageChunkDoubles"]
    # random level sizes, including levels wider than the staged chunks
    sizes = []
    left = n
    while left:
        s = int(min(left, rng.choice([1, 3, 31, 32, 33, 121, 400, 700])))
        sizes.append(s)
        left -= s
    b = 0
    for s in sizes:
        e = b + s
        nch = stage_chunks(b, e, cap)
        pieces = cd // 2
        src0 = dir_base + (b >> 5) * 2048
        copied = {}
        for kk in range(nch * pieces):  # sweep_stage_level, factor blocks
            ch, pc = divmod(kk, pieces)
            dst = ch * cd + 2 * pc
            src = src0 + ch * 2048 + 2 * pc
            assert 0 <= dst and dst + 2 <= k["kStageDoubles"]
            assert dir_base <= src and src + 2 <= dir_base + n32 * 64 <= pack_len
            assert src % 2 == 0 and dst % 2 == 0  # 16-byte pieces
            copied[dst], copied[dst + 1] = src, src + 1
        if not forward:  # D^-1
            srcD0 = 2 * n32 * 64 + (b >> 5) * 512
            for kk in range(nch * 256):
                dst = k["kStageBwdD"] + 2 * kk
                src = srcD0 + 2 * kk
                assert dst + 2 <= k["kStageDoubles"] and src + 2 <= pack_len
                copied[dst], copied[dst + 1] = src, src + 1
        for p in range(b, e):  # sweep_cta_row: staged reads equal the packed element
            ch = (p >> 5) - (b >> 5)
            assert ch >= 0
            if ch >= nch:
                continue
            for d in range(k["kStageSlots"]):
                for el in range(16):
                    smem = ch * cd + d * 512 + el * 32 + (p & 31)
                    glob = dir_base + (p >> 5) * 2048 + d * 512 + el * 32 + (p & 31)
                    assert copied[smem] == glob
            if not forward:
                for el in range(16):
                    smem = k["kStageBwdD"] + ch * 512 + el * 32 + (p & 31)
                    assert copied[smem] == 2 * n32 * 64 + (p >> 5) * 512 + el * 32 + (p & 31)
        b = e
    assert b == n

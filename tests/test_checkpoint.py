"""Binary state checkpoint (o2f_checkpoint_write / _read), on the CPU: the
values of the reference's text state file, bit for bit, and the errors the
reference's loadCellStates raises (src/utils.cpp:29-67) for a missing,
damaged or mismatched file."""
from __future__ import annotations

import numpy as np
import pytest

from optimisation2forme_b200 import (O2FError, load_cell_states, load_state_binary, save_cell_states,
                                     save_state_binary)


def _state(n, seed=0):
    rng = np.random.default_rng(seed)
    U = rng.standard_normal(4 * n) * np.tile([1.0, 300.0, 30.0, 2.5e5], n)
    U[::4] = np.abs(U[::4]) + 0.5
    U[5] = -0.0
    U[9] = np.nextafter(1.0, 2.0)
    U[13] = 5e-324  # subnormal
    return U


def test_round_trip_is_exact_and_matches_the_text_file(tmp_path):
    U = _state(1000)
    save_state_binary(tmp_path / "s.bin", U, time=0.125, steps=4321)
    V, t, steps = load_state_binary(tmp_path / "s.bin", 1000)
    assert np.array_equal(V.view(np.int64), U.view(np.int64)) and (t, steps) == (0.125, 4321)
    # text (reference format, 17 significant digits) -> binary -> same bits
    save_cell_states(tmp_path / "s.txt", U)
    W = load_cell_states(tmp_path / "s.txt", 1000)
    save_state_binary(tmp_path / "w.bin", W)
    X, _, _ = load_state_binary(tmp_path / "w.bin", 1000)
    assert np.array_equal(X.view(np.int64), U.view(np.int64))
    # layout: 64-byte header, then rho[], rho_u[], rho_v[], E[] as float64
    raw = (tmp_path / "s.bin").read_bytes()
    assert raw[:7] == b"O2FSOA1" and len(raw) == 64 + 32 * 1000
    fields = np.frombuffer(raw[64:], dtype="<f8").reshape(4, 1000)
    assert np.array_equal(fields.T.reshape(-1).view(np.int64), U.view(np.int64))


def _expect_io(path, n):
    with pytest.raises(O2FError) as e:
        load_state_binary(path, n)
    assert e.value.status == "O2F_ERR_IO"
    return str(e.value)


def test_damaged_or_mismatched_files_are_rejected(tmp_path):
    U = _state(64, seed=1)
    good = tmp_path / "g.bin"
    save_state_binary(good, U)
    raw = bytearray(good.read_bytes())
    assert "cannot open" in _expect_io(tmp_path / "missing.bin", 64)
    assert "65 in the mesh" in _expect_io(good, 65)  # wrong cell count
    (tmp_path / "t.bin").write_bytes(raw[:-8])
    assert "truncated" in _expect_io(tmp_path / "t.bin", 64)
    (tmp_path / "x.bin").write_bytes(raw + b"\0")
    assert "trailing" in _expect_io(tmp_path / "x.bin", 64)
    flipped = bytearray(raw)
    flipped[64 + 100] ^= 1
    (tmp_path / "c.bin").write_bytes(flipped)
    assert "checksum" in _expect_io(tmp_path / "c.bin", 64)
    foreign = bytearray(raw)
    foreign[0:4] = b"JUNK"
    (tmp_path / "f.bin").write_bytes(foreign)
    assert "not an o2f" in _expect_io(tmp_path / "f.bin", 64)
    (tmp_path / "s.txt").write_text("64\n")  # the text format is not a checkpoint
    _expect_io(tmp_path / "s.txt", 64)

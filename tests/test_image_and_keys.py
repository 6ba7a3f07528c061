"""Host pieces without a GPU: the image writer (PNG decoded back with zlib,
binary PPM read back) and the configuration keys added without a reference
counterpart (parsed from a reference-syntax file, mapped into o2f_params)."""
from __future__ import annotations

import struct
import zlib

import numpy as np


def _read_png(path):
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(data):
        n, tag = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(tag + body) & 0xFFFFFFFF
        if tag == b"IHDR":
            w, h, depth, colour = struct.unpack(">IIBB", body[:10])
            assert (depth, colour) == (8, 2)
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = [raw[r * (3 * w + 1):(r + 1) * (3 * w + 1)] for r in range(h)]
    assert all(row[0] == 0 for row in rows)  # filter type 0
    return np.frombuffer(b"".join(row[1:] for row in rows), dtype=np.uint8).reshape(h, w, 3)


def test_png_and_ppm_round_trip(tmp_path):
    from optimisation2forme_b200 import write_image
    img = np.random.default_rng(3).integers(0, 256, size=(17, 23, 3), dtype=np.uint8)
    write_image(tmp_path / "a.png", img)
    assert np.array_equal(_read_png(tmp_path / "a.png"), img)
    write_image(tmp_path / "b.ppm", img)
    raw = (tmp_path / "b.ppm").read_bytes()
    head = b"P6\n23 17\n255\n"
    assert raw.startswith(head) and np.array_equal(np.frombuffer(raw[len(head):], np.uint8).reshape(17, 23, 3), img)


def test_new_keys_parse_and_map(tmp_path):
    from optimisation2forme_b200 import load_config
    cfg = tmp_path / "c.txt"
    cfg.write_text("adjoint_jacobian = frozen_limiter\nadjoint_fd_step = 1e-8\ndt_mode = thermal\n"
                   "adjoint_precond = none\n# later keys override\nadjoint_jacobian = full\n")
    p = load_config(cfg)
    assert (p.adjoint_jacobian, p.adjoint_fd_step, p.dt_mode, p.adjoint_precond) == ("full", 1e-8, "thermal", "none")
    c = p.to_c()
    assert (c.adjoint_jacobian, c.adjoint_fd_step, c.dt_mode, c.adjoint_precond) == (1, 1e-8, 1, 0)
    from optimisation2forme_b200 import SimulationParams
    d = SimulationParams().to_c()  # defaults reproduce the reference
    assert (d.adjoint_jacobian, d.adjoint_precond, d.dt_mode, d.precision) == (0, 1, 0, 0)

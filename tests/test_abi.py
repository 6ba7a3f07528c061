"""The C-ABI library: loads without a GPU, exports every symbol that
include/o2f.h declares, and rejects bad host-side input with a status."""
from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, desc_of, small_mesh


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms.update(re.findall(r"\b(o2f_[a-z0-9_]+)\s*\(", txt))
    return sorted(syms)


def test_every_declared_symbol_is_exported():
    from optimisation2forme_b200 import LIB_PATH, lib
    lib()
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (o2f_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    assert len(declared_symbols()) >= 25


def test_library_targets_sm100a_only():
    from optimisation2forme_b200 import LIB_PATH
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", str(LIB_PATH)], capture_output=True,
                         text=True).stdout
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def test_defaults_mirror_reference_params():
    from optimisation2forme_b200 import _lib
    p = _lib.Params()
    _lib.lib().o2f_params_default(C.byref(p))
    assert (p.gamma, p.Pr, p.cp, p.rho_ref, p.p_ref, p.limiter_k) == (1.4, 0.71, 1005.0, 1.225, 101325.0, 1e-2)


def test_host_mesh_errors_are_statuses(tmp_path):
    from optimisation2forme_b200 import HostMesh, O2FError
    with pytest.raises(O2FError) as e:
        HostMesh(tmp_path / "missing.msh")
    assert e.value.status == "O2F_ERR_IO"
    m = small_mesh(triangles=True, n_surface=16, n_layers=4)
    bad = dict(m)
    bad["segments"] = m["segments"][:-2]  # a boundary edge without a code
    bad["segment_bc"] = m["segment_bc"][:-1]
    with pytest.raises(O2FError) as e:
        HostMesh(desc=desc_of(bad))
    assert e.value.status == "O2F_ERR_MESH"
    bad = dict(m)
    bad["cell_nodes"] = m["cell_nodes"].copy()
    bad["cell_nodes"][0] = 10 ** 9
    with pytest.raises(O2FError) as e:
        HostMesh(desc=desc_of(bad))
    assert e.value.status == "O2F_ERR_MESH"
    # the same triangle twice more: an edge shared by more than two cells
    bad = dict(m)
    extra = m["cell_nodes"][:3]
    bad["cell_nodes"] = np.concatenate([m["cell_nodes"], extra, extra])
    bad["cell_offsets"] = np.concatenate([m["cell_offsets"], m["cell_offsets"][-1] + np.array([3, 6])])
    with pytest.raises(O2FError):
        HostMesh(desc=desc_of(bad))


def test_msh_reader_errors(tmp_path):
    from optimisation2forme_b200 import HostMesh, O2FError
    f = tmp_path / "bad.msh"
    f.write_text("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
    with pytest.raises(O2FError) as e:
        HostMesh(f)
    assert e.value.status == "O2F_ERR_IO"


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """Every struct of include/o2f.h has the size and field offsets that the
    ctypes mirror in _lib.py uses (a C program compiled here prints them)."""
    import shutil
    from optimisation2forme_b200 import _lib
    if shutil.which("gcc") is None:
        pytest.skip("gcc is needed")
    mirrors = {"o2f_params": _lib.Params, "o2f_mesh_desc": _lib.MeshDesc, "o2f_shape_params": _lib.ShapeParams,
               "o2f_mesh_info": _lib.MeshInfo, "o2f_timing": _lib.Timing}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "o2f.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, out):
        cname, field, value = line.split()
        cls = mirrors[cname]
        want = C.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert int(value) == want, line

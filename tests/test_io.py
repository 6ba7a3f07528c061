"""Boundary formats: the reference config file, the shape parameter file,
the cell-state text file (src/params.cpp:18-83,
src/shape_optimization.cpp:19-145, src/utils.cpp:29-107)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN


def test_load_config_later_keys_win(tmp_path):
    from optimisation2forme_b200 import load_config
    f = tmp_path / "c.txt"
    f.write_text("# comment\ncfl_number = 0.2\ninflow_velocity = 0.3\nunknown_key = 7\n\ncfl_number   = 0.5\n"
                 "boundary_conditions = inflow_outflow_x\nmesh_name = a.msh\naoa_deg = 1.5\n")
    p = load_config(f)
    assert (p.cfl_number, p.inflow_velocity, p.mesh_name, p.aoa_deg) == (0.5, 0.3, "a.msh", 1.5)
    f.write_text("boundary_conditions = bogus\n")
    with pytest.raises(ValueError):
        load_config(f)


def test_load_params_generic_stars_and_overrides(tmp_path):
    from optimisation2forme_b200 import load_params_generic
    names, vals, opt = load_params_generic(GOLDEN / "naca_2D_shape_params_0.txt")
    assert names == ["pos_x", "c", "m", "p", "t", "beta"] and opt == ["m", "p"]
    assert vals == [0.355, 1.0, 0.0, 0.4, 0.12, 50.0]
    f = tmp_path / "p.txt"
    f.write_text("m *= 0.1 # camber\np *= 0.3\nm = 0.2\nq 3\n")
    names, vals, opt = load_params_generic(f)
    assert opt == ["p"] and dict(zip(names, vals)) == {"m": 0.2, "p": 0.3, "q": 3.0}


def test_cell_state_round_trip_and_errors(tmp_path, golden_dir):
    from optimisation2forme_b200 import load_cell_states, save_cell_states
    U = load_cell_states(golden_dir / "naca_2D_flow_1", 25274)
    save_cell_states(tmp_path / "s", U)
    assert np.array_equal(load_cell_states(tmp_path / "s", 25274), U)
    with pytest.raises(ValueError):
        load_cell_states(tmp_path / "s", 25273)
    (tmp_path / "t").write_text("3\n1 2 3 4\n")
    with pytest.raises(ValueError):
        load_cell_states(tmp_path / "t", 3)


def test_shape_log_format(tmp_path):
    from optimisation2forme_b200 import write_shape_log
    write_shape_log(tmp_path / "log", ["m", "p"], 14.35, [-216350.0, 1230.0])
    assert (tmp_path / "log").read_text() == " J=14.35000000 m=-2.163500e+05 p=1.230000e+03\n"

"""The C ABI on the CPU: the library loads, exports every declared symbol,
validates its arguments, and its host-only functions agree with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import alsvinn_b200
from alsvinn_b200 import _lib
from conftest import ROOT, load_golden

HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = []
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(als_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.PROTOTYPES, "binding missing for " + name


def test_ghost_cells():
    assert alsvinn_b200.ghost_cells("hll", "weno2") == 2
    assert alsvinn_b200.ghost_cells("hll3", "eno3") == 3
    assert alsvinn_b200.ghost_cells("central", "eno4") == 4
    assert alsvinn_b200.ghost_cells("hll", "none") == 1
    assert alsvinn_b200.ghost_cells("tecno1", "none") == 1
    assert alsvinn_b200.ghost_cells("tecno4", "none") == 3
    assert alsvinn_b200.ghost_cells("tecno6", "none") == 5
    with pytest.raises(_lib.AlsError):
        alsvinn_b200.ghost_cells("tecno4", "weno2")   # TeCNO fluxes: reconstruction "none"
    with pytest.raises(_lib.AlsError):
        alsvinn_b200.ghost_cells(7, 1)


def test_uniform_draws_match_reference_generator():
    z = load_golden("stlmersenne_40x3")
    np.testing.assert_array_equal(alsvinn_b200.uniform_draws(40, 0, 3), z["draws"])
    np.testing.assert_array_equal(alsvinn_b200.uniform_draws(40, 1, 2), z["draws"][1:])


def test_compute_timestep_matches_integrator_formula():
    lib = _lib.load()
    D = ctypes.POINTER(ctypes.c_double)
    ws = np.array([1.3, 0.7, 0.0])
    cl = np.array([1 / 512, 1.0, 1.0])
    dt = lib.als_compute_timestep(ws.ctypes.data_as(D), cl.ctypes.data_as(D), 0.45, 0.0, 0.2)
    total = 0.0
    for d in range(3):
        total += ws[d] / cl[d]
    assert dt == min(0.45 / total, 0.2)
    dt = lib.als_compute_timestep(ws.ctypes.data_as(D), cl.ctypes.data_as(D), 0.45, 0.19999, 0.2)
    assert dt == 0.2 - 0.19999


@pytest.mark.parametrize("field,value", [("dimension", 4), ("flux", 9), ("reconstruction", -1),
                                         ("integrator", 5), ("boundary", 3), ("members", 0),
                                         ("precision", 2), ("cfl", 0.0)])
def test_solver_rejects_invalid_configuration(field, value):
    lib = _lib.load()
    cfg = _lib.SolverConfig()
    cfg.dimension = 2
    cfg.n[0] = cfg.n[1] = 16
    cfg.n[2] = 1
    cfg.upper[0] = cfg.upper[1] = 1.0
    cfg.gamma = 1.4
    cfg.cfl = 0.4
    cfg.end_time = 1.0
    cfg.members = 1
    setattr(cfg, field, value)
    h = ctypes.c_void_p()
    rc = lib.als_solver_create(ctypes.byref(cfg), 0, ctypes.byref(h))
    assert rc == -1
    assert lib.als_last_error()


def test_solver_rejects_grids_smaller_than_two_ghost_widths():
    with pytest.raises(_lib.AlsError) as e:
        alsvinn_b200.Simulator(2, (3, 16), (0, 0), (1, 1), reconstruction="weno2")
    assert e.value.code == -1

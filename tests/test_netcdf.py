"""Snapshot files with the layout of alsfvm::io::NetCDFWriter, read back with
an independent reader (scipy.io.netcdf_file, classic NetCDF)."""
import ctypes
import os
import tempfile

import numpy as np
import pytest
from scipy.io import netcdf_file

from alsvinn_b200 import _lib

pytestmark = []


def _write(path, dim, n, arrays, names, time, attrs):
    lib = _lib.load()
    nn = (ctypes.c_int * 3)(*(list(n) + [1, 1, 1])[:3])
    cname = (ctypes.c_char_p * len(names))(*[s.encode() for s in names])
    data = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
    ptrs = (ctypes.c_void_p * len(data))(*[a.ctypes.data for a in data])
    an = (ctypes.c_char_p * len(attrs))(*[k.encode() for k in attrs])
    av = (ctypes.c_char_p * len(attrs))(*[v.encode() for v in attrs.values()])
    return lib.als_write_netcdf(path.encode(), dim, nn, len(names),
                                ctypes.cast(cname, ctypes.POINTER(ctypes.c_void_p)),
                                ctypes.cast(ptrs, ctypes.POINTER(ctypes.c_void_p)), time,
                                len(attrs), ctypes.cast(an, ctypes.POINTER(ctypes.c_void_p)),
                                ctypes.cast(av, ctypes.POINTER(ctypes.c_void_p)))


@pytest.mark.parametrize("dim,n", [(1, (17,)), (2, (5, 3)), (3, (4, 3, 2))])
def test_writer_layout_matches_the_reference_writer(dim, n):
    rng = np.random.default_rng(dim)
    names = {1: ["rho", "mx", "E"], 2: ["rho", "mx", "my", "E"],
             3: ["rho", "mx", "my", "mz", "E"]}[dim]
    nn = list(n) + [1] * (3 - dim)
    # interior cells in Volume::copyInternalCells order: x fastest
    arrays = [rng.normal(size=nn[0] * nn[1] * nn[2]) for _ in names]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "kh_3.nc")
        assert _write(path, dim, n, arrays, names, 0.125, {"alsvinn_b200.note": "test"}) == 0
        with netcdf_file(path, "r", mmap=False) as f:
            assert f.version_byte == 2
            assert f.dimensions == {"t": 1, "x": nn[0], "y": nn[1], "z": nn[2]}
            assert float(f.variables["time"][0]) == 0.125
            assert f.variables["time"].dimensions == ("t",)
            assert f._attributes["alsvinn_b200.note"] == b"test"
            for name, a in zip(names, arrays):
                v = f.variables[name]
                assert v.dimensions == ("x", "y", "z")
                # the reference's bytes: the flat array in x-fastest order
                np.testing.assert_array_equal(np.asarray(v[:]).reshape(-1), a)


def test_writer_rejects_bad_arguments():
    assert _write("/nonexistent-dir/x.nc", 2, (3, 3), [np.zeros(9)] * 4,
                  ["rho", "mx", "my", "E"], 0.0, {}) == -1
    assert _write("x.nc", 4, (3, 3), [np.zeros(9)] * 4, ["rho", "mx", "my", "E"], 0.0, {}) == -1


@pytest.mark.gpu
def test_solver_snapshot_holds_the_interior_state():
    import alsvinn_b200 as als
    states, _ = als.kh_ensemble(32, 0, 2)
    with als.Simulator(2, (32, 32), flux="hll3", reconstruction="weno2", cfl=0.4,
                       end_time=0.02, members=2) as sim:
        sim.set_state(states)
        sim.run()
        U = sim.get_state(1)[0]
        t = sim.info(1)["t"]
        with tempfile.TemporaryDirectory() as d:
            path = sim.write_netcdf(os.path.join(d, "kh"), snapshot=1, member=1)
            assert path.endswith("kh_1.nc")
            with netcdf_file(path, "r", mmap=False) as f:
                assert float(f.variables["time"][0]) == t
                for k, name in enumerate(["rho", "mx", "my", "E"]):
                    flat = np.asarray(f.variables[name][:]).reshape(-1)
                    np.testing.assert_array_equal(flat, U[k, 0, 2:-2, 2:-2].reshape(-1))

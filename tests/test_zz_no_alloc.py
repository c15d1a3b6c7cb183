"""The allocation-free flux entry point, als_compute_flux_static.

Some callers of the flux evaluation cannot let a library allocate device
memory (a runtime that owns and pre-plans all device memory, or one that
forbids allocation while it drives the time loop).  For them the library
keeps the wave-speed accumulators in a fixed device array.  These checks
call that entry point through the C ABI and compare it with the allocating
als_compute_flux on the same states: the net fluxes and wave speeds must be
identical (tolerance 0, like every FP64 comparison here), on two calls in a
row, because the fixed array keeps the previous call's contents.

This file sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from alsvinn_b200 import _lib
from oracle_lib import ghost_cells, smooth_random_state

pytestmark = pytest.mark.gpu

_D = ctypes.POINTER(ctypes.c_double)
FLUX = {"hll": 0, "hll3": 1, "central": 2}
RECON = {"none": 0, "weno2": 1, "eno2": 2, "eno3": 3, "eno4": 4}


def _grid(dim, n, g):
    grid = _lib.Grid()
    grid.dimension = dim
    nn = list(n) + [1] * (3 - len(n))
    for d in range(3):
        grid.n[d] = nn[d]
    grid.ghosts = g
    grid.gamma = 1.4
    return grid


def _states(seed, members, dim, n, g):
    lib = _lib.load()
    x = torch.from_numpy(np.stack([smooth_random_state(seed + k, dim, n, g)
                                   for k in range(members)])).cuda()
    grid = _grid(dim, n, g)
    for m in range(members):
        assert lib.als_fill_ghosts(ctypes.byref(grid), 1, _lib.plane_pointers(x[m]), dim + 2,
                                   None) == 0
    torch.cuda.synchronize()
    return x


def _allocating(x, dim, n, g, flux, recon):
    """als_compute_flux state by state (the entry point that allocates)."""
    lib = _lib.load()
    grid = _grid(dim, n, g)
    out = torch.zeros_like(x)
    ws = np.zeros((x.shape[0], 3))
    for m in range(x.shape[0]):
        w = np.zeros(3)
        rc = lib.als_compute_flux(ctypes.byref(grid), FLUX[flux], RECON[recon],
                                  _lib.plane_pointers(x[m]), _lib.plane_pointers(out[m]),
                                  None, None, w.ctypes.data_as(_D), None)
        assert rc == 0, lib.als_last_error()
        ws[m] = w
    return out, ws


def _static(x, dim, n, g, flux, recon):
    lib = _lib.load()
    grid = _grid(dim, n, g)
    out = torch.zeros_like(x)
    ws = np.zeros((x.shape[0], 3))
    rc = lib.als_compute_flux_static(ctypes.byref(grid), FLUX[flux], RECON[recon],
                                     ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     x.shape[0], ws.ctypes.data_as(_D), None)
    assert rc == 0, lib.als_last_error()
    return out, ws


@pytest.mark.parametrize("dim,n,flux,recon", [(2, (40, 36), "hll3", "weno2"),
                                              (1, (64,), "hll", "eno3"),
                                              (3, (10, 9, 12), "central", "weno2")])
def test_static_flux_matches_allocating_flux_twice(dim, n, flux, recon):
    g = ghost_cells(recon)
    # two calls in a row on different states: the second must not see the first's maxima
    for seed, members in ((11, 5), (901, 3)):
        x = _states(seed, members, dim, n, g)
        want_out, want_ws = _allocating(x, dim, n, g, flux, recon)
        got_out, got_ws = _static(x, dim, n, g, flux, recon)
        np.testing.assert_array_equal(got_ws, want_ws)
        np.testing.assert_array_equal(got_out.cpu().numpy(), want_out.cpu().numpy())


def test_static_flux_rejects_more_states_than_its_array_holds():
    lib = _lib.load()
    grid = _grid(2, (16, 16), 2)
    ws = np.zeros(3 * 1025)
    x = torch.zeros((4, 20, 20), dtype=torch.float64, device="cuda")
    rc = lib.als_compute_flux_static(ctypes.byref(grid), 0, 1, ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(x.data_ptr()), 1025, ws.ctypes.data_as(_D),
                                     None)
    assert rc == -1
    assert b"1024" in lib.als_last_error()


@pytest.mark.parametrize("entry", ["static", "allocating"])
def test_flux_calls_from_concurrent_threads(entry):
    """Four host threads, each on its own stream, call the flux entry point
    40 times on their own states; every result equals the serial one.  The
    static entry point shares one device array (calls on a device take
    turns), the allocating one keeps accumulators per thread."""
    import threading
    dim, n, g, flux, recon = 2, (48, 40), 2, "hll3", "weno2"
    states = [_states(900 + 10 * k, 2, dim, n, g) for k in range(4)]
    serial = [_static(x, dim, n, g, flux, recon) if entry == "static"
              else _allocating(x, dim, n, g, flux, recon) for x in states]
    lib = _lib.load()
    grid = _grid(dim, n, g)
    errors = []

    def worker(k):
        stream = torch.cuda.Stream()
        x = states[k]
        try:
            for _ in range(40):
                with torch.cuda.stream(stream):
                    out = torch.zeros_like(x)
                ws = np.zeros((x.shape[0], 3))
                handle = ctypes.c_void_p(stream.cuda_stream)
                if entry == "static":
                    rc = lib.als_compute_flux_static(
                        ctypes.byref(grid), FLUX[flux], RECON[recon], ctypes.c_void_p(x.data_ptr()),
                        ctypes.c_void_p(out.data_ptr()), x.shape[0], ws.ctypes.data_as(_D), handle)
                    assert rc == 0, lib.als_last_error()
                else:
                    for m in range(x.shape[0]):
                        w = np.zeros(3)
                        rc = lib.als_compute_flux(
                            ctypes.byref(grid), FLUX[flux], RECON[recon], _lib.plane_pointers(x[m]),
                            _lib.plane_pointers(out[m]), None, None, w.ctypes.data_as(_D), handle)
                        assert rc == 0, lib.als_last_error()
                        ws[m] = w
                stream.synchronize()
                assert torch.equal(out, serial[k][0])
                assert np.array_equal(ws, serial[k][1])
        except Exception as exc:   # reported by the main thread
            errors.append(exc)

    # each thread zeroes its outputs on its own stream; the states are
    # ready on every stream before the threads start
    torch.cuda.synchronize()
    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors[0]

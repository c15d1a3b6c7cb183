"""Python face of the C ABI, named after the reference's interfaces.

``Simulator`` wraps the fused device solver (``als_solver_*``): it is what
``alsvinncli``'s time loop (Simulator::performStep, Simulator.cpp:81-85,
191-214) and, with ``members > 1``, ``alsuqcli``'s sample loop
(alsuq/src/run/Runner.cpp:42-78) become.  The plug-in level calls
(``NumericalFlux``, ``Reconstruction``, ``Boundary``, ``Integrator``) take
device tensors and mirror one virtual call of the reference each.
"""
import ctypes

import numpy as np

from . import _lib
from .initial_data import padded_shape

FLUX = {"hll": 0, "hll3": 1, "central": 2}
RECONSTRUCTION = {"none": 0, "weno2": 1, "eno2": 2, "eno3": 3, "eno4": 4}
INTEGRATOR = {"forwardeuler": 0, "rungekutta2": 1, "rungekutta3": 2}
BOUNDARY = {"neumann": 0, "periodic": 1}
PRECISION = {"fp64": 0, "fp32": 1}
EQUATION = {"euler1": 1, "euler2": 2, "euler3": 3}

_D = ctypes.POINTER(ctypes.c_double)


def _choice(table, value, what):
    if isinstance(value, int):
        return value
    try:
        return table[value]
    except KeyError:
        raise ValueError("unknown %s %r (known: %s)" % (what, value, ", ".join(table))) from None


def ghost_cells(flux, reconstruction):
    lib = _lib.load()
    return _lib.check(lib.als_ghost_cells(_choice(FLUX, flux, "flux"),
                                          _choice(RECONSTRUCTION, reconstruction, "reconstruction")))


class Simulator:
    """Advances one simulation, or an ensemble of ``members`` simulations of
    the same grid, by whole time steps on the GPU."""

    def __init__(self, dimension, n, lower, upper, flux="hll3", reconstruction="weno2",
                 integrator="rungekutta3", boundary="periodic", gamma=1.4, cfl=0.4,
                 end_time=1.0, max_steps=0, precision="fp64", members=1, device=0):
        lib = _lib.load()
        self._lib = lib
        cfg = _lib.SolverConfig()
        cfg.dimension = dimension
        nn = list(n) + [1] * (3 - len(n))
        lo = list(lower) + [0.0] * (3 - len(lower))
        hi = list(upper) + [0.0] * (3 - len(upper))
        for d in range(3):
            cfg.n[d] = int(nn[d])
            cfg.lower[d] = float(lo[d])
            cfg.upper[d] = float(hi[d])
        cfg.flux = _choice(FLUX, flux, "flux")
        cfg.reconstruction = _choice(RECONSTRUCTION, reconstruction, "reconstruction")
        cfg.integrator = _choice(INTEGRATOR, integrator, "integrator")
        cfg.boundary = _choice(BOUNDARY, boundary, "boundary")
        cfg.gamma = gamma
        cfg.cfl = cfl
        cfg.end_time = end_time
        cfg.max_steps = int(max_steps)
        cfg.precision = _choice(PRECISION, precision, "precision")
        cfg.members = int(members)
        self.config = cfg
        self.dimension = dimension
        self.n = tuple(int(v) for v in nn[:dimension])
        self.members = int(members)
        handle = ctypes.c_void_p()
        _lib.check(lib.als_solver_create(ctypes.byref(cfg), device, ctypes.byref(handle)))
        self._h = handle
        plane = ctypes.c_longlong()
        g = ctypes.c_int()
        _lib.check(lib.als_solver_geometry(self._h, ctypes.byref(plane), ctypes.byref(g)))
        self.plane = plane.value
        self.ghosts = g.value
        self.shape = padded_shape(dimension, self.n, self.ghosts)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.als_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_state(self, states, first_member=0):
        """Uploads FP64 host states of shape (members, nvar, Nz, Ny, Nx) or (nvar, Nz, Ny, Nx)."""
        a = np.ascontiguousarray(states, dtype=np.float64)
        if a.shape == self.shape:
            a = a[None]
        if a.shape[1:] != self.shape:
            raise ValueError("state shape %s does not match %s" % (a.shape, self.shape))
        _lib.check(self._lib.als_solver_set_state(self._h, a.ctypes.data_as(_D), first_member,
                                                  a.shape[0]))

    def set_state_device(self, ptr, first_member=0, count=None):
        count = self.members - first_member if count is None else count
        _lib.check(self._lib.als_solver_set_state_device(self._h, ctypes.c_void_p(ptr),
                                                         first_member, count))

    def get_state(self, first_member=0, count=None):
        count = self.members - first_member if count is None else count
        out = np.zeros((count,) + self.shape)
        _lib.check(self._lib.als_solver_get_state(self._h, out.ctypes.data_as(_D), first_member,
                                                  count))
        return out

    def state_pointer(self):
        p = ctypes.c_void_p()
        _lib.check(self._lib.als_solver_state_pointer(self._h, ctypes.byref(p)))
        return p.value

    def advance(self, steps):
        _lib.check(self._lib.als_solver_advance(self._h, int(steps)))

    def run(self):
        """Runs to the end time; raises AlsError(ALS_E_CONSTRAINT) on a
        constraint violation, like Simulator::checkConstraints throws."""
        _lib.check(self._lib.als_solver_run(self._h))

    def synchronize(self):
        _lib.check(self._lib.als_solver_synchronize(self._h))

    def stream(self):
        return self._lib.als_solver_stream(self._h)

    def info(self, member=0):
        info = _lib.MemberInfo()
        _lib.check(self._lib.als_solver_info(self._h, member, ctypes.byref(info)))
        return {"t": info.t, "dt": info.dt, "steps": info.steps, "done": bool(info.done),
                "status": info.status, "bad_index": info.bad_index, "bad_step": info.bad_step}

    def launches_per_step(self):
        return _lib.check(self._lib.als_solver_launches_per_step(self._h))

    def profile_step(self):
        """Runs one step with events around each kernel; returns their durations in ms."""
        buf = (ctypes.c_float * 8)()
        k = _lib.check(self._lib.als_solver_profile_step(self._h, buf, 8))
        return [buf[i] for i in range(k)]


def _grid(dimension, n, ghosts, gamma):
    g = _lib.Grid()
    g.dimension = dimension
    nn = list(n) + [1] * (3 - len(n))
    for d in range(3):
        g.n[d] = int(nn[d])
    g.ghosts = ghosts
    g.gamma = gamma
    return g


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    return ctypes.c_void_p(stream) if stream else None


class NumericalFlux:
    """numflux::NumericalFlux (NumericalFlux.hpp:25-53) on device planes."""

    def __init__(self, dimension, n, flux="hll", reconstruction="weno2", gamma=1.4):
        self.dimension = dimension
        self.n = tuple(n)
        self.flux = _choice(FLUX, flux, "flux")
        self.reconstruction = _choice(RECONSTRUCTION, reconstruction, "reconstruction")
        self.gamma = gamma
        self.ghosts = ghost_cells(self.flux, self.reconstruction)

    def getNumberOfGhostCells(self):
        return self.ghosts

    def computeFlux(self, conserved, out, start=(0, 0, 0), end=(0, 0, 0), stream=0):
        """Net flux of the region into ``out`` (device FP64 tensors); returns the wave speeds."""
        lib = _lib.load()
        g = _grid(self.dimension, self.n, self.ghosts, self.gamma)
        ws = np.zeros(3)
        s = (ctypes.c_int * 3)(*start)
        e = (ctypes.c_int * 3)(*end)
        _lib.check(lib.als_compute_flux(ctypes.byref(g), self.flux, self.reconstruction,
                                        _ptr(conserved), _ptr(out), s, e, ws.ctypes.data_as(_D),
                                        _stream(stream)))
        return ws


class Reconstruction:
    """reconstruction::Reconstruction (Reconstruction.hpp:21-59) on device planes."""

    def __init__(self, dimension, n, reconstruction="weno2", gamma=1.4):
        self.dimension = dimension
        self.n = tuple(n)
        self.reconstruction = _choice(RECONSTRUCTION, reconstruction, "reconstruction")
        self.gamma = gamma
        self.ghosts = ghost_cells(0, self.reconstruction)

    def getNumberOfGhostCells(self):
        return self.ghosts

    def performReconstruction(self, conserved, direction, left, right, stream=0):
        lib = _lib.load()
        g = _grid(self.dimension, self.n, self.ghosts, self.gamma)
        _lib.check(lib.als_reconstruct(ctypes.byref(g), self.reconstruction, direction,
                                       _ptr(conserved), _ptr(left), _ptr(right), _stream(stream)))


class Boundary:
    """boundary::Boundary (Boundary.hpp:23-36) on device planes."""

    def __init__(self, dimension, n, ghosts, boundary="periodic"):
        self.dimension = dimension
        self.n = tuple(n)
        self.ghosts = ghosts
        self.boundary = _choice(BOUNDARY, boundary, "boundary")

    def applyBoundaryConditions(self, planes, nvar=None, members=1, stream=0):
        lib = _lib.load()
        nvar = self.dimension + 2 if nvar is None else nvar
        g = _grid(self.dimension, self.n, self.ghosts, 1.4)
        _lib.check(lib.als_fill_ghosts(ctypes.byref(g), self.boundary, _ptr(planes), nvar, members,
                                       _stream(stream)))


class Integrator:
    """integrator::Integrator (Integrator.hpp:52-115): the stage combination
    of performSubstep and computeTimestep, around a NumericalFlux."""

    def __init__(self, name, numerical_flux, cfl):
        self.integrator = _choice(INTEGRATOR, name, "integrator")
        self.flux = numerical_flux
        self.cfl = cfl

    def getNumberOfSubsteps(self):
        return self.integrator + 1

    def computeTimestep(self, wave_speeds, cell_lengths, t, end_time):
        lib = _lib.load()
        ws = np.ascontiguousarray(wave_speeds, dtype=np.float64)
        cl = np.ascontiguousarray(cell_lengths, dtype=np.float64)
        return lib.als_compute_timestep(ws.ctypes.data_as(_D), cl.ctypes.data_as(_D), self.cfl,
                                        t, end_time)

    def performSubstep(self, volumes, cell_lengths, dt, out, substep, t, end_time, stream=0):
        """volumes[k] = U_k (device tensors); returns dt (computed at substep 0)."""
        lib = _lib.load()
        ws = self.flux.computeFlux(volumes[substep], out, stream=stream)
        if substep == 0:
            dt = self.computeTimestep(ws, cell_lengths, t, end_time)
        c = dt / cell_lengths[0]
        _lib.check(lib.als_integrator_combine(self.integrator, substep, _ptr(out),
                                              _ptr(volumes[substep]), _ptr(volumes[0]),
                                              out.numel(), c, _stream(stream)))
        return dt

"""Python face of the C ABI, named after the reference's interfaces.

``Simulator`` wraps the fused device solver (``als_solver_*``): it is what
``alsvinncli``'s time loop (Simulator::performStep, Simulator.cpp:81-85,
191-214) and, with ``members > 1`` or several ``levels``, ``alsuqcli``'s
sample loop (alsuq/src/run/Runner.cpp:42-78) become.  ``MeanVariance``
wraps the FP64 ensemble statistics (alsuq/src/stats/MeanVariance.cpp).  The
plug-in level calls (``NumericalFlux``, ``Reconstruction``, ``Boundary``,
``Integrator``) take device tensors of shape (nvar, ...) and mirror one
virtual call of the reference each.
"""
import ctypes

import numpy as np

from . import _lib
from .initial_data import padded_shape

FLUX = {"hll": 0, "hll3": 1, "central": 2, "tecno1": 3, "tecno4": 4, "tecno6": 5}
RECONSTRUCTION = {"none": 0, "weno2": 1, "eno2": 2, "eno3": 3, "eno4": 4, "mc": 5, "mm": 6,
                  "wenof2": 7, "weno3": 8}
INTEGRATOR = {"forwardeuler": 0, "rungekutta2": 1, "rungekutta3": 2, "rungekutta4": 3}
BOUNDARY = {"neumann": 0, "periodic": 1}
PRECISION = {"fp64": 0, "fp32": 1}
EQUATION = {"euler1": 1, "euler2": 2, "euler3": 3}

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


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
    """Advances one simulation, an ensemble of ``members`` simulations of the
    same grid, or several grid ``levels`` (list of dicts with ``n``,
    ``members`` and optionally ``lower``/``upper``) by whole time steps on
    the GPU.  Members are numbered level after level."""

    def __init__(self, dimension, n=None, lower=None, upper=None, flux="hll3",
                 reconstruction="weno2", integrator="rungekutta3", boundary="periodic", gamma=1.4,
                 cfl=0.4, end_time=1.0, max_steps=0, precision="fp64", members=1, device=0,
                 levels=None):
        lib = _lib.load()
        self._lib = lib
        if levels is None:
            levels = [{"n": n, "members": members, "lower": lower, "upper": upper}]
        cfgs = (_lib.SolverConfig * len(levels))()
        for k, lev in enumerate(levels):
            cfg = cfgs[k]
            cfg.dimension = dimension
            nn = list(lev["n"]) + [1] * (3 - len(lev["n"]))
            lo = list(lev.get("lower") or [0.0] * dimension) + [0.0] * 3
            hi = list(lev.get("upper") or [1.0] * dimension) + [0.0] * 3
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
            cfg.members = int(lev.get("members", 1))
        self.config = cfgs[0]
        self.dimension = dimension
        self.precision = precision
        handle = ctypes.c_void_p()
        _lib.check(lib.als_solver_create_levels(cfgs, len(levels), device, ctypes.byref(handle)))
        self._h = handle
        g = ctypes.c_int()
        _lib.check(lib.als_solver_geometry(self._h, None, ctypes.byref(g)))
        self.ghosts = g.value
        self.levels = []
        for k, lev in enumerate(levels):
            first = ctypes.c_int()
            count = ctypes.c_int()
            plane = ctypes.c_longlong()
            _lib.check(lib.als_solver_level(self._h, k, ctypes.byref(first), ctypes.byref(count),
                                            ctypes.byref(plane)))
            nn = tuple(int(v) for v in lev["n"][:dimension])
            self.levels.append({"first": first.value, "members": count.value,
                                "plane": plane.value, "n": nn,
                                "shape": padded_shape(dimension, nn, self.ghosts)})
        self.members = sum(lev["members"] for lev in self.levels)
        self.n = self.levels[0]["n"]
        self.plane = self.levels[0]["plane"]
        self.shape = self.levels[0]["shape"]

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

    def _level_of(self, member):
        for k, lev in enumerate(self.levels):
            if lev["first"] <= member < lev["first"] + lev["members"]:
                return k
        raise ValueError("member %d out of range" % member)

    def decompose(self, procs):
        """Makes the members the subdomains of one grid split over ``procs``
        ranks per direction (als_solver_decompose): one time step for all,
        ghost layers written across subdomains by the stage kernels.  Call
        before set_state, which then takes each block with its ghosts."""
        p = list(procs) + [1] * (3 - len(procs))
        _lib.check(self._lib.als_solver_decompose(self._h, (ctypes.c_int * 3)(*p[:3])))

    def set_state(self, states, first_member=0):
        """Uploads FP64 host states, shape (count, nvar, Nz, Ny, Nx) or (nvar, Nz, Ny, Nx)."""
        shape = self.levels[self._level_of(first_member)]["shape"]
        a = np.ascontiguousarray(states, dtype=np.float64)
        if a.shape == shape:
            a = a[None]
        if a.shape[1:] != shape:
            raise ValueError("state shape %s does not match %s" % (a.shape, shape))
        _lib.check(self._lib.als_solver_set_state(self._h, a.ctypes.data_as(_D), first_member,
                                                  a.shape[0]))

    def set_state_device(self, ptr, first_member=0, count=None):
        count = self.members - first_member if count is None else count
        _lib.check(self._lib.als_solver_set_state_device(self._h, ctypes.c_void_p(ptr),
                                                         first_member, count))

    def get_state(self, first_member=0, count=None):
        lev = self.levels[self._level_of(first_member)]
        if count is None:
            count = lev["first"] + lev["members"] - first_member
        out = np.zeros((count,) + lev["shape"])
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
        """Runs one step with events between the stages; returns their durations in ms."""
        buf = (ctypes.c_float * 8)()
        k = _lib.check(self._lib.als_solver_profile_step(self._h, buf, 8))
        return [buf[i] for i in range(k)]

    def set_schedule(self, blocks_per_sm=0, level_order=None):
        order = None
        if level_order is not None:
            order = (ctypes.c_int * len(self.levels))(*level_order)
        _lib.check(self._lib.als_solver_set_schedule(self._h, int(blocks_per_sm), order))

    def schedule(self):
        bps = ctypes.c_int()
        order = (ctypes.c_int * len(self.levels))()
        _lib.check(self._lib.als_solver_get_schedule(self._h, ctypes.byref(bps), order))
        return {"blocks_per_sm": bps.value, "level_order": list(order)}

    def set_tiles(self, shapes):
        """Tile shape per level: 0 the dimension's box tile (2-D 32x16, 3-D
        8x8x4 cells); 1 the alternative where it is built (2-D 16x16 cells
        for WENO2 with HLL, HLL3 or Central; 3-D 16x16 columns marching along
        z, the 3-D default, for reconstructions reaching one cell with the
        two-point fluxes)."""
        arr = (ctypes.c_int * len(self.levels))(*[int(v) for v in shapes])
        _lib.check(self._lib.als_solver_set_tiles(self._h, arr))

    def tiles(self):
        """{"shapes": [shape per level], "extents": [(x, y, z) tile cells per level]}."""
        nl = len(self.levels)
        shapes = (ctypes.c_int * nl)()
        ext = (ctypes.c_int * (3 * nl))()
        _lib.check(self._lib.als_solver_get_tiles(self._h, shapes, ext))
        return {"shapes": list(shapes),
                "extents": [tuple(ext[3 * k:3 * k + 3]) for k in range(nl)]}

    def tune(self, steps=3):
        """Runs the schedule autotuner (tile shape per level, blocks per SM,
        level order); state and clocks are restored."""
        nl = len(self.levels)
        bps = ctypes.c_int()
        order = (ctypes.c_int * nl)()
        shapes = (ctypes.c_int * nl)()
        ms = ctypes.c_double()
        _lib.check(self._lib.als_solver_tune(self._h, int(steps), ctypes.byref(bps), order, shapes,
                                             ctypes.byref(ms)))
        return {"blocks_per_sm": bps.value, "level_order": list(order),
                "tile_shapes": list(shapes), "ms_per_step": ms.value}

    def write_netcdf(self, basename, snapshot=0, member=0):
        """Writes member's state to <basename>_<snapshot>.nc (NetCDFWriter layout)."""
        _lib.check(self._lib.als_solver_write_netcdf(self._h, member, basename.encode(),
                                                     int(snapshot)))
        return "%s_%d.nc" % (basename, snapshot)

    def region_sums(self, first_member=0, count=None, lo=None, hi=None):
        """FP64 sums of each conserved variable over the interior box [lo, hi)
        (interior cell coordinates, default the whole interior): (count, nvar)."""
        lev = self.levels[self._level_of(first_member)]
        if count is None:
            count = lev["first"] + lev["members"] - first_member
        nvar = self.dimension + 2
        out = np.zeros((count, nvar))
        clo = (ctypes.c_int * 3)(*(list(lo) + [0, 0, 0])[:3]) if lo is not None else None
        chi = (ctypes.c_int * 3)(*(list(hi) + [1, 1, 1])[:3]) if hi is not None else None
        _lib.check(self._lib.als_solver_region_sums(self._h, first_member, count, clo, chi,
                                                    out.ctypes.data_as(_D)))
        return out


class MeanVariance:
    """alsuq::stats::MeanVariance (MeanVariance.cpp:30-67) in FP64 Welford
    form: add ensemble states (any precision) and read mean and the biased
    variance as device tensors."""

    def __init__(self, count, device=0):
        self._lib = _lib.load()
        self.count = int(count)
        h = ctypes.c_void_p()
        _lib.check(self._lib.als_stats_create(self.count, device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.als_stats_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_solver(self, simulator, level=0):
        _lib.check(self._lib.als_stats_add_solver(self._h, simulator._h, level))

    def add(self, states, precision="fp64", stream=0):
        """Adds a (members, ...) device tensor of states."""
        members = states.shape[0]
        stride = states[0].numel()
        _lib.check(self._lib.als_stats_add(self._h, ctypes.c_void_p(states.data_ptr()),
                                           _choice(PRECISION, precision, "precision"), members,
                                           stride, ctypes.c_void_p(stream) if stream else None))

    def merge(self, n, mean, m2, stream=0):
        _lib.check(self._lib.als_stats_merge(self._h, int(n), ctypes.c_void_p(mean.data_ptr()),
                                             ctypes.c_void_p(m2.data_ptr()),
                                             ctypes.c_void_p(stream) if stream else None))

    def moments(self):
        """(n, mean device pointer, M2 device pointer)."""
        n = ctypes.c_longlong()
        mean = ctypes.c_void_p()
        m2 = ctypes.c_void_p()
        _lib.check(self._lib.als_stats_moments(self._h, ctypes.byref(n), ctypes.byref(mean),
                                               ctypes.byref(m2)))
        return n.value, mean.value, m2.value

    def result(self, mean, variance, stream=0):
        """Writes mean and variance into FP64 device tensors of `count` elements."""
        _lib.check(self._lib.als_stats_result(self._h, ctypes.c_void_p(mean.data_ptr()),
                                              ctypes.c_void_p(variance.data_ptr()),
                                              ctypes.c_void_p(stream) if stream else None))


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

    def __init__(self, dimension, n, flux="hll", reconstruction="weno2", gamma=1.4, ghosts=None):
        """``ghosts``: the planes' ghost width when wider than the flux needs
        (a diffusion operator with a wider stencil sets it)."""
        self.dimension = dimension
        self.n = tuple(n)
        self.flux = _choice(FLUX, flux, "flux")
        self.reconstruction = _choice(RECONSTRUCTION, reconstruction, "reconstruction")
        self.gamma = gamma
        self.ghosts = ghosts or ghost_cells(self.flux, self.reconstruction)

    def getNumberOfGhostCells(self):
        return self.ghosts

    def computeFlux(self, conserved, out, start=(0, 0, 0), end=(0, 0, 0), stream=0,
                    compute_wave_speed=True):
        """Net flux of the region into ``out`` ((nvar, ...) FP64 device tensors);
        returns the per-direction wave speeds (the call then waits for the
        stream), or None with ``compute_wave_speed`` False (the reference's
        computeWaveSpeed flag: the flux is only enqueued)."""
        lib = _lib.load()
        g = _grid(self.dimension, self.n, self.ghosts, self.gamma)
        ws = np.zeros(3) if compute_wave_speed else None
        s = (ctypes.c_int * 3)(*start)
        e = (ctypes.c_int * 3)(*end)
        _lib.check(lib.als_compute_flux(ctypes.byref(g), self.flux, self.reconstruction,
                                        _lib.plane_pointers(conserved), _lib.plane_pointers(out),
                                        s, e, ws.ctypes.data_as(_D) if ws is not None else None,
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
                                       _lib.plane_pointers(conserved), _lib.plane_pointers(left),
                                       _lib.plane_pointers(right), _stream(stream)))


class Boundary:
    """boundary::Boundary (Boundary.hpp:23-36) on device planes."""

    def __init__(self, dimension, n, ghosts, boundary="periodic"):
        self.dimension = dimension
        self.n = tuple(n)
        self.ghosts = ghosts
        self.boundary = _choice(BOUNDARY, boundary, "boundary")

    def applyBoundaryConditions(self, planes, stream=0):
        lib = _lib.load()
        g = _grid(self.dimension, self.n, self.ghosts, 1.4)
        _lib.check(lib.als_fill_ghosts(ctypes.byref(g), self.boundary, _lib.plane_pointers(planes),
                                       planes.shape[0], _stream(stream)))


DIFFUSION = {"tecnoroe": 0, "tecnorusanov": 1}
TECNO_RECONSTRUCTION = {"none": 0, "eno2": 2, "eno3": 3, "eno4": 4}


def diffusion_ghost_cells(reconstruction):
    """Ghost cells of a TeCNO diffusion operator over ``reconstruction``."""
    lib = _lib.load()
    return _lib.check(lib.als_diffusion_ghost_cells(
        _choice(TECNO_RECONSTRUCTION, reconstruction, "TeCNO reconstruction")))


class DiffusionOperator:
    """diffusion::DiffusionOperator (DiffusionOperator.hpp:25-47) as
    DiffusionFactory builds it for the Euler equations: TecnoDiffusionCPU with
    the "tecnoroe" or "tecnorusanov" matrix over the TeCNO reconstruction
    "none", "eno2", "eno3" or "eno4" of the scaled entropy variables.  Its
    work arrays persist between calls, as the reference's do."""

    def __init__(self, dimension, n, diffusion="tecnoroe", reconstruction="eno2", gamma=1.4,
                 ghosts=None):
        self.dimension = dimension
        self.n = tuple(n)
        self.kind = _choice(DIFFUSION, diffusion, "diffusion")
        self.reconstruction = _choice(TECNO_RECONSTRUCTION, reconstruction, "TeCNO reconstruction")
        self.ghosts = ghosts or diffusion_ghost_cells(reconstruction)
        self.gamma = gamma
        self._lib = _lib.load()
        g = _grid(dimension, self.n, self.ghosts, gamma)
        h = ctypes.c_void_p()
        _lib.check(self._lib.als_diffusion_create(ctypes.byref(g), self.kind, self.reconstruction,
                                                  ctypes.byref(h)))
        self._h = h

    def getNumberOfGhostCells(self):
        return diffusion_ghost_cells({v: k for k, v in TECNO_RECONSTRUCTION.items()}[
            self.reconstruction])

    def applyDiffusion(self, output, conserved, stream=0):
        """output += the diffusion of ``conserved`` ((nvar, ...) FP64 device
        tensors, ghosts filled)."""
        _lib.check(self._lib.als_diffusion_apply(self._h, _lib.plane_pointers(conserved),
                                                 _lib.plane_pointers(output), _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.als_diffusion_destroy(self._h)
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


class Integrator:
    """integrator::Integrator (Integrator.hpp:52-115): the stage combination
    of performSubstep and computeTimestep, around the system L(U) of a
    NumericalFlux and, optionally, a DiffusionOperator added to it
    (ConservedSystem.cpp:31-103)."""

    def __init__(self, name, numerical_flux, cfl, diffusion=None):
        self.integrator = _choice(INTEGRATOR, name, "integrator")
        self.flux = numerical_flux
        self.diffusion = diffusion
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
        # only the first stage's wave speeds set dt (Integrator.cpp:20-46); the
        # other stages are enqueued without a host round trip
        ws = self.flux.computeFlux(volumes[substep], out, stream=stream,
                                   compute_wave_speed=substep == 0)
        if self.diffusion is not None:
            self.diffusion.applyDiffusion(out, volumes[substep], stream=stream)
        if substep == 0:
            dt = self.computeTimestep(ws, cell_lengths, t, end_time)
        c = dt / cell_lengths[0]
        if self.integrator == 3 and substep == 3:
            # RungeKutta4.cpp:80-87
            _lib.check(lib.als_integrator_combine_rk4(_ptr(out), _ptr(volumes[0]),
                                                      _ptr(volumes[1]), _ptr(volumes[2]),
                                                      _ptr(volumes[3]), out.numel(), c,
                                                      _stream(stream)))
        else:
            _lib.check(lib.als_integrator_combine(self.integrator, substep, _ptr(out),
                                                  _ptr(volumes[substep]), _ptr(volumes[0]),
                                                  out.numel(), c, _stream(stream)))
        return dt

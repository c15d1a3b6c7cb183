"""ctypes bindings for the two test oracles.

TEST INFRASTRUCTURE ONLY.

* ``COracle`` wraps ``oracle/liboracle.so``: the plain-C restatement of the
  reference's hot path (``oracle/als_oracle.c``).  It is built on demand with
  ``make -C oracle`` (gcc only), so it is available on every machine.
* ``RefOracle`` wraps ``oracle/_ref/libalsref.so``: the reference's own CPU
  sources compiled by ``make -C oracle ref``.  It only exists where it was
  built (it needs the reference source tree); tests that need it skip
  otherwise, and the committed fixtures in ``tests/golden/`` carry its
  outputs everywhere else.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")

FLUX = {"hll": 0, "hll3": 1, "central": 2, "tecno1": 3, "tecno4": 4, "tecno6": 5}
RECON = {"none": 0, "weno2": 1, "eno2": 2, "eno3": 3, "eno4": 4, "mc": 5, "mm": 6,
         "wenof2": 7, "weno3": 8}
INTEGRATOR = {"forwardeuler": 0, "rungekutta2": 1, "rungekutta3": 2, "rungekutta4": 3}
DIFFUSION = {"tecnoroe": 0, "tecnorusanov": 1}
DIFFUSION_RECON = {"none": 0, "eno2": 2, "eno3": 3, "eno4": 4}
BC = {"neumann": 0, "periodic": 1}

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _dptr(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def ghost_cells(recon, flux="hll"):
    g = {"none": 1, "weno2": 2, "eno2": 2, "eno3": 3, "eno4": 4, "mc": 2, "mm": 2,
         "wenof2": 2, "weno3": 3}[recon]
    return max(g, {"tecno4": 3, "tecno6": 5}.get(flux, 1))


def padded_shape(dim, n, g):
    """(nvar, Nz, Ny, Nx) of a padded volume."""
    nn = [n[d] if d < dim else 1 for d in range(3)]
    N = [nn[d] + (2 * g if d < dim else 0) for d in range(3)]
    return (dim + 2, N[2], N[1], N[0])


class _Config(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("g", ctypes.c_int),
        ("gamma", ctypes.c_double),
        ("flux", ctypes.c_int),
        ("recon", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("bc", ctypes.c_int),
        ("dx", ctypes.c_double * 3),
        ("diffusion", ctypes.c_int),
        ("diffusion_recon", ctypes.c_int),
    ]


def build_c_oracle():
    path = os.path.join(ORACLE_DIR, "liboracle.so")
    src = os.path.join(ORACLE_DIR, "als_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return path


class FunctionalParams(ctypes.Structure):
    _fields_ = [("degree", ctypes.c_int), ("degree_k", ctypes.c_int), ("degree_n", ctypes.c_int),
                ("degree_m", ctypes.c_int), ("min_value", ctypes.c_double),
                ("max_value", ctypes.c_double), ("gamma", ctypes.c_double),
                ("lower", ctypes.c_double * 3), ("upper", ctypes.c_double * 3),
                ("direction", ctypes.c_int), ("number_of_h", ctypes.c_int)]


FUNCTIONAL = {"identity": 0, "moment": 1, "log_entropy": 2, "legendre": 3,
              "legendre_pointwise": 4, "bv": 5, "bv_direction": 6, "structure_2pt": 7}


class COracle:
    def __init__(self):
        self.lib = ctypes.CDLL(build_c_oracle())
        L = self.lib
        L.orc_configure.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, _I, _D, _D,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double]
        L.orc_simulate.argtypes = [ctypes.POINTER(_Config), ctypes.c_double, ctypes.c_double,
                                   ctypes.c_long, _D, _D, ctypes.c_long,
                                   ctypes.POINTER(ctypes.c_long), _D]
        L.orc_net_flux.argtypes = [ctypes.POINTER(_Config), _D, _D, _D]
        L.orc_reconstruct.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, _D, _D, _D]
        L.orc_fill_ghosts.argtypes = [ctypes.POINTER(_Config), _D, ctypes.c_int]
        L.orc_meanvar.argtypes = [ctypes.c_long, ctypes.c_long, _D, _D, _D]
        L.orc_obeys_constraints.argtypes = [ctypes.POINTER(_Config), _D]
        L.orc_diffusion_apply.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, ctypes.c_int,
                                          _D, _D, _D]
        L.orc_diffusion_ghost_cells.argtypes = [ctypes.c_int]
        L.orc_set_diffusion.argtypes = [ctypes.POINTER(_Config), ctypes.c_int, ctypes.c_int]
        L.orc_functional_size.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int]
        L.orc_functional_size.restype = ctypes.c_long
        L.orc_functional.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(FunctionalParams), _D, _D, ctypes.c_double]
        L.orc_structure_cube.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D]
        L.orc_structure_basic.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, _D, _D]

    def config(self, dim, n, lower, upper, flux, recon, integrator, bc, gamma):
        cfg = _Config()
        nn = (ctypes.c_int * 3)(*[int(v) for v in (list(n) + [1, 1, 1])[:3]])
        lo = (ctypes.c_double * 3)(*[float(v) for v in (list(lower) + [0, 0, 0])[:3]])
        hi = (ctypes.c_double * 3)(*[float(v) for v in (list(upper) + [0, 0, 0])[:3]])
        rc = self.lib.orc_configure(ctypes.byref(cfg), dim, nn, lo, hi, FLUX[flux],
                                    RECON[recon], INTEGRATOR[integrator], BC[bc], gamma)
        assert rc == 0
        return cfg

    def simulate(self, cfg, planes, cfl, end_time, max_steps=10 ** 9, dts_capacity=100000):
        out = np.ascontiguousarray(planes, dtype=np.float64).copy()
        dts = np.zeros(dts_capacity)
        steps = ctypes.c_long()
        t = ctypes.c_double()
        rc = self.lib.orc_simulate(ctypes.byref(cfg), cfl, end_time, max_steps, _dptr(out),
                                   _dptr(dts), dts_capacity, ctypes.byref(steps),
                                   ctypes.byref(t))
        return rc, out, dts[:min(steps.value, dts_capacity)], steps.value, t.value

    def net_flux(self, cfg, planes):
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        out = np.zeros_like(inp)
        ws = np.zeros(3)
        self.lib.orc_net_flux(ctypes.byref(cfg), _dptr(inp), _dptr(out), _dptr(ws))
        return out, ws

    def reconstruct(self, cfg, direction, planes):
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        left = np.zeros_like(inp)
        right = np.zeros_like(inp)
        self.lib.orc_reconstruct(ctypes.byref(cfg), direction, _dptr(inp), _dptr(left),
                                 _dptr(right))
        return left, right

    def fill_ghosts(self, cfg, planes):
        out = np.ascontiguousarray(planes, dtype=np.float64).copy()
        self.lib.orc_fill_ghosts(ctypes.byref(cfg), _dptr(out), out.shape[0])
        return out

    def meanvar(self, states):
        st = np.ascontiguousarray(states, dtype=np.float64)
        count = st[0].size
        mean = np.zeros(count)
        var = np.zeros(count)
        self.lib.orc_meanvar(count, st.shape[0], _dptr(st), _dptr(mean), _dptr(var))
        return mean.reshape(st.shape[1:]), var.reshape(st.shape[1:])

    def set_diffusion(self, cfg, kind, recon):
        """Adds a TeCNO diffusion operator to cfg's system (widens cfg.g)."""
        assert self.lib.orc_set_diffusion(ctypes.byref(cfg), DIFFUSION[kind],
                                          DIFFUSION_RECON[recon]) == 0
        return cfg

    def functional(self, dim, n, g, kind, planes, weight=1.0, out=None, degree=1, degree_k=0,
                   degree_n=0, degree_m=0, min_value=0.0, max_value=1.0, gamma=1.4,
                   lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), direction=0, number_of_h=1):
        """out (nvar, size) += weight * f(planes) for one padded state."""
        nn = (ctypes.c_int * 3)(*[int(v) for v in (list(n) + [1, 1, 1])[:3]])
        size = self.lib.orc_functional_size(dim, nn, g, FUNCTIONAL[kind], int(number_of_h))
        res = np.zeros((dim + 2, size)) if out is None else np.array(out, dtype=np.float64)
        p = FunctionalParams(int(degree), int(degree_k), int(degree_n), int(degree_m),
                             float(min_value), float(max_value), float(gamma))
        for d in range(3):
            p.lower[d] = float(lower[d]) if d < len(lower) else 0.0
            p.upper[d] = float(upper[d]) if d < len(upper) else 0.0
        p.direction, p.number_of_h = int(direction), int(number_of_h)
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        rc = self.lib.orc_functional(dim, nn, g, FUNCTIONAL[kind], ctypes.byref(p), _dptr(inp),
                                     _dptr(res), float(weight))
        if rc == -2:
            raise ValueError("functional %s: a Legendre argument outside [-1, 1]" % kind)
        if rc != 0:
            raise ValueError("functional %s not defined in %d-D" % (kind, dim))
        return res

    def diffusion_state(self, cfg):
        """The persistent work arrays of a diffusion operator as the
        reference creates them: four volumes from HostMemory (every entry
        42), then three zeroed difference planes."""
        shp = padded_shape(cfg.dim, list(cfg.n), cfg.g)
        plane = int(np.prod(shp[1:]))
        st = np.zeros(4 * shp[0] * plane + 3 * plane)
        st[:4 * shp[0] * plane] = 42.0
        return st

    def apply_diffusion(self, cfg, kind, recon, state, planes, out):
        """Adds the TeCNO diffusion of `planes` to a copy of `out`; `state`
        (from diffusion_state) is updated in place."""
        assert state.flags["C_CONTIGUOUS"] and state.dtype == np.float64
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        res = np.ascontiguousarray(out, dtype=np.float64).copy()
        self.lib.orc_diffusion_apply(ctypes.byref(cfg), DIFFUSION[kind], DIFFUSION_RECON[recon],
                                     _dptr(state), _dptr(inp), _dptr(res))
        return res

    def obeys_constraints(self, cfg, planes):
        p = np.ascontiguousarray(planes, dtype=np.float64)
        return bool(self.lib.orc_obeys_constraints(ctypes.byref(cfg), _dptr(p)))

    def structure_cube(self, dim, n, g, bc, H, p, planes):
        st = np.ascontiguousarray(planes, dtype=np.float64)
        out = np.zeros((st.shape[0], H))
        nn = (ctypes.c_int * 3)(*(list(n) + [1, 1, 1])[:3])
        self.lib.orc_structure_cube(dim, nn, g, 1 if bc == "periodic" else 0, st.shape[0], H,
                                    float(p), _dptr(st), _dptr(out))
        return out

    def structure_basic(self, dim, n, g, bc, direction, H, p, planes):
        st = np.ascontiguousarray(planes, dtype=np.float64)
        out = np.zeros((st.shape[0], H))
        nn = (ctypes.c_int * 3)(*(list(n) + [1, 1, 1])[:3])
        self.lib.orc_structure_basic(dim, nn, g, 1 if bc == "periodic" else 0, st.shape[0],
                                     direction, H, float(p), _dptr(st), _dptr(out))
        return out


def ref_library_path():
    return os.path.join(ORACLE_DIR, "_ref", "libalsref.so")


class RefOracle:
    """The reference's own CPU code (only where ``make -C oracle ref`` ran)."""

    def __init__(self, path=None):
        path = path or ref_library_path()
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.alsref_last_error.restype = ctypes.c_char_p
        L.alsref_last_loop_seconds.restype = ctypes.c_double
        L.alsref_simulate.argtypes = [ctypes.c_int, _I, _D, _D, ctypes.c_char_p,
                                      ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_long, _D, _D, ctypes.c_long,
                                      ctypes.POINTER(ctypes.c_long), _D]
        L.alsref_compute_flux.argtypes = [ctypes.c_int, _I, _D, _D, ctypes.c_char_p,
                                          ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                                          _D, _D, _D]
        L.alsref_reconstruct.argtypes = [ctypes.c_int, _I, ctypes.c_char_p, ctypes.c_double,
                                         ctypes.c_int, _D, _D, _D]
        L.alsref_apply_boundary.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_char_p, _D]
        L.alsref_meanvar.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_long, _D, _D, _D]
        L.alsref_stlmersenne.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, _D]
        L.alsref_ghost_cells.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p]
        L.alsref_structure_cube.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_char_p,
                                            ctypes.c_int, ctypes.c_double, _D, _D]
        L.alsref_set_diffusion.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        L.alsref_apply_diffusion.argtypes = [ctypes.c_int, _I, ctypes.c_char_p, ctypes.c_char_p,
                                             ctypes.c_double, ctypes.c_int, _D, _D,
                                             ctypes.POINTER(ctypes.c_int)]
        L.alsref_statistics.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, _I,
                                        ctypes.c_int, ctypes.c_long, _D, ctypes.c_double, _D, _D]
        L.alsref_functional_size.argtypes = [ctypes.c_int, _I, ctypes.c_int, ctypes.c_char_p,
                                             ctypes.c_int, ctypes.c_double]
        L.alsref_functional_size.restype = ctypes.c_long
        L.alsref_functional.argtypes = [ctypes.c_int, _I, _D, _D, ctypes.c_int, ctypes.c_char_p,
                                        ctypes.c_int, ctypes.c_double, _I, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, _D, _D]

    def set_diffusion(self, kind, recon="none"):
        """Diffusion operator of the following simulations (none by default)."""
        self._check(self.lib.alsref_set_diffusion(kind.encode(), recon.encode()))

    def apply_diffusion(self, dim, n, kind, recon, gamma, states, outs):
        """One operator object applied to states[k], adding into outs[k] in
        turn; returns the new outputs."""
        st = np.ascontiguousarray(states, dtype=np.float64)
        out = np.ascontiguousarray(outs, dtype=np.float64).copy()
        g = ctypes.c_int()
        self._check(self.lib.alsref_apply_diffusion(dim, self._vec(n, ctypes.c_int, 1),
                                                    kind.encode(), recon.encode(), gamma,
                                                    st.shape[0], _dptr(st), _dptr(out),
                                                    ctypes.byref(g)))
        return out

    def _check(self, rc):
        if rc < 0:
            raise RuntimeError(self.lib.alsref_last_error().decode())
        return rc

    @staticmethod
    def _vec(vals, ctype, fill):
        vals = (list(vals) + [fill, fill, fill])[:3]
        return (ctype * 3)(*vals)

    def simulate(self, dim, n, lower, upper, flux, recon, integrator, bc, gamma, cfl,
                 end_time, planes, max_steps=10 ** 9, dts_capacity=100000):
        out = np.ascontiguousarray(planes, dtype=np.float64).copy()
        dts = np.zeros(dts_capacity)
        steps = ctypes.c_long()
        t = ctypes.c_double()
        rc = self._check(self.lib.alsref_simulate(
            dim, self._vec(n, ctypes.c_int, 1), self._vec(lower, ctypes.c_double, 0.0),
            self._vec(upper, ctypes.c_double, 0.0), flux.encode(), recon.encode(),
            integrator.encode(), bc.encode(), gamma, cfl, end_time, max_steps, _dptr(out),
            _dptr(dts), dts_capacity, ctypes.byref(steps), ctypes.byref(t)))
        return rc, out, dts[:min(steps.value, dts_capacity)], steps.value, t.value

    def compute_flux(self, dim, n, lower, upper, flux, recon, bc, gamma, planes):
        inp = np.ascontiguousarray(planes, dtype=np.float64).copy()
        out = np.zeros_like(inp)
        ws = np.zeros(3)
        self._check(self.lib.alsref_compute_flux(
            dim, self._vec(n, ctypes.c_int, 1), self._vec(lower, ctypes.c_double, 0.0),
            self._vec(upper, ctypes.c_double, 0.0), flux.encode(), recon.encode(),
            bc.encode(), gamma, _dptr(inp), _dptr(out), _dptr(ws)))
        return inp, out, ws

    def reconstruct(self, dim, n, recon, gamma, direction, planes):
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        left = np.zeros_like(inp)
        right = np.zeros_like(inp)
        self._check(self.lib.alsref_reconstruct(dim, self._vec(n, ctypes.c_int, 1),
                                                recon.encode(), gamma, direction, _dptr(inp),
                                                _dptr(left), _dptr(right)))
        return left, right

    def apply_boundary(self, dim, n, ghosts, bc, planes):
        out = np.ascontiguousarray(planes, dtype=np.float64).copy()
        self._check(self.lib.alsref_apply_boundary(dim, self._vec(n, ctypes.c_int, 1), ghosts,
                                                   bc.encode(), _dptr(out)))
        return out

    def meanvar(self, dim, n, ghosts, states):
        st = np.ascontiguousarray(states, dtype=np.float64)
        mean = np.zeros(st.shape[1:])
        var = np.zeros(st.shape[1:])
        self._check(self.lib.alsref_meanvar(dim, self._vec(n, ctypes.c_int, 1), ghosts,
                                            st.shape[0], _dptr(st), _dptr(mean), _dptr(var)))
        return mean, var

    def structure_cube(self, dim, n, ghosts, bc, H, p, planes):
        st = np.ascontiguousarray(planes, dtype=np.float64)
        out = np.zeros((st.shape[0], H))
        self._check(self.lib.alsref_structure_cube(dim, self._vec(n, ctypes.c_int, 1), ghosts,
                                                   bc.encode(), H, float(p), _dptr(st),
                                                   _dptr(out)))
        return out

    def statistics(self, dim, n, ghosts, states, platform="cpu", name="meanvar", time=1.0):
        """The statistics `name` of `platform` made by the reference's
        StatisticsFactory over the padded states (samples first), combined,
        finalized and written like alsuq's Runner; returns its first two
        statistics (mean and variance for meanvar)."""
        st = np.ascontiguousarray(states, dtype=np.float64)
        first = np.zeros(st.shape[1:])
        second = np.zeros(st.shape[1:])
        self._check(self.lib.alsref_statistics(platform.encode(), name.encode(), dim,
                                               self._vec(n, ctypes.c_int, 1), ghosts,
                                               st.shape[0], _dptr(st), float(time),
                                               _dptr(first), _dptr(second)))
        return first, second

    def functional(self, dim, n, ghosts, kind, planes, weight=1.0, out=None, degree=1,
                   gamma=1.4, lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), degree_k=0,
                   degree_n=0, degree_m=0, min_value=0.0, max_value=1.0):
        """out (nvar, size) += weight * f(planes) by the reference's
        FunctionalFactory ("cpu") functional `kind`, for one padded state."""
        nn = self._vec(n, ctypes.c_int, 1)
        size = self.lib.alsref_functional_size(dim, nn, ghosts, kind.encode(), int(degree),
                                               float(gamma))
        self._check(size)
        res = np.zeros((dim + 2, size)) if out is None else np.array(out, dtype=np.float64)
        inp = np.ascontiguousarray(planes, dtype=np.float64)
        degrees = (ctypes.c_int * 3)(int(degree_k), int(degree_n), int(degree_m))
        self._check(self.lib.alsref_functional(dim, nn, self._vec(lower, ctypes.c_double, 0.0),
                                               self._vec(upper, ctypes.c_double, 0.0), ghosts,
                                               kind.encode(), int(degree), float(gamma), degrees,
                                               float(min_value), float(max_value),
                                               float(weight), _dptr(inp), _dptr(res)))
        return res

    def stlmersenne(self, dimension, first, count):
        out = np.zeros(dimension * count)
        self._check(self.lib.alsref_stlmersenne(dimension, first, count, _dptr(out)))
        return out.reshape(count, dimension)


def smooth_random_state(seed, dim, n, g, gamma=1.4, amplitude=0.1, velocity=0.2):
    """A seeded random state near rho = p = 1 (padded planes, ghosts random too).

    Uses numpy's PCG64, so the same seed gives the same state wherever the
    same numpy runs (fixtures store a digest of the reference outputs for
    such inputs)."""
    rng = np.random.default_rng(seed)
    shp = padded_shape(dim, n, g)
    rho = rng.uniform(1 - amplitude, 1 + amplitude, shp[1:])
    p = rng.uniform(1 - amplitude, 1 + amplitude, shp[1:])
    u = [rng.uniform(-velocity, velocity, shp[1:]) for _ in range(dim)]
    E = p / (gamma - 1) + 0.5 * rho * sum(x * x for x in u)
    return np.ascontiguousarray(np.stack([rho] + [rho * x for x in u] + [E]))


def digest(*arrays):
    """sha256 of the exact bytes of float64 arrays (bit-exact comparison)."""
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def ref_b200_library_path():
    return os.path.join(ROOT, "oracle", "_ref", "libalsref_b200.so")


class RefB200Oracle(RefOracle):
    """The reference's time loop whose flux can be numflux::NumericalFluxB200
    (oracle/adapter/), built by ``make -C oracle ref-b200``."""

    def __init__(self):
        super().__init__(ref_b200_library_path())
        self.lib.alsref_set_flux_platform.argtypes = [ctypes.c_char_p]

    def set_flux_platform(self, platform):
        self._check(self.lib.alsref_set_flux_platform(platform.encode()))

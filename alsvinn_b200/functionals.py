"""Observables of ensemble states (device tensors).

Python face of ``als_structure_functions`` and ``als_functional``
(include/als_b200.h): the reference's StructureCube and StructureBasic
statistics (alsuq/src/stats/StructureCube.cpp, StructureBasic.cpp) and its
functionals (alsfvm/src/functional/: identity, moment, log_entropy,
legendre, legendre_pointwise, bv), evaluated on the GPU for every member and
conserved variable at once.
"""
import ctypes

from . import _lib
from .simulator import BOUNDARY, PRECISION, _choice, _grid, _stream

KINDS = {"cube": 0, "basic": 1}


def structure_functions(states, dimension, n, ghosts, boundary="periodic", kind="cube", H=8,
                        p=1.0, direction=0, gamma=1.4, stream=0):
    """S[member, var, h] for a (members, nvar, Nz, Ny, Nx) FP64 or FP32 CUDA tensor.

    cube: h = 1..H-1 over the surface of the cube of half-width h around
    every cell (S[..., 0] = 0); basic: h = 0..H-1 along ``direction``.
    Returns an FP64 CUDA tensor (members, nvar, H)."""
    import torch
    lib = _lib.load()
    if states.dim() != 5 or not states.is_cuda or not states.is_contiguous():
        raise ValueError("states must be a contiguous (members, nvar, Nz, Ny, Nx) CUDA tensor")
    if states.dtype == torch.float64:
        precision = "fp64"
    elif states.dtype == torch.float32:
        precision = "fp32"
    else:
        raise ValueError("states must be float64 or float32")
    members, nvar = states.shape[0], states.shape[1]
    if nvar != dimension + 2:
        raise ValueError("expected %d conserved variables" % (dimension + 2))
    out = torch.zeros((members, nvar, H), dtype=torch.float64, device=states.device)
    g = _grid(dimension, n, ghosts, gamma)
    _lib.check(lib.als_structure_functions(
        ctypes.byref(g), _choice(BOUNDARY, boundary, "boundary"), _choice(KINDS, kind, "kind"),
        int(direction), int(H), float(p), ctypes.c_void_p(states.data_ptr()),
        _choice(PRECISION, precision, "precision"), states[0].numel(), members,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream) if stream else None))
    return out


FUNCTIONALS = {"identity": 0, "moment": 1, "log_entropy": 2, "legendre": 3,
               "legendre_pointwise": 4, "bv": 5, "bv_direction": 6, "structure_2pt": 7}


def functional_size(dimension, n, ghosts, kind, number_of_h=1):
    """Elements per variable of a functional's output (Functional::getFunctionalSize)."""
    lib = _lib.load()
    g = _grid(dimension, n, ghosts, 1.4)
    p = _lib.FunctionalParams()
    p.number_of_h = int(number_of_h)
    size = ctypes.c_longlong()
    _lib.check(lib.als_functional_size2(ctypes.byref(g), _choice(FUNCTIONALS, kind, "functional"),
                                        ctypes.byref(p), ctypes.byref(size)))
    return size.value


def functional(states, dimension, n, ghosts, kind, weight=1.0, out=None, degree=1, degree_k=0,
               degree_n=0, degree_m=0, min_value=0.0, max_value=1.0, gamma=1.4,
               lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0), direction=0, number_of_h=1,
               stream=0):
    """out += weight * f(U) for every member of a (members, nvar, Nz, Ny, Nx)
    FP64 or FP32 CUDA tensor; ``out`` (created zero when None) is an FP64
    CUDA tensor (members, nvar, functional_size).  ``kind``: identity,
    moment (``degree``), log_entropy (``gamma``), legendre (``degree_k``,
    ``degree_n``, ``degree_m``, ``min_value``, ``max_value``),
    legendre_pointwise (``degree``, ``min_value``, ``max_value``), bv (the
    power ``degree``), or the alsuq statistics bv_direction (``direction``,
    ``degree``) and structure_2pt (``direction``, ``number_of_h``);
    ``lower``/``upper`` are the domain corners.  An ensemble statistic of the
    reference (onepointmoment, bv, functional, structure_2pt) is the mean of
    these per-member results over the members."""
    import torch
    lib = _lib.load()
    if states.dim() != 5 or not states.is_cuda or not states.is_contiguous():
        raise ValueError("states must be a contiguous (members, nvar, Nz, Ny, Nx) CUDA tensor")
    precision = {torch.float64: "fp64", torch.float32: "fp32"}.get(states.dtype)
    if precision is None:
        raise ValueError("states must be float64 or float32")
    members, nvar = states.shape[0], states.shape[1]
    size = functional_size(dimension, n, ghosts, kind, number_of_h)
    if out is None:
        out = torch.zeros((members, nvar, size), dtype=torch.float64, device=states.device)
    if out.shape != (members, nvar, size) or out.dtype != torch.float64 or not out.is_contiguous():
        raise ValueError("out must be a contiguous FP64 tensor (members, nvar, %d)" % size)
    p = _lib.FunctionalParams()
    p.degree, p.degree_k, p.degree_n, p.degree_m = int(degree), int(degree_k), int(degree_n), \
        int(degree_m)
    p.min_value, p.max_value, p.gamma = float(min_value), float(max_value), float(gamma)
    p.direction, p.number_of_h = int(direction), int(number_of_h)
    for d in range(3):
        p.lower[d] = float(lower[d]) if d < len(lower) else 0.0
        p.upper[d] = float(upper[d]) if d < len(upper) else 0.0
    g = _grid(dimension, n, ghosts, gamma)
    _lib.check(lib.als_functional(
        ctypes.byref(g), _choice(FUNCTIONALS, kind, "functional"), ctypes.byref(p),
        ctypes.c_void_p(states.data_ptr()), PRECISION[precision], states[0].numel(), members,
        ctypes.c_void_p(out.data_ptr()), out[0].numel(), float(weight), _stream(stream)))
    return out


class TimeIntegratedFunctional:
    """TimeIntegrationFunctional (TimeIntegrationFunctional.cpp:20-63): a
    functional accumulated with weight dt = t - t_last at every write whose
    time lies within ``radius`` of ``time``."""

    def __init__(self, dimension, n, ghosts, kind, time, radius, **params):
        self.args = (dimension, n, ghosts, kind)
        self.params = params
        self.time = time
        self.radius = radius
        self.last_time = 0.0
        self.value = None

    def write(self, states, t):
        dt = t - self.last_time
        if abs(t - self.time) <= self.radius:
            self.value = functional(states, *self.args, weight=dt, out=self.value, **self.params)
        self.last_time = t
        return self.value

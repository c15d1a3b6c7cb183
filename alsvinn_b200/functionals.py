"""Structure-function statistics of ensemble states (device tensors).

Python face of ``als_structure_functions`` (include/als_b200.h): the
reference's StructureCube and StructureBasic statistics
(alsuq/src/stats/StructureCube.cpp, alsuq/src/stats/StructureBasic.cpp)
evaluated on the GPU for every member and conserved variable at once.
"""
import ctypes

from . import _lib
from .simulator import BOUNDARY, PRECISION, _choice, _grid

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

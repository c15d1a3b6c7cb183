"""B200-native cell-update hot path of alsvinn's finite-volume solver (alsfvm).

The compute lives in ``libals_b200.so`` (hand-written sm_100a CUDA behind the
C ABI in ``include/als_b200.h``); this package is the Python face of it.
"""
from . import _lib
from .initial_data import (kelvin_helmholtz, kh_ensemble, padded_shape, sod, uniform_draws)
from .simulator import (Boundary, DiffusionOperator, Integrator, MeanVariance, NumericalFlux,
                        Reconstruction, Simulator, diffusion_ghost_cells, ghost_cells)
from .surrogate import Surrogate
from . import uq

__all__ = [
    "Boundary", "DiffusionOperator", "Integrator", "MeanVariance", "NumericalFlux",
    "Reconstruction", "Simulator", "Surrogate", "diffusion_ghost_cells", "ghost_cells", "uq",
    "kelvin_helmholtz", "kh_ensemble", "padded_shape", "sod", "uniform_draws",
]


def library_path():
    return _lib.library_path()

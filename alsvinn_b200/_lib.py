"""ctypes binding of ``libals_b200.so`` (declared in ``include/als_b200.h``).

The library is the product: there is no fallback.  Loading fails loudly
when it has not been built (``python -m alsvinn_b200.build``).
"""
import ctypes
import os

from . import build as _build

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)   # array of plane pointers
_LL = ctypes.POINTER(ctypes.c_longlong)


class FunctionalParams(ctypes.Structure):
    _fields_ = [("degree", ctypes.c_int), ("degree_k", ctypes.c_int), ("degree_n", ctypes.c_int),
                ("degree_m", ctypes.c_int), ("min_value", ctypes.c_double),
                ("max_value", ctypes.c_double), ("gamma", ctypes.c_double),
                ("lower", ctypes.c_double * 3), ("upper", ctypes.c_double * 3),
                ("direction", ctypes.c_int), ("number_of_h", ctypes.c_int)]


class Grid(ctypes.Structure):
    _fields_ = [("dimension", ctypes.c_int), ("n", ctypes.c_int * 3), ("ghosts", ctypes.c_int),
                ("gamma", ctypes.c_double)]


class SolverConfig(ctypes.Structure):
    _fields_ = [
        ("dimension", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("lower", ctypes.c_double * 3),
        ("upper", ctypes.c_double * 3),
        ("flux", ctypes.c_int),
        ("reconstruction", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("boundary", ctypes.c_int),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("end_time", ctypes.c_double),
        ("max_steps", ctypes.c_longlong),
        ("precision", ctypes.c_int),
        ("members", ctypes.c_int),
    ]


class MlpConfig(ctypes.Structure):
    _fields_ = [("inputs", ctypes.c_int), ("width", ctypes.c_int), ("hidden", ctypes.c_int),
                ("max_batch", ctypes.c_int)]


class MemberInfo(ctypes.Structure):
    _fields_ = [("t", ctypes.c_double), ("dt", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("done", ctypes.c_int), ("status", ctypes.c_int),
                ("bad_index", ctypes.c_longlong), ("bad_step", ctypes.c_longlong)]


# name -> (restype, argtypes) for every function the header declares
PROTOTYPES = {
    "als_scratch_trim": (ctypes.c_int, [ctypes.c_int, ctypes.c_ulonglong]),
    "als_last_error": (ctypes.c_char_p, []),
    "als_version": (ctypes.c_int, []),
    "als_ghost_cells": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "als_fill_ghosts": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, _PP, ctypes.c_int,
                                       _VP]),
    "als_compute_flux": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int, _PP, _PP,
                                        _I, _I, _D, _VP]),
    "als_compute_flux_static": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int,
                                               _VP, _VP, ctypes.c_int, _D, _VP]),
    "als_reconstruct": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int, _PP, _PP,
                                       _PP, _VP]),
    "als_integrator_combine": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _VP, _VP, _VP,
                                              ctypes.c_size_t, ctypes.c_double, _VP]),
    "als_integrator_combine_rk4": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, ctypes.c_size_t,
                                                  ctypes.c_double, _VP]),
    "als_compute_timestep": (ctypes.c_double, [_D, _D, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double]),
    "als_solver_create": (ctypes.c_int, [ctypes.POINTER(SolverConfig), ctypes.c_int,
                                         ctypes.POINTER(_VP)]),
    "als_solver_create_levels": (ctypes.c_int, [ctypes.POINTER(SolverConfig), ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(_VP)]),
    "als_solver_level": (ctypes.c_int, [_VP, ctypes.c_int, _I, _I, _LL]),
    "als_solver_set_schedule": (ctypes.c_int, [_VP, ctypes.c_int, _I]),
    "als_solver_get_schedule": (ctypes.c_int, [_VP, _I, _I]),
    "als_solver_tune": (ctypes.c_int, [_VP, ctypes.c_int, _I, _I, _I, _D]),
    "als_solver_set_tiles": (ctypes.c_int, [_VP, _I]),
    "als_solver_get_tiles": (ctypes.c_int, [_VP, _I, _I]),
    "als_solver_region_sums": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _I, _I, _D]),
    "als_stats_create": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(_VP)]),
    "als_stats_destroy": (ctypes.c_int, [_VP]),
    "als_stats_add": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _VP]),
    "als_stats_add_solver": (ctypes.c_int, [_VP, _VP, ctypes.c_int]),
    "als_stats_merge": (ctypes.c_int, [_VP, ctypes.c_longlong, _VP, _VP, _VP]),
    "als_stats_moments": (ctypes.c_int, [_VP, _LL, ctypes.POINTER(_VP), ctypes.POINTER(_VP)]),
    "als_stats_result": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "als_solver_destroy": (ctypes.c_int, [_VP]),
    "als_solver_decompose": (ctypes.c_int, [_VP, _I]),
    "als_solver_geometry": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_longlong), _I]),
    "als_solver_set_state": (ctypes.c_int, [_VP, _D, ctypes.c_int, ctypes.c_int]),
    "als_solver_set_state_device": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_int]),
    "als_solver_get_state": (ctypes.c_int, [_VP, _D, ctypes.c_int, ctypes.c_int]),
    "als_solver_state_pointer": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "als_solver_advance": (ctypes.c_int, [_VP, ctypes.c_longlong]),
    "als_solver_run": (ctypes.c_int, [_VP]),
    "als_solver_info": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(MemberInfo)]),
    "als_solver_synchronize": (ctypes.c_int, [_VP]),
    "als_solver_stream": (_VP, [_VP]),
    "als_solver_launches_per_step": (ctypes.c_int, [_VP]),
    "als_solver_profile_step": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float), ctypes.c_int]),
    "als_uniform_draws": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                                         ctypes.c_double, ctypes.c_double, _D]),
    "als_structure_functions": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_double, _VP,
                                                ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                                _VP, _VP]),
    "als_write_netcdf": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _I, ctypes.c_int, _PP,
                                        _PP, ctypes.c_double, ctypes.c_int, _PP, _PP]),
    "als_solver_write_netcdf": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "als_functional_size": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, _LL]),
    "als_functional_size2": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int,
                                            ctypes.POINTER(FunctionalParams), _LL]),
    "als_functional": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int,
                                      ctypes.POINTER(FunctionalParams), _VP, ctypes.c_int,
                                      ctypes.c_longlong, ctypes.c_int, _VP, ctypes.c_longlong,
                                      ctypes.c_double, _VP]),
    "als_diffusion_ghost_cells": (ctypes.c_int, [ctypes.c_int]),
    "als_diffusion_create": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.c_int, ctypes.c_int, _PP]),
    "als_diffusion_apply": (ctypes.c_int, [_VP, _PP, _PP, _VP]),
    "als_diffusion_destroy": (ctypes.c_int, [_VP]),
    # include/als_surrogate.h
    "als_mlp_create": (ctypes.c_int, [ctypes.POINTER(MlpConfig), ctypes.c_int, _PP]),
    "als_mlp_destroy": (ctypes.c_int, [_VP]),
    "als_mlp_param_count": (ctypes.c_int, [_VP, _LL]),
    "als_mlp_init": (ctypes.c_int, [_VP, ctypes.c_ulonglong]),
    "als_mlp_set_params": (ctypes.c_int, [_VP, _VP]),
    "als_mlp_get_params": (ctypes.c_int, [_VP, _VP]),
    "als_mlp_forward": (ctypes.c_int, [_VP, _VP, ctypes.c_longlong, _VP, _VP]),
    "als_mlp_forward_layers": (ctypes.c_int, [_VP, _VP, ctypes.c_longlong, _VP, _VP]),
    "als_mlp_gradients": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, _VP,
                                         ctypes.POINTER(ctypes.c_float), _VP]),
    "als_mlp_train": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                     _VP, _VP]),
    "als_mlp_test_wait_timeout": (ctypes.c_int, [_VP, ctypes.c_uint, ctypes.c_int]),
    "als_mlp_sample_uniform": (ctypes.c_int, [_VP, ctypes.c_longlong, ctypes.c_ulonglong, _VP]),
}

_lib = None


class AlsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("als error %d: %s" % (code, message))
        self.code = code


def library_path():
    """The in-tree library, or the one named by ALS_B200_LIBRARY."""
    return os.environ.get("ALS_B200_LIBRARY") or _build.library_path()


def load():
    """Loads the shared library (once) and declares every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError("libals_b200.so is not built (%s); run `python -m alsvinn_b200.build`"
                           % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def plane_pointers(tensor):
    """ctypes array of the per-variable plane pointers of a (nvar, ...) device tensor."""
    nvar = tensor.shape[0]
    return (ctypes.c_void_p * nvar)(*[tensor[v].data_ptr() for v in range(nvar)])


def check(rc):
    if rc < 0:
        raise AlsError(rc, load().als_last_error().decode())
    return rc

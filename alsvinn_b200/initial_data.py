"""Initial data of the benchmark configurations, generated on the host.

The reference evaluates Python snippets per cell midpoint through an
embedded interpreter (alsfvm/src/init/PythonInitialData.cpp:106-276); that
machinery is not rebuilt here.  These generators produce the conserved
variables of the benchmark cases directly as padded planes (ghost cells
zero; every solver fills them with its boundary condition before the first
step, as Simulator::setInitialValue does, Simulator.cpp:161).

Primitive -> conserved follows Euler::computeConserved (Euler.hpp:236-245):
m = rho*u, E = p/(gamma-1) + 0.5*rho*(u.u).
"""
import ctypes

import numpy as np

from . import _lib

KH_PARAMETERS = 40


def padded_shape(dimension, n, ghosts):
    """(nvar, Nz, Ny, Nx) of a padded state."""
    nn = [n[d] if d < dimension else 1 for d in range(3)]
    N = [nn[d] + (2 * ghosts if d < dimension else 0) for d in range(3)]
    return (dimension + 2, N[2], N[1], N[0])


def midpoints(dimension, n, lower, upper, ghosts):
    """Cell-midpoint coordinates of the padded grid (ghost cells included)."""
    axes = []
    for d in range(3):
        if d < dimension:
            dx = (upper[d] - lower[d]) / n[d]
            idx = np.arange(n[d] + 2 * ghosts) - ghosts
            axes.append(lower[d] + (idx + 0.5) * dx)
        else:
            axes.append(np.zeros(1))
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return x, y, z


def _interior_mask(dimension, n, ghosts):
    shape = padded_shape(dimension, n, ghosts)[1:]
    mask = np.zeros(shape, dtype=bool)
    sl = []
    for d in (2, 1, 0):
        sl.append(slice(ghosts, ghosts + n[d]) if d < dimension else slice(0, 1))
    mask[tuple(sl)] = True
    return mask


def conserved(rho, velocities, p, gamma):
    """Stacks rho, m, E from primitive variables (Euler.hpp:236-245)."""
    uu = velocities[0] * velocities[0]
    for u in velocities[1:]:
        uu = uu + u * u
    E = p / (gamma - 1) + 0.5 * rho * uu
    return np.stack([rho] + [rho * u for u in velocities] + [E])


def sod(n=1024, ghosts=2, gamma=1.4):
    """Sod shock tube on [-1, 1]: (rho, u, p) = (1, 0, 1) for x < 0, else (0.125, 0, 0.1)."""
    x, _, _ = midpoints(1, (n,), (-1.0,), (1.0,), ghosts)
    left = x < 0
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    u = np.zeros_like(rho)
    U = conserved(rho, [u], p, gamma)
    U[:, ~_interior_mask(1, (n,), ghosts)] = 0.0
    return np.ascontiguousarray(U)


def uniform_draws(dimension, first_sample, count, lower=0.0, upper=1.0):
    """Parameter draws of alsuq's default generator (STLMersenne.cpp:38-85)."""
    lib = _lib.load()
    out = np.zeros((count, dimension))
    _lib.check(lib.als_uniform_draws(dimension, first_sample, count, lower, upper,
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out


def kh_perturbation(x, a, b):
    """0.01 * sum_{i=1..10} a_i cos(b_i + 2 pi i x), with a normalised to sum 1."""
    s = float(np.sum(a))
    if abs(s) < 1e-10:
        s = 1.0
    eps = np.zeros_like(x)
    for i in range(len(a)):
        eps = eps + (a[i] / s) * np.cos(b[i] + 2.0 * np.pi * (i + 1) * x)
    return 0.01 * eps


def kelvin_helmholtz(n, params, ghosts=2, gamma=1.4, dimension=2):
    """Kelvin-Helmholtz on the periodic unit square (cube for dimension 3).

    Base state rho=2, u=-0.5 in the band 0.25+eps_lo < y < 0.75+eps_hi, else
    rho=1, u=0.5; other velocities 0, p=2.5.  ``params`` holds the 40
    perturbation parameters: a_hi = params[0:10], a_lo = params[10:20],
    b_hi = params[20:30], b_lo = params[30:40].  In 3-D the interfaces are
    perturbed along x + z.  Evaluated at cell midpoints.
    """
    params = np.asarray(params, dtype=np.float64)
    if params.shape != (KH_PARAMETERS,):
        raise ValueError("Kelvin-Helmholtz takes 40 parameters")
    nn = (n, n, n)[:dimension]
    x, y, z = midpoints(dimension, nn, (0.0,) * 3, (1.0,) * 3, ghosts)
    s = x + z if dimension == 3 else x
    upper = 0.75 + kh_perturbation(s, params[0:10], params[20:30])
    lower = 0.25 + kh_perturbation(s, params[10:20], params[30:40])
    middle = (y > lower) & (y < upper)
    rho = np.where(middle, 2.0, 1.0)
    ux = np.where(middle, -0.5, 0.5)
    vel = [ux] + [np.zeros_like(ux) for _ in range(dimension - 1)]
    p = np.full_like(rho, 2.5)
    U = conserved(rho, vel, p, gamma)
    U[:, ~_interior_mask(dimension, nn, ghosts)] = 0.0
    return np.ascontiguousarray(U)


def kh_ensemble(n, first_sample, count, ghosts=2, gamma=1.4, dimension=2):
    """States of KH samples [first_sample, first_sample+count) and their parameters."""
    params = uniform_draws(KH_PARAMETERS, first_sample, count)
    states = np.stack([kelvin_helmholtz(n, params[k], ghosts, gamma, dimension)
                       for k in range(count)])
    return states, params

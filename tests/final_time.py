"""Helpers for the final-time parity fixtures (tests/golden/final_time_*.npz).

TEST INFRASTRUCTURE ONLY.  The fixtures hold the reference CPU time loop's
results on Kelvin-Helmholtz runs to T = 2 in a compact form (the full
states are too large to commit): the initial data as per-column band
limits, the step count, final time and dt sequence digest, and per
conserved variable the L1 norm, sum, 16 x 16 block sums and sha256 of the
final interior.  tests/golden/make_final_time.py writes them; the GPU tests
rebuild the initial state from the band limits and compare.
"""
import hashlib
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GAMMA = 1.4
GHOSTS = 2
BLOCK = 16
CASES = ("uq256_7", "uq256_4095", "kh1024")    # 2-D, initial data as band limits
CASES3 = ("kh3d48",)                           # 3-D, initial data by the generator
# KH 256^2 to T = 2 with other schemes: (reconstruction, flux, integrator, ghosts)
SCHEMES = {"kh256_eno3_hll_rk2": ("eno3", "hll", "rungekutta2", 3),
           "kh256_mc_hll3_rk3": ("mc", "hll3", "rungekutta3", 2),
           "kh256_weno3_hll3_rk3": ("weno3", "hll3", "rungekutta3", 3),
           "kh256_wenof2_hll_rk3": ("wenof2", "hll", "rungekutta3", 2)}
SCHEME_CASES = tuple(SCHEMES)


def fixture_path(name):
    return os.path.join(GOLDEN, "final_time_%s.npz" % name)


def load(name):
    z = np.load(fixture_path(name))
    out = {k: z[k] for k in z.files}
    for k in ("n", "sample", "ghosts", "steps", "block"):
        out[k] = int(out[k])
    for k in ("gamma", "cfl", "end_time", "t", "observable", "dts_min", "dts_max"):
        if k in out:
            out[k] = float(out[k])
    for k in ("flux", "recon", "integrator", "bc", "dts_sha256", "interior_sha256",
              "initial_sha256"):
        if k in out:
            out[k] = str(out[k])
    return out


def band_limits_of(U, n, ghosts=GHOSTS):
    """First and one-past-last interior row of the KH band (rho == 2) per column."""
    rho = U[0, 0, ghosts:ghosts + n, ghosts:ghosts + n]
    inside = rho == 2.0
    lo = np.zeros(n, dtype=np.int32)
    hi = np.zeros(n, dtype=np.int32)
    for x in range(n):
        rows = np.nonzero(inside[:, x])[0]
        lo[x], hi[x] = rows[0], rows[-1] + 1
        if rows.size != hi[x] - lo[x]:
            raise ValueError("band is not contiguous in column %d" % x)
    return lo, hi


def kh_state_from_bands(n, lo, hi, ghosts=GHOSTS, gamma=GAMMA):
    """The padded KH state whose band covers rows [lo[x], hi[x]) of column x
    (rho = 2, u = -0.5 inside, rho = 1, u = 0.5 outside, v = 0, p = 2.5;
    ghost cells zero), converted to conserved variables the way the
    initial-data generator does (Euler.hpp:236-245)."""
    N = n + 2 * ghosts
    rows = np.arange(n)[:, None]
    inside = (rows >= lo[None, :]) & (rows < hi[None, :])
    rho = np.where(inside, 2.0, 1.0)
    u = np.where(inside, -0.5, 0.5)
    v = np.zeros_like(u)
    p = np.full_like(rho, 2.5)
    uu = u * u + v * v
    E = p / (gamma - 1) + 0.5 * rho * uu
    U = np.zeros((4, 1, N, N))
    for k, plane in enumerate((rho, rho * u, rho * v, E)):
        U[k, 0, ghosts:ghosts + n, ghosts:ghosts + n] = plane
    return U


def interior(U, n, ghosts=GHOSTS):
    return np.ascontiguousarray(U[:, 0, ghosts:ghosts + n, ghosts:ghosts + n])


def summary(U, n, ghosts=GHOSTS):
    """Per-variable L1 norms and sums (math.fsum: exactly rounded), 16 x 16
    block sums and the sha256 of the final interior."""
    I = interior(U, n, ghosts)
    l1 = np.array([math.fsum(np.abs(I[v]).ravel()) for v in range(I.shape[0])])
    sums = np.array([math.fsum(I[v].ravel()) for v in range(I.shape[0])])
    b = n // BLOCK
    blocks = I.reshape(I.shape[0], b, BLOCK, b, BLOCK).sum(axis=(2, 4))
    return {"l1": l1, "sums": sums, "block_sums": blocks,
            "interior_sha256": hashlib.sha256(I.tobytes()).hexdigest()}


BLOCK3 = 8


def interior3(U, n, ghosts=GHOSTS):
    return np.ascontiguousarray(U[:, ghosts:ghosts + n, ghosts:ghosts + n, ghosts:ghosts + n])


def summary3(U, n, ghosts=GHOSTS):
    """summary() of a 3-D state: per-variable L1 norms and sums, 8 x 8 x 8
    block sums and the sha256 of the final interior."""
    I = interior3(U, n, ghosts)
    l1 = np.array([math.fsum(np.abs(I[v]).ravel()) for v in range(I.shape[0])])
    sums = np.array([math.fsum(I[v].ravel()) for v in range(I.shape[0])])
    b = n // BLOCK3
    blocks = I.reshape(I.shape[0], b, BLOCK3, b, BLOCK3, b, BLOCK3).sum(axis=(2, 4, 6))
    return {"l1": l1, "sums": sums, "block_sums": blocks,
            "interior_sha256": hashlib.sha256(I.tobytes()).hexdigest()}


# Riemann problems with Neumann boundaries, run to their final time:
# name: (dimension, n, reconstruction, flux, integrator, ghosts, end time)
RIEMANN = {"sod2d256_neumann": (2, 256, "weno2", "hll3", "rungekutta3", 2, 0.25),
           "sod3d32_neumann": (3, 32, "weno2", "hll3", "rungekutta3", 2, 0.2)}
RIEMANN_CASES = tuple(RIEMANN)


def riemann_state(dim, n, ghosts=GHOSTS, gamma=GAMMA):
    """Sod across the diagonal of the unit square / cube: rho = 1, p = 1
    where the cell midpoints' coordinates sum to less than dim / 2, else
    rho = 0.125, p = 0.1; at rest; ghost cells zero (padded planes)."""
    x = (np.arange(n) + 0.5) / n
    grids = np.meshgrid(*([x] * dim), indexing="ij")      # axis order z, y, x reversed below
    total = sum(grids)
    inside = total < dim / 2.0
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 1.0, 0.1)
    E = p / (gamma - 1)
    N = n + 2 * ghosts
    shape = (dim + 2,) + (1,) * (3 - dim) + (N,) * dim
    U = np.zeros(shape)
    inner = (slice(ghosts, ghosts + n),) * dim
    U[(0,) + (0,) * (3 - dim) + inner] = rho
    U[(dim + 1,) + (0,) * (3 - dim) + inner] = E
    return U


def state_digest(U):
    return hashlib.sha256(np.ascontiguousarray(U, dtype=np.float64).tobytes()).hexdigest()


def observable(U, n, ghosts=GHOSTS):
    """Mean density over [0.25, 0.75]^2 (cells round(0.25 n) .. round(0.75 n))."""
    lo, hi = int(round(0.25 * n)), int(round(0.75 * n))
    I = interior(U, n, ghosts)
    return math.fsum(I[0, lo:hi, lo:hi].ravel()) / float((hi - lo) ** 2)


def dts_digest(dts):
    return hashlib.sha256(np.ascontiguousarray(dts, dtype=np.float64).tobytes()).hexdigest()

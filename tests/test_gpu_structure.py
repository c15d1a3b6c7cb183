"""Structure-function statistics on the GPU against the C oracle.

The oracle (oracle/als_oracle.c) reproduces the reference's
dispatchComputeStructureCubeCPU bit for bit (tests/test_oracle.py); the GPU
sums the same positive terms in another order and divides once, so the
agreement bar is 1e-12 relative per entry (FP64 rounding of sums of up to
~1e5 terms).
"""
import numpy as np
import pytest
import torch

from alsvinn_b200.functionals import structure_functions
from oracle_lib import smooth_random_state

pytestmark = pytest.mark.gpu

CASES = [(1, (64,)), (2, (24, 20)), (2, (33, 17)), (3, (10, 9, 8))]


def _states(dim, n, g, members, seed):
    return np.stack([smooth_random_state(seed + m, dim, n, g) for m in range(members)])


@pytest.mark.parametrize("dim,n", CASES)
@pytest.mark.parametrize("bc", ["periodic", "neumann"])
@pytest.mark.parametrize("p", [1.0, 2.0, 3.0, 2.5])
def test_structure_cube_matches_oracle(c_oracle, dim, n, bc, p):
    g = 2
    H = 6 if dim < 3 else 4
    st = _states(dim, n, g, 3, 100 * dim + int(10 * p))
    out = structure_functions(torch.from_numpy(st).cuda(), dim, n, g, bc, "cube", H, p)
    out = out.cpu().numpy()
    for m in range(st.shape[0]):
        ref = c_oracle.structure_cube(dim, n, g, bc, H, p, st[m])
        np.testing.assert_allclose(out[m], ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("dim,n", CASES)
@pytest.mark.parametrize("bc", ["periodic", "neumann"])
def test_structure_basic_matches_oracle(c_oracle, dim, n, bc):
    g = 2
    H = 7
    st = _states(dim, n, g, 2, 500 + dim)
    for direction in range(dim):
        for p in (1.0, 2.0, 1.5):
            out = structure_functions(torch.from_numpy(st).cuda(), dim, n, g, bc, "basic", H, p,
                                      direction=direction).cpu().numpy()
            for m in range(st.shape[0]):
                ref = c_oracle.structure_basic(dim, n, g, bc, direction, H, p, st[m])
                # pow on the device vs the host's pow: a few ulp per term
                np.testing.assert_allclose(out[m], ref, rtol=1e-12, atol=1e-300)


def test_structure_cube_of_fp32_members(c_oracle):
    dim, n, g, H, p = 2, (40, 32), 2, 9, 2.0
    st = _states(dim, n, g, 4, 900).astype(np.float32)
    out = structure_functions(torch.from_numpy(st).cuda(), dim, n, g, "periodic", "cube", H, p)
    out = out.cpu().numpy()
    for m in range(st.shape[0]):
        ref = c_oracle.structure_cube(dim, n, g, "periodic", H, p, st[m].astype(np.float64))
        np.testing.assert_allclose(out[m], ref, rtol=1e-12)


def test_structure_cube_radius_beyond_the_grid_wraps(c_oracle):
    """H larger than the grid: periodic points wrap more than once, Neumann clamps."""
    dim, n, g, H = 2, (6, 5), 2, 9
    st = _states(dim, n, g, 1, 77)
    for bc in ("periodic", "neumann"):
        out = structure_functions(torch.from_numpy(st).cuda(), dim, n, g, bc, "cube", H, 1.0)
        ref = c_oracle.structure_cube(dim, n, g, bc, H, 1.0, st[0])
        np.testing.assert_allclose(out.cpu().numpy()[0], ref, rtol=1e-12)

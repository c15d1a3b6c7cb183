"""The TeCNO diffusion operator on the GPU (als_diffusion_*, the Python
DiffusionOperator), against the oracle and the reference's fixtures.

The operator evaluates entropy variables, which take logarithms: the CUDA
path calls the device `log`, the reference and the oracle the C library's,
and the two may differ in the last bit.  Comparisons therefore use a
relative tolerance of 1e-10 (absolute 1e-12 on values of order one); step
counts are compared exactly.  The operator's work arrays persist between
calls as the reference's do, so every check applies one operator to several
states in a row.
"""
import os

import numpy as np
import pytest
import torch

import alsvinn_b200 as als
from conftest import GOLDEN, load_golden
from oracle_lib import smooth_random_state
from plugin_loop import run_plugin_time_loop

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-10, 1e-12


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _fixtures(prefix):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.startswith(prefix) and f.endswith(".npz"))


@pytest.mark.parametrize("dim,n", [(1, (24,)), (2, (12, 11)), (3, (9, 10, 8))])
@pytest.mark.parametrize("kind", ["tecnoroe", "tecnorusanov"])
@pytest.mark.parametrize("recon", ["none", "eno2", "eno3", "eno4"])
def test_diffusion_operator_matches_oracle(c_oracle, dim, n, kind, recon):
    """Three calls of one operator against the oracle's restatement with
    its persistent state (relative 1e-10)."""
    g = als.diffusion_ghost_cells(recon)
    seed = 7000 + 31 * dim + 7 * ["none", "eno2", "eno3", "eno4"].index(recon) + len(kind)
    states = [smooth_random_state(seed + k, dim, n, g) for k in range(3)]
    outs = [np.random.default_rng(seed + k).uniform(-1, 1, states[0].shape) for k in range(3)]
    cfg = c_oracle.config(dim, n, [0.0] * dim, [1.0] * dim, "hll", "none", "rungekutta3",
                          "neumann", 1.4)
    cfg.g = g
    st = c_oracle.diffusion_state(cfg)
    with als.DiffusionOperator(dim, n, kind, recon) as op:
        assert op.getNumberOfGhostCells() == g
        for k in range(3):
            ref = c_oracle.apply_diffusion(cfg, kind, recon, st, states[k], outs[k])
            out = _dev(outs[k])
            op.applyDiffusion(out, _dev(states[k]))
            np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", _fixtures("diffusion_apply_"))
def test_diffusion_operator_reproduces_reference_calls(name):
    """Fixtures of three successive calls made by the reference build."""
    z = load_golden(name)
    dim = int(z["dim"])
    with als.DiffusionOperator(dim, tuple(z["n"]), str(z["diffusion"]),
                               str(z["diffusion_recon"]), ghosts=int(z["ghosts"])) as op:
        for k in range(z["states"].shape[0]):
            out = _dev(z["outs"][k])
            op.applyDiffusion(out, _dev(z["states"][k]))
            np.testing.assert_allclose(out.cpu().numpy(), z["result"][k], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("name", _fixtures("tecnodiff_"))
def test_plugin_time_loop_with_diffusion_reproduces_reference(name):
    """Whole simulations with flux + TeCNO diffusion through the plug-in
    classes against the reference's own time loop (relative 1e-10)."""
    z = load_golden(name)
    U, steps, t = run_plugin_time_loop(z, str(z["diffusion"]), str(z["diffusion_recon"]))
    assert steps == int(z["steps"])
    assert abs(t - float(z["t"])) <= 1e-15
    np.testing.assert_allclose(U, z["final"], rtol=RTOL, atol=ATOL)


def test_diffusion_of_a_constant_state_is_zero():
    """Equal neighbours: the reconstructed jumps vanish and so does the
    diffusion on the interior cells away from the last ones (2-D, Roe
    matrix, ENO2), to rounding of the ENO weights (which sum to 1 only up
    to rounding)."""
    dim, n = 2, (20, 18)
    g = als.diffusion_ghost_cells("eno2")
    shp = (4, 1, n[1] + 2 * g, n[0] + 2 * g)
    U = np.empty(shp)
    U[0], U[1], U[2], U[3] = 1.2, 0.3, -0.1, 2.5
    with als.DiffusionOperator(dim, n, "tecnoroe", "eno2") as op:
        out = torch.zeros(shp, dtype=torch.float64, device="cuda")
        # the first call reads never-written entries (42) next to the last
        # cells along each direction, as the reference does; the second call
        # sees every entry written
        op.applyDiffusion(out, _dev(U))
        out.zero_()
        op.applyDiffusion(out, _dev(U))
        inner = out.cpu().numpy()[:, 0, g + 1:-(g + 1), g + 1:-(g + 1)]
        assert np.abs(inner).max() < 1e-12

"""RungeKutta4 through the plug-in integrator (als_integrator_combine,
als_integrator_combine_rk4): whole simulations driven by the plug-in classes
against the reference's fixtures and the oracle, bit for bit."""
import os
import zlib

import numpy as np
import pytest

import alsvinn_b200 as als
from alsvinn_b200 import _lib
from conftest import GOLDEN, load_golden
from oracle_lib import ghost_cells, smooth_random_state
from plugin_loop import run_plugin_time_loop

pytestmark = pytest.mark.gpu

RK4_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                      if f.startswith("rk4_") and f.endswith(".npz"))


@pytest.mark.parametrize("name", RK4_FIXTURES)
def test_rk4_plugin_loop_reproduces_reference_fixture(name):
    z = load_golden(name)
    U, steps, t = run_plugin_time_loop(z)
    assert steps == int(z["steps"]) and t == float(z["t"])
    np.testing.assert_array_equal(U, z["final"])


@pytest.mark.parametrize("dim,n", [(1, (40,)), (2, (19, 21)), (3, (10, 9, 11))])
@pytest.mark.parametrize("recon,flux", [("weno2", "hll3"), ("eno3", "hll"), ("mc", "central"),
                                        ("none", "tecno4")])
@pytest.mark.parametrize("bc", ["neumann", "periodic"])
def test_rk4_plugin_loop_matches_oracle(c_oracle, dim, n, recon, flux, bc):
    """Fresh random states: the plug-in loop with RK4 against the oracle's
    RK4 time loop (bit for bit; tecno4 within 1e-10 for its logarithms)."""
    g = ghost_cells(recon, flux)
    seed = zlib.crc32(("rk4-%d-%s-%s-%s" % (dim, recon, flux, bc)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    cfg = c_oracle.config(dim, n, lo, hi, flux, recon, "rungekutta4", bc, 1.4)
    rc, U_ref, dts, steps, t = c_oracle.simulate(cfg, st, 0.4, 0.04)
    assert rc == 0
    z = dict(dim=dim, n=np.array(n), lower=np.array(lo), upper=np.array(hi), flux=flux,
             recon=recon, integrator="rungekutta4", bc=bc, cfl=0.4, end_time=0.04, gamma=1.4,
             initial=st)
    U, s, tt = run_plugin_time_loop(z)
    assert s == steps
    if flux.startswith("tecno"):
        np.testing.assert_allclose(U, U_ref, rtol=1e-10, atol=1e-12)
    else:
        assert tt == t
        np.testing.assert_array_equal(U, U_ref)


def test_fused_solver_refuses_rk4():
    """The fused solver runs FE/RK2/RK3; RK4 is the plug-in integrator's."""
    with pytest.raises(_lib.AlsError) as e:
        als.Simulator(1, (32,), integrator="rungekutta4")
    assert e.value.code == -4

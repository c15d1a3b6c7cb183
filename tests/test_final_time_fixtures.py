"""CPU checks of the final-time fixtures (reference CPU time loop to T = 2).

* The initial state rebuilt from the stored band limits equals the
  Kelvin-Helmholtz generator's for the stored parameters.
* The 4096-sample FP64 UQ oracle ensemble (made on the GPU by
  tests/golden/make_uq_oracle.py) is pinned to the reference's CPU path at
  T = 2 on members 7 and 4095: the same step counts and observables.
* Where the reference build is present, its STLMersenne draws equal the
  stored parameters.
"""
import os

import numpy as np
import pytest

import alsvinn_b200.initial_data as init
import final_time as ft


@pytest.mark.parametrize("name", ft.CASES + ft.SCHEME_CASES)
def test_band_limits_rebuild_the_generator_state(name):
    z = ft.load(name)
    U = init.kelvin_helmholtz(z["n"], z["params"], z["ghosts"], z["gamma"])
    np.testing.assert_array_equal(
        ft.kh_state_from_bands(z["n"], z["band_lo"], z["band_hi"], z["ghosts"]), U)
    if name in ft.SCHEMES:
        recon, flux, integrator, ghosts = ft.SCHEMES[name]
        assert (z["recon"], z["flux"], z["integrator"], z["ghosts"]) == \
            (recon, flux, integrator, ghosts)
    assert z["steps"] == len(z["dts_head"]) or z["steps"] > 64
    assert z["t"] == z["end_time"]


@pytest.mark.parametrize("name", ft.RIEMANN_CASES)
def test_riemann_state_is_the_fixture_initial_state(name):
    z = ft.load(name)
    dim, n, recon, flux, integrator, ghosts, end_time = ft.RIEMANN[name]
    assert (int(z["dim"]), z["n"], z["recon"], z["flux"], z["integrator"], z["ghosts"],
            z["end_time"], z["bc"]) == (dim, n, recon, flux, integrator, ghosts, end_time,
                                        "neumann")
    assert ft.state_digest(ft.riemann_state(dim, n, ghosts)) == z["initial_sha256"]
    assert z["t"] == z["end_time"]


@pytest.mark.parametrize("name", ft.CASES3)
def test_3d_generator_state_is_the_fixture_initial_state(name):
    z = ft.load(name)
    U = init.kelvin_helmholtz(z["n"], z["params"], z["ghosts"], z["gamma"], dimension=3)
    assert ft.state_digest(U) == z["initial_sha256"]
    assert z["t"] == z["end_time"] and z["steps"] > 64


@pytest.mark.parametrize("name", ("uq256_7", "uq256_4095"))
def test_uq_oracle_ensemble_pinned_to_reference_members(name):
    z = ft.load(name)
    oracle = np.load(ft.GOLDEN + "/uq_kh256_fp64_4096.npz")
    s = z["sample"]
    assert int(oracle["steps"][s]) == z["steps"]
    # the ensemble's observable is an FP64 device sum: equal to the reference
    # member's exactly rounded one within a few ulp
    assert abs(float(oracle["y"][s]) - z["observable"]) <= 1e-14 * abs(z["observable"])


def test_parameters_are_the_reference_draws(ref_oracle):
    """The stored parameters are the reference generator's draws.  Its
    engine is one per process and only moves forward, so the draws are
    taken in a fresh process, in increasing sample order."""
    import json
    import subprocess
    import sys
    zs = sorted((ft.load(name) for name in ft.CASES + ft.CASES3 + ft.SCHEME_CASES),
                key=lambda z: z["sample"])
    samples = sorted(set(z["sample"] for z in zs))
    code = ("import json, sys; sys.path.insert(0, %r); from oracle_lib import RefOracle; "
            "r = RefOracle(); print(json.dumps([r.stlmersenne(40, s, 1)[0].tolist() for s in %r]))"
            % (os.path.dirname(os.path.abspath(__file__)), samples))
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True)
    draws = dict(zip(samples, json.loads(out.stdout.strip().splitlines()[-1])))
    for z in zs:
        np.testing.assert_array_equal(np.array(draws[z["sample"]]), z["params"])

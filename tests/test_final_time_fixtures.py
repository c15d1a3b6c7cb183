"""CPU checks of the final-time fixtures (reference CPU time loop to T = 2).

* The initial state rebuilt from the stored band limits equals the
  Kelvin-Helmholtz generator's for the stored parameters.
* The 4096-sample FP64 UQ oracle ensemble (made on the GPU by
  tests/golden/make_uq_oracle.py) is pinned to the reference's CPU path at
  T = 2 on members 7 and 4095: the same step counts and observables.
* Where the reference build is present, its STLMersenne draws equal the
  stored parameters.
"""
import numpy as np
import pytest

import alsvinn_b200.initial_data as init
import final_time as ft


@pytest.mark.parametrize("name", ft.CASES)
def test_band_limits_rebuild_the_generator_state(name):
    z = ft.load(name)
    U = init.kelvin_helmholtz(z["n"], z["params"], z["ghosts"], z["gamma"])
    np.testing.assert_array_equal(ft.kh_state_from_bands(z["n"], z["band_lo"], z["band_hi"]), U)
    assert z["steps"] == len(z["dts_head"]) or z["steps"] > 64
    assert z["t"] == z["end_time"]


@pytest.mark.parametrize("name", ("uq256_7", "uq256_4095"))
def test_uq_oracle_ensemble_pinned_to_reference_members(name):
    z = ft.load(name)
    oracle = np.load(ft.GOLDEN + "/uq_kh256_fp64_4096.npz")
    s = z["sample"]
    assert int(oracle["steps"][s]) == z["steps"]
    # the ensemble's observable is an FP64 device sum: equal to the reference
    # member's exactly rounded one within a few ulp
    assert abs(float(oracle["y"][s]) - z["observable"]) <= 1e-14 * abs(z["observable"])


@pytest.mark.parametrize("name", ft.CASES)
def test_parameters_are_the_reference_draws(ref_oracle, name):
    z = ft.load(name)
    np.testing.assert_array_equal(ref_oracle.stlmersenne(40, z["sample"], 1)[0], z["params"])

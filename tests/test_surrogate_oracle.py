"""CPU checks of the surrogate's oracle and of the UQ estimators.

The MLP oracle (oracle/mlp_oracle.py) is the checker of the tensor-core
kernels, so its back-propagation is verified here against central finite
differences of its own FP64 forward pass.  The control-variate estimator is
checked on synthetic data with a known answer.
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as mo  # noqa: E402

from alsvinn_b200 import uq  # noqa: E402


def test_parameter_count_of_the_kh_network():
    assert mo.param_count(40, 256, 4) == 208129


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 1.0 + 2.0 ** -9, -2.5, 3.0e-3])
    r = mo.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                                # 1 + 2^-8 is halfway: even is 1.0
    assert r[2] == 1.0 + 2.0 ** -7                   # above halfway rounds up
    assert r[3] == 1.0
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8


@pytest.mark.parametrize("hidden", [1, 3])
def test_oracle_backprop_matches_finite_differences(hidden):
    rng = np.random.default_rng(3 + hidden)
    inputs, width, B = 5, 8, 7
    n = mo.param_count(inputs, width, hidden)
    p = rng.normal(0, 0.5, n)
    x = rng.uniform(0, 1, (B, inputs))
    t = rng.normal(0, 1, B)
    g, loss = mo.gradients(p, x, t, inputs, width, hidden, bf16_path=False)
    h = 1e-6
    for k in rng.choice(n, 25, replace=False):
        pp = p.copy()
        pm = p.copy()
        pp[k] += h
        pm[k] -= h
        lp = np.mean((mo.forward(pp, x, inputs, width, hidden, False)[0] - t) ** 2)
        lm = np.mean((mo.forward(pm, x, inputs, width, hidden, False)[0] - t) ** 2)
        assert abs((lp - lm) / (2 * h) - g[k]) <= 1e-6 * max(1.0, abs(g[k]))
    assert loss == pytest.approx(np.mean((mo.forward(p, x, inputs, width, hidden, False)[0] - t) ** 2))


def test_control_variate_with_exact_surrogate_is_exact():
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 1, 4096)
    y = 3.0 + 2.0 * x
    # surrogate = the observable itself: E[f] = 4, E[f^2] = Var + mean^2 = 4/12 + 16
    m, v, beta, _ = uq.control_variate(y[:64], y[:64], 4.0, 4.0 / 12.0 + 16.0)
    assert beta == pytest.approx(1.0)
    assert m == pytest.approx(4.0, abs=1e-12)
    assert v == pytest.approx(4.0 / 12.0, abs=1e-12)


def test_control_variate_reduces_the_error_of_plain_mc():
    rng = np.random.default_rng(1)
    err_plain, err_cv = [], []
    for _ in range(200):
        x = rng.uniform(0, 1, 128)
        y = np.sin(3 * x) + 0.05 * rng.normal(size=x.size)   # observable with noise
        f = np.sin(3 * x)                                     # surrogate
        ef = (1 - np.cos(3.0)) / 3.0
        ef2 = 0.5 - np.sin(6.0) / 12.0
        true_mean = ef
        err_plain.append(uq.plain_mc(y)[0] - true_mean)
        err_cv.append(uq.control_variate(y, f, ef, ef2)[0] - true_mean)
    rms_plain = np.sqrt(np.mean(np.square(err_plain)))
    rms_cv = np.sqrt(np.mean(np.square(err_cv)))
    assert rms_cv < 0.2 * rms_plain


def test_uq_oracle_ensemble_fixture():
    """The committed FP64 ensemble the UQ estimators are measured against."""
    from conftest import load_golden
    z = load_golden("uq_kh256_fp64_4096")
    y = z["y"]
    assert z["samples"] == 4096 and y.shape == (4096,) and z["n"] == 256
    assert z["end_time"] == 2.0 and z["first_sample"] == 0
    assert np.all(np.isfinite(y))
    # mean density over [0.25,0.75]^2 starts near 2 (heavy band) and mixes towards 1.5
    assert 1.5 < y.mean() < 2.0 and 0 < y.std() < 0.2
    assert z["steps"].min() > 5000
    m, v = uq.plain_mc(y)
    assert m == pytest.approx(y.mean(), rel=1e-15) and v == pytest.approx(y.var(), rel=1e-12)
    # the FP64 Welford density statistics cover the padded plane
    assert z["rho_mean"].shape == (1, 260, 260) and np.all(z["rho_var"] >= 0)

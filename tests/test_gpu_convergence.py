"""Convergence rates, as the reference's own tests measure them, on the GPU
path (the plug-in Reconstruction, Boundary and Integrator classes).

* test/library_tests/src/fvm/reconstruction/ReconstructionConvergenceTest.cpp:
  a 1-D periodic grid on [0, 1] of n = 2^5 .. 2^14 cells holding the cell
  averages of rho = sin(2 pi x) + 2 (p = 2.5, u = 0); the reconstructed
  left and right densities of every cell are compared with rho at the
  cell's faces, and the L1 and L-infinity errors' rates come from a
  least-squares line through (log2 n, log2 error).  Expected rates are the
  reference's double-precision ones.
* test/library_tests/src/uq/generators/MeanVarTest.cpp: uniform draws of
  the STLMersenne generator (40 dimensions, M = 2^4 .. 2^19 samples, each M
  continuing the sequence as the reference's process-wide engine does)
  accumulated by the FP64 Welford MeanVariance on the device; the RMS
  errors of mean and variance over the 40 dimensions must fall at rate
  1/2 (at least 0.49).
* test/library_tests/src/fvm/integrator/ForwardEulerTest.cpp and
  RungeKutta2Test.cpp: the same system (below); every rate between
  consecutive resolutions within 0.1 of -1 (N = 2^4 .. 2^14) and within
  0.05 of -2 (N = 2^6 .. 2^14).
* test/library_tests/src/fvm/integrator/IntegratorConvergenceTest.cpp:
  du/dt = u, u(0) = 1, integrated to t = 1 with N = 2^6 .. 2^9 constant
  steps through the integrator's stage combinations (the system returns
  dt u and a wave speed of 1, so that with CFL 1 and unit cells every step
  is one unit of the integrator's own time); the error |e - u(1)| has to
  fall at least at the reference's rate.
"""
import math

import numpy as np
import pytest
import torch

import alsvinn_b200 as als

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def _f(x):
    return np.sin(2 * np.pi * x) + 2


def _average_f(a, b):
    return (-np.cos(2 * np.pi * b) + np.cos(2 * np.pi * a)) / (2 * np.pi * (b - a)) + 2


def _rate(x, y):
    """-slope of the least-squares line through (x, y) (polyfit.hpp's linearFit)."""
    return -np.polyfit(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64), 1)[0]


# (name, L1 rate, L-infinity rate): ReconstructionConvergenceTest.cpp, FP64 values
RECONSTRUCTIONS = [("weno2", 1.99, 1.99), ("mc", 1.99, 1.99), ("wenof2", 1.99, 1.99),
                   ("eno2", 1.98, 1.99), ("eno3", 2.95, 2.99), ("none", 0.999, 0.999)]


@pytest.mark.parametrize("name,l1_rate,linf_rate", RECONSTRUCTIONS,
                         ids=[r[0] for r in RECONSTRUCTIONS])
def test_reconstruction_convergence(name, l1_rate, linf_rate):
    logs = {"n": [], "l1_left": [], "l1_right": [], "linf_left": [], "linf_right": []}
    for k in range(5, 15):
        n = 1 << k
        rec = als.Reconstruction(1, (n,), name, gamma=GAMMA)
        g = rec.getNumberOfGhostCells()
        dx = 1.0 / n
        a = np.arange(n) * dx
        b = (np.arange(n) + 1) * dx
        U = np.zeros((3, 1, 1, n + 2 * g))
        U[0, 0, 0, g:g + n] = _average_f(a, b)
        U[2, 0, 0, g:g + n] = 2.5 / (GAMMA - 1)       # p = 2.5, u = 0
        conserved = torch.from_numpy(U).cuda()
        als.Boundary(1, (n,), g, "periodic").applyBoundaryConditions(conserved)
        left = torch.zeros_like(conserved)
        right = torch.zeros_like(conserved)
        rec.performReconstruction(conserved, 0, left, right)
        torch.cuda.synchronize()
        lv = left[0, 0, 0, g:g + n].cpu().numpy()
        rv = right[0, 0, 0, g:g + n].cpu().numpy()
        dl = np.abs(lv - _f(a))
        dr = np.abs(rv - _f(b))
        logs["n"].append(math.log2(n))
        logs["l1_left"].append(math.log2(dl.sum() / n))
        logs["l1_right"].append(math.log2(dr.sum() / n))
        logs["linf_left"].append(math.log2(dl.max()))
        logs["linf_right"].append(math.log2(dr.max()))
    for key, expect in (("l1_left", l1_rate), ("l1_right", l1_rate),
                        ("linf_left", linf_rate), ("linf_right", linf_rate)):
        rate = _rate(logs["n"], logs[key])
        assert rate >= expect, (name, key, rate)


class _ODESystem:
    """The reference test's system: L(u) = dt u, wave speed (1, 0, 0)."""

    def __init__(self, dt):
        self.dt = dt

    def computeFlux(self, conserved, out, stream=0, compute_wave_speed=True):
        torch.mul(conserved, self.dt, out=out)
        return np.array([1.0, 0.0, 0.0])


# IntegratorConvergenceTest.cpp, FP64 values
INTEGRATORS = [("forwardeuler", 0.9), ("rungekutta2", 1.9), ("rungekutta3", 2.9),
               ("rungekutta4", 3.9)]


def _ode_errors(name, ks):
    """(log N, log |e - u(1)|) for N = 2 << k, k in ks."""
    errors, resolutions = [], []
    for k in ks:
        N = 2 << k
        dt = 1.0 / N
        integ = als.Integrator(name, _ODESystem(dt), cfl=1.0)
        volumes = [torch.ones(1, dtype=torch.float64, device="cuda")
                   for _ in range(integ.getNumberOfSubsteps() + 1)]
        t = 0.0
        for _ in range(N):
            for substep in range(integ.getNumberOfSubsteps()):
                step = integ.performSubstep(volumes, (1.0, 1.0, 1.0), 1.0, volumes[substep + 1],
                                            substep, t, 1e9)
                assert step == 1.0
            volumes[0], volumes[-1] = volumes[-1], volumes[0]
            t += dt
        assert t == 1.0
        torch.cuda.synchronize()
        u = float(volumes[0].item())
        errors.append(math.log(abs(math.exp(1.0) - u)))
        resolutions.append(math.log(N))
    return resolutions, errors


@pytest.mark.parametrize("name,expected", INTEGRATORS, ids=[i[0] for i in INTEGRATORS])
def test_integrator_convergence(name, expected):
    resolutions, errors = _ode_errors(name, range(5, 9))
    assert _rate(resolutions, errors) >= expected, (name, _rate(resolutions, errors))


@pytest.mark.parametrize("name,ks,rate,tol", [("forwardeuler", range(3, 14), -1.0, 0.1),
                                              ("rungekutta2", range(5, 14), -2.0, 5e-2)],
                         ids=["ForwardEulerTest", "RungeKutta2Test"])
def test_integrator_rate_between_resolutions(name, ks, rate, tol):
    resolutions, errors = _ode_errors(name, ks)
    slopes = np.diff(errors) / np.diff(resolutions)
    assert np.all(np.abs(slopes - rate) <= tol), slopes


def test_monte_carlo_mean_and_variance_converge_at_rate_one_half():
    D = 40
    log_m, log_mean_err, log_var_err = [], [], []
    first = 0
    for k in range(4, 20):
        M = 1 << k
        draws = als.uniform_draws(D, first, M)
        first += M
        mv = als.MeanVariance(D)
        try:
            mv.add(torch.from_numpy(draws).cuda())
            mean = torch.zeros(D, dtype=torch.float64, device="cuda")
            var = torch.zeros(D, dtype=torch.float64, device="cuda")
            mv.result(mean, var)
            torch.cuda.synchronize()
        finally:
            mv.close()
        mean_err = math.sqrt(float(((mean.cpu().numpy() - 0.5) ** 2).sum()))
        var_err = math.sqrt(float(((var.cpu().numpy() - 1.0 / 12.0) ** 2).sum()))
        log_m.append(math.log(M))
        log_mean_err.append(math.log(mean_err))
        log_var_err.append(math.log(var_err))
    assert _rate(log_m, log_mean_err) >= 0.49, _rate(log_m, log_mean_err)
    assert _rate(log_m, log_var_err) >= 0.49, _rate(log_m, log_var_err)


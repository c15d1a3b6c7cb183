"""Uncertainty quantification over Kelvin-Helmholtz ensembles.

The reference runs UQ samples one after another (alsuq/src/run/Runner.cpp:42-78,
one FiniteVolumeSimulator per sample) and accumulates raw moments
(alsuq/src/stats/MeanVariance.cpp:30-67).  Here a whole ensemble advances in
one batched simulator (one launch per RK stage over every member), the
observable of every member is an FP64 region sum read on the device, and
the estimators below are FP64:

* ``plain_mc``: the sample mean and the biased (1/M) variance of the
  observable, the reference's MeanVariance definition;
* ``control_variate``: the same two moments with a surrogate f(X) of the
  observable as control variate: E[Y] = E[Y - b (f - E f)] with
  b = cov(Y, f) / var(f) fitted on the samples, E[Y^2] likewise with f^2,
  and E f, E f^2 taken from many cheap surrogate evaluations.
"""
import time

import numpy as np

from .initial_data import KH_PARAMETERS, kelvin_helmholtz, uniform_draws
from .simulator import MeanVariance, Simulator

KH_BOX = (0.25, 0.75)


def _box_cells(n, box):
    lo = int(round(box[0] * n))
    hi = int(round(box[1] * n))
    return lo, hi


def kh_observable_ensemble(n, first_sample, count, precision="fp64", end_time=2.0, cfl=0.4,
                           box=KH_BOX, device=0, field_statistics=False, keep_statistics=False,
                           upload_chunk=256):
    """Solves the 2-D KH samples [first_sample, first_sample + count) at n x n
    to ``end_time`` (WENO2 + HLL3, RK3, periodic) as one batched ensemble.

    Returns ``(params, y, info)``: the (count, 40) perturbation parameters of
    alsuq's generator (STLMersenne order), the observable y = mean density
    over box x box at the end time (FP64 region sums), and a dict with the
    solve's wall-clock seconds (states resident on the device), the steps of
    every member and, with ``field_statistics``, the FP64 Welford mean and
    variance of every conserved variable over the ensemble (padded planes).
    With ``keep_statistics`` the FP64 accumulator itself is returned open in
    info["statistics"] (for merging across GPUs; the caller closes it).
    """
    params = uniform_draws(KH_PARAMETERS, first_sample, count)
    with Simulator(2, (n, n), (0.0, 0.0), (1.0, 1.0), flux="hll3", reconstruction="weno2",
                   integrator="rungekutta3", boundary="periodic", cfl=cfl, end_time=end_time,
                   precision=precision, members=count, device=device) as sim:
        g = sim.ghosts
        for a in range(0, count, upload_chunk):
            k = min(upload_chunk, count - a)
            states = np.stack([kelvin_helmholtz(n, params[a + j], g) for j in range(k)])
            sim.set_state(states, first_member=a)
        sim.synchronize()
        t0 = time.perf_counter()
        sim.run()
        sim.synchronize()
        seconds = time.perf_counter() - t0
        lo, hi = _box_cells(n, box)
        sums = sim.region_sums(0, count, lo=(lo, lo), hi=(hi, hi))
        y = sums[:, 0] / float((hi - lo) ** 2)
        steps = np.array([sim.info(m)["steps"] for m in range(count)])
        info = {"solve_seconds": seconds, "steps": steps, "n": n, "precision": precision,
                "end_time": end_time, "box_cells": (lo, hi), "shape": sim.shape,
                "stage_launches": int(steps.max()) * sim.launches_per_step()}
        if keep_statistics:
            mv = MeanVariance(4 * sim.plane, device=device)
            mv.add_solver(sim, 0)
            info["statistics"] = mv
        elif field_statistics:
            mv = MeanVariance(4 * sim.plane, device=device)
            mv.add_solver(sim, 0)
            import torch
            mean = torch.zeros(4 * sim.plane, dtype=torch.float64, device="cuda:%d" % device)
            var = torch.zeros_like(mean)
            mv.result(mean, var)
            mv.close()
            info["field_mean"] = mean.cpu().numpy().reshape(sim.shape)
            info["field_var"] = var.cpu().numpy().reshape(sim.shape)
    return params, y, info


def plain_mc(y):
    """Sample mean and biased variance (S2/M - mean^2 semantics, computed two-pass in FP64)."""
    y = np.asarray(y, dtype=np.float64)
    m = y.mean()
    return m, np.mean((y - m) ** 2)


def control_variate(y, f, f_mean, f2_mean, beta=None, beta2=None):
    """Control-variate estimates of E[Y] and Var[Y].

    ``y``: solver observables of M samples; ``f``: surrogate values at the same
    samples; ``f_mean``, ``f2_mean``: E[f] and E[f^2] under the parameter
    distribution (from many surrogate evaluations).  The coefficients are
    fitted on the samples unless given.  Returns (mean, variance, beta, beta2).
    """
    y = np.asarray(y, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    if beta is None:
        fc = f - f.mean()
        beta = float(np.dot(fc, y - y.mean()) / max(np.dot(fc, fc), 1e-300))
    mean = float(np.mean(y - beta * (f - f_mean)))
    y2 = y * y
    g = f * f
    if beta2 is None:
        gc = g - g.mean()
        beta2 = float(np.dot(gc, y2 - y2.mean()) / max(np.dot(gc, gc), 1e-300))
    second = float(np.mean(y2 - beta2 * (g - f2_mean)))
    return mean, second - mean * mean, beta, beta2

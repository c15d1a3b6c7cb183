"""The reference's time loop (Simulator::incrementSolution,
alsfvm/src/simulator/Simulator.cpp:191-214) driven with the plug-in classes
of alsvinn_b200: NumericalFlux (+ an optional DiffusionOperator) as the
system, Integrator for the stages, Boundary after every stage.  Test helper
for fixtures that store their configuration (see tests/golden/make_golden.py).
"""
import numpy as np
import torch

import alsvinn_b200 as als


def run_plugin_time_loop(z, diffusion=None, diffusion_recon="none"):
    """Runs fixture ``z`` to its end time; returns (final padded state, steps, t)."""
    dim = int(z["dim"])
    n = tuple(int(v) for v in z["n"])
    flux, recon = str(z["flux"]), str(z["recon"])
    g = als.ghost_cells(flux, recon)
    if diffusion is not None:
        g = max(g, als.diffusion_ghost_cells(diffusion_recon))
    lengths = [(float(z["upper"][d]) - float(z["lower"][d])) / n[d] for d in range(dim)]
    lengths += [0.0] * (3 - dim)
    bc = als.Boundary(dim, n, g, str(z["bc"]))
    nf = als.NumericalFlux(dim, n, flux, recon, gamma=float(z["gamma"]), ghosts=g)
    op = None
    if diffusion is not None:
        op = als.DiffusionOperator(dim, n, diffusion, diffusion_recon, gamma=float(z["gamma"]),
                                   ghosts=g)
    try:
        integ = als.Integrator(str(z["integrator"]), nf, float(z["cfl"]), diffusion=op)
        substeps = integ.getNumberOfSubsteps()
        init = torch.from_numpy(np.ascontiguousarray(z["initial"], dtype=np.float64)).cuda()
        vols = [init.clone() for _ in range(substeps + 1)]
        bc.applyBoundaryConditions(vols[0])
        t, steps, T = 0.0, 0, float(z["end_time"])
        while t < T:
            dt = 0.0
            for s in range(substeps):
                dt = integ.performSubstep(vols, lengths, dt, vols[s + 1], s, t, T)
                bc.applyBoundaryConditions(vols[s + 1])
            vols[0], vols[substeps] = vols[substeps], vols[0]
            t += dt
            steps += 1
        torch.cuda.synchronize()
        return vols[0].cpu().numpy(), steps, t
    finally:
        if op is not None:
            op.close()

"""Spatial decomposition on one GPU: the subdomains of a Cartesian
decomposition, each run by the plug-in calls, with their halos exchanged by
device copies (LocalExchange), reproduce the undivided grid bit for bit --
step count, every dt and every interior cell -- against the fused solver."""
import numpy as np
import pytest

import alsvinn_b200 as als
from alsvinn_b200 import domain
from oracle_lib import smooth_random_state

pytestmark = pytest.mark.gpu

CASES = [
    (1, (48,), (3,), "weno2", "hll3", "rungekutta3", "periodic"),
    (1, (48,), (2,), "eno3", "hll", "rungekutta2", "neumann"),
    (2, (24, 20), (2, 2), "weno2", "hll3", "rungekutta3", "periodic"),
    (2, (24, 20), (3, 1), "mc", "hll", "forwardeuler", "neumann"),
    (2, (24, 20), (1, 2), "eno2", "central", "rungekutta3", "periodic"),
    (2, (24, 20), (2, 2), "none", "tecno4", "rungekutta3", "periodic"),
    (3, (12, 10, 8), (1, 2, 2), "weno2", "hll3", "rungekutta3", "periodic"),
    (3, (12, 10, 8), (2, 1, 2), "eno2", "hll3", "rungekutta2", "neumann"),
]


@pytest.mark.parametrize("dim,n,procs,recon,flux,integ,bc", CASES,
                         ids=["d%d-%s-%s-%s-%s" % (c[0], "x".join(map(str, c[2])), c[3], c[4], c[6])
                              for c in CASES])
def test_decomposed_run_equals_the_undivided_grid(dim, n, procs, recon, flux, integ, bc):
    g = als.ghost_cells(flux, recon)
    st = smooth_random_state(800 + dim + len(recon), dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    T = 0.03
    with als.Simulator(dim, n, lo, hi, flux=flux, reconstruction=recon, integrator=integ,
                       boundary=bc, cfl=0.4, end_time=T) as sim:
        sim.set_state(st)
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    sl = tuple([slice(None)] + [slice(None)] * (3 - dim) +
               [slice(g, g + n[d]) for d in reversed(range(dim))])
    world = int(np.prod(procs))
    decs = [domain.CartesianDecomposition(dim, n, procs, r, bc) for r in range(world)]
    subs = [domain.Subdomain(dec, flux, recon, integ, 0.4, 1.4) for dec in decs]
    for s in subs:
        s.set_state(st)
    run = domain.DecomposedSimulation(subs, domain.LocalExchange(decs, g),
                                      [1.0 / n[d] for d in range(dim)], 0.4, T)
    steps, t = run.run()
    assert steps == info["steps"] and t == info["t"]
    # bit for bit, the TeCNO flux included (both runs call the same device log)
    np.testing.assert_array_equal(run.gather(U.shape), U[sl])

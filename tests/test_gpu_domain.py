"""Spatial decomposition on one GPU: the subdomains of a Cartesian
decomposition, each run by the plug-in calls, with their halos exchanged by
device copies (LocalExchange), reproduce the undivided grid bit for bit --
step count, every dt and every interior cell -- against the fused solver."""
import numpy as np
import pytest

import alsvinn_b200 as als
from alsvinn_b200 import _lib, domain
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


SPLIT_CASES = [
    (1, (48,), (3,), "weno2", "hll3", "rungekutta3", "periodic", "fp64"),
    (1, (48,), (2,), "eno3", "hll", "rungekutta2", "neumann", "fp64"),
    (2, (64, 48), (2, 2), "weno2", "hll3", "rungekutta3", "periodic", "fp64"),
    (2, (64, 48), (4, 1), "weno2", "hll3", "rungekutta3", "neumann", "fp64"),
    (2, (64, 48), (1, 3), "eno2", "hll", "rungekutta2", "periodic", "fp64"),
    (2, (64, 48), (2, 3), "none", "tecno4", "rungekutta3", "neumann", "fp64"),
    (2, (64, 48), (2, 2), "weno2", "hll3", "rungekutta3", "periodic", "fp32"),
    (3, (16, 16, 16), (2, 2, 2), "weno2", "hll3", "rungekutta3", "periodic", "fp64"),
    (3, (16, 12, 8), (1, 2, 2), "eno2", "hll3", "rungekutta2", "neumann", "fp64"),
]


@pytest.mark.parametrize("dim,n,procs,recon,flux,integ,bc,precision", SPLIT_CASES,
                         ids=["d%d-%s-%s-%s-%s-%s" % (c[0], "x".join(map(str, c[2])), c[3], c[4],
                                                      c[6], c[7]) for c in SPLIT_CASES])
@pytest.mark.parametrize("persistent", [False, True])
def test_split_fused_solver_equals_the_undivided_grid(dim, n, procs, recon, flux, integ, bc,
                                                      precision, persistent):
    """The fused solver over subdomains (one launch per stage for all of
    them, halos written into the neighbours' ghost layers by the stage
    kernels) against the undivided grid: same steps and time, every
    subdomain block -- interior, exchanged ghost layers, corners and
    physical ghosts -- equal to its slice of the undivided padded state."""
    g = als.ghost_cells(flux, recon)
    st = smooth_random_state(850 + dim + len(recon) + len(bc), dim, n, g)
    T = 0.03
    with als.Simulator(dim, n, [0.0] * dim, [1.0] * dim, flux=flux, reconstruction=recon,
                       integrator=integ, boundary=bc, cfl=0.4, end_time=T,
                       precision=precision) as sim:
        sim.set_state(st)
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    split = domain.SplitSimulation(dim, n, procs, flux=flux, reconstruction=recon,
                                   integrator=integ, boundary=bc, cfl=0.4, end_time=T,
                                   precision=precision)
    try:
        if persistent:
            split.sim.set_schedule(blocks_per_sm=2)
        split.set_state(st)
        got = split.run()
        assert got["steps"] == info["steps"] and got["t"] == info["t"] and got["status"] == 0
        for m in range(len(split.decs)):
            assert split.sim.info(m)["steps"] == info["steps"]
        blocks = split.sim.get_state()
        for r, dec in enumerate(split.decs):
            np.testing.assert_array_equal(blocks[r], U[dec.local_slice(g)])
    finally:
        split.close()


def test_split_solver_rejects_what_it_cannot_run():
    """Forward Euler, a member count that is not the number of subdomains,
    and a split of an inactive direction are refused."""
    with als.Simulator(2, (32, 32), integrator="forwardeuler", members=4) as sim:
        with pytest.raises(_lib.AlsError) as e:
            sim.decompose((2, 2))
        assert e.value.code == -4
    with als.Simulator(2, (32, 32), members=3) as sim:
        with pytest.raises(_lib.AlsError):
            sim.decompose((2, 2))
        with pytest.raises(_lib.AlsError):
            sim.decompose((1, 1, 3))


def test_split_solver_wants_its_whole_state_after_the_split():
    """A state set before the split has ghosts from the boundary condition,
    not from the neighbouring subdomains: advancing is refused until the
    whole split state is set again, and a split state is set in one call."""
    st = np.stack([smooth_random_state(5 + r, 2, (16, 16), 2) for r in range(4)])
    with als.Simulator(2, (16, 16), members=4, end_time=0.01) as sim:
        sim.set_state(st)
        sim.decompose((2, 2))
        with pytest.raises(_lib.AlsError):
            sim.advance(1)
        with pytest.raises(_lib.AlsError):
            sim.set_state(st[1:], first_member=1)
        with pytest.raises(_lib.AlsError):
            sim.set_state(st[:2])
        sim.set_state(st)
        sim.advance(1)
        assert sim.info(0)["steps"] == 1

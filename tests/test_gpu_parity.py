"""Parity of the CUDA path with the oracle, through the C ABI.

Every comparison of the FP64 path is bit-exact (assert_array_equal): the
kernels keep the reference's operation order and are compiled with
-fmad=false and IEEE division / square root.
"""
import zlib

import numpy as np
import pytest
import torch

import alsvinn_b200 as als
from alsvinn_b200 import _lib
from conftest import SIMULATION_FIXTURES, flux_cases, load_golden
from oracle_lib import digest, ghost_cells, padded_shape, smooth_random_state

pytestmark = pytest.mark.gpu


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _sim(z, **kw):
    return als.Simulator(z["dim"], tuple(z["n"]), tuple(z["lower"]), tuple(z["upper"]),
                         flux=z["flux"], reconstruction=z["recon"], integrator=z["integrator"],
                         boundary=z["bc"], gamma=z["gamma"], cfl=z["cfl"], end_time=z["end_time"],
                         **kw)


@pytest.mark.parametrize("name", SIMULATION_FIXTURES)
def test_fused_solver_reproduces_reference_fixture(name):
    z = load_golden(name)
    with _sim(z) as sim:
        sim.set_state(z["initial"])
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    assert info["steps"] == z["steps"]
    assert info["t"] == z["t"]
    assert info["dt"] == z["dts"][-1]
    np.testing.assert_array_equal(U, z["final"])


def test_sod_1024_reference_numbers():
    z = load_golden("sod1024_weno2_hll_rk3")
    with _sim(z) as sim:
        sim.set_state(als.sod(1024))
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    assert info["steps"] == 498 and info["t"] == 0.2
    assert U[0, 0, 0, 2 + 512] == 0.42568131167974621


CASES = []
for _dim, _n in ((1, (40,)), (2, (19, 21)), (3, (10, 9, 11))):
    for _recon in ("none", "weno2", "eno2", "eno3", "eno4", "mc", "mm", "wenof2", "weno3"):
        if min(_n) < 2 * ghost_cells(_recon):
            continue
        for _flux in ("hll", "hll3", "central"):
            for _integ in ("forwardeuler", "rungekutta2", "rungekutta3"):
                for _bc in ("neumann", "periodic"):
                    CASES.append((_dim, _n, _recon, _flux, _integ, _bc))


@pytest.mark.parametrize("dim,n,recon,flux,integ,bc", CASES,
                         ids=["d%d-%s-%s-%s-%s" % (c[0], c[2], c[3], c[4], c[5]) for c in CASES])
def test_fused_solver_matches_oracle(c_oracle, dim, n, recon, flux, integ, bc):
    g = ghost_cells(recon)
    seed = zlib.crc32(("%d-%s-%s-%s-%s" % (dim, recon, flux, integ, bc)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    cfg = c_oracle.config(dim, n, lo, hi, flux, recon, integ, bc, 1.4)
    rc, U_ref, dts, steps, t = c_oracle.simulate(cfg, st, 0.4, 0.04)
    assert steps >= 1
    with als.Simulator(dim, n, lo, hi, flux=flux, reconstruction=recon, integrator=integ,
                       boundary=bc, cfl=0.4, end_time=0.04) as sim:
        sim.set_state(st)
        if rc == 0:
            sim.run()
        else:
            # some combinations (central flux, high-order ENO on noise) blow up:
            # the reference stops with a constraint violation after `steps`
            with pytest.raises(_lib.AlsError) as e:
                sim.run()
            assert e.value.code == -3
        info = sim.info()
        U = sim.get_state()[0]
    assert info["steps"] == steps and info["t"] == t
    assert info["status"] == rc
    np.testing.assert_array_equal(U, U_ref)


@pytest.mark.parametrize("case", flux_cases(), ids=lambda c: "d%d_%s_%s_%s" % (
    c["dim"], c["recon"], c["flux"], c["bc"]))
def test_plugin_boundary_and_flux_match_reference(case):
    """Boundary::applyBoundaryConditions then NumericalFlux::computeFlux, compared
    with the digests of the reference's own outputs."""
    dim, n = case["dim"], case["n"]
    g = ghost_cells(case["recon"])
    st = _dev(smooth_random_state(case["seed"], dim, n, g))
    als.Boundary(dim, n, g, case["bc"]).applyBoundaryConditions(st)
    torch.cuda.synchronize()
    assert digest(st.cpu().numpy()) == case["filled"]
    out = torch.zeros_like(st)
    ws = als.NumericalFlux(dim, n, case["flux"], case["recon"]).computeFlux(st, out)
    assert digest(ws) == case["ws"]
    assert digest(out.cpu().numpy()) == case["net"]


@pytest.mark.parametrize("dim,n", [(1, (40,)), (2, (33, 18)), (3, (12, 9, 10))])
@pytest.mark.parametrize("flux,recon", [("hll3", "weno2"), ("hll", "eno3"), ("central", "none")])
def test_plugin_flux_without_wave_speeds(dim, n, flux, recon):
    """computeWaveSpeed == false (a null wave_speed in the C ABI): no wave
    speeds come back, the call only enqueues, and the net flux is the same
    bits as with them, also for a region inside the interior."""
    g = ghost_cells(recon)
    st = _dev(smooth_random_state(400 + dim, dim, n, g))
    als.Boundary(dim, n, g, "periodic").applyBoundaryConditions(st)
    nf = als.NumericalFlux(dim, n, flux, recon)
    start = (1, 1, 1)[:dim] + (0,) * (3 - dim)
    end = (-2, -1, -1)[:dim] + (0,) * (3 - dim)
    for region in (((0, 0, 0), (0, 0, 0)), (start, end)):
        ref = torch.full_like(st, 7.0)
        ws = nf.computeFlux(st, ref, *region)
        assert ws is not None and ws[0] > 0
        out = torch.full_like(st, 7.0)
        assert nf.computeFlux(st, out, *region, compute_wave_speed=False) is None
        torch.cuda.synchronize()
        assert torch.equal(out, ref)


@pytest.mark.parametrize("dim,n", [(1, (20,)), (2, (11, 12)), (3, (8, 9, 10))])
@pytest.mark.parametrize("recon", ["none", "weno2", "eno2", "eno3", "eno4", "mc", "mm", "wenof2", "weno3"])
def test_plugin_reconstruction_matches_oracle(c_oracle, dim, n, recon):
    g = ghost_cells(recon)
    if min(n) < 2 * g:
        pytest.skip("grid smaller than two ghost widths")
    st = smooth_random_state(99 + dim, dim, n, g)
    cfg = c_oracle.config(dim, n, [0] * dim, [1] * dim, "hll", recon, "rungekutta3", "neumann", 1.4)
    r = als.Reconstruction(dim, n, recon)
    x = _dev(st)
    for d in range(dim):
        lref, rref = c_oracle.reconstruct(cfg, d, st)
        left = torch.zeros_like(x)
        right = torch.zeros_like(x)
        r.performReconstruction(x, d, left, right)
        np.testing.assert_array_equal(left.cpu().numpy(), lref)
        np.testing.assert_array_equal(right.cpu().numpy(), rref)


def test_plugin_weno2_known_answer():
    """WenoTest.cpp:228-301 through the plug-in Reconstruction."""
    n, g = 10, 2
    st = np.zeros(padded_shape(1, (n,), g))
    st[0] = 1.0
    st[1] = 1.0
    st[2] = 10.0
    st[0, 0, 0, 1:4] = (2, 0, 1)
    x = _dev(st)
    left = torch.zeros_like(x)
    right = torch.zeros_like(x)
    als.Reconstruction(1, (n,), "weno2").performReconstruction(x, 0, left, right)
    eps = 1e-8
    a0, a1 = (2 / 3) / (1 + eps) ** 2, (1 / 3) / (4 + eps) ** 2
    a0t, a1t = (1 / 3) / (1 + eps) ** 2, (2 / 3) / (4 + eps) ** 2
    expect_r = a0 / (a0 + a1) * 0.5 - a1 / (a0 + a1)
    expect_l = -0.5 * a0t / (a0t + a1t) + a1t / (a0t + a1t)
    assert abs(right[0, 0, 0, 2].item() - expect_r) < 1e-8
    assert abs(left[0, 0, 0, 2].item() - expect_l) < 1e-8


@pytest.mark.parametrize("recon,value,tol", [("eno2", 0.0, 0.0), ("eno2", 1.0, 0.0),
                                             ("eno3", 0.0, 0.0), ("eno3", 1.0, 2e-6)],
                         ids=["ConstantZeroTestSecondOrder", "ConstantOneTestSecondOrder",
                              "ConstantZeroTestThirdOrder", "ConstantOneTestThirdOrder"])
def test_plugin_eno_constant_states(recon, value, tol):
    """EnoTest.cpp:47-220 through the plug-in Reconstruction: a 10 x 10
    state that is constant everywhere (0, or 1 with energy 10) reconstructs
    to itself along x on the reference's range (cells g-1 .. N-g along x,
    the interior rows), exactly for ENO2 and zero, within 2e-6 otherwise."""
    n = (10, 10)
    rec = als.Reconstruction(2, n, recon)
    g = rec.getNumberOfGhostCells()
    st = np.zeros(padded_shape(2, n, g))
    if value:
        st[:3] = value
        st[3] = 10 * value
    x = _dev(st)
    left = torch.zeros_like(x)
    right = torch.zeros_like(x)
    rec.performReconstruction(x, 0, left, right)
    N = n[0] + 2 * g
    box = (slice(None), 0, slice(g, n[1] + g), slice(g - 1, N - (g - 1)))
    expect = st[box]
    assert np.all(np.abs(left.cpu().numpy()[box] - expect) <= tol)
    assert np.all(np.abs(right.cpu().numpy()[box] - expect) <= tol)


@pytest.mark.parametrize("integ", ["forwardeuler", "rungekutta2", "rungekutta3"])
def test_plugin_time_loop_matches_oracle(c_oracle, integ):
    """Simulator::incrementSolution driven through the plug-in calls only."""
    dim, n, recon, flux, bc = 2, (14, 13), "weno2", "hll3", "periodic"
    g = ghost_cells(recon)
    st = smooth_random_state(4242, dim, n, g)
    cfg = c_oracle.config(dim, n, [0, 0], [1, 1], flux, recon, integ, bc, 1.4)
    rc, U_ref, dts, steps, t_ref = c_oracle.simulate(cfg, st, 0.4, 0.03)
    nf = als.NumericalFlux(dim, n, flux, recon)
    bnd = als.Boundary(dim, n, g, bc)
    it = als.Integrator(integ, nf, 0.4)
    vols = [_dev(st)] + [torch.zeros_like(_dev(st)) for _ in range(it.getNumberOfSubsteps())]
    bnd.applyBoundaryConditions(vols[0])
    cell = [1 / 14, 1 / 13, 1.0]
    t, k = 0.0, 0
    while t < 0.03:
        dt = 0.0
        for s in range(it.getNumberOfSubsteps()):
            dt = it.performSubstep(vols, cell, dt, vols[s + 1], s, t, 0.03)
            bnd.applyBoundaryConditions(vols[s + 1])
        vols[0], vols[-1] = vols[-1], vols[0]
        assert dt == dts[k]
        t += dt
        k += 1
    torch.cuda.synchronize()
    assert k == steps and t == t_ref
    np.testing.assert_array_equal(vols[0].cpu().numpy(), U_ref)


def test_ensemble_members_match_independent_runs(c_oracle):
    """Each member of a batched ensemble equals its own single simulation."""
    n = 32
    states, params = als.kh_ensemble(n, 0, 3)
    states[1] = smooth_random_state(7, 2, (n, n), 2)
    with als.Simulator(2, (n, n), (0, 0), (1, 1), flux="hll3", reconstruction="weno2",
                       cfl=0.4, end_time=0.05, members=3) as sim:
        sim.set_state(states)
        sim.run()
        U = sim.get_state()
        infos = [sim.info(m) for m in range(3)]
    cfg = c_oracle.config(2, (n, n), [0, 0], [1, 1], "hll3", "weno2", "rungekutta3", "periodic",
                          1.4)
    for m in range(3):
        rc, U_ref, dts, steps, t = c_oracle.simulate(cfg, states[m], 0.4, 0.05)
        assert infos[m]["steps"] == steps and infos[m]["t"] == t
        np.testing.assert_array_equal(U[m], U_ref)


def test_constraint_violation_flags_only_the_poisoned_member(c_oracle):
    """Simulator::checkConstraints: a member with negative pressure fails
    (status + first bad cell) while the others complete unaffected."""
    n = 24
    states = np.stack([smooth_random_state(300 + k, 2, (n, n), 2) for k in range(3)])
    # E below the kinetic energy in one cell -> p < 0 after the first step
    states[1, 3, 0, 10, 10] = -1.0
    with als.Simulator(2, (n, n), (0, 0), (1, 1), flux="hll", reconstruction="weno2",
                       cfl=0.4, end_time=0.02, members=3) as sim:
        sim.set_state(states)
        with pytest.raises(_lib.AlsError) as e:
            sim.run()
        assert e.value.code == -3
        infos = [sim.info(m) for m in range(3)]
        U = sim.get_state()
    assert infos[1]["status"] == 1 and infos[1]["done"]
    assert infos[1]["bad_step"] == 1 and infos[1]["bad_index"] >= 0
    cfg = c_oracle.config(2, (n, n), [0, 0], [1, 1], "hll", "weno2", "rungekutta3", "periodic", 1.4)
    for m in (0, 2):
        assert infos[m]["status"] == 0
        rc, U_ref, dts, steps, t = c_oracle.simulate(cfg, states[m], 0.4, 0.02)
        np.testing.assert_array_equal(U[m], U_ref)
    rc, _, _, steps, _ = c_oracle.simulate(cfg, states[1], 0.4, 0.02)
    assert rc == 1 and steps == infos[1]["steps"]


def test_max_steps_and_zero_end_time():
    z = load_golden("kh32_weno2_hll3_rk3")
    with _sim(z, max_steps=5) as sim:
        sim.set_state(z["initial"])
        sim.run()
        assert sim.info()["steps"] == 5
    z["end_time"] = 0.0
    with _sim(z) as sim:
        sim.set_state(z["initial"])
        sim.run()
        assert sim.info()["steps"] == 0


def test_fp32_members_stay_close_to_fp64():
    n = 64
    states, _ = als.kh_ensemble(n, 0, 2)
    out = {}
    for prec in ("fp64", "fp32"):
        with als.Simulator(2, (n, n), (0, 0), (1, 1), flux="hll3", reconstruction="weno2",
                           cfl=0.4, end_time=0.1, members=2, precision=prec) as sim:
            sim.set_state(states)
            sim.run()
            out[prec] = sim.get_state()
    g = 2
    a = out["fp64"][:, :, :, g:-g, g:-g]
    b = out["fp32"][:, :, :, g:-g, g:-g]
    # L1 error per conserved variable relative to the L1 norm of the density
    # (my starts at zero, so its own norm is no scale)
    rel = np.abs(a - b).sum(axis=(2, 3, 4)) / np.abs(a[:, :1]).sum(axis=(2, 3, 4))
    assert rel.max() < 1e-4, rel


@pytest.mark.parametrize("dim,n,steps", [(2, (1024, 1024), 6), (3, (128, 128, 128), 2)])
def test_full_size_steps_match_oracle(c_oracle, dim, n, steps):
    """The benchmark sizes themselves (KH 1024^2, KH 128^3; WENO2 + HLL3,
    RK3, periodic, FP64): a few whole time steps bit for bit, step for step."""
    g = 2
    params = als.uniform_draws(40, 3, 1)[0]
    st = als.kelvin_helmholtz(n[0], params, g, dimension=dim)
    lo, hi = [0.0] * dim, [1.0] * dim
    cfg = c_oracle.config(dim, n, lo, hi, "hll3", "weno2", "rungekutta3", "periodic", 1.4)
    rc, U_ref, dts, done, t = c_oracle.simulate(cfg, st, 0.4, 10.0, max_steps=steps)
    assert rc == 0 and done == steps
    with als.Simulator(dim, n, lo, hi, flux="hll3", reconstruction="weno2",
                       integrator="rungekutta3", boundary="periodic", cfl=0.4,
                       end_time=10.0, max_steps=steps) as sim:
        sim.set_state(st)
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    assert info["steps"] == steps and info["t"] == t and info["dt"] == dts[steps - 1]
    np.testing.assert_array_equal(U, U_ref)


def test_largest_grid_conserves_and_matches_its_halves():
    """A grid far above the benchmark (KH 4096^2 FP64, 0.5 GB per state):
    with periodic boundaries every conserved total stays at its start to
    rounding (FP64 sums over 16.8 M cells), and its left and right halves,
    run as two subdomains of a decomposition, give the same bits."""
    from alsvinn_b200 import domain
    n, g, steps = 4096, 2, 3
    st = als.kelvin_helmholtz(n, als.uniform_draws(40, 9, 1)[0], g)
    with als.Simulator(2, (n, n), (0, 0), (1, 1), flux="hll3", reconstruction="weno2",
                       integrator="rungekutta3", boundary="periodic", cfl=0.4, end_time=10.0,
                       max_steps=steps) as sim:
        sim.set_state(st)
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    assert info["steps"] == steps and info["status"] == 0
    inner = (slice(None), 0, slice(g, g + n), slice(g, g + n))
    before = st[inner].sum(axis=(1, 2))
    after = U[inner].sum(axis=(1, 2))
    # (y-momentum starts at exactly 0: its scale is the final |m_y| total)
    scale = np.maximum(np.abs(st[inner]).sum(axis=(1, 2)), np.abs(U[inner]).sum(axis=(1, 2)))
    assert np.all(np.abs(after - before) <= 1e-13 * scale), (after - before) / scale
    decs = [domain.CartesianDecomposition(2, (n, n), (2, 1), r, "periodic") for r in range(2)]
    subs = [domain.Subdomain(d, "hll3", "weno2", "rungekutta3", 0.4, 1.4) for d in decs]
    for s in subs:
        s.set_state(st)
    run = domain.DecomposedSimulation(subs, domain.LocalExchange(decs, g), [1.0 / n, 1.0 / n],
                                      0.4, 10.0)
    assert run.run(max_steps=steps) == (steps, info["t"])
    np.testing.assert_array_equal(run.gather(U.shape), U[:, :, g:g + n, g:g + n])

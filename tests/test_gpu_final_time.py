"""Final-time parity with the reference's CPU time loop (Simulator.cpp:191-214).

The plain FP64 method must match the reference on the same inputs with
identical step counts and a relative L1 difference of at most 1e-10 per
conserved variable at the final time.  The fixtures hold the reference
build's results at T = 2 (tests/golden/make_final_time.py):

* KH 1024^2, WENO2 + HLL3, RK3, CFL 0.4, periodic (about 23k steps): the
  benchmark configuration itself;
* KH 256^2 members 7 and 4095 of the 4096-sample FP64 UQ oracle ensemble;
* KH on the unit cube, 48^3 (1,475 steps), through both 3-D tile shapes;
* KH 256^2 with ENO3 + HLL + RK2, MC + HLL3 + RK3, WENO3 + HLL3 + RK3 and
  WENOF2 + HLL + RK3 (6,166 to 6,765 steps each);
* Sod across the diagonal with Neumann boundaries, 2-D 256^2 and 3-D 32^3.

Kelvin-Helmholtz at T = 2 is chaotic, so a single differing bit in any of
the steps would show at the end: the tests assert the dt sequence digest
and the sha256 of the final interior (bit equality), and the L1 bar.
"""
import numpy as np
import pytest

import alsvinn_b200 as als
import alsvinn_b200.initial_data as init
import final_time as ft

pytestmark = pytest.mark.gpu

L1_TOL = 1e-10


def _solver(z, members=1, **kw):
    n = z["n"]
    return als.Simulator(2, (n, n), (0.0, 0.0), (1.0, 1.0), flux=z["flux"],
                         reconstruction=z["recon"], integrator=z["integrator"], boundary=z["bc"],
                         gamma=z["gamma"], cfl=z["cfl"], end_time=z["end_time"], members=members,
                         **kw)


def _check_final(z, U, steps, t):
    n = z["n"]
    assert steps == z["steps"], (steps, z["steps"])
    assert t == z["t"], (t, z["t"])
    s = ft.summary(U, n, z["ghosts"])
    # relative L1 difference per conserved variable, bounded through the
    # 16 x 16 block sums (sum_b |A_b - B_b| <= sum_cells |a - b|) and the norms
    diff = np.abs(s["block_sums"] - z["block_sums"]).sum(axis=(1, 2))
    rel = diff / z["l1"]
    assert np.all(rel <= L1_TOL), rel
    assert np.all(np.abs(s["l1"] - z["l1"]) <= L1_TOL * z["l1"]), (s["l1"], z["l1"])
    # and bit equality of the whole interior
    assert s["interior_sha256"] == z["interior_sha256"]


def _step_by_step(sim):
    dts = []
    while not sim.info()["done"]:
        sim.advance(1)
        dts.append(sim.info()["dt"])
    return np.array(dts)


def test_kh1024_to_final_time_matches_reference():
    """The headline configuration to T = 2 one step at a time: every dt of
    the ~23k steps and the final state equal to the reference build's."""
    z = ft.load("kh1024")
    n = z["n"]
    U0 = ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"])
    with _solver(z) as sim:
        sim.set_state(U0)
        dts = _step_by_step(sim)
        info = sim.info()
        U = sim.get_state()[0]
    assert info["status"] == 0
    assert len(dts) == z["steps"]
    np.testing.assert_array_equal(dts[:64], z["dts_head"])
    np.testing.assert_array_equal(dts[-64:], z["dts_tail"])
    assert ft.dts_digest(dts) == z["dts_sha256"]
    _check_final(z, U, info["steps"], info["t"])


def test_uq_oracle_members_to_final_time_match_reference():
    """Members 7 and 4095 of the UQ oracle ensemble, advanced together as
    one batched FP64 ensemble (the path that generated the 4096-sample
    oracle) by the graph-captured run: final states equal to the
    reference's, and their observables equal to the ensemble fixture's."""
    zs = [ft.load(name) for name in ("uq256_7", "uq256_4095")]
    n = zs[0]["n"]
    states = np.stack([ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"]) for z in zs])
    with _solver(zs[0], members=len(zs)) as sim:
        sim.set_state(states)
        sim.run()
        infos = [sim.info(m) for m in range(len(zs))]
        U = sim.get_state()
    oracle = np.load(ft.GOLDEN + "/uq_kh256_fp64_4096.npz")
    for m, z in enumerate(zs):
        assert infos[m]["status"] == 0
        _check_final(z, U[m], infos[m]["steps"], infos[m]["t"])
        assert ft.observable(U[m], n) == z["observable"]
        assert int(oracle["steps"][z["sample"]]) == z["steps"]


def test_uq_member_dt_sequence_matches_reference():
    """Member 4095 alone, one step at a time: every dt equal to the reference's."""
    z = ft.load("uq256_4095")
    n = z["n"]
    with _solver(z) as sim:
        sim.set_state(ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"]))
        dts = _step_by_step(sim)
        info = sim.info()
        U = sim.get_state()[0]
    assert ft.dts_digest(dts) == z["dts_sha256"]
    _check_final(z, U, info["steps"], info["t"])


@pytest.mark.parametrize("name", ft.SCHEME_CASES)
def test_other_schemes_to_final_time_match_reference(name):
    """KH 256^2 to T = 2 one step at a time with the other reconstruction,
    flux and integrator combinations: every dt and the final interior
    equal to the reference build's."""
    z = ft.load(name)
    n = z["n"]
    U0 = ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"], z["ghosts"])
    with _solver(z) as sim:
        sim.set_state(U0)
        dts = _step_by_step(sim)
        info = sim.info()
        U = sim.get_state()[0]
    assert info["status"] == 0
    assert len(dts) == z["steps"]
    np.testing.assert_array_equal(dts[:64], z["dts_head"])
    np.testing.assert_array_equal(dts[-64:], z["dts_tail"])
    assert ft.dts_digest(dts) == z["dts_sha256"]
    _check_final(z, U, info["steps"], info["t"])


@pytest.mark.parametrize("name", ["uq256_7", "kh256_eno3_hll_rk2"])
def test_plugin_path_to_final_time_matches_reference(name):
    """The drop-in path itself to T = 2: the reference's time loop
    (Simulator.cpp:191-214) over the plug-in NumericalFlux, Integrator and
    Boundary calls, one host round trip per step for dt, as an alsvinn run
    with this platform selected would drive them.  Every dt and the final
    interior equal the reference build's."""
    import torch
    z = ft.load(name)
    n, g = z["n"], z["ghosts"]
    U0 = ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"], g)
    nf = als.NumericalFlux(2, (n, n), z["flux"], z["recon"], gamma=z["gamma"])
    bnd = als.Boundary(2, (n, n), nf.getNumberOfGhostCells(), z["bc"])
    it = als.Integrator(z["integrator"], nf, z["cfl"])
    first = torch.from_numpy(U0).cuda()
    vols = [first] + [torch.zeros_like(first) for _ in range(it.getNumberOfSubsteps())]
    bnd.applyBoundaryConditions(vols[0])
    cell = [1.0 / n, 1.0 / n, 1.0]
    t, dts = 0.0, []
    while t < z["end_time"]:
        dt = 0.0
        for s in range(it.getNumberOfSubsteps()):
            dt = it.performSubstep(vols, cell, dt, vols[s + 1], s, t, z["end_time"])
            bnd.applyBoundaryConditions(vols[s + 1])
        vols[0], vols[-1] = vols[-1], vols[0]
        dts.append(dt)
        t += dt
    torch.cuda.synchronize()
    dts = np.array(dts)
    assert len(dts) == z["steps"] and t == z["t"]
    assert ft.dts_digest(dts) == z["dts_sha256"]
    _check_final(z, vols[0].cpu().numpy(), len(dts), t)


@pytest.mark.parametrize("name,procs", [("uq256_7", (2, 2)), ("kh256_mc_hll3_rk3", (4, 1))])
def test_split_domain_to_final_time_matches_reference(name, procs):
    """The grid split into subdomains inside the fused solver (halos written
    into the neighbours' ghost layers by the stage kernels, the reference's
    Cartesian decomposition) to T = 2: the same step count and t, and the
    gathered interior equal to the reference build's undivided run."""
    import hashlib
    from alsvinn_b200 import domain
    z = ft.load(name)
    n, g = z["n"], z["ghosts"]
    U0 = ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"], g)
    split = domain.SplitSimulation(2, (n, n), procs, flux=z["flux"], reconstruction=z["recon"],
                                   integrator=z["integrator"], boundary=z["bc"],
                                   gamma=z["gamma"], cfl=z["cfl"], end_time=z["end_time"])
    try:
        split.set_state(U0)
        info = split.run()
        inner = np.ascontiguousarray(split.interior()[:, 0])
    finally:
        split.close()
    assert info["status"] == 0
    assert info["steps"] == z["steps"] and info["t"] == z["t"]
    assert hashlib.sha256(inner.tobytes()).hexdigest() == z["interior_sha256"]


def test_multilevel_batch_to_final_time_matches_reference():
    """One batched solver over two grid levels (UQ members 7 and 4095 at
    256^2, the headline KH at 1024^2), one launch per stage over all of
    them, run to T = 2: every member takes its own reference step count and
    ends on the reference build's exact bits."""
    import hashlib
    names = [["uq256_7", "uq256_4095"], ["kh1024"]]
    zs = [[ft.load(nm) for nm in level] for level in names]
    levels = [{"n": (z[0]["n"], z[0]["n"]), "members": len(z)} for z in zs]
    z0 = zs[0][0]
    with als.Simulator(2, levels=levels, flux=z0["flux"], reconstruction=z0["recon"],
                       integrator=z0["integrator"], boundary=z0["bc"], gamma=z0["gamma"],
                       cfl=z0["cfl"], end_time=z0["end_time"]) as sim:
        for k, lev in enumerate(sim.levels):
            sim.set_state(np.stack([ft.kh_state_from_bands(z["n"], z["band_lo"], z["band_hi"])
                                    for z in zs[k]]), first_member=lev["first"])
        sim.run()
        for k, lev in enumerate(sim.levels):
            out = sim.get_state(lev["first"])
            for m, z in enumerate(zs[k]):
                info = sim.info(lev["first"] + m)
                assert info["status"] == 0
                assert info["steps"] == z["steps"] and info["t"] == z["t"]
                inner = ft.interior(out[m], z["n"])
                assert hashlib.sha256(inner.tobytes()).hexdigest() == z["interior_sha256"]


@pytest.mark.parametrize("name", ft.RIEMANN_CASES)
def test_neumann_riemann_to_final_time_matches_reference(name):
    """Sod across the diagonal with Neumann boundaries (2-D 256^2 to
    T = 0.25, 3-D 32^3 to T = 0.2), one step at a time: every dt and the
    final interior equal to the reference build's."""
    z = ft.load(name)
    dim, n, g = int(z["dim"]), z["n"], z["ghosts"]
    U0 = ft.riemann_state(dim, n, g)
    assert ft.state_digest(U0) == z["initial_sha256"]
    with als.Simulator(dim, (n,) * dim, (0.0,) * dim, (1.0,) * dim, flux=z["flux"],
                       reconstruction=z["recon"], integrator=z["integrator"], boundary=z["bc"],
                       gamma=z["gamma"], cfl=z["cfl"], end_time=z["end_time"]) as sim:
        sim.set_state(U0)
        dts = _step_by_step(sim)
        info = sim.info()
        U = sim.get_state()[0]
    assert info["status"] == 0
    assert info["steps"] == z["steps"] and info["t"] == z["t"]
    np.testing.assert_array_equal(dts[:64], z["dts_head"])
    np.testing.assert_array_equal(dts[-64:], z["dts_tail"])
    assert ft.dts_digest(dts) == z["dts_sha256"]
    s = ft.summary(U, n, g) if dim == 2 else ft.summary3(U, n, g)
    axes = tuple(range(1, s["block_sums"].ndim))
    diff = np.abs(s["block_sums"] - z["block_sums"]).sum(axis=axes)
    assert np.all(diff <= L1_TOL * z["l1"]), (diff, z["l1"])
    assert s["interior_sha256"] == z["interior_sha256"]


@pytest.mark.parametrize("shape", [1, 0], ids=["z-marching columns", "8x8x4 boxes"])
def test_kh3d_to_final_time_matches_reference(shape):
    """3-D KH 48^3 to T = 2 one step at a time with each 3-D tile shape:
    every dt and the final interior equal to the reference build's (48
    cells along z are two z-marching segments, 32 + 16)."""
    z = ft.load("kh3d48")
    n = z["n"]
    U0 = init.kelvin_helmholtz(n, z["params"], ft.GHOSTS, ft.GAMMA, dimension=3)
    assert ft.state_digest(U0) == z["initial_sha256"]
    with als.Simulator(3, (n, n, n), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), flux=z["flux"],
                       reconstruction=z["recon"], integrator=z["integrator"], boundary=z["bc"],
                       gamma=z["gamma"], cfl=z["cfl"], end_time=z["end_time"]) as sim:
        sim.set_tiles([shape])
        assert sim.tiles()["shapes"] == [shape]
        sim.set_state(U0)
        dts = _step_by_step(sim)
        info = sim.info()
        U = sim.get_state()[0]
    assert info["status"] == 0
    assert info["steps"] == z["steps"] and info["t"] == z["t"]
    np.testing.assert_array_equal(dts[:64], z["dts_head"])
    np.testing.assert_array_equal(dts[-64:], z["dts_tail"])
    assert ft.dts_digest(dts) == z["dts_sha256"]
    s = ft.summary3(U, n)
    # (the z momentum stays zero: its L1 norm is 0 in both, so its block
    # differences must be 0)
    diff = np.abs(s["block_sums"] - z["block_sums"]).sum(axis=(1, 2, 3))
    assert np.all(diff <= L1_TOL * z["l1"]), (diff, z["l1"])
    assert s["interior_sha256"] == z["interior_sha256"]

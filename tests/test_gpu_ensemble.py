"""Ensembles on the GPU: multilevel batches in one launch per stage, the
schedule autotuner, FP64 statistics and conservation sums.

Every member of a batched or multilevel run must equal its own single
simulation bit for bit (the reference runs samples one after another,
alsuq/src/run/Runner.cpp:42-78)."""
import numpy as np
import pytest
import torch

import alsvinn_b200 as als
from alsvinn_b200 import _lib
from conftest import load_golden
from oracle_lib import ghost_cells, padded_shape, smooth_random_state

pytestmark = pytest.mark.gpu

LEVELS = [{"n": (24, 24), "members": 3}, {"n": (40, 36), "members": 2},
          {"n": (16, 20), "members": 2}]


def _level_states(levels, g, seed0):
    states = []
    for k, lev in enumerate(levels):
        states.append(np.stack([smooth_random_state(seed0 + 10 * k + m, 2, lev["n"], g)
                                for m in range(lev["members"])]))
    return states


def _run_levels(levels, states, order=None, tune=False, shapes=None, **kw):
    with als.Simulator(2, levels=levels, flux="hll3", reconstruction="weno2", cfl=0.4,
                       end_time=0.03, **kw) as sim:
        if shapes is not None:
            sim.set_tiles(shapes)
            assert sim.tiles()["shapes"] == list(shapes)
        for k, lev in enumerate(sim.levels):
            sim.set_state(states[k], first_member=lev["first"])
        if tune:
            before = [sim.get_state(lev["first"]) for lev in sim.levels]
            choice = sim.tune(steps=2)
            after = [sim.get_state(lev["first"]) for lev in sim.levels]
            for a, b in zip(before, after):
                np.testing.assert_array_equal(a, b)
            assert all(sim.info(m)["steps"] == 0 for m in range(sim.members))
            assert sim.schedule()["blocks_per_sm"] == choice["blocks_per_sm"]
            assert sim.tiles()["shapes"] == choice["tile_shapes"]
        if order is not None:
            sim.set_schedule(0, order)
        sim.run()
        out = [sim.get_state(lev["first"]) for lev in sim.levels]
        infos = [sim.info(m) for m in range(sim.members)]
    return out, infos


@pytest.mark.parametrize("integ", ["rungekutta3", "rungekutta2", "forwardeuler"])
def test_multilevel_members_equal_single_runs(c_oracle, integ):
    g = ghost_cells("weno2")
    states = _level_states(LEVELS, g, 500)
    out, infos = _run_levels(LEVELS, states, integrator=integ)
    m = 0
    for k, lev in enumerate(LEVELS):
        n = lev["n"]
        cfg = c_oracle.config(2, n, (0, 0), (1, 1), "hll3", "weno2", integ, "periodic", 1.4)
        for j in range(lev["members"]):
            rc, U, dts, steps, t = c_oracle.simulate(cfg, states[k][j], 0.4, 0.03)
            assert rc == 0
            assert infos[m]["steps"] == steps and infos[m]["t"] == t
            np.testing.assert_array_equal(out[k][j], U)
            m += 1


def test_level_order_and_tuning_do_not_change_results():
    g = ghost_cells("weno2")
    states = _level_states(LEVELS, g, 700)
    base, base_info = _run_levels(LEVELS, states)
    for order in ([2, 0, 1], [1, 2, 0]):
        out, info = _run_levels(LEVELS, states, order=order)
        for a, b in zip(base, out):
            np.testing.assert_array_equal(a, b)
        assert [i["steps"] for i in info] == [i["steps"] for i in base_info]
    out, info = _run_levels(LEVELS, states, tune=True)
    for a, b in zip(base, out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("integ", ["rungekutta3", "rungekutta2", "forwardeuler"])
def test_tile_shape_per_level_does_not_change_results(precision, integ):
    """Levels on the 16x16 tile, the 32x16 tile or a mix (one launch per
    shape and stage), and persistent launches over them, give the same bits."""
    g = ghost_cells("weno2")
    states = _level_states(LEVELS, g, 800)
    base, base_info = _run_levels(LEVELS, states, precision=precision, integrator=integ)
    for shapes in ([1, 1, 1], [0, 1, 0], [1, 0, 1]):
        out, info = _run_levels(LEVELS, states, shapes=shapes, precision=precision,
                                integrator=integ)
        for a, b in zip(base, out):
            np.testing.assert_array_equal(a, b)
        assert [i["steps"] for i in info] == [i["steps"] for i in base_info]


def test_tile_shapes_report_extents_and_reject_unbuilt():
    with als.Simulator(2, levels=LEVELS, flux="hll3", reconstruction="weno2", cfl=0.4,
                       end_time=0.03) as sim:
        t = sim.tiles()
        assert t["shapes"] == [0, 0, 0] and t["extents"][0] == (32, 16, 1)
        sim.set_tiles([1, 0, 1])
        assert sim.tiles()["extents"] == [(16, 16, 1), (32, 16, 1), (16, 16, 1)]
    with als.Simulator(2, levels=LEVELS, flux="hll3", reconstruction="eno3", cfl=0.4,
                       end_time=0.03) as sim:
        with pytest.raises(_lib.AlsError):
            sim.set_tiles([1, 0, 0])
    with als.Simulator(3, (8, 8, 8), (0, 0, 0), (1, 1, 1), flux="hll3",
                       reconstruction="eno3") as sim:
        with pytest.raises(_lib.AlsError):
            sim.set_tiles([1])
    with als.Simulator(3, (8, 8, 8), (0, 0, 0), (1, 1, 1), flux="hll3",
                       reconstruction="weno2") as sim:
        sim.set_tiles([1])
        assert sim.tiles()["extents"] == [(16, 16, 32)]


def test_fp32_multilevel_against_fp64():
    g = ghost_cells("weno2")
    states = _level_states(LEVELS, g, 900)
    a, _ = _run_levels(LEVELS, states)
    b, _ = _run_levels(LEVELS, states, precision="fp32")
    # noisy initial data through WENO weights: FP32 rounding grows to ~1e-4
    for x, y in zip(a, b):
        err = np.abs(x - y).max()
        assert err < 1e-3, err


def test_meanvariance_matches_reference_and_welford():
    z = load_golden("meanvar_7")
    states = np.stack([smooth_random_state(int(s), 2, (6, 5), 2) for s in z["seeds"]])
    x = torch.from_numpy(states).cuda()
    mv = als.MeanVariance(states[0].size)
    mv.add(x[:4])
    mv.add(x[4:])
    mean = torch.zeros(states[0].size, dtype=torch.float64, device="cuda")
    var = torch.zeros_like(mean)
    mv.result(mean, var)
    mean = mean.cpu().numpy().reshape(states.shape[1:])
    var = var.cpu().numpy().reshape(states.shape[1:])
    # the reference's raw moments (S2/M - mean^2) and Welford agree to rounding
    np.testing.assert_allclose(mean, z["mean"], rtol=1e-14, atol=0)
    np.testing.assert_allclose(var, z["var"], rtol=1e-9, atol=1e-14)
    # and Welford matches a two-pass FP64 variance much more tightly
    np.testing.assert_allclose(var, states.var(axis=0), rtol=1e-12, atol=1e-16)


def test_meanvariance_fp32_members_and_merge():
    rng = np.random.default_rng(5)
    data = rng.normal(3.0, 0.01, size=(150, 1000)).astype(np.float32)
    x = torch.from_numpy(data).cuda()
    a = als.MeanVariance(1000)
    a.add(x[:90], precision="fp32")
    b = als.MeanVariance(1000)
    b.add(x[90:], precision="fp32")
    n, mean_b, m2_b = b.moments()
    mb = torch.zeros(1000, dtype=torch.float64, device="cuda")
    vb = torch.zeros_like(mb)
    b.result(mb, vb)
    # merge b's (n, mean, M2) into a
    m2t = torch.zeros_like(mb)
    torch.cuda.synchronize()
    m2t.copy_(vb * n)
    a.merge(n, mb, m2t)
    mean = torch.zeros_like(mb)
    var = torch.zeros_like(mb)
    a.result(mean, var)
    d = data.astype(np.float64)
    np.testing.assert_allclose(mean.cpu().numpy(), d.mean(axis=0), rtol=1e-14)
    np.testing.assert_allclose(var.cpu().numpy(), d.var(axis=0), rtol=1e-10)


def test_region_sums_and_conservation():
    n = 48
    states, _ = als.kh_ensemble(n, 0, 2)
    g = 2
    with als.Simulator(2, (n, n), flux="hll3", reconstruction="weno2", cfl=0.4, end_time=0.05,
                       members=2) as sim:
        sim.set_state(states)
        s0 = sim.region_sums()
        np.testing.assert_allclose(s0, states[:, :, 0, g:-g, g:-g].sum(axis=(2, 3)), rtol=1e-14)
        sim.run()
        s1 = sim.region_sums()
        U = sim.get_state()
        box = sim.region_sums(lo=(12, 12), hi=(36, 36))
    # periodic: mass, momentum and energy are conserved to rounding
    np.testing.assert_allclose(s1, s0, rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(box, U[:, :, 0, g + 12:g + 36, g + 12:g + 36].sum(axis=(2, 3)),
                               rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("sample", [7, 4095])
def test_uq_oracle_members_equal_single_runs_at_full_size(sample):
    """Members of the 4096-sample FP64 ensemble (256^2 to T = 2, committed
    observables) re-solved alone: identical observable and step count."""
    z = load_golden("uq_kh256_fp64_4096")
    params, y, info = als.uq.kh_observable_ensemble(256, sample, 1, precision="fp64",
                                                    end_time=2.0)
    assert info["steps"][0] == z["steps"][sample]
    assert y[0] == z["y"][sample]


Z_CASES = [((20, 18, 40), "weno2", "hll3", "rungekutta3", "periodic", 2),
           ((17, 16, 33), "eno2", "hll", "rungekutta2", "neumann", 1),
           ((16, 21, 18), "mc", "central", "forwardeuler", "periodic", 3),
           ((18, 17, 35), "wenof2", "hll3", "rungekutta3", "neumann", 1),
           ((16, 16, 16), "none", "hll", "rungekutta3", "periodic", 2),
           ((19, 16, 20), "mm", "hll3", "rungekutta2", "periodic", 1)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("n,recon,flux,integ,bc,members", Z_CASES,
                         ids=["%s-%s-%s-%s" % (c[1], c[2], c[3], c[4]) for c in Z_CASES])
def test_z_marching_3d_tiles_equal_the_box_tiles(n, recon, flux, integ, bc, members, precision):
    """3-D shape 1 (16x16 columns marching along z in segments) gives the
    bits of shape 0 (8x8x4 boxes): every member, ghosts included, with
    partial columns and segments, both boundaries, every integrator."""
    g = ghost_cells(recon)
    states = np.stack([smooth_random_state(300 + k, 3, n, g) for k in range(members)])
    out = {}
    for shape in (0, 1):
        with als.Simulator(3, n, (0, 0, 0), (1, 1, 1), flux=flux, reconstruction=recon,
                           integrator=integ, boundary=bc, cfl=0.4, end_time=0.02,
                           precision=precision, members=members) as sim:
            sim.set_tiles([shape])
            sim.set_state(states)
            sim.run()
            out[shape] = (sim.get_state(), [sim.info(m) for m in range(members)])
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert [(i["steps"], i["t"], i["dt"]) for i in out[0][1]] == \
        [(i["steps"], i["t"], i["dt"]) for i in out[1][1]]
    assert out[0][1][0]["steps"] >= 2


def test_z_marching_3d_against_the_oracle(c_oracle):
    """Shape 1 on KH-like 3-D data against the C oracle directly (WENO2 +
    HLL3, RK3, periodic), a grid of two z segments plus a partial one."""
    n, g = (17, 16, 70), 2
    st = smooth_random_state(41, 3, n, g)
    cfg = c_oracle.config(3, n, (0, 0, 0), (1, 1, 1), "hll3", "weno2", "rungekutta3", "periodic",
                          1.4)
    rc, U_ref, dts, steps, t = c_oracle.simulate(cfg, st, 0.4, 10.0, max_steps=3)
    with als.Simulator(3, n, (0, 0, 0), (1, 1, 1), flux="hll3", reconstruction="weno2",
                       integrator="rungekutta3", boundary="periodic", cfl=0.4, end_time=10.0,
                       max_steps=3) as sim:
        sim.set_tiles([1])
        assert sim.tiles()["extents"][0][:2] == (16, 16)
        sim.set_state(st)
        sim.run()
        info = sim.info()
        U = sim.get_state()[0]
    assert rc == 0 and info["steps"] == steps == 3 and info["t"] == t
    np.testing.assert_array_equal(U, U_ref)

"""The oracle itself: pinned against the reference's own CPU code.

CPU only.  The C restatement (oracle/als_oracle.c) must reproduce, bit for
bit, every golden fixture produced by the reference's unmodified CPU
sources (tests/golden/make_golden.py), and, where the reference build is
present, fresh random cases.  The reference's own unit tests that pin this
path (test/library_tests/src/fvm/...) are ported here against the oracle.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, SIMULATION_FIXTURES, flux_cases, load_golden
from oracle_lib import digest, ghost_cells, padded_shape, smooth_random_state


@pytest.mark.parametrize("name", SIMULATION_FIXTURES)
def test_c_oracle_reproduces_reference_simulation(c_oracle, name):
    z = load_golden(name)
    dim = z["dim"]
    cfg = c_oracle.config(dim, z["n"], z["lower"], z["upper"], z["flux"], z["recon"],
                          z["integrator"], z["bc"], z["gamma"])
    rc, U, dts, steps, t = c_oracle.simulate(cfg, z["initial"], z["cfl"], z["end_time"])
    assert rc == 0
    assert steps == z["steps"]
    assert t == z["t"]
    np.testing.assert_array_equal(dts, z["dts"])
    np.testing.assert_array_equal(U, z["final"])


def test_sod_reference_numbers():
    """Sod 1024, WENO2+HLL, RK3, CFL 0.45, T=0.2: 498 steps ending at T exactly."""
    z = load_golden("sod1024_weno2_hll_rk3")
    assert z["steps"] == 498
    assert z["t"] == 0.2
    g = 2
    assert z["final"][0, 0, 0, g + 512] == 0.42568131167974621


@pytest.mark.parametrize("case", flux_cases(), ids=lambda c: "d%d_%s_%s_%s" % (
    c["dim"], c["recon"], c["flux"], c["bc"]))
def test_c_oracle_net_flux_matches_reference(c_oracle, case):
    dim, n = case["dim"], case["n"]
    g = ghost_cells(case["recon"])
    st = smooth_random_state(case["seed"], dim, n, g)
    cfg = c_oracle.config(dim, n, [0] * dim, [1] * dim, case["flux"], case["recon"],
                          "rungekutta3", case["bc"], 1.4)
    filled = c_oracle.fill_ghosts(cfg, st)
    assert digest(filled) == case["filled"]
    net, ws = c_oracle.net_flux(cfg, filled)
    assert digest(ws) == case["ws"]
    assert digest(net) == case["net"]


def test_c_oracle_meanvar_matches_reference(c_oracle):
    z = load_golden("meanvar_7")
    states = np.stack([smooth_random_state(int(s), 2, (6, 5), 2) for s in z["seeds"]])
    mean, var = c_oracle.meanvar(states)
    np.testing.assert_array_equal(mean, z["mean"])
    np.testing.assert_array_equal(var, z["var"])


@pytest.mark.parametrize("dim,n", [(1, (24,)), (2, (10, 11)), (3, (8, 9, 8))])
@pytest.mark.parametrize("recon", ["none", "weno2", "eno2", "eno3", "eno4", "mc", "mm", "wenof2", "weno3"])
def test_c_oracle_matches_reference_build(c_oracle, ref_oracle, dim, n, recon):
    """Fresh random cases against the reference build (skipped without it)."""
    g = ghost_cells(recon)
    if min(n) < 2 * g:
        pytest.skip("grid smaller than two ghost widths")
    seed = 5000 + 17 * dim + 3 * ["none", "weno2", "eno2", "eno3", "eno4", "mc", "mm",
                                  "wenof2", "weno3"].index(recon)
    for flux in ("hll", "hll3", "central"):
        for bc in ("neumann", "periodic"):
            st = smooth_random_state(seed, dim, n, g)
            lo, hi = [0.0] * dim, [1.0] * dim
            for integ in ("forwardeuler", "rungekutta2", "rungekutta3", "rungekutta4"):
                cfg = c_oracle.config(dim, n, lo, hi, flux, recon, integ, bc, 1.4)
                r = ref_oracle.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, 0.4, 0.03, st)
                c = c_oracle.simulate(cfg, st, 0.4, 0.03)
                assert r[0] == c[0] and r[3] == c[3] and r[4] == c[4]
                np.testing.assert_array_equal(r[1], c[1])
                np.testing.assert_array_equal(r[2], c[2])
            for d in range(dim):
                lr = ref_oracle.reconstruct(dim, n, recon, 1.4, d, st)
                cfg = c_oracle.config(dim, n, lo, hi, flux, recon, "rungekutta3", bc, 1.4)
                lc = c_oracle.reconstruct(cfg, d, st)
                np.testing.assert_array_equal(lr[0], lc[0])
                np.testing.assert_array_equal(lr[1], lc[1])


# --------------------------------------------------------------------------
# ports of the reference's unit tests for this path, against the oracle


def test_weno2_known_answer(c_oracle):
    """WenoTest.cpp:228-301: rho = (.., 2, 0, 1, ..) gives closed-form weights."""
    n = 10
    g = 2
    st = np.zeros(padded_shape(1, (n,), g))
    st[0] = 1.0
    st[1] = 1.0
    st[2] = 10.0
    st[0, 0, 0, 1] = 2
    st[0, 0, 0, 2] = 0
    st[0, 0, 0, 3] = 1
    cfg = c_oracle.config(1, (n,), (0,), (1,), "hll", "weno2", "rungekutta3", "neumann", 1.4)
    left, right = c_oracle.reconstruct(cfg, 0, st)
    eps = 1e-8
    d0, d1 = 2.0 / 3.0, 1.0 / 3.0
    b0, b1 = 1.0, 4.0
    a0, a1 = d0 / (b0 + eps) ** 2, d1 / (b1 + eps) ** 2
    a0t, a1t = d1 / (b0 + eps) ** 2, d0 / (b1 + eps) ** 2
    w0, w1 = a0 / (a0 + a1), a1 / (a0 + a1)
    w0t, w1t = a0t / (a0t + a1t), a1t / (a0t + a1t)
    assert abs((w0 * 0.5 + w1 * -1) - right[0, 0, 0, 2]) < 1e-8
    assert abs((w0t * -0.5 + w1t * 1) - left[0, 0, 0, 2]) < 1e-8


@pytest.mark.parametrize("recon", ["none", "weno2", "eno2", "eno3", "eno4"])
def test_reconstruction_of_constants_is_exact(c_oracle, recon):
    """WenoTest.cpp:32-227: zero reconstructs exactly, one within 1e-8."""
    g = ghost_cells(recon)
    for value, tol in ((0.0, 0.0), (1.0, 1e-8)):
        st = np.full(padded_shape(2, (10, 10), g), value)
        cfg = c_oracle.config(2, (10, 10), (0, 0), (1, 1), "hll", recon, "rungekutta3",
                              "neumann", 1.4)
        for d in range(2):
            left, right = c_oracle.reconstruct(cfg, d, st)
            sl = (slice(None), slice(None), slice(g, -g), slice(g, -g))
            assert np.all(np.abs(left[sl] - value) <= tol)
            assert np.all(np.abs(right[sl] - value) <= tol)


@pytest.mark.parametrize("flux", ["hll", "hll3", "central"])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_constant_state_has_zero_net_flux(c_oracle, flux, dim):
    """numericalfluxtest.cpp:65-126: a constant state with Neumann gives net flux 0."""
    n = (10,) * dim
    g = 2
    st = np.zeros(padded_shape(dim, n, g))
    st[0] = 1.0
    st[1] = 0.3
    st[-1] = 3.0
    cfg = c_oracle.config(dim, n, [0] * dim, [1] * dim, flux, "weno2", "rungekutta3", "neumann",
                          1.4)
    net, ws = c_oracle.net_flux(cfg, st)
    assert np.all(net == 0.0)
    assert ws[0] > 0


def test_boundary_fills(c_oracle):
    """BoundaryTest.cpp:52-334: Neumann mirrors, periodic wraps (2 ghost cells)."""
    n = 6
    g = 2
    st = np.zeros(padded_shape(2, (n, n), g))
    inner = np.arange(n * n, dtype=float).reshape(n, n) + 1
    st[:, 0, g:-g, g:-g] = inner
    cfgN = c_oracle.config(2, (n, n), (0, 0), (1, 1), "hll", "weno2", "rungekutta3", "neumann", 1.4)
    cfgP = c_oracle.config(2, (n, n), (0, 0), (1, 1), "hll", "weno2", "rungekutta3", "periodic", 1.4)
    N = c_oracle.fill_ghosts(cfgN, st)[0, 0]
    P = c_oracle.fill_ghosts(cfgP, st)[0, 0]
    for k in range(1, g + 1):
        np.testing.assert_array_equal(N[g:-g, g - k], N[g:-g, g + k - 1])
        np.testing.assert_array_equal(N[g:-g, -g - 1 + k], N[g:-g, -g - k])
        np.testing.assert_array_equal(P[g:-g, g - k], P[g:-g, g - k + n])
        np.testing.assert_array_equal(P[g - k, :], P[g - k + n, :])


def _structure_cases():
    rows = []
    with open(os.path.join(GOLDEN, "structure_cube_cases.txt")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            dim, n, bc, H, p, seed, dg, mx = line.split()
            rows.append((int(dim), tuple(int(v) for v in n.split(",")), bc, int(H), float(p),
                         int(seed), dg, float(mx)))
    return rows


@pytest.mark.parametrize("case", _structure_cases(), ids=lambda c: "d%d_%s_H%d_p%g" % (
    c[0], c[2], c[3], c[4]))
def test_c_oracle_structure_cube_matches_reference(c_oracle, case):
    """structure_common.hpp:39-160 through the reference's own code: bit for bit."""
    dim, n, bc, H, p, seed, dg, mx = case
    st = smooth_random_state(seed, dim, n, 2)
    out = c_oracle.structure_cube(dim, n, 2, bc, H, p, st)
    assert digest(out) == dg
    assert out.max() == mx


@pytest.mark.parametrize("bc", ["periodic", "neumann"])
def test_c_oracle_structure_functions_against_reference_build(c_oracle, ref_oracle, bc):
    for dim, n in ((2, (9, 11)), (3, (5, 6, 4))):
        st = smooth_random_state(4242 + dim, dim, n, 3)
        for H, p in ((7, 2.0), (3, 1.5)):
            np.testing.assert_array_equal(c_oracle.structure_cube(dim, n, 3, bc, H, p, st),
                                          ref_oracle.structure_cube(dim, n, 3, bc, H, p, st))


def test_structure_basic_small_case_by_hand(c_oracle):
    """StructureBasic.cpp:74-118 on a 1-D ramp: |u_i - u_{i+h}| = h*step away from the edge."""
    n = 8
    st = np.zeros(padded_shape(1, (n,), 2))
    st[:, 0, 0, 2:-2] = np.arange(n, dtype=float)
    out = c_oracle.structure_basic(1, (n,), 2, "neumann", 0, 4, 1.0, st)
    # Neumann clamps: sum_i |i - min(i+h, n-1)| / n
    for h in range(4):
        expect = sum(abs(i - min(i + h, n - 1)) for i in range(n)) / n
        assert out[0, h] == pytest.approx(expect, rel=1e-15)
    per = c_oracle.structure_basic(1, (n,), 2, "periodic", 0, 4, 2.0, st)
    for h in range(4):
        expect = sum((i - (i + h) % n) ** 2 for i in range(n)) / n
        assert per[0, h] == pytest.approx(expect, rel=1e-15)


def test_reference_driver_with_adapter_loads_and_matches_on_cpu(ref_oracle):
    """oracle/_ref/libalsref_b200.so (the reference time loop that can take the
    B200 flux adapter) gives the plain reference's results with its CPU flux."""
    from oracle_lib import RefB200Oracle, ref_b200_library_path
    if not os.path.exists(ref_b200_library_path()):
        pytest.skip("libalsref_b200.so not built")
    rb = RefB200Oracle()
    rb.set_flux_platform("cpu")
    st = smooth_random_state(8, 2, (10, 12), 2)
    a = ref_oracle.simulate(2, (10, 12), (0, 0), (1, 1), "hll3", "weno2", "rungekutta3",
                            "periodic", 1.4, 0.4, 0.02, st)
    b = rb.simulate(2, (10, 12), (0, 0), (1, 1), "hll3", "weno2", "rungekutta3", "periodic",
                    1.4, 0.4, 0.02, st)
    assert a[0] == b[0] and a[3] == b[3] and a[4] == b[4]
    np.testing.assert_array_equal(a[1], b[1])
    with pytest.raises(RuntimeError):
        rb.set_flux_platform("tpu")


@pytest.mark.parametrize("dim,n", [(1, (24,)), (2, (12, 11)), (3, (10, 11, 10))])
@pytest.mark.parametrize("flux", ["tecno1", "tecno4", "tecno6"])
def test_c_oracle_tecno_matches_reference_build(c_oracle, ref_oracle, dim, n, flux):
    """The TeCNO fluxes (reconstruction none) against the reference build:
    simulations with every integrator and boundary, and one net flux with its
    wave speeds, bit for bit (both sides call the C library's log).  In 3-D
    this includes the reference's z-direction flux, which stays 0 between
    unequal states (Tecno1.hpp writes the 2-D formulas only)."""
    g = ghost_cells("none", flux)
    if min(n) < 2 * g:
        pytest.skip("grid smaller than two ghost widths")
    seed = 5400 + 17 * dim + 3 * ["tecno1", "tecno4", "tecno6"].index(flux)
    lo, hi = [0.0] * dim, [1.0] * dim
    for bc in ("neumann", "periodic"):
        st = smooth_random_state(seed, dim, n, g)
        for integ in ("forwardeuler", "rungekutta2", "rungekutta3"):
            cfg = c_oracle.config(dim, n, lo, hi, flux, "none", integ, bc, 1.4)
            r = ref_oracle.simulate(dim, n, lo, hi, flux, "none", integ, bc, 1.4, 0.4, 0.03, st)
            c = c_oracle.simulate(cfg, st, 0.4, 0.03)
            assert r[0] == c[0] and r[3] == c[3] and r[4] == c[4]
            np.testing.assert_array_equal(r[1], c[1])
            np.testing.assert_array_equal(r[2], c[2])
        cfg = c_oracle.config(dim, n, lo, hi, flux, "none", "rungekutta3", bc, 1.4)
        filled, rf, rws = ref_oracle.compute_flux(dim, n, lo, hi, flux, "none", bc, 1.4, st)
        np.testing.assert_array_equal(filled, c_oracle.fill_ghosts(cfg, st))
        cf, cws = c_oracle.net_flux(cfg, filled)
        np.testing.assert_array_equal(rws, cws)
        np.testing.assert_array_equal(rf, cf)


TECNO_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                        if f.startswith("tecno_") and f.endswith(".npz"))


@pytest.mark.parametrize("name", TECNO_FIXTURES)
def test_c_oracle_reproduces_reference_tecno_simulation(c_oracle, name):
    """TeCNO fixtures made by the reference build, reproduced bit for bit
    (the oracle calls the same C library log as the reference)."""
    z = load_golden(name)
    dim = int(z["dim"])
    cfg = c_oracle.config(dim, z["n"], z["lower"], z["upper"], str(z["flux"]), str(z["recon"]),
                          str(z["integrator"]), str(z["bc"]), float(z["gamma"]))
    rc, U, dts, steps, t = c_oracle.simulate(cfg, z["initial"], float(z["cfl"]),
                                             float(z["end_time"]))
    assert rc == 0 and steps == z["steps"] and t == z["t"]
    np.testing.assert_array_equal(dts, z["dts"])
    np.testing.assert_array_equal(U, z["final"])


@pytest.mark.parametrize("dim,n", [(1, (64,)), (2, (32, 30))])
def test_tecno_entropy_production(c_oracle, dim, n):
    """tecno1 and tecno4 are entropy conservative (the periodic entropy
    production sum_i v(u_i) . L_i vanishes to rounding); tecno6 is not, since
    the reference's six-point stencil reads u_i where u_{i+3} belongs; HLL3
    dissipates entropy."""
    gamma = 1.4

    def production(flux):
        g = ghost_cells("none", flux)
        st = smooth_random_state(3, dim, n, g)
        cfg = c_oracle.config(dim, n, [0.0] * dim, [1.0] * dim, flux, "none", "rungekutta3",
                              "periodic", gamma)
        f = c_oracle.fill_ghosts(cfg, st)
        net, _ = c_oracle.net_flux(cfg, f)
        sl = (slice(None), slice(None), slice(g, g + n[1]) if dim > 1 else slice(None),
              slice(g, g + n[0]))
        U, L = f[sl], net[sl]
        rho, m, E = U[0], U[1:1 + dim], U[1 + dim]
        mm = sum(m[k] * m[k] for k in range(dim))
        p = (gamma - 1) * (E - 0.5 * mm / rho)
        s = np.log(p) - gamma * np.log(rho)
        v = np.stack([(gamma - s) / (gamma - 1) - mm / (rho * 2 * p)]
                     + [m[k] / p for k in range(dim)] + [-rho / p])
        return (v * L).sum() / np.abs(v * L).sum()

    assert abs(production("tecno1")) < 1e-14
    assert abs(production("tecno4")) < 1e-14
    assert abs(production("tecno6")) > 1e-7
    assert production("hll3") < -1e-3


# --------------------------------------------------------------------------
# TeCNO diffusion (TecnoDiffusionCPU with the tecno reconstructions)

DIFFUSION_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                            if f.startswith("tecnodiff_") and f.endswith(".npz"))
DIFFUSION_APPLY_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                                  if f.startswith("diffusion_apply_") and f.endswith(".npz"))


@pytest.mark.parametrize("name", DIFFUSION_FIXTURES)
def test_c_oracle_reproduces_reference_diffusion_simulation(c_oracle, name):
    """Time loops with a TeCNO diffusion operator in the system, made by the
    reference build, reproduced bit for bit."""
    z = load_golden(name)
    dim = int(z["dim"])
    cfg = c_oracle.config(dim, z["n"], z["lower"], z["upper"], str(z["flux"]), str(z["recon"]),
                          str(z["integrator"]), str(z["bc"]), float(z["gamma"]))
    c_oracle.set_diffusion(cfg, str(z["diffusion"]), str(z["diffusion_recon"]))
    rc, U, dts, steps, t = c_oracle.simulate(cfg, z["initial"], float(z["cfl"]),
                                             float(z["end_time"]))
    assert rc == 0 and steps == z["steps"] and t == z["t"]
    np.testing.assert_array_equal(dts, z["dts"])
    np.testing.assert_array_equal(U, z["final"])


@pytest.mark.parametrize("name", DIFFUSION_APPLY_FIXTURES)
def test_c_oracle_reproduces_reference_diffusion_calls(c_oracle, name):
    """One operator applied to three states in a row: the reference reads
    entries of its work arrays that only earlier calls wrote, and the
    oracle's persistent state reproduces that bit for bit."""
    z = load_golden(name)
    dim = int(z["dim"])
    cfg = c_oracle.config(dim, z["n"], [0.0] * dim, [1.0] * dim, "hll", "none", "rungekutta3",
                          "neumann", float(z["gamma"]))
    cfg.g = int(z["ghosts"])
    st = c_oracle.diffusion_state(cfg)
    for k in range(z["states"].shape[0]):
        res = c_oracle.apply_diffusion(cfg, str(z["diffusion"]), str(z["diffusion_recon"]), st,
                                       z["states"][k], z["outs"][k])
        np.testing.assert_array_equal(res, z["result"][k])


@pytest.mark.parametrize("dim,n", [(1, (24,)), (2, (12, 11)), (3, (9, 10, 8))])
@pytest.mark.parametrize("kind", ["tecnoroe", "tecnorusanov"])
@pytest.mark.parametrize("recon", ["none", "eno2", "eno3", "eno4"])
def test_c_oracle_diffusion_matches_reference_build(c_oracle, ref_oracle, dim, n, kind, recon):
    """Every operator of the reference's diffusion factory for the Euler
    equations, three calls in a row on fresh random states (skipped without
    the reference build)."""
    g = 1 if recon == "none" else int(recon[-1])
    seed = 6000 + 31 * dim + 7 * ["none", "eno2", "eno3", "eno4"].index(recon) + len(kind)
    states = np.stack([smooth_random_state(seed + k, dim, n, g) for k in range(3)])
    outs = np.stack([np.random.default_rng(seed + k).uniform(-1, 1, states.shape[1:])
                     for k in range(3)])
    ref = ref_oracle.apply_diffusion(dim, n, kind, recon, 1.4, states, outs)
    cfg = c_oracle.config(dim, n, [0.0] * dim, [1.0] * dim, "hll", "none", "rungekutta3",
                          "neumann", 1.4)
    cfg.g = g
    st = c_oracle.diffusion_state(cfg)
    for k in range(3):
        np.testing.assert_array_equal(
            c_oracle.apply_diffusion(cfg, kind, recon, st, states[k], outs[k]), ref[k])


RK4_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                      if f.startswith("rk4_") and f.endswith(".npz"))


@pytest.mark.parametrize("name", RK4_FIXTURES)
def test_c_oracle_reproduces_reference_rk4_simulation(c_oracle, name):
    """RungeKutta4 time loops made by the reference build (RungeKutta4.cpp),
    reproduced bit for bit."""
    z = load_golden(name)
    dim = int(z["dim"])
    cfg = c_oracle.config(dim, z["n"], z["lower"], z["upper"], str(z["flux"]), str(z["recon"]),
                          str(z["integrator"]), str(z["bc"]), float(z["gamma"]))
    rc, U, dts, steps, t = c_oracle.simulate(cfg, z["initial"], float(z["cfl"]),
                                             float(z["end_time"]))
    assert rc == 0 and steps == z["steps"] and t == z["t"]
    np.testing.assert_array_equal(dts, z["dts"])
    np.testing.assert_array_equal(U, z["final"])

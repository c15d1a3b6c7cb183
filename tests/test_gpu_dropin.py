"""The drop-in boundary end to end: the reference's own time loop
(Simulator::incrementSolution's substep loop over ConservedSystem, the
end-time adjuster, the constraint check) with the adapter classes a
maintainer adds to alsvinn — compiled against the reference's headers
(oracle/adapter/) — in place of the reference's NumericalFluxCPU,
Reconstruction, BoundaryCPU and integrators.  Every whole simulation must
equal the reference's own, bit for bit.
"""
import os
import zlib

import numpy as np
import pytest

from oracle_lib import RefB200Oracle, ghost_cells, ref_b200_library_path, smooth_random_state

pytestmark = pytest.mark.gpu

CASES = []
for _dim, _n in ((1, (32,)), (2, (14, 12)), (3, (8, 9, 8))):
    for _recon in ("weno2", "eno3", "mc", "wenof2", "weno3", "none"):
        for _flux, _integ, _bc in (("hll3", "rungekutta3", "periodic"),
                                   ("hll", "rungekutta2", "neumann"),
                                   ("central", "forwardeuler", "periodic")):
            CASES.append((_dim, _n, _recon, _flux, _integ, _bc))


@pytest.fixture(scope="module")
def ref_b200():
    if not os.path.exists(ref_b200_library_path()):
        pytest.skip("oracle/_ref/libalsref_b200.so not built (make -C oracle ref-b200)")
    return RefB200Oracle()


@pytest.mark.parametrize("platform", ["b200", "b200-parts", "b200-all"])
@pytest.mark.parametrize("dim,n,recon,flux,integ,bc", CASES,
                         ids=["d%d-%s-%s-%s-%s" % (c[0], c[2], c[3], c[4], c[5]) for c in CASES])
def test_reference_time_loop_with_b200_classes(ref_b200, platform, dim, n, recon, flux, integ, bc):
    """b200: NumericalFluxB200 as the flux; b200-parts: the reference's
    NumericalFluxCPU over ReconstructionB200, with BoundaryB200 and
    IntegratorB200; b200-all: NumericalFluxB200, BoundaryB200, IntegratorB200."""
    g = ghost_cells(recon)
    seed = zlib.crc32(("dropin-%d-%s-%s-%s" % (dim, recon, flux, integ)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    out = {}
    for p in ("cpu", platform):
        ref_b200.set_flux_platform(p)
        out[p] = ref_b200.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, 0.4, 0.03, st)
    ref_b200.set_flux_platform("cpu")
    a, b = out["cpu"], out[platform]
    assert a[0] == b[0]            # status
    assert a[3] == b[3] >= 1       # steps
    assert a[4] == b[4]            # final time
    np.testing.assert_array_equal(a[2], b[2])   # every dt
    np.testing.assert_array_equal(a[1], b[1])   # final state, ghosts included


TECNO_CASES = [(1, (32,), "tecno6", "rungekutta3", "periodic"),
               (2, (14, 12), "tecno1", "rungekutta2", "neumann"),
               (2, (14, 12), "tecno4", "rungekutta3", "periodic"),
               (3, (10, 11, 10), "tecno4", "forwardeuler", "periodic")]


@pytest.mark.parametrize("platform", ["b200-all"])
def test_reference_time_loop_with_b200_classes_to_final_time(ref_b200, platform):
    """The reference's own loop with all the adapter classes (flux,
    reconstruction, boundary, integrator) to T = 2 on the KH 256^2 UQ member
    7 (WENO2 + HLL3 + RK3, 6,330 steps; about 90 s, the adapters exchange
    host volumes with the device on every call): the dt sequence and the
    final interior equal the reference's CPU classes' (the committed
    final-time fixture)."""
    import hashlib
    import final_time as ft
    z = ft.load("uq256_7")
    n = z["n"]
    U0 = ft.kh_state_from_bands(n, z["band_lo"], z["band_hi"])
    ref_b200.set_flux_platform(platform)
    try:
        rc, U, dts, steps, t = ref_b200.simulate(2, (n, n), (0.0, 0.0), (1.0, 1.0), z["flux"],
                                                 z["recon"], z["integrator"], z["bc"], z["gamma"],
                                                 z["cfl"], z["end_time"], U0)
    finally:
        ref_b200.set_flux_platform("cpu")
    assert rc == 0
    assert steps == z["steps"] and t == z["t"]
    assert ft.dts_digest(dts) == z["dts_sha256"]
    assert hashlib.sha256(ft.interior(U, n).tobytes()).hexdigest() == z["interior_sha256"]


@pytest.mark.parametrize("platform", ["b200", "b200-all"])
@pytest.mark.parametrize("dim,n,flux,integ,bc", TECNO_CASES,
                         ids=["d%d-%s-%s-%s" % (c[0], c[2], c[3], c[4]) for c in TECNO_CASES])
def test_reference_time_loop_with_b200_tecno_flux(ref_b200, platform, dim, n, flux, integ, bc):
    """The TeCNO fluxes (reconstruction none) through NumericalFluxB200 in the
    reference's time loop: same status and step count as the reference's own
    NumericalFluxCPU; states within relative 1e-10 (the device log and the C
    library's log may differ in the last bit)."""
    g = ghost_cells("none", flux)
    seed = zlib.crc32(("dropin-tecno-%d-%s-%s" % (dim, flux, integ)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    out = {}
    for p in ("cpu", platform):
        ref_b200.set_flux_platform(p)
        out[p] = ref_b200.simulate(dim, n, lo, hi, flux, "none", integ, bc, 1.4, 0.4, 0.03, st)
    ref_b200.set_flux_platform("cpu")
    a, b = out["cpu"], out[platform]
    assert a[0] == b[0] == 0
    assert a[3] == b[3] >= 1
    assert abs(a[4] - b[4]) <= 1e-15
    np.testing.assert_allclose(a[2], b[2], rtol=1e-10)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-10, atol=1e-12)


DIFFUSION_CASES = [(1, (32,), "tecno1", "tecnoroe", "eno2", "rungekutta3", "periodic", 0.03),
                   (1, (40,), "tecno4", "tecnorusanov", "eno3", "rungekutta2", "neumann", 0.03),
                   (2, (14, 12), "tecno1", "tecnoroe", "eno2", "rungekutta3", "periodic", 0.01),
                   (3, (10, 11, 10), "tecno1", "tecnorusanov", "eno4", "rungekutta3", "neumann",
                    0.01)]


@pytest.mark.parametrize("dim,n,flux,dkind,drec,integ,bc,T", DIFFUSION_CASES,
                         ids=["d%d-%s-%s-%s" % (c[0], c[2], c[3], c[4]) for c in DIFFUSION_CASES])
def test_reference_time_loop_with_b200_diffusion(ref_b200, dim, n, flux, dkind, drec, integ, bc, T):
    """The reference's time loop with every part from the B200 library
    (NumericalFluxB200, DiffusionB200, BoundaryB200, IntegratorB200) against
    the reference's own classes, TeCNO diffusion in the system: same status
    and steps, states within relative 1e-10 (device vs C library log)."""
    g = max(ghost_cells("none", flux), 1 if drec == "none" else int(drec[-1]))
    seed = zlib.crc32(("dropin-diff-%d-%s-%s" % (dim, flux, drec)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    out = {}
    ref_b200.set_diffusion(dkind, drec)
    try:
        for p in ("cpu", "b200-all"):
            ref_b200.set_flux_platform(p)
            out[p] = ref_b200.simulate(dim, n, lo, hi, flux, "none", integ, bc, 1.4, 0.4, T, st)
    finally:
        ref_b200.set_flux_platform("cpu")
        ref_b200.set_diffusion("none")
    a, b = out["cpu"], out["b200-all"]
    assert a[0] == b[0] == 0
    assert a[3] == b[3] >= 1
    assert abs(a[4] - b[4]) <= 1e-15
    np.testing.assert_allclose(a[2], b[2], rtol=1e-10)
    np.testing.assert_allclose(a[1], b[1], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("dim,n,recon,flux,bc", [(1, (32,), "weno2", "hll3", "periodic"),
                                                 (2, (14, 12), "eno2", "hll", "neumann"),
                                                 (3, (8, 9, 8), "weno2", "hll3", "periodic")])
def test_reference_time_loop_with_b200_rk4(ref_b200, dim, n, recon, flux, bc):
    """RungeKutta4 in the reference's own loop with IntegratorB200 (and the
    other B200 classes) against the reference's RungeKutta4, bit for bit."""
    g = ghost_cells(recon, flux)
    seed = zlib.crc32(("dropin-rk4-%d-%s-%s" % (dim, recon, flux)).encode()) % 100000
    st = smooth_random_state(seed, dim, n, g)
    lo, hi = [0.0] * dim, [1.0] * dim
    out = {}
    for p in ("cpu", "b200-all"):
        ref_b200.set_flux_platform(p)
        out[p] = ref_b200.simulate(dim, n, lo, hi, flux, recon, "rungekutta4", bc, 1.4, 0.4, 0.03,
                                   st)
    ref_b200.set_flux_platform("cpu")
    a, b = out["cpu"], out["b200-all"]
    assert a[0] == b[0] and a[3] == b[3] >= 1 and a[4] == b[4]
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("dim,n,samples", [(1, (33,), 5), (2, (14, 12), 9), (3, (7, 6, 8), 4)])
def test_meanvar_statistics_adapter_against_reference_class(ref_b200, dim, n, samples):
    """MeanVarianceB200 (oracle/adapter/StatisticsB200.hpp, registered as
    REGISTER_STATISTICS(b200, meanvar, ...)) and the reference's own
    MeanVariance, both made by name through the reference's
    StatisticsFactory and run like alsuq's Runner (write per sample,
    combine, finalize, write): the FP64 Welford mean equals the raw-sum mean
    to 1e-14 of the samples' magnitude mean(|U|) (a mean near zero, e.g. of
    a momentum, has no relative scale of its own), and the Welford variance
    M2/M equals S2/M - (S1/M)^2 to 1e-14 of the second moment's scale (the
    raw-moment difference cancels; its own rounding error is of that size)."""
    g = 2
    states = np.stack([smooth_random_state(4000 + 13 * k + dim, dim, n, g)
                       for k in range(samples)])
    mean_ref, var_ref = ref_b200.statistics(dim, n, g, states, platform="cpu", name="meanvar")
    mean, var = ref_b200.statistics(dim, n, g, states, platform="b200", name="meanvar")
    scale = np.mean(np.abs(states), axis=0)
    assert np.all(np.abs(mean - mean_ref) <= 1e-14 * scale)
    second = np.mean(states * states, axis=0)
    assert np.all(np.abs(var - var_ref) <= 1e-14 * np.maximum(second, 1e-300))
    # and the Welford variance against an exactly rounded two-pass variance
    exact = np.var(states.astype(np.longdouble), axis=0).astype(np.float64)
    assert np.all(np.abs(var - exact) <= 1e-13 * np.maximum(exact, 1e-300) + 1e-300)

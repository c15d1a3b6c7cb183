"""Generates tests/golden/final_time_*.npz: final-time results of the
reference's own CPU time loop on the Kelvin-Helmholtz configurations.

TEST INFRASTRUCTURE ONLY.  Run where the reference tree is available:

    make -C oracle ref && python tests/golden/make_final_time.py [uq256] [kh1024]

The reference build (oracle/_ref/libalsref.so: NumericalFluxCPU with
HLL3, ReconstructionCPU with WENO2, RungeKutta3, BoundaryCPU periodic,
driven like Simulator::incrementSolution, alsfvm/src/simulator/
Simulator.cpp:191-214, with the end-time clamp of
alsfvm/src/io/FixedIntervalWriter.cpp:45-53) runs each case to T = 2:

* kh1024: KH 1024^2, parameters = alsuq STLMersenne sample 0, CFL 0.4
  (about 23k steps; about half an hour on eight host cores);
* uq256_<s>: KH 256^2 members s = 7 and 4095 of the 4096-sample UQ
  oracle ensemble (parameters = STLMersenne sample s), CFL 0.4;
* kh256_<scheme>: KH 256^2, parameters = STLMersenne samples 1, 2, 3, 4, CFL 0.4,
  with the other reconstruction / flux / integrator combinations of
  tests/final_time.py's SCHEMES (ENO3, MC, WENO3, WENOF2; HLL, HLL3; RK2,
  RK3);
* sod2d256_neumann, sod3d32_neumann: Sod across the diagonal of the unit
  square (256^2, T = 0.25) and cube (32^3, T = 0.2) with Neumann
  boundaries, WENO2 + HLL3, RK3;
* kh3d48: KH on the unit cube, 48^3, parameters = STLMersenne sample 0,
  CFL 0.4 (the 3-D path, whose z-marching tiles cover 48 = 32 + 16 cells
  in two segments).

What is stored, and why it is enough, is described in tests/final_time.py.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import final_time as ft  # noqa: E402
from oracle_lib import RefOracle  # noqa: E402

CFL = 0.4
END_TIME = 2.0


def run_case(ref, name, n, sample, recon="weno2", flux="hll3", integrator="rungekutta3",
             ghosts=ft.GHOSTS):
    import alsvinn_b200.initial_data as init
    params = np.asarray(ref.stlmersenne(40, sample, 1)[0])
    U_gen = init.kelvin_helmholtz(n, params, ghosts, ft.GAMMA)
    lo, hi = ft.band_limits_of(U_gen, n, ghosts)
    U0 = ft.kh_state_from_bands(n, lo, hi, ghosts)
    assert np.array_equal(U0, U_gen), "band reconstruction differs from the generator"
    t0 = time.perf_counter()
    rc, U, dts, steps, t = ref.simulate(2, (n, n), (0.0, 0.0), (1.0, 1.0), flux, recon,
                                        integrator, "periodic", ft.GAMMA, CFL, END_TIME, U0,
                                        dts_capacity=200000)
    seconds = time.perf_counter() - t0
    assert rc == 0, name
    assert len(dts) == steps
    s = ft.summary(U, n, ghosts)
    out = dict(n=n, sample=sample, params=params, band_lo=lo, band_hi=hi, ghosts=ghosts,
               gamma=ft.GAMMA, cfl=CFL, end_time=END_TIME, flux=flux, recon=recon,
               integrator=integrator, bc="periodic", steps=steps, t=t,
               dts_sha256=ft.dts_digest(dts), dts_head=dts[:64], dts_tail=dts[-64:],
               dts_min=dts.min(), dts_max=dts.max(), l1=s["l1"], sums=s["sums"],
               block_sums=s["block_sums"], interior_sha256=s["interior_sha256"],
               block=ft.BLOCK, observable=ft.observable(U, n, ghosts), ref_loop_seconds=seconds,
               ref_threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
    np.savez_compressed(ft.fixture_path(name), **out)
    print("%s: %d steps, t=%r, %.1f s, observable %.17g, sha %s"
          % (name, steps, t, seconds, out["observable"], s["interior_sha256"][:16]))


def run_case_3d(ref, name, n, sample):
    """KH on the periodic unit cube (interfaces perturbed along x + z),
    n^3 cells, the same scheme to T = 2; the initial state is the
    generator's (its digest stored), the final one summarised per 8^3 block."""
    import alsvinn_b200.initial_data as init
    params = np.asarray(ref.stlmersenne(40, sample, 1)[0])
    U0 = init.kelvin_helmholtz(n, params, ft.GHOSTS, ft.GAMMA, dimension=3)
    t0 = time.perf_counter()
    rc, U, dts, steps, t = ref.simulate(3, (n, n, n), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "hll3",
                                        "weno2", "rungekutta3", "periodic", ft.GAMMA, CFL,
                                        END_TIME, U0, dts_capacity=200000)
    seconds = time.perf_counter() - t0
    assert rc == 0, name
    assert len(dts) == steps
    s = ft.summary3(U, n)
    out = dict(n=n, sample=sample, params=params, initial_sha256=ft.state_digest(U0),
               ghosts=ft.GHOSTS, gamma=ft.GAMMA, cfl=CFL, end_time=END_TIME, flux="hll3",
               recon="weno2", integrator="rungekutta3", bc="periodic", steps=steps, t=t,
               dts_sha256=ft.dts_digest(dts), dts_head=dts[:64], dts_tail=dts[-64:],
               dts_min=dts.min(), dts_max=dts.max(), l1=s["l1"], sums=s["sums"],
               block_sums=s["block_sums"], interior_sha256=s["interior_sha256"],
               block=ft.BLOCK3, ref_loop_seconds=seconds,
               ref_threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
    np.savez_compressed(ft.fixture_path(name), **out)
    print("%s: %d steps, t=%r, %.1f s, sha %s" % (name, steps, t, seconds,
                                                  s["interior_sha256"][:16]))


def run_case_riemann(ref, name):
    """A diagonal Sod problem with Neumann boundaries to its final time;
    the initial state is rebuilt by tests/final_time.py (digest stored)."""
    dim, n, recon, flux, integrator, ghosts, end_time = ft.RIEMANN[name]
    U0 = ft.riemann_state(dim, n, ghosts)
    t0 = time.perf_counter()
    rc, U, dts, steps, t = ref.simulate(dim, (n,) * dim, (0.0,) * dim, (1.0,) * dim, flux, recon,
                                        integrator, "neumann", ft.GAMMA, CFL, end_time, U0,
                                        dts_capacity=200000)
    seconds = time.perf_counter() - t0
    assert rc == 0, name
    assert len(dts) == steps
    s = ft.summary(U, n, ghosts) if dim == 2 else ft.summary3(U, n, ghosts)
    out = dict(n=n, dim=dim, sample=-1, initial_sha256=ft.state_digest(U0), ghosts=ghosts,
               gamma=ft.GAMMA, cfl=CFL, end_time=end_time, flux=flux, recon=recon,
               integrator=integrator, bc="neumann", steps=steps, t=t,
               dts_sha256=ft.dts_digest(dts), dts_head=dts[:64], dts_tail=dts[-64:],
               dts_min=dts.min(), dts_max=dts.max(), l1=s["l1"], sums=s["sums"],
               block_sums=s["block_sums"], interior_sha256=s["interior_sha256"],
               block=ft.BLOCK if dim == 2 else ft.BLOCK3, ref_loop_seconds=seconds,
               ref_threads=int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
    np.savez_compressed(ft.fixture_path(name), **out)
    print("%s: %d steps, t=%r, %.1f s, sha %s" % (name, steps, t, seconds,
                                                  s["interior_sha256"][:16]))


def main(which):
    ref = RefOracle()
    if "uq256" in which:
        for s in (7, 4095):
            run_case(ref, "uq256_%d" % s, 256, s)
    if "kh1024" in which:
        run_case(ref, "kh1024", 1024, 0)
    if "kh3d48" in which:
        run_case_3d(ref, "kh3d48", 48, 0)
    if "riemann" in which:
        for name in ft.RIEMANN_CASES:
            run_case_riemann(ref, name)
    if "schemes" in which:
        # samples 1, 2, ... in increasing order: the reference's generator is
        # one engine per process that only moves forward
        for i, name in enumerate(ft.SCHEME_CASES):
            recon, flux, integrator, ghosts = ft.SCHEMES[name]
            run_case(ref, name, 256, 1 + i, recon, flux, integrator, ghosts)


if __name__ == "__main__":
    main(sys.argv[1:] or ["uq256", "kh1024", "kh3d48", "schemes", "riemann"])

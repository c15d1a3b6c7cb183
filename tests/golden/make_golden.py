"""Generates the golden fixtures in tests/golden/ from the reference's own CPU code.

TEST INFRASTRUCTURE ONLY.  Run where the reference tree is available:

    make -C oracle ref && python tests/golden/make_golden.py

Every fixture is produced by oracle/_ref/libalsref.so, i.e. the reference's
unmodified CPU sources (NumericalFluxCPU, ReconstructionCPU, ENOCPU,
ForwardEuler/RungeKutta2/RungeKutta3, BoundaryCPU, ConservedSystem,
MeanVariance arithmetic, STLMersenne), driven like Simulator::incrementSolution.
Inputs are stored next to the outputs so the fixtures do not depend on the
initial-data generators that made them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle_lib import RefOracle, digest, ghost_cells, smooth_random_state  # noqa: E402

# name: (dim, n, lower, upper, flux, recon, integrator, bc, cfl, end_time, init)
SIMULATIONS = {
    "sod1024_weno2_hll_rk3": (1, (1024,), (-1.0,), (1.0,), "hll", "weno2", "rungekutta3",
                              "neumann", 0.45, 0.2, "sod"),
    "sod256_eno3_hll3_rk2": (1, (256,), (-1.0,), (1.0,), "hll3", "eno3", "rungekutta2",
                             "neumann", 0.45, 0.2, "sod"),
    "sod128_none_hll_fe": (1, (128,), (-1.0,), (1.0,), "hll", "none", "forwardeuler",
                           "neumann", 0.45, 0.2, "sod"),
    "kh16_weno2_central_rk3": (2, (16, 16), (0.0, 0.0), (1.0, 1.0), "central", "weno2",
                               "rungekutta3", "periodic", 0.4, 0.02, "kh"),
    "kh32_weno2_hll3_rk3": (2, (32, 32), (0.0, 0.0), (1.0, 1.0), "hll3", "weno2", "rungekutta3",
                            "periodic", 0.4, 0.3, "kh"),
    "kh24_eno2_hll_rk2": (2, (24, 24), (0.0, 0.0), (1.0, 1.0), "hll", "eno2", "rungekutta2",
                          "periodic", 0.4, 0.1, "kh"),
    "kh20_eno4_hll3_fe_neumann": (2, (20, 20), (0.0, 0.0), (1.0, 1.0), "hll3", "eno4",
                                  "forwardeuler", "neumann", 0.3, 0.05, "kh"),
    "kh3d_12_weno2_hll3_rk3": (3, (12, 12, 12), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "hll3", "weno2",
                               "rungekutta3", "periodic", 0.4, 0.05, "kh3"),
    # seeded smooth random states: variation along every direction
    "rand2d_20x18_weno2_hll3_rk3": (2, (20, 18), (0.0, 0.0), (1.0, 1.0), "hll3", "weno2",
                                    "rungekutta3", "periodic", 0.4, 0.05, "seed:11"),
    "rand2d_16x17_eno3_hll_rk3_neumann": (2, (16, 17), (0.0, 0.0), (1.0, 1.0), "hll", "eno3",
                                          "rungekutta3", "neumann", 0.4, 0.05, "seed:12"),
    "rand3d_9x8x10_weno2_hll3_rk3": (3, (9, 8, 10), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "hll3",
                                     "weno2", "rungekutta3", "periodic", 0.4, 0.03, "seed:13"),
    "rand3d_8x8x8_eno2_central_rk2": (3, (8, 8, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "central",
                                      "eno2", "rungekutta2", "neumann", 0.3, 0.02, "seed:14"),
    # slope-limited reconstructions (MC.hpp, MM.hpp)
    "sod256_mc_hll3_rk3": (1, (256,), (-1.0,), (1.0,), "hll3", "mc", "rungekutta3", "neumann",
                           0.45, 0.2, "sod"),
    "kh24_mm_hll_rk2": (2, (24, 24), (0.0, 0.0), (1.0, 1.0), "hll", "mm", "rungekutta2", "periodic",
                        0.4, 0.1, "kh"),
    "rand3d_9x8x7_mc_hll3_rk3": (3, (9, 8, 7), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "hll3", "mc",
                                 "rungekutta3", "periodic", 0.4, 0.03, "seed:15"),
    # WENO2 in primitive variables with bounds (WENOF2.hpp)
    "sod512_wenof2_hll3_rk3": (1, (512,), (-1.0,), (1.0,), "hll3", "wenof2", "rungekutta3",
                               "neumann", 0.45, 0.2, "sod"),
    "kh32_wenof2_hll3_rk3": (2, (32, 32), (0.0, 0.0), (1.0, 1.0), "hll3", "wenof2", "rungekutta3",
                             "periodic", 0.4, 0.2, "kh"),
    # WENO of order 3 (WENOCPU<3>)
    "sod256_weno3_hll_rk3": (1, (256,), (-1.0,), (1.0,), "hll", "weno3", "rungekutta3", "neumann",
                             0.45, 0.2, "sod"),
    "kh24_weno3_hll3_rk3": (2, (24, 24), (0.0, 0.0), (1.0, 1.0), "hll3", "weno3", "rungekutta3",
                            "periodic", 0.4, 0.2, "kh"),
}


def initial_state(kind, dim, n, g):
    import alsvinn_b200.initial_data as init
    if kind.startswith("seed:"):
        return smooth_random_state(int(kind[5:]), dim, n, g)
    if kind == "sod":
        return init.sod(n[0], g)
    params = np.asarray(RefOracle().stlmersenne(40, 0, 1)[0])
    return init.kelvin_helmholtz(n[0], params, g, dimension=3 if kind == "kh3" else 2)


def write_limiter_cases(ref):
    """One spatial-operator evaluation per (dim, MC/MM/WENOF2/WENO3, flux, boundary)."""
    cases = []
    seed = 2000
    for dim, n in ((1, (16,)), (2, (10, 9)), (3, (8, 8, 9))):
        for recon in ("mc", "mm"):
            for flux in ("hll", "hll3", "central"):
                for bc in ("neumann", "periodic"):
                    seed += 1
                    st = smooth_random_state(seed, dim, n, 2)
                    filled, net, ws = ref.compute_flux(dim, n, [0.0] * dim, [1.0] * dim, flux,
                                                       recon, bc, 1.4, st)
                    cases.append((dim, ",".join(map(str, n)), recon, flux, bc, seed,
                                  digest(filled), digest(net), digest(ws), float(ws.max())))
    seed = 2500
    for dim, n in ((1, (16,)), (2, (10, 9)), (3, (8, 8, 9))):
        for flux in ("hll", "hll3", "central"):
            for bc in ("neumann", "periodic"):
                seed += 1
                st = smooth_random_state(seed, dim, n, 2)
                filled, net, ws = ref.compute_flux(dim, n, [0.0] * dim, [1.0] * dim, flux,
                                                   "wenof2", bc, 1.4, st)
                cases.append((dim, ",".join(map(str, n)), "wenof2", flux, bc, seed,
                              digest(filled), digest(net), digest(ws), float(ws.max())))
    seed = 2700
    for dim, n in ((1, (16,)), (2, (10, 9)), (3, (8, 8, 9))):
        for flux in ("hll", "hll3", "central"):
            for bc in ("neumann", "periodic"):
                seed += 1
                st = smooth_random_state(seed, dim, n, 3)
                filled, net, ws = ref.compute_flux(dim, n, [0.0] * dim, [1.0] * dim, flux,
                                                   "weno3", bc, 1.4, st)
                cases.append((dim, ",".join(map(str, n)), "weno3", flux, bc, seed,
                              digest(filled), digest(net), digest(ws), float(ws.max())))
    with open(os.path.join(HERE, "compute_flux_cases_limiters.txt"), "w") as f:
        f.write("# dim n recon flux bc seed sha256(ghost-filled input) sha256(net flux) "
                "sha256(wave speeds) max_wave_speed\n")
        for c in cases:
            f.write("%d %s %s %s %s %d %s %s %s %.17g\n" % c)


# TeCNO fluxes (reconstruction none), prefixed "tecno_": the CUDA path calls
# the device log, so these are matched to a tolerance on the GPU; the oracle
# matches them bit for bit
TECNO_SIMULATIONS = {
    "tecno_kh32_tecno1_rk3": (2, (32, 32), (0.0, 0.0), (1.0, 1.0), "tecno1", "none",
                              "rungekutta3", "periodic", 0.4, 0.05, "kh"),
    "tecno_rand2d_18x20_tecno4_rk2": (2, (18, 20), (0.0, 0.0), (1.0, 1.0), "tecno4", "none",
                                      "rungekutta2", "neumann", 0.4, 0.04, "seed:21"),
    "tecno_rand1d_64_tecno6_rk3": (1, (64,), (0.0,), (1.0,), "tecno6", "none", "rungekutta3",
                                   "periodic", 0.4, 0.05, "seed:22"),
    "tecno_rand3d_10x11x10_tecno4_fe": (3, (10, 11, 10), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "tecno4",
                                        "none", "forwardeuler", "periodic", 0.3, 0.02, "seed:23"),
}


def write_tecno_fixtures(ref):
    for name, (dim, n, lo, hi, flux, recon, integ, bc, cfl, T, kind) in TECNO_SIMULATIONS.items():
        g = ghost_cells(recon, flux)
        U0 = initial_state(kind, dim, n, g)
        rc, U, dts, steps, t = ref.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, cfl, T, U0)
        assert rc == 0, name
        np.savez_compressed(os.path.join(HERE, name + ".npz"), initial=U0, final=U, dts=dts,
                            steps=steps, t=t, dim=dim, n=np.array(n), lower=np.array(lo),
                            upper=np.array(hi), flux=flux, recon=recon, integrator=integ, bc=bc,
                            cfl=cfl, end_time=T, gamma=1.4)
        print(name, "steps=%d t=%r" % (steps, t))


# TeCNO diffusion in the reference's time loop (ConservedSystem with
# TecnoDiffusionCPU), prefixed "tecnodiff_": (..., diffusion, its reconstruction)
DIFFUSION_SIMULATIONS = {
    "tecnodiff_rand1d_64_tecno1_roe_eno2_rk3": (1, (64,), (0.0,), (1.0,), "tecno1", "none",
                                                "rungekutta3", "periodic", 0.4, 0.05, "seed:31",
                                                "tecnoroe", "eno2"),
    "tecnodiff_sod128_tecno4_rusanov_eno3_rk2": (1, (128,), (-1.0,), (1.0,), "tecno4", "none",
                                                 "rungekutta2", "neumann", 0.4, 0.05, "sod",
                                                 "tecnorusanov", "eno3"),
    "tecnodiff_rand2d_14x12_tecno1_roe_eno2_rk3": (2, (14, 12), (0.0, 0.0), (1.0, 1.0), "tecno1",
                                                   "none", "rungekutta3", "periodic", 0.4, 0.01,
                                                   "seed:32", "tecnoroe", "eno2"),
    "tecnodiff_rand3d_10x11x10_tecno1_rusanov_eno4_rk3": (3, (10, 11, 10), (0.0, 0.0, 0.0),
                                                          (1.0, 1.0, 1.0), "tecno1", "none",
                                                          "rungekutta3", "neumann", 0.4, 0.01,
                                                          "seed:33", "tecnorusanov", "eno4"),
}


def diffusion_ghosts(flux, recon, diffusion_recon):
    return max(ghost_cells(recon, flux), 1 if diffusion_recon == "none" else int(diffusion_recon[-1]))


def write_diffusion_fixtures(ref):
    for name, (dim, n, lo, hi, flux, recon, integ, bc, cfl, T, kind, dkind, drec) in \
            DIFFUSION_SIMULATIONS.items():
        g = diffusion_ghosts(flux, recon, drec)
        U0 = initial_state(kind, dim, n, g)
        ref.set_diffusion(dkind, drec)
        rc, U, dts, steps, t = ref.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, cfl, T, U0)
        ref.set_diffusion("none")
        assert rc == 0, name
        np.savez_compressed(os.path.join(HERE, name + ".npz"), initial=U0, final=U, dts=dts,
                            steps=steps, t=t, dim=dim, n=np.array(n), lower=np.array(lo),
                            upper=np.array(hi), flux=flux, recon=recon, integrator=integ, bc=bc,
                            cfl=cfl, end_time=T, gamma=1.4, diffusion=dkind,
                            diffusion_recon=drec)
        print(name, "steps=%d t=%r" % (steps, t))
    # one operator applied three times in a row (its work arrays carry over)
    for dim, n, dkind, drec, seed in ((2, (12, 11), "tecnoroe", "eno3", 41),
                                      (3, (9, 10, 8), "tecnorusanov", "eno2", 42)):
        g = 1 if drec == "none" else int(drec[-1])
        states = np.stack([smooth_random_state(seed + k, dim, n, g) for k in range(3)])
        outs = np.stack([np.random.default_rng(seed + k).uniform(-1, 1, states.shape[1:])
                         for k in range(3)])
        res = ref.apply_diffusion(dim, n, dkind, drec, 1.4, states, outs)
        name = "diffusion_apply_%dd_%s_%s" % (dim, dkind, drec)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), states=states, outs=outs,
                            result=res, dim=dim, n=np.array(n), ghosts=g, diffusion=dkind,
                            diffusion_recon=drec, gamma=1.4)
        print(name)


# RungeKutta4 (the plug-in integrator path), prefixed "rk4_"
RK4_SIMULATIONS = {
    "rk4_sod256_weno2_hll3": (1, (256,), (-1.0,), (1.0,), "hll3", "weno2", "rungekutta4",
                              "neumann", 0.45, 0.2, "sod"),
    "rk4_kh32_eno2_hll": (2, (32, 32), (0.0, 0.0), (1.0, 1.0), "hll", "eno2", "rungekutta4",
                          "periodic", 0.4, 0.1, "kh"),
    "rk4_rand3d_9x8x10_weno2_hll3": (3, (9, 8, 10), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "hll3",
                                     "weno2", "rungekutta4", "periodic", 0.4, 0.03, "seed:51"),
}


def write_rk4_fixtures(ref):
    for name, (dim, n, lo, hi, flux, recon, integ, bc, cfl, T, kind) in RK4_SIMULATIONS.items():
        g = ghost_cells(recon, flux)
        U0 = initial_state(kind, dim, n, g)
        rc, U, dts, steps, t = ref.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, cfl, T, U0)
        assert rc == 0, name
        np.savez_compressed(os.path.join(HERE, name + ".npz"), initial=U0, final=U, dts=dts,
                            steps=steps, t=t, dim=dim, n=np.array(n), lower=np.array(lo),
                            upper=np.array(hi), flux=flux, recon=recon, integrator=integ, bc=bc,
                            cfl=cfl, end_time=T, gamma=1.4)
        print(name, "steps=%d t=%r" % (steps, t))


# Functionals of the reference's FunctionalFactory (Identity, Moment,
# LogEntropy, BoundedVariation), on seeded states: (dim, n, kind, degree)
FUNCTIONAL_CASES = [(dim, n, kind, degree)
                    for dim, n in ((1, (37,)), (2, (13, 11)), (3, (7, 6, 5)))
                    for kind, degrees in (("identity", (1,)), ("moment", (2, 3)),
                                          ("log_entropy", (1,)), ("bv", (1, 2)))
                    for degree in degrees
                    if not (kind == "bv" and dim > 2)]
FUNCTIONAL_MEMBERS = 2
FUNCTIONAL_WEIGHT = 0.75
FUNCTIONAL_BOX = ((0.0, -1.0, 0.0), (2.0, 1.0, 1.0))


def functional_case_name(dim, kind, degree):
    return "d%d-%s-p%d" % (dim, kind, degree)


# Legendre and LegendrePointWise (2-D only) with their value range
# [min, max] = LEGENDRE_RANGE, which maps every variable of the seeded
# states into [0, 1]; degree -3 is evaluated as degree 2 by Boost.
LEGENDRE_N = (13, 11)
LEGENDRE_RANGE = (-3.0, 3.0)
LEGENDRE_CASES = [("legendre", dict(degree_k=1, degree_n=2, degree_m=3)),
                  ("legendre", dict(degree_k=0, degree_n=0, degree_m=6)),
                  ("legendre", dict(degree_k=4, degree_n=1, degree_m=2)),
                  ("legendre_pointwise", dict(degree=2)),
                  ("legendre_pointwise", dict(degree=7)),
                  ("legendre_pointwise", dict(degree=-3))]


def legendre_case_name(kind, params):
    if kind == "legendre":
        return "d2-legendre-k%dn%dm%d" % (params["degree_k"], params["degree_n"],
                                          params["degree_m"])
    return "d2-legendre_pointwise-p%d" % params["degree"]


def write_functional_fixtures(ref):
    """tests/golden/functionals_ref.npz: for every case and member k, the
    state smooth_random_state(600 + 7 k + dim) (ghost width 2), an output
    that starts at 0.5 + k, and the reference's out + 0.75 f(state)."""
    out = {}
    for dim, n, kind, degree in FUNCTIONAL_CASES:
        name = functional_case_name(dim, kind, degree)
        results, starts = [], []
        for k in range(FUNCTIONAL_MEMBERS):
            st = smooth_random_state(600 + 7 * k + dim, dim, n, 2)
            size = ref.functional(dim, n, 2, kind, st, weight=0.0, degree=degree).shape[1]
            start = np.full((dim + 2, size), 0.5 + k)
            starts.append(start)
            results.append(ref.functional(dim, n, 2, kind, st, weight=FUNCTIONAL_WEIGHT,
                                          out=start, degree=degree, gamma=1.4,
                                          lower=FUNCTIONAL_BOX[0], upper=FUNCTIONAL_BOX[1]))
        out[name + "/start"] = np.stack(starts)
        out[name + "/result"] = np.stack(results)
    lo, hi = LEGENDRE_RANGE
    for kind, params in LEGENDRE_CASES:
        name = legendre_case_name(kind, params)
        results, starts = [], []
        for k in range(FUNCTIONAL_MEMBERS):
            st = smooth_random_state(600 + 7 * k + 2, 2, LEGENDRE_N, 2)
            size = ref.functional(2, LEGENDRE_N, 2, kind, st, weight=0.0, min_value=lo,
                                  max_value=hi, **params).shape[1]
            start = np.full((4, size), 0.5 + k)
            starts.append(start)
            results.append(ref.functional(2, LEGENDRE_N, 2, kind, st, weight=FUNCTIONAL_WEIGHT,
                                          out=start, min_value=lo, max_value=hi,
                                          lower=FUNCTIONAL_BOX[0], upper=FUNCTIONAL_BOX[1],
                                          **params))
        out[name + "/start"] = np.stack(starts)
        out[name + "/result"] = np.stack(results)
    np.savez_compressed(os.path.join(HERE, "functionals_ref.npz"), **out)
    print("functionals_ref.npz: %d cases" % (len(FUNCTIONAL_CASES) + len(LEGENDRE_CASES)))


def main():
    ref = RefOracle()
    out = {}
    # the generator is a process-wide singleton: draw first, in sample order
    draws = ref.stlmersenne(40, 0, 3)
    np.savez_compressed(os.path.join(HERE, "stlmersenne_40x3.npz"), draws=draws)
    for name, (dim, n, lo, hi, flux, recon, integ, bc, cfl, T, kind) in SIMULATIONS.items():
        g = ghost_cells(recon)
        U0 = initial_state(kind, dim, n, g)
        rc, U, dts, steps, t = ref.simulate(dim, n, lo, hi, flux, recon, integ, bc, 1.4, cfl, T, U0)
        assert rc == 0, name
        np.savez_compressed(os.path.join(HERE, name + ".npz"), initial=U0, final=U, dts=dts,
                            steps=steps, t=t, dim=dim, n=np.array(n), lower=np.array(lo),
                            upper=np.array(hi), flux=flux, recon=recon, integrator=integ, bc=bc,
                            cfl=cfl, end_time=T, gamma=1.4)
        out[name] = (steps, t)
    # one spatial-operator evaluation per (dim, reconstruction, flux, boundary):
    # seeded inputs, digest of the reference's net flux and wave speeds
    cases = []
    seed = 1000
    for dim, n in ((1, (16,)), (2, (10, 9)), (3, (8, 8, 9))):
        for recon in ("none", "weno2", "eno2", "eno3", "eno4"):
            g = ghost_cells(recon)
            if min(n) < 2 * g:
                continue
            for flux in ("hll", "hll3", "central"):
                for bc in ("neumann", "periodic"):
                    seed += 1
                    st = smooth_random_state(seed, dim, n, g)
                    lo = [0.0] * dim
                    hi = [1.0] * dim
                    filled, net, ws = ref.compute_flux(dim, n, lo, hi, flux, recon, bc, 1.4, st)
                    cases.append((dim, ",".join(map(str, n)), recon, flux, bc, seed,
                                  digest(filled), digest(net), digest(ws), float(ws.max())))
    write_limiter_cases(ref)
    write_tecno_fixtures(ref)
    write_diffusion_fixtures(ref)
    write_rk4_fixtures(ref)
    with open(os.path.join(HERE, "compute_flux_cases.txt"), "w") as f:
        f.write("# dim n recon flux bc seed sha256(ghost-filled input) sha256(net flux) "
                "sha256(wave speeds) max_wave_speed\n")
        for c in cases:
            f.write("%d %s %s %s %s %d %s %s %s %.17g\n" % c)
    # structure-function cubes through the reference's dispatchComputeStructureCubeCPU
    rows = []
    seed = 3000
    for dim, n in ((1, (32,)), (2, (12, 10)), (3, (7, 6, 8))):
        for bc in ("periodic", "neumann"):
            for H, p in ((6, 1.0), (5, 2.0), (4, 3.0), (5, 2.5)):
                seed += 1
                st = smooth_random_state(seed, dim, n, 2)
                out = ref.structure_cube(dim, n, 2, bc, H, p, st)
                rows.append((dim, ",".join(map(str, n)), bc, H, p, seed, digest(out),
                             float(out.max())))
    with open(os.path.join(HERE, "structure_cube_cases.txt"), "w") as f:
        f.write("# dim n bc H p seed sha256(out, nvar x H) max\n")
        for r in rows:
            f.write("%d %s %s %d %.17g %d %s %.17g\n" % r)
    write_functional_fixtures(ref)
    # alsuq's MeanVariance made by name through its StatisticsFactory
    states = np.stack([smooth_random_state(77 + k, 2, (6, 5), 2) for k in range(7)])
    mean, var = ref.statistics(2, (6, 5), 2, states, platform="cpu", name="meanvar")
    np.savez_compressed(os.path.join(HERE, "meanvar_7.npz"), mean=mean, var=var,
                        seeds=np.arange(77, 84))
    for k, v in out.items():
        print(k, "steps=%d t=%r" % v)


if __name__ == "__main__":
    if sys.argv[1:] == ["functionals"]:
        write_functional_fixtures(RefOracle())
    else:
        main()

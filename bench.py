"""Benchmark of the cell-update hot path: cell-updates/s on B200.

Default workload: 2-D Euler Kelvin-Helmholtz, 1024x1024 periodic unit
square, FP64, WENO2 + HLL3, SSP-RK3, CFL 0.4 (the plain GPU drop-in
configuration).  One bench step = one full time step (CFL reduction and
three Runge-Kutta stages) over the whole grid.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank advances its own Kelvin-Helmholtz sample (sample
index = rank): ensemble members are independent, so ranks share no data and
no collective runs inside the timed region (weak scaling).  Timing: per-step
CUDA events on the solver's stream with an L2 flush (a 512 MiB write)
between timed steps, barrier + synchronize around the timed region, max over
ranks.  `--impl reference` times the reference's own CPU implementation
(oracle/_ref, the unmodified reference sources) on the host cores.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

N = 1024
DIM = 2
NVAR = 4
GHOSTS = 2
FLUX, RECON, INTEG, BC, CFL = "hll3", "weno2", "rungekutta3", "periodic", 0.4
METRIC = "cell-updates/s (2-D Euler KH 1024^2, WENO2+HLL3, RK3, FP64)"
WORKLOAD = {"workload": "kelvin-helmholtz 2-D Euler 1024x1024 periodic, FP64, weno2+hll3, "
                        "rungekutta3, cfl 0.4; one step = one full time step",
            "cells": N * N, "precision": "fp64", "l2": "flushed between timed steps (512 MiB write)"}
# algorithmic bytes per interior cell and launch (FP64, 4 planes):
#   stage 0 reads U^n, writes L                    -> 2 plane passes
#   stage 1 reads L and U^n, writes U2             -> 3
#   stage 2 reads U2 and U^n, writes U^{n+1}       -> 3
ALG_BYTES_PER_CELL = {"flux0": 2 * NVAR * 8, "rk3_1": 3 * NVAR * 8, "rk3_2": 3 * NVAR * 8}
KERNEL_NAMES = ["flux0", "rk3_1", "rk3_2"]


# time steps per CUDA graph of the solver (als_solver_advance)
GRAPH_STEPS = 8


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def tensor_peak():
    """(burst, sustained, source) dense BF16 TFLOP/s."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("bf16_tflops", 1590.0), p.get("bf16_tflops", 1590.0), "measured (burst)"
    return 1590.0, 1590.0, "fallback (burst)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, val in zip(names, p[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_issue_peak():
    """(FP64 thread instructions/s, source): 148 SMs x 64 FP64 lanes per
    clock (half the 128 FP32 lanes; B200's 37 TFLOP/s FP64 = 2 flops per
    FMA lane) at the measured maximum SM clock."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    mhz, src = 1965.0, "nominal clock"
    if os.path.exists(path):
        with open(path) as f:
            mhz = json.load(f).get("sm_max_mhz", mhz)
        src = "sm_max_mhz of MEASURED_PEAKS.json"
    return 148 * 64 * mhz * 1e6, "148 SMs x 64 FP64 lanes/clock x %.0f MHz (%s)" % (mhz, src)


def fp64_roofline(dom, cells, hbm_peak, peak_kind, traffic, per_kernel):
    """The binding ceiling of the plain FP64 method: FP64 instruction issue.
    achieved = FP64 thread instructions per cell and stage (ncu
    sm__sass_thread_inst_executed_op_fp64_pred_on over a launch, divided by
    its cells; profiles/traffic_kh1024.json) x cells / the stage kernel's
    event duration.  Beside it: the issue of all instructions (ncu
    smsp__thread_inst_executed per cell against 148 SMs x 4 schedulers x 32
    lanes per clock; predicated-off lanes are not counted, so this fraction
    is a lower bound of the issue slots used) and the HBM fraction of the
    same launch."""
    tpath = os.path.join(ROOT, "profiles", "traffic_kh1024.json")
    per_cell = all_per_cell = None
    if os.path.exists(tpath):
        with open(tpath) as f:
            t = json.load(f)
        per_cell = t.get("fp64_inst_per_cell", {}).get(dom["kernel"])
        all_per_cell = t.get("inst_per_cell", {}).get(dom["kernel"])
    peak, src = fp64_issue_peak()
    out = {"bound": "fp64", "unit": "FP64 thread-inst/s", "peak": peak, "peak_source": src,
           "kernel": "stage kernel '%s' (%.4f ms)" % (dom["kernel"], dom["ms"])}
    if per_cell:
        out["achieved"] = per_cell * cells / (dom["ms"] * 1e-3)
        out["frac"] = out["achieved"] / peak
        out["fp64_inst_per_cell"] = per_cell
    if all_per_cell:
        issue_peak = peak * 2          # 128 thread-instructions per SM and clock
        achieved = all_per_cell * cells / (dom["ms"] * 1e-3)
        out["issue"] = {"achieved": achieved, "peak": issue_peak, "unit": "thread-inst/s",
                        "frac": achieved / issue_peak, "inst_per_cell": all_per_cell,
                        "peak_source": "148 SMs x 4 schedulers x 32 lanes per clock"}
    out["hbm"] = {"achieved": dom["achieved_gbs"], "peak": hbm_peak, "unit": "GB/s",
                  "frac": dom["achieved_gbs"] / hbm_peak, "traffic": traffic,
                  "peak_source": peak_kind}
    out["per_kernel"] = per_kernel
    return out


def kh_state(sample):
    import alsvinn_b200 as als
    params = als.uniform_draws(40, sample, 1)[0]
    return als.kelvin_helmholtz(N, params, GHOSTS)


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the CPU records."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(state, target_seconds=12.0):
    """The reference's own CPU path (oracle/_ref) on a bounded sample of the
    same workload, all host threads; falls back to the C restatement."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import COracle, RefOracle, ref_library_path
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if os.path.exists(ref_library_path()):
        ref = RefOracle()
        # a 2-step probe sizes one timed sample of about target_seconds
        ref.simulate(DIM, (N, N), (0, 0), (1, 1), FLUX, RECON, INTEG, BC, 1.4, CFL, 2.0, state,
                     max_steps=2)
        per_step = max(ref.lib.alsref_last_loop_seconds() / 2, 1e-4)
        steps = int(min(max(target_seconds / per_step, 2), 2000))
        rc, _, _, done, _ = ref.simulate(DIM, (N, N), (0, 0), (1, 1), FLUX, RECON, INTEG, BC,
                                         1.4, CFL, 2.0, state, max_steps=steps)
        secs = ref.lib.alsref_last_loop_seconds()
        kind, sample = "reference", "%d time steps of the same KH 1024^2 state" % done
        threads = int(os.environ.get("OMP_NUM_THREADS", cores))
    else:
        c = COracle()
        cfg = c.config(DIM, (N, N), (0, 0), (1, 1), FLUX, RECON, INTEG, BC, 1.4)
        done = 2
        t0 = time.perf_counter()
        c.simulate(cfg, state, CFL, 2.0, max_steps=done)
        secs = time.perf_counter() - t0
        kind, sample, threads = "port", "%d time steps of the same KH 1024^2 state" % done, 1
    return {"value": N * N * done / secs, "unit": "cell-updates/s", "cores": threads,
            "kind": kind, "sample": sample, "seconds": secs, "cpu_model": cpu_model(),
            "host_threads": os.cpu_count()}


def run_reference_arm(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import RefOracle, ref_library_path
    if not os.path.exists(ref_library_path()):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref (reference CPU build) missing on this machine"}))
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    ref = RefOracle()
    # the sample's parameters from the reference's own generator
    # (STLMersenne.cpp:38-85); the initial-data formula is plain NumPy, so
    # this arm loads none of the B200 library
    import alsvinn_b200.initial_data as init
    state = init.kelvin_helmholtz(N, ref.stlmersenne(40, 0, 1)[0], GHOSTS)
    # each bench step: one full KH 1024^2 time step by the reference's CPU code
    ref.simulate(DIM, (N, N), (0, 0), (1, 1), FLUX, RECON, INTEG, BC, 1.4, CFL, 2.0, state,
                 max_steps=args.warmup)
    rc, _, _, steps, _ = ref.simulate(DIM, (N, N), (0, 0), (1, 1), FLUX, RECON, INTEG, BC, 1.4,
                                      CFL, 2.0, state, max_steps=args.steps)
    secs = ref.lib.alsref_last_loop_seconds()
    value = N * N * steps / secs
    out = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
           "steps": steps, "warmup": args.warmup, "ms_per_step": secs / steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": WORKLOAD, "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "cell-updates/s",
                            "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "reference",
                            "sample": "%d time steps of KH 1024^2 (reference CPU sources, OpenMP)"
                            % steps, "cpu_model": cpu_model(), "host_threads": os.cpu_count()},
           "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# Ensemble workloads: (dimension, [(n, members), ...]).  "ensemble": 512 KH
# samples at 256^2; "multilevel": four KH levels (2048x128^2, 512x256^2,
# 128x512^2, 32x1024^2) in one launch per stage; "kh3d": 8 3-D KH samples
# at 128^3 (FP64 spot check).
BATCHES = {
    "ensemble": (2, [(256, 512)]),
    "multilevel": (2, [(128, 2048), (256, 512), (512, 128), (1024, 32)]),
    "kh3d": (3, [(128, 8)]),
}


def run_batch(args, rank, world, local):
    """Times `steps` time steps of every member of every level (one launch
    per stage over all of them); value = member cell-updates / s."""
    import torch
    import torch.distributed as dist
    import alsvinn_b200 as als
    from alsvinn_b200 import distributed
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dim, levels = BATCHES[args.workload]
    if (args.n or args.members) and len(levels) == 1:
        levels = [(args.n or levels[0][0], args.members or levels[0][1])]
    precision = "fp64" if args.workload == "kh3d" else args.precision
    nvar = dim + 2
    elem = 8 if precision == "fp64" else 4
    lv = [{"n": (n,) * dim, "members": m} for n, m in levels]
    sim = als.Simulator(dim, levels=lv, flux=FLUX, reconstruction=RECON, integrator=INTEG,
                        boundary=BC, cfl=CFL, end_time=1e9, precision=precision, device=local)
    first = 0
    for lev in sim.levels:
        n = lev["n"][0]
        for a in range(0, lev["members"], 64):
            k = min(64, lev["members"] - a)
            params = als.uniform_draws(40, rank * sim.members + first + a, k)
            states = np.stack([als.kelvin_helmholtz(n, params[j], GHOSTS, dimension=dim)
                               for j in range(k)])
            sim.set_state(states, first_member=lev["first"] + a)
        first += lev["members"]
    if args.kernels_only:
        sim.advance(args.warmup + args.steps)
        sim.synchronize()
        sim.close()
        return
    schedule = sim.tune(steps=2)
    # the tuned choice against every level on one fixed tile shape (each
    # timed over the same number of steps from the current state)
    shape_ms = {}
    for shape in (0, 1):
        try:
            sim.set_tiles([shape] * len(sim.levels))
        except Exception:
            continue
        sim.advance(2)
        sim.synchronize()
        t0 = time.perf_counter()
        sim.advance(4)
        sim.synchronize()
        shape_ms["all levels shape %d" % shape] = (time.perf_counter() - t0) * 1e3 / 4
    sim.set_tiles(schedule["tile_shapes"])
    sim.advance(2)
    sim.synchronize()
    t0 = time.perf_counter()
    sim.advance(4)
    sim.synchronize()
    shape_ms["tuned %s" % schedule["tile_shapes"]] = (time.perf_counter() - t0) * 1e3 / 4
    schedule["ms_per_step_by_tiles"] = shape_ms
    # the warm-up also captures the solver's 8-step CUDA graph, which the
    # first advance of 8 or more steps builds: at least 8 steps, so that the
    # capture is not part of the timed region
    warmup = max(args.warmup, GRAPH_STEPS)
    sim.advance(warmup)
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    sim.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    bad = [m for m in range(sim.members) if sim.info(m)["status"] != 0]
    nbad = len(bad)
    if world > 1:
        tb = torch.tensor([nbad], dtype=torch.int64, device="cuda")
        dist.all_reduce(tb, op=dist.ReduceOp.MAX)
        nbad = int(tb.item())
    if nbad:
        raise RuntimeError("constraint violation in members %r (this rank)" % bad[:8])
    cells = sum((lev["n"][0] ** dim) * lev["members"] for lev in sim.levels)
    value = world * cells * args.steps / (ms * 1e-3)
    kms = np.array([sim.profile_step() for _ in range(3)]).mean(axis=0)
    hbm_peak, peak_kind = peaks()
    per_cell = {"flux0": 2 * nvar * elem, "rk3_1": 3 * nvar * elem, "rk3_2": 3 * nvar * elem}
    roof = [{"kernel": k, "ms": float(t), "achieved_gbs": per_cell[k] * cells / (t * 1e-3) / 1e9}
            for k, t in zip(KERNEL_NAMES, kms)]
    dom = max(range(3), key=lambda i: roof[i]["ms"])
    # FP64 statistics of the final states (every level) and the FP64 conservation sums
    # (one all_gather of (n, mean, M2) per level and a rank-ordered merge across GPUs)
    t0 = time.perf_counter()
    for k, lev in enumerate(sim.levels):
        mv = als.MeanVariance(nvar * lev["plane"], device=local)
        mv.add_solver(sim, k)
        if world > 1:
            merged = distributed.merge_statistics(mv)
            merged.close()
        mv.close()
    torch.cuda.synchronize()
    stats_s = time.perf_counter() - t0
    result = {
        "metric": "member cell-updates/s (%s, KH, WENO2+HLL3, RK3, %s)" % (args.workload, precision),
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == "fp64" else "f32",
        "data": "synthetic (Kelvin-Helmholtz samples from the reference's generator)",
        "warmup": warmup,
        "config": {"workload": args.workload, "levels": levels, "dimension": dim,
                   "precision": precision, "member_cells": cells,
                   "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": roof[dom]["achieved_gbs"], "peak": hbm_peak,
                     "unit": "GB/s", "frac": roof[dom]["achieved_gbs"] / hbm_peak,
                     "traffic": None, "kernel": roof[dom]["kernel"], "peak_source": peak_kind,
                     "per_kernel": roof},
        "schedule": schedule, "statistics_seconds": stats_s,
        "gpu_launches": args.steps * sim.launches_per_step(), "clocks": clock_info,
    }
    if rank == 0:
        print(json.dumps(result))
    sim.close()
    if world > 1:
        dist.destroy_process_group()


UQ_ORACLE = os.path.join(ROOT, "tests", "golden", "uq_kh256_fp64_4096.npz")


def run_uq(args, rank, world, local):
    """UQ time-to-error: plain batched Monte Carlo against the surrogate
    control variate, KH 256^2 to T = 2, observable = mean density over
    [0.25, 0.75]^2, both measured against the 4096-sample FP64 ensemble.

    The surrogate (40 -> 256 x4 -> 1, BF16 tensor cores) is trained on the
    FP64 ensemble's samples 0..1023 (Adam, lr 1e-3, up to 2000 steps, early
    stopping on samples 1024..2047) and evaluated on samples 2048..4095: there
    the residual variance Var(Y - b f) / Var(Y) (and the same for Y^2) says
    how many fewer solver samples the control-variate estimator needs for
    the RMS error of plain MC with M samples.  Both arms are then run for
    real on fresh samples (FP32 members, FP64 statistics): plain MC with M
    samples, the control variate with the reduced count plus the surrogate's
    E[f], E[f^2] from 2^22 evaluations.  value = plain wall-clock / control
    variate wall-clock (training included, training data reused from the
    oracle ensemble; the ratio with the training data's solves counted too
    is reported beside it)."""
    import torch
    import alsvinn_b200 as als
    from alsvinn_b200 import uq
    if rank != 0:
        return
    torch.cuda.set_device(local)
    if not os.path.exists(UQ_ORACLE):
        raise RuntimeError("missing %s (python tests/golden/make_uq_oracle.py)" % UQ_ORACLE)
    z = np.load(UQ_ORACLE)
    y_or = np.asarray(z["y"], dtype=np.float64)
    n_or = y_or.size
    n = int(z["n"])
    T = float(z["end_time"])
    p_or = als.uniform_draws(40, 0, n_or)
    mu_or, var_or = uq.plain_mc(y_or)
    M = args.samples
    prec = args.precision

    def now():
        torch.cuda.synchronize()
        return time.perf_counter()

    clocks = ClockSampler(local)
    clocks.start()
    t0 = now()
    sur = als.Surrogate(seed=0, device=local)
    losses = sur.fit(p_or[:1024], y_or[:1024], steps=2000, lr=1e-3,
                     validation=(p_or[1024:2048], y_or[1024:2048]))
    t_train = now() - t0
    fj = sur(p_or[2048:]).double().cpu().numpy()
    yj = y_or[2048:]
    fc = fj - fj.mean()
    beta = np.dot(fc, yj - yj.mean()) / np.dot(fc, fc)
    r_mean = float(np.var(yj - beta * fj) / np.var(yj))
    g2 = fj * fj
    y2 = yj * yj
    gc = g2 - g2.mean()
    beta2 = np.dot(gc, y2 - y2.mean()) / np.dot(gc, gc)
    r_var = float(np.var(y2 - beta2 * g2) / np.var(y2))
    rho2 = float(np.corrcoef(yj, fj)[0, 1] ** 2)
    t0 = now()
    m1, m2 = sur.moments(1 << 22, seed=3)
    t_moments = now() - t0

    # plain batched MC, M fresh samples
    p_pl, y_pl, info_pl = uq.kh_observable_ensemble(n, n_or, M, precision=prec, end_time=T,
                                                    device=local)
    t_plain = info_pl["solve_seconds"]
    mean_pl, var_pl = uq.plain_mc(y_pl)
    # control variate: the sample count that matches plain MC's RMS errors
    m_cv = int(np.ceil(M * max(r_mean, r_var))) + 1
    m_cv = min(max(m_cv, 8), M)
    p_cv, y_cv, info_cv = uq.kh_observable_ensemble(n, n_or + M, m_cv, precision=prec,
                                                    end_time=T, device=local)
    t0 = now()
    f_cv = sur(p_cv).double().cpu().numpy()
    mean_cv, var_cv, _, _ = uq.control_variate(y_cv, f_cv, m1, m2)
    t_eval = now() - t0
    clock_info = clocks.stop()
    sur.close()
    t_cv = info_cv["solve_seconds"] + t_train + t_moments + t_eval
    per_sample = t_plain / M
    t_cv_with_data = t_cv + 1024 * per_sample
    curve = uq_error_curve(y_or, fj, m1, m2, per_sample, t_train + t_moments)
    result = {
        "metric": "UQ time-to-error, plain batched MC / surrogate control variate "
                  "(KH %d^2, T=%g, mean and variance of mean rho over [0.25,0.75]^2)" % (n, T),
        "value": t_plain / t_cv, "unit": "x (plain wall-clock / control-variate wall-clock)",
        "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * t_cv,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 members, f64 statistics, bf16 surrogate",
        "data": "synthetic (Kelvin-Helmholtz samples from the reference's generator)",
        "config": {"workload": "uq", "n": n, "end_time": T, "plain_samples": M,
                   "cv_samples": m_cv, "member_precision": prec,
                   "oracle": "%d-sample FP64 ensemble (tests/golden)" % n_or,
                   "surrogate": "40-256x4-1 GELU, Adam lr 1e-3, <=2000 steps, early stop"},
        "uq": {
            "oracle_mean": mu_or, "oracle_var": var_or,
            "heldout_rho2": rho2, "residual_ratio_mean": r_mean, "residual_ratio_var": r_var,
            "surrogate_best_step": int(sur.best_step), "final_train_loss": float(losses[-1]),
            "plain": {"mean": mean_pl, "var": var_pl, "err_mean": mean_pl - mu_or,
                      "err_var": var_pl - var_or, "rms_err_mean_expected": np.sqrt(var_or / M),
                      "seconds": t_plain},
            "cv": {"mean": mean_cv, "var": var_cv, "err_mean": mean_cv - mu_or,
                   "err_var": var_cv - var_or,
                   "rms_err_mean_expected": np.sqrt(r_mean * var_or / m_cv),
                   "seconds_solve": info_cv["solve_seconds"], "seconds_train": t_train,
                   "seconds_moments": t_moments, "seconds_eval": t_eval},
            "ratio_including_training_data": t_plain / t_cv_with_data,
            "per_sample_seconds": per_sample,
            "time_to_error_curve": curve,
        },
        # stage launches of both solves, plus the surrogate's (about 20 per
        # training step, 6 per inference chunk of 32768 rows)
        "gpu_launches": int(info_pl["stage_launches"] + info_cv["stage_launches"]
                            + 20 * 2000 + 6 * (((1 << 22) + 32767) // 32768)),
        "clocks": clock_info,
    }
    print(json.dumps(result, default=float))


def uq_error_curve(y_or, f_held, f_mean, f2_mean, per_sample, cv_fixed_seconds,
                   counts=(128, 256, 512, 1024)):
    """Errors of both estimators against the 4096-sample FP64 oracle at
    several sample counts, over disjoint repetitions drawn from the held-out
    samples 2048..4095 (their FP64 observables and surrogate values; no
    training sample is reused).  Each point: sample count, RMS error of the
    mean and of the variance over the repetitions for plain MC and for the
    control variate, and the GPU wall-clock each arm needs for that count
    (per-sample solve time of this run; the control variate adds its
    training and E[f], E[f^2] passes)."""
    from alsvinn_b200 import uq
    mu, var = uq.plain_mc(y_or)
    held = y_or[2048:]
    out = []
    for M in counts:
        reps = held.size // M
        ep, ev, cp, cv = [], [], [], []
        for r in range(reps):
            y = held[r * M:(r + 1) * M]
            f = f_held[r * M:(r + 1) * M]
            m_pl, v_pl = uq.plain_mc(y)
            m_cv, v_cv, _, _ = uq.control_variate(y, f, f_mean, f2_mean)
            ep.append(m_pl - mu)
            ev.append(v_pl - var)
            cp.append(m_cv - mu)
            cv.append(v_cv - var)
        rms = lambda e: float(np.sqrt(np.mean(np.square(e))))  # noqa: E731
        out.append({"samples": M, "repetitions": reps,
                    "plain": {"rms_err_mean": rms(ep), "rms_err_var": rms(ev),
                              "seconds": M * per_sample},
                    "cv": {"rms_err_mean": rms(cp), "rms_err_var": rms(cv),
                           "seconds": M * per_sample + cv_fixed_seconds}})
    return out


def run_surrogate(args, rank, world, local):
    """The surrogate's tensor-core kernels: inference over 2^20 parameter
    rows (the E[f], E[f^2] pass of the control variate) and full-batch
    training steps on 1024 rows.  Rates are taken around whole library
    calls (each call ends synchronised); FLOPs are algorithmic (2 per
    multiply-add of the 40 -> 256 x4 -> 1 network, K unpadded)."""
    import torch
    import alsvinn_b200 as als
    from alsvinn_b200 import _lib
    if rank != 0:
        return
    torch.cuda.set_device(local)
    rows = 1 << 20
    flop_row = 2 * (40 * 256 + 3 * 256 * 256 + 256)
    sur = als.Surrogate(seed=0, device=local)
    x = torch.empty(rows * 40, dtype=torch.float32, device="cuda")
    _lib.check(sur._lib.als_mlp_sample_uniform(x.data_ptr(), x.numel(), 5, 0))
    x = x.view(rows, 40)
    # each call ends synchronised (about 0.8 ms): at least 20 timed calls
    steps = max(args.steps, 20)
    for _ in range(max(args.warmup, 3)):
        sur.forward_raw(x)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    t0 = time.perf_counter()
    for _ in range(steps):
        sur.forward_raw(x)
    torch.cuda.synchronize()
    infer_s = (time.perf_counter() - t0) / steps
    # the same rows through one kernel per layer (activations via HBM)
    for _ in range(2):
        sur.forward_raw(x, per_layer=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        sur.forward_raw(x, per_layer=True)
    torch.cuda.synchronize()
    layers_s = (time.perf_counter() - t0) / steps
    xt = x[:1024].clone()
    tt = torch.sin(xt.sum(dim=1))
    sur.train_raw(xt, tt, 5)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    train_steps = 200
    sur.train_raw(xt, tt, train_steps)
    torch.cuda.synchronize()
    train_s = (time.perf_counter() - t0) / train_steps
    clock_info = clocks.stop()
    sur.close()
    _, bf16_peak, kind = tensor_peak()
    achieved = rows * flop_row / infer_s / 1e12
    result = {
        "metric": "surrogate inference rows/s (40-256x4-1 MLP, BF16 tcgen05, FP32 accumulate)",
        "value": rows / infer_s, "unit": "rows/s", "n_gpus": 1, "steps": steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * infer_s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
        "data": "synthetic (U[0,1) parameter draws)",
        "config": {"workload": "surrogate", "rows": rows, "train_batch": 1024},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": bf16_peak,
                     "unit": "TFLOP/s", "frac": achieved / bf16_peak, "traffic": None,
                     "kernel": "whole forward call: per 262,144 rows one input-packing "
                               "kernel and one whole-network tcgen05 kernel (4 layers + head); "
                               "wall clock around calls that each end synchronised",
                     "peak_source": kind},
        "per_layer_ms_per_step": 1e3 * layers_s,
        "per_layer_frac": rows * flop_row / layers_s / 1e12 / bf16_peak,
        "train_step_ms": 1e3 * train_s,
        "train_tflops": 3 * 1024 * flop_row / train_s / 1e12,
        "gpu_launches": steps * 2 * (rows // 262144),
        "clocks": clock_info,
    }
    print(json.dumps(result))

def run_plugin(args, rank, world, local):
    """KH 1024^2 FP64 through the plug-in classes: the reference's time loop
    (Simulator.cpp:191-214) with NumericalFlux as the system, Integrator for
    the stages and Boundary after every stage, each one C-ABI call -- what a
    user of the reference gets by switching only the platform of those
    objects.  The time step takes one host round trip per step (the wave
    speeds of the first stage), as in the reference."""
    import torch
    import torch.distributed as dist
    import alsvinn_b200 as als
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n = (N, N)
    lengths = [1.0 / N, 1.0 / N, 0.0]
    nf = als.NumericalFlux(DIM, n, FLUX, RECON)
    bc = als.Boundary(DIM, n, nf.getNumberOfGhostCells(), BC)
    integ = als.Integrator(INTEG, nf, CFL)
    substeps = integ.getNumberOfSubsteps()
    first = torch.from_numpy(kh_state(rank)).cuda()
    vols = [first] + [first.clone() for _ in range(substeps)]
    bc.applyBoundaryConditions(vols[0])
    state = {"t": 0.0}

    def step():
        dt = 0.0
        for s in range(substeps):
            dt = integ.performSubstep(vols, lengths, dt, vols[s + 1], s, state["t"], 1e9)
            bc.applyBoundaryConditions(vols[s + 1])
        vols[0], vols[substeps] = vols[substeps], vols[0]
        state["t"] += dt

    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        flush.fill_(1.0)
        step()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    for k in range(args.steps):
        flush.fill_(float(k))
        starts[k].record()
        step()
        ends[k].record()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    cells = N * N
    result = {
        "metric": "cell-updates/s (KH 1024^2 FP64 through the plug-in classes)",
        "value": world * cells * args.steps / (total_ms * 1e-3), "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Kelvin-Helmholtz initial data, sample index = rank)",
        "config": dict(WORKLOAD, parallelism="independent replicas",
                       path="NumericalFlux.computeFlux + Integrator.performSubstep + "
                            "Boundary.applyBoundaryConditions per stage"),
        "gpu_launches": args.steps * substeps * 3,
        "clocks": clock_info,
    }
    if rank == 0:
        print(json.dumps(result))
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernels-only", action="store_true",
                    help="only run warmup+steps time steps (for profiler captures)")
    ap.add_argument("--workload", default="kh1024",
                    choices=sorted(["kh1024", "plugin", "uq", "surrogate"] + list(BATCHES)),
                    help="kh1024 (default, the plain FP64 drop-in through the fused solver), "
                         "plugin (the same through the plug-in classes), an ensemble workload, "
                         "or uq (time-to-error of the surrogate control variate)")
    ap.add_argument("--samples", type=int, default=1024, help="plain MC samples of --workload uq")
    ap.add_argument("--n", type=int, default=0,
                    help="grid size of a one-level batch workload (profiler captures)")
    ap.add_argument("--members", type=int, default=0,
                    help="members of a one-level batch workload (profiler captures)")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="member precision of the ensemble workloads")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload == "uq":
        run_uq(args, rank, world, local)
        return
    if args.workload == "surrogate":
        run_surrogate(args, rank, world, local)
        return
    if args.workload == "plugin":
        run_plugin(args, rank, world, local)
        return
    if args.workload != "kh1024":
        run_batch(args, rank, world, local)
        return

    import torch
    import torch.distributed as dist
    import alsvinn_b200 as als

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    state = kh_state(rank)
    sim = als.Simulator(DIM, (N, N), (0, 0), (1, 1), flux=FLUX, reconstruction=RECON,
                        integrator=INTEG, boundary=BC, cfl=CFL, end_time=1e9, device=local)
    sim.set_state(state)
    if args.kernels_only:
        for _ in range(args.warmup + args.steps):
            sim.advance(1)
        sim.synchronize()
        if sim.info()["status"] != 0:
            raise RuntimeError("constraint violation")
        sim.close()
        return
    # the schedule autotuner (state and clocks are restored afterwards)
    schedule = sim.tune(steps=3)
    stream = torch.cuda.ExternalStream(sim.stream(), device=local)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1.0)
            sim.advance(1)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        for k in range(args.steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            sim.advance(1)
            ends[k].record(stream)
        torch.cuda.synchronize()
        clock_info = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    merge_ms = None
    if world > 1:
        # the ensemble's end: FP64 Welford statistics of the members, merged
        # across the ranks in rank order (NCCL all_gather + Chan merge)
        from alsvinn_b200 import distributed
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        m0.record()
        mv = als.MeanVariance(NVAR * sim.plane, device=local)
        mv.add_solver(sim, 0)
        merged = distributed.merge_statistics(mv)
        merged.close()
        mv.close()
        m1.record()
        torch.cuda.synchronize()
        merge_ms = m0.elapsed_time(m1)
        total_ms += merge_ms
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    total_ms = float(t.item())
    info = sim.info()
    if info["status"] != 0:
        raise RuntimeError("constraint violation during the bench: %r" % info)

    # per-kernel durations for the roofline (events around each kernel)
    kms = np.array([sim.profile_step() for _ in range(5)])
    avg_k = kms.mean(axis=0)
    hbm_peak, peak_kind = peaks()
    cells = N * N
    roof = []
    for name, ms in zip(KERNEL_NAMES, avg_k):
        achieved = ALG_BYTES_PER_CELL[name] * cells / (ms * 1e-3) / 1e9
        roof.append({"kernel": name, "ms": float(ms), "achieved_gbs": achieved})
    dom = max(range(len(roof)), key=lambda i: roof[i]["ms"])
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_kh1024.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic = json.load(f).get(KERNEL_NAMES[dom])

    # end to end through the public API with host buffers: upload the state
    # from pinned memory, advance the same number of steps, download it
    pinned_in = torch.from_numpy(state).pin_memory()
    pinned_out = torch.empty_like(pinned_in).pin_memory()
    # the warm-up runs the same three calls once (first calls set up staging,
    # and an advance of 8 or more steps captures the solver's CUDA graph)
    out = pinned_out.numpy()
    sim.set_state(pinned_in.numpy())
    sim.advance(max(args.warmup, GRAPH_STEPS))
    sim._lib.als_solver_get_state(sim._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, 1)
    sim.synchronize()
    e2e_steps = args.steps
    t0 = time.perf_counter()
    sim.set_state(pinned_in.numpy())
    sim.advance(e2e_steps)
    sim._lib.als_solver_get_state(sim._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, 1)
    e2e_secs = time.perf_counter() - t0
    tt = torch.tensor([e2e_secs], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_secs = float(tt.item())
    state_bytes = state.nbytes

    value = world * cells * args.steps / (total_ms * 1e-3)
    result = {
        "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (Kelvin-Helmholtz initial data, sample index = rank)",
        "config": WORKLOAD,
        "sharding": "one ensemble member per GPU (sample index = rank); with N > 1 the "
                    "timed region ends with the FP64 statistics merge across ranks",
        "roofline": fp64_roofline(roof[dom], cells, hbm_peak, peak_kind, traffic, roof),
        "e2e": {"value": world * cells * e2e_steps / e2e_secs, "unit": "cell-updates/s",
                "h2d_bytes_per_step": state_bytes / e2e_steps,
                "d2h_bytes_per_step": state_bytes / e2e_steps,
                "definition": "als_solver_set_state(pinned host) + %d steps + als_solver_get_state"
                              "(pinned host), wall clock" % e2e_steps},
        "gpu_launches": args.steps * sim.launches_per_step(),
        "schedule": schedule,
        "clocks": clock_info,
    }
    if merge_ms is not None:
        result["statistics_merge_ms"] = merge_ms
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU baseline is timed at N = 1 only
        result["cpu_baseline"] = cpu_baseline(state)
    if rank == 0:
        print(json.dumps(result))
    sim.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

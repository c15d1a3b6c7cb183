"""Generates tests/golden/uq_kh256_fp64_4096.npz: the FP64 oracle ensemble of
the UQ benchmark (needs a GPU, about ten minutes on one B200).

    python tests/golden/make_uq_oracle.py

4096 Kelvin-Helmholtz samples (alsuq's STLMersenne draws 0..4095, 40
parameters each) at 256 x 256, WENO2 + HLL3, RK3, CFL 0.4, periodic, run to
T = 2 with the plain FP64 method (bit-identical per member to the
reference's CPU path on the same inputs).  Stored per sample: the
observable y = mean density over [0.25, 0.75]^2 at T, the step count and
the final time; the parameters are not stored (they are re-drawn from the
sample indices).  Also stored: the FP64 Welford mean and variance of the
density field over the ensemble.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import alsvinn_b200 as als  # noqa: E402

N = 256
SAMPLES = 4096
END_TIME = 2.0


def main(out=os.path.join(HERE, "uq_kh256_fp64_4096.npz")):
    t0 = time.perf_counter()
    params, y, info = als.uq.kh_observable_ensemble(N, 0, SAMPLES, precision="fp64",
                                                    end_time=END_TIME, field_statistics=True)
    np.savez_compressed(out, y=y, steps=info["steps"], n=N, samples=SAMPLES, end_time=END_TIME,
                        first_sample=0, solve_seconds=info["solve_seconds"],
                        rho_mean=info["field_mean"][0], rho_var=info["field_var"][0])
    print("wrote %s: %d samples, steps %d..%d, solve %.1f s, total %.1f s, y mean %.8f std %.8f"
          % (out, SAMPLES, info["steps"].min(), info["steps"].max(), info["solve_seconds"],
             time.perf_counter() - t0, y.mean(), y.std()))


if __name__ == "__main__":
    main(*sys.argv[1:])

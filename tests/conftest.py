import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

from oracle_lib import COracle, RefOracle, ref_library_path  # noqa: E402

SIMULATION_FIXTURES = sorted(f[:-4] for f in os.listdir(GOLDEN)
                             if f.endswith(".npz") and (f.startswith("sod") or f.startswith("kh")
                                                        or f.startswith("rand")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


@pytest.fixture(scope="session")
def c_oracle():
    return COracle()


@pytest.fixture(scope="session")
def ref_oracle():
    if not os.path.exists(ref_library_path()):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    return RefOracle()


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {k: z[k] for k in z.files}
    # scalars stored as 0-d arrays become Python values
    for k in ("flux", "recon", "integrator", "bc"):
        if k in out and np.ndim(out[k]) == 0:
            out[k] = str(out[k])
    for k in ("cfl", "end_time", "gamma", "t"):
        if k in out and np.ndim(out[k]) == 0:
            out[k] = float(out[k])
    for k in ("dim", "steps", "n", "samples", "first_sample"):
        if k in out and np.ndim(out[k]) == 0:
            out[k] = int(out[k])
    return out


def flux_cases():
    rows = []
    for name in ("compute_flux_cases.txt", "compute_flux_cases_limiters.txt"):
        with open(os.path.join(GOLDEN, name)) as f:
            for line in f:
                if line.startswith("#"):
                    continue
                p = line.split()
                rows.append({"dim": int(p[0]), "n": tuple(int(v) for v in p[1].split(",")),
                             "recon": p[2], "flux": p[3], "bc": p[4], "seed": int(p[5]),
                             "filled": p[6], "net": p[7], "ws": p[8], "ws_max": float(p[9])})
    return rows

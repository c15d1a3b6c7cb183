"""Builds the B200 shared library in-tree (``alsvinn_b200/_lib/libals_b200.so``).

Every CUDA translation unit is compiled for sm_100a only, in parallel, with
nvcc.  FP64 units use ``-fmad=false`` and IEEE division/square root so the
plain FP64 method reproduces the reference CPU path bit for bit; FP32
ensemble units may contract multiply-adds.

Usage: ``python -m alsvinn_b200.build`` (or ``build()`` from Python).
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(ROOT, "_build", "obj")
LIB_NAME = "libals_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
EXACT = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
FAST32 = ["-fmad=true"]
# FP32 ensemble members: contracted multiply-adds and the hardware-approximate
# divide and square root (at most a few ulp; the FP64 path stays IEEE), and
# in 2-D three resident blocks per SM (the FP32 tile needs half the shared
# memory and registers of the FP64 one).  Measured on 512 x 256^2 KH members
# (member cell-updates/s): IEEE, 2 blocks 4.2e9; approximate, 2 blocks 5.1e9;
# approximate, 3 blocks 5.9e9 (6.3e9 with the reciprocal forms that
# euler_math.cuh uses for FP32); 16x16 tiles / 288 threads / 4 blocks 5.3e9;
# 32x8 / 320 / 4 3.9e9.
STAGE32 = ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-DALS_STAGE2_BLOCKS=3", "-DALS_STAGE2S_BLOCKS=4"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    """(source, extra flags) of every translation unit."""
    units = []
    for name in sorted(os.listdir(CSRC)):
        if not name.endswith(".cu"):
            continue
        flags = STAGE32 if "_f32_" in name else (FAST32 if name.startswith("mlp") else EXACT)
        units.append((os.path.join(CSRC, name), flags))
    return units


def _headers_mtime():
    latest = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for name in os.listdir(d):
            if name.endswith((".cuh", ".h", ".hpp")):
                latest = max(latest, os.path.getmtime(os.path.join(d, name)))
    return latest


def _compile(nvcc, src, flags, force, obj_dir=OBJ_DIR):
    obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
    cmd = [nvcc] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    # the command an object was built with sits beside it: a change of flags
    # rebuilds it like a change of its sources
    stamp = obj + ".cmd"
    same_cmd = os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
    if (not force and same_cmd and os.path.exists(obj) and
            os.path.getmtime(obj) > os.path.getmtime(src) and
            os.path.getmtime(obj) > _headers_mtime()):
        return obj
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (src, res.stdout))
    with open(stamp, "w") as f:
        f.write(" ".join(cmd))
    return obj


def library_path():
    return os.path.join(OUT_DIR, LIB_NAME)


def build(force=False, jobs=None, verbose=False, extra_flags=(), out=None, obj_dir=None):
    """Compiles every unit (only what changed unless ``force``) and links the library.

    ``extra_flags`` (e.g. tuning defines), ``out`` and ``obj_dir`` build a
    variant elsewhere; the default is the in-tree library."""
    nvcc = nvcc_path()
    obj_dir = obj_dir or OBJ_DIR
    lib = out or library_path()
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    units = sources()
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    extra = list(extra_flags)
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda u: _compile(nvcc, u[0], u[1] + extra, force, obj_dir), units))
    if force or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if res.returncode != 0:
            raise RuntimeError("link failed:\n%s" % res.stdout)
    if verbose:
        print("built", lib)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

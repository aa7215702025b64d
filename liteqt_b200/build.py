"""Build the sm_100a CUDA library liteqt_b200/librgf_b200.so in-tree with nvcc.

    python -m liteqt_b200.build [--force] [--ptxas]

Every .cu file is compiled separately (in parallel) as relocatable device
code: each kernel variant's task function lives in its own translation unit
(rgf_task_*.cu) and the persistent kernel (rgf_fp64.cu) calls them across
units, resolved by the device link of the final shared library.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librgf_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-rdc=true",
    # the persistent kernel runs 2 CTAs of 256 threads per SM: every task
    # function it calls must fit the same 128-register budget
    "-maxrregcount=128",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


# Units whose kernels run one CTA per SM (their __launch_bounds__ give them up
# to 255 registers a thread): the mixed-precision form holds a 128 x 128 FP32
# matrix in registers during its inverse.
ONE_CTA_PER_SM = {"rgf_mixed.cu"}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    jobs = []
    hdrs = headers()
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            flags = list(NVCC_FLAGS)
            if os.path.basename(src) in ONE_CTA_PER_SM:
                flags.remove("-maxrregcount=128")
            cmd = [nvcc(), *flags, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    if jobs:
        workers = max(1, min(len(jobs), os.cpu_count() or 1))
        with concurrent.futures.ThreadPoolExecutor(workers) as pool:
            futs = []
            for cmd in jobs:
                if verbose:
                    print(" ".join(cmd), flush=True)
                futs.append(pool.submit(subprocess.run, cmd, capture_output=True, text=True))
            failed = None
            for cmd, f in zip(jobs, futs):
                r = f.result()
                if r.stdout or r.stderr:
                    sys.stdout.write(r.stdout + r.stderr)
                if r.returncode != 0 and failed is None:
                    failed = subprocess.CalledProcessError(r.returncode, cmd)
            if failed is not None:
                raise failed
    if force or _stale(LIB, objs):
        # device link of the relocatable objects + host link; exported symbols:
        # the extern "C" rgf_* entry points (visibility default via the map)
        # cuFFT (the GW convolutions' FFT form) from the CUDA toolkit, found at
        # run time through the toolkit's library directory
        cudalib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc()))), "lib64")
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-shared", "-o", LIB, *objs,
               "-Xlinker", "--version-script=" + os.path.join(CSRC, "exports.map"),
               "-L" + cudalib, "-lcufft", "-Xlinker", "-rpath=" + cudalib]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)

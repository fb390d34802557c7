"""Build the engine shared library ``marqov_b200/libmarqov_b200.so`` for sm_100a.

nvcc compiles every ``csrc/*.cu`` for ``-gencode arch=compute_100a,code=sm_100a``
and links them with the static CUDA runtime into one C-ABI library (no torch
types cross it).  Host code is built with ``-ffp-contract=off`` so the FP64
acceptance-rule thresholds computed on the host round like the device code.
"""
from __future__ import annotations

import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmarqov_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden"]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                  + [os.path.join(HERE, "..", "include", "marqov_b200.h")])


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(f) <= t for f in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []
    objs = [os.path.join(objdir, os.path.basename(src)[:-3] + ".o") for src in sources()]
    cmds = [[NVCC, *ARCH, *FLAGS, *extra, "-c", "-o", obj, src] for src, obj in zip(sources(), objs)]
    # one nvcc per translation unit, side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    tmp = OUT + ".tmp"
    subprocess.check_call([NVCC, *ARCH, "-shared", "-o", tmp, *objs])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
